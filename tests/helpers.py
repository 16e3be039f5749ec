"""Shared test helpers: drive a model (native GPU or CPU oracle) through update!-style steps and
compare states exactly."""
import math

import numpy as np

from PlanktonIndividuals import _abi


def forcing_indices(t, wl, time_offset_i=None):
    """Snapshot indices (0-based) that update! selects at model time t (update.jl:14-26)."""
    tv = int(math.floor(t / wl.dT_vel))
    tp = int(math.floor(t / wl.dT_PAR))
    tt = int(math.floor(t / wl.dT_temp))
    return tv, tp, tt


class VelCache:
    def __init__(self, wl):
        self.wl, self.cache = wl, {}

    def __call__(self, i):
        if i not in self.cache:
            self.cache[i] = self.wl.velocity(i)
        return self.cache[i]


def drive(model, wl, steps, vel=None):
    """update!(sim) with vels, one step at a time through the set_* entry points."""
    vel = vel or VelCache(wl)
    for _ in range(steps):
        _, t = model.get_time()
        tv, tp, tt = forcing_indices(t, wl)
        model.set_velocity(*vel(tv))
        model.set_PARF(wl.parf[:, :, tp])
        model.set_temp(wl.temp[:, :, :, tt])
        model.time_step(wl.dT)


def same(a, b):
    a = np.asarray(a); b = np.asarray(b)
    if a.dtype.kind == "f":
        return a.shape == b.shape and np.array_equal(a, b, equal_nan=True)
    return np.array_equal(a, b)


def compare_states(ref, gpu, nsp, fields_only_active=False):
    """Returns a list of mismatch descriptions (empty when everything is identical)."""
    bad = []
    for s in range(nsp):
        A, B = ref.get_individuals(s), gpu.get_individuals(s)
        for k in A:
            a, b = np.asarray(A[k]), np.asarray(B[k])
            if not same(a, b):
                if a.dtype.kind == "f":
                    neq = ~((a == b) | (np.isnan(a) & np.isnan(b)))
                else:
                    neq = a != b
                diff = np.nonzero(neq)[0]
                i = int(diff[0])
                bad.append(f"sp{s} {k}: {len(diff)} slots differ, first {i}: {a[i]!r} vs {b[i]!r}")
    for n in range(_abi.NTRACERS):
        a, b = ref.get_tracer(n), gpu.get_tracer(n)
        if not same(a, b):
            d = np.argwhere(a != b)
            bad.append(f"tracer {_abi.tracer_names[n]}: {len(d)} cells differ, first {tuple(d[0])}: "
                       f"{a[tuple(d[0])]!r} vs {b[tuple(d[0])]!r}")
    kinds = [(_abi.PI_DIAG_PAR, 0)] + [(k, s) for s in range(nsp) for k in
                                         (_abi.PI_DIAG_NUM, _abi.PI_DIAG_GRAZ, _abi.PI_DIAG_MORT, _abi.PI_DIAG_DVID)]
    for k, s in kinds:
        a, b = ref.get_diag(k, s), gpu.get_diag(k, s)
        if not same(a, b):
            bad.append(f"diag {k} sp{s}: {int(np.sum(a != b))} cells differ")
    return bad
