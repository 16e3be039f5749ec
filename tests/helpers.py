"""Shared test helpers: drive a model (native GPU or CPU oracle) through update!-style steps and
compare states exactly."""
import numpy as np

from PlanktonIndividuals import _abi
from PlanktonIndividuals.stepping import VelCache, drive, forcing_indices  # noqa: F401


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
