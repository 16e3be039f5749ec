"""Batched FP32 form: many independent models advanced together (pi_batch_* of include/pib200.h).

The reference runs an ensemble as separate PlanktonModels, one `update!` after another. Here every
member keeps its own grid, parameters, capacity, individuals, tracers, forcing and seed, and each
phase of TimeStep! is one launch over all members, replayed from a CUDA graph. A member computes
the same bits it would compute alone as a PlanktonModel(FT=Float32).

    members = [Member(grid, bgc_params, phyt_params, capacity, seed), ...]
    batch = PlanktonBatch(members, nspecies=1)
    batch.set_state(m, individuals, tracers)
    batch.set_series(m, vels=dict(u=..., v=..., w=...), PARF=..., temp=..., ΔT_vel=..., ΔT_PAR=..., ΔT_temp=...)
    batch.autotune(ΔT)
    batch.step(ΔT, nsteps)
"""
import ctypes as ct
from dataclasses import dataclass

import numpy as np

from . import _abi, _lib
from ._abi import IND_DOUBLE, IND_INT, NTRACERS, PI_BOUNDED, PI_OK, pi_individuals
from ._native import CapacityError, PIError, _dptr, make_bgc_struct, make_grid_struct, make_species_structs


@dataclass
class Member:
    grid: object            # RectilinearGrid
    bgc_params: dict
    phyt_params: dict
    capacity: int
    seed: int = 0


def _f64(a, shape=None):
    a = np.asarray(a, dtype=np.float64)
    if shape is not None and a.shape != tuple(shape):
        raise ValueError(f"expected shape {tuple(shape)}, got {a.shape}")
    return np.asfortranarray(a)


class PlanktonBatch:
    def __init__(self, members, nspecies=1):
        self.lib = _lib.load()
        self.members = list(members)
        self.nsp = int(nspecies)
        self._keep = []
        arr = (_abi.pi_member * len(self.members))()
        for m, mb in enumerate(self.members):
            g, keep = make_grid_struct(mb.grid)
            b = make_bgc_struct(mb.bgc_params)
            sp = make_species_structs(mb.phyt_params, self.nsp)
            self._keep += [g, keep, b, sp]
            arr[m].grid = ct.pointer(g)
            arr[m].bgc = ct.pointer(b)
            arr[m].species = ct.cast(sp, ct.POINTER(_abi.pi_quota_params))
            arr[m].capacity = int(mb.capacity)
            arr[m].seed = int(mb.seed)
        h = ct.c_void_p()
        rc = self.lib.pi_batch_create(arr, len(self.members), self.nsp, ct.byref(h))
        if rc != PI_OK:
            raise PIError(rc, self._errmsg(None))
        self.h = h

    # ---- plumbing ------------------------------------------------------------------------------
    def _errmsg(self, h):
        buf = ct.create_string_buffer(1024)
        self.lib.pi_batch_last_error(h, buf, 1024)
        return buf.value.decode(errors="replace")

    def _check(self, rc, what):
        if rc != PI_OK:
            msg = self._errmsg(self.h)
            if rc == _abi.PI_ERR_CAPACITY:
                raise CapacityError(rc, msg)
            raise PIError(rc, f"{what}: status {rc}: {msg}")

    def close(self):
        if getattr(self, "h", None):
            self.lib.pi_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return len(self.members)

    def member(self, m):
        """A view of member m with the model-level calls (set/get individuals, tracers, ...)."""
        return BatchMember(self, m)

    # ---- state -------------------------------------------------------------------------------
    def set_individuals(self, m, sp, data):
        C = self.members[m].capacity
        keep = {}
        st = pi_individuals()
        for k in IND_DOUBLE:
            a = np.ascontiguousarray(data[k], dtype=np.float64)
            if a.shape != (C,):
                raise ValueError(f"individual attribute {k} must have length {C}")
            keep[k] = a
            setattr(st, k, _dptr(a))
        for k in IND_INT:
            a = np.ascontiguousarray(data[k], dtype=np.int64)
            keep[k] = a
            setattr(st, k, a.ctypes.data_as(ct.POINTER(ct.c_int64)))
        ac = np.ascontiguousarray(data["ac"], dtype=np.uint8)
        keep["ac"] = ac
        st.ac = ac.ctypes.data_as(ct.POINTER(ct.c_uint8))
        self._check(self.lib.pi_batch_set_individuals(self.h, m, sp, ct.byref(st)), "set_individuals")

    def get_individuals(self, m, sp):
        C = self.members[m].capacity
        out = {k: np.empty(C, dtype=np.float64) for k in IND_DOUBLE}
        out.update({k: np.empty(C, dtype=np.int64) for k in IND_INT})
        out["ac"] = np.empty(C, dtype=np.uint8)
        st = pi_individuals()
        for k in IND_DOUBLE:
            setattr(st, k, _dptr(out[k]))
        for k in IND_INT:
            setattr(st, k, out[k].ctypes.data_as(ct.POINTER(ct.c_int64)))
        st.ac = out["ac"].ctypes.data_as(ct.POINTER(ct.c_uint8))
        self._check(self.lib.pi_batch_get_individuals(self.h, m, sp, ct.byref(st)), "get_individuals")
        out["ac"] = out["ac"].astype(bool)
        return out

    def set_tracer(self, m, n, data):
        a = _f64(data, self.members[m].grid.total_size)
        self._check(self.lib.pi_batch_set_tracer(self.h, m, n, _dptr(a.ravel(order="F"))), "set_tracer")

    def get_tracer(self, m, n):
        g = self.members[m].grid
        out = np.empty(int(np.prod(g.total_size)), dtype=np.float64)
        self._check(self.lib.pi_batch_get_tracer(self.h, m, n, _dptr(out)), "get_tracer")
        return out.reshape(g.total_size, order="F")

    def set_state(self, m, individuals, tracers):
        for s, d in enumerate(individuals):
            self.set_individuals(m, s, d)
        for n in range(NTRACERS):
            self.set_tracer(m, n, tracers[n])

    # ---- forcing ------------------------------------------------------------------------------
    def _vel_shapes(self, m):
        g = self.members[m].grid
        b = [int(t == PI_BOUNDED) for t in g.topo]
        return (g.Nx + b[0], g.Ny, g.Nz), (g.Nx, g.Ny + b[1], g.Nz), (g.Nx, g.Ny, g.Nz + b[2])

    def set_velocity(self, m, u, v, w):
        su, sv, sw = self._vel_shapes(m)
        u, v, w = _f64(u, su), _f64(v, sv), _f64(w, sw)
        self._check(self.lib.pi_batch_set_velocity(self.h, m, _dptr(u.ravel(order="F")), _dptr(v.ravel(order="F")),
                                                   _dptr(w.ravel(order="F"))), "set_velocity")

    def set_velocity0(self, m, u, v, w):
        su, sv, sw = self._vel_shapes(m)
        u, v, w = _f64(u, su), _f64(v, sv), _f64(w, sw)
        self._check(self.lib.pi_batch_set_velocity0(self.h, m, _dptr(u.ravel(order="F")), _dptr(v.ravel(order="F")),
                                                    _dptr(w.ravel(order="F"))), "set_velocity0")

    def set_PARF(self, m, parf):
        g = self.members[m].grid
        a = _f64(parf, (g.Nx, g.Ny))
        self._check(self.lib.pi_batch_set_PARF(self.h, m, _dptr(a.ravel(order="F"))), "set_PARF")

    def set_temp(self, m, temp):
        g = self.members[m].grid
        a = _f64(temp, g.size)
        self._check(self.lib.pi_batch_set_temp(self.h, m, _dptr(a.ravel(order="F"))), "set_temp")

    def set_flux_bc(self, m, tracer, face, kind, values=None, nt=0):
        if values is None:
            p = ct.POINTER(ct.c_double)()
        else:
            values = np.asfortranarray(np.atleast_1d(np.asarray(values, dtype=np.float64)))
            self._keep.append(values)
            p = _dptr(values.ravel(order="F"))
        self._check(self.lib.pi_batch_set_flux_bc(self.h, m, int(tracer), int(face), int(kind), p, int(nt)),
                    "set_flux_bc")

    def set_series(self, m, *, PARF, temp, ΔT_PAR=3600.0, ΔT_temp=3600.0, vels=None, ΔT_vel=None,
                   time_offset=0):
        """Device-resident forcing series of member m (PlanktonSimulation's arrays): vels u, v, w of
        shape (Nx[+1], Ny[+1], Nz[+1], n), PARF (Nx, Ny, n), temp (Nx, Ny, Nz, n)."""
        g = self.members[m].grid
        PARF = np.asfortranarray(np.asarray(PARF, dtype=np.float64).reshape(g.Nx, g.Ny, -1, order="F"))
        temp = np.asfortranarray(np.asarray(temp, dtype=np.float64).reshape(g.Nx, g.Ny, g.Nz, -1, order="F"))
        null = ct.POINTER(ct.c_double)()
        if vels:
            su, sv, sw = self._vel_shapes(m)
            u = np.asfortranarray(np.asarray(vels["u"], dtype=np.float64).reshape(su + (-1,), order="F"))
            v = np.asfortranarray(np.asarray(vels["v"], dtype=np.float64).reshape(sv + (-1,), order="F"))
            w = np.asfortranarray(np.asarray(vels["w"], dtype=np.float64).reshape(sw + (-1,), order="F"))
            pu, pv, pw, nvel = _dptr(u), _dptr(v), _dptr(w), u.shape[3]
        else:
            pu = pv = pw = null
            nvel, ΔT_vel = 0, 1.0
        self._check(self.lib.pi_batch_set_series(self.h, m, pu, pv, pw, int(nvel), float(ΔT_vel or 1.0),
                                                 _dptr(PARF), int(PARF.shape[2]), float(ΔT_PAR),
                                                 _dptr(temp), int(temp.shape[3]), float(ΔT_temp), int(time_offset)),
                    "set_series")

    def clear_series(self, m):
        self._check(self.lib.pi_batch_clear_series(self.h, m), "clear_series")

    # ---- stepping -----------------------------------------------------------------------------
    def step(self, ΔT, nsteps=1, sync=True):
        self._check(self.lib.pi_batch_step(self.h, float(ΔT), int(nsteps), 1 if sync else 0), "step")

    def set_tracer_kernel(self, fused, levels=32):
        """Tracer update kernels: fused (one kernel per column run of `levels` levels) or the x-y
        and z kernels with the halo fill (pi_batch_set_tracer_kernel); results are identical."""
        self._check(self.lib.pi_batch_set_tracer_kernel(self.h, 1 if fused else 0, int(levels)), "set_tracer_kernel")

    def set_option(self, name, value):
        """One launch-shape option by name (pi_batch_set_option); results are identical for every
        choice."""
        self._check(self.lib.pi_batch_set_option(self.h, name.encode(), int(value)), "set_option")

    def synchronize(self):
        self._check(self.lib.pi_batch_synchronize(self.h), "synchronize")

    def set_diags(self, tracer_mask=0, proc_mask=0):
        """Optional diagnostics of every member (bits as pi_batch_set_diags)."""
        self._check(self.lib.pi_batch_set_diags(self.h, ct.c_uint32(tracer_mask), ct.c_uint32(proc_mask)), "set_diags")

    def check_finite(self, m):
        """Raises PIError (PI_ERR_NAN) naming the first tracer cell or active individual of member
        m holding a NaN or Inf."""
        self._check(self.lib.pi_batch_check_finite(self.h, int(m)), "check_finite")

    def guard_stats(self):
        """(decisions recomputed in Float64 near their threshold, decisions that changed)."""
        r, c = ct.c_int64(), ct.c_int64()
        self._check(self.lib.pi_batch_guard_stats(self.h, ct.byref(r), ct.byref(c)), "guard_stats")
        return r.value, c.value

    def set_sort_interval(self, steps):
        """Steps between the counting sorts that keep the stored individuals grouped by cell
        (0: never); changes speed only, no result."""
        self._check(self.lib.pi_batch_set_sort_interval(self.h, int(steps)), "set_sort_interval")

    def autotune(self, ΔT, steps_per_candidate=2):
        buf = ct.create_string_buffer(4096)
        self._check(self.lib.pi_batch_autotune(self.h, float(ΔT), int(steps_per_candidate), buf, 4096), "autotune")
        return buf.value.decode()

    def get_time(self):
        it = ct.c_int64()
        t = ct.c_double()
        self._check(self.lib.pi_batch_get_time(self.h, ct.byref(it), ct.byref(t)), "get_time")
        return it.value, t.value

    def set_time(self, iteration, t):
        self._check(self.lib.pi_batch_set_time(self.h, int(iteration), float(t)), "set_time")

    # ---- outputs ------------------------------------------------------------------------------
    def count_active(self, m=-1, sp=-1):
        n = ct.c_int64()
        self._check(self.lib.pi_batch_count_active(self.h, int(m), int(sp), ct.byref(n)), "count_active")
        return n.value

    def get_diag(self, m, kind, sp=0):
        g = self.members[m].grid
        out = np.empty(int(np.prod(g.total_size)), dtype=np.float64)
        self._check(self.lib.pi_batch_get_diag(self.h, m, int(kind), int(sp), _dptr(out)), "get_diag")
        return out.reshape(g.total_size, order="F")

    def reset_diags(self):
        self._check(self.lib.pi_batch_reset_diags(self.h), "reset_diags")

    def budget(self, m):
        """FP64 mass budgets (mmol): dict with tracer and individual C, N, P."""
        out = (ct.c_double * 6)()
        self._check(self.lib.pi_batch_budget(self.h, m, out), "budget")
        v = list(out)
        return dict(tracer_C=v[0], tracer_N=v[1], tracer_P=v[2], ind_C=v[3], ind_N=v[4], ind_P=v[5])

    def stream(self):
        s = ct.c_void_p()
        self._check(self.lib.pi_batch_get_stream(self.h, ct.byref(s)), "get_stream")
        return s.value

    def profile_enable(self, on=True):
        self._check(self.lib.pi_batch_profile_enable(self.h, 1 if on else 0), "profile_enable")

    def profile_read(self):
        n = ct.c_int32()
        names = ct.create_string_buffer(8192)
        launches = (ct.c_int64 * 64)()
        ms = (ct.c_double * 64)()
        self._check(self.lib.pi_batch_profile_read(self.h, 64, names, 8192, launches, ms, ct.byref(n)), "profile_read")
        raw = names.raw.split(b"\0")
        return {raw[q].decode(): (launches[q], ms[q]) for q in range(min(n.value, 64))}


class BatchMember:
    """Member m of a batch with the per-model calls of CModel (stepping stays batch-wide)."""

    def __init__(self, batch, m):
        self.batch, self.m = batch, m
        self.grid = batch.members[m].grid

    def get_individuals(self, sp):
        return self.batch.get_individuals(self.m, sp)

    def set_individuals(self, sp, data):
        self.batch.set_individuals(self.m, sp, data)

    def get_tracer(self, n):
        return self.batch.get_tracer(self.m, n)

    def set_tracer(self, n, data):
        self.batch.set_tracer(self.m, n, data)

    def set_velocity(self, u, v, w):
        self.batch.set_velocity(self.m, u, v, w)

    def set_PARF(self, parf):
        self.batch.set_PARF(self.m, parf)

    def set_temp(self, temp):
        self.batch.set_temp(self.m, temp)

    def get_diag(self, kind, sp=0):
        return self.batch.get_diag(self.m, kind, sp)

    def get_time(self):
        return self.batch.get_time()

    def count_active(self, sp):
        return self.batch.count_active(self.m, sp)

    def set_state(self, individuals, tracers):
        self.batch.set_state(self.m, individuals, tracers)


def shard_members(costs, world_size):
    """Split ensemble members over `world_size` ranks with balanced work: members sorted by cost
    (largest first) go, one by one, to the rank with the least total so far (ties: lowest rank).
    `costs` are per-member work estimates (individuals + interior cells). Returns, per rank, the
    sorted list of member indices. Deterministic, so every rank computes the same partition
    without communicating."""
    order = sorted(range(len(costs)), key=lambda m: (-costs[m], m))
    load = [0.0] * world_size
    parts = [[] for _ in range(world_size)]
    for m in order:
        r = min(range(world_size), key=lambda q: (load[q], q))
        parts[r].append(m)
        load[r] += costs[m]
    return [sorted(p) for p in parts]


def member_cost(wl):
    """Work estimate of a member: active individuals plus interior cells."""
    return float(sum(wl.N)) + float(wl.grid.Nx * wl.grid.Ny * wl.grid.Nz)
