"""Thin object wrapper over a C library that exports the pib200.h entry points.

`CModel` owns one model handle and converts numpy arrays (Julia column-major layout) to the
pointer arguments of the C ABI. The product package instantiates it over libpib200 only.
"""
import ctypes as ct

import numpy as np

from . import _abi
from ._abi import (IND_DOUBLE, IND_INT, NTRACERS, PI_OK, pi_bgc_params, pi_grid, pi_grid_metrics, pi_individuals,
                   pi_quota_params, BGC_FIELDS, QUOTA_FIELDS)


class PIError(RuntimeError):
    """Error returned by the C ABI; `.code` is the pi_status value."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class CapacityError(PIError, ValueError):
    """Division overflow, the reference's ArgumentError at QuotaMode/plankton_update.jl:20-22."""


def _dptr(a):
    return a.ctypes.data_as(ct.POINTER(ct.c_double))


def _f64(a, shape=None):
    a = np.asarray(a, dtype=np.float64)
    if shape is not None and a.shape != tuple(shape):
        raise ValueError(f"expected shape {tuple(shape)}, got {a.shape}")
    return np.asfortranarray(a)


def make_grid_struct(grid):
    g = pi_grid()
    g.Nx, g.Ny, g.Nz = grid.Nx, grid.Ny, grid.Nz
    g.Hx, g.Hy, g.Hz = grid.Hx, grid.Hy, grid.Hz
    for a in range(3):
        g.topo[a] = grid.topo[a]
    g.dx, g.dy = float(grid.Δx), float(grid.Δy)
    keep = [np.ascontiguousarray(grid.dzF, dtype=np.float64),
            np.ascontiguousarray(grid.dzC, dtype=np.float64),
            np.asfortranarray(grid.landmask, dtype=np.uint8)]
    g.dzF = _dptr(keep[0])
    g.dzC = _dptr(keep[1])
    g.landmask = keep[2].ctypes.data_as(ct.POINTER(ct.c_uint8))
    if getattr(grid, "is_latlon", False):
        # LatLonGrid: the metric arrays as the reference stores them (halos included)
        mt = pi_grid_metrics()
        for name in ("dxC", "dyC", "dxF", "dyF", "Az", "Ax", "Ay", "Vol"):
            arr = np.asfortranarray(getattr(grid, name), dtype=np.float64)
            keep.append(arr)
            setattr(mt, name, _dptr(arr))
        keep.append(mt)
        g.metrics = ct.pointer(mt)
    return g, keep


def make_bgc_struct(params):
    b = pi_bgc_params()
    for cname, key in BGC_FIELDS:
        setattr(b, cname, float(params[key]))
    return b


def make_species_structs(phyt_params, nsp, mode="quota"):
    struct, fields = {"carbon": (_abi.pi_carbon_params, _abi.CARBON_FIELDS),
                      "macro": (_abi.pi_macro_params, _abi.MACRO_FIELDS),
                      "iron": (_abi.pi_iron_params, _abi.IRON_FIELDS)}.get(mode, (pi_quota_params, QUOTA_FIELDS))
    arr = (struct * nsp)()
    for s in range(nsp):
        for cname, key in fields:
            v = phyt_params[key]
            v = v[s] if hasattr(v, "__len__") else v
            setattr(arr[s], cname, float(v))
    return arr


class CModel:
    """One model handle of a library exporting `<prefix>create` ... `<prefix>last_error`."""

    def __init__(self, lib, prefix, grid, bgc_params, phyt_params, nsp, capacity, seed,
                 precision=None, mode="quota"):
        """mode: "quota" (QuotaMode), "carbon" (CarbonMode, `<prefix>create_carbon`), "macro"
        (MacroMolecularMode, `<prefix>create_macro`) or "iron" (IronEnergyMode, `<prefix>create_iron`)."""
        if mode not in ("quota", "carbon", "macro", "iron"):
            raise ValueError(f"mode must be 'quota', 'carbon', 'macro' or 'iron', not {mode!r}")
        self.lib = _abi.declare(lib, prefix)
        self.prefix = prefix
        self.mode = mode
        self.precision = _abi.PI_FP64 if precision is None else int(precision)
        self.nsa = 0
        self.grid = grid
        self.nsp = int(nsp)
        self.capacity = int(capacity)
        g, self._keep = make_grid_struct(grid)
        b = make_bgc_struct(bgc_params)
        sp = make_species_structs(phyt_params, self.nsp, mode)
        h = ct.c_void_p()
        fn = self._fn({"carbon": "create_carbon", "macro": "create_macro", "iron": "create_iron"}.get(mode, "create"))
        if precision is None:
            rc = fn(ct.byref(g), ct.byref(b), sp, self.nsp, self.capacity, ct.c_uint64(seed), ct.byref(h))
        else:
            rc = fn(ct.byref(g), ct.byref(b), sp, self.nsp, self.capacity, int(precision),
                    ct.c_uint64(seed), ct.byref(h))
        if rc != PI_OK:
            raise PIError(rc, f"{prefix}create failed ({rc}): {self._errmsg(None)}")
        self.h = h

    def _fn(self, name):
        return getattr(self.lib, self.prefix + name)

    def _errmsg(self, h):
        buf = ct.create_string_buffer(512)
        self._fn("last_error")(h, buf, 512)
        return buf.value.decode(errors="replace")

    def _check(self, rc, what):
        if rc != PI_OK:
            msg = self._errmsg(self.h)
            if rc == _abi.PI_ERR_CAPACITY:
                raise CapacityError(rc, msg)
            raise PIError(rc, f"{what}: status {rc}: {msg}")

    def close(self):
        if getattr(self, "h", None):
            self._fn("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def G(self):
        g = self.grid
        return (g.Nx + 2 * g.Hx) * (g.Ny + 2 * g.Hy) * (g.Nz + 2 * g.Hz)

    @property
    def gshape(self):
        return self.grid.total_size

    # ---- individuals ---------------------------------------------------------------------
    def set_individuals(self, sp, data):
        C = self.capacity
        keep = {}
        st = pi_individuals()
        carbon, macro, iron = self.mode == "carbon", self.mode == "macro", self.mode == "iron"
        for k in IND_DOUBLE + (("Bd",) if carbon else ()) + (_abi.MACRO_POOLS if macro else ()) + \
                (_abi.IRON_POOLS if iron else ()):
            if carbon and k in ("Cq", "Nq", "Pq", "Bd") and k not in data:
                continue                      # CarbonMode keeps no quotas; Bd defaults to zero
            if iron and (k in ("Cq", "Nq", "Pq") or (k in ("exEn", "tdark") and k not in data)):
                continue                      # IronEnergyMode keeps its own quotas instead
            if macro and k in ("Sz", "Bm", "Cq", "Nq", "Pq"):
                continue                      # MacroMolecularMode keeps its six pools instead
            a = np.ascontiguousarray(data[k], dtype=np.float64)
            if a.shape != (C,):
                raise ValueError(f"individual attribute {k} must have length {C}")
            keep[k] = a
            setattr(st, k, _dptr(a))
        for k in IND_INT:
            a = np.ascontiguousarray(data[k], dtype=np.int64)
            if a.shape != (C,):
                raise ValueError(f"individual attribute {k} must have length {C}")
            keep[k] = a
            setattr(st, k, a.ctypes.data_as(ct.POINTER(ct.c_int64)))
        ac = np.ascontiguousarray(data["ac"], dtype=np.uint8)
        keep["ac"] = ac
        st.ac = ac.ctypes.data_as(ct.POINTER(ct.c_uint8))
        if data.get("ptc") is not None:           # abiotic particles held; zeros when absent
            a = np.ascontiguousarray(data["ptc"], dtype=np.float64)
            if a.shape != (C,):
                raise ValueError(f"individual attribute ptc must have length {C}")
            keep["ptc"] = a
            st.ptc = _dptr(a)
        self._check(self._fn("set_individuals")(self.h, int(sp), ct.byref(st)), "set_individuals")

    def get_individuals(self, sp):
        C = self.capacity
        carbon, macro = self.mode == "carbon", self.mode == "macro"
        if macro:
            names = tuple(k for k in IND_DOUBLE if k not in ("Sz", "Bm", "Cq", "Nq", "Pq")) + _abi.MACRO_POOLS
        elif self.mode == "iron":
            names = tuple(k for k in IND_DOUBLE if k not in ("Cq", "Nq", "Pq")) + _abi.IRON_POOLS
        else:
            names = tuple(k for k in IND_DOUBLE if not (carbon and k in ("Cq", "Nq", "Pq"))) + (("Bd",) if carbon else ())
        if self.precision == _abi.PI_FP64:
            names = names + ("ptc",)
        out = {k: np.empty(C, dtype=np.float64) for k in names}
        out.update({k: np.empty(C, dtype=np.int64) for k in IND_INT})
        out["ac"] = np.empty(C, dtype=np.uint8)
        st = pi_individuals()
        for k in names:
            setattr(st, k, _dptr(out[k]))
        for k in IND_INT:
            setattr(st, k, out[k].ctypes.data_as(ct.POINTER(ct.c_int64)))
        st.ac = out["ac"].ctypes.data_as(ct.POINTER(ct.c_uint8))
        self._check(self._fn("get_individuals")(self.h, int(sp), ct.byref(st)), "get_individuals")
        out["ac"] = out["ac"].astype(bool)
        return out

    # ---- fields ----------------------------------------------------------------------------
    def set_tracer(self, idx, data):
        a = _f64(data, self.gshape)
        self._check(self._fn("set_tracer")(self.h, int(idx), _dptr(a.ravel(order="F"))), "set_tracer")

    def get_tracer(self, idx):
        out = np.empty(self.G, dtype=np.float64)
        self._check(self._fn("get_tracer")(self.h, int(idx), _dptr(out)), "get_tracer")
        return out.reshape(self.gshape, order="F")

    def set_velocity(self, u, v, w):
        g = self.grid
        b = [int(t == _abi.PI_BOUNDED) for t in g.topo]
        u = _f64(u, (g.Nx + b[0], g.Ny, g.Nz))
        v = _f64(v, (g.Nx, g.Ny + b[1], g.Nz))
        w = _f64(w, (g.Nx, g.Ny, g.Nz + b[2]))
        self._check(self._fn("set_velocity")(self.h, _dptr(u.ravel(order="F")), _dptr(v.ravel(order="F")),
                                             _dptr(w.ravel(order="F"))), "set_velocity")

    def set_velocity0(self, u, v, w):
        """vel₀ (previous step's velocity), for restarting from a checkpoint."""
        g = self.grid
        b = [int(t == _abi.PI_BOUNDED) for t in g.topo]
        u = _f64(u, (g.Nx + b[0], g.Ny, g.Nz))
        v = _f64(v, (g.Nx, g.Ny + b[1], g.Nz))
        w = _f64(w, (g.Nx, g.Ny, g.Nz + b[2]))
        self._check(self._fn("set_velocity0")(self.h, _dptr(u.ravel(order="F")), _dptr(v.ravel(order="F")),
                                              _dptr(w.ravel(order="F"))), "set_velocity0")

    def set_PARF(self, parf):
        a = _f64(parf, (self.grid.Nx, self.grid.Ny))
        self._check(self._fn("set_PARF")(self.h, _dptr(a.ravel(order="F"))), "set_PARF")

    def set_temp(self, temp):
        a = _f64(temp, self.grid.size)
        self._check(self._fn("set_temp")(self.h, _dptr(a.ravel(order="F"))), "set_temp")

    def set_flux_bc(self, tracer, face, kind, values=None, nt=0):
        if values is None:
            p = ct.POINTER(ct.c_double)()
        else:
            values = np.asfortranarray(np.atleast_1d(np.asarray(values, dtype=np.float64)))
            self._keep.append(values)
            p = _dptr(values.ravel(order="F"))
        self._check(self._fn("set_flux_bc")(self.h, int(tracer), int(face), int(kind), p, int(nt)),
                    "set_flux_bc")

    # ---- stepping ----------------------------------------------------------------------------
    def time_step(self, dT):
        self._check(self._fn("time_step")(self.h, float(dT)), "time_step")

    def get_time(self):
        it = ct.c_int64()
        t = ct.c_double()
        self._check(self._fn("get_time")(self.h, ct.byref(it), ct.byref(t)), "get_time")
        return it.value, t.value

    def set_time(self, iteration, t):
        self._check(self._fn("set_time")(self.h, int(iteration), float(t)), "set_time")

    def count_active(self, sp):
        n = ct.c_int64()
        self._check(self._fn("count_active")(self.h, int(sp), ct.byref(n)), "count_active")
        return n.value

    def set_diags(self, tracer_mask=0, proc_mask=0):
        """PlanktonDiagnostics(model; tracer, phytoplankton) beyond the defaults: bit n of
        tracer_mask adds tracer n, bit q of proc_mask the QuotaMode process q (PROC_NAMES)."""
        self._check(self._fn("set_diags")(self.h, ct.c_uint32(tracer_mask), ct.c_uint32(proc_mask)), "set_diags")

    def budget(self):
        """Mass budgets (mmol): interior tracer C, N, P and the active individuals' C, N, P
        (pi_get_budget)."""
        out = np.zeros(6, dtype=np.float64)
        self._check(self._fn("get_budget")(self.h, _dptr(out)), "get_budget")
        return out

    def check_finite(self):
        """Raises PIError (PI_ERR_NAN) naming the first tracer cell or active individual holding a
        NaN or Inf."""
        self._check(self._fn("check_finite")(self.h), "check_finite")

    def get_diag(self, kind, sp=0):
        out = np.empty(self.G, dtype=np.float64)
        self._check(self._fn("get_diag")(self.h, int(kind), int(sp), _dptr(out)), "get_diag")
        return out.reshape(self.gshape, order="F")

    # ---- abiotic particles (src/Individuals/Abiotic/) --------------------------------------------
    def set_abiotics(self, params, nsa, intac=(), release=(), max_candidates=25, max_ptc=None):
        """abiotic_setup(params, N, Nsa, Palat(intac, release)) and max_candidates of PlanktonModel:
        params maps each of ABIOTIC_FIELDS to nsa values; intac and release are (phytoplankton
        species, abiotic species) 0-based pairs; max_ptc holds each phytoplankton species'
        max_ptc (NaN where the mode has none, the default)."""
        ps = (_abi.pi_abiotic_params * nsa)()
        for a in range(nsa):
            for k in _abi.ABIOTIC_FIELDS:
                setattr(ps[a], k, float(np.asarray(params[k], dtype=np.float64).ravel()[a]))
        def pairs(lst):
            arr = (ct.c_int32 * max(1, 2 * len(lst)))()
            for q, (p, a) in enumerate(lst):
                arr[2 * q], arr[2 * q + 1] = int(p), int(a)
            return arr
        mp = np.full(self.nsp, np.nan) if max_ptc is None else np.asarray(max_ptc, dtype=np.float64)
        mp = np.ascontiguousarray(mp)
        self._keep.append(mp)
        self._check(self._fn("set_abiotics")(self.h, int(nsa), ps, len(intac), pairs(intac), len(release),
                                             pairs(release), int(max_candidates), _dptr(mp)), "set_abiotics")
        self.nsa = nsa

    def set_abiotic_particles(self, sa, data):
        C = self.capacity
        st = _abi.pi_abiotic_particles()
        keep = []
        for k in ("x", "y", "z"):
            a = np.ascontiguousarray(data[k], dtype=np.float64)
            if a.shape != (C,):
                raise ValueError(f"abiotic attribute {k} must have length {C}")
            keep.append(a)
            setattr(st, k, _dptr(a))
        for k in IND_INT:
            if data.get(k) is not None:
                a = np.ascontiguousarray(data[k], dtype=np.int64)
                keep.append(a)
                setattr(st, k, a.ctypes.data_as(ct.POINTER(ct.c_int64)))
        ac = np.ascontiguousarray(data["ac"], dtype=np.uint8)
        keep.append(ac)
        st.ac = ac.ctypes.data_as(ct.POINTER(ct.c_uint8))
        self._check(self._fn("set_abiotic_particles")(self.h, int(sa), ct.byref(st)), "set_abiotic_particles")

    def get_abiotic_particles(self, sa):
        C = self.capacity
        out = {k: np.empty(C, dtype=np.float64) for k in ("x", "y", "z")}
        out.update({k: np.empty(C, dtype=np.int64) for k in IND_INT})
        out["ac"] = np.empty(C, dtype=np.uint8)
        st = _abi.pi_abiotic_particles()
        for k in ("x", "y", "z"):
            setattr(st, k, _dptr(out[k]))
        for k in IND_INT:
            setattr(st, k, out[k].ctypes.data_as(ct.POINTER(ct.c_int64)))
        st.ac = out["ac"].ctypes.data_as(ct.POINTER(ct.c_uint8))
        self._check(self._fn("get_abiotic_particles")(self.h, int(sa), ct.byref(st)), "get_abiotic_particles")
        out["ac"] = out["ac"].astype(bool)
        return out

    def count_abiotic(self, sa):
        n = ct.c_int64()
        self._check(self._fn("count_abiotic")(self.h, int(sa), ct.byref(n)), "count_abiotic")
        return n.value

    def set_abiotic_bc(self, sa, face, kind, values=None, nt=0):
        if values is None:
            p = ct.POINTER(ct.c_double)()
        else:
            values = np.asfortranarray(np.atleast_1d(np.asarray(values, dtype=np.float64)))
            self._keep.append(values)
            p = _dptr(values.ravel(order="F"))
        self._check(self._fn("set_abiotic_bc")(self.h, int(sa), int(face), int(kind), p, int(nt)), "set_abiotic_bc")

    def set_state(self, individuals, tracers):
        """Upload a full initial state: individuals = list (per species) of attribute dicts,
        tracers = sequence of NTRACERS halo-padded arrays."""
        for s, d in enumerate(individuals):
            self.set_individuals(s, d)
        for n in range(NTRACERS):
            self.set_tracer(n, tracers[n])
