"""PlanktonSimulation and update! (src/Simulation/simulations.jl, src/Simulation/update.jl,
src/Simulation/utils.jl). The forcing series are copied to device memory once; each step binds
its velocity, PAR and temperature snapshot on the device."""
import ctypes as ct

import numpy as np

from ._abi import PI_BOUNDED, PI_OK
from ._native import CapacityError, PIError, _dptr
from .model import PlanktonDiagnostics
from .parameters import default_PARF, default_temperature


def _f64_fortran(a, ndim):
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == ndim - 1:
        a = a[..., None]
    return np.asfortranarray(a)


class PlanktonSimulation:
    """PlanktonSimulation(model; ΔT, iterations, PARF, temp, diags, vels, ΔT_vel, ΔT_PAR, ΔT_temp,
    output_writer). `vels` is a dict with u, v, w of shape (Nx[+1], Ny[+1], Nz[+1], nΔT), the +1
    on Bounded axes; PARF is (Nx, Ny, nΔT); temp is (Nx, Ny, Nz, nΔT)."""

    def __init__(self, model, *, ΔT, iterations, PARF=None, temp=None, diags=None, vels=None,
                 ΔT_vel=None, ΔT_PAR=3600.0, ΔT_temp=3600.0, output_writer=None):
        FT = model.FT
        self.output_writer = output_writer
        g = model.grid
        self.model = model
        self.ΔT = float(FT(ΔT))
        self.iterations = int(iterations)
        if PARF is None:
            PARF = default_PARF(g, ΔT, iterations)
        if temp is None:
            temp = default_temperature(g, ΔT, iterations)
        ΔT_vel = ΔT if ΔT_vel is None else ΔT_vel
        self.ΔT_vel, self.ΔT_PAR, self.ΔT_temp = float(FT(ΔT_vel)), float(FT(ΔT_PAR)), float(FT(ΔT_temp))
        PARF = _f64_fortran(np.asarray(PARF).astype(FT), 3)
        temp = _f64_fortran(np.asarray(temp).astype(FT), 4)
        self.diags = diags if diags is not None else PlanktonDiagnostics(model)
        # validate_temp / validate_PARF / validate_velocity (Simulation/utils.jl:213-304)
        if temp.shape[:3] != g.size:
            raise ValueError(f"Dimension mismatch: the size of temperature must be {g.size}.")
        if PARF.shape[:2] != (g.Nx, g.Ny):
            raise ValueError(f"Dimension mismatch: the size of PARF must be {(g.Nx, g.Ny)}.")
        keep = [PARF, temp]
        null = ct.POINTER(ct.c_double)()
        if vels:
            b = [int(t == PI_BOUNDED) for t in g.topo]
            u = _f64_fortran(np.asarray(vels["u"]).astype(FT), 4)
            v = _f64_fortran(np.asarray(vels["v"]).astype(FT), 4)
            w = _f64_fortran(np.asarray(vels["w"]).astype(FT), 4)
            names = ("Periodic", "Bounded")
            for a, shp, ax in ((u, (g.Nx + b[0], g.Ny, g.Nz), 0), (v, (g.Nx, g.Ny + b[1], g.Nz), 1),
                               (w, (g.Nx, g.Ny, g.Nz + b[2]), 2)):
                if a.shape[:3] != shp:
                    raise ValueError(f"Dimension mismatch: the size of {'uvw'[ax]} must be {shp}, "
                                     f"for {names[b[ax]]} topology.")
            if not (u.shape[3] == v.shape[3] == w.shape[3]):
                raise ValueError("u, v and w must have the same number of snapshots")
            keep += [u, v, w]
            pu, pv, pw, nvel = _dptr(u), _dptr(v), _dptr(w), u.shape[3]
        else:
            pu = pv = pw = null
            nvel = 0
        self.input = dict(PARF=PARF, temp=temp, vels=vels, ΔT_vel=self.ΔT_vel,
                          ΔT_PAR=self.ΔT_PAR, ΔT_temp=self.ΔT_temp)
        nat = model._native
        h = ct.c_void_p()
        rc = nat.lib.pi_sim_create(nat.h, self.ΔT, self.iterations, pu, pv, pw, int(nvel), self.ΔT_vel,
                                   _dptr(PARF), int(PARF.shape[2]), self.ΔT_PAR,
                                   _dptr(temp), int(temp.shape[3]), self.ΔT_temp, ct.byref(h))
        if rc != PI_OK:
            raise ValueError(nat._errmsg(nat.h))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self.model._native.lib.pi_sim_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __repr__(self):
        return (f"PlanktonSimulation:\n├── ΔT: {self.ΔT}s\n├── model time: {self.model.t}s\n"
                f"├── simulation stops after: {self.iterations} iterations")


def update_b(sim, time_offset=None, sync=True):
    """update!(sim; time_offset) (src/Simulation/update.jl:11-48). `sync=False` returns once the
    steps are queued on the GPU; call `synchronize(sim.model)` to wait and collect errors. With an
    output writer, every step is followed by write_output! (update.jl:30), so the steps run one
    call each."""
    to = time_offset or {}
    mask = (1 if to.get("vels") else 0) | (2 if to.get("PARF") else 0) | (4 if to.get("temp") else 0)
    nat = sim.model._native

    def check(rc):
        if rc != PI_OK:
            msg = nat._errmsg(nat.h)
            if rc == 4:
                raise CapacityError(rc, msg)
            raise PIError(rc, msg)

    if sim.output_writer is None:
        check(nat.lib.pi_sim_update(sim._h, mask, 1 if sync else 0))
        return
    from .output import write_output_b
    for i in range(1, sim.iterations + 1):
        check(nat.lib.pi_sim_update_steps(sim._h, ct.c_int64(i), ct.c_int64(1), mask, 1))
        write_output_b(sim.output_writer, sim.model, sim.diags)


def synchronize(model):
    nat = model._native
    rc = nat.lib.pi_synchronize(nat.h)
    if rc != PI_OK:
        msg = nat._errmsg(nat.h)
        if rc == 4:
            raise CapacityError(rc, msg)
        raise PIError(rc, msg)
