"""Per-output error of the FP32 form against the FP64 form on the same workload.

The FP64 form computes the reference's step in Float64 (bit for bit equal to the CPU oracle in the
GPU tests); the FP32 form computes the bulk of the step in Float32. These helpers run both from
the same initial state and forcing series (device-resident, as PlanktonSimulation keeps them) and
report population counts, active-slot and cell mismatches, quota errors and interior tracer-mass
errors."""
import ctypes as ct

import numpy as np

from . import _abi

_SNAPS = {}


def snapshots(wl, nsnap):
    """Velocity snapshots 0..nsnap-1 of a workload, computed once per process."""
    have = _SNAPS.setdefault(id(wl), [])
    while len(have) < nsnap:
        have.append(wl.velocity(len(have)))
    return have[:nsnap]


def series_arrays(wl, nsnap):
    """u, v, w snapshot series (…, nsnap) of a workload, as PlanktonSimulation takes them."""
    snaps = snapshots(wl, nsnap)
    return {c: np.stack([sn[q] for sn in snaps], axis=-1) for q, c in enumerate("uvw")}


def interior_mass(get, g):
    """Σ tracer · volume over the interior, per tracer (get(n) returns tracer n with halos)."""
    from .grids import cell_volumes
    vol = cell_volumes(g)[g.Hx:g.Hx + g.Nx, g.Hy:g.Hy + g.Ny, g.Hz:g.Hz + g.Nz]
    out = {}
    for n, name in enumerate(_abi.tracer_names):
        a = get(n)[g.Hx:g.Hx + g.Nx, g.Hy:g.Hy + g.Ny, g.Hz:g.Hz + g.Nz]
        out[name] = float(np.sum(a * vol))
    return out


def mass_rel(M32, M64):
    return {k: (abs(M32[k] - M64[k]) / abs(M64[k]) if M64[k] else abs(M32[k])) for k in M64}


def fp64_sim(lib, wl, steps):
    """A PI_FP64 model of the workload with its forcing series on the device (pi_sim_create);
    returns (model, sim handle, arrays kept alive)."""
    from ._native import CModel
    m = CModel(lib, "pi_", wl.grid, wl.bgc, wl.phyt, wl.nsp, wl.capacity, wl.seed, precision=_abi.PI_FP64)
    m.set_state(wl.individuals, wl.tracers)
    nsnap = wl.snapshots_needed(steps + 1)
    vv = series_arrays(wl, nsnap)
    u, v, w = (np.asfortranarray(vv[c]) for c in "uvw")
    dp = lambda a: a.ctypes.data_as(ct.POINTER(ct.c_double))
    sim = ct.c_void_p()
    rc = lib.pi_sim_create(m.h, wl.dT, 1, dp(u), dp(v), dp(w), nsnap, wl.dT_vel, dp(wl.parf), wl.parf.shape[2],
                           wl.dT_PAR, dp(wl.temp), wl.temp.shape[3], wl.dT_temp, ct.byref(sim))
    if rc != 0:
        raise RuntimeError(m._errmsg(m.h))
    return m, sim, (u, v, w)


def fp32_batch(members, steps):
    """The FP32 batched form of the workloads (one member each) with their forcing series."""
    from .batch import Member, PlanktonBatch
    b = PlanktonBatch([Member(w.grid, w.bgc, w.phyt, w.capacity, w.seed) for w in members], nspecies=members[0].nsp)
    for m, wl in enumerate(members):
        b.set_state(m, wl.individuals, wl.tracers)
        b.set_series(m, vels=series_arrays(wl, wl.snapshots_needed(steps + 1)), ΔT_vel=wl.dT_vel, PARF=wl.parf,
                     ΔT_PAR=wl.dT_PAR, temp=wl.temp, ΔT_temp=wl.dT_temp)
    return b


def individual_errors(A, B):
    """Errors of the FP32 individuals B against the FP64 individuals A of one species."""
    both = A["ac"] & B["ac"]
    out = {"ac_mismatch": int(np.sum(A["ac"] != B["ac"])),
           "cell_mismatch": int(np.sum(both & ((A["xi"] != B["xi"]) | (A["yi"] != B["yi"]) | (A["zi"] != B["zi"])))),
           "quota_rel_max": {k: (float(np.max(np.abs(A[k][both] - B[k][both]) / np.abs(A[k][both]))) if both.any() else 0.0)
                             for k in ("Bm", "Cq", "Nq", "Pq", "Chl")},
           "z_abs_max": float(np.max(np.abs(A["z"][both] - B["z"][both]))) if both.any() else 0.0}
    # population totals: meaningful also after a decision flip has moved daughters to other slots
    tot = {}
    for k in ("Bm", "Cq", "Nq", "Pq", "Chl"):
        t64, t32 = float(np.sum(A[k][A["ac"]])), float(np.sum(B[k][B["ac"]]))
        tot[k] = abs(t32 - t64) / abs(t64) if t64 else abs(t32)
    n64, n32 = int(A["ac"].sum()), int(B["ac"].sum())
    out["count_rel_diff"] = abs(n32 - n64) / n64 if n64 else float(n32)
    out["total_rel_diff"] = tot
    return out


def fp32_vs_fp64(lib, wl, steps, check_every=100):
    """Runs `steps` steps of the workload in both forms; population counts are compared every
    `check_every` steps, everything else at the end."""
    m64, sim, keep = fp64_sim(lib, wl, steps)
    b = fp32_batch([wl], steps)
    hist = []
    try:
        for s0 in range(0, steps, check_every):
            n = min(check_every, steps - s0)
            for _ in range(n):
                if lib.pi_sim_update(sim, 0, 0) != 0:
                    raise RuntimeError(m64._errmsg(m64.h))
            if lib.pi_synchronize(m64.h) != 0:
                raise RuntimeError(m64._errmsg(m64.h))
            b.step(wl.dT, n)
            hist.append({"step": s0 + n, "fp64": [m64.count_active(s) for s in range(wl.nsp)],
                         "fp32": [b.count_active(0, s) for s in range(wl.nsp)]})
        rel = mass_rel(interior_mass(lambda n: b.get_tracer(0, n), wl.grid), interior_mass(m64.get_tracer, wl.grid))
        inds = {f"sp{s}": individual_errors(m64.get_individuals(s), b.get_individuals(0, s)) for s in range(wl.nsp)}
        return {"steps": steps, "counts_equal_at_every_check": all(h["fp64"] == h["fp32"] for h in hist),
                "counts": hist, "tracer_mass_rel_err": rel, "max_tracer_mass_rel_err": max(rel.values()),
                "individuals": inds, "budget_fp32": b.budget(0),
                "guard_band": dict(zip(("recomputed", "changed"), b.guard_stats()))}
    finally:
        b.close()
        lib.pi_sim_destroy(sim)
        m64.close()
