"""The optional diagnostics of the CPU oracle (PlanktonDiagnostics(model; tracer, phytoplankton),
src/Diagnostics/diagnostics_struct.jl:23-105, diags_spcs! in diagnostics_kernels.jl:14-33 and the
tracer sums of time_step.jl:168-172), checked against sums formed here from the oracle's own
state: after one step each process field equals the ascending-slot sum of the process over the
active individuals of each find_inds! cell (tolerance 0); tracer fields equal the sum of the
tracer after each step (tolerance 0); over several steps the totals agree to rounding."""
import numpy as np

import oracle
from PlanktonIndividuals import _abi, workloads as W
from helpers import VelCache, drive

ALL_PROC = (1 << len(_abi.PROC_NAMES)) - 1


def _values(ref, s):
    A, R = ref.get_individuals(s), ref.get_rates(s)
    v = {k: R[k] for k in ("PS", "BS", "VDOC", "VNH4", "VNO3", "VPO4", "resp", "exu")}
    v.update({k: A[k] for k in ("Bm", "Cq", "Nq", "Pq", "Chl")})
    return A, v


def _cell_sums(ref, A, vals, g):
    out = np.zeros(g.total_size, order="F")
    for i in np.nonzero(A["ac"])[0]:          # ascending slot, as diags_proc! on one thread
        c = (A["xi"][i] - 1, A["yi"][i] - 1, A["zi"][i] - 1)
        out[c] = out[c] + vals[i]
    return out


def test_oracle_optional_diagnostics():
    over = {"dvid_P": [1e-3, 2e-3], "dvid_reg": [1.0, 1.1], "mort_P": [3e-4, 3e-4], "grz_P": [1e-4, 0.0]}
    wl = W.config2(nx=10, nz=6, N_per_species=400, steps=6, nmodes=8, seed=71, phyt_over=over)
    wl.parf = np.asfortranarray(np.roll(wl.parf, -10, axis=2))
    g = wl.grid
    ref = oracle.from_workload(wl)
    tmask = (1 << _abi.tracer_names.index("NO3")) | (1 << _abi.tracer_names.index("DOC")) | (1 << 13)
    ref.set_diags(tmask, ALL_PROC)
    vel = VelCache(wl)
    drive(ref, wl, 1, vel)
    for s in range(wl.nsp):
        A, vals = _values(ref, s)
        for q, name in enumerate(_abi.PROC_NAMES):
            assert np.array_equal(ref.get_diag(_abi.PI_DIAG_PROC + q, s), _cell_sums(ref, A, vals[name], g)), name
    trsum = {n: ref.get_tracer(n).copy() for n in range(_abi.NTRACERS) if tmask >> n & 1}
    tot = {(s, name): float(np.sum(_values(ref, s)[1][name][_values(ref, s)[0]["ac"]]))
           for s in range(wl.nsp) for name in _abi.PROC_NAMES}
    for _ in range(4):
        drive(ref, wl, 1, vel)
        for n in trsum:
            trsum[n] = trsum[n] + ref.get_tracer(n)
        for s in range(wl.nsp):
            A, vals = _values(ref, s)
            for name in _abi.PROC_NAMES:
                tot[(s, name)] += float(np.sum(vals[name][A["ac"]]))
    for n, a in trsum.items():
        assert np.array_equal(ref.get_diag(_abi.PI_DIAG_TRACER + n, 0), a), _abi.tracer_names[n]
    for (s, name), t in tot.items():
        got = float(np.sum(ref.get_diag(_abi.PI_DIAG_PROC + _abi.PROC_NAMES.index(name), s)))
        assert abs(got - t) <= 1e-12 * max(abs(t), 1e-300), (s, name, got, t)
    # disabled kinds are rejected
    ref.set_diags(0, 0)
    import pytest
    from PlanktonIndividuals._native import PIError
    with pytest.raises(PIError):
        ref.get_diag(_abi.PI_DIAG_PROC, 0)
