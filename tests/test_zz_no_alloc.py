"""The allocation-free advection entry point against the regular step.

pi_tracer_advection_noalloc is for callers that cannot allocate device memory (a host runtime
that owns every device allocation through its own pool, or a loop that must not allocate after
start-up); its scratch is a fixed device array inside the library. Here it must reproduce, bit for
bit, the advection part of pi_time_step: with only DIC non-zero and no individuals, one step
changes DIC's interior by exactly the advection tendency (its forcing, diffusion and particle
terms are zero). Two calls in a row on different fields check that the shared scratch carries
nothing from one call into the next. The tolerance is 0, as in the other parity tests.
"""
import ctypes as ct

import numpy as np
import pytest

from PlanktonIndividuals import _abi, grids as G, workloads as W
from PlanktonIndividuals._native import CModel, make_grid_struct
from PlanktonIndividuals.init import empty_individuals

pytestmark = pytest.mark.gpu


def _declare(lib):
    dp = ct.POINTER(ct.c_double)
    f = lib.pi_tracer_advection_noalloc
    f.restype = ct.c_int32
    f.argtypes = [ct.POINTER(_abi.pi_grid), ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                  ct.c_double, ct.c_void_p, ct.c_void_p]
    lib.pi_noalloc_last_error.restype = ct.c_int32
    lib.pi_noalloc_last_error.argtypes = [ct.c_char_p, ct.c_size_t]
    return f


def _step_reference(lib, wl, dic, vel):
    """pi_time_step on a model whose only non-zero tracer is `dic` and which has no individuals."""
    m = CModel(lib, "pi_", wl.grid, wl.bgc, wl.phyt, 1, 8, seed=0, precision=_abi.PI_FP64)
    zeros = np.zeros(wl.grid.total_size, order="F")
    m.set_state([empty_individuals(8)], [dic] + [zeros] * (_abi.NTRACERS - 1))
    m.set_velocity(*vel)
    m.set_PARF(np.zeros((wl.grid.Nx, wl.grid.Ny)))
    m.set_temp(np.zeros(wl.grid.size))
    m.time_step(wl.dT)
    out = m.get_tracer(0)
    m.close()
    return out


def _padded(a, g):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a.ravel(order="F"))).cuda()


def test_noalloc_advection_matches_time_step_twice(gpu_lib):
    import torch
    lib = gpu_lib
    f = _declare(lib)
    wl = W.config2(nx=20, nz=10, N_per_species=10, nsp=1, steps=2, nmodes=16, seed=11)
    g = wl.grid
    u, v, w = wl.velocity(0)
    # halo-padded velocities exactly as vel_copy! builds them
    U, V, Wf = (np.zeros(g.total_size, order="F") for _ in range(3))
    U[g.Hx:g.Hx + g.Nx, g.Hy:g.Hy + g.Ny, g.Hz:g.Hz + g.Nz] = u
    V[g.Hx:g.Hx + g.Nx, g.Hy:g.Hy + g.Ny, g.Hz:g.Hz + g.Nz] = v
    Wf[g.Hx:g.Hx + g.Nx, g.Hy:g.Hy + g.Ny, g.Hz:g.Hz + g.Nz + 1] = w
    G.fill_halo_vel(U, V, Wf, g)
    dU, dV, dW = _padded(U, g), _padded(V, g), _padded(Wf, g)
    gs, keep = make_grid_struct(g)
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(5)
    for call in range(2):
        dic = np.asfortranarray(20.0 * rng.uniform(0.5, 1.5, g.total_size))
        G.fill_halo_tracer(dic, g)
        ref = _step_reference(lib, wl, dic, (u, v, w))
        dc = _padded(dic, g)
        dGc = torch.full((dic.size,), np.nan, dtype=torch.float64, device="cuda")
        rc = f(ct.byref(gs), dc.data_ptr(), dU.data_ptr(), dV.data_ptr(), dW.data_ptr(), wl.dT,
               dGc.data_ptr(), stream)
        assert rc == 0
        torch.cuda.synchronize()
        Gc = dGc.cpu().numpy().reshape(g.total_size, order="F")
        got = G.interior(dic, g) + G.interior(Gc, g)
        assert np.array_equal(got, G.interior(ref, g)), f"call {call + 1} differs from pi_time_step"


def test_noalloc_rejects_grids_beyond_the_fixed_scratch(gpu_lib):
    import torch
    f = _declare(gpu_lib)
    g = G.RectilinearGrid(size=(100, 100, 60), x=(0, 1e3), y=(0, 1e3), z=(0, -60), FT=np.float64)
    gs, keep = make_grid_struct(g)
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = f(ct.byref(gs), x.data_ptr(), x.data_ptr(), x.data_ptr(), x.data_ptr(), 1.0, x.data_ptr(), None)
    assert rc == _abi.PI_ERR_ARG
    buf = ct.create_string_buffer(256)
    gpu_lib.pi_noalloc_last_error(buf, 256)
    assert b"exceeds the fixed scratch" in buf.value
