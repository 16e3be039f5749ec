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


def _step_reference(lib, wl, dic, vel, grid=None):
    """pi_time_step on a model whose only non-zero tracer is `dic` and which has no individuals."""
    g = grid if grid is not None else wl.grid
    m = CModel(lib, "pi_", g, wl.bgc, wl.phyt, 1, 8, seed=0, precision=_abi.PI_FP64)
    zeros = np.zeros(g.total_size, order="F")
    m.set_state([empty_individuals(8)], [dic] + [zeros] * (_abi.NTRACERS - 1))
    m.set_velocity(*vel)
    m.set_PARF(np.zeros((g.Nx, g.Ny)))
    m.set_temp(np.zeros(g.size))
    m.time_step(wl.dT)
    out = m.get_tracer(0)
    m.close()
    return out


def _padded_velocity(g, u, v, w):
    """Halo-padded u, v, w exactly as vel_copy! + fill_halo_vel! build them (the +1 face on
    Bounded axes included)."""
    U, V, Wf = (np.zeros(g.total_size, order="F") for _ in range(3))
    bx = 1 if g.topo[0] == _abi.PI_BOUNDED else 0
    by = 1 if g.topo[1] == _abi.PI_BOUNDED else 0
    U[g.Hx:g.Hx + g.Nx + bx, g.Hy:g.Hy + g.Ny, g.Hz:g.Hz + g.Nz] = u
    V[g.Hx:g.Hx + g.Nx, g.Hy:g.Hy + g.Ny + by, g.Hz:g.Hz + g.Nz] = v
    Wf[g.Hx:g.Hx + g.Nx, g.Hy:g.Hy + g.Ny, g.Hz:g.Hz + g.Nz + 1] = w
    G.fill_halo_vel(U, V, Wf, g)
    return U, V, Wf


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


def _masked_grid(size, topology, z, seed):
    """A grid with land: a sloping bottom under the western columns and a block of land through
    the upper levels (the mask differs with the size and seed)."""
    Nx, Ny, Nz = size
    rng = np.random.default_rng(seed)
    lm = np.ones(size, dtype=bool)
    for i in range(Nx // 3):
        lm[i, :, Nz - 1 - (Nx // 3 - i) * Nz // (Nx // 3 + 1):] = False
    i0, j0 = int(rng.integers(Nx // 3, Nx - 3)), int(rng.integers(1, Ny - 4))
    lm[i0:i0 + 2, j0:j0 + 3, :max(1, Nz // 2)] = False
    return G.RectilinearGrid(size=size, x=(0.0, Nx * 800.0), y=(0.0, Ny * 700.0), z=z, FT=np.float64,
                             topology=topology, landmask=lm)


def test_noalloc_bounded_landmask_and_changing_grid(gpu_lib):
    """Bounded x/y (zero flux through the last face), a partial 3D land mask and a stretched
    vertical grid, then a second call on another grid (other size, spacing, topology and mask):
    each call must equal the advection of pi_time_step bit for bit, so nothing of the first
    call's metrics, mask or intermediates may leak into the second."""
    import torch
    lib = gpu_lib
    f = _declare(lib)
    wl = W.config2(nx=8, nz=4, N_per_species=10, nsp=1, steps=2, nmodes=8, seed=3)
    stretched = tuple(-np.concatenate([[0.0], np.cumsum(np.linspace(1.0, 4.0, 6))]))
    grids = [_masked_grid((14, 12, 6), (G.Bounded, G.Bounded, G.Bounded), np.array(stretched), seed=1),
             _masked_grid((18, 10, 5), (G.Periodic, G.Bounded, G.Bounded), (0.0, -15.0), seed=2)]
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(9)
    for call, g in enumerate(grids):
        bx = 1 if g.topo[0] == _abi.PI_BOUNDED else 0
        by = 1 if g.topo[1] == _abi.PI_BOUNDED else 0
        u = np.asfortranarray(rng.uniform(-0.3, 0.3, (g.Nx + bx, g.Ny, g.Nz)))
        v = np.asfortranarray(rng.uniform(-0.3, 0.3, (g.Nx, g.Ny + by, g.Nz)))
        w = np.asfortranarray(rng.uniform(-2e-3, 2e-3, (g.Nx, g.Ny, g.Nz + 1)))
        w[:, :, 0] = 0.0
        w[:, :, -1] = 0.0
        if bx:
            u[0] = u[-1] = 0.0
        if by:
            v[:, 0] = v[:, -1] = 0.0
        dU, dV, dW = (_padded(a, g) for a in _padded_velocity(g, u, v, w))
        dic = np.asfortranarray(20.0 * rng.uniform(0.5, 1.5, g.total_size)) * g.landmask
        dic = np.asfortranarray(dic)
        G.fill_halo_tracer(dic, g)
        ref = _step_reference(lib, wl, dic, (u, v, w), grid=g)
        gs, keep = make_grid_struct(g)
        dc = _padded(dic, g)
        dGc = torch.full((dic.size,), np.nan, dtype=torch.float64, device="cuda")
        rc = f(ct.byref(gs), dc.data_ptr(), dU.data_ptr(), dV.data_ptr(), dW.data_ptr(), wl.dT,
               dGc.data_ptr(), stream)
        assert rc == 0
        del keep, gs     # the host metrics may go once the call has returned
        torch.cuda.synchronize()
        Gc = dGc.cpu().numpy().reshape(g.total_size, order="F")
        got = G.interior(dic, g) + G.interior(Gc, g)
        assert np.array_equal(got, G.interior(ref, g)), f"call {call + 1} differs from pi_time_step"
        assert not np.array_equal(G.interior(Gc, g), np.zeros_like(G.interior(Gc, g)))
