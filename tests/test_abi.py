"""The C ABI library loads without a GPU and exports every entry point include/pib200.h declares;
host-side validation that needs no device."""
import ctypes as ct
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "pib200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:pi_status|const char\*)\s+(pi_\w+)\s*\(", txt, re.M)))


def test_library_exports_every_declared_symbol():
    import build
    build.build()
    from PlanktonIndividuals import _lib
    lib = _lib.load()
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(_lib.EXPORTS) <= set(names)


def test_status_strings_and_create_without_gpu():
    from PlanktonIndividuals import _lib
    lib = _lib.load()
    assert lib.pi_status_string(0) == b"ok"
    assert lib.pi_status_string(4).startswith(b"number of individuals")


def test_simulation_requires_gpu_arch():
    from PlanktonIndividuals import CPU, PlanktonModel, RectilinearGrid
    g = RectilinearGrid(size=(4, 4, 1), x=(0, 4), y=(0, 4), z=(0, -1))
    with pytest.raises(ValueError, match="GPU"):
        PlanktonModel(CPU(), g)


def test_header_mentions_reference_interfaces():
    txt = open(os.path.join(ROOT, "include", "pib200.h")).read()
    for ref in ("models.jl:51", "time_step.jl:12", "update.jl:11", "simulations.jl:98", "utils.jl:5"):
        assert ref in txt


def _batch_create_status(grid_over):
    """pi_batch_create on one member whose grid fields are overridden; returns (status, message)."""
    from PlanktonIndividuals import _abi, _lib
    from PlanktonIndividuals._native import make_bgc_struct, make_species_structs
    from PlanktonIndividuals.parameters import bgc_params_default, phyt_params_default
    lib = _lib.load()
    g = _abi.pi_grid()
    g.Nx, g.Ny, g.Nz, g.Hx, g.Hy, g.Hz = 8, 8, 4, 2, 2, 2
    for a in range(3):
        g.topo[a] = [_abi.PI_PERIODIC, _abi.PI_PERIODIC, _abi.PI_BOUNDED][a]
    g.dx = g.dy = 10.0
    for k, v in grid_over.items():
        if k == "topo":
            for a in range(3):
                g.topo[a] = v[a]
        else:
            setattr(g, k, v)
    dz = np.ones(g.Nz + 2 * g.Hz)
    g.dzF = dz.ctypes.data_as(ct.POINTER(ct.c_double))
    g.dzC = dz.ctypes.data_as(ct.POINTER(ct.c_double))
    b = make_bgc_struct(bgc_params_default(np.float64))
    sp = make_species_structs(phyt_params_default(1), 1)
    mem = (_abi.pi_member * 1)()
    mem[0].grid = ct.pointer(g)
    mem[0].bgc = ct.pointer(b)
    mem[0].species = ct.cast(sp, ct.POINTER(_abi.pi_quota_params))
    mem[0].capacity = 16
    mem[0].seed = 1
    h = ct.c_void_p()
    rc = lib.pi_batch_create(mem, 1, 1, ct.byref(h))
    buf = ct.create_string_buffer(512)
    lib.pi_batch_last_error(None, buf, 512)
    if rc == _abi.PI_OK:
        lib.pi_batch_destroy(h)
    return rc, buf.value.decode()


def test_batch_create_rejects_bad_members_before_touching_a_device():
    from PlanktonIndividuals import _abi
    rc, msg = _batch_create_status({"Hx": 1})
    assert rc == _abi.PI_ERR_ARG and "halo must be 2..8" in msg
    rc, msg = _batch_create_status({"topo": (_abi.PI_PERIODIC, _abi.PI_PERIODIC, _abi.PI_PERIODIC)})
    assert rc == _abi.PI_ERR_ARG and "z must be Bounded" in msg
    # 4097 × 4097 × 64 halo-padded cells fit in 31 bits, but the three bit fields of a cell code
    # need 13 + 13 + 7 bits
    rc, msg = _batch_create_status({"Nx": 4093, "Ny": 4093, "Nz": 60})
    assert rc == _abi.PI_ERR_ARG and "too large" in msg
    rc, _ = _batch_create_status({})
    assert rc in (_abi.PI_OK, _abi.PI_ERR_CUDA)      # a valid member: created, or no device here


def test_julia_binding_calls_only_declared_symbols():
    """The Julia module (untested here: no Julia) binds symbols that include/pib200.h declares."""
    src = open(os.path.join(ROOT, "planktonindividuals.jl_b200", "julia", "PIB200.jl")).read()
    called = set(re.findall(r"ccall\(\(:(pi_\w+), lib\)", src))
    assert len(called) >= 20
    assert called <= set(declared_symbols())
