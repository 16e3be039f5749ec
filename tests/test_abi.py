"""The C ABI library loads without a GPU and exports every entry point include/pib200.h declares;
host-side validation that needs no device."""
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
