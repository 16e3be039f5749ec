"""PlanktonIndividuals — the model time step of PlanktonIndividuals.jl on NVIDIA B200 (sm_100a).

The Python names follow the Julia API with `!` written as `_b`:

    grid  = RectilinearGrid(size=(128, 128, 1), x=(0, 128e3), y=(0, 128e3), z=(0, -10), FT=np.float64)
    model = PlanktonModel(GPU(), grid, FT=np.float64, max_individuals=2**15,
                          phyto=phyto_setup(None, [2**14], 1))
    sim   = PlanktonSimulation(model, ΔT=60.0, iterations=1440, vels=dict(u=u, v=v, w=w))
    update_b(sim)

All numerical work runs in libpib200.so (CUDA); there is no CPU fallback.
"""
from ._abi import tracer_names
from ._native import CapacityError, PIError
from .architectures import CPU, GPU, CarbonMode, IronEnergyMode, MacroMolecularMode, QuotaMode
from .grids import (Ax, Ay, Az, Bounded, LatLonGrid, LoadLatLonGrid, Periodic, RectilinearGrid, interior,
                    volume, ΔxC, ΔxF, ΔyC, ΔyF, ΔzC, ΔzF)
from .model import (Palat, PlanktonDiagnostics, PlanktonModel, TimeStep_b, abiotic_setup, phyto_setup,
                    set_bc_b, set_bc_particle_b)
from .parameters import (abiotic_params_default, bgc_params_default, default_PARF, default_temperature,
                         default_tracer_init, phyt_params_default, update_abiotic_params, update_bgc_params,
                         update_phyt_params)
from .simulation import PlanktonSimulation, synchronize, update_b
from .output import PlanktonOutputWriter, write_output_b
from .batch import BatchMember, Member, PlanktonBatch
from . import units

__all__ = ["RectilinearGrid", "LatLonGrid", "LoadLatLonGrid", "Periodic", "Bounded", "PlanktonModel", "PlanktonSimulation",
           "PlanktonDiagnostics", "update_b", "TimeStep_b", "synchronize", "phyto_setup", "GPU", "CPU",
           "QuotaMode", "CarbonMode", "MacroMolecularMode", "IronEnergyMode", "tracer_names",
           "bgc_params_default", "phyt_params_default", "update_bgc_params", "update_phyt_params",
           "default_PARF", "default_temperature", "default_tracer_init", "interior", "units",
           "CapacityError", "PIError", "ΔxC", "ΔyC", "ΔzC", "ΔxF", "ΔyF", "ΔzF", "Ax", "Ay", "Az",
           "volume", "PlanktonBatch", "Member", "BatchMember", "PlanktonOutputWriter", "write_output_b",
           "abiotic_setup", "Palat", "abiotic_params_default", "update_abiotic_params", "set_bc_b",
           "set_bc_particle_b"]
