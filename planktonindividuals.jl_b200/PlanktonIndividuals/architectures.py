"""Architectures and physiology modes (src/Architectures.jl, src/PlanktonIndividuals.jl:59-83).
GPU() with QuotaMode() (both precisions), CarbonMode(), MacroMolecularMode() and IronEnergyMode()
(Float64) are implemented."""


class Architecture:
    pass


class GPU(Architecture):
    """One CUDA GPU (sm_100a)."""

    def __repr__(self):
        return "GPU()"


class CPU(Architecture):
    """Present for API compatibility; constructing a model on CPU() raises (no CPU fallback)."""

    def __repr__(self):
        return "CPU()"


class AbstractMode:
    pass


class QuotaMode(AbstractMode):
    """C, N and P quotas (the reference default)."""

    def __repr__(self):
        return "QuotaMode()"


class CarbonMode(AbstractMode):
    """Carbon only: biomass, damaged biomass and Chl (src/Individuals/Plankton/CarbonMode/)."""

    def __repr__(self):
        return "CarbonMode()"


class MacroMolecularMode(AbstractMode):
    """Protein, DNA, RNA, carbohydrate/lipid and N/P reserves
    (src/Individuals/Plankton/MacroMolecularMode/)."""

    def __repr__(self):
        return "MacroMolecularMode()"


class IronEnergyMode(AbstractMode):
    """Energy budget with N, P and Fe quotas, iron allocation to photosynthesis, nitrate reduction
    and nitrogen fixation (src/Individuals/Plankton/IronEnergyMode/)."""

    def __repr__(self):
        return "IronEnergyMode()"
