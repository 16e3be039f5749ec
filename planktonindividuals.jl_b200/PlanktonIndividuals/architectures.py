"""Architectures and physiology modes (src/Architectures.jl, src/PlanktonIndividuals.jl:59-83).
Only GPU() and QuotaMode() are implemented; the others exist so that code naming them fails
with a clear message."""


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
    pass


class MacroMolecularMode(AbstractMode):
    pass


class IronEnergyMode(AbstractMode):
    pass
