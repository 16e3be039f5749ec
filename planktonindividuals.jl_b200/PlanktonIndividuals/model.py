"""PlanktonModel, TimeStep! and PlanktonDiagnostics over libpib200 (src/Model/models.jl,
src/Model/time_step.jl, src/Diagnostics/diagnostics_struct.jl)."""
import numpy as np

from . import _abi, _lib
from ._abi import NTRACERS, PI_FP32, PI_FP64, tracer_names
from ._native import CModel
from .architectures import GPU, CarbonMode, MacroMolecularMode, QuotaMode
from .init import generate_tracers, initialize_plankton, initialize_plankton_carbon, initialize_plankton_macro
from .parameters import (bgc_params_default, default_tracer_init, phyt_params_default,
                         update_bgc_params, update_phyt_params)


class phyto_setup:
    """phyto_setup(params, N, Nsp) (src/PlanktonIndividuals.jl:109-113)."""

    def __init__(self, params=None, N=(2 ** 10,), Nsp=1):
        self.params = params
        self.N = list(N)
        self.Nsp = int(Nsp)


class _Attrs(dict):
    __getattr__ = dict.__getitem__


class phytoplankton:
    """phytoplankton{data, p} of one species; `data` is downloaded from the device on access."""

    def __init__(self, model, s, p):
        self._model, self._s, self.p = model, s, p

    @property
    def data(self):
        return _Attrs(self._model._native.get_individuals(self._s))


class individuals:
    def __init__(self, model, params, nsp):
        self.phytos = _Attrs({f"sp{s + 1}": phytoplankton(model, s, _Attrs(
            {k: (v[s] if hasattr(v, "__len__") else v) for k, v in params.items()})) for s in range(nsp)})
        self.abiotics = _Attrs()


class _Field:
    def __init__(self, model, n):
        self._model, self._n = model, n

    @property
    def data(self):
        return self._model._native.get_tracer(self._n)


class PlanktonModel:
    """PlanktonModel(arch, grid; FT, mode, max_individuals, bgc_params, tracer_initial, phyto,
    abiotic, t) (src/Model/models.jl:51-155). Individuals and tracers are initialised on the host
    with a seeded generator (`seed`), then copied to the GPU; the same seed keys the step's
    random draws."""

    def __init__(self, arch, grid, *, FT=np.float32, mode=None, max_individuals=8 * 1024,
                 bgc_params=None, tracer_initial=None, phyto=None, abiotic=None, t=0.0,
                 max_candidates=25, seed=0, initial_state=None):
        if not isinstance(arch, GPU) and arch is not GPU:
            raise ValueError("PlanktonModel: this implementation runs on GPU() only (no CPU fallback)")
        if mode is CarbonMode:
            mode = CarbonMode()
        if mode is MacroMolecularMode:
            mode = MacroMolecularMode()
        carbon = isinstance(mode, CarbonMode)
        macro = isinstance(mode, MacroMolecularMode)
        if mode is not None and not carbon and not macro and not isinstance(mode, QuotaMode) and mode is not QuotaMode:
            raise NotImplementedError(f"{mode}: QuotaMode(), CarbonMode() and MacroMolecularMode() are implemented")
        if abiotic is not None:
            raise NotImplementedError("abiotic particles are not implemented")
        FT = np.dtype(FT).type
        if FT not in (np.float32, np.float64):
            raise ValueError("FT must be Float32 or Float64")
        if carbon and FT is not np.float64:
            raise NotImplementedError("CarbonMode() is built in the FP64 form: use FT = Float64")
        if macro and FT is not np.float64:
            raise NotImplementedError("MacroMolecularMode() is built in the FP64 form: use FT = Float64")
        if getattr(grid, "is_latlon", False) and FT is not np.float64:
            raise NotImplementedError("LatLonGrid is built in the FP64 form: use FT = Float64")
        self.FT = FT
        self.arch = GPU()
        self.mode = mode if (carbon or macro) else QuotaMode()
        self.grid = grid
        self.max_candidates = max_candidates
        if bgc_params is None:
            bgc_final = update_bgc_params({}, FT)
        elif isinstance(bgc_params, dict):
            bgc_final = update_bgc_params(bgc_params, FT)
        else:
            raise ValueError("Phytoplankton parameters must be either Nothing or Dict!")
        pmode = self.mode
        if phyto is None:
            phyto = phyto_setup(update_phyt_params({}, FT, N=1, mode=pmode), [2 ** 10], 1)
        elif isinstance(phyto, phyto_setup):
            if max(phyto.N) > max_individuals:
                raise ValueError("maximum(phyto.N) ≤ max_individuals")
            if len(phyto.N) != phyto.Nsp:
                raise ValueError(f"PlanktonModel: `phyto`: The length of `N` must be {phyto.Nsp}, the same as "
                                 f"`Nsp`, each species has its own initial condition")
            if phyto.params is None:
                phyto.params = update_phyt_params({}, FT, N=phyto.Nsp, mode=pmode)
            elif isinstance(phyto.params, dict):
                phyto.params = update_phyt_params(phyto.params, FT, N=phyto.Nsp, mode=pmode)
            else:
                raise ValueError("Phytoplankton parameters must be either Nothing or Dict!")
        else:
            raise ValueError("PlanktonModel:`phyto` must be either Nothing or `phyto_setup`!")
        self.bgc_params = bgc_final
        self.phyto = phyto
        nsp = phyto.Nsp
        self.max_individuals = int(max_individuals)
        lib = _lib.load()
        precision = PI_FP64 if FT is np.float64 else PI_FP32
        self._native = CModel(lib, "pi_", grid, bgc_final, phyto.params, nsp, max_individuals,
                              seed, precision=precision, mode="carbon" if carbon else "macro" if macro else "quota")
        if initial_state is None:
            rng = np.random.default_rng(seed)
            init = initialize_plankton_carbon if carbon else initialize_plankton_macro if macro else initialize_plankton
            inds = [init(grid, phyto.params, s, phyto.N[s], max_individuals, rng) for s in range(nsp)]
            trs = generate_tracers(grid, tracer_initial or default_tracer_init(), rng)
        else:
            inds, trs = initial_state
        self._native.set_state(inds, trs)
        if t:
            self._native.set_time(0, float(t))
        self.individuals = individuals(self, phyto.params, nsp)
        self.tracers = _Attrs({name: _Field(self, n) for n, name in enumerate(tracer_names)})

    @property
    def t(self):
        return self._native.get_time()[1]

    @property
    def iteration(self):
        return self._native.get_time()[0]

    def count_active(self):
        """calc_active_individuals (models.jl:157-164)."""
        return [self._native.count_active(s) for s in range(self.phyto.Nsp)]

    def set_velocity(self, u, v, w):
        self._native.set_velocity(u, v, w)

    def set_PARF(self, parf):
        self._native.set_PARF(parf)

    def set_temp(self, temp):
        self._native.set_temp(temp)

    def __repr__(self):
        return (f"PlanktonModel:\n├── floating point data type: {np.dtype(self.FT).name}\n"
                f"├── grid: {self.grid!r}\n├── {self.mode!r} is selected for phytoplankton physiology\n"
                f"├── phytoplankton: {self.phyto.Nsp} species with {self.count_active()} individuals for each species\n"
                f"└── maximum number of individuals: {self.max_individuals} per species")


class PlanktonDiagnostics:
    """PlanktonDiagnostics(model; tracer, phytoplankton, iteration_interval)
    (diagnostics_struct.jl:23-105). The default diagnostics (PAR and num/graz/mort/dvid per
    species) and the requested ones — tracer fields (any of the 14 tracer names) and the mode's
    processes (QuotaMode: PS, BS, VDOC, VNH4, VNO3, VPO4, resp, exu, Bm, Cq, Nq, Pq, Chl; CarbonMode:
    PS, BS, RP, RS, TD, Bm, Bd, Chl; MacroMolecularMode: PS, VDOC, VNH4, VNO3, VPO4, resp, ρChl,
    S_PRO, S_DNA, S_RNA, exu, CH, NST, PST, PRO, DNA, RNA, Chl, of which VNH4 and exu stay zero as
    in the reference) — are accumulated on the device by every step; fields download on access."""

    DEFAULT = ("num", "graz", "mort", "dvid", "ptc")

    def __init__(self, model, tracer=(), phytoplankton=("num", "graz", "mort", "dvid", "ptc"),
                 abiotic_particle=("num",), iteration_interval=1):
        if not isinstance(tracer, tuple) or not isinstance(phytoplankton, tuple):
            raise ValueError("tracer and phytoplankton must be Tuples")
        # diag_avail (diagnostics_struct.jl:115-136): names available for the model's mode
        proc_names = (_abi.CARBON_PROC_NAMES if isinstance(model.mode, CarbonMode) else
                      _abi.MACRO_PROC_NAMES if isinstance(model.mode, MacroMolecularMode) else _abi.PROC_NAMES)
        for t in tracer:
            if t not in tracer_names and t != "PAR":
                raise ValueError(f"{t} is not one of the diagnostics")
        for p in phytoplankton:
            if p not in self.DEFAULT and p not in proc_names:
                raise ValueError(f"{p} is not one of the diagnostics")
        for a in abiotic_particle:
            if a != "num":
                raise ValueError(f"{a} is not one of the diagnostics")
        self._model = model
        self.iteration_interval = iteration_interval
        nat = model._native
        tmask = 0
        for t in tracer:
            if t in tracer_names:
                tmask |= 1 << tracer_names.index(t)
        pmask = 0
        for p in phytoplankton:
            if p in proc_names:
                pmask |= 1 << proc_names.index(p)
        nat.set_diags(tmask, pmask)
        G = model.grid.total_size
        procs = tuple(dict.fromkeys(tuple(phytoplankton) + self.DEFAULT))

        class _Sp:
            def __init__(self, s):
                self.s = s

            def keys(self):
                return procs

            def __getattr__(self, k):
                kinds = {"num": _abi.PI_DIAG_NUM, "graz": _abi.PI_DIAG_GRAZ,
                         "mort": _abi.PI_DIAG_MORT, "dvid": _abi.PI_DIAG_DVID}
                if k == "ptc":
                    return np.zeros(G, order="F")
                if k in kinds:
                    return nat.get_diag(kinds[k], self.s)
                if k in procs:
                    return nat.get_diag(_abi.PI_DIAG_PROC + proc_names.index(k), self.s)
                raise AttributeError(k)

            def __getitem__(self, k):
                return getattr(self, k)

        names = tuple(t for t in tracer if t in tracer_names) + ("PAR",)

        class _Tr:
            def keys(self):
                return names

            def __getattr__(self, k):
                if k == "PAR":
                    return nat.get_diag(_abi.PI_DIAG_PAR, 0)
                if k in names:
                    return nat.get_diag(_abi.PI_DIAG_TRACER + tracer_names.index(k), 0)
                raise AttributeError(k)

            def __getitem__(self, k):
                return getattr(self, k)

        self.tracer = _Tr()
        self.phytos = _Attrs({f"sp{s + 1}": _Sp(s) for s in range(model.phyto.Nsp)})
        self.abiotics = _Attrs()

    def reset(self):
        r = self._model._native.lib.pi_reset_diags(self._model._native.h)
        if r:
            raise RuntimeError("pi_reset_diags failed")


def TimeStep_b(model, ΔT, diags=None):
    """TimeStep!(model, ΔT, diags) (src/Model/time_step.jl:12-180)."""
    model._native.time_step(float(ΔT))
