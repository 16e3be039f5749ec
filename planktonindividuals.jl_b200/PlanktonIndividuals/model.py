"""PlanktonModel, TimeStep! and PlanktonDiagnostics over libpib200 (src/Model/models.jl,
src/Model/time_step.jl, src/Diagnostics/diagnostics_struct.jl)."""
import numpy as np

from . import _abi, _lib
from ._abi import NTRACERS, PI_FP32, PI_FP64, tracer_names
from ._native import CModel
from .architectures import GPU, CarbonMode, IronEnergyMode, MacroMolecularMode, QuotaMode
from .init import (generate_tracers, initialize_abiotic_particle, initialize_plankton, initialize_plankton_carbon,
                   initialize_plankton_iron, initialize_plankton_macro)
from .parameters import (abiotic_params_default, bgc_params_default, default_tracer_init, phyt_params_default,
                         update_abiotic_params, update_bgc_params, update_phyt_params)


class phyto_setup:
    """phyto_setup(params, N, Nsp) (src/PlanktonIndividuals.jl:109-113)."""

    def __init__(self, params=None, N=(2 ** 10,), Nsp=1):
        self.params = params
        self.N = list(N)
        self.Nsp = int(Nsp)


class Palat:
    """Palat(intac, release) (src/PlanktonIndividuals.jl:118-121): the (phytoplankton, abiotic)
    species name pairs that interact (particle_interaction!) and release (particle_release!), e.g.
    Palat([("sp1", "sa1")], [("sp1", "sa1")])."""

    def __init__(self, intac=(), release=()):
        self.intac = [tuple(p) for p in intac]
        self.release = [tuple(p) for p in release]


class abiotic_setup:
    """abiotic_setup(params, N, Nsa, palat) (src/PlanktonIndividuals.jl:122-127)."""

    def __init__(self, params=None, N=(2 ** 10,), Nsa=1, palat=None):
        self.params = params
        self.N = list(N)
        self.Nsa = int(Nsa)
        self.palat = palat if palat is not None else Palat()


class _Attrs(dict):
    __getattr__ = dict.__getitem__


class phytoplankton:
    """phytoplankton{data, p} of one species; `data` is downloaded from the device on access."""

    def __init__(self, model, s, p):
        self._model, self._s, self.p = model, s, p

    @property
    def data(self):
        return _Attrs(self._model._native.get_individuals(self._s))


class abiotic_particle:
    """abiotic_particle{data, p, bc} of one abiotic species (src/PlanktonIndividuals.jl:100-105);
    `data` (x, y, z, xi, yi, zi, ac) is downloaded from the device on access."""

    def __init__(self, model, a, p):
        self._model, self._a, self.p = model, a, p

    @property
    def data(self):
        return _Attrs(self._model._native.get_abiotic_particles(self._a))


class individuals:
    def __init__(self, model, params, nsp, abiotic_params=None, nsa=0):
        self.phytos = _Attrs({f"sp{s + 1}": phytoplankton(model, s, _Attrs(
            {k: (v[s] if hasattr(v, "__len__") else v) for k, v in params.items()})) for s in range(nsp)})
        self.abiotics = _Attrs({f"sa{a + 1}": abiotic_particle(model, a, _Attrs(
            {k: v[a] for k, v in abiotic_params.items()})) for a in range(nsa)})


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
        if mode is IronEnergyMode:
            mode = IronEnergyMode()
        carbon = isinstance(mode, CarbonMode)
        macro = isinstance(mode, MacroMolecularMode)
        iron = isinstance(mode, IronEnergyMode)
        if mode is not None and not (carbon or macro or iron) and not isinstance(mode, QuotaMode) and mode is not QuotaMode:
            raise NotImplementedError(f"{mode}: QuotaMode(), CarbonMode(), MacroMolecularMode() and IronEnergyMode() "
                                      f"are implemented")
        FT = np.dtype(FT).type
        if FT not in (np.float32, np.float64):
            raise ValueError("FT must be Float32 or Float64")
        if carbon and FT is not np.float64:
            raise NotImplementedError("CarbonMode() is built in the FP64 form: use FT = Float64")
        if macro and FT is not np.float64:
            raise NotImplementedError("MacroMolecularMode() is built in the FP64 form: use FT = Float64")
        if iron and FT is not np.float64:
            raise NotImplementedError("IronEnergyMode() is built in the FP64 form: use FT = Float64")
        if getattr(grid, "is_latlon", False) and FT is not np.float64:
            raise NotImplementedError("LatLonGrid is built in the FP64 form: use FT = Float64")
        if abiotic is not None:                                  # models.jl:99-117
            if not isinstance(abiotic, abiotic_setup):
                raise ValueError("PlanktonModel:`abiotic` must be either Nothing or `abiotic_setup`!")
            if FT is not np.float64:
                raise NotImplementedError("abiotic particles are built in the FP64 form: use FT = Float64")
            if max(abiotic.N) > max_individuals:
                raise ValueError("maximum(abiotic.N) ≤ max_individuals")
            if len(abiotic.N) != abiotic.Nsa:
                raise ValueError(f"PlanktonModel: `abiotic`: The length of `N` must be {abiotic.Nsa}, the same as "
                                 f"`Nsa`, each species has its own initial condition")
            if abiotic.params is None:
                abiotic.params = update_abiotic_params(abiotic_params_default(abiotic.Nsa), FT, N=abiotic.Nsa)
            elif isinstance(abiotic.params, dict):
                abiotic.params = update_abiotic_params(abiotic.params, FT, N=abiotic.Nsa)
            else:
                raise ValueError("Abiotic parameters must be either Nothing or Dict!")
        self.FT = FT
        self.arch = GPU()
        self.mode = mode if (carbon or macro or iron) else QuotaMode()
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
        self.abiotic = abiotic
        nsp = phyto.Nsp
        pal_intac, pal_release = [], []
        if abiotic is not None:                                  # models.jl:121-143
            sps = [f"sp{s + 1}" for s in range(nsp)]
            sas = [f"sa{a + 1}" for a in range(abiotic.Nsa)]
            for lst, out in ((abiotic.palat.intac, pal_intac), (abiotic.palat.release, pal_release)):
                for pr in lst:
                    sp, sa = (str(q).lstrip(":") for q in pr)
                    if sp not in sps:
                        raise ValueError(f"Abiotic: {sp} is not generated")
                    if sa not in sas:
                        raise ValueError(f"Abiotic: {sa} is not generated")
                    out.append((sps.index(sp), sas.index(sa)))
        self.max_individuals = int(max_individuals)
        lib = _lib.load()
        precision = PI_FP64 if FT is np.float64 else PI_FP32
        self._native = CModel(lib, "pi_", grid, bgc_final, phyto.params, nsp, max_individuals,
                              seed, precision=precision,
                              mode="carbon" if carbon else "macro" if macro else "iron" if iron else "quota")
        if initial_state is None:
            rng = np.random.default_rng(seed)
            init = (initialize_plankton_carbon if carbon else initialize_plankton_macro if macro else
                    initialize_plankton_iron if iron else initialize_plankton)
            inds = [init(grid, phyto.params, s, phyto.N[s], max_individuals, rng) for s in range(nsp)]
            trs = generate_tracers(grid, tracer_initial or default_tracer_init(), rng)
        else:
            inds, trs = initial_state
        self._native.set_state(inds, trs)
        nsa = 0
        if abiotic is not None:
            nsa = abiotic.Nsa
            # max_ptc exists only where the mode's parameters define it (IronEnergyMode); NaN
            # otherwise, where a merge raises as the reference's field access does
            mp = phyto.params.get("max_ptc")
            max_ptc = [float(mp[s]) for s in range(nsp)] if mp is not None else [float("nan")] * nsp
            self._native.set_abiotics(abiotic.params, nsa, pal_intac, pal_release, max_candidates, max_ptc)
            if initial_state is None:
                for a in range(nsa):
                    self._native.set_abiotic_particles(a, initialize_abiotic_particle(grid, abiotic.N[a],
                                                                                      max_individuals, rng))
        if t:
            self._native.set_time(0, float(t))
        self.individuals = individuals(self, phyto.params, nsp, abiotic.params if abiotic else None, nsa)
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

    def count_abiotic(self):
        """calc_active_individuals of the abiotic species (models.jl:170-176)."""
        return [self._native.count_abiotic(a) for a in range(self._native.nsa)]

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
                      _abi.MACRO_PROC_NAMES if isinstance(model.mode, MacroMolecularMode) else
                      _abi.IRON_PROC_NAMES if isinstance(model.mode, IronEnergyMode) else _abi.PROC_NAMES)
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
                if k == "ptc":                   # time_step.jl:140-149: kept only with abiotic particles
                    if not nat.nsa:
                        return np.zeros(G, order="F")
                    return nat.get_diag(_abi.PI_DIAG_PTC, self.s)
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
        anames = tuple(abiotic_particle)

        class _Sa:
            def __init__(self, a):
                self.a = a

            def keys(self):
                return anames

            def __getattr__(self, k):
                if k == "num":
                    return nat.get_diag(_abi.PI_DIAG_ABIO_NUM, self.a)
                raise AttributeError(k)

            def __getitem__(self, k):
                return getattr(self, k)

        self.abiotics = _Attrs({f"sa{a + 1}": _Sa(a) for a in range(nat.nsa)})

    def reset(self):
        r = self._model._native.lib.pi_reset_diags(self._model._native.h)
        if r:
            raise RuntimeError("pi_reset_diags failed")


def _bc_kind(model, pos, bc_value):
    if pos not in _abi.FACES:
        raise ValueError(f"pos must be one of {tuple(_abi.FACES)}")
    if np.ndim(bc_value) == 0:
        return _abi.FACES[pos], _abi.PI_BC_CONST, [float(bc_value)], 0
    a = np.asfortranarray(np.asarray(bc_value, dtype=np.float64))
    if a.ndim == 2:
        return _abi.FACES[pos], _abi.PI_BC_ARRAY2D, a, 0
    if a.ndim == 3:
        return _abi.FACES[pos], _abi.PI_BC_ARRAY3D, a, a.shape[2]
    raise ValueError("bc_value must be a Number, a 2D or a 3D array")


def set_bc_b(model, *, tracer, pos, bc_value):
    """set_bc!(model; tracer, pos, bc_value) (src/Biogeochemistry/HaloRegions/boundary_conditions.jl:21-31):
    a constant, a face array (n1, n2) or a time series (n1, n2, nt) indexed by model.iteration."""
    tracer = str(tracer).lstrip(":")
    if tracer not in tracer_names:
        raise ValueError(f"{tracer} is not a tracer")
    face, kind, v, nt = _bc_kind(model, str(pos).lstrip(":"), bc_value)
    model._native.set_flux_bc(tracer_names.index(tracer), face, kind, v, nt)


def set_bc_particle_b(model, *, sa, pos, bc_value):
    """set_bc_particle!(model; sa, pos, bc_value) (boundary_conditions.jl:33-41): the particle flux
    of abiotic species `sa` through a face, turned into particles by particles_from_bcs!."""
    sa = str(sa).lstrip(":")
    if sa not in model.individuals.abiotics:
        raise ValueError(f"Abiotic: {sa} is not generated")
    face, kind, v, nt = _bc_kind(model, str(pos).lstrip(":"), bc_value)
    model._native.set_abiotic_bc(int(sa[2:]) - 1, face, kind, v, nt)


def TimeStep_b(model, ΔT, diags=None):
    """TimeStep!(model, ΔT, diags) (src/Model/time_step.jl:12-180)."""
    model._native.time_step(float(ΔT))
