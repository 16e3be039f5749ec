"""Output writers (src/Output/output_writers.jl, write_outputs.jl) on the CPU, driven by the oracle
model through the same interface as a GPU model: archives hold the individuals and the
interval-averaged interior diagnostics under the reference's dataset paths at every write, roll
over to _part1/_part2 files past max_filesize, and species logs follow the QuotaMode format."""
import os

import numpy as np

import oracle
from PlanktonIndividuals import _abi, workloads as W
from PlanktonIndividuals.output import PlanktonOutputWriter, read_archive, write_output_b
from helpers import VelCache, drive


class _Data:
    def __init__(self, ref, s):
        self.ref, self.s = ref, s

    @property
    def data(self):
        return self.ref.get_individuals(self.s)


class _Phytos(dict):
    pass


class _Model:
    """The attributes write_output! reads, from an oracle model."""

    def __init__(self, ref, wl):
        self.ref, self.grid = ref, wl.grid
        self.individuals = type("I", (), {})()
        self.individuals.phytos = _Phytos({f"sp{s + 1}": _Data(ref, s) for s in range(wl.nsp)})
        self.individuals.abiotics = _Phytos()

    @property
    def t(self):
        return self.ref.get_time()[1]

    @property
    def iteration(self):
        return self.ref.get_time()[0]


class _Diags:
    """PAR and num diagnostics of an oracle model, cleared by reset()."""

    def __init__(self, ref, nsp, interval):
        self.ref, self.iteration_interval = ref, interval
        self.base = {}
        self.reset()
        outer = self

        class Tr:
            def keys(self):
                return ("PAR",)

            def __getitem__(self, k):
                return outer.ref.get_diag(_abi.PI_DIAG_PAR, 0) - outer.base[("PAR", 0)]

        class Sp:
            def __init__(self, s):
                self.s = s

            def keys(self):
                return ("num",)

            def __getitem__(self, k):
                return outer.ref.get_diag(_abi.PI_DIAG_NUM, self.s) - outer.base[("num", self.s)]

        self.tracer = Tr()
        self.phytos = {f"sp{s + 1}": Sp(s) for s in range(nsp)}

    def reset(self):
        self.base[("PAR", 0)] = self.ref.get_diag(_abi.PI_DIAG_PAR, 0)
        for s in range(2):
            try:
                self.base[("num", s)] = self.ref.get_diag(_abi.PI_DIAG_NUM, s)
            except Exception:
                pass


def test_writer_archives_logs_and_rollover(tmp_path):
    wl = W.config2(nx=8, nz=4, N_per_species=200, nsp=2, steps=6, nmodes=8, seed=91)
    wl.parf = np.asfortranarray(np.roll(wl.parf, -10, axis=2))
    ref = oracle.from_workload(wl)
    model, diags = _Model(ref, wl), _Diags(ref, 2, 2)
    out = str(tmp_path / "results")
    w = PlanktonOutputWriter(dir=out, write_log=True, save_diags=True, save_phytoplankton=True,
                             phytoplankton_include=("x", "Bm", "ac"), max_filesize=40_000)
    vel = VelCache(wl)
    snaps = {}
    for step in range(6):
        drive(ref, wl, 1, vel)
        snaps[step + 1] = [ref.get_individuals(s) for s in range(2)]
        write_output_b(w, model, diags)
    files = sorted(os.listdir(out))
    assert "dynamic_species001.txt" in files and "dynamic_species002.txt" in files
    parts = sorted(f for f in files if f.startswith("phytoplankton_part"))
    assert len(parts) >= 2 and "phytoplankton.npz" not in files       # rolled over
    got = {}
    for f in parts:
        got.update(read_archive(os.path.join(out, f)))
    for it in range(1, 7):
        assert got[f"timeseries/t/{it}"] == it * wl.dT
        for s in range(2):
            for att in ("x", "Bm", "ac"):
                assert np.array_equal(got[f"timeseries/sp{s + 1}/{att}/{it}"], snaps[it][s][att])
    dg = {}
    for f in files:
        if f.startswith("diags"):
            dg.update(read_archive(os.path.join(out, f)))
    assert sorted(k for k in dg if k.startswith("timeseries/t/")) == ["timeseries/t/2", "timeseries/t/4", "timeseries/t/6"]
    g = wl.grid
    pop = dg["timeseries/phyto/sp1/num/2"]
    assert pop.shape == (g.Nx, g.Ny, g.Nz)
    assert abs(pop.sum() - (len(np.nonzero(snaps[1][0]["ac"])[0]) + len(np.nonzero(snaps[2][0]["ac"])[0])) / 2) < 1e-9
    lines = open(os.path.join(out, "dynamic_species001.txt")).read().splitlines()
    assert len(lines) == 6
    f = lines[-1].split()
    assert len(f) == 11 and int(float(f[2])) == int(snaps[6][0]["ac"].sum())
    assert "E" in f[6] and abs(float(f[6]) - snaps[6][0]["Bm"][snaps[6][0]["ac"]].mean()) <= 1e-8 * abs(float(f[6]))
