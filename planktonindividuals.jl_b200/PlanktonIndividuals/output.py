"""PlanktonOutputWriter and write_output! (src/Output/output_writers.jl, src/Output/write_outputs.jl).

The reference writes JLD2 (HDF5) files; this image has no HDF5 library, so each file is a NumPy
archive (.npz: a zip of .npy arrays, readable from Julia with NPZ.jl) holding the same datasets
under the same paths — `timeseries/t/<iteration>`, `timeseries/<species>/<attribute>/<iteration>`
for individuals, `timeseries/<tracer>/<iteration>` and
`timeseries/phyto/<species>/<process>/<iteration>` for diagnostics (interior fields averaged over
the diagnostics interval, which are then cleared). Archives are appended to after every write,
roll over to `_part1`, `_part2`, ... files past `max_filesize`, and species logs
(`dynamic_species001.txt`, ...) get one line per step in the reference's QuotaMode format.
"""
import io
import math
import os
import re
import shutil
import zipfile

import numpy as np

from . import _abi


class PlanktonOutputWriter:
    """PlanktonOutputWriter(; dir, diags_prefix, phytoplankton_prefix, abiotic_particle_prefix,
    write_log, save_diags, save_phytoplankton, save_abiotic_particle, phytoplankton_include,
    abiotic_particle_include, phytoplankton_iteration_interval, abiotic_particle_iteration_interval,
    max_filesize) (output_writers.jl:54-92). As in the reference, an existing `dir` is removed and
    created again."""

    def __init__(self, dir="./results", diags_prefix="diags", phytoplankton_prefix="phytoplankton",
                 abiotic_particle_prefix="abiotic_particle", write_log=False, save_diags=False,
                 save_phytoplankton=False, save_abiotic_particle=False, phytoplankton_include=("x", "y", "z"),
                 abiotic_particle_include=("x", "y", "z"), phytoplankton_iteration_interval=1,
                 abiotic_particle_iteration_interval=1, max_filesize=math.inf):
        if os.path.isdir(dir):
            shutil.rmtree(dir)
        os.mkdir(dir)
        self.filepath = dir
        self.write_log = write_log
        self.save_diags = save_diags
        self.save_phytoplankton = save_phytoplankton
        self.save_abiotic_particle = save_abiotic_particle
        self.diags_file = os.path.join(dir, diags_prefix + ".npz") if save_diags else ""
        self.phytoplankton_file = os.path.join(dir, phytoplankton_prefix + ".npz") if save_phytoplankton else ""
        self.abiotic_particle_file = os.path.join(dir, abiotic_particle_prefix + ".npz") if save_abiotic_particle else ""
        self.phytoplankton_include = tuple(phytoplankton_include)
        self.phytoplankton_iteration_interval = int(phytoplankton_iteration_interval)
        self.abiotic_particle_include = tuple(abiotic_particle_include)
        self.abiotic_particle_iteration_interval = int(abiotic_particle_iteration_interval)
        self.max_filesize = max_filesize
        self.part_diags = self.part_phytoplankton = self.part_abiotic_particle = 1

    def __repr__(self):
        return (f"PlanktonOutputWriter:\n├── files are saved at {self.filepath}\n"
                f"├── {'diagnostics are saved as ' + self.diags_file if self.save_diags else 'diagnostics are not saved'}\n"
                f"├── {'phytoplankton is saved as ' + self.phytoplankton_file if self.save_phytoplankton else 'phytoplankton are not saved'}\n"
                f"├── write log: {str(self.write_log).lower()}\n"
                f"└── Maximum file size: {humanize_filesize(self.max_filesize)}")


def humanize_filesize(s):
    """humanize_filesize (output_writers.jl:130-143)."""
    suffix = ["B", "KiB", "MiB", "GiB", "TiB", "PiB", "EiB", "ZiB", "YiB"]
    value, unit, big = s, 1024.0, suffix[0]
    for power in range(1, len(suffix) + 1):
        unit = 1024.0 ** power
        big = suffix[power - 1]
        if value < unit:
            break
    return "%3.1f %s" % (1024 * value / unit, big)


def _filesize(path):
    return os.path.getsize(path) if os.path.exists(path) else 0


def _next_part(path, part):
    """start_next_*_file (write_outputs.jl:43-75): the first rollover renames the file to _part1."""
    if part == 1:
        p1 = re.sub(r"\.npz$", "_part1.npz", path)
        if os.path.exists(path):
            os.replace(path, p1)
        path = p1
    part += 1
    return re.sub(r"part\d+\.npz$", f"part{part}.npz", path), part


def _append(path, items):
    """Appends arrays to the archive (jldopen(path, "a+")): name → value."""
    with zipfile.ZipFile(path, "a", compression=zipfile.ZIP_STORED) as z:
        for name, value in items:
            buf = io.BytesIO()
            np.lib.format.write_array(buf, np.asarray(value), allow_pickle=False)
            z.writestr(name + ".npy", buf.getvalue())


def read_archive(path):
    """All datasets of an output archive: {dataset path: array}."""
    out = {}
    with zipfile.ZipFile(path) as z:
        for name in z.namelist():
            with z.open(name) as f:
                out[name[:-4] if name.endswith(".npy") else name] = np.lib.format.read_array(f, allow_pickle=False)
    return out


def _interior(a, g):
    return np.asarray(a)[g.Hx:g.Hx + g.Nx, g.Hy:g.Hy + g.Ny, g.Hz:g.Hz + g.Nz]


def write_individuals(phytos, path, t, it, atts):
    """write_individuals_to_jld2 (write_outputs.jl:159-169)."""
    items = [(f"timeseries/t/{it}", np.float64(t))]
    for sp in phytos.keys():
        data = phytos[sp].data
        for att in atts:
            items.append((f"timeseries/{sp}/{att}/{it}", np.asarray(data[att])))
    _append(path, items)


def write_diags(diags, path, t, it, ncounts, grid):
    """write_diags_to_jld2 (write_outputs.jl:171-202): interior fields over the interval, then the
    diagnostics start again from zero."""
    items = [(f"timeseries/t/{it}", np.float64(t))]
    for key in diags.tracer.keys():
        items.append((f"timeseries/{key}/{it}", _interior(diags.tracer[key], grid) / ncounts))
    for sp in diags.phytos.keys():
        for proc in diags.phytos[sp].keys():
            items.append((f"timeseries/phyto/{sp}/{proc}/{it}", _interior(diags.phytos[sp][proc], grid) / ncounts))
    abiotics = getattr(diags, "abiotics", {})
    for sa in abiotics.keys():
        for proc in abiotics[sa].keys():
            items.append((f"timeseries/abiotic/{sa}/{proc}/{it}", _interior(abiotics[sa][proc], grid) / ncounts))
    _append(path, items)
    diags.reset()


def write_species_dynamics(t, phytos, filepath, carbon=False):
    """write_species_dynamics for QuotaMode (write_outputs.jl:98-117) or CarbonMode (:142-157): one
    line per species file."""
    for i, sp in enumerate(phytos.keys(), start=1):
        d = phytos[sp].data
        ac = np.asarray(d["ac"], dtype=bool)
        pop = int(ac.sum())
        keys = ("gen", "age", "Sz", "Bm") if carbon else ("gen", "age", "Sz", "Bm", "Cq", "Nq", "Pq", "Chl")
        ave = {k: (float(np.sum(np.asarray(d[k])[ac])) / pop if pop else float("nan")) for k in keys}
        day, hour = t // 86400, (t % 86400) / 3600
        with open(os.path.join(filepath, "dynamic_species%03d.txt" % i), "a") as f:
            if carbon:
                f.write("%3.0f  %2.2f  %6.0f  %1.2f  %1.2f  %1.2f  %.8E\n" %
                        (day, hour, pop, ave["gen"], ave["age"], ave["Sz"], ave["Bm"]))
            else:
                f.write("%3.0f  %2.2f  %6.0f  %1.2f  %1.2f  %1.2f  %.8E  %.8E  %.8E  %.8E  %.8E\n" %
                        (day, hour, pop, ave["gen"], ave["age"], ave["Sz"], ave["Bm"], ave["Cq"], ave["Nq"],
                         ave["Pq"], ave["Chl"]))


def write_output_b(writer, model, diags):
    """write_output!(writer, model, diags) (write_outputs.jl:2-41)."""
    if writer is None:
        return
    t, it = model.t, model.iteration
    phytos = model.individuals.phytos
    if writer.write_log:
        from .architectures import CarbonMode, IronEnergyMode, MacroMolecularMode
        if isinstance(getattr(model, "mode", None), IronEnergyMode):
            # write_species_dynamics for IronEnergyMode (write_outputs.jl:118-141) reads data.En,
            # which IronEnergyMode individuals do not have (their field is exEn)
            raise ValueError("type has no field En: write_species_dynamics fails for IronEnergyMode (use write_log = false)")
        if isinstance(getattr(model, "mode", None), MacroMolecularMode):
            # the reference defines write_species_dynamics for QuotaMode, IronEnergyMode and
            # CarbonMode only (write_outputs.jl:98-157)
            raise ValueError("write_species_dynamics has no method for MacroMolecularMode (use write_log = false)")
        write_species_dynamics(t, phytos, writer.filepath, carbon=isinstance(getattr(model, "mode", None), CarbonMode))
    if writer.save_diags and it % diags.iteration_interval == 0:
        if _filesize(writer.diags_file) >= writer.max_filesize:
            writer.diags_file, writer.part_diags = _next_part(writer.diags_file, writer.part_diags)
        write_diags(diags, writer.diags_file, t, it, diags.iteration_interval, model.grid)
    if writer.save_phytoplankton and it % writer.phytoplankton_iteration_interval == 0:
        if _filesize(writer.phytoplankton_file) >= writer.max_filesize:
            writer.phytoplankton_file, writer.part_phytoplankton = _next_part(writer.phytoplankton_file,
                                                                              writer.part_phytoplankton)
        write_individuals(phytos, writer.phytoplankton_file, t, it, writer.phytoplankton_include)
    if writer.save_abiotic_particle and it % writer.abiotic_particle_iteration_interval == 0:
        if _filesize(writer.abiotic_particle_file) >= writer.max_filesize:
            writer.abiotic_particle_file, writer.part_abiotic_particle = _next_part(writer.abiotic_particle_file,
                                                                                    writer.part_abiotic_particle)
        write_individuals(model.individuals.abiotics, writer.abiotic_particle_file, t, it,
                          writer.abiotic_particle_include)
