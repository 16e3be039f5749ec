#!/usr/bin/env python
"""Throughput of the PlanktonIndividuals model time step on B200: FP32 batched form vs FP64 plain.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload config2|config3|config4|config5]

Default workload: config 2 — 256×256×64 grid (50 m × 50 m × 2 m), 2 species × 2,097,152
individuals seeded in the top 40 m, divergence-free random-Fourier velocity refreshed every 60
steps, dt = 30 s (seeded synthetic inputs). A step is one TimeStep! of the whole model. The headline
`value` is individual-steps/s (active individuals × steps ÷ device time) of the FP32 batched form
(the batch engine with its CUDA graph and autotuned launch shapes; config 2 is a batch of one
member) with every input resident in HBM; `fp64` gives the plain FP64 form on the same workload
in the same run, and `cell_steps_per_s` the tracer cell-steps/s. `e2e` is the FP32 form through
the C-ABI (pi_create(PI_FP32) + pi_set_velocity/PARF/temp + pi_time_step + pi_count_active) with
host buffers: each step uploads its forcing snapshot from pinned host memory and reads back the
population counts.

--workload config3 runs the mixed-precision case at scale (512×512×128, 4 species × 16,777,216
individuals with their own size distributions, dt = 20 s) the same way as config 2.
--workload config4 / config5 run the batched ensembles (64 uneven 3D members; 4096 0D boxes) in
the FP32 batched form; the members are split across ranks (scaling "strong").

`step_roofline` relates the whole step to HBM bandwidth with per-unit bytes of the FP32 form:
106 B per active individual (read and write of its persistent state) and 308 B per interior cell
(14 tracers read and written, velocities, temperature, PAR, fixed-point sums).

Multi-GPU (config 2): the model domain is not partitioned; each rank runs an independent replica
(scaling "weak") and `value` sums the replicas' individual-steps over the slowest rank's time.

--accuracy reports each output's error of the FP32 batched form against the FP64 form, which the
GPU parity tests show to be bit-identical to the CPU oracle: config 2 over --acc-steps steps
(population counts every 100 steps, active-slot and cell mismatches, quota and position errors,
interior tracer-mass errors), the same for config 3 with --workload config3, or, with --workload
config5, --acc-boxes boxes over 2880 steps, or with --workload config4 the first --acc-boxes
ensemble members over 500 steps (per-member counts and tracer-mass errors).

--impl reference times the reference algorithm's CPU implementation: the reference is Julia
(absent here), so this is the CPU oracle (a Float64 restatement of TimeStep!) with all host
threads, on a bounded sample of the same workload (a 128×128×64 sub-domain with the same
individual density).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "planktonindividuals.jl_b200"))

import numpy as np  # noqa: E402

from PlanktonIndividuals.accuracy import (fp32_batch, fp32_vs_fp64, fp64_sim,  # noqa: E402,F401
                                          interior_mass, mass_rel, series_arrays, snapshots)

METRIC = "individual-steps/s (FP32 batched form; FP64 plain form reported beside)"
SORT_INTERVAL = 32      # steps between the counting sorts that keep individuals grouped by cell
UNIT = "ind-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="config2", choices=["config2", "config3", "config4", "config5"])
    ap.add_argument("--fp64-steps", type=int, default=50)
    ap.add_argument("--e2e-steps", type=int, default=30)
    ap.add_argument("--profile-steps", type=int, default=5)
    ap.add_argument("--tune-steps", type=int, default=2)
    ap.add_argument("--cpu-steps", type=int, default=16)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--nx", type=int, default=None, help="config 2/3 horizontal size (smaller for profiling); "
                    "default 256 (config 2), 512 (config 3)")
    ap.add_argument("--nz", type=int, default=None, help="default 64 (config 2), 128 (config 3)")
    ap.add_argument("--n-per-species", type=int, default=None, help="default 2,097,152 (config 2), 16,777,216 (config 3)")
    ap.add_argument("--accuracy", action="store_true",
                    help="report the FP32 form's errors against the FP64 form (bit-exact to the CPU oracle)")
    ap.add_argument("--acc-steps", type=int, default=1000)
    ap.add_argument("--acc-boxes", type=int, default=16)
    return ap.parse_args()


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "20"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        # start timing only once the sampler is producing rows
        t0 = time.time()
        while self.p is not None and time.time() - t0 < 5.0:
            self.f.flush()
            if os.path.getsize(self.f.name) > 0:
                break
            time.sleep(0.05)

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except (ValueError, IndexError):
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ------------------------------------------------------------------------------------------
# algorithmic bytes per launch (the minimum each kernel must move)
# ------------------------------------------------------------------------------------------

def algorithmic_bytes(name, members, n_active_total, n_slots_total):
    V = sum(w.grid.Nx * w.grid.Ny * w.grid.Nz for w in members)
    inactive = n_slots_total - n_active_total
    if name == "k32_ztail":
        # tracer_temp, tracer read; new tracer written (14 each); w and pop per cell
        return V * (3 * 14 * 4 + 4 + 4)
    if name == "k32_xy":
        # tracer read, tracer_temp written (14 each); u and v per cell
        return V * (2 * 14 * 4 + 8)
    if name == "k32_move":
        # active: cell, 3 offsets, flags, stat, Chl read; cell, offsets, flags, stat written;
        # pop (4) and Chl (8) sums; inactive slots: flags and cell read; the velocity field
        # (u, v, w: 12 bytes per cell) read once
        return n_active_total * (4 + 12 + 1 + 1 + 4 + 4 + 12 + 1 + 1 + 4 + 8) + inactive * 5 + V * 12
    if name == "k32_physiology":
        # flags, stat, cell, Bm..age read; Bm..age, flags written; 7 gathers; 5 consumption sums
        return n_active_total * (1 + 1 + 4 + 24 + 24 + 1 + 7 * 4 + 5 * 8) + inactive * 1
    # FP64 plain form (k_* kernels)
    if name == "k_particles_sorted":
        return n_active_total * (4 + 1 + 1 + 4 + 24 + 24 + 4 + 4 + 8)
    if name in ("k_sweep_y", "k_sweep_z"):
        return V * (14 * 8 * 3 + 8)
    return None


B_IND_FP32, B_CELL_FP32 = 106, 308      # algorithmic bytes per active individual / interior cell


def step_roofline(n_ind, n_cells, ms_per_step):
    hbm, kind = measured_peaks()
    byts = n_ind * B_IND_FP32 + n_cells * B_CELL_FP32
    ach = byts / (ms_per_step / 1e3) / 1e9
    return {"bytes_per_step": int(byts), "achieved": round(ach, 1), "peak": hbm, "peak_source": kind,
            "unit": "GB/s", "frac": round(ach / hbm, 4)}


def gpu_launches(prof, P, K, workload):
    """Own kernels launched in K timed steps, from the kernels one profiled step launched: one per
    profiled scope, except the halo fill (three passes in the 0D boxes, whose N < H) and the
    storage-order sort (count, three scan passes, scatter; once per SORT_INTERVAL steps), plus
    k32_copy_if_err and k32_end_step in every step."""
    per_step = 2
    for name, (n, _) in prof.items():
        if name == "k32_sort":
            continue
        per_step += (3 if (name == "k32_halo" and workload == "config5") else 1) * n // P
    return K * per_step + 5 * (-(-K // SORT_INTERVAL))


# DRAM traffic per launch measured with ncu (dram__bytes_read.sum + dram__bytes_write.sum, one pass,
# --clock-control none) on config 2 (256x256x64, 2 x 2,097,152 individuals), per interior cell or per
# active individual; a launch's traffic is this figure times its units
MEASURED_TRAFFIC = {"k32_xy": ("cell", 113.0), "k32_ztail": ("cell", 214.4),
                    "k32_move": ("active", 78.0), "k32_physiology": ("active", 123.8)}


def profile_roofline(prof, members, nact, nslots):
    tot_ms = sum(v[1] for v in prof.values())
    order = sorted(prof, key=lambda k: -prof[k][1])
    hbm, peak_kind = measured_peaks()
    roof = None
    for dom in order:
        byts = algorithmic_bytes(dom, members, nact, nslots)
        if byts:
            per_launch_ms = prof[dom][1] / prof[dom][0]
            ach = byts / (per_launch_ms / 1e3) / 1e9
            traffic = None
            if dom in MEASURED_TRAFFIC:
                unit, per = MEASURED_TRAFFIC[dom]
                V = sum(w.grid.Nx * w.grid.Ny * w.grid.Nz for w in members)
                traffic = int(per * (V if unit == "cell" else nact))
            roof = {"kernel": dom, "bound": "hbm", "achieved": round(ach, 1), "peak": hbm,
                    "peak_source": peak_kind, "unit": "GB/s", "frac": round(ach / hbm, 4),
                    "traffic": traffic, "algorithmic_bytes_per_launch": int(byts),
                    "avg_launch_ms": round(per_launch_ms, 4),
                    "traffic_source": "ncu dram bytes per " + MEASURED_TRAFFIC[dom][0] + " on config 2, times this launch's units"
                    if traffic else None}
            break
    return roof, tot_ms


def run_fp32(members, args, dist, local, clocks_cls):
    import torch
    from PlanktonIndividuals.batch import Member, PlanktonBatch
    K, Wm = args.steps, args.warmup
    nsp = members[0].nsp
    dT = members[0].dT
    b = PlanktonBatch([Member(w.grid, w.bgc, w.phyt, w.capacity, w.seed) for w in members], nspecies=nsp)
    total = 100 + Wm + K + args.profile_steps + 10      # tuning takes fewer than 100 steps
    for m, wl in enumerate(members):
        b.set_state(m, wl.individuals, wl.tracers)
        nsnap = wl.snapshots_needed(total)
        b.set_series(m, vels=series_arrays(wl, nsnap), ΔT_vel=wl.dT_vel, PARF=wl.parf, ΔT_PAR=wl.dT_PAR,
                     temp=wl.temp, ΔT_temp=wl.dT_temp)
    tune = b.autotune(dT, args.tune_steps) if args.tune_steps > 0 else ""
    n_tune = b.get_time()[0]
    b.step(dT, Wm)
    n0 = b.count_active()
    it0 = b.get_time()[0]
    # the timed steps start a storage-order cycle: they include one counting sort per SORT_INTERVAL
    # steps, the first before their first step
    b.set_sort_interval(SORT_INTERVAL)
    stream = torch.cuda.ExternalStream(b.stream())
    clocks = clocks_cls(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.step(dT, K, sync=False)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ck = clocks.stop()
    b.synchronize()
    ms = e0.elapsed_time(e1)
    n1 = b.count_active()
    if b.get_time()[0] != it0 + K:
        raise RuntimeError(f"the timed region advanced the model by {b.get_time()[0] - it0} steps, not {K}")
    prof = {}
    if args.profile_steps > 0:
        b.set_sort_interval(SORT_INTERVAL)          # the profiled steps include one sort
        # each kernel timed on its own: the x-y tracer kernel in line with the particle kernels
        # (results are the same either way)
        b.set_option("xy_beside_particles", 0)
        b.profile_enable(True)
        b.step(dT, args.profile_steps)
        prof = b.profile_read()
        b.profile_enable(False)
        if "k32_sort" in prof:
            # a sort runs once per SORT_INTERVAL steps: its share of a step
            n_sort, ms_sort = prof["k32_sort"]
            prof["k32_sort"] = (n_sort, ms_sort / n_sort / SORT_INTERVAL * args.profile_steps)
    nslots = sum(w.capacity * w.nsp for w in members)
    roof, tot = profile_roofline(prof, members, b.count_active(), nslots) if prof else (None, 1.0)
    budgets = b.budget(0)
    b.close()
    return dict(ms=ms, ind_steps=K * (n0 + n1) / 2.0, n0=n0, n1=n1, clocks=ck, prof=prof, roof=roof,
                tot_ms=tot, tune=tune, n_tune=n_tune, budget0=budgets)


def run_fp64(wl, args, lib):
    import ctypes as ct
    import torch
    from PlanktonIndividuals import _abi
    from PlanktonIndividuals._native import CModel
    K = args.fp64_steps
    Wm = 3
    m = CModel(lib, "pi_", wl.grid, wl.bgc, wl.phyt, wl.nsp, wl.capacity, wl.seed, precision=_abi.PI_FP64)
    m.set_state(wl.individuals, wl.tracers)
    nsnap = wl.snapshots_needed(Wm + K + 2)
    vv = series_arrays(wl, nsnap)
    u, v, w = (np.asfortranarray(vv[c]) for c in "uvw")
    dp = lambda a: a.ctypes.data_as(ct.POINTER(ct.c_double))
    sim = ct.c_void_p()
    rc = lib.pi_sim_create(m.h, wl.dT, 1, dp(u), dp(v), dp(w), nsnap, wl.dT_vel, dp(wl.parf),
                           wl.parf.shape[2], wl.dT_PAR, dp(wl.temp), wl.temp.shape[3], wl.dT_temp, ct.byref(sim))
    assert rc == 0, m._errmsg(m.h)
    sp = ct.c_void_p()
    lib.pi_get_stream(m.h, ct.byref(sp))
    stream = torch.cuda.ExternalStream(sp.value)
    for _ in range(Wm):
        lib.pi_sim_update(sim, 0, 0)
    assert lib.pi_synchronize(m.h) == 0, m._errmsg(m.h)
    n0 = sum(m.count_active(s) for s in range(wl.nsp))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(K):
        lib.pi_sim_update(sim, 0, 0)
    e1.record(stream)
    e1.synchronize()
    assert lib.pi_synchronize(m.h) == 0, m._errmsg(m.h)
    ms = e0.elapsed_time(e1)
    n1 = sum(m.count_active(s) for s in range(wl.nsp))
    lib.pi_sim_destroy(sim)
    m.close()
    V = wl.grid.Nx * wl.grid.Ny * wl.grid.Nz
    return {"value": round(K * (n0 + n1) / 2.0 / (ms / 1e3), 1), "unit": UNIT, "steps": K,
            "ms_per_step": round(ms / K, 4), "cell_steps_per_s": round(K * V / (ms / 1e3), 1), "dtype": "f64"}


def run_e2e(wl, args, lib, precision, inputs="f32"):
    """The same metric through the C-ABI with host buffers (pinned), one step per call: every step
    uploads its forcing (vel_copy!, copyto!, copy_interior!) from host arrays with the pi_set_*
    calls (Float32 arrays through the _f32 setters, the reference's arrays when FT = Float32, or
    Float64 arrays), queues TimeStep! (pi_time_step_async) and reads its population counts back
    into host memory (pi_count_active_async). The setters return once their host arrays are copied;
    the copies overlap the step queued before them."""
    import ctypes as ct
    import torch
    from PlanktonIndividuals._native import CModel
    m = CModel(lib, "pi_", wl.grid, wl.bgc, wl.phyt, wl.nsp, wl.capacity, wl.seed, precision=precision)
    m.set_state(wl.individuals, wl.tracers)
    nsnap = wl.snapshots_needed(args.e2e_steps + 2)
    snaps = snapshots(wl, nsnap)
    sp = ct.c_void_p()
    m.lib.pi_get_stream(m.h, ct.byref(sp))
    stream = torch.cuda.ExternalStream(sp.value)
    tdt = torch.float32 if inputs == "f32" else torch.float64

    def pin(a):
        t = torch.empty(int(a.size), dtype=tdt, pin_memory=True)
        out = t.numpy().reshape(a.shape, order="F")
        out[...] = a
        return out

    # every step's inputs staged in pinned host memory before the timed region: the snapshot,
    # PAR and temperature that update! would pick for it (update.jl:18-26)
    vel_p, par_p, tmp_p = {}, {}, {}
    for it in range(args.e2e_steps + 1):
        tnow = it * wl.dT
        tv = min(int(np.floor(tnow / wl.dT_vel)), nsnap - 1)
        tp = int(np.floor(tnow / wl.dT_PAR))
        tt = int(np.floor(tnow / wl.dT_temp))
        if tv not in vel_p:
            vel_p[tv] = tuple(pin(x) for x in snaps[tv])
        if tp not in par_p:
            par_p[tp] = pin(np.asfortranarray(wl.parf[:, :, tp]))
        if tt not in tmp_p:
            tmp_p[tt] = pin(np.asfortranarray(wl.temp[:, :, :, tt]))
    h2d = sum(x.nbytes for x in vel_p[0]) + par_p[0].nbytes + tmp_p[0].nbytes
    counts = torch.zeros((args.e2e_steps + 1) * wl.nsp, dtype=torch.int64, pin_memory=True)
    cbase = counts.data_ptr()
    ptr = ((lambda a: ct.c_void_p(a.ctypes.data)) if inputs == "f32"
           else (lambda a: a.ctypes.data_as(ct.POINTER(ct.c_double))))
    sfx = "_f32" if inputs == "f32" else ""
    set_vel, set_par, set_tmp = (getattr(m.lib, f"pi_set_{k}{sfx}") for k in ("velocity", "PARF", "temp"))

    def check(rc, what):
        if rc != 0:
            raise RuntimeError(f"{what}: {m._errmsg(m.h)}")

    def one_step(i):
        tnow = i * wl.dT
        tv = min(int(np.floor(tnow / wl.dT_vel)), nsnap - 1)
        tp = int(np.floor(tnow / wl.dT_PAR)); tt = int(np.floor(tnow / wl.dT_temp))
        check(set_vel(m.h, *(ptr(x) for x in vel_p[tv])), "set velocity")
        check(set_par(m.h, ptr(par_p[tp])), "set PARF")
        check(set_tmp(m.h, ptr(tmp_p[tt])), "set temp")
        check(m.lib.pi_time_step_async(m.h, ct.c_double(wl.dT)), "time step")
        for s in range(wl.nsp):
            check(m.lib.pi_count_active_async(m.h, s, ct.c_void_p(cbase + 8 * (i * wl.nsp + s))), "count")

    one_step(0)          # untimed: first launch of the step (graph capture of the FP32 form)
    check(m.lib.pi_synchronize(m.h), "synchronize")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ee0, ee1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ee0.record(stream)
    for i in range(1, args.e2e_steps + 1):
        one_step(i)
    ee1.record(stream)
    ee1.synchronize()
    wall = time.perf_counter() - t0
    check(m.lib.pi_synchronize(m.h), "synchronize")
    ev_ms = ee0.elapsed_time(ee1)
    ne = int(counts[wl.nsp:].sum())
    m.close()
    return {"value": round(ne / (ev_ms / 1e3), 1), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": 8 * wl.nsp, "steps": args.e2e_steps,
            "ms_per_step": round(ev_ms / args.e2e_steps, 3), "wall_ms_per_step": round(1e3 * wall / args.e2e_steps, 3),
            "form": "fp32" if precision else "fp64", "inputs": "float32" if inputs == "f32" else "float64",
            "note": "each step uploads its forcing from pinned host arrays through pi_set_velocity/PARF/temp"
                    f"{sfx}, queues pi_time_step_async and reads the population counts with "
                    "pi_count_active_async; CUDA events on the model stream bracket the loop"}


def run_ours(args):
    import torch
    from PlanktonIndividuals import _abi, _lib, workloads as W

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", device_id=torch.device("cuda", local))
    lib = _lib.load()
    if args.workload == "config2":
        args.nx, args.nz = args.nx or 256, args.nz or 64
        args.n_per_species = args.n_per_species or 2_097_152
        members = [W.config2(nx=args.nx, nz=args.nz, N_per_species=args.n_per_species, seed=2 + rank)]
        wdesc = (f"config2: {args.nx}x{args.nx}x{args.nz} grid, 2 species x {args.n_per_species:,} individuals, "
                 f"random-Fourier velocity refreshed every 60 steps, dt=30 s")
        scaling = "weak"
    elif args.workload == "config3":
        args.nx, args.nz = args.nx or 512, args.nz or 128
        args.n_per_species = args.n_per_species or 16_777_216
        members = [W.config3(nx=args.nx, nz=args.nz, N_per_species=args.n_per_species, seed=3 + rank)]
        wdesc = (f"config3: {args.nx}x{args.nx}x{args.nz} grid, 4 species x {args.n_per_species:,} individuals "
                 "(lognormal sizes, mu -0.5/0/0.5/1), random-Fourier velocity refreshed every 60 steps, dt=20 s")
        scaling = "weak"
    elif args.workload == "config4":
        from PlanktonIndividuals.batch import member_cost, shard_members
        allm = W.config4()
        members = [allm[q] for q in shard_members([member_cost(w) for w in allm], ws)[rank]]
        wdesc = "config4: 64 members, grids U{64..256}^2 x U{16..32}, populations 2^U(14,20), 1 species, dt=30 s"
        scaling = "strong"
    else:
        from PlanktonIndividuals.batch import member_cost, shard_members
        allm = W.config5()
        members = [allm[q] for q in shard_members([member_cost(w) for w in allm], ws)[rank]]
        wdesc = "config5: 4096 0D boxes, populations 2^U(8,13), no advection, per-box light phase, dt=60 s"
        scaling = "strong"
    r32 = run_fp32(members, args, dist, local, Clocks)
    ms = r32["ms"]
    t_max, ind_all = ms, r32["ind_steps"]
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
        tot = torch.tensor([ind_all], device="cuda", dtype=torch.float64)
        dist.all_reduce(tot)
        ind_all = float(tot.item())
    K = args.steps
    V = sum(w.grid.Nx * w.grid.Ny * w.grid.Nz for w in members)
    Vall = V
    if dist:
        tv = torch.tensor([float(V)], device="cuda", dtype=torch.float64)
        dist.all_reduce(tv)
        Vall = float(tv.item())
    value = ind_all / (t_max / 1e3)
    cell_steps = K * Vall / (t_max / 1e3)
    print(f"[bench] fp32 {t_max / K:.4f} ms/step, {value:.4g} {UNIT}; kernels (ms/step): "
          + json.dumps({k: round(v[1] / max(args.profile_steps, 1), 4)
                        for k, v in sorted(r32['prof'].items(), key=lambda kv: -kv[1][1])[:14]}),
          file=sys.stderr, flush=True)
    fp64 = e2e = None
    if args.workload in ("config2", "config3"):
        if args.fp64_steps > 0:
            fp64 = run_fp64(members[0], args, lib)
            print(f"[bench] fp64 {fp64['ms_per_step']} ms/step", file=sys.stderr, flush=True)
        if args.e2e_steps > 0:
            e2e = run_e2e(members[0], args, lib, _abi.PI_FP32, "f32")
            print(f"[bench] e2e {e2e['ms_per_step']} ms/step", file=sys.stderr, flush=True)
            e2e["float64_inputs"] = {k: v for k, v in run_e2e(members[0], args, lib, _abi.PI_FP32, "f64").items()
                                     if k in ("value", "ms_per_step", "wall_ms_per_step", "h2d_bytes_per_step")}
    out = None
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline and ws == 1 and args.workload == "config2":
            cpu = cpu_baseline(args.cpu_steps)
        prof = r32["prof"]
        P = max(args.profile_steps, 1)
        out = {
            "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": ws, "steps": K,
            "warmup": args.warmup, "ms_per_step": round(t_max / K, 4), "higher_is_better": True,
            "scaling": scaling, "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": wdesc, "form": "fp32 batched (CUDA graph, autotuned launch shapes)",
                       "members_per_rank": len(members),
                       "l2": "inputs larger than L2 (tracer and particle state of every member over 1 GB)",
                       "parallelism": f"{'replicas' if scaling == 'weak' else 'members split'} x{ws}"},
            "cell_steps_per_s": round(cell_steps, 1),
            "individuals": int(r32["n0"]),
            "fp64": fp64,
            "fp32_over_fp64": (round(value / ws / fp64["value"], 3) if fp64 else None),
            "kernel_profile_ms_per_step": {k: round(v[1] / P, 4) for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])},
            "profile_share": {k: round(v[1] / r32["tot_ms"], 4) for k, v in prof.items()},
            "roofline": r32["roof"],
            "step_roofline": step_roofline(ind_all / K, Vall, t_max / K),
            "cpu_baseline": cpu, "e2e": e2e, "clocks": r32["clocks"],
            "gpu_launches": gpu_launches(prof, P, K, args.workload),
            "sort_interval": SORT_INTERVAL,
            "autotune": {"steps": r32["n_tune"], "choices": r32["tune"].strip().splitlines()},
        }
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return out


# ------------------------------------------------------------------------------------------
# FP32 form against the FP64 form (the FP64 form equals the CPU oracle bit for bit)
# ------------------------------------------------------------------------------------------

def run_accuracy(args):
    from PlanktonIndividuals import _lib, workloads as W
    lib = _lib.load()
    t0 = time.time()
    if args.workload in ("config4", "config5"):
        boxes = W.config5(n_max=args.acc_boxes) if args.workload == "config5" else W.config4(n_max=args.acc_boxes)
        steps = boxes[0].steps
        b = fp32_batch(boxes, steps)
        b.step(boxes[0].dT, steps)
        c32 = [b.count_active(m, 0) for m in range(len(boxes))]
        c64, mass = [], []
        for m, wl in enumerate(boxes):
            mm, sim, keep = fp64_sim(lib, wl, steps)
            for _ in range(steps):
                lib.pi_sim_update(sim, 0, 0)
            assert lib.pi_synchronize(mm.h) == 0, mm._errmsg(mm.h)
            c64.append(mm.count_active(0))
            mass.append(max(mass_rel(interior_mass(lambda n: b.get_tracer(m, n), wl.grid),
                                     interior_mass(mm.get_tracer, wl.grid)).values()))
            lib.pi_sim_destroy(sim)
            mm.close()
        n0 = [wl.N[0] for wl in boxes]
        return {"accuracy": args.workload, "members": len(boxes), "steps": steps, "initial": n0, "fp32": c32, "fp64": c64,
                "members_with_equal_counts": int(sum(int(a == c) for a, c in zip(c32, c64))),
                "max_tracer_mass_rel_err_per_member": [float(x) for x in mass],
                "max_count_diff": int(max(abs(a - c) for a, c in zip(c32, c64))),
                "mean_growth_factor": round(float(np.mean(np.array(c64) / np.array(n0))), 4),
                "max_tracer_mass_rel_err": float(max(mass)),
                "guard_band": dict(zip(("recomputed", "changed"), b.guard_stats())),
                "seconds": round(time.time() - t0, 1)}
    wl = W.config3(seed=3) if args.workload == "config3" else W.config2(seed=2)
    out = {"accuracy": args.workload}
    out.update(fp32_vs_fp64(lib, wl, args.acc_steps))
    out["seconds"] = round(time.time() - t0, 1)
    return out


def cpu_sample_workload():
    from PlanktonIndividuals import workloads as W
    # bounded sample of config2: a 128×128×64 sub-domain with the same individual density
    return W.config2(nx=128, nz=64, N_per_species=2_097_152 // 4, seed=2)


def cpu_baseline(steps):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from PlanktonIndividuals.stepping import VelCache, drive
    wl = cpu_sample_workload()
    m = oracle.from_workload(wl)
    vel = VelCache(wl)
    vel(0)
    drive(m, wl, 1, vel)                  # untimed first step (page-in)
    n0 = sum(m.count_active(s) for s in range(wl.nsp))
    t0 = time.perf_counter()
    drive(m, wl, steps, vel)
    dt = time.perf_counter() - t0
    n1 = sum(m.count_active(s) for s in range(wl.nsp))
    val = steps * (n0 + n1) / 2.0 / dt
    return {"value": round(val, 1), "unit": UNIT, "cores": oracle.num_threads(), "kind": "port",
            "sample": f"{steps} steps of config2 on a 128x128x64 sub-domain, 2x524,288 individuals "
                      f"(same density), CPU oracle (Float64 restatement) with OpenMP",
            "seconds": round(dt, 2)}


def run_reference(args):
    ws, rank, local = dist_setup()
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from PlanktonIndividuals.stepping import VelCache, drive
    wl = cpu_sample_workload()
    m = oracle.from_workload(wl)
    vel = VelCache(wl)
    vel(0)
    drive(m, wl, args.warmup, vel)
    n0 = sum(m.count_active(s) for s in range(wl.nsp))
    t0 = time.perf_counter()
    drive(m, wl, args.steps, vel)
    dt = time.perf_counter() - t0
    n1 = sum(m.count_active(s) for s in range(wl.nsp))
    val = args.steps * (n0 + n1) / 2.0 / dt
    cores = oracle.num_threads()
    sample = (f"config2 128x128x64 sub-domain, 2x524,288 individuals (same density); the reference "
              f"is Julia and not runnable here, so its algorithm runs as the CPU oracle (Float64 "
              f"restatement of TimeStep!) with {cores} OpenMP threads")
    return {"impl": "reference", "metric": METRIC, "value": round(val, 1), "unit": UNIT,
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * dt / args.steps, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": "config2 sample (see cpu_baseline.sample)", "form": "fp64"},
            "cpu_baseline": {"value": round(val, 1), "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(val, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    if args.accuracy:
        out = run_accuracy(args)
    else:
        out = run_reference(args) if args.impl == "reference" else run_ours(args)
    if out is not None:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
