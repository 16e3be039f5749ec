#!/usr/bin/env python
"""Throughput of the PlanktonIndividuals model time step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: config 2 — 256×256×64 grid (50 m × 50 m × 2 m), 2 species × 2,097,152 individuals
seeded in the top 40 m, divergence-free random-Fourier velocity, dt = 30 s (seeded synthetic
inputs). A step is one TimeStep! of the whole model. The headline `value` is individual-steps/s
(active individuals × steps ÷ device time) with every input resident in HBM; `cell_steps_per_s`
gives the tracer cell-steps/s of the same run. `e2e` is the same metric through the C-ABI with
host buffers: each step uploads its velocity/PAR/temperature snapshot from pinned host memory
(vel_copy!/copyto!/copy_interior!, update.jl:18-26), runs pi_time_step, and reads back the
population counts.

Multi-GPU: the model domain is not partitioned; each rank runs an independent replica
(scaling "weak") and `value` sums the replicas' individual-steps over the slowest rank's time.

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

METRIC = "individual-steps/s (config2, FP64 plain)"
UNIT = "ind-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--profile-steps", type=int, default=5)
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
                                       "--format=csv,noheader,nounits", "-lms", "50"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

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
# algorithmic bytes per launch (Float64 form)
# ------------------------------------------------------------------------------------------

def algorithmic_bytes(name, wl, n_active_total):
    """Bytes each launch must move at minimum (Float64 form); see DESIGN.md section 4."""
    g = wl.grid
    V = g.Nx * g.Ny * g.Nz
    NC = wl.nsp * wl.capacity
    inactive = NC - n_active_total
    occupied_layers = min(g.Nz, 20)
    vel_cells = g.Nx * g.Ny * occupied_layers
    if name == "k_particles_sorted":
        # per individual: list entry, flags, stat, cell, x, y, z read; x, y, z, cell, key written;
        # one count update; vel₀, vel½, vel₁ (9 fields) read once over the occupied layers
        return n_active_total * (4 + 1 + 1 + 4 + 24 + 24 + 4 + 4 + 8) + 9 * 8 * vel_cells
    if name == "k_particles":
        # slot pass: flags, stat for every slot; inactive slots: cell, x, y, z read, cell, key written
        return NC * 2 + inactive * (4 + 24 + 8)
    if name == "k_sweep_x":
        return V * (14 * 8 * 2 + 8)
    if name == "k_sweep_y":
        return V * (14 * 8 * 3 + 8)
    if name == "k_sweep_z":
        return V * (14 * 8 * 3 + 8)
    if name == "k_tracer_tail":
        # advective tendency + tracer read, new tracer written, offsets, each entry's 5 terms
        return V * (14 * 8 * 3 + 4) + n_active_total * (4 + 1 + 40)
    if name == "k_physiology":
        # per species launch over C slots: state r/w (Bm,Cq,Nq,Pq,Chl,age r; +Sz w), flags, stat,
        # cell, pos, 7 gathers, 5 consumption terms
        per_active = (6 * 8 + 7 * 8) + 3 + 4 + 4 + 7 * 8 + 40
        return (n_active_total / wl.nsp) * per_active + (wl.capacity - n_active_total / wl.nsp) * 2
    return None


def run_ours(args):
    import ctypes as ct
    import torch
    from PlanktonIndividuals import _abi, _lib, workloads as W
    from PlanktonIndividuals._native import CModel

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", device_id=torch.device("cuda", local))
    lib = _lib.load()
    K, Wm = args.steps, args.warmup
    wl = W.config2(seed=2 + rank)
    total = Wm + K + args.profile_steps
    nsnap = wl.snapshots_needed(total + 1)
    snaps = [wl.velocity(i) for i in range(nsnap)]
    m = CModel(lib, "pi_", wl.grid, wl.bgc, wl.phyt, wl.nsp, wl.capacity, wl.seed, precision=_abi.PI_FP64)
    m.set_state(wl.individuals, wl.tracers)
    # PlanktonSimulation with the forcing series in HBM; one update! call per step
    u = np.asfortranarray(np.stack([s[0] for s in snaps], axis=3))
    v = np.asfortranarray(np.stack([s[1] for s in snaps], axis=3))
    w = np.asfortranarray(np.stack([s[2] for s in snaps], axis=3))
    dp = lambda a: a.ctypes.data_as(ct.POINTER(ct.c_double))
    sim = ct.c_void_p()
    rc = lib.pi_sim_create(m.h, wl.dT, 1, dp(u), dp(v), dp(w), nsnap, wl.dT_vel, dp(wl.parf),
                           wl.parf.shape[2], wl.dT_PAR, dp(wl.temp), wl.temp.shape[3], wl.dT_temp, ct.byref(sim))
    assert rc == 0, m._errmsg(m.h)
    stream_ptr = ct.c_void_p()
    lib.pi_get_stream(m.h, ct.byref(stream_ptr))
    stream = torch.cuda.ExternalStream(stream_ptr.value)

    def step_async():
        r = lib.pi_sim_update(sim, 0, 0)
        if r:
            raise RuntimeError(m._errmsg(m.h))

    for _ in range(Wm):
        step_async()
    assert lib.pi_synchronize(m.h) == 0, m._errmsg(m.h)
    n0 = sum(m.count_active(s) for s in range(wl.nsp))
    clocks = Clocks(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(K):
        step_async()
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ck = clocks.stop()
    assert lib.pi_synchronize(m.h) == 0, m._errmsg(m.h)
    ms = e0.elapsed_time(e1)
    n1 = sum(m.count_active(s) for s in range(wl.nsp))
    ind_steps = K * (n0 + n1) / 2.0
    cells = wl.grid.Nx * wl.grid.Ny * wl.grid.Nz
    t_max = ms
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
        tot = torch.tensor([ind_steps], device="cuda", dtype=torch.float64)
        dist.all_reduce(tot)
        ind_steps_all = float(tot.item())
    else:
        ind_steps_all = ind_steps
    value = ind_steps_all / (t_max / 1e3)
    cell_steps = ws * K * cells / (t_max / 1e3)

    # ---- per-kernel profile (CUDA events around each launch, separate pass) ----
    prof, roof, tot_ms = {}, None, 1.0
    if args.profile_steps > 0:
        prof, roof, tot_ms = kernel_profile(lib, m, wl, args, step_async)
    # ---- end to end through the C-ABI with pinned host buffers ----
    lib.pi_sim_destroy(sim)
    e2e = None
    if args.e2e_steps > 0:
        e2e = run_e2e(m, wl, snaps, nsnap, args, stream)

    out = None
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline and ws == 1:
            cpu = cpu_baseline(args.cpu_steps)
        out = {
            "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": ws, "steps": K,
            "warmup": Wm, "ms_per_step": round(t_max / K, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": "config2: 256x256x64 grid, 2 species x 2,097,152 individuals, "
                                   "random-Fourier velocity, dt=30 s, FP64 plain",
                       "form": "fp64", "l2": "inputs larger than L2 (state ~1.5 GB per model)",
                       "parallelism": f"replicas x{ws}"},
            "cell_steps_per_s": round(cell_steps, 1),
            "individuals": int(n0),
            "kernel_profile_ms_per_step": {k: round(v[1] / args.profile_steps, 4) for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])},
            "profile_share": {k: round(v[1] / tot_ms, 4) for k, v in prof.items()},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": ck,
            "gpu_launches": K * (12 + 4 * wl.nsp),
        }
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    m.close()
    return out


def kernel_profile(lib, m, wl, args, step_async):
    import ctypes as ct
    lib.pi_profile_enable(m.h, 1)
    for _ in range(args.profile_steps):
        step_async()
    nmax = 64
    names = ct.create_string_buffer(4096)
    launches = (ct.c_int64 * nmax)()
    kms = (ct.c_double * nmax)()
    nk = ct.c_int32()
    lib.pi_profile_read(m.h, nmax, names, 4096, launches, kms, ct.byref(nk))
    lib.pi_profile_enable(m.h, 0)
    knames = names.raw.split(b"\0")[:nk.value]
    prof = {kn.decode(): (int(launches[i]), float(kms[i])) for i, kn in enumerate(knames)}
    tot_ms = sum(v[1] for v in prof.values())
    dom = max(prof, key=lambda k: prof[k][1])
    nact = sum(m.count_active(s) for s in range(wl.nsp))
    hbm, peak_kind = measured_peaks()
    byts = algorithmic_bytes(dom, wl, nact)
    roof = None
    if byts:
        per_launch_ms = prof[dom][1] / prof[dom][0]
        ach = byts / (per_launch_ms / 1e3) / 1e9
        roof = {"kernel": dom, "bound": "hbm", "achieved": round(ach, 1), "peak": hbm,
                "peak_source": peak_kind, "unit": "GB/s", "frac": round(ach / hbm, 4),
                "traffic": None, "algorithmic_bytes_per_launch": int(byts),
                "avg_launch_ms": round(per_launch_ms, 4)}
    return prof, roof, tot_ms


def run_e2e(m, wl, snaps, nsnap, args, stream):
    import torch
    g = wl.grid
    pin = lambda shape: torch.empty(int(np.prod(shape)), dtype=torch.float64, pin_memory=True).numpy().reshape(shape, order="F")
    hu, hv, hw = pin(snaps[0][0].shape), pin(snaps[0][1].shape), pin(snaps[0][2].shape)
    hp, ht = pin((g.Nx, g.Ny)), pin((g.Nx, g.Ny, g.Nz))
    h2d = (hu.nbytes + hv.nbytes + hw.nbytes + hp.nbytes + ht.nbytes)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ee0, ee1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ee0.record(stream)
    ne = 0
    for _ in range(args.e2e_steps):
        it, tnow = m.get_time()
        tv = int(np.floor(tnow / wl.dT_vel)); tp = int(np.floor(tnow / wl.dT_PAR)); tt = int(np.floor(tnow / wl.dT_temp))
        src = snaps[min(tv, nsnap - 1)]
        hu[...] = src[0]; hv[...] = src[1]; hw[...] = src[2]
        hp[...] = wl.parf[:, :, tp]; ht[...] = wl.temp[:, :, :, tt]
        m.set_velocity(hu, hv, hw)
        m.set_PARF(hp)
        m.set_temp(ht)
        m.time_step(wl.dT)
        ne += sum(m.count_active(s) for s in range(wl.nsp))
    ee1.record(stream)
    ee1.synchronize()
    wall = time.perf_counter() - t0
    ev_ms = ee0.elapsed_time(ee1)
    return {"value": round(ne / (ev_ms / 1e3), 1), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": 8 * wl.nsp, "steps": args.e2e_steps,
            "ms_per_step": round(ev_ms / args.e2e_steps, 3), "wall_ms_per_step": round(1e3 * wall / args.e2e_steps, 3),
            "note": "each step copies its snapshot into pinned host buffers, uploads it (vel_copy!, "
                    "copyto!, copy_interior!), runs pi_time_step and reads the population counts; "
                    "CUDA events on the model stream bracket the whole loop"}


def cpu_sample_workload():
    from PlanktonIndividuals import workloads as W
    # bounded sample of config2: a 128×128×64 sub-domain with the same individual density
    return W.config2(nx=128, nz=64, N_per_species=2_097_152 // 4, seed=2)


def cpu_baseline(steps):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    from helpers import VelCache, drive
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
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    from helpers import VelCache, drive
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
    out = run_reference(args) if args.impl == "reference" else run_ours(args)
    if out is not None:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
