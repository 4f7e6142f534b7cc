"""Benchmark of the fused B200 time step on the single-grid plain-FP32 workload:
hydro scheme, 4096 x 4096 periodic Kelvin-Helmholtz shear layer (tanh profile, seeded
noise), FP32 state, CFL time step kept on the device, 1000 RK3 steps per run.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl fused|reference]

One process per GPU (torchrun for N > 1); the single grid does not shard, so N GPUs run N
independent replicas and `value` is their aggregate (weak scaling).  Rank 0 prints one
JSON line.  `--impl reference` times the reference's CPU arithmetic (oracle/_ref, the
reference's own stencil/RHS headers compiled for the host; the CPU port where that build is
absent) on the host cores instead, on rank 0 only.
"""
import argparse
import datetime
import glob
import json
import os
import re
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N1 = N2 = 4096
SCHEME, SETUP, SEED = "hydro", "kh", 2
NVAR = 4
ELEM = 4
# Algorithmic HBM bytes per cell and stage: stage 0 reads u, writes v and u'; stage 1
# reads u and v, writes v and u'; stage 2 reads u and v, writes u' (v is dead).
B_STAGE = [3 * NVAR * ELEM, 4 * NVAR * ELEM, 3 * NVAR * ELEM]
B_ALG = sum(B_STAGE)  # 160 B per cell-step
METRIC = "Gcell-steps/s"
CPU_DT = 1.8e-5  # fixed step of the CPU samples: inside this workload's CFL/diffusive limit (~1.86e-5)
DATA = "synthetic: seeded tanh Kelvin-Helmholtz shear layer (setup kh, seed 2)"
WORKLOAD = "hydro 4096x4096 periodic tanh Kelvin-Helmholtz, plain FP32 fused RK3 step, device-resident CFL dt"


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(key):
    """Per-launch DRAM bytes of the substage kernel from a committed ncu summary line
    `bench-traffic: <key> <bytes>` in profiles/*.md, or None."""
    for p in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        for line in open(p):
            m = re.match(r"\s*bench-traffic:\s*(\S+)\s+([0-9.eE+]+)", line)
            if m and m.group(1) == key:
                return float(m.group(2))
    return None


# ---- distributed plumbing (also exercised by tests/test_bench_dist.py with gloo) ---------
def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def dist_init(world, backend):
    import torch.distributed as dist
    if world > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return dist if world > 1 else None


def reduce_max(x, dist, device):
    """Max of a float over ranks (the timing rule: slowest rank)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist, device):
    if dist is not None:
        import torch
        t = torch.zeros(1, device=device)
        dist.all_reduce(t)


def aggregate_rate(cells_per_rank, steps, world, max_seconds):
    """Whole-job Gcell-steps/s: all ranks' cell-steps over the slowest rank's time."""
    return world * cells_per_rank * steps / max_seconds / 1e9


# ---- clocks --------------------------------------------------------------------------
CLOCK_QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


class ClockSampler:
    def __init__(self, index, interval_ms=200):
        self.index = index
        self.interval_ms = interval_ms
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={CLOCK_QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.interval_ms)],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.file.flush()
        rows = []
        with open(self.file.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    rows.append((float(parts[1]), float(parts[2]), float(parts[3]), parts[5:9]))
                except ValueError:
                    continue
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        loaded = [r for r in rows if r[2] > 200.0] or rows  # samples under load (power draw)
        reasons = sorted({names[k] for r in loaded for k in range(4) if r[3][k].lower().startswith("active")})
        return {"sm_mhz": float(np.median([r[0] for r in loaded])), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(loaded), "power_w_max": max(r[2] for r in rows)}


# ---- CPU arithmetic of the reference ------------------------------------------------------
def host_cpu():
    """The host's logical CPU count and model name (/proc/cpuinfo), recorded beside CPU rates."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.lower().startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"nproc": os.cpu_count(), "model": model}


def flop_model(nvar, eqns_flop):
    """The reference's flop model per cell-step, 3 (eqns_flop + 2 NVAR) (src/config.cpp:33)."""
    return 3 * (eqns_flop + 2 * nvar)


def cpu_sample(state, rows, steps, dt):
    """Time `steps` RK3 steps of the reference's CPU arithmetic on a periodic 4096-wide strip
    of `rows` rows cut from the workload's state.  Returns (Gcell-steps/s, kind, cores)."""
    from oracle.oracle import Oracle, available, reference_delta
    kind = "reference" if available(SCHEME, "f32", "reference") else "port"
    o = Oracle(SCHEME, "f32", kind)
    cores = o.threads(os.cpu_count() or 1)
    o.set_delta(*reference_delta(N1, N2, 1.0, 1.0))
    u = o.padded(np.ascontiguousarray(state[:rows]))
    v = o.empty(rows, N2)
    t0 = time.perf_counter()
    o.run(u, v, 0.0, dt, steps)
    el = time.perf_counter() - t0
    return rows * N2 * steps / el / 1e9, kind, cores, el


def calibrated_sample(state, dt, budget_s, min_steps=1):
    """(rows, steps) of a CPU sample that takes about `budget_s` seconds: a strip of the
    state for short budgets, the whole grid and more steps for long ones."""
    rate, _, _, _ = cpu_sample(state, 256, 1, dt)
    cells = budget_s * rate * 1e9
    steps = max(min_steps, int(cells // (N1 * N2)))
    rows = int(cells / (N2 * steps))
    return max(16, min(N1, rows)), steps


# The reference's own benchmark (bench/bench.txt:3-73): hydro-isot FP32 on a Tesla M2090, ms
# per step at each resolution, the best of its four block shapes.
REFERENCE_SWEEP_MS = {1024: 5.468, 1280: 12.136, 1536: 14.992, 1792: 18.016, 2048: 21.188, 2560: 47.83,
                      3072: 59.318, 3584: 71.384, 4096: 84.107, 5120: 151.282, 6144: 189.339, 7168: 285.987,
                      8192: 337.53, 10240: 526.947, 12288: 758.47, 14336: 1036.88}


def run_sweep_leg(device, steps=50, warmup=5, sizes=None):
    """The reference's benchmark sweep re-run here: hydro-isot FP32, periodic 2 pi box, Gaussian
    velocity noise (sigma 0.01, seed 7), the reference's dt, at each of its resolutions
    1024^2 .. 14336^2; steps replayed from the two-step graph, timed with events on the
    simulation's stream.  Beside each, the reference's published ms per step (Tesla M2090)."""
    import torch
    import fg2_b200
    rows = []
    for n, ref_ms in REFERENCE_SWEEP_MS.items():
        if sizes and n not in sizes:
            continue
        with fg2_b200.Sim(n, n, scheme="hydro-isot") as s:
            s.config()
            s.init("noise", seed=7)
            dt = s.getdt()
            stream = torch.cuda.ExternalStream(s.stream, device=device)
            s.set_time(0.0)
            s.advance(warmup, dt, graph=True)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            s.advance(steps, dt, graph=True)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / steps
            status = s.sync()
        rows.append([n, ms, n * n / (ms / 1e3) / 1e9, status, ref_ms, ref_ms / ms])
    return {"workload": "hydro-isot FP32 periodic, noise sigma 0.01 seed 7, reference dt, "
                        f"{steps} steps per size (the reference's bench/bench.txt sweep)",
            "columns": ["n", "ms_per_step", "gcell_steps_per_s", "status", "reference_m2090_ms_per_step",
                        "speedup_vs_reference"], "rows": rows}


def accuracy_vs_f64(scheme, n1, n2, x0, steps, dt, para=()):
    """Per-field RMS and max errors of `steps` FP32 steps against FP64 steps of the same
    scheme from the same state, with one fixed dt (the FP64 oracle on the GPU: the same kernel
    in double, itself pinned to the reference's arithmetic at R = double)."""
    import fg2_b200
    outs = {}
    for storage in ("f64", "f32"):
        with fg2_b200.Sim(n1, n2, scheme=scheme, storage=storage) as s:
            for kv in para:
                s.para(kv)
            s.config()
            s.upload(x0.astype(np.float64 if storage == "f64" else np.float32))
            s.set_time(0.0)
            s.advance(steps, dt)
            status = s.sync()
            outs[storage] = s.download().astype(np.float64)
    err = (outs["f32"] - outs["f64"]).reshape(-1, x0.shape[-1])
    return {"steps": steps, "dt": dt, "status": status, "l2_rms": np.sqrt((err ** 2).mean(0)).tolist(),
            "linf": np.abs(err).max(0).tolist()}


def run_small_leg(device):
    """The small plain configuration in full on both sides: hydro 256^2 periodic, rho = 1,
    p = 1/gamma, Gaussian velocity noise (sigma 0.01, seed 1), the reference's dt, 100 steps;
    on the GPU (steps replayed from the two-step graph, events on the simulation's stream) and
    through the reference's CPU arithmetic on all host cores, from the same state."""
    import torch
    import fg2_b200
    from oracle.oracle import Oracle, available, reference_delta
    n, nsteps = 256, 100
    with fg2_b200.Sim(n, n) as s:
        s.config()
        s.init("noise", seed=1)
        x0 = s.download()
        dt = s.getdt()
        stream = torch.cuda.ExternalStream(s.stream, device=device)
        s.set_time(0.0)
        s.advance(10, dt, graph=True)
        s.upload(x0)
        s.set_time(0.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        s.advance(nsteps, dt, graph=True)
        e1.record(stream)
        e1.synchronize()
        gpu_ms = e0.elapsed_time(e1)
        status = s.sync()
    kind = "reference" if available(SCHEME, "f32", "reference") else "port"
    o = Oracle(SCHEME, "f32", kind)
    cores = o.threads(os.cpu_count() or 1)
    o.set_delta(*reference_delta(n, n, 1.0, 1.0))
    u = o.padded(x0)
    v = o.empty(n, n)
    t0 = time.perf_counter()
    o.run(u, v, 0.0, dt, nsteps)
    cpu_s = time.perf_counter() - t0
    cells = n * n * nsteps
    return {"workload": "hydro 256x256 periodic, noise sigma 0.01 seed 1, reference dt, 100 steps (in full)",
            "gpu": {"value": cells / (gpu_ms / 1e3) / 1e9, "unit": "Gcell-steps/s", "ms_per_step": gpu_ms / nsteps,
                    "status": status, "note": "launch-bound: 64 Kcells per step, all in L2"},
            "cpu": {"value": cells / cpu_s / 1e9, "unit": "Gcell-steps/s", "seconds": cpu_s, "cores": cores,
                    "kind": kind}}


def initial_state():
    import fg2_b200
    q, _ = fg2_b200.setup_evaluate(SETUP, N1, N2, SCHEME, seed=SEED)
    return q.astype(np.float32)


def config_of(storage, world):
    """The workload's `config` object, the same in both arms."""
    return {"workload": WORKLOAD if storage == "f32" else WORKLOAD.replace("plain FP32", f"{storage} deviation storage"),
            "storage": storage, "scheme": SCHEME, "grid": [N1, N2], "setup": SETUP, "seed": SEED,
            "dt": "CFL + diffusive limit, FP64, device-resident", "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (u, u' and v are 268 MB each)"}


def run_reference(args):
    rank, _, world = dist_env()
    if rank != 0:
        return
    # the input comes from the numpy restatement of the setup, so this process maps no
    # library of the product: only the reference's arithmetic compiled for the host
    from oracle.setups import kh
    state = kh(N1, N2, seed=SEED).astype(np.float32)
    dt = CPU_DT
    rows, per = calibrated_sample(state, dt, 120.0 / max(1, args.steps + args.warmup))
    for _ in range(args.warmup):
        cpu_sample(state, rows, per, dt)
    el = 0.0
    for _ in range(args.steps):
        _, kind, cores, e = cpu_sample(state, rows, per, dt)
        el += e
    value = rows * N2 * per * args.steps / el / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Gcell-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / (args.steps * per) * 1e3 * (N1 / rows),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": DATA,
        "config": config_of(args.storage, world),
        "cpu_baseline": {"value": value, "unit": "Gcell-steps/s", "cores": cores, "kind": kind,
                         "sample": f"each step: {per} RK3 step(s) on a periodic {rows}x{N2} strip of the 4096^2 state",
                         "ns_per_cell_step": 1.0 / value, "host": host_cpu()},
        "e2e": {"value": value, "unit": "Gcell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "ns_per_cell_step": 1.0 / value,
    }
    print(json.dumps(line), flush=True)


# ---- the fused GPU path -------------------------------------------------------------------
def run_e2e(sim, state, stream, args, dist, device, world, cells):
    """One frame through the C ABI with host buffers: the pinned host state is uploaded,
    K steps run (graph replay, device-resident dt), the status word and the state are read
    back; all inside the timed region."""
    import torch
    host = torch.empty((N1, N2, NVAR), dtype=torch.float32, pin_memory=True).numpy()
    host[...] = state
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(dist, device)
    torch.cuda.synchronize()
    e0.record(stream)
    sim.upload(host)
    sim.set_time(0.0)
    sim.advance(args.steps, 0.0, graph=True)
    status = sim.sync()
    sim.download(out=host)
    e1.record(stream)
    e1.synchronize()
    e2e_ms = reduce_max(e0.elapsed_time(e1), dist, device)
    state_bytes = cells * NVAR * ELEM

    # the reference's solve loop (src/solve.cpp:38-41) through the same C ABI: per step getdt()
    # (the FP64 CFL + diffusive reduction, read back) and step() (status read back)
    k_loop = min(args.steps, 200)
    barrier(dist, device)
    torch.cuda.synchronize()
    e0.record(stream)
    sim.upload(host)
    t, loop_status = 0.0, 0
    for _ in range(k_loop):
        dt = sim.getdt()
        loop_status |= sim.step(t, dt)
        t += dt
    sim.download(out=host)
    e1.record(stream)
    e1.synchronize()
    loop_ms = reduce_max(e0.elapsed_time(e1), dist, device)
    status_bytes = 48  # the status block one getdt() or step() reads back
    per_step = {"value": aggregate_rate(cells, k_loop, world, loop_ms / 1e3), "unit": "Gcell-steps/s",
                "steps": k_loop, "status": loop_status,
                "h2d_bytes_per_step": state_bytes / k_loop,
                "d2h_bytes_per_step": state_bytes / k_loop + 2 * status_bytes,
                "what": "per step: getdt() (CFL reduction kernel, read back) then step() (three substage "
                        "launches, status read back); pinned state uploaded before and downloaded after"}
    return {"value": aggregate_rate(cells, args.steps, world, e2e_ms / 1e3), "unit": "Gcell-steps/s",
            "h2d_bytes_per_step": state_bytes / args.steps,
            "d2h_bytes_per_step": (state_bytes + status_bytes) / args.steps,
            "what": "one frame through the C ABI: pinned host state uploaded, K graph-replayed steps, "
                    "status read, state downloaded",
            "reference_solve_loop": per_step}, status



# ---- single-grid tiling -------------------------------------------------------------------
def tune_single(sim, cache=None, key=None):
    """Autotune a single grid's tiling (fg2_sim_autotune, state left unchanged), or apply the
    tiling already found for the same key (grid size, scheme, storage).  Returns the tiling."""
    if cache is not None and key in cache:
        sim.set_tiling(*cache[key])
        return cache[key]
    sim.autotune(reps=3)
    t = sim.tiling()
    if cache is not None:
        cache[key] = t
    return t


# ---- the batch path (secondary result) -----------------------------------------------------
BATCH_SIDES = (64, 96, 128, 192, 256, 384, 512)
BATCH_COUNT, BATCH_SEED = 512, 4
B_ALG_ISOT = 10 * 3 * 4  # 120 B per cell-step: hydro-isot, FP32


def batch_sizes(count=BATCH_COUNT, seed=BATCH_SEED):
    """Square sides drawn uniformly from BATCH_SIDES with the seed."""
    rng = np.random.default_rng(seed)
    return [(int(x), int(x)) for x in rng.choice(BATCH_SIDES, size=count)]


def batch_accuracy(sizes, x0, steps=20, dt=1.0e-3):
    """FP32 batch against the same batch in FP64 from the same member states, one fixed dt:
    RMS and max errors per field over all members."""
    import fg2_b200
    outs = {}
    for storage in ("f64", "f32"):
        with fg2_b200.Batch(sizes, scheme="hydro-isot", storage=storage) as b:
            b.config()
            for m, x in zip(b.members, x0):
                m.upload(x.astype(np.float64 if storage == "f64" else np.float32))
            b.set_time(0.0)
            b.advance(steps, dt, graph=True)
            status = b.sync()
            outs[storage] = [m.download().astype(np.float64).reshape(-1, 3) for m in b.members]
    err = np.concatenate([a - c for a, c in zip(outs["f32"], outs["f64"])])
    return {"steps": steps, "dt": dt, "status": status, "l2_rms": np.sqrt((err ** 2).mean(0)).tolist(),
            "linf": np.abs(err).max(0).tolist()}


def run_batch_leg(steps, warmup, device, tiling=None, one_at_a_time=True, rank=0, world=1, dist=None):
    """512 independent hydro-isot simulations (sides 64..512, box 2 pi, random-phase k^-2
    velocity at rms Mach 0.3): one persistent launch per substage over every member's tiles,
    two-step CUDA graph, per-member device-resident CFL steps, autotuned tiling.  Beside it,
    the same simulations advanced one after another through the single-grid path on one
    stream (one two-step graph per simulation).  With world > 1 every rank steps its share of
    the 512 members (fg2_b200.shard_members, by cell count; member k keeps its seed), with no
    exchange; the rate is all members' cell-steps over the slowest rank's time."""
    import torch
    import fg2_b200
    all_sizes = batch_sizes()
    isot_fpc = flop_model(3, fg2_b200.load_library("hydro-isot").fg2_eqns_flop())  # 660
    mine = fg2_b200.shard_members(all_sizes, world)[rank]
    sizes = [all_sizes[k] for k in mine]
    two_pi = 2 * np.pi
    b = fg2_b200.Batch(sizes, scheme="hydro-isot")
    b.set_box(two_pi, two_pi)
    b.config()
    for m, k in zip(b.members, mine):
        m.init("turb", seed=BATCH_SEED * 100000 + k)
    x0 = [m.download() for m in b.members]
    if tiling:
        b.set_tiling(*tiling[:2])
        if len(tiling) > 2:
            b.set_strip(tiling[2])
        tune_ms = None
    else:
        tune_ms = b.autotune(reps=4)
    nb, ctas = b.tiling()
    strip = b.strip()
    cells = b.cells
    stream = torch.cuda.ExternalStream(b.stream, device=device)
    b.set_time(0.0)
    b.advance(max(warmup, 4), 0.0, graph=True)
    if b.sync() != 0:
        raise RuntimeError("batch warm-up produced a bad status")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    barrier(dist, device)
    torch.cuda.synchronize()
    e0.record(stream)
    b.advance(steps, 0.0, graph=True)
    e1.record(stream)
    e1.synchronize()
    ms = reduce_max(e0.elapsed_time(e1), dist, device)
    status = int(reduce_max(b.sync(), dist, device))
    total_cells = sum(a * c for a, c in all_sizes)
    value = total_cells * steps / (ms / 1e3) / 1e9
    peak, _ = peaks()
    b.close()
    accuracy = batch_accuracy(sizes, x0) if one_at_a_time else None

    result = {"workload": f"{len(all_sizes)} hydro-isot sims, sides {list(BATCH_SIDES)} drawn with seed {BATCH_SEED}, "
                          "box 2 pi, k^-2 random-phase velocity rms Mach 0.3, FP32, per-member CFL dt",
              "cells": total_cells, "steps": steps, "value": value, "unit": "Gcell-steps/s", "ms_per_step": ms / steps,
              "status": status, "accuracy_vs_f64": accuracy, "tiling": {"strip_columns": strip, "warps_per_cta": strip // 32, "blocks_of_7_rows": nb,
                         "ctas_per_sm": ctas, "autotune_step_ms": tune_ms},
              "roofline": {"bound": "hbm", "bytes_per_cell_step": B_ALG_ISOT,
                           "achieved": value * B_ALG_ISOT, "peak": peak, "unit": "GB/s",
                           "frac": value * B_ALG_ISOT / peak,
                           "traffic": profiled_traffic("substage_batch_isot_c4"),
                           "traffic_unit": "DRAM bytes per step (three launches), one ncu capture",
                           "algorithmic_bytes_per_step": B_ALG_ISOT * total_cells},
              "flops_ref_model": {"gflops": value * isot_fpc, "flop_per_cell_step": isot_fpc},
              "gpu_launches_per_step": 4}
    if world > 1:
        result.update(n_gpus=world, scaling="strong", sharding="members by cell count, no exchange",
                      rank0_members=len(sizes), rank0_cells=cells, ms_per_step_max_over_ranks=ms / steps)
    if not one_at_a_time:
        return result

    # the same simulations one at a time through the single-grid path, on one stream
    k_alone = min(steps, 20)
    alone_stream = torch.cuda.Stream(device=device)
    sims = []
    tuned = {}
    for k, (n1, n2) in enumerate(sizes):
        s = fg2_b200.Sim(n1, n2, scheme="hydro-isot", stream=alone_stream.cuda_stream)
        s.set_box(two_pi, two_pi)
        s.config()
        s.upload(x0[k])
        tune_single(s, tuned, (n1, n2))  # every grid size autotuned once
        s.set_time(0.0)
        s.advance(4, 0.0, graph=True)
        sims.append(s)
    # one untimed pass over every simulation: the first pass's host-side enqueue of 512
    # graphs runs up to 1.3x slower than later ones
    for s in sims:
        s.advance(k_alone, 0.0, graph=True)
    torch.cuda.synchronize()
    e0.record(alone_stream)
    for s in sims:
        s.advance(k_alone, 0.0, graph=True)
    e1.record(alone_stream)
    e1.synchronize()
    ms_alone = e0.elapsed_time(e1)
    for s in sims:
        s.close()
    alone = cells * k_alone / (ms_alone / 1e3) / 1e9
    result["one_at_a_time"] = {"value": alone, "steps": k_alone, "ms_per_step": ms_alone / k_alone,
                               "what": "same members, single-grid path (tiling autotuned per grid size), "
                                       "one simulation after another"}
    result["speedup_vs_one_at_a_time"] = value / alone
    return result


# ---- the 16-bit deviation-storage path (secondary results) ----------------------------------
# 16-bit storage: u, v and the rounding residual r of u, 2 B per value.  Every stage reads u
# with its residual r (the stencil reads the compensated state) and writes u' with its
# residual; stage 0 also writes v, stage 1 reads and writes v, stage 2 reads v: 16 array
# passes, 128 B per cell-step for hydro (80 B of them the plain RK3 traffic of u and v, 48 B
# the compensation)
B_ALG_F16 = 16 * NVAR * 2


def run_mixed_leg(state, steps, warmup, device, plain_value):
    """The headline workload with the state stored as FP16 / BF16 deviations (per-field
    background, per-64x64-tile scales), FP32 stencil, compensated update (every rounding
    residual kept)."""
    import torch
    import fg2_b200
    out = {}
    peak, _ = peaks()
    for storage in ("f16", "bf16"):
        sim = fg2_b200.Sim(N1, N2, scheme=SCHEME, storage=storage)
        sim.config()
        sim.upload(state)
        tiling = tune_single(sim)
        sim.set_dt_mode("cfl")
        stream = torch.cuda.ExternalStream(sim.stream, device=device)
        sim.set_time(0.0)
        sim.advance(max(warmup, 3), 0.0, graph=True)
        if sim.sync() != 0:
            raise RuntimeError(f"{storage} warm-up produced a bad status")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        sim.advance(steps, 0.0, graph=True)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        status = sim.sync()
        sim.close()
        value = N1 * N2 * steps / (ms / 1e3) / 1e9
        out[storage] = {"value": value, "unit": "Gcell-steps/s", "ms_per_step": ms / steps, "status": status,
                        "speedup_vs_plain_f32": value / plain_value, "tiling": list(tiling),
                        "roofline": {"bound": "hbm", "bytes_per_cell_step": B_ALG_F16, "achieved": value * B_ALG_F16,
                                     "peak": peak, "unit": "GB/s", "frac": value * B_ALG_F16 / peak}}
    return out


DISK_N = 2048
DISK_DT = 1.0e-7  # inside the explicit radiation-diffusion limit (~0.28 Delta^2 = 6.6e-7 here)
DISK_FLOP = 3 * (733 + 2 * 6)  # the reference's flop model per cell-step (src/config.cpp:33)
DISK_B_ALG = 10 * 6 * 4  # 240 B per cell-step (six FP32 fields)


def run_disk_leg(steps, warmup, device, tiling=None):
    """The disk scheme (six fields, log-r / theta grid, 733-flop right-hand side) at
    2048 x 2048 on the smooth torus-like state, FP32, fixed dt, steps replayed from the
    two-step CUDA graph, tiling autotuned (or fixed by `tiling`).  Compute-heavy: reported
    against the reference's flop model and against HBM."""
    import torch
    import fg2_b200
    peak, _ = peaks()
    with fg2_b200.Sim(DISK_N, DISK_N, scheme="disk") as sim:
        sim.config()
        sim.init("smooth", seed=3)
        if tiling:
            sim.set_tiling(*tiling)
        else:
            sim.autotune(reps=3)
        tiled = sim.tiling()
        stream = torch.cuda.ExternalStream(sim.stream, device=device)
        sim.set_time(0.0)
        sim.advance(max(warmup, 3), DISK_DT, graph=True)
        if sim.sync() != 0:
            raise RuntimeError("disk warm-up produced a bad status")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with ClockSampler(device.index or 0, 50) as clk:
            e0.record(stream)
            sim.advance(steps, DISK_DT, graph=True)
            e1.record(stream)
            e1.synchronize()
        ms = e0.elapsed_time(e1)
        status = sim.sync()
    cells = DISK_N * DISK_N
    value = cells * steps / (ms / 1e3) / 1e9
    nd = 512  # FP32 against FP64 on a smaller grid of the same setup (FP64 disk kernels are slow)
    x0, _ = fg2_b200.setup_evaluate("smooth", nd, nd, scheme="disk", seed=3)
    acc = accuracy_vs_f64("disk", nd, nd, x0, 20, 2.0e-6)
    return {"workload": f"disk {DISK_N}x{DISK_N} smooth torus-like state (seed 3), FP32, fixed dt {DISK_DT:g}, walls",
            "value": value, "unit": "Gcell-steps/s", "steps": steps, "ms_per_step": ms / steps, "status": status,
            "gflops_ref_model": value * DISK_FLOP, "flop_per_cell_step": DISK_FLOP,
            "tiling": {"blocks_of_7_rows": tiled[0], "ctas_per_sm": tiled[1], "tail_bands": tiled[2],
                       "how": "fixed" if tiling else "fg2_sim_autotune"},
            "clocks": clk.summary(),
            "accuracy_vs_f64": dict(acc, grid=[nd, nd]),
            "roofline": {"bound": "compute", "bytes_per_cell_step": DISK_B_ALG, "hbm_achieved": value * DISK_B_ALG,
                         "hbm_peak": peak, "unit": "GB/s", "hbm_frac": value * DISK_B_ALG / peak,
                         "traffic": profiled_traffic("substage_disk_f32_2048"),
                         "traffic_unit": "DRAM bytes per step (three launches), one ncu capture"}}


def f16_numbers(x):
    """The values of the FP16 numbers that deviation storage holds for the state x (per-field
    mean as background, 0 for u2; per-64x64-tile largest deviation as scale), without their
    rounding residual."""
    n1, n2, nv = x.shape
    bg = x.reshape(-1, nv).astype(np.float64).mean(0).astype(np.float32)
    bg[2] = 0.0
    t = 64
    d = np.abs(x - bg).reshape(n1 // t, t, n2 // t, t, nv).max(axis=(1, 3))
    d[~(d > 0)] = 1.0
    s = np.repeat(np.repeat(d, t, 0), t, 1)
    return (bg + s * ((x - bg) / s).astype(np.float16).astype(np.float32)).astype(np.float32)


def run_precision_leg(n, steps, device):
    """Kelvin-Helmholtz at n x n, the same fixed step sequence in FP64, FP32 and the 16-bit
    deviation storages; per-field L2 (RMS) and Linf errors against the FP64 run, and the
    relative L2 error of the density rho = exp(lnd).  Also FP32 steps from the initial state
    rounded once to the FP16 numbers of deviation storage, residual dropped (`f32_from_f16_start`):
    the error that a single uncompensated 16-bit rounding of the state leaves."""
    import fg2_b200
    state = fg2_b200.setup_evaluate(SETUP, n, n, SCHEME, seed=SEED)[0]
    with fg2_b200.Sim(n, n, scheme=SCHEME, storage="f64") as s:
        s.config()
        s.upload(state)
        s.set_dt_mode("cfl")
        dt = 0.9 * s.getdt()
        s.advance(steps, dt)
        ref = s.download()
    state32 = state.astype(np.float32)
    del state
    rho_ref = np.exp(ref[..., 0])
    rho_norm = np.sqrt((rho_ref ** 2).sum())
    result = {"grid": [n, n], "steps": steps, "dt": dt, "fields": ["lnd", "u1", "u2", "lne"]}
    rounded_start = f16_numbers(state32)  # bg + s h: one FP16 rounding of the state, residual dropped
    for storage in ("f32", "f16", "bf16", "f32_from_f16_start"):
        with fg2_b200.Sim(n, n, scheme=SCHEME, storage="f32" if storage == "f32_from_f16_start" else storage) as s:
            s.config()
            s.upload(rounded_start if storage == "f32_from_f16_start" else state32)
            s.advance(steps, dt)
            status = s.sync()
            out = s.download()
        err = out.astype(np.float64) - ref
        rms = np.sqrt((err.reshape(-1, NVAR) ** 2).mean(0))
        linf = np.abs(err.reshape(-1, NVAR)).max(0)
        rho_l2 = float(np.sqrt(((np.exp(out[..., 0].astype(np.float64)) - rho_ref) ** 2).sum()) / rho_norm)
        result[storage] = {"status": status, "l2_rms": rms.tolist(), "linf": linf.tolist(), "rho_rel_l2": rho_l2}
        del out, err
    for storage in ("f16", "bf16", "f32_from_f16_start"):
        result[storage]["rho_rel_l2_vs_f32"] = result[storage]["rho_rel_l2"] / max(result["f32"]["rho_rel_l2"], 1e-300)
    return result


# ---- batch + 16-bit storage (secondary result) ----------------------------------------------
COMBINED_SIDES = (512, 1024, 2048)
COMBINED_COUNT, COMBINED_SEED, COMBINED_STEPS = 64, 5, 300


def run_combined_leg(device):
    """64 hydro sims (sides from {512, 1024, 2048} by seed 5, k^-2 random-phase velocity at rms
    Mach 0.5, rho = 1, p = 1/gamma): the FP16 batch against the same sims advanced one at a
    time in plain FP32 (and, for reference, as an FP32 batch), all with one fixed dt (0.9 x the
    smallest member CFL step) for 300 steps, replayed from graphs; errors against an FP64
    batch with the same steps."""
    import torch
    import fg2_b200
    rng = np.random.default_rng(COMBINED_SEED)
    sizes = [(int(x), int(x)) for x in rng.choice(COMBINED_SIDES, size=COMBINED_COUNT)]
    states = [fg2_b200.setup_evaluate("turb", n1, n2, SCHEME, seed=COMBINED_SEED * 1000 + k)[0]
              for k, (n1, n2) in enumerate(sizes)]
    cells = sum(n1 * n2 for n1, n2 in sizes)

    def timed(fn, stream):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    # the common step: 0.9 x the FP64 CFL step of the finest member (the smallest over members)
    k_fine = max(range(len(sizes)), key=lambda k: sizes[k][0])
    with fg2_b200.Sim(*sizes[k_fine], scheme=SCHEME, storage="f64") as s:
        s.config()
        s.upload(states[k_fine])
        s.set_dt_mode("cfl")
        dt = 0.9 * s.getdt()

    def run_batch(storage, time_it):
        b = fg2_b200.Batch(sizes, scheme=SCHEME, storage=storage)
        b.config()
        for k, m in enumerate(b.members):
            m.upload(states[k] if storage == "f64" else states[k].astype(np.float32))
        stream = torch.cuda.ExternalStream(b.stream, device=device)
        if time_it:
            b.autotune(reps=2)
        b.advance(2, dt, graph=True)  # warm-up: captures the graph ...
        for k, m in enumerate(b.members):  # ... then back to the initial states
            m.upload(states[k] if storage == "f64" else states[k].astype(np.float32))
        ms = timed(lambda: b.advance(COMBINED_STEPS, dt, graph=True), stream)
        status = b.sync()
        outs = [m.download() for m in b.members]
        b.close()
        return ms, status, outs

    ms64, st64, ref = run_batch("f64", False)
    ms16, st16, out16 = run_batch("f16", True)
    msb32, stb32, outb32 = run_batch("f32", True)
    # the plain FP32 path, one simulation after another on one stream
    stream = torch.cuda.Stream(device=device)
    sims = []
    tuned = {}
    for k, (n1, n2) in enumerate(sizes):
        s = fg2_b200.Sim(n1, n2, scheme=SCHEME, storage="f32", stream=stream.cuda_stream)
        s.config()
        s.upload(states[k].astype(np.float32))
        tune_single(s, tuned, (n1, n2))  # every grid size autotuned once
        s.advance(2, dt, graph=True)
        s.upload(states[k].astype(np.float32))
        sims.append(s)
    ms32 = timed(lambda: [s.advance(COMBINED_STEPS, dt, graph=True) for s in sims], stream)
    st32 = max(s.sync() for s in sims)
    out32 = [s.download() for s in sims]
    for s in sims:
        s.close()

    def rho_err(outs):
        num = sum(((np.exp(o[..., 0].astype(np.float64)) - np.exp(r[..., 0])) ** 2).sum() for o, r in zip(outs, ref))
        den = sum((np.exp(r[..., 0]) ** 2).sum() for r in ref)
        return float(np.sqrt(num / den))

    v16 = cells * COMBINED_STEPS / (ms16 / 1e3) / 1e9
    v32 = cells * COMBINED_STEPS / (ms32 / 1e3) / 1e9
    vb32 = cells * COMBINED_STEPS / (msb32 / 1e3) / 1e9
    e16, e32, eb32 = rho_err(out16), rho_err(out32), rho_err(outb32)
    return {"workload": f"{len(sizes)} hydro sims, sides {list(COMBINED_SIDES)} drawn with seed {COMBINED_SEED}, "
                        f"k^-2 random-phase velocity rms Mach 0.5, fixed dt {dt:.4g}, {COMBINED_STEPS} steps",
            "cells": cells, "dt": dt,
            "f16_batch": {"value": v16, "unit": "Gcell-steps/s", "ms_per_step": ms16 / COMBINED_STEPS, "status": st16,
                          "rho_rel_l2_vs_f64": e16},
            "f32_one_at_a_time": {"value": v32, "unit": "Gcell-steps/s", "ms_per_step": ms32 / COMBINED_STEPS,
                                  "status": st32, "rho_rel_l2_vs_f64": e32,
                                  "tiling": {f"{k[0]}x{k[1]}": list(v) for k, v in tuned.items()}},
            "f32_batch": {"value": vb32, "unit": "Gcell-steps/s", "ms_per_step": msb32 / COMBINED_STEPS,
                          "status": stb32, "rho_rel_l2_vs_f64": eb32},
            "speedup": v16 / v32, "error_ratio": e16 / max(e32, 1e-300), "f64_status": st64}


def compact(x, digits=5):
    """Floats rounded to `digits` significant digits (the JSON line stays short)."""
    if isinstance(x, float):
        return float(f"{x:.{digits}g}") if np.isfinite(x) else x
    if isinstance(x, dict):
        return {k: compact(v, digits) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [compact(v, digits) for v in x]
    return x


def summary_of(line):
    """The secondary legs' headline numbers in a few hundred bytes (the last key of the line,
    so a truncated tail of the output still shows them)."""
    def g(d, *keys):  # nested lookup, None where a level is missing
        for k in keys:
            d = d.get(k) if isinstance(d, dict) else None
        return d

    out = {}
    out["plain_f32"] = {"gcs": line.get("value"), "hbm_frac": g(line, "roofline", "frac"),
                        "e2e_gcs": g(line, "e2e", "value"), "tiling": [g(line, "tiling", "blocks_of_7_rows"),
                                                                       g(line, "tiling", "ctas_per_sm"),
                                                                       g(line, "tiling", "tail_bands")]}
    if line.get("batch"):
        b = line["batch"]
        out["c4_batch"] = {"gcs": b.get("value"), "hbm_frac": g(b, "roofline", "frac"),
                           "one_at_a_time_gcs": g(b, "one_at_a_time", "value")}
    if line.get("mixed"):
        out["mixed_4096"] = {k: {"gcs": v.get("value"), "x_f32": v.get("speedup_vs_plain_f32")}
                             for k, v in line["mixed"].items()}
    if line.get("precision"):
        p = line["precision"]
        out["c3_rho_rel_l2"] = {k: g(p, k, "rho_rel_l2") for k in ("f32", "f16", "bf16", "f32_from_f16_start")}
    if line.get("combined"):
        c = line["combined"]
        out["c5"] = {"f16_batch_gcs": g(c, "f16_batch", "value"), "f32_alone_gcs": g(c, "f32_one_at_a_time", "value"),
                     "f32_batch_gcs": g(c, "f32_batch", "value"), "speedup": c.get("speedup"),
                     "rho_err_ratio": c.get("error_ratio")}
    if line.get("disk"):
        out["disk_gcs"] = line["disk"].get("value")
    if line.get("small"):
        out["c1"] = {"gpu_gcs": g(line, "small", "gpu", "value"), "cpu_gcs": g(line, "small", "cpu", "value")}
    if line.get("sweep"):
        cols = line["sweep"]["columns"]
        out["sweep_gcs"] = {str(r[0]): r[cols.index("gcell_steps_per_s")] for r in line["sweep"]["rows"]}
    out["cpu_baseline_gcs"] = g(line, "cpu_baseline", "value")
    return compact(out, 4)


def run_fused(args):
    import torch
    import fg2_b200

    if args.only_batch:  # the batch leg alone (profiling): fixed tiling, no one-at-a-time leg
        torch.cuda.set_device(0)
        tiling = tuple(int(x) for x in args.batch_tiling.split(",")) if args.batch_tiling else None
        print(json.dumps(run_batch_leg(args.steps, args.warmup, torch.device("cuda", 0), tiling, False)), flush=True)
        return
    if args.only_sweep:  # the reference's benchmark sweep alone
        torch.cuda.set_device(0)
        sizes = [int(x) for x in args.sweep_sizes.split(",")] if args.sweep_sizes else None
        print(json.dumps(run_sweep_leg(torch.device("cuda", 0), sizes=sizes)), flush=True)
        return
    if args.only_combined:  # the combined (64-sim FP16 batch) leg alone
        torch.cuda.set_device(0)
        print(json.dumps(run_combined_leg(torch.device("cuda", 0))), flush=True)
        return
    if args.only_precision:  # the 8192^2 precision leg alone
        torch.cuda.set_device(0)
        print(json.dumps(run_precision_leg(8192, 500, torch.device("cuda", 0))), flush=True)
        return
    if args.only_disk:  # the disk-scheme leg alone (profiling: --tiling fixes its tiling)
        torch.cuda.set_device(0)
        tiling = tuple(int(x) for x in args.tiling.split(",")) if args.tiling else None
        print(json.dumps(run_disk_leg(args.steps, args.warmup, torch.device("cuda", 0), tiling)), flush=True)
        return

    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    dist = dist_init(world, "nccl")

    sim = fg2_b200.Sim(N1, N2, scheme=SCHEME, storage=args.storage)
    b_alg = B_ALG_F16 if args.storage in ("f16", "bf16") else B_ALG  # 160 B FP32, 128 B 16-bit
    fpc = flop_model(NVAR, sim.lib.fg2_eqns_flop())  # 891 for hydro
    sim.config()
    state = initial_state()
    sim.upload(state)
    if args.tiling:  # fixed tiling (profiling runs: no autotune launches before the captured ones)
        sim.set_tiling(*[int(x) for x in args.tiling.split(",")])
        tiling = sim.tiling()
    else:
        tiling = tune_single(sim)  # the successor of the reference's block-size heuristic
    sim.set_dt_mode("cfl")
    stream = torch.cuda.ExternalStream(sim.stream, device=device)
    cells = N1 * N2

    # warm-up (graph capture happens here)
    sim.set_time(0.0)
    sim.advance(max(args.warmup, 3), 0.0, graph=True)
    if sim.sync() != 0:
        raise RuntimeError("warm-up produced a bad status")

    # timed region: K steps through the graph, device-resident CFL dt
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(dist, device)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        sim.advance(args.steps, 0.0, graph=True)
        ev1.record(stream)
        ev1.synchronize()
    status = sim.sync()
    torch.cuda.synchronize()
    barrier(dist, device)
    ms = reduce_max(ev0.elapsed_time(ev1), dist, device)
    value = aggregate_rate(cells, args.steps, world, ms / 1e3)
    sim_time = sim.time()

    # per-launch duration of the substage kernel, live, on the launching stream
    dt_fixed = sim.last_dt()
    reps = 20
    evs = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
           for _ in range(3)]
    for r in range(reps):
        for k in range(3):
            evs[k][r][0].record(stream)
            sim.stage(k, dt_fixed)
            evs[k][r][1].record(stream)
    torch.cuda.synchronize()
    stage_ms = [float(np.mean([a.elapsed_time(b) for a, b in evs[k][2:]])) for k in range(3)]
    if sim.sync() != 0:
        raise RuntimeError("stage timing produced a bad status")
    peak, peak_kind = peaks()
    achieved = b_alg * cells / (sum(stage_ms) / 1e3) / 1e9  # GB/s over the three launches
    traffic = profiled_traffic(f"substage_hydro_{args.storage}_4096")

    # end to end through the public API: pinned host state in, K steps, state out
    e2e, e2e_status = None, None
    if not args.no_e2e:
        e2e, e2e_status = run_e2e(sim, state, stream, args, dist, device, world, cells)

    accuracy = None
    if rank == 0 and world == 1 and not args.no_accuracy and args.storage == "f32":
        accuracy = accuracy_vs_f64(SCHEME, N1, N2, state, 100, CPU_DT)

    batch = None
    if not args.no_batch and args.storage == "f32":
        # N > 1: every rank steps its share of the members (the same collective steps on all)
        batch = run_batch_leg(200, args.warmup, device, one_at_a_time=world == 1, rank=rank, world=world,
                              dist=dist)

    mixed, precision, combined = None, None, None
    if rank == 0 and world == 1 and not args.no_mixed and args.storage == "f32":
        mixed = run_mixed_leg(state, args.steps, args.warmup, device, value / world)
        precision = run_precision_leg(8192, 500, device)
        combined = run_combined_leg(device)

    disk = None
    if rank == 0 and world == 1 and not args.no_disk and args.storage == "f32":
        disk = run_disk_leg(200, args.warmup, device)

    small = None
    if rank == 0 and world == 1 and not args.no_cpu and args.storage == "f32":
        small = run_small_leg(device)

    sweep = None
    if rank == 0 and world == 1 and not args.no_sweep and args.storage == "f32":
        sweep = run_sweep_leg(device)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rows, per = calibrated_sample(state, CPU_DT, 20.0, 2)
        rate, kind, cores, el = cpu_sample(state, rows, per, CPU_DT)
        cpu = {"value": rate, "unit": "Gcell-steps/s", "cores": cores, "kind": kind,
               "sample": f"{per} RK3 steps on a periodic {rows}x{N2} strip of the 4096^2 state ({el:.1f} s)",
               "ns_per_cell_step": 1.0 / rate, "host": host_cpu()}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Gcell-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if args.storage == "f32" else f"{args.storage} storage, f32 math",
            "data": DATA,
            "config": config_of(args.storage, world),
            "ns_per_cell_step": 1.0 / (value / world),
            "status": status, "sim_time": sim_time,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "frac_nominal_8tbs": achieved / 8000.0,
                         "bytes_per_cell_step": b_alg, "stage_ms": stage_ms,
                         "dram_gbs_from_traffic": traffic / (sum(stage_ms) / 1e3) / 1e9 if traffic else None},
            "flops_ref_model": {"gflops": value * fpc, "flop_per_cell_step": fpc,
                                "what": "the reference's model 3 (eqns_flop + 2 NVAR) per cell-step (src/config.cpp:33); "
                                        "a secondary figure: the path is HBM-bound"},
            "step_hbm_frac": value / world * b_alg / peak,
            "tiling": {"blocks_of_7_rows": tiling[0], "ctas_per_sm": tiling[1], "tail_bands": tiling[2],
                       "strip_columns": 128,
                       "how": "--tiling" if args.tiling else "fg2_sim_autotune on the workload's own state"},
            "cpu_baseline": cpu,
            "accuracy_vs_f64": accuracy,
            "e2e": e2e, "e2e_status": e2e_status,
            "batch": batch,
            "mixed": mixed,
            "precision": precision,
            "combined": combined,
            "disk": disk,
            "small": small,
            "sweep": sweep,
            "gpu_launches": 4 * args.steps,
            "clocks": clk.summary(),
        }
        line["summary"] = summary_of(line)
        print(json.dumps(compact(line)), flush=True)
    sim.close()
    if dist is not None:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="fused", choices=["fused", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the batch (secondary) leg")
    ap.add_argument("--no-mixed", action="store_true", help="skip the 16-bit storage and precision legs")
    ap.add_argument("--no-disk", action="store_true", help="skip the disk-scheme leg")
    ap.add_argument("--only-disk", action="store_true", help="run the disk-scheme leg alone and print it")
    ap.add_argument("--only-precision", action="store_true", help="run the 8192^2 precision leg alone and print it")
    ap.add_argument("--only-combined", action="store_true", help="run the combined 64-sim leg alone and print it")
    ap.add_argument("--no-sweep", action="store_true", help="skip the reference's benchmark sweep")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the FP32-against-FP64 error of the headline workload")
    ap.add_argument("--only-sweep", action="store_true", help="run the reference's benchmark sweep alone and print it")
    ap.add_argument("--sweep-sizes", default="", help="comma-separated sides of the sweep to run (default: all)")
    ap.add_argument("--only-batch", action="store_true", help="run the batch leg alone and print it")
    ap.add_argument("--batch-tiling", default="",
                    help="nb,ctas_per_sm[,strip] for the batch leg (default: autotune)")
    ap.add_argument("--tiling", default="",
                    help="nb,ctas_per_sm[,tail_bands] of the headline workload's launches (default: autotune)")
    ap.add_argument("--storage", default="f32", choices=["f32", "f16", "bf16"],
                    help="state storage of the headline workload (f16/bf16: deviation storage)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_fused(args)


if __name__ == "__main__":
    main()
