"""Benchmark of the Barnes-Hut force path on one B200 per rank.

Default workload (the headline configuration): Plummer sphere, N=1,048,576,
scale radius 1 AU, total mass 1 Msun, seed 1; softening 1e-4, dt 1e-4;
Barnes-Hut with the geometric MAC theta=0.5, monopole+quadrupole, FP64 state,
FP32 pair forces.  A step is one velocity-Verlet step on device-resident
state (kick-drift + bbox, keys, sort, tree, multipoles, walk, kick).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 runs N independent replicas (the path does not shard across GPUs:
one system per GPU), one process per GPU under torchrun; time is the max
over ranks.  --impl reference times the reference's own CPU Barnes-Hut
(oracle/_ref: BarnesHutSolver with its job system on all host threads).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "celestial-mechanics-desktop_b200"))
sys.path.insert(0, str(ROOT / "oracle"))

METRIC = "steps/s and body-interactions/s at fixed force error: learned vs geometric MAC"
N_BODIES = 1 << 20
THETA, EPS, DT, SEED = 0.5, 1e-4, 1e-4, 1
# FP32 flops per interaction, counted from the walk's own arithmetic
# (FMA = 2, add/mul/rsqrt = 1): body-body 20, body-cell monopole+quadrupole 51.
FLOPS_BODY, FLOPS_CELL_QUAD = 20, 51
# Algorithmic bytes per body of the integer stages (each array read or
# written once): sort stage = kick-drift+bbox 129 (read pos/vel/acc/mass/
# active, write pos/vel) + zero acc 24 + keys 37 (read pos+active, write
# key+row) + 8 radix passes x 24 (read and write key+row) + gather 68 (read
# row, pos, mass; write double4) = 450; tree stage = radix tree 29 (read key,
# write children/range/prefix/parent) + mark 35 + scan/base 8 + emit 40 +
# multipoles 32 + 0.45 nodes/body x 100 = 189.
SORT_BYTES_PER_BODY, TREE_BYTES_PER_BODY = 450, 189
DISK_RADIUS_SCALE = 30.0


def workload_name(n: int) -> str:
    return "bh_plummer_1m" if n == N_BODIES else f"bh_plummer_n{n}"


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(ws, x: float) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(ws, x: float) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device),
                                          f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            if len(r) < 9:
                continue
            for name, v in zip(names, r[5:9]):
                if v.strip() == "Active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d, "measured"
    return {"hbm_gbs": 6650.0, "sm_max_mhz": 1965.0}, "fallback"


def walk_traffic_per_launch():
    """DRAM bytes of one walk launch from the committed ncu summary, or None."""
    f = ROOT / "profiles" / "k_walk_group_bh_plummer.md"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith("dram_bytes_per_launch:"):
            return float(line.split(":", 1)[1])
    return None


def reference_bh_seconds(b, threads: int) -> tuple[float, str]:
    """One reference Barnes-Hut force evaluation (tree build + parallel walk)
    on the host: the reference's own code when oracle/_ref is built, else
    the oracle restatement.  Returns (seconds, kind)."""
    import oracle

    if oracle.ref() is not None:
        t = time.perf_counter()
        oracle.ref_bh_forces(b.px, b.py, b.pz, b.mass, b.active, EPS, THETA, True, threads)
        return time.perf_counter() - t, "reference"
    t = time.perf_counter()
    oracle.bh_forces(b.px, b.py, b.pz, b.mass, b.active, EPS, THETA, nthreads=threads)
    return time.perf_counter() - t, "port"


def run_reference(args, ws, rank):
    if rank != 0:
        return
    from nbody_b200 import scenarios

    b = scenarios.plummer(args.n, 1.0, 1.0, seed=SEED)
    threads = os.cpu_count() or 1
    warm = min(args.warmup, 1)
    steps = max(1, min(args.steps, 3))
    for _ in range(warm):
        reference_bh_seconds(b, threads)
    total = 0.0
    kind = "port"
    for _ in range(steps):
        s, kind = reference_bh_seconds(b, threads)
        total += s
    value = steps / total
    sample = (f"N=1,048,576 Plummer seed 1: {steps} full force evaluations (serial tree build + "
              f"parallel walk, theta 0.5, monopole), {warm} warm-up")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "steps/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": warm, "ms_per_step": 1e3 * total / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Plummer sphere)",
        "config": {"workload": workload_name(args.n), "n": args.n, "theta": THETA, "eps": EPS,
                   "multipole": "monopole (reference)", "mac": "geometric"},
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": threads, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }))


def run_b200(args, ws, rank, local):
    import torch

    from nbody_b200 import MODE_BARNES_HUT, Engine, scenarios
    from nbody_b200 import _native as N

    dev = local
    torch.cuda.set_device(dev)
    b = scenarios.plummer(args.n, 1.0, 1.0, seed=SEED)
    eng = Engine(args.n, device=dev)
    eng.set_param(N.PARAM_THETA, THETA)
    flags = MODE_BARNES_HUT
    stream = torch.cuda.ExternalStream(eng.stream, device=dev)
    eng.set_state(b, old_acc=False)
    eng.step(max(args.warmup, 3), DT, EPS, flags)
    torch.cuda.synchronize(dev)

    # ---- device-resident timed region ---------------------------------
    clocks = Clocks(dev)
    barrier(ws)
    torch.cuda.synchronize(dev)
    clocks.start()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    walk_ms, build_ms, sort_ms, tree_ms, inter, flops = 0.0, 0.0, 0.0, 0.0, 0, 0.0
    for _ in range(args.steps):
        eng.step(1, DT, EPS, flags)
        tm = eng.timings()
        c = eng.counters()
        walk_ms += tm[N.T_TRAVERSAL]
        build_ms += tm[N.T_BUILD]
        sort_ms += tm[N.T_SORT]
        tree_ms += tm[N.T_TREE]
        inter += int(c[N.C_CELL_INTERACTIONS] + c[N.C_BODY_INTERACTIONS])
        flops += FLOPS_CELL_QUAD * c[N.C_CELL_INTERACTIONS] + FLOPS_BODY * c[N.C_BODY_INTERACTIONS]
    t1.record(stream)
    torch.cuda.synchronize(dev)
    barrier(ws)
    clk = clocks.stop()
    ms = t0.elapsed_time(t1)
    ms_max = max_over_ranks(ws, ms)
    steps_total = sum_over_ranks(ws, args.steps)
    value = steps_total / (ms_max / 1e3)
    inter_total = sum_over_ranks(ws, inter)

    # ---- force error of the last step against the FP64 direct sum -----
    err = eng.force_error(4096, 12345, EPS)

    # ---- end to end through the seam with host buffers -----------------
    st, _ = eng.get_state()
    n = st.n
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    hp = [pin(st.px), pin(st.py), pin(st.pz), pin(st.mass), pin(st.active)]
    out = [pin(np.empty(n)), pin(np.empty(n)), pin(np.empty(n))]
    eng.compute_forces(*hp[:4], hp[4], EPS, flags, out=out)
    barrier(ws)
    torch.cuda.synchronize(dev)
    e0 = time.perf_counter()
    e_steps = max(1, args.steps)
    for _ in range(e_steps):
        eng.compute_forces(*hp[:4], hp[4], EPS, flags, out=out)
    e_s = max_over_ranks(ws, time.perf_counter() - e0)
    e2e_value = sum_over_ranks(ws, e_steps) / e_s
    h2d = 4 * 8 * n + n
    d2h = 3 * 8 * n

    # ---- roofline of the dominant kernel (the walk) --------------------
    pk, pk_kind = peaks()
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    fp32_peak = sms * 128 * 2 * pk.get("sm_max_mhz", 1965.0) * 1e6 / 1e12
    achieved = (flops / args.steps) / (walk_ms / args.steps / 1e3) / 1e12
    traffic = walk_traffic_per_launch()

    line = None
    if rank == 0:
        cpu = None
        if ws == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            s, kind = reference_bh_seconds(b, threads)
            cpu = {"value": 1.0 / s, "unit": "steps/s", "cores": threads, "kind": kind,
                   "sample": "one full force evaluation of the same N=1,048,576 Plummer input "
                             "(reference BarnesHutSolver: serial tree build + parallel walk, "
                             "theta 0.5, monopole)"}
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": ws,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Plummer sphere, numpy PCG64)",
            "config": {"workload": workload_name(args.n), "n": args.n, "theta": THETA, "eps": EPS,
                       "dt": DT, "seed": SEED, "multipole": "monopole+quadrupole",
                       "mac": "geometric", "state": "f64", "pair_forces": "f32",
                       "parallelism": f"replicas x{ws}",
                       "l2": "inputs larger than L2 (state, sort and tree buffers > 300 MB)"},
            "interactions_per_s": inter_total / (ms_max / 1e3),
            "interactions_per_step": inter / args.steps,
            "force_error": {"mean": err[0], "max": err[1], "rms": err[2],
                            "vs": "FP64 direct sum, 4096 uniformly sampled bodies"},
            "stage_ms": {"build": build_ms / args.steps, "walk": walk_ms / args.steps,
                         "sort": sort_ms / args.steps, "tree": tree_ms / args.steps},
            "stage_gbs": {
                "sort": SORT_BYTES_PER_BODY * args.n / (sort_ms / args.steps / 1e3) / 1e9,
                "tree": TREE_BYTES_PER_BODY * args.n / (tree_ms / args.steps / 1e3) / 1e9,
                "hbm_peak": pk.get("hbm_gbs", 6458.1),
                "bytes_per_body": {"sort": SORT_BYTES_PER_BODY, "tree": TREE_BYTES_PER_BODY},
                "note": "sort = kick-drift+bbox, keys+histograms, 8 radix passes, gather; "
                        "tree = radix tree, octree mark/scan/emit, multipoles; at N=2^20 the "
                        "sort buffers (24 MB) stay in the 126 MB L2"},
            "gpu_launches": None,
            "roofline": {"bound": "fp32", "kernel": "k_walk_group", "achieved": achieved,
                         "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                         "peak_kind": f"SMs x 128 x 2 x sm_max_mhz ({pk_kind} max clock)",
                         "frac_at_median_clock": (achieved / (fp32_peak * clk["sm_mhz"] /
                                                              pk.get("sm_max_mhz", 1965.0))
                                                  if clk.get("sm_mhz") else None),
                         "traffic": traffic},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "path": "nb_compute_forces (IPhysicsComputeBackend.ComputeForces) on pinned "
                            "host arrays: H2D pos+mass+active, BH force evaluation, D2H acc"},
            "clocks": clk,
        }
    eng.close()
    return line


def launches_per_step() -> int:
    """Kernels of one device step: kick-drift-bbox, cube, keys, 8 sort passes,
    gather, zero-acc, radix tree, octree mark, block scan, octree base,
    octree emit, multipoles, walk groups, walk, kick."""
    return 1 + 1 + 1 + 8 + 1 + 1 + 6 + 1 + 1 + 1


def _timed_steps(eng, stream, steps, dt, eps, flags, dev, ws):
    """K device steps bracketed by a barrier, synchronise and CUDA events
    on the engine's stream; returns (ms over ranks' max, clocks)."""
    import torch

    clocks = Clocks(dev)
    barrier(ws)
    torch.cuda.synchronize(dev)
    clocks.start()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    eng.step(steps, dt, eps, flags)
    t1.record(stream)
    torch.cuda.synchronize(dev)
    barrier(ws)
    clk = clocks.stop()
    return max_over_ranks(ws, t0.elapsed_time(t1)), clk


def run_ds1000(args, ws, rank, local):
    """FP64 direct sum + velocity Verlet: N=1000 Plummer (scale 1 AU, 1 Msun,
    seed 0), eps 1e-4, dt 1e-3, 10,000 steps; energy drift against the CPU
    restatement of CpuParallelBackend + SoAVerletIntegrator run on the same
    input (its trajectory is bit-identical)."""
    import torch

    import oracle
    from nbody_b200 import MODE_DIRECT_FP64, Engine, scenarios

    dev = local
    torch.cuda.set_device(dev)
    n, eps, dt, steps = 1000, 1e-4, 1e-3, args.steps if args.steps != 20 else 10_000
    b = scenarios.plummer(n, 1.0, 1.0, seed=0)
    eng = Engine(n, device=dev)
    stream = torch.cuda.ExternalStream(eng.stream, device=dev)
    eng.set_state(b, old_acc=False)
    eng.step(max(args.warmup, 3), dt, eps, MODE_DIRECT_FP64)  # warm-up on a copy of the state
    eng.set_state(b, old_acc=False)
    e0 = eng.diagnostics(eps)["e"]
    ms, clk = _timed_steps(eng, stream, steps, dt, eps, MODE_DIRECT_FP64, dev, ws)
    e1 = eng.diagnostics(eps)["e"]
    drift = (e1 - e0) / abs(e0)
    line = None
    if rank == 0:
        d = {k: getattr(b, k) for k in ("px", "py", "pz", "vx", "vy", "vz", "ax", "ay", "az",
                                         "mass", "active")}
        threads = os.cpu_count() or 1
        t = time.perf_counter()
        cpu_steps = steps if not args.no_cpu_baseline else 0
        w = oracle.verlet_direct(d, eps, dt, cpu_steps, nthreads=threads) if cpu_steps else None
        cpu_s = time.perf_counter() - t
        cpu_drift = None
        if w is not None:
            w["active"] = b.active
            cpu_drift = (oracle.energy(w, eps)["e"] - oracle.energy(d, eps)["e"]) / abs(e0)
        line = {"metric": METRIC, "value": steps / (ms / 1e3), "unit": "steps/s", "n_gpus": ws,
                "steps": steps, "warmup": max(args.warmup, 3), "ms_per_step": ms / steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded Plummer sphere)",
                "config": {"workload": "ds_plummer_1000", "n": n, "eps": eps, "dt": dt,
                           "seed": 0, "force": "direct sum FP64, CpuParallelBackend rounding"},
                "energy_drift": drift, "cpu_energy_drift": cpu_drift,
                "pairs_per_s": n * (n - 1) * steps / (ms / 1e3),
                "cpu_baseline": None if w is None else {
                    "value": steps / cpu_s, "unit": "steps/s", "cores": threads, "kind": "port",
                    "sample": f"the same {steps} steps with the CpuParallelBackend restatement "
                              "(OpenMP over targets)"},
                "clocks": clk, "gpu_launches": 5 * steps}
    eng.close()
    return line


def run_disk(args, ws, rank, local):
    """Collisional disk: 262,144 bodies + a 1 Msun central body, Barnes-Hut
    theta 0.5 with shell-theorem leaves, merges (64/frame, 2/body) and
    compaction every step, eps 1e-4, dt 1e-3."""
    import torch

    from nbody_b200 import (FLAG_COLLISIONS, FLAG_SHELL_THEOREM, MODE_BARNES_HUT, Engine,
                            scenarios)
    from nbody_b200 import _native as N

    dev = local
    torch.cuda.set_device(dev)
    n, eps, dt = 262_144, 1e-4, 1e-3
    steps = args.steps if args.steps != 20 else 1000
    # radius scale 30: calibrated so ~1 % of the bodies merge per 1000 steps
    # (a scale of 1000 makes every body overlap ~3 others at the start)
    d = scenarios.collisional_disk(n, seed=2, radius_scale=DISK_RADIUS_SCALE)
    eng = Engine(n + 1, device=dev)
    eng.set_param(N.PARAM_THETA, THETA)
    stream = torch.cuda.ExternalStream(eng.stream, device=dev)
    flags = MODE_BARNES_HUT | FLAG_SHELL_THEOREM | FLAG_COLLISIONS
    eng.set_state(d, old_acc=False)
    eng.step(max(args.warmup, 3), dt, eps, flags)
    eng.set_state(d, old_acc=False)
    p0 = eng.diagnostics(eps, pe_mode=1)
    ms, clk = _timed_steps(eng, stream, steps, dt, eps, flags, dev, ws)
    p1 = eng.diagnostics(eps, pe_mode=1)
    st, ids = eng.get_state()
    line = None
    if rank == 0:
        dp = np.sqrt(sum((p1[k] - p0[k]) ** 2 for k in ("px", "py", "pz")))
        pn = np.sqrt(sum(p0[k] ** 2 for k in ("px", "py", "pz")))
        line = {"metric": METRIC, "value": steps / (ms / 1e3), "unit": "steps/s", "n_gpus": ws,
                "steps": steps, "warmup": max(args.warmup, 3), "ms_per_step": ms / steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded Keplerian disk)",
                "config": {"workload": "disk_262k", "n": n + 1, "eps": eps, "dt": dt, "seed": 2,
                           "theta": THETA, "radius_scale": DISK_RADIUS_SCALE,
                           "collisions": "broad phase + merge + compaction every step"},
                "bodies_left": int(len(ids)), "merged": int(n + 1 - len(ids)),
                "merges_per_1000_steps_frac": (n + 1 - len(ids)) / (n + 1) * 1000.0 / steps,
                "energy_drift": (p1["e"] - p0["e"]) / abs(p0["e"]),
                "momentum_drift_abs": dp, "momentum_scale": pn,
                "mass_drift": (p1["m"] - p0["m"]) / p0["m"], "clocks": clk}
    eng.close()
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--n", type=int, default=N_BODIES,
                    help="bodies (default the 1,048,576-body workload; smaller for profiling)")
    ap.add_argument("--workload", default="bh1m", choices=["bh1m", "ds1000", "disk"],
                    help="bh1m: the headline Barnes-Hut line; ds1000: FP64 direct sum N=1000, "
                         "10k steps; disk: collisional disk N=262,145, 1000 steps")
    args = ap.parse_args()
    ws, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank)
        elif args.workload == "ds1000":
            line = run_ds1000(args, ws, rank, local)
            if line is not None:
                print(json.dumps(line))
        elif args.workload == "disk":
            line = run_disk(args, ws, rank, local)
            if line is not None:
                print(json.dumps(line))
        else:
            line = run_b200(args, ws, rank, local)
            if line is not None:
                line["gpu_launches"] = launches_per_step() * args.steps
                print(json.dumps(line))
    finally:
        if ws > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
