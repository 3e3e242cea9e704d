"""Benchmark of the bundle-adjustment operator on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config cfg2] [--impl ours|reference]

A step is one bundle adjustment of the configuration's full synthetic scene (seeded; see
typecv_b200/synthetic.py), ``--iterations`` LM iterations.  ``value`` is LM steps per second of the
whole job, measured on the device with CUDA events (the library's solve time: inputs already in
HBM), the max over ranks; ``e2e`` is the same metric through the public call
(``tba_bundle_adjust`` with pinned host buffers: host checks, host-to-device copies, the solve and
the device-to-host read inside the timed region).  The working set of configuration 2 (~1.5 GB)
is larger than L2, so no flush is needed between steps.

Multi-GPU runs are replicas (the operator does not shard): each rank solves its own copy of the
scene, no collective touches the data path, and ``scaling`` is "weak".

``--impl reference`` times the reference operator's algorithm as the oracle restates it in C++
(oracle/ba_oracle.cpp, OpenMP over the host cores; the reference itself is TypeScript and needs
Node, absent here): each step is one LM iteration of the same scene (a bounded sample).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import signal
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "BA LM steps/s & Schur matvec HBM GB/s, mixed vs FP64 at equal final cost, 1 B200"
UNIT = "LM steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="cfg2", choices=["cfg0", "cfg1", "cfg2"])
    ap.add_argument("--iterations", type=int, default=None, help="LM iterations per step")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="fraction of the configuration's points (profiling)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def make_scene(config, scale=1.0):
    from typecv_b200 import synthetic as S
    if config == "cfg0":
        return S.ring_scene(points=max(50, int(2000 * scale)))
    if config == "cfg1":
        return S.helix_scene(points=max(1000, int(100_000 * scale)))
    return S.sphere_scene(points=max(1000, int(1_000_000 * scale)))


def workload(scene, config, iterations):
    return {"workload": f"{config}: {scene.C} cameras / {scene.P} points / {scene.M} observations, shared focal, "
                        f"{iterations} LM iterations per step, PCG tolerance 1e-6, Huber 2 px",
            "cameras": scene.C, "points": scene.P, "observations": scene.M, "lm_iterations_per_step": iterations,
            "l2": "working set larger than the 126 MB L2; no flush"}


def product_bytes(scene, shared, prod_blocks, factor_bytes=8):
    """Algorithmic DRAM bytes of one launch of the one-pass Schur product k_product_f: per
    observation its 12 stored Jacobian factors (8 B each in FP64, 4 B in the mixed form) and its
    camera and point index (8 B); per point V_p^-1 (6 words) and its offset (4 B); the direction
    vector p (m words) and the per-block partial rows (prod_blocks x m words, written)."""
    m = 6 * scene.C + (1 if shared else 0)
    return scene.M * (12 * factor_bytes + 8) + scene.P * (6 * 8 + 4) + 8 * m + 8 * m * prod_blocks


def two_pass_bytes(scene, shared):
    """The two-pass Schur product's algorithmic bytes (W read twice, y written and read)."""
    s = 8
    b = scene.M * (2 * 18 * s + 2 * 4) + scene.P * (6 * s + 2 * 3 * s) + scene.C * (21 * s + 12 * s)
    return b + (scene.M * 2 * 3 * s if shared else 0)


class Clocks:
    """nvidia-smi samples of the SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.file = tempfile.NamedTemporaryFile(prefix="clocks", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.send_signal(signal.SIGTERM)
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.file.close()

    def summary(self):
        rows = []
        for line in open(self.file.name).read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 9:
                rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": float(rows[0][2]),
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def dram_traffic(scene, shared):
    """Per-launch DRAM bytes of k_product from the committed ncu summary, scaled to this scene by
    its observations (the capture ran a smaller scene; traffic grows with the observations)."""
    path = os.path.join(ROOT, "profiles", "k_product_traffic.json")
    try:
        d = json.load(open(path))
    except OSError:
        return None
    key = "shared" if shared else "fixed"
    if key not in d:
        return None
    return d[key]["dram_bytes_per_observation"] * scene.M


def cpu_baseline_run(scene, iterations=1):
    """The oracle (the reference operator's algorithm in C++, OpenMP over the host cores) on
    `iterations` LM iterations of the full scene; returns (seconds, LM iterations run, threads)."""
    from oracle import bundle_adjust as ob
    s, i = scene.packed()
    packed = {"C": scene.C, "P": scene.P, "M": scene.M, "scene": s, "index": i}
    t0 = time.perf_counter()
    out = ob.gpu_operator_packed(packed, 0, 1, iterations=iterations, huber=2.0, shared=True)
    dt = time.perf_counter() - t0
    st = out[12 * scene.C + 3 * scene.P:]
    ran = max(1, int(st[10] + st[11]))
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return dt, ran, threads


def init_dist(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    import torch
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()


def max_over_ranks(world, value):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(world, value):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def run_reference(args, world, rank):
    if rank != 0:
        return
    scene = make_scene(args.config, args.scale)
    for _ in range(args.warmup):
        cpu_baseline_run(scene, 1)
    times, ran = [], 0
    threads = 1
    for _ in range(args.steps):
        dt, k, threads = cpu_baseline_run(scene, 1)
        times.append(dt)
        ran += k
    total = sum(times)
    value = ran / total
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": workload(scene, args.config, 1), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"1 LM iteration of the full {args.config} scene per step (the reference "
                                       "operator's algorithm restated in C++, oracle/ba_oracle.cpp)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world, rank, local = init_dist(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    import torch
    import typecv_b200 as tb
    from typecv_b200 import _lib

    scene = make_scene(args.config, args.scale)
    iterations = args.iterations or scene.options.get("iterations", 10)
    shared = True
    s_np, i_np = scene.packed()
    # pinned host buffers for the end-to-end path
    s_pin = torch.empty(s_np.size, dtype=torch.float64, pin_memory=True).numpy()
    i_pin = torch.empty(i_np.size, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    s_pin[:] = s_np
    i_pin[:] = i_np
    precision = _lib.TBA_PRECISION_MIXED if args.precision == "mixed" else _lib.TBA_PRECISION_FP64
    ctl = tb.make_control(scene.C, scene.P, scene.M, anchor=0, scale_view=1, iterations=iterations,
                          shared_focal=shared, huber=2.0, tolerance=1e-6, precision=precision,
                          flags=_lib.TBA_FLAG_TIME_PRODUCTS)
    out = torch.empty(12 * scene.C + 3 * scene.P + 27, dtype=torch.float64, pin_memory=True).numpy()
    dev = tb.ShadeDevice.open(local)
    try:
        for _ in range(max(args.warmup, 0)):
            tb.solve_packed(dev, ctl, s_pin, i_pin, out)
        reports, walls = [], []
        barrier(world)
        with Clocks(local) as clocks:
            for _ in range(args.steps):
                t0 = time.perf_counter()
                _, rep = tb.solve_packed(dev, ctl, s_pin, i_pin, out)
                walls.append(time.perf_counter() - t0)
                reports.append(rep)
            barrier(world)
        clk = clocks.summary()
    finally:
        dev.close()
    solve_s = sum(r["solve_ms"] for r in reports) / 1000
    lm = sum(r["lm_iterations"] for r in reports)
    cg = sum(r["cg_iterations"] for r in reports)
    t_max = max_over_ranks(world, solve_s)
    lm_all = sum_over_ranks(world, lm)
    e2e_max = max_over_ranks(world, sum(walls))
    base = 12 * scene.C + 3 * scene.P
    final_cost, final_rmse = float(out[base + 6]), float(out[base + 25])
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    pk, pk_kind = peaks()
    prod_ms = sum(r["product_ms"] for r in reports)
    prod_n = sum(r["product_launches"] for r in reports)
    n_sms = torch.cuda.get_device_properties(local).multi_processor_count
    prod_blocks = n_sms  # one 512-thread block per SM (the product kernel's occupancy)
    bytes_launch = product_bytes(scene, shared, prod_blocks, 4 if args.precision == "mixed" else 8)
    t_launch = prod_ms / max(prod_n, 1) / 1000
    achieved = bytes_launch / t_launch / 1e9 if prod_n else None
    traffic = dram_traffic(scene, shared)
    line = {
        "metric": METRIC, "value": lm_all / t_max, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * t_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
        "data": "synthetic (seeded; typecv_b200/synthetic.py)",
        "config": {**workload(scene, args.config, iterations), "precision": args.precision,
                   "parallelism": f"replicas x{world}"},
        "pcg_iterations_per_s": sum_over_ranks(world, cg) / t_max if world > 1 else cg / t_max,
        "final_cost": final_cost, "final_rmse_px": final_rmse,
        "e2e": {"value": lm_all / e2e_max, "unit": UNIT, "h2d_bytes_per_step": int(reports[-1]["h2d_bytes"]),
                "d2h_bytes_per_step": int(reports[-1]["d2h_bytes"])},
        "roofline": {"bound": "hbm", "kernel": "k_product_f (one-pass Schur product S p over stored Jacobian factors)",
                     "achieved": achieved, "peak": pk["hbm_gbs"], "peak_kind": pk_kind, "unit": "GB/s",
                     "frac": achieved / pk["hbm_gbs"] if achieved else None,
                     "traffic": traffic, "algorithmic_bytes": bytes_launch,
                     "launch_ms": 1000 * t_launch, "launches": prod_n,
                     "two_pass_equivalent_gbs": two_pass_bytes(scene, shared) / t_launch / 1e9 if prod_n else None},
        "clocks": clk,
        "gpu_launches": sum(r["kernel_launches"] for r in reports),
    }
    if world == 1 and not args.no_cpu_baseline:
        dt, ran, threads = cpu_baseline_run(scene, 1)
        line["cpu_baseline"] = {"value": ran / dt, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"1 LM iteration of the full {args.config} scene, {dt:.1f} s (the "
                                          "reference operator's algorithm restated in C++, oracle/ba_oracle.cpp)"}
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
