"""Benchmark of the bundle-adjustment operator on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config cfg2] [--precision both|fp64|mixed]
                    [--impl ours|reference]

Configuration 2 (the default; 1,500 cameras / 1M points / ~6.2M observations): a step is one
bundle adjustment of the full seeded synthetic scene (typecv_b200/synthetic.py), 10 LM iterations.
``value`` is LM steps per second of the whole job in the mixed-precision form, measured on the device
with CUDA events (the library's solve time: inputs already in HBM), the max over ranks; the same
figures of the FP64 form, run on the same scene in the same process, are under ``fp64``, with the two
forms' final costs.  ``e2e`` is the same metric through the public call (``tba_bundle_adjust`` with
pinned host buffers: host checks, host-to-device copies, the solve and the device-to-host read inside
the timed region).  The working set (~1.5 GB) is larger than the 126 MB L2, so no flush is needed.
``roofline`` describes the dominant kernel, the one-pass Schur product, from CUDA-event pairs the
library records around every product launch of one more solve after the timed steps (the events
would cost the timed solves about 3%).

``--config cfg3`` runs the batched local-window solve (512 arc windows, one persistent launch) and
``--config cfg4`` the adjoint of a 200-camera / 50k-point solve; ``--config invdepth`` the
inverse-depth measurement linearisation (4M seeded measurements per call, ``tba_linearize_inverse_depth``);
``--config observations`` the evaluation and depth filtering of every observation of the configuration-2
scene at its true poses (``tba_evaluate_observations``); each prints its own line.

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
    ap.add_argument("--config", default="cfg2", choices=["cfg0", "cfg1", "cfg2", "cfg3", "cfg4", "invdepth", "observations"])
    ap.add_argument("--iterations", type=int, default=None, help="LM iterations per step")
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "mixed"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="fraction of the configuration's points (profiling)")
    ap.add_argument("--count", type=int, default=512, help="cfg3: problems in the batch")
    ap.add_argument("--fd", type=int, default=256, help="cfg4: finite-difference coordinates")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--host-pcg-loop", action="store_true",
                    help="cfg0-cfg2: PCG steps launched from the host in chunks instead of the device-side "
                         "graph loop (for profilers that do not follow conditional graph nodes)")
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
    camera and point indices (8 B); per point V_p^-1 (6 values of the factors' size: the mixed form
    reads an FP32 copy); per warp task its first observation (4 B, about one task per 28
    observations, counted per point here); the direction in world axes (6C FP64 words) and the
    per-block partial rows (prod_blocks x m values of the factors' size, written by the product and
    read by the column reduction)."""
    m = 6 * scene.C + (1 if shared else 0)
    return (scene.M * (12 * factor_bytes + 8) + scene.P * (6 * factor_bytes + 4) + 8 * 6 * scene.C
            + 2 * factor_bytes * m * prod_blocks)


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


def dram_traffic(scene, precision):
    """Per-launch DRAM bytes of k_product_f from the committed ncu summary, scaled to this scene by
    its observations (the capture ran a smaller scene; traffic grows with the observations)."""
    path = os.path.join(ROOT, "profiles", "k_product_f_traffic.json")
    try:
        d = json.load(open(path))
    except OSError:
        return None
    if precision not in d:
        return None
    return d[precision]["dram_bytes_per_observation"] * scene.M


def cpu_baseline_run(scene, iterations=1):
    """The oracle (the reference operator's algorithm in C++, OpenMP over the host cores) on
    `iterations` LM iterations of the full scene; returns (seconds, LM iterations run, threads,
    the oracle's output array)."""
    from oracle import bundle_adjust as ob
    s, i = scene.packed()
    packed = {"C": scene.C, "P": scene.P, "M": scene.M, "scene": s, "index": i}
    t0 = time.perf_counter()
    out = ob.gpu_operator_packed(packed, 0, 1, iterations=iterations, huber=2.0, shared=True)
    dt = time.perf_counter() - t0
    st = out[12 * scene.C + 3 * scene.P:]
    ran = max(1, int(st[10] + st[11]))
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return dt, ran, threads, out


def parity_against_oracle(local, scene, ref, iterations):
    """The FP64 form through tba_bundle_adjust on the same scene and options as the oracle's run
    (`ref`, `iterations` LM iterations of the reference operator's algorithm restated in C++):
    cost, RMS, accepted and rejected steps, PCG iterations, and the largest pose and point
    differences.  Measured outside every timed region."""
    import typecv_b200 as tb
    s_np, i_np = scene.packed()
    ctl = tb.make_control(scene.C, scene.P, scene.M, anchor=0, scale_view=1, iterations=iterations, shared_focal=True,
                          huber=2.0, tolerance=1e-6, precision=0)
    with tb.ShadeDevice.open(local) as dev:
        out, _ = tb.solve_packed(dev, ctl, s_np, i_np)
    C, n = scene.C, 12 * scene.C + 3 * scene.P
    g, w = out[n:], ref[n:]
    return {"against": f"the oracle (reference operator's algorithm, C++), {iterations} LM iteration(s), FP64 form",
            "final_cost_rel_diff": float(abs(g[6] - w[6]) / w[6]),
            "final_rmse_diff_px": float(abs(g[25] - w[25])),
            "accepted": [int(g[10]), int(w[10])], "rejected": [int(g[11]), int(w[11])],
            "cg_iterations": [int(g[16]), int(w[16])],
            "max_pose_diff": float(np.max(np.abs(out[:12 * C] - ref[:12 * C]))),
            "max_point_diff": float(np.max(np.abs(out[12 * C:n] - ref[12 * C:n]))),
            "log_focal_diff": float(abs(g[26] - w[26]))}


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


def _reduce_device():
    """Where the reductions' one-word tensors live: the GPU under NCCL, the host under gloo."""
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def barrier(world):
    import torch
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    if torch.cuda.is_available():
        torch.cuda.synchronize()


def _all_reduce(world, value, op):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(world, value):
    import torch.distributed as dist
    return _all_reduce(world, value, dist.ReduceOp.MAX)


def sum_over_ranks(world, value):
    import torch.distributed as dist
    return _all_reduce(world, value, dist.ReduceOp.SUM)


def finish_dist(world):
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def invdepth_cpu(rows):
    """The oracle's C++ CPU linearisation (the reference's inverseDepthJacobian, OpenMP over the host
    cores) over `rows`: (seconds, output rows, threads)."""
    from oracle import inverse_depth as oid
    oid.linearize_rows(rows[:16])
    t0 = time.perf_counter()
    out = oid.linearize_rows(rows)
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return time.perf_counter() - t0, out, threads


INVDEPTH_METRIC = "inverse-depth measurement linearisations/s, 1 B200"
INVDEPTH_UNIT = "measurements/s"
INVDEPTH_ROWS = 4 << 20


def run_reference(args, world, rank):
    if rank != 0:
        return
    if args.config == "invdepth":
        from typecv_b200 import synthetic as S
        rows = S.inverse_depth_rows(measurements=max(1, int(INVDEPTH_ROWS * args.scale)))
        for _ in range(args.warmup):
            invdepth_cpu(rows[:4096])
        total, threads = 0.0, 1
        for _ in range(args.steps):
            dt, _, threads = invdepth_cpu(rows)
            total += dt
        value = len(rows) * args.steps / total
        line = {"metric": INVDEPTH_METRIC, "value": value, "unit": INVDEPTH_UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded)",
                "config": {"workload": f"invdepth: {len(rows)} inverse-depth measurement rows"}, "impl": "reference",
                "cpu_baseline": {"value": value, "unit": INVDEPTH_UNIT, "cores": threads, "kind": "port",
                                 "sample": f"all {len(rows)} rows per step through the CPU inverseDepthJacobian "
                                           "restated in C++ (oracle/ba_oracle.cpp)"},
                "e2e": {"value": value, "unit": INVDEPTH_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    cfg = args.config if args.config in ("cfg0", "cfg1", "cfg2") else "cfg2"
    scene = make_scene(cfg, args.scale)
    for _ in range(args.warmup):
        cpu_baseline_run(scene, 1)
    times, ran, cg = [], 0, 0
    threads = 1
    n = 12 * scene.C + 3 * scene.P
    for _ in range(args.steps):
        dt, k, threads, out = cpu_baseline_run(scene, 1)
        times.append(dt)
        ran += k
        cg += int(out[n + 16])
    total = sum(times)
    value = ran / total
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": workload(scene, cfg, 1), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"1 LM iteration of the full {cfg} scene per step (the reference "
                                       "operator's algorithm restated in C++, oracle/ba_oracle.cpp)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "pcg_iterations_per_s": cg / total}
    print(json.dumps(line), flush=True)


def pinned_like(a, torch):
    if a.dtype == np.uint32:
        p = torch.empty(a.size, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    else:
        p = torch.empty(a.size, dtype=torch.float64, pin_memory=True).numpy()
    p[:] = a
    return p


def time_form(args, world, local, scene, precision, iterations):
    """Warm-up and timed solves of one form, then one solve with CUDA events around every Schur
    product (for the roofline: the events cost about 3% of the solve, so they stay out of the
    timed steps); returns (reports of the timed steps, wall times, output, clocks, the
    instrumented report)."""
    import torch
    import typecv_b200 as tb
    from typecv_b200 import _lib
    s_np, i_np = scene.packed()
    s_pin, i_pin = pinned_like(s_np, torch), pinned_like(i_np, torch)
    kw = dict(anchor=0, scale_view=1, iterations=iterations, shared_focal=True, huber=2.0, tolerance=1e-6,
              precision=precision)
    ctl = tb.make_control(scene.C, scene.P, scene.M, **kw,
                          flags=_lib.TBA_FLAG_HOST_PCG_LOOP if args.host_pcg_loop else 0)
    ctl_timed = tb.make_control(scene.C, scene.P, scene.M, **kw, flags=_lib.TBA_FLAG_TIME_PRODUCTS)
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
        result = out.copy()
        _, instrumented = tb.solve_packed(dev, ctl_timed, s_pin, i_pin, out)
    finally:
        dev.close()
    return reports, walls, result, clk, instrumented


def time_resident(args, world, local, scene, precision, iterations):
    """Row f2: the same solve through a resident scene (tba_scene_create once; per step
    tba_scene_write of the initial poses and points, then tba_scene_adjust, which reads back only the
    state words).  Returns LM steps/s end to end (host wall time) and on the device."""
    import torch
    import typecv_b200 as tb
    from typecv_b200 import _lib
    from typecv_b200.resident import ResidentScene
    s_np, i_np = scene.packed()
    C, P = scene.C, scene.P
    poses = pinned_like(np.ascontiguousarray(s_np[:12 * C]), torch)
    points = pinned_like(np.ascontiguousarray(s_np[12 * C:12 * C + 3 * P]), torch)
    ctl = tb.make_control(C, P, scene.M, anchor=0, scale_view=1, iterations=iterations, shared_focal=True,
                          huber=2.0, tolerance=1e-6, precision=precision,
                          flags=_lib.TBA_FLAG_HOST_PCG_LOOP if args.host_pcg_loop else 0)
    dev = tb.ShadeDevice.open(local)
    try:
        with ResidentScene(dev, ctl, s_np, i_np) as rs:
            for _ in range(max(args.warmup, 1)):
                rs.write(poses, points)
                rs.adjust()
            walls, reps = [], []
            barrier(world)
            for _ in range(args.steps):
                t0 = time.perf_counter()
                rs.write(poses, points)
                _, state, rep = rs.adjust()
                walls.append(time.perf_counter() - t0)
                reps.append(rep)
            barrier(world)
    finally:
        dev.close()
    lm = sum_over_ranks(world, sum(r["lm_iterations"] for r in reps))
    wall_s = max_over_ranks(world, sum(walls))
    solve_s = max_over_ranks(world, sum(r["solve_ms"] for r in reps) / 1000)
    return {"e2e": lm / wall_s, "value": lm / solve_s, "unit": UNIT, "final_cost": float(state[6]),
            "h2d_bytes_per_step": 8 * (12 * C + 3 * P), "d2h_bytes_per_step": 8 * len(state),
            "check_ms": reps[-1].get("check_ms", 0.0),
            "note": "tba_scene_write of the initial poses and points + tba_scene_adjust per step, mixed form"}


def form_summary(world, scene, reports, walls, out):
    solve_s = sum(r["solve_ms"] for r in reports) / 1000
    lm = sum(r["lm_iterations"] for r in reports)
    cg = sum(r["cg_iterations"] for r in reports)
    t_max = max_over_ranks(world, solve_s)
    lm_all = sum_over_ranks(world, lm)
    e2e_max = max_over_ranks(world, sum(walls))
    cg_all = sum_over_ranks(world, cg)
    base = 12 * scene.C + 3 * scene.P
    return {"value": lm_all / t_max, "e2e": lm_all / e2e_max, "t_max": t_max,
            "pcg_iterations_per_s": cg_all / t_max, "final_cost": float(out[base + 6]),
            "final_rmse_px": float(out[base + 25]), "lm_iterations": lm, "cg_iterations": cg,
            "refinements": sum(r.get("refinements", 0) for r in reports),
            "fp64_iterations": sum(r.get("fp64_iterations", 0) for r in reports)}


def roofline(scene, reports, precision):
    pk, pk_kind = peaks()
    prod_ms = sum(r["product_ms"] for r in reports)
    prod_n = sum(r["product_launches"] for r in reports)
    blocks = reports[-1].get("product_blocks", 0) or 1
    bytes_launch = product_bytes(scene, True, blocks, 4 if precision == "mixed" else 8)
    t_launch = prod_ms / max(prod_n, 1) / 1000
    achieved = bytes_launch / t_launch / 1e9 if prod_n else None
    kernel = "k_product_f<FP32 factors>" if precision == "mixed" else "k_product_f<FP64 factors>"
    return {"bound": "hbm", "kernel": kernel + " (one-pass Schur product S p over the stored Jacobian factors)",
            "achieved": achieved, "peak": pk["hbm_gbs"], "peak_kind": pk_kind, "unit": "GB/s",
            "frac": achieved / pk["hbm_gbs"] if achieved else None,
            "traffic": dram_traffic(scene, precision), "algorithmic_bytes": bytes_launch,
            "launch_ms": 1000 * t_launch, "launches": prod_n, "product_blocks": blocks,
            "two_pass_bytes_over_one_pass_time": two_pass_bytes(scene, True) / t_launch / 1e9 if prod_n else None}


def run_single(args, world, rank, local):
    scene = make_scene(args.config, args.scale)
    iterations = args.iterations or scene.options.get("iterations", 10)
    from typecv_b200 import _lib
    forms = ["mixed", "fp64"] if args.precision == "both" else [args.precision]
    results = {}
    for form in forms:
        prec = _lib.TBA_PRECISION_MIXED if form == "mixed" else _lib.TBA_PRECISION_FP64
        reports, walls, out, clk, instrumented = time_form(args, world, local, scene, prec, iterations)
        results[form] = (reports, walls, out, clk, form_summary(world, scene, reports, walls, out), instrumented)
    if args.config == "cfg2" and forms[0] == "mixed":
        results["resident"] = time_resident(args, world, local, scene, _lib.TBA_PRECISION_MIXED, iterations)
    if rank != 0:
        return
    head = forms[0]
    reports, walls, out, clk, summ, instrumented = results[head]
    line = {
        "metric": METRIC, "value": summ["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * summ["t_max"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if head == "fp64" else "f32+f64",
        "data": "synthetic (seeded; typecv_b200/synthetic.py)",
        "config": {**workload(scene, args.config, iterations), "precision": head, "parallelism": f"replicas x{world}",
                   "pcg_loop": "host chunks" if args.host_pcg_loop else "device graph (conditional while node)"},
        "pcg_iterations_per_s": summ["pcg_iterations_per_s"],
        "final_cost": summ["final_cost"], "final_rmse_px": summ["final_rmse_px"],
        "e2e": {"value": summ["e2e"], "unit": UNIT, "h2d_bytes_per_step": int(reports[-1]["h2d_bytes"]),
                "d2h_bytes_per_step": int(reports[-1]["d2h_bytes"])},
        "roofline": roofline(scene, [instrumented], head),
        "clocks": clk,
        "gpu_launches": sum(r["kernel_launches"] for r in reports),
    }
    if head == "mixed":
        base = 12 * scene.C + 3 * scene.P
        line["mixed"] = {"refinements": summ["refinements"], "cg_iterations": summ["cg_iterations"],
                         "fp64_iterations": summ["fp64_iterations"], "pcg_failures": int(out[base + 17])}
    if len(forms) == 2:
        r64, _, _, clk64, s64, inst64 = results["fp64"]
        line["fp64"] = {"value": s64["value"], "e2e": s64["e2e"], "pcg_iterations_per_s": s64["pcg_iterations_per_s"],
                        "final_cost": s64["final_cost"], "final_rmse_px": s64["final_rmse_px"],
                        "roofline": roofline(scene, [inst64], "fp64"), "clocks": clk64,
                        "gpu_launches": sum(r["kernel_launches"] for r in r64)}
        out64 = results["fp64"][2]
        n = 12 * scene.C + 3 * scene.P
        line["mixed_vs_fp64"] = {"lm_steps_ratio": summ["value"] / s64["value"],
                                 "final_cost_rel_diff": abs(summ["final_cost"] - s64["final_cost"]) / s64["final_cost"],
                                 "max_pose_diff": float(np.max(np.abs(out[:12 * scene.C] - out64[:12 * scene.C]))),
                                 "max_point_diff": float(np.max(np.abs(out[12 * scene.C:n] - out64[12 * scene.C:n]))),
                                 "final_rmse_diff_px": abs(summ["final_rmse_px"] - s64["final_rmse_px"])}
        line["fp64"]["pcg"] = {"iterations": s64["cg_iterations"], "failures": int(out64[n + 17])}
    if head == "mixed" or len(forms) == 2:
        line["resident"] = results.get("resident")
    if world == 1 and not args.no_cpu_baseline:
        dt, ran, threads, ref = cpu_baseline_run(scene, 1)
        cg = int(ref[12 * scene.C + 3 * scene.P + 16])
        line["cpu_baseline"] = {"value": ran / dt, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"1 LM iteration of the full {args.config} scene, {dt:.1f} s (the "
                                          "reference operator's algorithm restated in C++, oracle/ba_oracle.cpp)",
                                # The first LM iteration's PCG steps against the solve's average: the
                                # same comparison per PCG iteration.
                                "pcg_iterations": cg, "pcg_iterations_per_s": cg / dt}
        line["parity"] = parity_against_oracle(local, scene, ref, 1)
    print(json.dumps(line), flush=True)


def run_batch(args, world, rank, local):
    """Configuration 3: 512 arc windows (C 5-40, P log-uniform 500-20k, tracks 2-10), 10 LM
    iterations each, one persistent launch per batch, against one grid-engine call per problem."""
    import torch
    import typecv_b200 as tb
    from typecv_b200 import batch as B
    from typecv_b200 import synthetic as S
    scenes = S.batch_scenes(count=args.count)
    probs = [B.PackedProblem(s.C, s.P, s.M, *s.packed(), s.anchor, s.scale_view) for s in scenes]
    n_scene = sum(p.scene.size for p in probs)
    n_index = sum(p.index.size for p in probs)
    s_pin = torch.empty(n_scene, dtype=torch.float64, pin_memory=True).numpy()
    i_pin = torch.empty(n_index, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    packed = B.pack_batch(probs, False, scene=s_pin, index=i_pin)
    out = torch.empty(packed.output_len, dtype=torch.float64, pin_memory=True).numpy()
    iterations, max_cg = 10, 256
    dev = tb.ShadeDevice.open(local)
    res = {}
    try:
        for prec in ("mixed", "fp64"):
            tune = None
            for _ in range(max(args.warmup, 1)):
                _, rep = B.batch_adjust(dev, packed, iterations=iterations, precision=prec, max_cg=max_cg, output=out)
                tune = tune or rep
            reps, walls = [], []
            barrier(world)
            with Clocks(local) as clocks:
                for _ in range(args.steps):
                    t0 = time.perf_counter()
                    recs, rep = B.batch_adjust(dev, packed, iterations=iterations, precision=prec, max_cg=max_cg,
                                               output=out)
                    walls.append(time.perf_counter() - t0)
                    reps.append(rep)
                barrier(world)
            res[prec] = (reps, walls, [r.copy() for r in recs], clocks.summary(), tune)
        # The mixed form's own kernel at the tuned shape (a forced schedule keeps the requested form),
        # beside whichever form the tuner chose for the headline.
        forced = res["mixed"][4]["schedule"] + 1
        B.batch_adjust(dev, packed, iterations=iterations, precision="mixed", max_cg=max_cg, output=out, schedule=forced)
        mixed_kernel = []
        for _ in range(args.steps):
            _, rep = B.batch_adjust(dev, packed, iterations=iterations, precision="mixed", max_cg=max_cg, output=out,
                                    schedule=forced)
            mixed_kernel.append(rep)
        mixed_kernel_recs = [r.copy() for r in B.batch_adjust(dev, packed, iterations=iterations, precision="mixed",
                                                                max_cg=max_cg, output=out, schedule=forced)[0]]
        seq_ms, seq = 0.0, []
        for sc, p in zip(scenes, probs):
            ctl = tb.make_control(sc.C, sc.P, sc.M, anchor=0, scale_view=1, iterations=iterations, max_cg=max_cg)
            o, rep = tb.solve_packed(dev, ctl, p.scene, p.index)
            seq_ms += rep["solve_ms"]
            seq.append(o.copy())
    finally:
        dev.close()
    reps, walls, recs, clk, tune = res["mixed"]
    solve_s = max_over_ranks(world, sum(r["solve_ms"] for r in reps) / 1000)
    lm = sum_over_ranks(world, sum(r["lm_iterations"] for r in reps))
    wall_s = max_over_ranks(world, sum(walls))
    if rank != 0:
        return

    def worst(records):
        w = 0.0
        for sc, a, b in zip(scenes, records, seq):
            base = 12 * sc.C + 3 * sc.P
            w = max(w, abs(a[base + 6] - b[base + 6]) / b[base + 6])
        return w

    r64 = res["fp64"][0]
    lm_seq = sum(int(o[12 * s.C + 3 * s.P + 10] + o[12 * s.C + 3 * s.P + 11]) for s, o in zip(scenes, seq))
    line = {"metric": "batched local-window BA: LM steps/s over the batch (one persistent launch)",
            "value": lm / solve_s, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * solve_s / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if reps[-1].get("form", 1) == 1 else "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": f"cfg3: {len(scenes)} arc windows, {sum(s.C for s in scenes)} cameras / "
                                   f"{sum(s.P for s in scenes)} points / {sum(s.M for s in scenes)} observations in "
                                   f"total, 10 LM iterations each, PCG tolerance 1e-6 (max 256), mixed precision",
                       "l2": "working set larger than L2"},
            "problems_per_s": world * len(scenes) * args.steps / solve_s,
            "e2e": {"value": lm / wall_s, "unit": UNIT, "h2d_bytes_per_step": int(reps[-1]["h2d_bytes"]),
                    "d2h_bytes_per_step": int(reps[-1]["d2h_bytes"])},
            "schedule": {"shape": reps[-1]["schedule"], "threads": reps[-1]["threads"], "blocks": reps[-1]["blocks"],
                         "tune_ms": tune["tune_ms"], "graph_replayed": reps[-1]["graph_replayed"],
                         "form": "mixed" if reps[-1].get("form", 1) == 1 else "fp64",
                         "note": "a mixed request runs the form the autotuner timed faster for this batch shape"},
            "mixed_kernel": {"value": sum(r["lm_iterations"] for r in mixed_kernel) /
                                      (sum(r["solve_ms"] for r in mixed_kernel) / 1000),
                             "worst_cost_rel_vs_sequential": worst(mixed_kernel_recs),
                             "note": "the mixed form itself (FP32 product, FP64 refinement), forced at the same shape"},
            "fp64_batch": {"value": sum(r["lm_iterations"] for r in r64) / (sum(r["solve_ms"] for r in r64) / 1000),
                           "worst_cost_rel_vs_sequential": worst(res["fp64"][2])},
            "mixed_worst_cost_rel_vs_sequential": worst(recs),
            "sequential_fp64": {"value": lm_seq / (seq_ms / 1000), "solve_ms": seq_ms,
                                "note": "the same problems, one tba_bundle_adjust call each (grid engine, FP64)"},
            "clocks": clk, "gpu_launches": sum(r["kernel_launches"] for r in reps)}
    line["speedup_vs_sequential_fp64"] = line["value"] / line["sequential_fp64"]["value"]
    print(json.dumps(line), flush=True)


def run_adjoint(args, world, rank, local):
    """Configuration 4: the vector-Jacobian product of the converged 200-camera / 50k-point solve
    (configuration 1's generator), and its central-difference check on `--fd` pixel coordinates
    (h = 1e-6 px) of the same configuration without outliers."""
    import typecv_b200 as tb
    from typecv_b200 import adjoint as AD
    from typecv_b200 import synthetic as S

    def solved(dev, sc):
        s, i = sc.packed()
        ctl = tb.make_control(sc.C, sc.P, sc.M, anchor=0, scale_view=1, iterations=30, shared_focal=True,
                              tolerance=1e-10, max_cg=256)
        out, _ = tb.solve_packed(dev, ctl, s, i)
        n = 12 * sc.C + 3 * sc.P
        s2 = s.copy()
        s2[:n] = out[:n]
        s2[n:n + 6 * sc.C].reshape(sc.C, 6)[:, :2] *= np.exp(out[n + 26])
        return s2, i

    dev = tb.ShadeDevice.open(local)
    try:
        # The configuration-1 scene with its outliers: the solve, then the adjoint at that solution.
        sc = S.helix_scene(seed=24, cameras=200, points=50_000)
        s, i = solved(dev, sc)
        g = np.random.default_rng(6).normal(size=12 * sc.C + 3 * sc.P)
        g /= np.linalg.norm(g)
        _, _, _, rep_out = AD.bundle_vjp(dev, sc.C, sc.P, sc.M, s, i, g)
        # Without the outliers: Newton steps to a stationary point, the timed products there, and the
        # central differences.
        clean = S.helix_scene(seed=24, cameras=200, points=50_000, outlier_rate=0.0)
        cs, ci = solved(dev, clean)
        ybar, kbar, sol, rep_fd = AD.bundle_vjp(dev, clean.C, clean.P, clean.M, cs, ci, g, newton_steps=6,
                                                want_solution=True)
        base = cs.copy()
        base[:sol.size] = sol
        for _ in range(max(args.warmup, 1)):
            AD.bundle_vjp(dev, clean.C, clean.P, clean.M, base, ci, g)
        times, reps = [], []
        with Clocks(local) as clocks:
            for _ in range(args.steps):
                t0 = time.perf_counter()
                _, _, _, rep = AD.bundle_vjp(dev, clean.C, clean.P, clean.M, base, ci, g)
                times.append(time.perf_counter() - t0)
                reps.append(rep)
        clk = clocks.summary()
        # One more product with CUDA events around every one-pass Schur product (roofline).
        _, _, _, rep_t = AD.bundle_vjp(dev, clean.C, clean.P, clean.M, base, ci, g, time_products=True)
        # The CPU baseline: the dense FP64 reference gradient (oracle/adjoint_dense.py) on the
        # 10-camera / 500-point subproblem, beside the device on the same subproblem.
        from oracle.adjoint_dense import Problem
        small = S.helix_scene(seed=22, cameras=10, points=500)
        ss, si = solved(dev, small)
        gs = np.random.default_rng(5).normal(size=12 * small.C + 3 * small.P)
        gs /= np.linalg.norm(gs)
        ys, _, sols, _ = AD.bundle_vjp(dev, small.C, small.P, small.M, ss, si, gs, newton_steps=4, want_solution=True)
        sbase = ss.copy()
        sbase[:sols.size] = sols
        _, _, _, rep_small = AD.bundle_vjp(dev, small.C, small.P, small.M, sbase, si, gs)
        t0 = time.perf_counter()
        ys_dense, _ = Problem(small.C, small.P, small.M, sbase, si).vjp(gs)
        dense_s = time.perf_counter() - t0
        dense_rel = float(np.linalg.norm(ys.ravel() - ys_dense.ravel()) / np.linalg.norm(ys_dense))
        coords = np.random.default_rng(7).choice(2 * clean.M, args.fd, replace=False)
        off = 18 * clean.C + 3 * clean.P
        h = 1e-6
        fd = np.zeros(coords.size)
        t0 = time.perf_counter()
        for n, k in enumerate(coords):
            sp, sm = base.copy(), base.copy()
            sp[off + k] += h
            sm[off + k] -= h
            tp, _ = AD.newton_solution(dev, clean.C, clean.P, clean.M, sp, ci, steps=2)
            tm, _ = AD.newton_solution(dev, clean.C, clean.P, clean.M, sm, ci, steps=2)
            fd[n] = g @ (tp - tm) / (2 * h)
        fd_s = time.perf_counter() - t0
    finally:
        dev.close()
    if rank != 0:
        return
    an = ybar.ravel()[coords]
    scale = float(np.max(np.abs(an)))
    err = np.abs(fd - an)
    solve_ms = statistics.median(r["solve_ms"] for r in reps)
    line = {"metric": "BA adjoint: vector-Jacobian products of the converged solve per second",
            "value": 1000.0 / solve_ms, "unit": "vjp/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": solve_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": f"cfg4: {clean.C} cameras / {clean.P} points / {clean.M} observations "
                                   "(configuration 1's generator without its 3% outliers), solved with the shared "
                                   "focal refined and then fixed, Newton steps to a stationary point; unit random "
                                   "cotangent on poses and points; exact Hessian, PCG tolerance 1e-12"},
            "e2e": {"value": args.steps / sum(times), "unit": "vjp/s",
                    "h2d_bytes_per_step": int(base.nbytes + ci.nbytes + g.nbytes),
                    "d2h_bytes_per_step": 16 * clean.M + 16},
            "adjoint_cg_iterations": reps[-1]["cg_iterations"], "adjoint_residual": reps[-1]["adjoint_residual"],
            "gradient_norm_at_point": reps[-1]["gradient_norm_initial"], "failed_bits": reps[-1]["failed"],
            "fd_check": {"coordinates": int(args.fd), "h_px": h,
                         "median_abs_err_over_max": float(np.median(err) / scale),
                         "max_abs_err_over_max": float(np.max(err) / scale),
                         "median_rel_err": float(np.median(err / np.maximum(np.abs(an), 1e-3 * scale))),
                         "newton_gradient_norm": rep_fd["gradient_norm_final"], "seconds": fd_s},
            "with_outliers": {"observations": sc.M, "gradient_norm_at_lm_solution": rep_out["gradient_norm_initial"],
                              "point_blocks_shifted": rep_out["point_failures"], "failed_bits": rep_out["failed"],
                              "adjoint_residual": rep_out["adjoint_residual"]},
            "clocks": clk, "gpu_launches": sum(r["kernel_launches"] for r in reps)}
    # The dominant kernel: the one-pass exact-Hessian Schur product k_adj_product.  Per launch: per
    # observation its 18-word cross block and camera and point index (152 B); per point V_p^-1
    # (6 words) and its task's first observation (counted per point, 4 B); the direction (6C
    # words); the per-block partial rows (6C words each, written here and read by k_adj_columns).
    pk, pk_kind = peaks()
    blocks = rep_t.get("product_blocks", 0)
    if rep_t.get("product_launches", 0) and blocks:
        nbytes = clean.M * (18 * 8 + 8) + clean.P * (6 * 8 + 4) + 8 * 6 * clean.C + 2 * 8 * 6 * clean.C * blocks
        t_launch = rep_t["product_ms"] / rep_t["product_launches"] / 1000
        achieved = nbytes / t_launch / 1e9
        line["roofline"] = {"bound": "hbm", "kernel": "k_adj_product (one-pass exact-Hessian Schur product)",
                            "achieved": achieved, "peak": pk["hbm_gbs"], "peak_kind": pk_kind, "unit": "GB/s",
                            "frac": achieved / pk["hbm_gbs"], "traffic": None, "algorithmic_bytes": nbytes,
                            "launch_ms": 1000 * t_launch, "launches": rep_t["product_launches"],
                            "product_blocks": blocks}
    line["cpu_baseline"] = {"value": 1.0 / dense_s, "unit": "vjp/s", "cores": os.cpu_count() or 1, "kind": "port",
                            "sample": f"one vjp of the 10-camera / 500-point subproblem ({small.M} observations) by "
                                      f"the dense FP64 reference gradient (oracle/adjoint_dense.py, numpy with its BLAS threads: Hessian by "
                                      f"central differences, KKT solve), {dense_s:.1f} s; a smaller workload than "
                                      "the line's, so no ratio to `value` is implied",
                            "device_same_subproblem_vjp_per_s": 1000.0 / rep_small["solve_ms"],
                            "device_vs_dense_rel_err": dense_rel}
    print(json.dumps(line), flush=True)


def run_inverse_depth(args, world, rank, local):
    """Row f4: one tba_linearize_inverse_depth call over 4M seeded measurement rows per step (scaled
    by --scale), pinned host buffers.  ``value`` from the kernel's CUDA events, ``e2e`` from the
    call's wall time (host-to-device copy of the rows, the kernel, the read of the results)."""
    import torch
    import ctypes
    import typecv_b200 as tb
    from typecv_b200 import _lib
    from typecv_b200 import synthetic as S
    M = max(1, int(INVDEPTH_ROWS * args.scale))
    rows = S.inverse_depth_rows(measurements=M)
    src = torch.empty(34 * M, dtype=torch.float64, pin_memory=True).numpy()
    src[:] = rows.ravel()
    dst = torch.empty(23 * M, dtype=torch.float64, pin_memory=True).numpy()
    lib = _lib.load()
    dev = tb.ShadeDevice.open(local)

    def call():
        rep = _lib.ObservationReport()
        st = lib.tba_linearize_inverse_depth(dev.handle, M, _lib.dptr(src), src.size, _lib.dptr(dst), dst.size,
                                             ctypes.byref(rep))
        if st != _lib.TBA_OK:
            raise RuntimeError(lib.tba_last_error(dev.handle).decode())
        return rep.as_dict()

    try:
        for _ in range(max(3, args.warmup)):
            call()
        reps, walls = [], []
        barrier(world)
        with Clocks(local) as clocks:
            for _ in range(args.steps):
                t0 = time.perf_counter()
                reps.append(call())
                walls.append(time.perf_counter() - t0)
            barrier(world)
        joint = joint_inverse_depth(dev, args) if rank == 0 else None
    finally:
        dev.close()
    kernel_s = max_over_ranks(world, sum(r["evaluate_ms"] for r in reps) / 1000)
    wall_s = max_over_ranks(world, sum(walls))
    if rank != 0:
        return
    # Every row against the oracle (flags equal, values within 1e-8 of max(1, |value|)).
    dt, want, threads = invdepth_cpu(rows)
    got = dst.reshape(M, 23)
    flags_equal = bool(np.array_equal(want[:, 0], got[:, 0]))
    ok = want[:, 0] == 1
    worst = float(np.max(np.abs(want[ok] - got[ok]) / np.maximum(1, np.abs(want[ok])))) if ok.any() else 0.0
    invalid = int(M - ok.sum())
    pk, kind = peaks()
    per_launch_s = kernel_s / args.steps
    achieved = 456 * M / per_launch_s / 1e9
    cpu = None
    if not args.no_cpu_baseline:
        cpu = {"value": M / dt, "unit": INVDEPTH_UNIT, "cores": threads, "kind": "port",
               "sample": f"all {M} rows through the CPU inverseDepthJacobian restated in C++ "
                         "(oracle/ba_oracle.cpp, OpenMP)"}
    line = {"metric": INVDEPTH_METRIC, "value": world * M * args.steps / kernel_s, "unit": INVDEPTH_UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": max(3, args.warmup),
            "ms_per_step": 1000 * kernel_s / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": f"invdepth: {M} inverse-depth measurement rows (34 words in, 23 out), "
                                   "512 ring cameras, one call per step",
                       "l2": "working set (1.9 GB at 4M rows) larger than L2"},
            "e2e": {"value": world * M * args.steps / wall_s, "unit": INVDEPTH_UNIT,
                    "h2d_bytes_per_step": int(reps[-1]["h2d_bytes"]), "d2h_bytes_per_step": int(reps[-1]["d2h_bytes"]),
                    "upload_ms": reps[-1]["upload_ms"], "download_ms": reps[-1]["download_ms"]},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / pk["hbm_gbs"], "traffic": None,
                         "note": f"k_linearize_inverse_depth, 456 algorithmic bytes per measurement; peak of {kind}"},
            "parity": {"rows_checked": M, "flags_equal": flags_equal, "max_rel_vs_oracle": worst,
                       "invalid_rows": invalid},
            "cpu_baseline": cpu, "clocks": clocks.summary(), "gpu_launches": sum(r["kernel_launches"] for r in reps),
            "joint": joint}
    print(json.dumps(line), flush=True)


def joint_inverse_depth(dev, args, iterations=4):
    """The joint inverse-depth bundle adjustment (bundleAdjustInverseDepthGpu) on the seeded
    120-view corridor: wall time of the call (device linearisations and projections, host FP64
    steps), its device time and launches; beside it, unless --no-cpu-baseline, the oracle's loop
    restatement of the reference's CPU bundleAdjustInverseDepth on the same input."""
    from typecv_b200 import synthetic as S
    from typecv_b200.inverse_depth_bundle import bundle_adjust_inverse_depth_gpu
    inp = S.inverse_depth_corridor()
    bundle_adjust_inverse_depth_gpu(dev, inp, [], {"iterations": 1})
    # The median of three calls (the host steps' time varies by tens of milliseconds between calls).
    walls = []
    for _ in range(3):
        t0 = time.perf_counter()
        got = bundle_adjust_inverse_depth_gpu(dev, inp, [], {"iterations": iterations})
        walls.append(time.perf_counter() - t0)
    wall = float(np.median(walls))
    d = got["diagnostics"]
    out = {"workload": "inverse_depth_corridor: 120 views, 1404 tracks of 4 views, 5616 measurements, "
                       f"{iterations} LM iterations", "ms": 1000 * wall, "ms_note": "median of three calls",
           "device_ms": d["deviceMs"],
           "gpu_launches": d["kernelLaunches"], "camera_parameters": d["cameraParameters"],
           "linear_solver": d["linearSolver"], "initial_cost": d["initialCost"], "final_cost": d["finalCost"],
           "accepted_steps": d["acceptedSteps"]}
    if not args.no_cpu_baseline:
        from oracle import inverse_depth as oid
        from typecv_b200.inverse_depth_bundle import drive, inverse_depth_bundle_steps
        # CPU baseline: the same array-wise host steps, every linearisation and projection answered
        # on the host by the C++ restatement of the CPU inverseDepthJacobian (OpenMP).
        def cpu_call(k):
            return drive(inverse_depth_bundle_steps(inp, [], {"iterations": k}),
                         lambda job: oid.linearize_rows(np.asarray(job["rows"]).reshape(-1, 34)))
        cpu_call(1)
        cpu_walls = []
        for _ in range(3):
            t0 = time.perf_counter()
            cpu = cpu_call(iterations)
            cpu_walls.append(time.perf_counter() - t0)
        out["cpu_baseline"] = {"ms": 1000 * float(np.median(cpu_walls)), "kind": "port",
                               "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)),
                               "sample": "the whole call on the host, median of three after one warm-up call: the "
                                         "same array-wise FP64 steps, linearisations by the C++ CPU "
                                         "inverseDepthJacobian (OpenMP)"}
        out["final_cost_rel_diff_vs_cpu_baseline"] = abs(d["finalCost"] - cpu["diagnostics"]["finalCost"]) / \
            cpu["diagnostics"]["finalCost"]
        # The oracle's loop-for-loop restatement of the reference's CPU steps: a parity check of the
        # result, not a timing baseline (its time is a Python loop's).
        want = oid.bundle_adjust_inverse_depth(inp, [], {"iterations": iterations})
        out["final_cost_rel_diff_vs_loop_restatement"] = abs(d["finalCost"] - want["diagnostics"]["finalCost"]) / \
            want["diagnostics"]["finalCost"]
    return out


def observation_request(scene, limit=0.05, noise=1.0, max_error=3.0):
    """The packed arrays of tba_evaluate_observations for the scene at its true poses and points."""
    cams = np.ascontiguousarray(np.concatenate([scene.truth_poses, scene.truth_cameras], axis=1).ravel())
    idx = np.empty(2 * scene.M, dtype=np.uint32)
    idx[0::2] = scene.obs_camera
    idx[1::2] = scene.obs_point
    offsets = np.searchsorted(scene.obs_point, np.arange(scene.P + 1)).astype(np.uint32)
    return {"cameras": cams, "points": np.ascontiguousarray(scene.truth_points.ravel()),
            "pixels": np.ascontiguousarray(scene.pixels.ravel()), "indices": idx, "offsets": offsets,
            "count": scene.M, "P": scene.P, "C": scene.C, "guarded": limit > 0, "limit": limit, "noise": noise,
            "max_error": max_error}


def run_observations(args, world, rank, local):
    """Row f3: one tba_evaluate_observations call over every observation of the configuration-2
    scene at its true state per step (3 px threshold, relative depth bound 0.05 at 1 px noise),
    pinned host buffers.  ``value`` from the kernels' CUDA events, ``e2e`` from the call's wall time."""
    import ctypes
    import torch
    import typecv_b200 as tb
    from typecv_b200 import _lib
    scene = make_scene("cfg2", args.scale)
    req = observation_request(scene)
    C, P, M = scene.C, scene.P, scene.M

    def pinned(a):
        p = pinned_like(a, torch)
        p[:] = a
        return p

    arrs = {k: pinned(req[k]) for k in ("cameras", "points", "pixels", "indices", "offsets")}
    flags = pinned_like(np.zeros(M + P, dtype=np.uint32), torch)
    summary = np.zeros(2)
    lib = _lib.load()
    dev = tb.ShadeDevice.open(local)
    ctl = _lib.ObservationControl(C, P, M, 0, req["max_error"], req["limit"], req["noise"])

    def call():
        rep = _lib.ObservationReport()
        st = lib.tba_evaluate_observations(dev.handle, ctypes.byref(ctl), _lib.dptr(arrs["cameras"]), arrs["cameras"].size,
                                           _lib.dptr(arrs["points"]), arrs["points"].size, _lib.dptr(arrs["pixels"]),
                                           arrs["pixels"].size, _lib.uptr(arrs["indices"]), arrs["indices"].size,
                                           _lib.uptr(arrs["offsets"]), arrs["offsets"].size, _lib.uptr(flags),
                                           flags.size, _lib.dptr(summary), ctypes.byref(rep))
        if st != _lib.TBA_OK:
            raise RuntimeError(lib.tba_last_error(dev.handle).decode())
        return rep.as_dict()

    try:
        for _ in range(max(3, args.warmup)):
            call()
        reps, walls = [], []
        barrier(world)
        with Clocks(local) as clocks:
            for _ in range(args.steps):
                t0 = time.perf_counter()
                reps.append(call())
                walls.append(time.perf_counter() - t0)
            barrier(world)
    finally:
        dev.close()
    kernel_s = max_over_ranks(world, sum(r["evaluate_ms"] for r in reps) / 1000)
    wall_s = max_over_ranks(world, sum(walls))
    if rank != 0:
        return
    # Every flag against the oracle (the restated kernels in C++, OpenMP over the host cores).
    from oracle import observations as oo
    oo.evaluate_cpp({**req, "count": 64, "P": 1, "offsets": req["offsets"][:2]})
    t0 = time.perf_counter()
    want = oo.evaluate_cpp(req)
    cpu_s = time.perf_counter() - t0
    mismatches = int(np.sum(want["flags"] != flags[:M + P]))
    summary_rel = abs(want["summary"][0] - summary[0]) / max(abs(want["summary"][0]), 1e-300)
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    pk, kind = peaks()
    per_launch_s = kernel_s / args.steps
    algorithmic = 56 * M + 32 * P + 144 * C
    achieved = algorithmic / per_launch_s / 1e9
    line = {"metric": "observation evaluation and depth filtering: observations/s, 1 B200",
            "value": world * M * args.steps / kernel_s, "unit": "observations/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": 1000 * kernel_s / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": f"observations: cfg2 scene at its true state, {C} cameras / {P} points / {M} "
                                   "observations, 3 px threshold, relative depth bound 0.05 at 1 px noise",
                       "l2": "working set larger than L2"},
            "inliers": float(summary[1]), "mean_error_px": float(summary[0] / max(summary[1], 1)),
            "depth_rejected_tracks": int(np.sum(flags[M:M + P])),
            "e2e": {"value": world * M * args.steps / wall_s, "unit": "observations/s",
                    "h2d_bytes_per_step": int(reps[-1]["h2d_bytes"]), "d2h_bytes_per_step": int(reps[-1]["d2h_bytes"]),
                    "upload_ms": reps[-1]["upload_ms"], "download_ms": reps[-1]["download_ms"]},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / pk["hbm_gbs"], "traffic": None,
                         "note": "the whole evaluation (projection, depth filter, partials, summary: "
                                 f"{reps[-1]['kernel_launches']} launches) against 56 B per observation + 32 B per "
                                 f"point + 144 B per camera; peak of {kind}"},
            "parity": {"observations_checked": M, "tracks_checked": P, "flag_mismatches": mismatches,
                       "inlier_count_equal": bool(want["summary"][1] == summary[1]),
                       "error_sum_rel_diff": summary_rel},
            "cpu_baseline": {"value": M / cpu_s, "unit": "observations/s", "cores": threads, "kind": "port",
                             "sample": "every observation of the scene through the restated kernels in C++ "
                                       "(oracle/ba_oracle.cpp, OpenMP)"},
            "clocks": clocks.summary(), "gpu_launches": sum(r["kernel_launches"] for r in reps)}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world, rank, local = init_dist(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        elif args.config == "cfg3":
            run_batch(args, world, rank, local)
        elif args.config == "cfg4":
            run_adjoint(args, world, rank, local)
        elif args.config == "invdepth":
            run_inverse_depth(args, world, rank, local)
        elif args.config == "observations":
            run_observations(args, world, rank, local)
        else:
            run_single(args, world, rank, local)
    finally:
        finish_dist(world)


if __name__ == "__main__":
    main()
