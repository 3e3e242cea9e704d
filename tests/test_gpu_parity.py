"""Parity of the CUDA operator (libtba.so, through its C ABI) with the oracle.

* the reference's recorded GPU results on its own fixtures (tests/golden/reference_records.json);
* the reference GPU operator's algorithm restated on the CPU (oracle.gpu_operator), same inputs;
* the reference's CPU bundle adjustment (oracle.cpu_bundle_adjust, exact dense solve) at a tight
  PCG tolerance: final robust cost within 1e-9 relative and RMS within 1e-6 px;
* the reference's own test assertions (tests/typeshade/cpu.test.mjs, focal.test.mjs) on the
  GPU result, and edge cases: zero iterations, rejected solves, windows, bearings, long tracks.
"""
import json
import math
import os

import numpy as np
import pytest

import typecv_b200 as tb
from typecv_b200 import _lib
from typecv_b200 import synthetic as S
from oracle import bundle_adjust as ob
from reference_cases import bundle_fixture, bundle_metrics, joint_focal_fixture, skew_bundle_fixture

pytestmark = pytest.mark.gpu

RECORDS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_records.json")))["records"]
COST_REL = 1e-9   # final robust cost, FP64 form
RMS_PX = 1e-6     # reprojection RMS, FP64 form


@pytest.fixture(scope="module")
def device():
    dev = tb.ShadeDevice.open(0)
    yield dev
    dev.close()


def record_fixture(rec):
    f = rec["fixture"]
    return skew_bundle_fixture(f["views"], f["count"]) if f["skew"] else bundle_fixture(views=f["views"], count=f["count"])


@pytest.mark.parametrize("rec", RECORDS, ids=lambda r: r["name"] + "/" + str(r["options"]["iterations"]))
def test_reproduces_reference_gpu_records(device, rec):
    out = tb.bundle_adjust_gpu(device, record_fixture(rec), rec["options"])
    serial = rec["variants"][0]
    costs = [v["finalCost"] for v in rec["variants"]]
    cg = [v["cgIterations"] for v in rec["variants"]]
    final = out["diagnostics"]["finalCost"]
    assert abs(final - serial["finalCost"]) <= COST_REL * serial["finalCost"], (final, serial)
    assert min(costs) * (1 - 1e-10) <= final <= max(costs) * (1 + 1e-10)
    assert min(cg) - 2 <= out["cgIterations"] <= max(cg) + 2
    assert out["linearSolverFailures"] == 0


def _compare_operator(device, model, options, pose_tol=1e-7):
    got = tb.bundle_adjust_gpu(device, model, options)
    want = ob.gpu_operator(model, options)
    gd, wd = got["diagnostics"], want["diagnostics"]
    assert abs(gd["initialCost"] - wd["initialCost"]) <= 1e-12 * wd["initialCost"]
    assert abs(gd["finalCost"] - wd["finalCost"]) <= COST_REL * max(wd["finalCost"], 1e-300) + 1e-18
    assert abs(gd["finalRmsePx"] - wd["finalRmsePx"]) <= RMS_PX
    assert gd["acceptedSteps"] == wd["acceptedSteps"] and gd["rejectedSteps"] == wd["rejectedSteps"]
    for a, b in zip(got["reconstruction"]["views"], want["reconstruction"]["views"]):
        assert np.max(np.abs(np.asarray(a["pose"]["t"]) - b["pose"]["t"])) < pose_tol
        assert np.max(np.abs(np.asarray(a["pose"]["R"]) - b["pose"]["R"])) < pose_tol
        assert abs(a["camera"]["fx"] - b["camera"]["fx"]) <= 1e-9 * b["camera"]["fx"]
    return got, want


@pytest.mark.parametrize("options", [
    {"iterations": 15, "huberPx": 1},
    {"iterations": 15, "huberPx": 1, "refineSharedFocal": True},
    {"iterations": 10, "variableViewIds": [30, 40]},
    {"iterations": 5, "variableViewIds": []},
    {"iterations": 12, "cgRelativeTolerance": 1e-10, "maxCgIterations": 200, "stallTolerance": 1e-4},
])
def test_matches_operator_oracle_on_reference_fixture(device, options):
    for settings in ({}, {"outlier": True}, {"shift": (7, -3, 2)}):
        model = bundle_fixture(**settings)
        opts = dict(options)
        if "shift" in settings and "variableViewIds" not in opts:
            opts.update(anchorViewId=20, scaleViewId=40)
        _compare_operator(device, model, opts)


def test_cpu_tier_assertions(device):
    # tests/typeshade/cpu.test.mjs:533-607 on the CUDA operator.
    for settings in ({}, {"outlier": True}, {"shift": (7, -3, 2)}):
        inp = bundle_fixture(**settings)
        snapshot = json.dumps([list(map(float, p["xyz"])) for p in inp["landmarks"]])
        initial = bundle_metrics(inp, 1)
        shifted = "shift" in settings
        anchor, scale_view = (1, 3) if shifted else (0, 1)
        r = tb.bundle_adjust_gpu(device, inp, {"iterations": 15, "huberPx": 1,
                                               **({"anchorViewId": 20, "scaleViewId": 40} if shifted else {})})
        actual = bundle_metrics(r["reconstruction"], 1)
        assert r["diagnostics"]["acceptedSteps"] > 0
        assert actual["cost"] < initial["cost"] * 0.05
        assert abs(actual["cost"] - r["diagnostics"]["finalCost"]) < 1e-6
        assert json.dumps([list(map(float, p["xyz"])) for p in inp["landmarks"]]) == snapshot
        v = r["reconstruction"]["views"][anchor]["pose"]
        assert np.array_equal(v["R"], inp["views"][anchor]["pose"]["R"]) and np.array_equal(v["t"], inp["views"][anchor]["pose"]["t"])
        a = ob.camera_center(r["reconstruction"]["views"][anchor]["pose"])
        b = ob.camera_center(r["reconstruction"]["views"][scale_view]["pose"])
        assert abs(np.linalg.norm(a - b) - r["diagnostics"]["baseline"]) < 1e-9
        assert actual["observations"] == 160
        assert r["execution"]["cpuStages"] == []
    inp = bundle_fixture()
    local = tb.bundle_adjust_gpu(device, inp, {"iterations": 10, "variableViewIds": [30, 40]})
    assert local["diagnostics"]["finalCost"] < local["diagnostics"]["initialCost"]
    for i in (0, 1):
        assert np.array_equal(local["reconstruction"]["views"][i]["pose"]["t"], inp["views"][i]["pose"]["t"])
    unchanged = tb.bundle_adjust_gpu(device, inp, {"iterations": 0})
    for a, b in zip(unchanged["reconstruction"]["landmarks"], inp["landmarks"]):
        assert np.array_equal(a["xyz"], b["xyz"])
    points_only = tb.bundle_adjust_gpu(device, inp, {"iterations": 5, "variableViewIds": []})
    assert points_only["diagnostics"]["finalCost"] < points_only["diagnostics"]["initialCost"]
    for a, b in zip(points_only["reconstruction"]["views"], inp["views"]):
        assert np.array_equal(a["pose"]["t"], b["pose"]["t"])
    rejected = tb.bundle_adjust_gpu(device, inp, {"iterations": 1, "maxCgIterations": 1, "cgRelativeTolerance": 1e-12})
    assert rejected["diagnostics"]["acceptedSteps"] == 0 and rejected["linearSolverFailures"] > 0
    for a, b in zip(rejected["reconstruction"]["landmarks"], inp["landmarks"]):
        assert np.array_equal(a["xyz"], b["xyz"])
    zero = {**inp, "views": [{**v, "pose": inp["views"][0]["pose"]} if i == 1 else v for i, v in enumerate(inp["views"])]}
    with pytest.raises(tb.RangeError, match="baseline"):
        tb.bundle_adjust_gpu(device, zero, {"iterations": 0})
    behind = {**inp, "landmarks": [{**p, "xyz": np.array([0.0, 0, -5])} if i == 0 else p for i, p in enumerate(inp["landmarks"])]}
    with pytest.raises(tb.RangeError, match="in front"):
        tb.bundle_adjust_gpu(device, behind, {"iterations": 0})


FOCAL = {"iterations": 40, "refineSharedFocal": True, "maxCgIterations": 256, "cgRelativeTolerance": 1e-10}


def test_joint_focal_recovers_truth_and_matches_cpu_reference(device):
    # tests/typeshade/focal.test.mjs:13-45
    jf = joint_focal_fixture()
    inp, truth = jf["input"], jf["truth"]
    expected = ob.cpu_bundle_adjust(inp, FOCAL)
    actual = tb.bundle_adjust_gpu(device, inp, FOCAL)
    d = actual["diagnostics"]
    assert d["finalCost"] < 1e-7 and d["finalRmsePx"] < 1e-4 and d["initialCost"] > 50000
    views = actual["reconstruction"]["views"]
    scale = views[0]["camera"]["fx"] / inp["views"][0]["camera"]["fx"]
    assert abs(views[0]["camera"]["fx"] - truth["views"][0]["camera"]["fx"]) < 0.001
    for v, v0 in zip(views, inp["views"]):
        assert abs(v["camera"]["fx"] / v0["camera"]["fx"] - scale) < 1e-12
        assert abs(v["camera"]["fy"] / v0["camera"]["fy"] - scale) < 1e-12
        assert v["camera"]["k1"] == v0["camera"]["k1"] and v["camera"]["k2"] == v0["camera"]["k2"]
    assert np.array_equal(views[0]["pose"]["R"], inp["views"][0]["pose"]["R"])
    assert abs(actual["diagnostics"]["finalCost"] - expected["diagnostics"]["finalCost"]) < 1e-7


def test_joint_focal_zero_iterations_and_fixed_poses(device):
    # tests/typeshade/focal.test.mjs:47-71
    inp = joint_focal_fixture(points=20, views=4)["input"]
    zero = tb.bundle_adjust_gpu(device, inp, {**FOCAL, "iterations": 0})
    assert zero["diagnostics"]["finalCost"] == zero["diagnostics"]["initialCost"]
    assert zero["diagnostics"]["acceptedSteps"] == 0
    for a, b in zip(zero["reconstruction"]["views"], inp["views"]):
        assert a["camera"] == b["camera"] and np.array_equal(a["pose"]["R"], b["pose"]["R"])
    local = tb.bundle_adjust_gpu(device, inp, {**FOCAL, "iterations": 15, "variableViewIds": []})
    assert local["diagnostics"]["finalCost"] < local["diagnostics"]["initialCost"]
    for a, b in zip(local["reconstruction"]["views"], inp["views"]):
        assert np.array_equal(a["pose"]["t"], b["pose"]["t"])
    assert local["reconstruction"]["views"][0]["camera"]["fx"] > inp["views"][0]["camera"]["fx"]


@pytest.mark.parametrize("shared", [True, False])
def test_synthetic_ring_matches_cpu_reference(device, shared):
    # Configuration 0 (10 cameras / 2,000 points), tight PCG: the exact dense CPU solve.
    scene = S.ring_scene()
    rec = scene.as_reconstruction()
    opts = {"iterations": 20, "huberPx": 2.0, "refineSharedFocal": shared, "cgRelativeTolerance": 1e-12,
            "maxCgIterations": 256}
    got = tb.bundle_adjust_gpu(device, rec, opts)
    want = ob.cpu_bundle_adjust(rec, opts)
    gd, wd = got["diagnostics"], want["diagnostics"]
    assert abs(gd["finalCost"] - wd["finalCost"]) <= COST_REL * wd["finalCost"], (gd, wd)
    assert abs(gd["finalRmsePx"] - wd["finalRmsePx"]) <= RMS_PX
    # 3% uniform outliers keep the Huber cost high; the inliers converge.
    assert gd["finalCost"] < gd["initialCost"] and gd["acceptedSteps"] > 0


def test_helix_full_size_matches_cpu_reference(device):
    # Configuration 1 at its full size: 200 cameras on a 3-lap helix, 100k points each in 3-12
    # cameras (751,555 observations), shared focal, PCG tolerance 1e-12 with a budget of 256, against
    # the exact dense CPU bundle adjustment (bundle-adjustment.ts:80-291, joint-focal.ts:45-287; a
    # 1,201-unknown reduced system per iteration).  Ten LM iterations: beyond them the reference
    # operator's own algorithm (the oracle's restatement, same budget) starts to fail PCG solves
    # that do not reach 1e-12 in 256 iterations and rejects steps the exact solve accepts; by 30
    # iterations it has failed 7 and ends 6.9e-5 above the CPU cost, so no implementation of the
    # operator matches the CPU solve there.  Over these ten both take 7 steps and reject 3, and the
    # oracle's operator ends within 3.2e-14 of the CPU cost.
    scene = S.helix_scene()
    assert (scene.C, scene.P) == (200, 100_000) and scene.M > 700_000
    rec = scene.as_reconstruction()
    opts = {"iterations": 10, "huberPx": 2.0, "refineSharedFocal": True, "cgRelativeTolerance": 1e-12,
            "maxCgIterations": 256}
    got = tb.bundle_adjust_gpu(device, rec, opts)
    want = ob.cpu_bundle_adjust(rec, opts)
    gd, wd = got["diagnostics"], want["diagnostics"]
    assert abs(gd["initialCost"] - wd["initialCost"]) <= 1e-12 * wd["initialCost"]
    assert abs(gd["finalCost"] - wd["finalCost"]) <= COST_REL * wd["finalCost"], (gd, wd)
    assert abs(gd["finalRmsePx"] - wd["finalRmsePx"]) <= RMS_PX, (gd, wd)
    assert gd["acceptedSteps"] == wd["acceptedSteps"] and gd["rejectedSteps"] == wd["rejectedSteps"]
    fx = [v["camera"]["fx"] for v in got["reconstruction"]["views"]]
    fx_ref = [v["camera"]["fx"] for v in want["reconstruction"]["views"]]
    assert np.max(np.abs(np.asarray(fx) / np.asarray(fx_ref) - 1)) < 1e-9


def test_long_tracks_and_skewed_cameras(device):
    # Points seen by more than 32 cameras take the multi-round warp path.
    scene = S.ring_scene(seed=3, cameras=40, points=200)
    assert np.bincount(scene.obs_point).max() > 32
    rec = scene.as_reconstruction()
    for shared in (False, True):
        _compare_operator(device, rec, {"iterations": 6, "refineSharedFocal": shared}, pose_tol=1e-6)
    _compare_operator(device, skew_bundle_fixture(17, 512), {"iterations": 3, "maxCgIterations": 96})


def test_directional_constraints(device):
    inp = bundle_fixture()
    direction = {"trackId": 1000, "direction": np.array([0.1, 0.05, 1.0]),
                 "observations": [{"viewId": 10, "featureId": 500, "pixel": [560.0, 300.0]},
                                  {"viewId": 20, "featureId": 500, "pixel": [548.0, 301.0]}]}
    opts = {"iterations": 8, "directionalConstraints": [direction]}
    got = tb.bundle_adjust_gpu(device, inp, opts)
    want = ob.gpu_operator(inp, opts)
    assert abs(got["diagnostics"]["finalCost"] - want["diagnostics"]["finalCost"]) <= COST_REL * want["diagnostics"]["finalCost"]
    d = got["directionalConstraints"][0]["direction"]
    assert abs(np.linalg.norm(d) - 1) < 1e-12
    assert np.max(np.abs(d - want["directionalConstraints"][0]["direction"])) < 1e-7
    assert got["diagnostics"]["pointParameters"] == 3 * 40 + 2


def test_helix_midsize_matches_operator_oracle(device):
    scene = S.helix_scene(cameras=40, points=4000)
    s, i = scene.packed()
    for shared in (True, False):
        ctl = tb.make_control(scene.C, scene.P, scene.M, anchor=0, scale_view=1, iterations=6, shared_focal=shared)
        out, rep = tb.solve_packed(device, ctl, s, i)
        packed = {"C": scene.C, "P": scene.P, "M": scene.M, "scene": s, "index": i}
        ref = ob.gpu_operator_packed(packed, 0, 1, iterations=6, huber=2.0, max_cg=ctl.max_cg, shared=shared)
        base = 12 * scene.C + 3 * scene.P
        assert abs(out[base + 6] - ref[base + 6]) <= COST_REL * ref[base + 6]
        assert abs(out[base + 16] - ref[base + 16]) <= 2 * 6
        assert rep["lm_iterations"] >= 1


MIXED_REL = 1e-6  # mixed form: final cost against the FP64 form and the FP64 oracle


@pytest.mark.parametrize("kind", ["ring", "helix"])
def test_mixed_precision_reaches_the_fp64_cost(device, kind):
    # The mixed form (FP32 Jacobian factors and Schur product inside the FP64 LM loop; each PCG
    # solution refined by its FP64 residual, and finished on the FP64 product when the FP32 run
    # stops short) has no reference counterpart; it is held to the FP64 form and to the FP64
    # oracle on the same inputs.
    scene = S.ring_scene(seed=11) if kind == "ring" else S.helix_scene(cameras=40, points=4000)
    s, i = scene.packed()
    packed = {"C": scene.C, "P": scene.P, "M": scene.M, "scene": s, "index": i}
    base = 12 * scene.C + 3 * scene.P
    for shared in (True, False):
        kw = dict(anchor=0, scale_view=1, iterations=10, shared_focal=shared, tolerance=1e-8, max_cg=200)
        o64, _ = tb.solve_packed(device, tb.make_control(scene.C, scene.P, scene.M, precision=0, **kw), s, i)
        o32, rep = tb.solve_packed(device, tb.make_control(scene.C, scene.P, scene.M, precision=1, **kw), s, i)
        ref = ob.gpu_operator_packed(packed, 0, 1, iterations=10, huber=2.0, max_cg=200, tolerance=1e-8, shared=shared)
        c64, c32, cr = o64[base + 6], o32[base + 6], ref[base + 6]
        assert abs(c32 - c64) <= MIXED_REL * c64, (c32, c64)
        assert abs(c32 - cr) <= MIXED_REL * cr, (c32, cr)
        assert o32[base + 10] > 0 and o32[base + 17] == 0
        assert np.max(np.abs(o32[:12 * scene.C] - o64[:12 * scene.C])) < 1e-5


@pytest.mark.parametrize("kind", ["ring", "helix"])
def test_schur_product_error_against_the_fp64_two_pass_product(device, kind):
    # On the first PCG direction of the first LM iteration, S p from the solve's own product against
    # the FP64 two-pass product (Jacobians recomputed from poses, points and pixels): the FP64
    # one-pass product over stored factors differs by rounding only; the mixed form's FP32 product
    # (FP32 factors, FP32 warp segment sums, FP64 sums across segments) by its FP32 error, which the
    # FP64 refinement of each PCG solution then removes.
    scene = S.ring_scene(seed=11) if kind == "ring" else S.helix_scene(cameras=40, points=4000)
    s, i = scene.packed()
    errors = {}
    for precision in (0, 1):
        for shared in (True, False):
            ctl = tb.make_control(scene.C, scene.P, scene.M, anchor=0, scale_view=1, iterations=2,
                                  shared_focal=shared, tolerance=1e-8, max_cg=200, precision=precision,
                                  flags=_lib.TBA_FLAG_PRODUCT_ERROR)
            _, rep = tb.solve_packed(device, ctl, s, i)
            errors[(precision, shared)] = (rep["product_error_max"], rep["product_error_norm"])
    print(f"{kind}: product error (max, norm) {errors}")
    for shared in (True, False):
        fp64_max, fp64_norm = errors[(0, shared)]
        mixed_max, mixed_norm = errors[(1, shared)]
        assert fp64_max < 1e-12 and fp64_norm < 1e-12, errors
        assert 0 < mixed_norm < 1e-5 and mixed_max < 1e-4, errors


def test_mixed_precision_through_the_operator(device):
    jf = joint_focal_fixture()
    inp = jf["input"]
    mixed = tb.bundle_adjust_gpu(device, inp, FOCAL, precision="mixed")
    fp64 = tb.bundle_adjust_gpu(device, inp, FOCAL)
    assert mixed["diagnostics"]["finalCost"] < 1e-7 and mixed["diagnostics"]["finalRmsePx"] < 1e-4
    assert abs(mixed["reconstruction"]["views"][0]["camera"]["fx"] - jf["truth"]["views"][0]["camera"]["fx"]) < 0.001
    assert abs(mixed["diagnostics"]["finalCost"] - fp64["diagnostics"]["finalCost"]) < 1e-7


@pytest.mark.parametrize("precision", [0, 1])
def test_device_pcg_loop_matches_the_host_chunked_loop(device, precision):
    # Each PCG run is one launch of a CUDA graph whose while node repeats the PCG step until the PCG
    # stops or its budget is spent; with product timing on, the host issues the same steps in
    # guarded chunks instead (also on request, without the events).  Both run the same kernels in the
    # same order; the products' camera sums
    # are atomic adds, whose order varies from run to run, so the results agree to the rounding that
    # a PCG stopped at its tolerance carries through the LM iterations.  A second solve with the same
    # launch parameters launches the graph built by the first.
    scene = S.helix_scene(cameras=40, points=4000)
    s, i = scene.packed()
    base = 12 * scene.C + 3 * scene.P
    cost_rel, pose_abs = (1e-12, 1e-6) if precision == 0 else (MIXED_REL, 1e-5)
    for shared in (True, False):
        kw = dict(anchor=0, scale_view=1, iterations=6, shared_focal=shared, tolerance=1e-8, max_cg=200,
                  precision=precision)
        chunked, rc = tb.solve_packed(device, tb.make_control(scene.C, scene.P, scene.M,
                                                              flags=_lib.TBA_FLAG_TIME_PRODUCTS, **kw), s, i)
        graph, rg = tb.solve_packed(device, tb.make_control(scene.C, scene.P, scene.M, **kw), s, i)
        again, ra = tb.solve_packed(device, tb.make_control(scene.C, scene.P, scene.M, **kw), s, i)
        host, rh = tb.solve_packed(device, tb.make_control(scene.C, scene.P, scene.M,
                                                           flags=_lib.TBA_FLAG_HOST_PCG_LOOP, **kw), s, i)
        assert rc["product_launches"] > 0 and rg["product_launches"] == 0 and ra["product_launches"] == 0
        assert rh["product_launches"] == 0
        for out, rep in ((graph, rg), (again, ra), (host, rh)):
            assert abs(out[base + 6] - chunked[base + 6]) <= cost_rel * chunked[base + 6]
            assert np.max(np.abs(out[:12 * scene.C] - chunked[:12 * scene.C])) < pose_abs
            assert rep["lm_iterations"] == rc["lm_iterations"]
            if precision == 0:  # the mixed form's restarts turn rounding into whole PCG runs
                assert abs(rep["cg_iterations"] - rc["cg_iterations"]) <= rc["lm_iterations"]
        if precision == 0:
            # The budget: with 3 PCG steps a solve, the loop stops at its budget, not at convergence.
            budget = dict(kw, max_cg=3)
            _, rb = tb.solve_packed(device, tb.make_control(scene.C, scene.P, scene.M, **budget), s, i)
            _, rbc = tb.solve_packed(device, tb.make_control(scene.C, scene.P, scene.M,
                                                             flags=_lib.TBA_FLAG_TIME_PRODUCTS, **budget), s, i)
            assert rb["lm_iterations"] == rbc["lm_iterations"] > 0
            assert 0 < rb["cg_iterations"] == rbc["cg_iterations"] <= 3 * rb["lm_iterations"]


def test_beyond_the_shared_memory_limit_the_two_pass_engine_matches_the_oracle(device):
    # 5,000 cameras: 30,000+ camera unknowns do not fit one block's shared memory, so the engine
    # takes the two-pass recompute product (report engine 1) in both forms.
    scene = S.helix_scene(seed=31, cameras=5000, points=20000, laps=12, pitch=0.3)
    s, i = scene.packed()
    packed = {"C": scene.C, "P": scene.P, "M": scene.M, "scene": s, "index": i}
    ctl = tb.make_control(scene.C, scene.P, scene.M, anchor=0, scale_view=1, iterations=3, shared_focal=True)
    out, rep = tb.solve_packed(device, ctl, s, i)
    assert rep["engine"] == 1 and rep["product_blocks"] == 0
    ref = ob.gpu_operator_packed(packed, 0, 1, iterations=3, huber=2.0, max_cg=ctl.max_cg, shared=True)
    base = 12 * scene.C + 3 * scene.P
    assert abs(out[base + 6] - ref[base + 6]) <= COST_REL * ref[base + 6]
    assert abs(out[base + 16] - ref[base + 16]) <= 2 * 3
    ctl_m = tb.make_control(scene.C, scene.P, scene.M, anchor=0, scale_view=1, iterations=3, shared_focal=True,
                            precision=tb._lib.TBA_PRECISION_MIXED)
    out_m, rep_m = tb.solve_packed(device, ctl_m, s, i)
    assert rep_m["engine"] == 1
    assert abs(out_m[base + 6] - out[base + 6]) <= COST_REL * out[base + 6]


@pytest.mark.parametrize("name", ["all-fixed", "local", "all-fixed-shared", "local-shared", "global"])
def test_fixed_camera_observations_still_optimize_points_and_focal(device, name):
    # fixedJacobianCases / assertFixedJacobianCases (tests/typeshade/bundle-fixed-jacobian-cases.mjs:3-128).
    import copy
    local = name.startswith("local")
    model = bundle_fixture(count=24, views=6, outlier=local)
    shared = name.endswith("shared")
    if shared:
        model = {**model, "views": [{**v, "camera": {**v["camera"], "fx": v["camera"]["fx"] * 0.97,
                                                     "fy": v["camera"]["fy"] * 0.97}} for v in model["views"]]}
    variable_ids = None if name == "global" else ([v["id"] for v in model["views"][-2:]] if local else [])
    variable = set(variable_ids if variable_ids is not None else [v["id"] for v in model["views"][1:]])
    fixed_obs = sum(1 for p in model["landmarks"] for o in p["observations"] if o["viewId"] not in variable)
    options = {"iterations": 3, "huberPx": 2, "refineSharedFocal": shared}
    if variable_ids is not None:
        options["variableViewIds"] = variable_ids
    before = copy.deepcopy(model)
    result = tb.bundle_adjust_gpu(device, model, options)
    assert repr(model) == repr(before)
    moved = {v["id"]: v for v in result["reconstruction"]["views"]}
    for v in model["views"]:
        if v["id"] not in variable:
            assert np.array_equal(np.asarray(moved[v["id"]]["pose"]["R"]), np.asarray(v["pose"]["R"]))
            assert np.array_equal(np.asarray(moved[v["id"]]["pose"]["t"]), np.asarray(v["pose"]["t"]))
    d = result["diagnostics"]
    assert d["acceptedSteps"] > 0 and d["finalCost"] < d["initialCost"] and fixed_obs > 0
    ratio = result["reconstruction"]["views"][0]["camera"]["fx"] / model["views"][0]["camera"]["fx"]
    if shared:
        assert abs(ratio - 1) > 1e-6
    else:
        assert ratio == 1
