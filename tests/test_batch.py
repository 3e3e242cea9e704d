"""The batched local-window solver (tba_batch_adjust) against one-call-per-problem solves.

Each problem of a batch must get the result record that ``tba_bundle_adjust`` (the grid engine)
gives for the same packed arrays and options, and that the oracle's restatement of the reference
GPU operator gives: final robust cost within 1e-9 relative in FP64, within 1e-6 in the mixed form.
The problems are arc windows of uneven sizes (configuration 3's generator at smaller sizes).
"""
import numpy as np
import pytest

import typecv_b200 as tb
from typecv_b200 import batch as B
from typecv_b200 import synthetic as S
from oracle import bundle_adjust as ob

pytestmark = pytest.mark.gpu

COST_REL = 1e-9
MIXED_REL = 1e-6


@pytest.fixture(scope="module")
def device():
    dev = tb.ShadeDevice.open(0)
    yield dev
    dev.close()


@pytest.fixture(scope="module")
def windows():
    sizes = [(5, 300), (40, 2500), (12, 900), (27, 4000), (8, 500), (33, 1200), (19, 3000), (6, 2000), (40, 700)]
    scenes = [S.arc_scene(seed=100 + k, cameras=c, points=p) for k, (c, p) in enumerate(sizes)]
    return scenes, [problem(s) for s in scenes]


def problem(scene):
    s, i = scene.packed()
    return B.PackedProblem(scene.C, scene.P, scene.M, s, i, scene.anchor, scene.scale_view)


def single(device, scene, *, iterations, shared, precision=0, max_cg=None, tolerance=1e-6):
    s, i = scene.packed()
    ctl = tb.make_control(scene.C, scene.P, scene.M, anchor=scene.anchor, scale_view=scene.scale_view,
                          iterations=iterations, shared_focal=shared, max_cg=max_cg, tolerance=tolerance,
                          precision=precision)
    out, _ = tb.solve_packed(device, ctl, s, i)
    return out


def base(scene):
    return 12 * scene.C + 3 * scene.P


@pytest.mark.parametrize("shared", [False, True])
def test_batch_fp64_matches_one_call_per_problem(device, windows, shared):
    scenes, probs = windows
    max_cg = 200
    recs, rep = B.batch_adjust(device, probs, iterations=8, shared_focal=shared, precision="fp64", max_cg=max_cg)
    assert rep["problems"] == len(scenes) and rep["blocks"] >= 1
    for sc, rec in zip(scenes, recs):
        want = single(device, sc, iterations=8, shared=shared, max_cg=max_cg)
        b = base(sc)
        assert rec.size == want.size
        assert abs(rec[b + 6] - want[b + 6]) <= COST_REL * want[b + 6], (sc.name, rec[b + 6], want[b + 6])
        assert abs(rec[b + 25] - want[b + 25]) <= 1e-6
        assert rec[b + 10] == want[b + 10] and rec[b + 11] == want[b + 11]  # accepted, rejected
        assert abs(rec[b + 16] - want[b + 16]) <= 2 * 8  # CG steps: summation order only
        assert rec[b + 14] == 0 and rec[b + 17] == want[b + 17]
        assert np.max(np.abs(rec[:12 * sc.C] - want[:12 * sc.C])) < 1e-7
        if shared:
            assert abs(rec[b + 26] - want[b + 26]) < 1e-9


def test_batch_fp64_matches_the_operator_oracle(device, windows):
    scenes, probs = windows
    pick = [0, 2, 4]
    recs, _ = B.batch_adjust(device, [probs[k] for k in pick], iterations=6, shared_focal=True, precision="fp64",
                             max_cg=200)
    for k, rec in zip(pick, recs):
        sc = scenes[k]
        s, i = sc.packed()
        packed = {"C": sc.C, "P": sc.P, "M": sc.M, "scene": s, "index": i}
        ref = ob.gpu_operator_packed(packed, sc.anchor, sc.scale_view, iterations=6, huber=2.0, max_cg=200,
                                     shared=True)
        b = base(sc)
        assert abs(rec[b + 6] - ref[b + 6]) <= COST_REL * ref[b + 6]
        assert rec[b + 10] == ref[b + 10]


@pytest.mark.parametrize("shared", [False, True])
def test_batch_mixed_reaches_the_fp64_cost(device, windows, shared):
    scenes, probs = windows
    recs, rep = B.batch_adjust(device, probs, iterations=10, shared_focal=shared, precision="mixed", max_cg=200)
    for sc, rec in zip(scenes, recs):
        want = single(device, sc, iterations=10, shared=shared, max_cg=200)
        b = base(sc)
        assert abs(rec[b + 6] - want[b + 6]) <= MIXED_REL * want[b + 6], (sc.name, rec[b + 6], want[b + 6])
        assert rec[b + 17] == 0
        assert np.max(np.abs(rec[:12 * sc.C] - want[:12 * sc.C])) < 1e-5
    assert rep["cg_iterations"] > 0 and rep["lm_iterations"] > 0


def test_every_launch_shape_gives_the_same_solution(device, windows):
    scenes, probs = windows
    first = None
    for k in range(len(B.batch_shapes())):
        recs, rep = B.batch_adjust(device, probs[:5], iterations=5, precision="fp64", schedule=k + 1, max_cg=200)
        assert rep["schedule"] == k and rep["tune_ms"] == 0
        if first is None:
            first = recs
            continue
        for sc, a, b in zip(scenes, recs, first):
            assert abs(a[base(sc) + 6] - b[base(sc) + 6]) <= COST_REL * b[base(sc) + 6]


def test_autotuner_caches_and_graph_replays(device, windows):
    _, probs = windows
    packed = B.pack_batch(probs, False)
    r1, rep1 = B.batch_adjust(device, packed, iterations=4, precision="mixed")
    r2, rep2 = B.batch_adjust(device, packed, iterations=4, precision="mixed")
    assert rep2["tune_ms"] == 0 and rep2["schedule"] == rep1["schedule"]
    assert rep2["graph_replayed"] == 1
    for sc, a, b in zip(windows[0], r1, r2):
        assert abs(a[base(sc) + 6] - b[base(sc) + 6]) <= COST_REL * b[base(sc) + 6]


def test_input_errors_stay_with_their_problem(device, windows):
    scenes, probs = windows
    bad = S.arc_scene(seed=7, cameras=6, points=400)
    s, i = bad.packed()
    s = s.copy()
    s[12 * 1:12 * 2] = s[0:12]  # scale camera on top of the anchor: zero gauge baseline
    bad_p = B.PackedProblem(bad.C, bad.P, bad.M, s, i, 0, 1)
    recs, _ = B.batch_adjust(device, [probs[0], bad_p, probs[2]], iterations=3, precision="fp64", max_cg=96)
    assert recs[1][base(bad) + 14] == 1 and recs[1][base(bad) + 10] == 0
    for k in (0, 2):
        sc, rec = scenes[k], recs[k]
        want = single(device, sc, iterations=3, shared=False, max_cg=96)
        assert rec[base(sc) + 14] == 0
        assert rec[base(sc) + 10] == want[base(sc) + 10] and rec[base(sc) + 11] == want[base(sc) + 11]
        assert abs(rec[base(sc) + 6] - want[base(sc) + 6]) <= COST_REL * want[base(sc) + 6]


def test_batch_rejects_invalid_problems(device, windows):
    scenes, probs = windows
    big = B.max_cameras() + 1
    wide = S.arc_scene(seed=9, cameras=big, points=200, spacing=np.pi / (2 * big))
    with pytest.raises(tb.RangeError, match="at most"):
        B.batch_adjust(device, [probs[0], problem(wide)], iterations=1)
    packed = B.pack_batch(probs[:2], False)
    packed.table[1].output_offset = 5  # overlaps the first record
    with pytest.raises(tb.RangeError, match="overlap"):
        B.batch_adjust(device, packed, iterations=1, output=np.zeros(packed.output_len + 10))
    s, i = probs[3].scene, probs[3].index.copy()
    i[0] = probs[3].C + 5
    with pytest.raises(tb.RangeError, match="camera out of range"):
        B.batch_adjust(device, [probs[0], B.PackedProblem(probs[3].C, probs[3].P, probs[3].M, s, i)], iterations=1)
