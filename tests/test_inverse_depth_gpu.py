"""Inverse-depth linearisation on the device against the oracle (tba_linearize_inverse_depth).

Restates the linearisation half of the reference's inverseDepthGpuCases
(tests/typeshade/inverse-depth-cases.mjs:126-165): every view of inverseDepthScene against one
anchored point at rho in {0, 1e-9, 0.2, -0.01}; rows unchanged by batching; validity and every
value within 1e-8 of the CPU linearisation (relative to max(1, |value|)).  Plus the admission checks
of tests/typeshade/inverse-depth.test.mjs:17-79 that apply to a synchronous host, rows that leave
the model's domain, and the long scene in batches of 127.
"""
import numpy as np
import pytest

import typecv_b200 as tb
from oracle import inverse_depth as oid
from reference_cases import inverse_depth_long_scene, inverse_depth_scene
from test_inverse_depth import anchored
from typecv_b200 import inverse_depth as ID
from typecv_b200.bundle import RangeError

pytestmark = pytest.mark.gpu

KEYS = ("pixel", "point", "pose", "focal")


@pytest.fixture(scope="module")
def device():
    dev = tb.ShadeDevice.open(0)
    yield dev
    dev.close()


def compare(measurements, rows):
    worst = 0.0
    for m, gpu in zip(measurements, rows):
        cpu = oid.inverse_depth_jacobian(m["view"]["camera"], m["view"]["pose"], m["point"])
        assert (cpu is None) == (gpu is None)
        if cpu is None:
            continue
        for key in KEYS:
            a, b = np.asarray(cpu[key], float), np.asarray(gpu[key], float)
            worst = max(worst, float(np.max(np.abs(a - b) / np.maximum(1, np.abs(a)))))
    return worst


def test_linearization_matches_cpu_and_is_unchanged_by_batching(device):
    model = inverse_depth_scene()
    measurements = [{"view": v, "point": anchored(model, rho=rho)} for rho in (0, 1e-9, 0.2, -0.01)
                    for v in model["views"]]
    whole = ID.linearize_batches(device, {"measurements": measurements})
    chunked = ID.linearize_batches(device, {"measurements": measurements}, 5)
    assert whole["batches"] == 1 and chunked["batches"] == 4 and chunked["batchSize"] == 5
    for a, b in zip(whole["rows"], chunked["rows"]):
        assert (a is None) == (b is None)
        if a is not None:
            for key in KEYS:
                assert np.array_equal(np.asarray(a[key]), np.asarray(b[key]))
    assert compare(measurements, whole["rows"]) <= 1e-8
    rep = whole["reports"][0]
    assert rep["kernel_launches"] == 1 and rep["h2d_bytes"] == 34 * 8 * 16 and rep["d2h_bytes"] == 23 * 8 * 16


def test_rows_outside_the_model_domain_come_back_empty(device):
    model = inverse_depth_scene()
    measurements = [{"view": v, "point": anchored(model, track=t, rho=-5)} for t in (0, 7) for v in model["views"]]
    rows = ID.linearize_inverse_depth_gpu(device, {"measurements": measurements})
    assert [r is not None for r in rows[:4]] == [True, True, False, False]
    assert compare(measurements, rows) <= 1e-8
    # Beyond the radial model's injective branch (r^2 >= -1/(3 k1)) for some of the points.
    wide = {**model["views"][1], "camera": {"fx": 800, "fy": 760, "cx": 320, "cy": 240, "k1": -10.0}}
    measurements = [{"view": wide, "point": anchored(model, t)} for t in range(25)]
    rows = ID.linearize_inverse_depth_gpu(device, {"measurements": measurements})
    assert [t for t, r in enumerate(rows) if r is None] == [1, 6, 11, 16, 21]
    assert compare(measurements, rows) <= 1e-8


def test_admission_checks(device):
    model = inverse_depth_scene()
    job = {"measurements": [{"view": model["views"][1], "point": anchored(model)}]}
    device.working_bytes = 1
    try:
        with pytest.raises(RangeError, match="budget"):
            ID.linearize_inverse_depth_gpu(device, job)
    finally:
        device.working_bytes = None
    with pytest.raises(RangeError, match="batch"):
        ID.linearize_inverse_depth_gpu(device, job, 0)
    device.working_bytes = 456  # one measurement's 57 words
    try:
        repeat = ID.linearize_batches(device, {"measurements": job["measurements"] * 3})
    finally:
        device.working_bytes = None
    assert len(repeat["rows"]) == 3 and repeat["batches"] == 3 and repeat["batchSize"] == 1
    for key in KEYS:
        assert np.array_equal(np.asarray(repeat["rows"][0][key]), np.asarray(repeat["rows"][2][key]))
    # The job is snapshotted: the caller's arrays are not read after the call returns, nor changed.
    before = job["measurements"][0]["point"]["parameters"].copy()
    rows = ID.linearize_inverse_depth_gpu(device, job, 1)
    assert np.array_equal(job["measurements"][0]["point"]["parameters"], before)
    want = oid.inverse_depth_jacobian(model["views"][1]["camera"], model["views"][1]["pose"], job["measurements"][0]["point"])
    assert abs(rows[0]["pixel"][0] - want["pixel"][0]) < 1e-9
    assert ID.linearize_inverse_depth_gpu(device, {"measurements": []}) == []


def test_long_scene_in_tail_batches(device):
    model = inverse_depth_long_scene()
    views = {v["id"]: v for v in model["views"]}
    measurements = []
    for p in model["landmarks"]:
        first = views[p["observations"][0]["viewId"]]
        point = oid.initialize_inverse_depth(first, p["observations"][0]["pixel"], p["xyz"])
        measurements += [{"view": views[o["viewId"]], "point": point} for o in p["observations"]]
    out = ID.linearize_batches(device, {"measurements": measurements}, 127)
    assert len(measurements) == 1008 and out["batches"] == 8 and out["batchSize"] == 127
    assert all(r is not None for r in out["rows"])
    assert compare(measurements, out["rows"]) <= 1e-8


def test_joint_bundle_on_the_device_matches_the_cpu_arm(device):
    """inverseDepthGpuCases' joint half (inverse-depth-cases.mjs:166-184)."""
    from typecv_b200.inverse_depth_bundle import bundle_adjust_inverse_depth_gpu
    model = inverse_depth_scene()
    cpu = oid.bundle_adjust_inverse_depth(model, [], {"iterations": 1})
    gpu = bundle_adjust_inverse_depth_gpu(device, model, [], {"iterations": 1, "solver": "sparse",
                                                              "measurementBatchSize": 31})
    assert cpu["uncertainty"]["observable"] and gpu["uncertainty"]["observable"]
    for a, b in zip(cpu["estimates"], gpu["estimates"]):
        assert abs(a["covariance"][8] - b["covariance"][8]) / a["covariance"][8] <= 1e-6
    d = gpu["diagnostics"]
    assert d["backend"] == "cuda-jacobians/host-f64-Schur"
    assert d["measurementBatchSize"] == 31 and d["measurementBatches"] == 2 * 4
    assert d["kernelLaunches"] == d["measurementBatches"] + d["costBatches"]


def test_large_sparse_joint_solve_in_tail_batches(device):
    """inverseDepthLargeGpuCase (inverse-depth-cases.mjs:87-123)."""
    from typecv_b200.inverse_depth_bundle import bundle_adjust_inverse_depth_gpu
    model = inverse_depth_long_scene()
    cpu = oid.bundle_adjust_inverse_depth(model, [], {"iterations": 1, "solver": "sparse"})
    gpu = bundle_adjust_inverse_depth_gpu(device, model, [], {"iterations": 1, "solver": "sparse",
                                                              "measurementBatchSize": 127})
    assert cpu["uncertainty"]["observable"] and gpu["uncertainty"]["observable"]
    worst = max(abs(b["covariance"][8] / a["covariance"][8] - 1) for a, b in zip(cpu["estimates"], gpu["estimates"]))
    assert worst <= 1e-4
    d = gpu["diagnostics"]
    assert d["cameraParameters"] > 96 and d["linearSolver"] == "sparse" and gpu["uncertainty"]["poses"] == "joint"
    assert d["measurementBatches"] == 16
    assert abs(d["finalCost"] - cpu["diagnostics"]["finalCost"]) <= 1e-9 * max(1.0, cpu["diagnostics"]["finalCost"])


def test_sliced_call_matches_the_oracle(device):
    """A call of more than 262,144 rows runs as slices of whole 128-row tiles whose downloads overlap
    the next slices' uploads: 600,001 rows make three launches, the last slice ragged, and every row
    equals the C++ CPU linearisation (flags equal, values within 1e-8)."""
    from typecv_b200.synthetic import inverse_depth_rows
    rows = inverse_depth_rows(seed=9, measurements=600_001)
    out = ID.linearize_rows(device, rows)
    assert out["batches"] == 1 and out["reports"][0]["kernel_launches"] == 3
    want = oid.linearize_rows(rows)
    assert np.array_equal(out["out"][:, 0], want[:, 0])
    ok = want[:, 0] == 1
    assert ok.sum() > 500_000
    assert np.max(np.abs(out["out"][ok] - want[ok]) / np.maximum(1, np.abs(want[ok]))) < 1e-8
    again = ID.linearize_rows(device, rows, 262_145)
    assert again["batches"] == 3 and np.array_equal(again["out"], out["out"])


def test_tile_wait_that_runs_out_reports_an_error_and_the_handle_recovers(device):
    # The kernel's bounded mbarrier waits are its failure detection.  With the main-loop waits cut
    # to zero polls, every block gives up on its first tile at once; the loads it issued still land
    # (the drain keeps the full bound), the call returns TBA_ERROR_CUDA with its message, and the
    # next call on the same handle, at the default bound, is correct.
    import ctypes

    from typecv_b200 import _lib
    from typecv_b200.synthetic import inverse_depth_rows
    lib = _lib.load()
    n = 3000  # 24 tiles: several blocks, each with both stages loaded when its first wait fails
    rows = np.ascontiguousarray(inverse_depth_rows(measurements=n).ravel())
    out = np.full(23 * n, np.nan)

    def call():
        return lib.tba_linearize_inverse_depth(device.handle, n, _lib.dptr(rows), rows.size, _lib.dptr(out), out.size,
                                               ctypes.byref(_lib.ObservationReport()))

    try:
        assert lib.tba_device_set_wait_limit(device.handle, 0) == _lib.TBA_OK
        assert call() == _lib.TBA_ERROR_CUDA
        msg = lib.tba_last_error(device.handle).decode()
        assert "did not complete" in msg and "in flight" not in msg, msg
    finally:
        assert lib.tba_device_set_wait_limit(device.handle, _lib.TBA_WAIT_LIMIT_DEFAULT) == _lib.TBA_OK
    out[:] = np.nan
    assert call() == _lib.TBA_OK, lib.tba_last_error(device.handle)
    want = oid.linearize_rows(rows.reshape(n, 34))
    got = out.reshape(n, 23)
    assert np.max(np.abs(got - want) / np.maximum(1, np.abs(want))) < 1e-8
