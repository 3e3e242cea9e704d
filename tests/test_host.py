"""Host-side logic of the operator, the packed layout and the C ABI surface (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

import typecv_b200 as tb
from typecv_b200 import _lib, build
from typecv_b200 import bundle as B
from typecv_b200 import synthetic as S
from oracle import bundle_adjust as ob
from reference_cases import bundle_fixture, joint_focal_fixture

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _lib.load()


def test_library_exports_every_header_symbol(lib):
    header = open(os.path.join(ROOT, "include", "tba.h")).read()
    declared = set(re.findall(r"\b(tba_[a-z_]+)\s*\(", header))
    assert declared == set(_lib.EXPORTS)
    for name in declared:
        assert hasattr(lib, name), name


def test_sizes_follow_the_reference_layout(lib):
    c = B.make_control(7, 11, 40, anchor=0, scale_view=1, shared_focal=True)
    assert lib.tba_scene_size(ctypes.byref(c)) == 18 * 7 + 3 * 11 + 2 * 40
    assert lib.tba_index_size(ctypes.byref(c)) == 3 * 40 + 11 + 2 * 7 + 2
    assert lib.tba_output_size(ctypes.byref(c)) == 12 * 7 + 3 * 11 + 27
    c.shared_focal = 0
    assert lib.tba_output_size(ctypes.byref(c)) == 12 * 7 + 3 * 11 + 26


@pytest.mark.parametrize("struct, cname", [
    (_lib.Control, "tba_control"), (_lib.Report, "tba_report"), (_lib.BatchProblem, "tba_batch_problem"),
    (_lib.BatchControl, "tba_batch_control"), (_lib.BatchReport, "tba_batch_report"),
    (_lib.VjpControl, "tba_vjp_control"), (_lib.VjpReport, "tba_vjp_report"),
    (_lib.ObservationControl, "tba_observation_control"), (_lib.ObservationReport, "tba_observation_report"),
])
def test_ctypes_structures_match_the_header_layout(struct, cname, tmp_path):
    # The Python mirrors of the C ABI's structures: the size and every field's offset as the C
    # compiler lays out include/tba.h.
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    fields = [f[0] for f in struct._fields_]
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "tba.h"\nint main(void) {\n'
                   + f'  printf("%zu\\n", sizeof({cname}));\n'
                   + "".join(f'  printf("%zu\\n", offsetof({cname}, {f}));\n' for f in fields)
                   + "  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(root, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert got[0] == ctypes.sizeof(struct), (cname, got[0], ctypes.sizeof(struct))
    assert got[1:] == [getattr(struct, f).offset for f in fields], cname


def test_device_open_reports_errors_without_crashing(lib):
    h = ctypes.c_void_p()
    status = lib.tba_device_open(0, ctypes.byref(h))
    if status == 0:
        lib.tba_device_close(h)
        pytest.skip("a GPU is present")
    assert not h.value and lib.tba_last_error(None)
    assert lib.tba_device_open(-1, ctypes.byref(h)) != 0


def test_packers_agree_with_the_oracle():
    for model in (bundle_fixture(views=5, count=50), joint_focal_fixture()["input"]):
        pb = B.bundle_problem(model, {}, lambda C: 24)
        s, i = B.pack_bundle_scene(pb["input"], pb["byId"], pb["active"])
        o = ob.pack(pb["input"], [int(a) for a in pb["active"]])
        assert np.array_equal(s, o["scene"]) and np.array_equal(i, o["index"])
    sc = S.ring_scene(cameras=5, points=60)
    s1, i1 = sc.packed()
    rec = sc.as_reconstruction()
    pb = B.bundle_problem(rec, {}, lambda C: 24)
    s2, i2 = B.pack_bundle_scene(pb["input"], pb["byId"], pb["active"])
    assert np.array_equal(s1, s2) and np.array_equal(i1, i2)


class _NoDevice:
    @property
    def handle(self):
        raise AssertionError("the device must not be reached")


@pytest.mark.parametrize("case,options,match", [
    ("owned", {}, "owned"),
    ("gauge", {"anchorViewId": 999}, "gauge"),
    ("window", {"variableViewIds": [10]}, "window"),
    ("scale", {"variableViewIds": [20]}, "scale camera"),
    ("disconnected", {}, "connected observation graph"),
    ("options", {"iterations": 101}, "Invalid GPU BA scene/options"),
    ("options", {"maxCgIterations": 0}, "Invalid GPU BA scene/options"),
    ("options", {"cgRelativeTolerance": 1.0}, "Invalid GPU BA scene/options"),
    ("stall", {"stallTolerance": 1.0}, "stallTolerance"),
    ("groups", {"refineSharedFocal": True, "focalGroups": {10: 0, 20: 1, 30: 0, 40: 1}}, "Per-group"),
    ("wg", {"cameraProductWorkgroupSize": 48}, "cameraProductWorkgroupSize"),
    ("mode", {"schurReduction": "fast"}, "Schur reduction"),
    ("camera", {}, "GPU geometry bounds"),
])
def test_operator_rejects_invalid_problems_before_device_work(case, options, match):
    # bundle.ts:808-838, bundle-host.ts:31-113; tests/typeshade/cpu.test.mjs:507.
    inp = bundle_fixture()
    if case == "owned":
        inp = {**inp, "landmarks": [inp["landmarks"][0], {**inp["landmarks"][1], "observations": inp["landmarks"][0]["observations"]}]}
    if case == "disconnected":
        inp = {**inp, "landmarks": [{**p, "observations": [o for o in p["observations"] if o["viewId"] != 40]}
                                    for p in inp["landmarks"]]}
    if case == "camera":
        inp = {**inp, "views": [{**v, "camera": {**v["camera"], "k1": 2.0}} for v in inp["views"]]}
    with pytest.raises(tb.RangeError, match=match):
        tb.bundle_adjust_gpu(_NoDevice(), inp, options)
