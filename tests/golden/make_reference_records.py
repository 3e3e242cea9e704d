"""Extract the reference's recorded GPU bundle-adjustment results into reference_records.json.

    python tests/golden/make_reference_records.py <path of the reference checkout>

The reference checkout's path is a required argument.  The records are
the reference's own `bundleAdjustGpu` runs (WebGPU, emulated f64) on fixtures of
tests/typeshade/geometry-cases.mjs, from:

* docs/experiments/gpu/ba-camera-products-software.json (scripts/benchmark-gpu-invariants.mjs:
  iterations 4, maxCgIterations 64; the record's fixture file hash equals the current one)
* docs/experiments/gpu/ba-camera-workgroups-software.json
  (scripts/benchmark-ba-camera-products.mjs: iterations 3, maxCgIterations 96)

Every variant of a row is kept, so a test can see the spread of the reference's own variants.
"""
import json
import os
import sys

if len(sys.argv) != 2:
    sys.exit("usage: make_reference_records.py <path of the reference checkout>")
REFERENCE = sys.argv[1]
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_records.json")

sources = [
    ("docs/experiments/gpu/ba-camera-products-software.json", {"iterations": 4, "maxCgIterations": 64},
     "scripts/benchmark-gpu-invariants.mjs:82-83,124-130"),
    ("docs/experiments/gpu/ba-camera-workgroups-software.json", {"iterations": 3, "maxCgIterations": 96},
     "scripts/benchmark-ba-camera-products.mjs:76-85,124-129"),
]
records = []
for path, options, script in sources:
    data = json.load(open(os.path.join(REFERENCE, path)))
    for row in data["rows"]:
        variants = [{"name": v["name"], "finalCost": v["raw"][0]["cost"], "cgIterations": v["raw"][0]["cgIterations"],
                     "failures": v["raw"][0]["failures"]} for v in row["variants"]]
        records.append({
            "source": path, "script": script, "name": row["name"],
            "fixture": {"views": row["views"], "count": row["count"], "skew": bool(row.get("skew"))},
            "options": {**options, "refineSharedFocal": bool(row["shared"])},
            "inputSha256": row["inputSha256"], "variants": variants,
        })
json.dump({"records": records}, open(OUT, "w"), indent=1)
print(f"wrote {len(records)} records to {OUT}")
