"""Generates tests/golden/*.npz: inputs and outputs of the reference's own CPU backend.

Run from the repository root where the reference tree is present:

    make -C oracle ref && python tests/golden/make_golden.py

Each fixture is one case of the reference's pipeline tests
(modules/isp/tests/pipeline_test.cpp), rendered by the reference's synthetic
camera (modules/isp/src/synthetic_raw.cpp) or a flat/ramp frame built the way
those tests build them, then processed frame after frame by
oracle/_ref/libisp_ref.so, which is the reference's cpu_pipeline.cpp,
isp_params.cpp and synthetic_raw.cpp compiled unmodified. The file records
the raw bytes, the settings, and per frame the image bytes, the histogram,
the statistics and the white balance state after the frame.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle  # noqa: E402
from goldens import CASES, GOLDEN_DIR, build_case  # noqa: E402
from isp_b200 import abi  # noqa: E402


def main() -> None:
    if not oracle.reference_available():
        raise SystemExit("oracle/_ref/libisp_ref.so is missing: run `make -C oracle ref` with the reference tree")
    os.makedirs(GOLDEN_DIR, exist_ok=True)
    total = 0
    for name in CASES:
        case = build_case(name)
        ref = oracle.ReferencePipeline(case.params)
        arrays = {}
        for i, raw in enumerate(case.raws):
            arrays[f"raw{i}"] = raw.data
        for f, raw in enumerate(case.frame_raws()):
            r = ref.process(raw, case.out_format, case.with_stats, case.exposure)
            arrays[f"image{f}"] = r.image
            if case.with_stats:
                arrays[f"hist{f}"] = r.histogram
                arrays[f"stats{f}"] = r.stats
            gains, valid = ref.awb()
            arrays[f"awb{f}"] = np.array([*gains.view(np.uint32), valid], np.uint32)
        if case.params.lens_shading is not None:
            arrays["lsc"] = np.asarray(case.params.lens_shading.gains, np.float32)
        meta = {
            "name": name,
            "raws": [
                {"width": r.width, "height": r.height, "pitch": r.pitch, "format": r.format,
                 "bit_depth": r.bit_depth, "pattern": r.pattern}
                for r in case.raws
            ],
            "sequence": case.sequence,
            "out_format": case.out_format,
            "with_stats": case.with_stats,
            "exposure": list(case.exposure),
            "params": case.params.to_dict(),
        }
        arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), np.uint8)
        path = os.path.join(GOLDEN_DIR, f"{name}.npz")
        np.savez_compressed(path, **arrays)
        size = os.path.getsize(path)
        total += size
        print(f"{name:48s} {size / 1024:8.1f} KiB")
    print(f"total {total / 1024:.1f} KiB")


if __name__ == "__main__":
    main()
