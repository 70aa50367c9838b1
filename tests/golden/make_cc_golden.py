"""Makes tests/golden/cc_golden.npz: outputs of the reference's own
reference_convert (oracle/_ref/libcc_ref.so, built from the reference's
sources by oracle/Makefile) on seeded noise images, for the colour
converter's parity tests where the reference build is absent.

    python tests/golden/make_cc_golden.py

Each case row: src, sw, sh, dst, dw, dh, matrix, range, mode, seed, has_crop,
crop x, y, w, h, letterbox; the fill is (200, 30, 90). The source bytes are
regenerated from the seed (oracle.cc.noise), so only outputs are stored.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "tests"), os.path.join(ROOT, "holoscan-zozo-modules_b200")]

from cc_cases import FORMATS, needs_even_width  # noqa: E402
from isp_b200 import cc  # noqa: E402
from oracle import cc as occ  # noqa: E402


def cases():
    # Every pair, each matrix and range once in turn, at 18x10.
    k = 0
    for src in FORMATS:
        for dst in FORMATS:
            matrix, rng = k % 3, (k // 3) % 2
            k += 1
            yield (src, 18, 10, dst, 18, 10, matrix, rng, cc.NEAREST, 17 + src, 0, 0, 0, 0, 0, 0)
    # Resizes: every mode, a crop and a letterbox, 40x22 sources.
    sizes = ((24, 13, None, 0), (52, 30, None, 0), (20, 20, (5, 3, 30, 15), 0), (22, 26, None, 1),
             (17, 32, (6, 4, 28, 16), 1))
    for mode in (cc.NEAREST, cc.BILINEAR, cc.AREA):
        for src, dst in ((cc.NV12, cc.RGB8), (cc.YUYV, cc.I420), (cc.RGBA8, cc.NV12), (cc.MONO16, cc.UYVY),
                         (cc.RGB16, cc.BGRA8), (cc.I420, cc.MONO8)):
            for w, h, crop, box in sizes:
                if needs_even_width(dst) and w % 2:
                    w += 1
                c = crop or (0, 0, 0, 0)
                yield (src, 40, 22, dst, w, h, cc.BT709, cc.LIMITED, mode, 23 + mode, int(crop is not None), *c, box)


def main() -> None:
    rows, outs = [], {}
    for i, row in enumerate(cases()):
        src, sw, sh, dst, dw, dh, matrix, rng, mode, seed, has_crop, cx, cy, cw, ch, box = row
        p = cc.params(matrix, rng, mode, (cx, cy, cw, ch) if has_crop else None, bool(box), (200, 30, 90))
        outs[f"out{i}"] = occ.ref_convert(occ.noise(src, sw, sh, seed), src, sw, sh, dst, dw, dh, p)
        rows.append(row)
    np.savez_compressed(os.path.join(HERE, "cc_golden.npz"), cases=np.array(rows, np.int32), **outs)
    print(len(rows), "cases")


if __name__ == "__main__":
    main()
