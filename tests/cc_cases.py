"""Case lists of the colour converter's parity tests, after the reference's own
tests (modules/color-convert/tests/converter_test.cpp:126-229 and
tests/host/conversion_math_test.cpp:138-508): the same formats, sizes,
crops, letterboxes, matrices and ranges; the expected side is the checker."""
from __future__ import annotations

import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for _p in (ROOT, os.path.join(ROOT, "holoscan-zozo-modules_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

from isp_b200 import cc  # noqa: E402

FORMATS = cc.ALL_FORMATS
NAMES = ("nv12", "nv16", "i420", "yuyv", "uyvy", "rgb8", "bgr8", "rgba8", "bgra8", "mono8", "mono16", "rgb16")


def needs_even_width(fmt: int) -> bool:
    return fmt in (cc.YUYV, cc.UYVY)


def every_pair():
    """(src, dst, matrix, range): every format into every format, 66x38, nearest
    (converter_test.cpp:126-144)."""
    for matrix in (cc.BT601, cc.BT709, cc.BT2020):
        for rng in (cc.LIMITED, cc.FULL):
            for src in FORMATS:
                for dst in FORMATS:
                    yield src, dst, matrix, rng


# (width, height, crop, letterbox) of converter_test.cpp:155-158, from a 98x54 source.
RESIZE_SIZES = ((64, 36, None, False), (200, 120, None, False), (30, 17, None, False),
                (48, 48, (7, 3, 50, 29), False), (64, 64, None, True), (41, 64, (10, 6, 61, 40), True))
RESIZE_SOURCES = (cc.NV12, cc.YUYV, cc.RGB8, cc.BGRA8, cc.MONO16)
RESIZE_DESTS = (cc.RGB8, cc.NV12, cc.I420, cc.UYVY, cc.MONO8, cc.RGB16)


def resize_modes():
    """(mode, src, dst, w, h, crop, letterbox) of converter_test.cpp:146-178;
    BT.709, fill (200, 30, 90)."""
    for mode in (cc.NEAREST, cc.BILINEAR, cc.AREA):
        for src in RESIZE_SOURCES:
            for dst in RESIZE_DESTS:
                for w, h, crop, box in RESIZE_SIZES:
                    if needs_even_width(dst) and w % 2:
                        continue
                    yield mode, src, dst, w, h, crop, box


def odd_sizes():
    """(src, dst, sw, dw, h): 1x1, 3x5, 17x9 between every pair, bilinear
    (converter_test.cpp:180-193)."""
    for src in FORMATS:
        for dst in FORMATS:
            for w, h in ((1, 1), (3, 5), (17, 9)):
                yield src, dst, w + 1 if needs_even_width(src) else w, w + 1 if needs_even_width(dst) else w, h


# Published colour bars (Y, Cb, Cr) of 100% bars white .. black, the figures the
# reference's test checks (conversion_math_test.cpp:150-184): ITU-R BT.601 and
# BT.709 with 219-code luma, and JPEG/JFIF for BT.601 full range.
BARS_RGB = ((255, 255, 255), (255, 255, 0), (0, 255, 255), (0, 255, 0), (255, 0, 255), (255, 0, 0), (0, 0, 255),
            (0, 0, 0))
BARS_601_LIMITED = ((235, 128, 128), (210, 16, 146), (170, 166, 16), (145, 54, 34), (106, 202, 222), (81, 90, 240),
                    (41, 240, 110), (16, 128, 128))
BARS_709_LIMITED = ((235, 128, 128), (219, 16, 138), (188, 154, 16), (173, 42, 26), (78, 214, 230), (63, 102, 240),
                    (32, 240, 118), (16, 128, 128))
BARS_601_FULL = ((255, 128, 128), (226, 0, 149), (179, 171, 0), (150, 44, 21), (105, 212, 235), (76, 85, 255),
                 (29, 255, 107), (0, 128, 128))

# Letterbox geometry known answers (conversion_math_test.cpp:406-443):
# (sw, sh, w, h, dst format, crop, expected source rect, expected content rect or
# a predicate name).
LETTERBOX = (
    (1920, 1080, 640, 640, cc.RGB8, None, (0, 0, 1920, 1080), (0, 140, 640, 360)),
    (1080, 1920, 640, 640, cc.RGB8, None, (0, 0, 1080, 1920), (140, 0, 360, 640)),
    (1000, 600, 333, 333, cc.RGB8, None, (0, 0, 1000, 600), (0, 66, 333, 200)),
    (1000, 600, 333, 333, cc.NV12, None, (0, 0, 1000, 600), (0, 66, 333, 200)),
    (1280, 720, 640, 360, cc.NV12, None, (0, 0, 1280, 720), (0, 0, 640, 360)),
    (1920, 1080, 300, 300, cc.RGB8, (100, 100, 400, 200), (100, 100, 400, 200), (0, 75, 300, 150)),
)

from isp_b200.cc_workloads import BENCH_CASES  # noqa: E402,F401  (the reference benchmark's cases)
