"""The colour converter's benchmark cases: those of the reference's own
benchmark (modules/color-convert/tests/benchmark.cpp:71-103), each run at
1920x1080 and 3840x2160 with BT.709 on the synthetic camera's test pattern
converted into the source format, as that benchmark does (:120-135)."""
from __future__ import annotations

from . import cc

# (source, destination, output width, output height (0: the input's), mode, letterbox, label)
BENCH_CASES = (
    (cc.NV12, cc.RGB8, 0, 0, cc.NEAREST, False, "convert"),
    (cc.NV12, cc.RGBA8, 0, 0, cc.NEAREST, False, "convert"),
    (cc.NV12, cc.BGR8, 0, 0, cc.NEAREST, False, "convert"),
    (cc.NV12, cc.MONO8, 0, 0, cc.NEAREST, False, "convert"),
    (cc.NV16, cc.RGB8, 0, 0, cc.NEAREST, False, "convert"),
    (cc.I420, cc.RGB8, 0, 0, cc.NEAREST, False, "convert"),
    (cc.YUYV, cc.RGB8, 0, 0, cc.NEAREST, False, "convert"),
    (cc.YUYV, cc.RGBA8, 0, 0, cc.NEAREST, False, "convert"),
    (cc.UYVY, cc.RGBA8, 0, 0, cc.NEAREST, False, "convert"),
    (cc.YUYV, cc.NV12, 0, 0, cc.NEAREST, False, "convert"),
    (cc.RGB8, cc.NV12, 0, 0, cc.NEAREST, False, "convert"),
    (cc.RGBA8, cc.NV12, 0, 0, cc.NEAREST, False, "convert"),
    (cc.RGB8, cc.BGR8, 0, 0, cc.NEAREST, False, "convert"),
    (cc.RGB16, cc.RGB8, 0, 0, cc.NEAREST, False, "convert"),
    (cc.NV12, cc.RGBA8, 1280, 720, cc.BILINEAR, False, "resize bilinear"),
    (cc.NV12, cc.RGB8, 640, 640, cc.BILINEAR, True, "resize bilinear, letterbox"),
    (cc.YUYV, cc.RGBA8, 640, 360, cc.NEAREST, False, "resize nearest"),
    (cc.NV12, cc.RGB8, 1280, 720, cc.AREA, False, "resize area"),
    (cc.NV12, cc.NV12, 1280, 720, cc.BILINEAR, False, "resize bilinear"),
)
SIZES = ((1920, 1080), (3840, 2160))

# The headline: the ISP's RGB8 output of a 4K frame into NV12, the format an
# encoder or an inference stage takes next.
HEADLINE = (cc.RGB8, cc.NV12, 3840, 2160)
