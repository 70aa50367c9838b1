"""CPU tests of the colour converter's checker and host side.

The C oracle (oracle/cc_oracle.c) is pinned to the reference's own
reference_convert built from its sources (oracle/_ref/libcc_ref.so) on the
reference test's case lists, to the published colour-bar codes and
letterbox geometry the reference's tests hold, and to the fixtures in
tests/golden/cc_golden.npz (made by tests/golden/make_cc_golden.py from the
reference build). The product's host side (names, sizes, geometry, checks
and their messages) is checked against the same, through the C ABI, with no
kernel launched.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from cc_cases import (BARS_601_FULL, BARS_601_LIMITED, BARS_709_LIMITED, BARS_RGB, FORMATS, LETTERBOX, NAMES,
                      every_pair, needs_even_width, odd_sizes, resize_modes)
from isp_b200 import cc
from oracle import cc as occ

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cc_golden.npz")
need_ref = pytest.mark.skipif(not occ.have_ref(), reason="reference build absent (oracle/_ref/libcc_ref.so)")


def convert_both(src_bytes, src, sw, sh, dst, dw, dh, p):
    got = occ.convert(src_bytes, src, sw, sh, dst, dw, dh, p)
    want = occ.ref_convert(src_bytes, src, sw, sh, dst, dw, dh, p)
    return got, want


@need_ref
def test_oracle_every_pair_matches_reference():
    bad = []
    for src, dst, matrix, rng in every_pair():
        img = occ.noise(src, 66, 38, 17)
        got, want = convert_both(img, src, 66, 38, dst, 66, 38, cc.params(matrix, rng, cc.NEAREST))
        if not np.array_equal(got, want):
            bad.append((NAMES[src], NAMES[dst], matrix, rng, int((got != want).sum())))
    assert not bad, bad[:10]


@need_ref
def test_oracle_resize_modes_match_reference():
    bad = []
    srcs = {s: occ.noise(s, 98, 54, 23) for s in (cc.NV12, cc.YUYV, cc.RGB8, cc.BGRA8, cc.MONO16)}
    for mode, src, dst, w, h, crop, box in resize_modes():
        p = cc.params(cc.BT709, cc.LIMITED, mode, crop, box, (200, 30, 90))
        got, want = convert_both(srcs[src], src, 98, 54, dst, w, h, p)
        if not np.array_equal(got, want):
            bad.append((mode, NAMES[src], NAMES[dst], w, h, crop, box))
    assert not bad, bad[:10]


@need_ref
def test_oracle_odd_sizes_match_reference():
    bad = []
    for src, dst, sw, dw, h in odd_sizes():
        img = occ.noise(src, sw, h, 5)
        got, want = convert_both(img, src, sw, h, dst, dw, h, cc.params(mode=cc.BILINEAR))
        if not np.array_equal(got, want):
            bad.append((NAMES[src], NAMES[dst], sw, dw, h))
    assert not bad, bad[:10]


@need_ref
def test_oracle_upscale_and_area_match_reference():
    """Upscaling and non-integer area footprints, every mode, with and without a crop."""
    for mode in (cc.NEAREST, cc.BILINEAR, cc.AREA):
        for src, dst in ((cc.NV12, cc.RGBA8), (cc.RGB16, cc.NV16), (cc.UYVY, cc.MONO16), (cc.I420, cc.YUYV)):
            img = occ.noise(src, 30, 22, 3)
            for dw, dh, crop in ((70, 41, None), (12, 9, (3, 2, 21, 17)), (30, 22, (1, 1, 28, 20))):
                p = cc.params(cc.BT2020, cc.FULL, mode, crop, False)
                got, want = convert_both(img, src, 30, 22, dst, dw, dh, p)
                assert np.array_equal(got, want), (mode, NAMES[src], NAMES[dst], dw, dh, crop)


@need_ref
def test_oracle_pitched_matches_reference():
    """NV12 50x20 with 64-byte rows into RGBA8 40x16 (converter_test.cpp:195-227)."""
    packed = occ.noise(cc.NV12, 50, 20, 9)
    buf = np.zeros(64 * 30, np.uint8)
    for y in range(20):
        buf[64 * y:64 * y + 50] = packed[50 * y:50 * y + 50]
    for y in range(10):
        buf[64 * (20 + y):64 * (20 + y) + 50] = packed[1000 + 50 * y:1000 + 50 * y + 50]
    view = occ.host_view(buf, cc.NV12, 50, 20, pitches=(64, 64), offsets=(0, 64 * 20))
    p = cc.params(mode=cc.BILINEAR)
    got = occ.convert(None, cc.NV12, 50, 20, cc.RGBA8, 40, 16, p, src_view=view)
    want = occ.ref_convert(packed, cc.NV12, 50, 20, cc.RGBA8, 40, 16, p)
    assert np.array_equal(got, want)
    assert np.array_equal(got, occ.convert(packed, cc.NV12, 50, 20, cc.RGBA8, 40, 16, p))


def bars_image():
    """Bars two pixels wide and two high (conversion_math_test.cpp:187-196)."""
    img = np.zeros((2, 16, 3), np.uint8)
    for x in range(16):
        img[:, x] = BARS_RGB[x // 2]
    return img.reshape(-1)


def read_ycc(buf, fmt, x, y, w, h):
    planes = occ.planes_of(fmt, w, h)
    if fmt in (cc.NV12, cc.NV16):
        cy = y // 2 if fmt == cc.NV12 else y
        uv = planes[0][0] * planes[0][1] + cy * planes[1][0] + 2 * (x // 2)
        return buf[y * w + x], buf[uv], buf[uv + 1]
    if fmt == cc.I420:
        u0 = planes[0][0] * planes[0][1]
        v0 = u0 + planes[1][0] * planes[1][1]
        c = (y // 2) * planes[1][0] + x // 2
        return buf[y * w + x], buf[u0 + c], buf[v0 + c]
    row = y * 2 * w
    pair = row + 4 * (x // 2)
    if fmt == cc.YUYV:
        return buf[pair + 2 * (x & 1)], buf[pair + 1], buf[pair + 3]
    return buf[pair + 1 + 2 * (x & 1)], buf[pair], buf[pair + 2]


@pytest.mark.parametrize("fmt", [cc.NV12, cc.NV16, cc.I420, cc.YUYV, cc.UYVY])
def test_oracle_colour_bars_published(fmt):
    """The published bar codes within the one-code slack the reference allows at
    an exact tie (conversion_math_test.cpp:202-241); and back to RGB within one."""
    rgb = bars_image()
    for matrix, rng, published in ((cc.BT601, cc.LIMITED, BARS_601_LIMITED), (cc.BT709, cc.LIMITED, BARS_709_LIMITED),
                                   (cc.BT601, cc.FULL, BARS_601_FULL)):
        p = cc.params(matrix, rng)
        ycc = occ.convert(rgb, cc.RGB8, 16, 2, fmt, 16, 2, p)
        for bar in range(8):
            got = read_ycc(ycc, fmt, 2 * bar, 1, 16, 2)
            for i in range(3):
                assert abs(int(got[i]) - published[bar][i]) <= 1, (fmt, matrix, rng, bar, i, got)
                if (matrix, rng) != (cc.BT601, cc.FULL):
                    assert int(got[i]) == published[bar][i], (fmt, matrix, rng, bar, i, got)
        back = occ.convert(ycc, fmt, 16, 2, cc.RGB8, 16, 2, p).reshape(2, 16, 3)
        for bar in range(8):
            assert np.abs(back[0, 2 * bar].astype(int) - np.array(BARS_RGB[bar])).max() <= 1


def test_oracle_letterbox_geometry():
    for sw, sh, w, h, fmt, crop, source, content in LETTERBOX:
        p = cc.params(crop=crop, letterbox=True)
        assert occ.mapping(sw, sh, w, h, fmt, p) == (source, content)
        assert cc.compute_mapping(sw, sh, w, h, fmt, p) == (source, content)
    # NV12 keeps the bordered axis even; YUYV only across.
    for fmt, (sw, sh, w, h) in ((cc.NV12, (1000, 601, 334, 335)), (cc.YUYV, (601, 1000, 335, 334))):
        _, (x, y, cw, ch) = cc.compute_mapping(sw, sh, w, h, fmt, cc.params(letterbox=True))
        if fmt == cc.NV12:
            assert cw == 334 and x == 0 and ch % 2 == 0 and y % 2 == 0
        else:
            assert cw % 2 == 0 and x % 2 == 0 and ch == 334
    assert cc.compute_mapping(1920, 1080, 640, 640, cc.RGB8, cc.params())[1] == (0, 0, 640, 640)


def test_letterbox_fill_is_the_fill_colour():
    """A letterboxed NV12 border holds the fill colour's BT.601 limited YCbCr
    (conversion_math_test.cpp:444-456): blue (0, 0, 255) is (41, 240, 110)."""
    src = occ.noise(cc.RGB8, 64, 32, 1)
    out = occ.convert(src, cc.RGB8, 64, 32, cc.NV12, 32, 32, cc.params(letterbox=True, fill_rgb=(0, 0, 255)))
    assert tuple(int(v) for v in read_ycc(out, cc.NV12, 0, 0, 32, 32)) == (41, 240, 110)


@need_ref
def test_mapping_matches_reference_sweep():
    rng = np.random.default_rng(4)
    for _ in range(300):
        sw, sh, w, h = (int(v) for v in rng.integers(1, 700, 4))
        fmt = int(rng.integers(0, 12))
        crop = None
        if rng.random() < 0.4:
            cw, ch = int(rng.integers(1, sw + 1)), int(rng.integers(1, sh + 1))
            crop = (int(rng.integers(0, sw - cw + 1)), int(rng.integers(0, sh - ch + 1)), cw, ch)
        p = cc.params(crop=crop, letterbox=bool(rng.random() < 0.8))
        want = occ.mapping(sw, sh, w, h, fmt, p, ref=True)
        assert occ.mapping(sw, sh, w, h, fmt, p) == want
        assert cc.compute_mapping(sw, sh, w, h, fmt, p) == want


def test_rejects_with_the_reference_messages():
    """Odd YUYV width, short pitch, missing plane, crop outside, host images
    (conversion_math_test.cpp:459-475, converter_test.cpp:269-290)."""
    buf = np.zeros(4096, np.uint8)
    rgb = occ.host_view(buf, cc.RGB8, 3, 2, location=cc.DEVICE)
    odd = occ.host_view(buf, cc.YUYV, 3, 2, pitches=(8,), location=cc.DEVICE)
    short = occ.host_view(buf, cc.RGB8, 3, 2, pitches=(8,), location=cc.DEVICE)
    nodata = occ.host_view(buf, cc.NV12, 4, 4, location=cc.DEVICE)
    nodata.planes[1].data = None
    cases = [(odd, rgb, cc.params(), "source image: yuyv needs an even width, not 3"),
             (rgb, short, cc.params(), "destination image plane 0 pitch 8 is shorter than a row of 9 bytes"),
             (nodata, rgb, cc.params(), "source image plane 1 has no data"),
             (rgb, rgb, cc.params(crop=(4, 4, 8, 8)), "crop 8x8+4+4 is not inside the 3x2 source")]
    for src, dst, p, message in cases:
        with pytest.raises(ValueError, match=message.replace("+", r"\+")):
            cc.validate_conversion(src, dst, p)
        if occ.have_ref():
            assert occ.ref_validate(src, dst, p) == message
    host = occ.host_view(buf, cc.RGB8, 3, 2)
    with pytest.raises(ValueError, match="source image must be in CUDA device memory"):
        cc.Converter().convert(host, rgb, cc.params())


def test_names_and_sizes():
    for f, name in enumerate(NAMES):
        assert cc.format_name(f) == name and cc.parse_format(name) == f
        for w, h in ((5, 3), (1, 1), (1920, 1080), (17, 9)):
            assert cc.packed_size(f, w, h) == occ.packed_size(f, w, h)
            for k, (rb, rows) in enumerate(occ.planes_of(f, w, h)):
                assert cc.plane_size(f, w, h, k) == (rb, rows)
    assert cc.format_name(99) == "unknown" and cc.parse_format("nv21") is None
    assert [cc.matrix_name(m) for m in range(3)] == ["bt601", "bt709", "bt2020"]
    assert [cc.range_name(r) for r in range(2)] == ["limited", "full"]
    assert [cc.resize_mode_name(m) for m in range(3)] == ["nearest", "bilinear", "area"]
    assert cc.parse_matrix("bt709") == cc.BT709 and cc.parse_range("full") == cc.FULL
    assert cc.parse_resize_mode("area") == cc.AREA and cc.parse_resize_mode("cubic") is None
    # Odd sizes: chroma planes round up (conversion_math_test.cpp:259-262).
    assert cc.packed_size(cc.NV12, 5, 3) == 5 * 3 + 3 * 2 * 2
    assert cc.packed_size(cc.I420, 5, 3) == 5 * 3 + 2 * 3 * 2
    assert cc.packed_size(cc.NV16, 5, 3) == 5 * 3 + 3 * 2 * 3
    assert not needs_even_width(cc.NV12) and needs_even_width(cc.UYVY)


@need_ref
def test_test_pattern_matches_reference():
    for w, h, frame in ((1920, 1080, 0), (1920, 1080, 7), (641, 37, 1000), (1, 1, 3)):
        assert np.array_equal(occ.test_pattern(w, h, frame), occ.ref_test_pattern(w, h, frame))


def test_oracle_matches_golden_fixtures():
    """The fixtures made from the reference build (tests/golden/make_cc_golden.py)."""
    data = np.load(GOLDEN)
    cases = data["cases"]
    assert len(cases) > 100
    for i, (src, sw, sh, dst, dw, dh, matrix, rng, mode, seed, has_crop, cx, cy, cw, ch, box) in enumerate(cases):
        crop = (int(cx), int(cy), int(cw), int(ch)) if has_crop else None
        p = cc.params(int(matrix), int(rng), int(mode), crop, bool(box), (200, 30, 90))
        img = occ.noise(int(src), int(sw), int(sh), int(seed))
        got = occ.convert(img, int(src), int(sw), int(sh), int(dst), int(dw), int(dh), p)
        assert np.array_equal(got, data[f"out{i}"]), (i, NAMES[src], NAMES[dst])


@need_ref
def test_validation_matches_reference_fuzz():
    """Random views and settings: the converter's checks accept exactly what
    the reference's validate_conversion accepts and refuse the rest with its
    message (conversion.cpp:170-192, :403-408)."""
    rng = np.random.default_rng(11)
    buf = np.zeros(1 << 16, np.uint8)
    for _ in range(2000):
        views = []
        for _side in range(2):
            fmt = int(rng.integers(0, 12))
            w, h = int(rng.integers(-2, 40)), int(rng.integers(-2, 30))
            v = occ.host_view(buf, fmt, max(w, 1), max(h, 1), location=cc.DEVICE)
            v.width, v.height = w, h
            for k in range(3):
                if rng.random() < 0.05:
                    v.planes[k].data = None
                if rng.random() < 0.1:
                    v.planes[k].pitch = max(0, int(v.planes[k].pitch) - int(rng.integers(1, 4)))
            views.append(v)
        crop = None
        if rng.random() < 0.4:
            crop = tuple(int(x) for x in rng.integers(-3, 45, 4))
        p = cc.params(int(rng.integers(0, 3)), int(rng.integers(0, 2)), int(rng.integers(0, 3)), crop,
                      bool(rng.random() < 0.5))
        want = occ.ref_validate(views[0], views[1], p)
        try:
            cc.validate_conversion(views[0], views[1], p)
            got = None
        except ValueError as e:
            got = str(e)
        assert got == want, (got, want)
