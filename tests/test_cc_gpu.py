"""GPU parity of the B200 colour converter, through the C ABI
(cc_b200_convert), against the C oracle on the same bytes: bit-exact, as the
reference's own GPU test demands of its kernel
(modules/color-convert/tests/converter_test.cpp:105-113). The case lists are
the reference test's (tests/cc_cases.py), plus full-size frames of its
benchmark cases, unaligned and pitched planes, and the direct path with a
letterbox border or a crop.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from cc_cases import BENCH_CASES, NAMES, every_pair, needs_even_width, odd_sizes, resize_modes
from isp_b200 import cc
from oracle import cc as occ

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cc_golden.npz")
POISON = 0xAB


def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("no CUDA device")
    return torch


class DeviceImage:
    """A packed image in device memory at `offset` bytes past a fresh
    allocation (so plane starts need not be aligned), rows `pad` bytes longer
    than packed."""

    def __init__(self, fmt: int, width: int, height: int, data: np.ndarray = None, offset: int = 0, pad: int = 0):
        torch = torch_cuda()
        self.fmt, self.width, self.height, self.offset, self.pad = fmt, width, height, offset, pad
        self.planes = occ.planes_of(fmt, width, height)
        total = sum((rb + pad) * rows for rb, rows in self.planes)
        self.buf = torch.full((total + offset + 64,), POISON, dtype=torch.uint8, device="cuda")
        if data is not None:
            self.upload(data)

    def view(self) -> cc.CcImageC:
        v = cc.CcImageC()
        v.format, v.width, v.height, v.location = self.fmt, self.width, self.height, cc.DEVICE
        base = self.buf.data_ptr() + self.offset
        for k, (rb, rows) in enumerate(self.planes):
            v.planes[k].data = base
            v.planes[k].pitch = rb + self.pad
            base += (rb + self.pad) * rows
        return v

    def upload(self, packed: np.ndarray) -> None:
        torch = torch_cuda()
        host = np.full(self.buf.numel(), POISON, np.uint8)
        src = dst = 0
        dst = self.offset
        for rb, rows in self.planes:
            for _ in range(rows):
                host[dst:dst + rb] = packed[src:src + rb]
                src += rb
                dst += rb + self.pad
        self.buf.copy_(torch.from_numpy(host))

    def download(self) -> np.ndarray:
        host = self.buf.cpu().numpy()
        out, src = [], self.offset
        for rb, rows in self.planes:
            for _ in range(rows):
                out.append(host[src:src + rb])
                assert (host[src + rb:src + rb + self.pad] == POISON).all(), "row padding was written"
                src += rb + self.pad
        assert (host[src:] == POISON).all(), "bytes past the image were written"
        return np.concatenate(out)


def gpu_convert(src_bytes, src, sw, sh, dst, dw, dh, p, offsets=(0, 0), pads=(0, 0), stream=0) -> np.ndarray:
    torch = torch_cuda()
    s = DeviceImage(src, sw, sh, src_bytes, offsets[0], pads[0])
    d = DeviceImage(dst, dw, dh, None, offsets[1], pads[1])
    cc.Converter().convert(s.view(), d.view(), p, stream)
    torch.cuda.synchronize()
    return d.download()


def expect_same(src_bytes, src, sw, sh, dst, dw, dh, p, **kw):
    got = gpu_convert(src_bytes, src, sw, sh, dst, dw, dh, p, **kw)
    want = occ.convert(src_bytes, src, sw, sh, dst, dw, dh, p, threads=8)
    wrong = int((got != want).sum())
    return wrong


def test_every_pair_every_matrix_and_range():
    bad = []
    for src, dst, matrix, rng in every_pair():
        img = occ.noise(src, 66, 38, 17)
        wrong = expect_same(img, src, 66, 38, dst, 66, 38, cc.params(matrix, rng, cc.NEAREST))
        if wrong:
            bad.append((NAMES[src], NAMES[dst], matrix, rng, wrong))
    assert not bad, bad[:10]


def test_resize_modes_crops_and_letterboxes():
    bad = []
    srcs = {s: occ.noise(s, 98, 54, 23) for s in (cc.NV12, cc.YUYV, cc.RGB8, cc.BGRA8, cc.MONO16)}
    for mode, src, dst, w, h, crop, box in resize_modes():
        p = cc.params(cc.BT709, cc.LIMITED, mode, crop, box, (200, 30, 90))
        wrong = expect_same(srcs[src], src, 98, 54, dst, w, h, p)
        if wrong:
            bad.append((mode, NAMES[src], NAMES[dst], w, h, crop, box, wrong))
    assert not bad, bad[:10]


def test_odd_sizes():
    bad = []
    for src, dst, sw, dw, h in odd_sizes():
        img = occ.noise(src, sw, h, 5)
        wrong = expect_same(img, src, sw, h, dst, dw, h, cc.params(mode=cc.BILINEAR))
        if wrong:
            bad.append((NAMES[src], NAMES[dst], sw, dw, h, wrong))
    assert not bad, bad[:10]


def test_direct_path_with_border_crop_and_upscale():
    """Same-size content beside a letterbox border, a crop the size of the
    destination, and upscales, for every destination format."""
    bad = []
    for src in (cc.NV12, cc.UYVY, cc.RGB8, cc.BGRA8, cc.MONO16, cc.RGB16, cc.I420):
        img = occ.noise(src, 40, 22, 11)
        for dst in cc.ALL_FORMATS:
            for dw, dh, crop, box in ((40, 40, None, True), (60, 22, None, True), (26, 15, (7, 3, 26, 15), False), (24, 15, (8, 2, 24, 15), False),
                                      (80, 47, None, False), (22, 40, (9, 0, 22, 22), True)):
                if needs_even_width(dst) and dw % 2:
                    continue
                for mode in (cc.NEAREST, cc.AREA):
                    p = cc.params(cc.BT2020, cc.FULL, mode, crop, box, (10, 250, 128))
                    wrong = expect_same(img, src, 40, 22, dst, dw, dh, p)
                    if wrong:
                        bad.append((NAMES[src], NAMES[dst], dw, dh, crop, box, mode, wrong))
    assert not bad, bad[:10]


@pytest.mark.parametrize("offsets,pads", [((1, 3), (0, 0)), ((2, 1), (5, 7)), ((3, 2), (64, 13)), ((0, 0), (16, 3))])
def test_unaligned_and_pitched_planes(offsets, pads):
    """Planes that start off word boundaries and rows with padding: the
    kernels' word stores fall back to bytes and never touch the padding."""
    bad = []
    for src, dst in ((cc.RGB8, cc.NV12), (cc.NV12, cc.RGBA8), (cc.YUYV, cc.I420), (cc.RGBA8, cc.RGB16),
                     (cc.MONO16, cc.UYVY), (cc.BGR8, cc.NV16), (cc.I420, cc.MONO16), (cc.RGB16, cc.BGR8)):
        img = occ.noise(src, 50, 20, 9)
        for dw, dh, mode in ((50, 20, cc.NEAREST), (38, 16, cc.BILINEAR), (21, 9, cc.AREA)):
            if needs_even_width(dst) and dw % 2:
                dw += 1
            wrong = expect_same(img, src, 50, 20, dst, dw, dh, cc.params(cc.BT709, cc.LIMITED, mode),
                                offsets=offsets, pads=pads)
            if wrong:
                bad.append((NAMES[src], NAMES[dst], dw, dh, mode, wrong))
    assert not bad, bad


def test_pitched_nv12_as_the_reference_test():
    """NV12 50x20 with 64-byte rows into RGBA8 40x16 with 256-byte rows
    (converter_test.cpp:195-227)."""
    img = occ.noise(cc.NV12, 50, 20, 9)
    assert expect_same(img, cc.NV12, 50, 20, cc.RGBA8, 40, 16, cc.params(mode=cc.BILINEAR), pads=(14, 96)) == 0


def test_every_16bit_sample():
    """All 65,536 16-bit values, as MONO16 and RGB16 sources, through the
    direct and the resample paths: the kernels' division by 257 is the
    correctly rounded one for every input."""
    values = np.arange(65536, dtype=np.uint16)
    mono = values.view(np.uint8).copy()  # 256x256, little-endian
    rgb16 = np.stack([values, values[::-1], np.roll(values, 12345)], axis=1).reshape(-1).view(np.uint8).copy()
    bad = []
    for src, img in ((cc.MONO16, mono), (cc.RGB16, rgb16)):
        for dst in (cc.MONO16, cc.RGB16, cc.RGB8, cc.NV12):
            for dw, dh, mode in ((256, 256, cc.NEAREST), (255, 129, cc.BILINEAR), (100, 37, cc.AREA)):
                wrong = expect_same(img, src, 256, 256, dst, dw, dh, cc.params(cc.BT601, cc.FULL, mode))
                if wrong:
                    bad.append((NAMES[src], NAMES[dst], dw, dh, mode, wrong))
    assert not bad, bad


def test_golden_fixtures():
    data = np.load(GOLDEN)
    bad = []
    for i, (src, sw, sh, dst, dw, dh, matrix, rng, mode, seed, has_crop, cx, cy, cw, ch, box) in enumerate(
            data["cases"]):
        crop = (int(cx), int(cy), int(cw), int(ch)) if has_crop else None
        p = cc.params(int(matrix), int(rng), int(mode), crop, bool(box), (200, 30, 90))
        got = gpu_convert(occ.noise(int(src), int(sw), int(sh), int(seed)), int(src), int(sw), int(sh), int(dst),
                          int(dw), int(dh), p)
        if not np.array_equal(got, data[f"out{i}"]):
            bad.append(i)
    assert not bad, bad[:10]


def test_test_pattern():
    torch = torch_cuda()
    for w, h, frame in ((1920, 1080, 0), (1920, 1080, 7), (1920, 1080, 1000), (641, 37, 3)):
        img = DeviceImage(cc.RGB8, w, h)
        cc.test_pattern(img.view(), frame)
        torch.cuda.synchronize()
        assert np.array_equal(img.download(), occ.test_pattern(w, h, frame)), (w, h, frame)


def test_camera_sizes():
    """The pattern in NV12 and YUYV at 1080p to RGBA8 1080p and to a
    letterboxed RGB8 640x640 (converter_test.cpp:243-263)."""
    rgb = occ.test_pattern(1920, 1080, 3)
    for camera in (cc.NV12, cc.YUYV):
        frame = occ.convert(rgb, cc.RGB8, 1920, 1080, camera, 1920, 1080, cc.params(cc.BT709), threads=8)
        assert expect_same(frame, camera, 1920, 1080, cc.RGBA8, 1920, 1080, cc.params(cc.BT709, mode=cc.NEAREST)) == 0
        assert expect_same(frame, camera, 1920, 1080, cc.RGB8, 640, 640, cc.params(cc.BT709, letterbox=True)) == 0


@pytest.mark.parametrize("width,height", [(1920, 1080), (3840, 2160)])
def test_benchmark_cases_full_size(width, height):
    """Every case of the reference's benchmark at its sizes, on noise input."""
    bad = []
    for src, dst, ow, oh, mode, box, label in BENCH_CASES:
        dw, dh = (ow or width), (oh or height)
        img = occ.noise(src, width, height, 7) if width < 3000 else np.random.default_rng(7).integers(
            0, 256, occ.packed_size(src, width, height), dtype=np.uint8)
        wrong = expect_same(img, src, width, height, dst, dw, dh, cc.params(cc.BT709, mode=mode, letterbox=box))
        if wrong:
            bad.append((NAMES[src], NAMES[dst], dw, dh, label, wrong))
    assert not bad, bad


def test_determinism_across_streams():
    """YUYV 640x360 to a letterboxed NV12 300x200 by area, three times on two
    streams (converter_test.cpp:265-277)."""
    torch = torch_cuda()
    img = occ.noise(cc.YUYV, 640, 360, 31)
    p = cc.params(mode=cc.AREA, letterbox=True)
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    outs = [gpu_convert(img, cc.YUYV, 640, 360, cc.NV12, 300, 200, p, stream=s.cuda_stream) for s in (s1, s2, s1)]
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])
    assert np.array_equal(outs[0], occ.convert(img, cc.YUYV, 640, 360, cc.NV12, 300, 200, p))


@pytest.mark.skipif(not occ.have_ref_cuda(), reason="reference CUDA build absent")
def test_reference_cuda_kernel_agrees():
    """The reference's own kernel, built for sm_100a, gives the same bytes on
    a few benchmark cases (a second witness beside the oracle)."""
    torch = torch_cuda()
    for src, dst, ow, oh, mode, box, label in BENCH_CASES[::3]:
        img = np.random.default_rng(1).integers(0, 256, occ.packed_size(src, 1920, 1080), dtype=np.uint8)
        dw, dh = (ow or 1920), (oh or 1080)
        p = cc.params(cc.BT709, mode=mode, letterbox=box)
        s = DeviceImage(src, 1920, 1080, img)
        d = DeviceImage(dst, dw, dh)
        occ.ref_cuda_convert(s.view(), d.view(), p)
        torch.cuda.synchronize()
        assert np.array_equal(d.download(), gpu_convert(img, src, 1920, 1080, dst, dw, dh, p)), label
