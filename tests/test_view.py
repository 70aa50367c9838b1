"""The demo's side-by-side view (applications/isp/src/view_op.cu:35-75):
raw mosaic as square-rooted gray on the left, the ISP's RGB8 image on the
right. The C oracle is checked here against an independent numpy restatement
(float32 arithmetic, one rounding per step); the GPU kernel, through
isp_b200_view_compose, against the oracle byte for byte, and against the
demo's own view kernel: view_op.cu built from its source for sm_100a with
the SDK's declarations stubbed (oracle/_ref/libview_ref_cuda.so, where the
reference tree was present at build time), run on the same device buffers."""
from __future__ import annotations

import numpy as np
import pytest

import isp_b200
import oracle
from isp_b200 import abi

FORMATS = ((abi.U8, 8), (abi.U16, 12), (abi.U16, 16), (abi.RAW10, 10), (abi.RAW12, 12),
           (abi.U16, 10))


def random_raw(fmt: int, bits: int, width: int, height: int, seed: int, pad: int = 0) -> abi.RawFrame:
    rng = np.random.default_rng(seed)
    pitch = abi.raw_row_bytes(fmt, width) + pad
    data = rng.integers(0, 256, pitch * height, dtype=np.uint8)
    return abi.RawFrame(data, width, height, pitch, fmt, bits, abi.RGGB)


def unpack(raw: abi.RawFrame) -> np.ndarray:
    """Sample counts [H, W] (isp_math.hpp:101-119)."""
    rows = raw.data.reshape(raw.height, raw.pitch).astype(np.int64)
    w = raw.width
    if raw.format == abi.U8:
        return rows[:, :w]
    if raw.format == abi.U16:
        return rows[:, 0:2 * w:2] | (rows[:, 1:2 * w:2] << 8)
    x = np.arange(w)
    if raw.format == abi.RAW10:
        g = 5 * (x >> 2)
        return (rows[:, g + (x & 3)] << 2) | ((rows[:, g + 4] >> (2 * (x & 3))) & 3)
    g = 3 * (x >> 1)
    return (rows[:, g + (x & 1)] << 4) | ((rows[:, g + 2] >> (4 * (x & 1))) & 15)


def numpy_view(raw: abi.RawFrame, black: float, rgb: np.ndarray) -> np.ndarray:
    f = np.float32
    white = f((1 << raw.bit_depth) - 1)
    scale = f(1) / (white - f(black))
    v = (unpack(raw).astype(f) - f(black)) * scale
    v = np.where(v < 0, f(0), np.where(v > 1, f(1), v)).astype(f)
    g = (np.sqrt(v) * f(255) + f(0.5)).astype(np.uint8)  # truncation of a value in [0.5, 255.5]
    out = np.empty((raw.height, 2 * raw.width, 3), np.uint8)
    out[:, :raw.width] = g[:, :, None]
    out[:, raw.width:] = rgb
    return out


@pytest.mark.parametrize("fmt,bits", FORMATS)
def test_oracle_view_matches_numpy(fmt, bits):
    for w, h, black in ((37, 11, 64.0), (64, 8, 0.0), (5, 3, 200.5)):
        raw = random_raw(fmt, bits, w, h, seed=w * 7 + bits, pad=3)
        rgb = np.random.default_rng(w).integers(0, 256, (h, w, 3), dtype=np.uint8)
        black = min(black, float((1 << bits) - 2))
        assert np.array_equal(oracle.view_compose(raw, black, rgb), numpy_view(raw, black, rgb))


@pytest.mark.gpu
@pytest.mark.parametrize("fmt,bits", FORMATS)
def test_view_kernel_matches_oracle(fmt, bits):
    import torch

    for w, h, black, pads in ((3840, 2160, 64.0, (0, 0, 0)), (37, 11, 16.0, (3, 5, 7)), (1, 1, 0.0, (0, 0, 0)),
                              (130, 9, 255.0 if bits > 8 else 17.0, (16, 1, 2))):
        raw = random_raw(fmt, bits, w, h, seed=w + bits, pad=pads[0])
        rgb = np.random.default_rng(w).integers(0, 256, (h, w, 3), dtype=np.uint8)
        rgb_pitch = 3 * w + pads[1]
        view_pitch = 6 * w + pads[2]
        rgb_rows = np.zeros((h, rgb_pitch), np.uint8)
        rgb_rows[:, :3 * w] = rgb.reshape(h, 3 * w)
        d_raw = torch.from_numpy(raw.data).cuda()
        d_rgb = torch.from_numpy(rgb_rows.reshape(-1)).cuda()
        d_out = torch.full((h * view_pitch,), 0xAB, dtype=torch.uint8, device="cuda")
        isp_b200.view_compose(raw.view(d_raw.data_ptr()), black, d_rgb.data_ptr(), rgb_pitch, d_out.data_ptr(),
                              view_pitch)
        torch.cuda.synchronize()
        got = d_out.cpu().numpy().reshape(h, view_pitch)
        want = oracle.view_compose(raw, black, rgb)
        assert np.array_equal(got[:, :6 * w].reshape(h, 2 * w, 3), want), (fmt, bits, w, h)
        assert (got[:, 6 * w:] == 0xAB).all(), "row padding was written"


@pytest.mark.gpu
@pytest.mark.skipif(not oracle.reference_view_available(), reason="the reference view kernel is not built")
@pytest.mark.parametrize("fmt,bits", FORMATS)
def test_view_kernel_matches_the_demos_kernel(fmt, bits):
    import torch

    for w, h, black in ((3840, 2160, 64.0), (37, 11, 16.0), (1, 1, 0.0), (130, 9, 255.0 if bits > 8 else 17.0),
                        (640, 480, float((1 << bits) - 2))):
        raw = random_raw(fmt, bits, w, h, seed=3 * w + bits)
        rgb = np.random.default_rng(w + 1).integers(0, 256, (h, w, 3), dtype=np.uint8)
        d_raw = torch.from_numpy(raw.data).cuda()
        d_rgb = torch.from_numpy(rgb.reshape(-1)).cuda()
        ours = torch.full((h * 6 * w,), 0xAB, dtype=torch.uint8, device="cuda")
        theirs = torch.full((h * 6 * w,), 0x5C, dtype=torch.uint8, device="cuda")
        isp_b200.view_compose(raw.view(d_raw.data_ptr()), black, d_rgb.data_ptr(), 3 * w, ours.data_ptr(), 6 * w)
        oracle.reference_view_compose(d_raw.data_ptr(), raw.pitch, w, h, fmt, bits, black, d_rgb.data_ptr(),
                                      theirs.data_ptr())
        torch.cuda.synchronize()
        assert torch.equal(ours, theirs), (fmt, bits, w, h, black)


def test_view_rejects():
    raw = random_raw(abi.RAW10, 10, 8, 2, 1)
    buf = 1 << 20  # never dereferenced: every call below is refused before a launch
    with pytest.raises(ValueError, match="pitch"):
        isp_b200.view_compose(raw.view(buf), 0.0, buf, 23, buf, 48)
    with pytest.raises(ValueError, match="view pitch"):
        isp_b200.view_compose(raw.view(buf), 0.0, buf, 24, buf, 47)
    bad = abi.RawFrame(raw.data, 8, 2, raw.pitch, abi.RAW10, 12, abi.RGGB)
    with pytest.raises(ValueError, match="bit depth"):
        isp_b200.view_compose(bad.view(buf), 0.0, buf, 24, buf, 48)
