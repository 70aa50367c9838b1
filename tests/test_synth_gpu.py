"""Seeded synthetic raw frames rendered on the device (isp_b200_synthetic_raw):
deterministic per seed, the same counts in every packing, the noise-free
scene equal (to within a count, the device's expf against numpy's) to a
numpy restatement of the documented scene model drawn from the same SplitMix64
stream, and shot plus read noise with the documented mean and variance."""
import numpy as np
import pytest

import isp_b200
from isp_b200 import abi

pytestmark = pytest.mark.gpu
M64 = (1 << 64) - 1


def mix64(z):
    z = (z + 0x9E3779B97F4A7C15) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def f32(x):
    return np.float32(x)


class Draw:
    def __init__(self, seed):
        self.state = seed & M64

    def uniform(self, lo, hi):
        self.state = mix64(self.state)
        u = f32(f32(self.state >> 40) * f32(5.9604645e-8))
        return f32(f32(lo) + f32(f32(f32(hi) - f32(lo)) * u))


COLOUR = {abi.RGGB: (0, 1, 1, 2), abi.BGGR: (2, 1, 1, 0), abi.GRBG: (1, 0, 2, 1), abi.GBRG: (1, 2, 0, 1)}


def restated_counts(width, height, pattern, bits, black, seed, edge=0.5):
    """The noise-free frame by the scene model of isp_synth.cu, in float32."""
    d = Draw(seed)
    w, h = f32(width), f32(height)
    base = [d.uniform(0.05, 0.35) for _ in range(3)]
    gx = [f32(d.uniform(-0.25, 0.25) / max(f32(w - f32(1)), f32(1))) for _ in range(3)]
    gy = [f32(d.uniform(-0.25, 0.25) / max(f32(h - f32(1)), f32(1))) for _ in range(3)]
    blobs = []
    for _ in range(8):
        bx, by = d.uniform(0.0, w), d.uniform(0.0, h)
        sigma = d.uniform(50.0, 300.0)
        k = f32(f32(-1.0) / f32(f32(2.0) * sigma * sigma))
        blobs.append((bx, by, k, [d.uniform(0.05, 0.5) for _ in range(3)]))
    rects = []
    for _ in range(64):
        rw = int(d.uniform(0.02, 0.2) * w) + 1
        rh = int(d.uniform(0.02, 0.2) * h) + 1
        x0 = int(d.uniform(0.0, max(f32(w - f32(rw)), f32(1.0))))
        y0 = int(d.uniform(0.0, max(f32(h - f32(rh)), f32(1.0))))
        rects.append((x0, y0, x0 + rw, y0 + rh, [d.uniform(0.0, 1.0) for _ in range(3)]))
    ys, xs = np.mgrid[0:height, 0:width]
    fx, fy = xs.astype(np.float32), ys.astype(np.float32)
    chan = np.array(COLOUR[pattern])[((ys & 1) << 1) | (xs & 1)]
    v = np.zeros((height, width), np.float32)
    for c in range(3):
        vc = (base[c] + gx[c] * fx) + gy[c] * fy
        for bx, by, k, amp in blobs:
            vc = vc + amp[c] * np.exp(((fx - bx) * (fx - bx) + (fy - by) * (fy - by)) * k)
        for x0, y0, x1, y1, rgb in rects:
            vc[y0:y1, x0:x1] = rgb[c]
        v = np.where(chan == c, vc, v)
    v = np.clip(v, 0, 1).astype(np.float32)
    cx, cy = f32((w - 1) / 2), f32((h - 1) / 2)
    inv_rc = f32(1) / f32(np.hypot(cx, cy))
    tan_edge = f32(np.tan(np.arccos(f32(edge) ** f32(0.25))))
    dxc, dyc = (fx - cx) * inv_rc, (fy - cy) * inv_rc
    u2 = (dxc * dxc + dyc * dyc) * tan_edge * tan_edge
    vig = f32(1) / ((f32(1) + u2) * (f32(1) + u2))
    white = (1 << bits) - 1
    counts = np.rint(f32(black) + v * vig * f32(white - black))
    return np.clip(counts, 0, white).astype(np.int64)


def _render(torch, width, height, fmt, bits, pattern, black, seed, **noise):
    pitch = abi.raw_row_bytes(fmt, width)
    buf = torch.zeros(pitch * height, dtype=torch.uint8, device="cuda")
    isp_b200.synthetic_raw(width, height, fmt, bits, pattern, black, seed, buf.data_ptr(), pitch, **noise)
    torch.cuda.synchronize()
    return buf.cpu().numpy().reshape(height, pitch)


def _unpack(data, fmt, width):
    d = data.astype(np.int64)
    if fmt == abi.U8:
        return d[:, :width]
    if fmt == abi.U16:
        return (d[:, 0:2 * width:2] | (d[:, 1:2 * width:2] << 8))
    if fmt == abi.RAW10:
        g = d[:, :5 * ((width + 3) // 4)].reshape(d.shape[0], -1, 5)
        out = np.stack([(g[:, :, k] << 2) | ((g[:, :, 4] >> (2 * k)) & 3) for k in range(4)], axis=2)
        return out.reshape(d.shape[0], -1)[:, :width]
    g = d[:, :3 * ((width + 1) // 2)].reshape(d.shape[0], -1, 3)
    out = np.stack([(g[:, :, 0] << 4) | (g[:, :, 2] & 15), (g[:, :, 1] << 4) | (g[:, :, 2] >> 4)], axis=2)
    return out.reshape(d.shape[0], -1)[:, :width]


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    if not t.cuda.is_available():
        pytest.skip("no CUDA device")
    return t


def test_deterministic_per_seed(torch):
    a = _render(torch, 257, 131, abi.RAW10, 10, abi.GRBG, 64.0, 7)
    b = _render(torch, 257, 131, abi.RAW10, 10, abi.GRBG, 64.0, 7)
    c = _render(torch, 257, 131, abi.RAW10, 10, abi.GRBG, 64.0, 8)
    assert np.array_equal(a, b) and not np.array_equal(a, c)


@pytest.mark.parametrize("fmt,bits", [(abi.RAW10, 10), (abi.RAW12, 12), (abi.U8, 8)])
def test_packings_carry_the_same_counts(torch, fmt, bits):
    w, h = 203, 77
    ref = _unpack(_render(torch, w, h, abi.U16, bits, abi.BGGR, 16.0, 11), abi.U16, w)
    got = _unpack(_render(torch, w, h, fmt, bits, abi.BGGR, 16.0, 11), fmt, w)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("pattern", [abi.RGGB, abi.GBRG])
def test_noise_free_scene_matches_its_restatement(torch, pattern):
    w, h, bits, black = 320, 200, 12, 256.0
    got = _unpack(_render(torch, w, h, abi.U16, bits, pattern, black, 2024, gain=0.0, read_noise=0.0), abi.U16, w)
    exp = restated_counts(w, h, pattern, bits, black, 2024)
    diff = np.abs(got - exp)
    assert diff.max() <= 1, f"max difference {diff.max()} counts"
    assert (diff == 0).mean() > 0.95


def test_noise_has_the_documented_moments(torch):
    w, h, bits, black = 512, 256, 12, 256.0
    clean = _unpack(_render(torch, w, h, abi.U16, bits, abi.RGGB, black, 5, gain=0.0, read_noise=0.0), abi.U16, w)
    noisy = _unpack(_render(torch, w, h, abi.U16, bits, abi.RGGB, black, 5, gain=0.5, read_noise=3.0), abi.U16, w)
    inside = (clean > black + 8) & (clean < (1 << bits) - 200)  # away from the clips
    delta = (noisy - clean)[inside].astype(np.float64)
    expected_var = (0.5 * (clean[inside] - black) + 9.0).mean()
    assert abs(delta.mean()) < 0.2
    assert delta.var() == pytest.approx(expected_var, rel=0.05)


def test_rejects_unusable_settings(torch):
    buf = torch.zeros(64, dtype=torch.uint8, device="cuda")
    with pytest.raises(ValueError):
        isp_b200.synthetic_raw(4, 4, abi.U16, 17, abi.RGGB, 0.0, 1, buf.data_ptr(), 8)
    with pytest.raises(ValueError):
        isp_b200.synthetic_raw(4, 4, abi.U16, 12, abi.RGGB, 5000.0, 1, buf.data_ptr(), 8)
