"""Batches: frames of many cameras (uneven sizes, formats, Bayer patterns and
settings) through one launch per pass, directly and as a replayed CUDA graph,
must give every frame the bytes the single-frame path gives it (and so the
reference's): images, histograms, statistics and white balance states, batch
after batch."""
import numpy as np
import pytest

import isp_b200
import oracle
from gpu_support import DeviceFrame, first_mismatch, same_bits, torch_cuda
from isp_b200 import abi, scene

pytestmark = pytest.mark.gpu

# (width, height, raw format, bits, black, pattern, demosaic, sharpen, wb, out, lut entries)
MIX = [
    (64, 40, abi.U8, 8, 16.0, abi.RGGB, abi.BILINEAR, 0.0, abi.MANUAL, abi.RGB8, 1024),
    (200, 150, abi.U16, 12, 256.0, abi.GBRG, abi.MALVAR, 0.0, abi.GRAY_WORLD, abi.RGB8, 1024),
    (333, 217, abi.RAW10, 10, 64.0, abi.GRBG, abi.MALVAR, 0.5, abi.GRAY_WORLD, abi.RGB16, 1024),
    (640, 480, abi.U8, 8, 16.0, abi.RGGB, abi.BILINEAR, 0.0, abi.WHITE_PATCH, abi.RGB8, 512),
    (130, 66, abi.RAW12, 12, 256.0, abi.BGGR, abi.MALVAR, 1.5, abi.WHITE_PATCH, abi.RGBA8, 1024),
    (256, 128, abi.U16, 16, 4096.0, abi.BGGR, abi.BILINEAR, 0.5, abi.MANUAL, abi.RGB32F, 256),
    (96, 64, abi.RAW10, 10, 64.0, abi.GBRG, abi.BILINEAR, 0.0, abi.GRAY_WORLD, abi.RGB8, 1024),
    (1920, 1080, abi.U16, 12, 256.0, abi.GBRG, abi.MALVAR, 0.0, abi.GRAY_WORLD, abi.RGB8, 1024),
    (67, 35, abi.RAW12, 12, 256.0, abi.RGGB, abi.MALVAR, 0.5, abi.MANUAL, abi.RGB16, 1024),
    (500, 300, abi.RAW12, 12, 256.0, abi.GRBG, abi.BILINEAR, 1.0, abi.WHITE_PATCH, abi.RGBA8, 1024),
]


def _params(spec, seed):
    w, h, fmt, bits, black, pattern, dem, sharpen, wb, out, lut_n = spec
    rng = np.random.default_rng(seed)
    lut = scene.srgb_table(lut_n) if seed % 2 == 0 else scene.filmic_table(lut_n)
    return abi.IspParams(black_level=black, lens_shading=scene.lens_shading_grid(w, h), white_balance=wb,
                         wb_gains=(float(rng.uniform(1.2, 2.2)), 1.0, float(rng.uniform(1.1, 1.9))),
                         demosaic=dem, ccm=scene.CCM, tone_curve=abi.LUT, lut=lut, sharpen=sharpen)


def _raw(spec, seed, pitch_pad=0):
    w, h, fmt, bits, black, pattern = spec[:6]
    counts = scene.mosaic_counts(w, h, pattern, black, (1 << bits) - 1, bits, seed)
    row = abi.raw_row_bytes(fmt, w)
    data, pitch = scene.pack(counts, fmt, row + pitch_pad)
    return abi.RawFrame(data, w, h, pitch, fmt, bits, pattern)


_RAWS = {}


def _frame_raws(round_):
    if round_ not in _RAWS:
        # One frame (index 6) has a pitch that rules out TMA, among TMA frames.
        _RAWS[round_] = [_raw(spec, 1000 * round_ + i, 2 if i == 6 else 0) for i, spec in enumerate(MIX)]
    return _RAWS[round_]


def _frames(round_):
    return [DeviceFrame(raw, spec[9], True) for raw, spec in zip(_frame_raws(round_), MIX)]


def _run_batch(use_graph, rounds=2, tune=False, tile_rows=0):
    torch = torch_cuda()
    cams = [isp_b200.Pipeline(_params(spec, i)) for i, spec in enumerate(MIX)]
    batch = isp_b200.Batch(len(MIX))
    if tile_rows:
        batch.set_tile_rows(tile_rows)
    stream = torch.cuda.Stream()
    results = []
    for r in range(rounds):
        frames = _frames(r)
        batch.clear()
        for cam, f in zip(cams, frames):
            rv, ov = f.views()
            batch.add(cam, rv, ov, f.hist.data_ptr(), f.stats.data_ptr(), (8_000_000, 1.5))
        if tune and r == 0:
            batch.autotune(stream.cuda_stream)
        batch.launch(stream.cuda_stream, use_graph)
        torch.cuda.synchronize()
        results.append([(f.result(), cam.awb()) for f, cam in zip(frames, cams)])
        assert all(cam.device_status() == 0 for cam in cams), "a kernel gave up a bounded wait"
    info = batch.info()
    batch.close()
    return results, info


def _run_single(rounds=2):
    cams = [isp_b200.Pipeline(_params(spec, i)) for i, spec in enumerate(MIX)]
    results = []
    for r in range(rounds):
        frames = _frames(r)
        row = []
        for cam, f in zip(cams, frames):
            f.run(cam, (8_000_000, 1.5))
            row.append((f.result(), cam.awb()))
        results.append(row)
    return results


def _compare(got, want):
    for r, (grow, wrow) in enumerate(zip(got, want)):
        for i, ((g, gawb), (w, wawb)) in enumerate(zip(grow, wrow)):
            what = f"batch {r} frame {i} {MIX[i][:3]}"
            assert same_bits(g.image, w.image), f"{what}: {first_mismatch(g.image, w.image)}"
            assert np.array_equal(g.histogram, w.histogram), f"{what}: histogram"
            assert same_bits(g.stats, w.stats), f"{what}: stats {g.stats} vs {w.stats}"
            assert np.array_equal(gawb[0], wawb[0]) and gawb[1] == wawb[1], f"{what}: white balance state"


@pytest.fixture(scope="module")
def single():
    return _run_single()


def test_batch_direct_matches_single_frames(single):
    got, _ = _run_batch(False)
    _compare(got, single)


def test_batch_graph_replays_match_single_frames(single):
    got, info = _run_batch(True, rounds=2)
    _compare(got, single)
    assert info["graph_replays"] == 2 and info["graph_main_ctas"] > 0 and info["graph_awb_ctas"] > 0


def test_batch_after_autotune_matches(single):
    got, info = _run_batch(True, rounds=2, tune=True)
    assert info["tuned"] and info["tile_rows"] in (64, 32) and info["block_threads"] == 256
    _compare(got, single)


@pytest.mark.parametrize("rows", [32, 64])
def test_batch_each_tile_height_matches_single_frames(single, rows):
    got, info = _run_batch(True, rounds=2, tile_rows=rows)
    assert info["tile_rows"] == rows
    _compare(got, single)


def test_batch_matches_oracle():
    """The batch against the C oracle itself, one round (frames and settings as above)."""
    got, _ = _run_batch(True, rounds=1)
    for i, spec in enumerate(MIX):
        ref = oracle.OraclePipeline(_params(spec, i))
        exp = ref.process(_frame_raws(0)[i], spec[9], True, (8_000_000, 1.5))
        g = got[0][i][0]
        assert same_bits(g.image, exp.image), f"frame {i}: {first_mismatch(g.image, exp.image)}"
        assert np.array_equal(g.histogram, exp.histogram) and same_bits(g.stats, exp.stats)


def test_batch_rejects_a_camera_twice():
    torch_cuda()
    cam = isp_b200.Pipeline(_params(MIX[0], 0))
    f = DeviceFrame(_raw(MIX[0], 0), abi.RGB8, True)
    batch = isp_b200.Batch(4)
    rv, ov = f.views()
    batch.add(cam, rv, ov)
    with pytest.raises(ValueError):
        batch.add(cam, rv, ov)
    small = isp_b200.Batch(1)
    small.add(cam, rv, ov)
    with pytest.raises(isp_b200.IspBusy):
        small.add(isp_b200.Pipeline(_params(MIX[0], 0)), rv, ov)
