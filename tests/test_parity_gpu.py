"""Parity of the sm_100a kernels with the reference CPU backend, through the C ABI.

Every golden fixture (the reference's own outputs, tests/golden/) is replayed
frame after frame through libisp_b200.so, in device memory and in host
memory; every image byte, histogram bin, statistic (the auto-exposure fields
included) and white balance state must be identical. The full-size
workloads are checked against the C oracle run on the same bytes.
Case lists follow modules/isp/tests/pipeline_test.cpp.
"""
import numpy as np
import pytest

import isp_b200
import oracle
from goldens import CASES, load_case
from gpu_support import DeviceFrame, first_mismatch, run_device, same_bits, torch_cuda
from isp_b200 import abi, scene

pytestmark = pytest.mark.gpu


def _check(name, f, got, expected, with_stats):
    assert same_bits(got.image, expected["image"]), f"{name} frame {f}: image {first_mismatch(got.image, expected['image'])}"
    if with_stats:
        assert np.array_equal(got.histogram, expected["hist"]), f"{name} frame {f}: histogram differs"
        bad = np.nonzero(got.stats.view(np.uint32) != expected["stats"].view(np.uint32))[0]
        assert bad.size == 0, f"{name} frame {f}: stats {bad.tolist()}: {got.stats[bad]} vs {expected['stats'][bad]}"


@pytest.mark.parametrize("name", CASES)
def test_device_matches_reference(name):
    case = load_case(name)
    pipe = isp_b200.Pipeline(case.params)
    for f, raw in enumerate(case.frame_raws()):
        got = run_device(pipe, raw, case.out_format, case.with_stats, case.exposure)
        _check(name, f, got, case.expected[f], case.with_stats)
        gains, valid = pipe.awb()
        assert np.array_equal(np.array([*gains.view(np.uint32), valid], np.uint32), case.expected[f]["awb"])
    assert pipe.device_status() == 0, "a kernel gave up a bounded wait"
    pipe.close()


@pytest.mark.parametrize("name", CASES)
def test_short_tiles_match_reference(name):
    """Every golden fixture again through the 32-row tile pass (three CTAs per SM)."""
    case = load_case(name)
    pipe = isp_b200.Pipeline(case.params)
    pipe.set_tile_rows(32)
    for f, raw in enumerate(case.frame_raws()):
        got = run_device(pipe, raw, case.out_format, case.with_stats, case.exposure)
        _check(name, f, got, case.expected[f], case.with_stats)
        gains, valid = pipe.awb()
        assert np.array_equal(np.array([*gains.view(np.uint32), valid], np.uint32), case.expected[f]["awb"])
    assert pipe.device_status() == 0
    pipe.close()


def test_autotune_picks_a_height_per_shape_and_leaves_no_trace():
    """isp_b200_autotune times both tile heights on a frame, keeps the faster
    for that shape and puts the white balance state back: the frames after it
    are the reference's first frames, at whichever height it picked."""
    torch = torch_cuda()
    case = load_case("malvar_gray_world")
    pipe = isp_b200.Pipeline(case.params)
    stream = torch.cuda.Stream()
    raws = case.frame_raws()
    tune = DeviceFrame(raws[0], case.out_format, True)
    rv, ov = tune.views()
    rows = pipe.autotune(rv, ov, tune.hist.data_ptr(), tune.stats.data_ptr(), case.exposure, stream.cuda_stream)
    assert rows in (64, 32)
    assert pipe.awb()[1] == 0, "the white balance state is the fresh pipeline's again"
    for f, raw in enumerate(raws):
        got = run_device(pipe, raw, case.out_format, case.with_stats, case.exposure)
        _check("malvar_gray_world", f, got, case.expected[f], case.with_stats)
    with pytest.raises(ValueError, match="tile_rows"):
        pipe.set_tile_rows(48)
    pipe.close()


@pytest.mark.parametrize("name", [n for n in CASES if not n.startswith(("sweep_", "edge_"))])
def test_host_buffers_match_reference(name):
    case = load_case(name)
    pipe = isp_b200.Pipeline(case.params)
    for f, raw in enumerate(case.frame_raws()):
        got = pipe.process_host(raw, case.out_format, case.with_stats, case.exposure)
        _check(name, f, got, case.expected[f], case.with_stats)
    pipe.close()


def test_two_streams_in_call_order():
    """two_streams (pipeline_test.cpp:270-362): frames queued on two streams in
    turn, never waited for in between, come out as the reference's in call order."""
    torch = torch_cuda()
    case = load_case("sequence_two_streams")
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    pipe = isp_b200.Pipeline(case.params)
    frames = [DeviceFrame(raw, case.out_format, True) for raw in case.frame_raws()]
    torch.cuda.synchronize()
    for f, frame in enumerate(frames):
        frame.run(pipe, case.exposure, streams[f % 2].cuda_stream)
    torch.cuda.synchronize()
    for f, frame in enumerate(frames):
        _check("two_streams", f, frame.result(), case.expected[f], True)


@pytest.mark.parametrize("overlap", [True, False])
@pytest.mark.parametrize("name", ["sequence_two_streams", "awb_smoothing", "malvar_gray_world", "white_patch_sharp_rgba"])
def test_frames_back_to_back_on_one_stream(name, overlap):
    """Frames of one camera queued on one stream with nothing in between: each
    frame's statistics pass may overlap the previous frame's tile pass (frame
    overlap on) or follow it (off); either way every frame, white balance
    smoothing included, is the reference's."""
    torch = torch_cuda()
    case = load_case(name)
    stream = torch.cuda.Stream()
    pipe = isp_b200.Pipeline(case.params)
    pipe.set_frame_overlap(overlap)
    frames = [DeviceFrame(raw, case.out_format, case.with_stats) for raw in case.frame_raws()]
    torch.cuda.synchronize()
    for frame in frames:
        frame.run(pipe, case.exposure, stream.cuda_stream)
    torch.cuda.synchronize()
    for f, frame in enumerate(frames):
        _check(name, f, frame.result(), case.expected[f], case.with_stats)
    gains, valid = pipe.awb()
    assert np.array_equal(np.array([*gains.view(np.uint32), valid], np.uint32), case.expected[-1]["awb"])
    assert pipe.device_status() == 0
    pipe.close()


def test_determinism_and_fresh_instances():
    """determinism (pipeline_test.cpp:621-634)."""
    case = load_case("malvar_sharpened")
    raw = case.raws[0]
    first = run_device(isp_b200.Pipeline(case.params), raw, abi.RGB8)
    for _ in range(3):
        again = run_device(isp_b200.Pipeline(case.params), raw, abi.RGB8)
        assert same_bits(again.image, first.image) and np.array_equal(again.histogram, first.histogram)
        assert same_bits(again.stats, first.stats)


def test_histograms_count_the_output_pixels():
    """histograms_count_pixels (pipeline_test.cpp:239-265), rebuilt from the image."""
    case = load_case("bilinear_sharpened")
    for fmt in (abi.RGB8, abi.RGBA8):
        r = run_device(isp_b200.Pipeline(case.params), case.raws[0], fmt)
        img = r.image.reshape(-1, abi.output_channels(fmt)).astype(np.int64)
        luma = (2126 * img[:, 0] + 7152 * img[:, 1] + 722 * img[:, 2] + 5000) // 10000
        rebuilt = np.stack([np.bincount(luma, minlength=256), np.bincount(img[:, 0], minlength=256),
                            np.bincount(img[:, 1], minlength=256), np.bincount(img[:, 2], minlength=256)])
        assert np.array_equal(rebuilt, r.histogram)


def test_padded_output_rows_untouched():
    """Output rows padded beyond the pixels: padding keeps its bytes."""
    case = load_case("malvar_odd_size")
    raw = case.raws[0]
    pitch = raw.width * 6 + 26
    f = DeviceFrame(raw, abi.RGB16, True, out_pitch=pitch)
    f.run(isp_b200.Pipeline(case.params), case.exposure)
    got = f.result()
    assert same_bits(got.image, case.expected[0]["image"])
    full = f.out.cpu().numpy().reshape(raw.height, pitch)
    assert np.all(full[:, raw.width * 6:] == 0xAB)


def test_rejects_before_launch():
    """rejects (pipeline_test.cpp:723-744): bad views raise ValueError, nothing queued."""
    torch = torch_cuda()
    pipe = isp_b200.Pipeline(abi.IspParams())
    buf = torch.zeros(64, dtype=torch.uint8, device="cuda")
    out = torch.zeros(4 * 4 * 3, dtype=torch.uint8, device="cuda")
    good = abi.RawViewC(buf.data_ptr(), 4, 4, 8, abi.U16, 12, abi.RGGB)
    rgb = abi.RgbViewC(out.data_ptr(), 12, abi.RGB8)
    pipe.process(good, rgb)
    torch.cuda.synchronize()
    for field, value in (("width", 1), ("pitch", 6), ("bit_depth", 17), ("format", abi.RAW10), ("data", None)):
        v = abi.RawViewC(good.data, 4, 4, 8, abi.U16, 12, abi.RGGB)
        setattr(v, field, value)
        with pytest.raises(ValueError):
            pipe.process(v, rgb)
    with pytest.raises(ValueError):
        pipe.process(good, abi.RgbViewC(out.data_ptr(), 6, abi.RGB8))


@pytest.fixture(scope="module")
def full_size_frames():
    frames = {}
    for make in (scene.config0, scene.config1):
        w = make()
        frames[w.name] = (w, w.raw(7))
    return frames


@pytest.mark.parametrize("rows", [64, 32])
@pytest.mark.parametrize("which", ["c0_1080p_u16_rggb_bilinear", "c1_4k_raw10_grbg_malvar_sharpen"])
def test_full_size_configs_match_oracle(full_size_frames, which, rows):
    w, raw = full_size_frames[which]
    pipe = isp_b200.Pipeline(w.params)
    pipe.set_tile_rows(rows)
    ref = oracle.OraclePipeline(w.params)
    for f in range(2):  # two frames: the white balance smoothing runs too
        got = run_device(pipe, raw, w.out_format, True, (10_000_000, 2.0))
        exp = ref.process(raw, w.out_format, True, (10_000_000, 2.0))
        assert same_bits(got.image, exp.image), f"{which} frame {f}: {first_mismatch(got.image, exp.image)}"
        assert np.array_equal(got.histogram, exp.histogram)
        assert same_bits(got.stats, exp.stats), f"{got.stats} vs {exp.stats}"


def test_a_bounded_wait_that_runs_out_is_reported_and_the_next_frame_is_clean():
    """The kernels' barrier waits are bounded: a wait that runs out returns,
    flags the camera (isp_b200_device_status reads 1 once), and leaves the
    context and the pipeline usable. The check kernel waits on a barrier that
    no copy completes; no GPU fault is involved."""
    torch = torch_cuda()
    case = load_case("malvar_gray_world")
    pipe = isp_b200.Pipeline(case.params)
    stream = torch.cuda.Stream()
    pipe.check_bounded_wait(256, stream.cuda_stream)
    assert pipe.device_status() == 1
    assert pipe.device_status() == 0, "the status is cleared once read"
    for f, raw in enumerate(case.frame_raws()):
        got = run_device(pipe, raw, case.out_format, case.with_stats, case.exposure)
        _check("malvar_gray_world", f, got, case.expected[f], case.with_stats)
    assert pipe.device_status() == 0
    with pytest.raises(ValueError, match="polls must be"):
        pipe.check_bounded_wait(0)
    pipe.close()
