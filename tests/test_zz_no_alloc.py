"""The entry point that allocates no memory, through the C ABI.

isp_b200_process_noalloc serves callers that cannot allocate device memory:
code running where cudaMalloc is forbidden or unsafe, such as a host
framework that owns every allocation or a real-time loop that must not touch
the allocator. Its scratch (tone table, lens shading grid, statistics sums,
white balance state) is one fixed device array inside the library. Two calls
with different frames and settings, queued back to back on one stream with
no wait in between, must give exactly what the regular entry point gives on
a fresh pipeline (the tolerance of the parity tests: none), and the device's
free memory must not move while they run. This file is collected last, so a
failure here comes after every other test has run; it also passes alone in a
fresh process.
"""
import numpy as np
import pytest

import isp_b200
from gpu_support import DeviceFrame, first_mismatch, same_bits, torch_cuda
from isp_b200 import abi, scene

pytestmark = pytest.mark.gpu


def _case(width, height, fmt, bits, black, pattern, seed, **settings):
    counts = scene.mosaic_counts(width, height, pattern, black, (1 << bits) - 1, bits, seed)
    data, pitch = scene.pack(counts, fmt)
    raw = abi.RawFrame(data, width, height, pitch, fmt, bits, pattern)
    params = abi.IspParams(black_level=black, lens_shading=scene.lens_shading_grid(width, height), ccm=scene.CCM,
                           **settings)
    return raw, params


CASES = [
    # RAW10, gray world, Malvar, sharpening, 1024-entry table, 16-bit output.
    (_case(333, 217, abi.RAW10, 10, 64.0, abi.GRBG, 5, white_balance=abi.GRAY_WORLD, demosaic=abi.MALVAR,
           sharpen=0.5, tone_curve=abi.LUT, lut=scene.srgb_table(1024)), abi.RGB16),
    # uint16 12-bit, white patch, bilinear, built-in sRGB (4097 entries), RGBA.
    (_case(200, 150, abi.U16, 12, 256.0, abi.BGGR, 6, white_balance=abi.WHITE_PATCH, demosaic=abi.BILINEAR,
           white_patch_percentile=0.995), abi.RGBA8),
]
EXPOSURE = (12_000_000, 1.0)


def _expected():
    """Each case through the regular entry point, a fresh pipeline each."""
    out = []
    for (raw, params), fmt in CASES:
        frame = DeviceFrame(raw, fmt, True)
        frame.run(isp_b200.Pipeline(params), EXPOSURE)
        out.append(frame.result())
    return out


def _queue_noalloc(frames, stream):
    for ((raw, params), fmt), frame in zip(CASES, frames):
        rv, ov = frame.views()
        isp_b200.process_noalloc(params, rv, ov, frame.hist.data_ptr(), frame.stats.data_ptr(), EXPOSURE, stream)


def test_noalloc_matches_the_regular_entry_point_twice_in_a_row():
    torch = torch_cuda()
    stream = torch.cuda.Stream()
    want = _expected()
    # A first round loads the kernels the calls use; the second is measured.
    for attempt in range(2):
        frames = [DeviceFrame(raw, fmt, True) for (raw, _), fmt in CASES]
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        _queue_noalloc(frames, stream.cuda_stream)  # both calls queued, no wait in between
        stream.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        for f, (frame, w) in enumerate(zip(frames, want)):
            got = frame.result()
            assert same_bits(got.image, w.image), f"round {attempt} case {f}: {first_mismatch(got.image, w.image)}"
            assert np.array_equal(got.histogram, w.histogram), f"round {attempt} case {f}: histogram"
            assert same_bits(got.stats, w.stats), f"round {attempt} case {f}: {got.stats} vs {w.stats}"
        assert isp_b200.noalloc_status(stream.cuda_stream) == 0, "a kernel gave up a bounded wait"
        if attempt == 1:
            assert free_after == free_before, f"device free memory moved by {free_before - free_after} bytes"


def test_noalloc_refuses_tables_beyond_its_array():
    torch_cuda()
    raw, params = CASES[0][0]
    frame = DeviceFrame(raw, abi.RGB8, False)
    rv, ov = frame.views()
    big = abi.IspParams(black_level=64.0, tone_curve=abi.LUT, lut=np.linspace(0, 1, 5000).astype(np.float32))
    with pytest.raises(ValueError, match="at most 4097"):
        isp_b200.process_noalloc(big, rv, ov)


def test_noalloc_queues_nothing_while_its_stream_is_capturing():
    torch = torch_cuda()
    (raw, params), fmt = CASES[0]
    frame = DeviceFrame(raw, fmt, True)
    rv, ov = frame.views()
    stream = torch.cuda.Stream()
    x = torch.zeros(4, device="cuda")
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        x.add_(1.0)
        with pytest.raises(ValueError, match="capturing"):
            isp_b200.process_noalloc(params, rv, ov, frame.hist.data_ptr(), frame.stats.data_ptr(), EXPOSURE,
                                     stream.cuda_stream)
    graph.replay()
    torch.cuda.synchronize()
    assert x.cpu().tolist() == [1.0] * 4
