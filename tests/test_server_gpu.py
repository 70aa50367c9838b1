"""Serving: camera streams through the continuous-batching server.

Each stream's frames, submitted interleaved with other streams' frames and
batched with them, must come out exactly as the same frames processed alone
in order by their own pipeline (the white balance smoothing chains across a
stream's frames). Admission against the memory budget, refusals when a
stream's queue is full (host-side failure injection: the submit is turned
away, nothing reaches the GPU) and a short Poisson-arrival run with latency
percentiles are checked too."""
import numpy as np
import pytest

import isp_b200
from isp_b200 import abi, scene

pytestmark = pytest.mark.gpu

# (width, height, format, bits, black, pattern, wb, demosaic, sharpen, out)
STREAMS = [
    (640, 480, abi.U8, 8, 16.0, abi.RGGB, abi.GRAY_WORLD, abi.BILINEAR, 0.0, abi.RGB8),
    (320, 180, abi.U16, 12, 256.0, abi.GBRG, abi.WHITE_PATCH, abi.MALVAR, 0.0, abi.RGB8),
    (384, 216, abi.RAW10, 10, 64.0, abi.GRBG, abi.GRAY_WORLD, abi.MALVAR, 0.5, abi.RGB16),
    (256, 192, abi.U16, 16, 4096.0, abi.BGGR, abi.MANUAL, abi.BILINEAR, 0.0, abi.RGBA8),
    (130, 66, abi.RAW12, 12, 256.0, abi.BGGR, abi.WHITE_PATCH, abi.MALVAR, 1.0, abi.RGB32F),
    (200, 150, abi.U8, 8, 16.0, abi.GRBG, abi.MANUAL, abi.MALVAR, 0.0, abi.RGB8),
]


def _params(spec, i):
    w, h, fmt, bits, black, pattern, wb, dem, sharpen, out = spec
    lut = scene.srgb_table(1024) if i % 2 == 0 else scene.filmic_table(1024)
    return abi.IspParams(black_level=black, lens_shading=scene.lens_shading_grid(w, h), white_balance=wb,
                         wb_gains=(1.7, 1.0, 1.4), demosaic=dem, ccm=scene.CCM, tone_curve=abi.LUT, lut=lut,
                         sharpen=sharpen)


def _raw(spec, seed):
    w, h, fmt, bits, black, pattern = spec[:6]
    counts = scene.mosaic_counts(w, h, pattern, black, (1 << bits) - 1, bits, seed)
    data, pitch = scene.pack(counts, fmt)
    return abi.RawFrame(data, w, h, pitch, fmt, bits, pattern)


def _buffers(spec):
    w, h, out = spec[0], spec[1], spec[9]
    img = np.zeros((h, w, abi.output_channels(out)), abi.output_dtype(out))
    return img, np.zeros((4, 256), np.uint32), np.zeros(12, np.float32)


@pytest.mark.parametrize("per_frame", [False, True], ids=["batched", "per_frame"])
def test_each_stream_is_the_same_alone_and_in_the_mix(per_frame):
    frames = 3
    raws = [[_raw(spec, 100 * i + k) for k in range(frames)] for i, spec in enumerate(STREAMS)]
    # Alone: each stream's frames in order through its own pipeline.
    alone = []
    for i, spec in enumerate(STREAMS):
        pipe = isp_b200.Pipeline(_params(spec, i))
        alone.append([pipe.process_host(raws[i][k], spec[9], True) for k in range(frames)])
        pipe.close()
    # In the mix: interleaved submissions to the server.
    server = isp_b200.Server(max_batch=8, max_inflight=2, queue_depth=frames, slots_per_stream=2, per_frame=per_frame)
    ids = [server.add_stream(_params(spec, i), *spec[:3], spec[3], spec[5], spec[9]) for i, spec in enumerate(STREAMS)]
    server.start()
    outs = [[_buffers(spec) for _ in range(frames)] for spec in STREAMS]
    for k in range(frames):
        for i in range(len(STREAMS)):
            img, hist, st = outs[i][k]
            server.submit(ids[i], raws[i][k], img, hist, st)
    server.drain(60.0)
    results = server.poll(1024)
    stats = server.stats()
    server.close()
    assert stats["completed"] == len(STREAMS) * frames and stats["error"] == 0
    assert len(results) == len(STREAMS) * frames
    for i, spec in enumerate(STREAMS):
        for k in range(frames):
            img, hist, st = outs[i][k]
            want = alone[i][k]
            assert np.array_equal(img.view(np.uint8), want.image.view(np.uint8)), f"stream {i} frame {k}: image"
            assert np.array_equal(hist, want.histogram), f"stream {i} frame {k}: histogram"
            assert np.array_equal(st.view(np.uint32), want.stats.view(np.uint32)), f"stream {i} frame {k}: stats"
    # Frames of a stream complete in arrival order.
    for i in range(len(STREAMS)):
        order = [r.frame for r in results if r.stream == ids[i]]
        assert order == sorted(order)


def test_admission_budget_of_one_frame_still_completes_everything():
    spec = STREAMS[0]
    raw = _raw(spec, 7)
    frame_bytes = abi.raw_row_bytes(spec[2], spec[0]) * spec[1] + spec[0] * spec[1] * 3
    server = isp_b200.Server(max_batch=8, max_inflight=2, queue_depth=4, slots_per_stream=2,
                             memory_budget=frame_bytes + 4096)
    a = server.add_stream(_params(spec, 0), *spec[:3], spec[3], spec[5], spec[9])
    b = server.add_stream(_params(spec, 1), *spec[:3], spec[3], spec[5], spec[9])
    server.start()
    for _ in range(3):
        server.submit(a, raw)
        server.submit(b, raw)
    server.drain(60.0)
    st = server.stats()
    server.close()
    assert st["completed"] == 6 and st["refused"] == 0 and st["error"] == 0
    assert st["mean_batch_frames"] == 1.0  # the budget admits one frame at a time


def test_full_queue_refuses_frames():
    spec = STREAMS[2]
    raw = _raw(spec, 9)
    server = isp_b200.Server(max_batch=4, max_inflight=1, queue_depth=1, slots_per_stream=1)
    sid = server.add_stream(_params(spec, 2), *spec[:3], spec[3], spec[5], spec[9])
    server.start()
    refused = 0
    for _ in range(40):
        try:
            server.submit(sid, raw)
        except isp_b200.IspBusy:
            refused += 1
    server.drain(60.0)
    st = server.stats()
    server.close()
    assert refused > 0 and st["refused"] == refused
    assert st["completed"] == st["submitted"] - refused


def test_poisson_arrivals_report_latency_percentiles():
    server = isp_b200.Server(max_batch=16, max_inflight=2, queue_depth=4, slots_per_stream=2)
    ids = [server.add_stream(_params(spec, i), *spec[:3], spec[3], spec[5], spec[9]) for i, spec in enumerate(STREAMS)]
    for i, spec in zip(ids, STREAMS):
        server.add_source(i, _raw(spec, 55 + i))
        server.add_source(i, _raw(spec, 56 + i))
    server.start()
    server.run_poisson([60.0] * len(ids), 0.5, seed=3)
    server.drain(60.0)
    st = server.stats()
    server.close()
    assert st["error"] == 0 and st["completed"] > 50
    assert 0.0 < st["p50_ms"] <= st["p99_ms"] <= st["p999_ms"] <= st["max_ms"]
    assert st["gpix_per_s"] > 0.0


def test_device_arrivals_match_host_arrivals():
    """Frames submitted in device memory (read in place) give the same results
    as the same frames submitted from host memory."""
    torch = pytest.importorskip("torch")
    frames = 2
    raws = [[_raw(spec, 300 + 10 * i + k) for k in range(frames)] for i, spec in enumerate(STREAMS)]
    results = {}
    for on_device in (False, True):
        server = isp_b200.Server(max_batch=8, max_inflight=2, queue_depth=frames, slots_per_stream=2)
        ids = [server.add_stream(_params(spec, i), *spec[:3], spec[3], spec[5], spec[9])
               for i, spec in enumerate(STREAMS)]
        server.start()
        keep = []
        outs = [[_buffers(spec) for _ in range(frames)] for spec in STREAMS]
        for k in range(frames):
            for i in range(len(STREAMS)):
                img, hist, st = outs[i][k]
                raw = raws[i][k]
                if on_device:
                    d = torch.from_numpy(raw.data.reshape(-1).copy()).cuda()
                    keep.append(d)
                    torch.cuda.synchronize()
                    server.submit_device(ids[i], d.data_ptr(), raw.pitch, img, hist, st)
                else:
                    server.submit(ids[i], raw, img, hist, st)
        server.drain(60.0)
        assert server.stats()["error"] == 0
        server.close()
        results[on_device] = outs
    for i in range(len(STREAMS)):
        for k in range(frames):
            for a, b in zip(results[False][i][k], results[True][i][k]):
                assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), f"stream {i} frame {k}"


@pytest.mark.parametrize("on_device", [False, True], ids=["host_sources", "device_sources"])
def test_closed_loop_saturation_completes_frames(on_device):
    server = isp_b200.Server(max_batch=16, max_inflight=2, queue_depth=2, slots_per_stream=2)
    ids = [server.add_stream(_params(spec, i), *spec[:3], spec[3], spec[5], spec[9], copy_back=True)
           for i, spec in enumerate(STREAMS)]
    for i, spec in zip(ids, STREAMS):
        server.add_source(i, _raw(spec, 70 + i), on_device)
    server.start()
    server.run_closed(0.5)
    server.drain(60.0)
    st = server.stats()
    server.close()
    assert st["error"] == 0 and st["refused"] == 0
    assert st["completed"] == st["submitted"] > len(STREAMS)
    assert st["mean_batch_frames"] > 1.0  # queues stay full: batches carry several streams
