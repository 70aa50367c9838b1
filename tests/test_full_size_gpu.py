"""The full-size workloads against the oracle, through the C ABI.

c2: 8192x6144 MIPI RAW12 BGGR with white patch (99.5 %), Malvar-He-Cutler,
sharpening 0.5, the colour matrix, the 4096-entry filmic table and RGBA8,
over three consecutive fresh-seed frames queued back to back on one stream,
so that the white patch estimate is smoothed from frame to frame at size
(as pipeline_test.cpp:164-235 runs two frames per case).

c3: the whole 48-camera mixed batch (16 x 640x480 RAW8 RGGB, 16 x 1920x1080
RAW12-in-u16 GBRG, 12 x 3840x2160 RAW10 GRBG, 4 x 4096x3072 RAW16 BGGR), two
batches through the replayed graph, every frame against the oracle run on
the same bytes with each camera's state carried.

Frames are rendered on the device (isp_b200_synthetic_raw) and copied back
for the oracle; every comparison is bit for bit.
"""
import numpy as np
import pytest

import isp_b200
import oracle
from gpu_support import DeviceFrame, first_mismatch, same_bits, torch_cuda
from isp_b200 import abi, scene
from oracle_jobs import run_pool

pytestmark = pytest.mark.gpu


def _render(torch, width, height, fmt, bits, pattern, black, seed):
    """A fresh frame rendered on the device: (device bytes, host RawFrame of the same bytes)."""
    row = abi.raw_row_bytes(fmt, width)
    pitch = (row + 15) // 16 * 16
    data = torch.empty(pitch * height, dtype=torch.uint8, device="cuda")
    isp_b200.synthetic_raw(width, height, fmt, bits, pattern, black, seed, data.data_ptr(), pitch)
    torch.cuda.synchronize()
    return data, abi.RawFrame(data.cpu().numpy(), width, height, pitch, fmt, bits, pattern)


def test_config2_three_fresh_frames_back_to_back_match_oracle():
    torch = torch_cuda()
    w = scene.config2()
    exposure = (20_000_000, 1.5)
    raws = [_render(torch, w.width, w.height, w.fmt, w.bits, w.pattern, w.black, 200 + k)[1] for k in range(3)]
    frames = [DeviceFrame(raw, w.out_format, True) for raw in raws]
    pipe = isp_b200.Pipeline(w.params)
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    for frame in frames:
        frame.run(pipe, exposure, stream.cuda_stream)
    torch.cuda.synchronize()
    ref = oracle.OraclePipeline(w.params)
    for f, (frame, raw) in enumerate(zip(frames, raws)):
        got = frame.result()
        exp = ref.process(raw, w.out_format, True, exposure)
        assert same_bits(got.image, exp.image), f"frame {f}: {first_mismatch(got.image, exp.image)}"
        assert np.array_equal(got.histogram, exp.histogram), f"frame {f}: histogram"
        assert same_bits(got.stats, exp.stats), f"frame {f}: stats {got.stats} vs {exp.stats}"
    gains, valid = pipe.awb()
    rgains, rvalid = ref.awb()
    assert same_bits(gains, rgains) and valid == rvalid == 1, "white patch state after three frames"
    assert pipe.device_status() == 0
    pipe.close()


def test_config3_whole_batch_twice_matches_oracle():
    torch = torch_cuda()
    cams = scene.mixed_cameras(seed=2024)
    assert len(cams) == 48
    exposure = (10_000_000, 1.5)
    stream = torch.cuda.Stream()
    pipes, inputs, sets = [], [], []
    for i, c in enumerate(cams):
        data, raw = _render(torch, c.width, c.height, c.fmt, c.bits, c.pattern, c.black, 7000 + i)
        pipes.append(isp_b200.Pipeline(c.params))
        inputs.append((data, raw))
    for _ in range(2):  # two batches: each camera's second frame follows its first
        sets.append([DeviceFrame(raw, abi.RGB8, True) for _, raw in inputs])
    batch = isp_b200.Batch(len(cams))
    for frames in sets:
        batch.clear()
        for pipe, frame in zip(pipes, frames):
            rv, ov = frame.views()
            batch.add(pipe, rv, ov, frame.hist.data_ptr(), frame.stats.data_ptr(), exposure)
        batch.launch(stream.cuda_stream, True)
    torch.cuda.synchronize()
    got = [[frames[i].result() for frames in sets] for i in range(len(cams))]
    states = [p.awb() for p in pipes]
    batch.close()
    jobs = [(i, c.params, [raw, raw], abi.RGB8, exposure) for i, (c, (_, raw)) in enumerate(zip(cams, inputs))]
    for i, outs, rgains, rvalid in run_pool(jobs):
        c = cams[i]
        for f, (image, hist, stats) in enumerate(outs):
            g = got[i][f]
            what = f"camera {i} ({c.width}x{c.height} format {c.fmt}) frame {f}"
            assert same_bits(g.image, image), f"{what}: {first_mismatch(g.image, image)}"
            assert np.array_equal(g.histogram, hist), f"{what}: histogram"
            assert same_bits(g.stats, stats), f"{what}: stats {g.stats} vs {stats}"
        gains, valid = states[i]
        assert same_bits(gains, rgains) and valid == rvalid, f"camera {i}: white balance state"
