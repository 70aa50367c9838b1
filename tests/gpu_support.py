"""Helpers of the GPU tests: device buffers (torch, plumbing only) around the C ABI."""
from __future__ import annotations

from typing import Optional, Tuple

import numpy as np

import isp_b200
from isp_b200 import abi


def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("no CUDA device")
    return torch


class DeviceFrame:
    """A raw frame uploaded to the device, with poisoned output buffers."""

    def __init__(self, raw: abi.RawFrame, fmt: int, with_stats: bool = True, out_pitch: Optional[int] = None,
                 poison: int = 0xAB):
        torch = torch_cuda()
        self.raw_host = raw
        self.fmt = fmt
        self.raw = torch.from_numpy(raw.data.copy()).cuda()
        ch = abi.output_channels(fmt)
        cb = abi.output_channel_bytes(fmt)
        row = raw.width * ch * cb
        self.out_pitch = row if out_pitch is None else out_pitch
        self.out = torch.full((raw.height * self.out_pitch,), poison, dtype=torch.uint8, device="cuda")
        self.hist = torch.full((abi.HISTOGRAM_CHANNELS * abi.HISTOGRAM_BINS,), 0x5A5A5A5A, dtype=torch.int32,
                               device="cuda") if with_stats else None
        self.stats = torch.full((abi.STATS_SIZE,), float("nan"), dtype=torch.float32,
                                device="cuda") if with_stats else None

    def views(self):
        r = self.raw_host
        raw = abi.RawViewC(self.raw.data_ptr(), r.width, r.height, r.pitch, r.format, r.bit_depth, r.pattern)
        out = abi.RgbViewC(self.out.data_ptr(), self.out_pitch, self.fmt)
        return raw, out

    def run(self, pipe: isp_b200.Pipeline, exposure=(0, 0.0), stream: int = 0) -> None:
        raw, out = self.views()
        pipe.process(raw, out, self.hist.data_ptr() if self.hist is not None else 0,
                     self.stats.data_ptr() if self.stats is not None else 0, exposure, stream)

    def result(self):
        torch = torch_cuda()
        torch.cuda.synchronize()
        r = self.raw_host
        ch = abi.output_channels(self.fmt)
        cb = abi.output_channel_bytes(self.fmt)
        buf = self.out.cpu().numpy().reshape(r.height, self.out_pitch)[:, : r.width * ch * cb]
        image = np.ascontiguousarray(buf).view(abi.output_dtype(self.fmt)).reshape(r.height, r.width, ch)
        hist = self.hist.cpu().numpy().view(np.uint32).reshape(4, 256) if self.hist is not None else None
        stats = self.stats.cpu().numpy() if self.stats is not None else None
        return isp_b200.Result(image, hist, stats)


def run_device(pipe: isp_b200.Pipeline, raw: abi.RawFrame, fmt: int, with_stats: bool = True,
               exposure: Tuple[int, float] = (0, 0.0)):
    f = DeviceFrame(raw, fmt, with_stats)
    f.run(pipe, exposure)
    return f.result()


def same_bits(a: np.ndarray, b: np.ndarray) -> bool:
    return a.shape == b.shape and np.array_equal(np.ascontiguousarray(a).view(np.uint8),
                                                 np.ascontiguousarray(b).view(np.uint8))


def first_mismatch(a: np.ndarray, b: np.ndarray) -> str:
    if a.shape != b.shape:
        return f"shapes {a.shape} vs {b.shape}"
    ia = np.ascontiguousarray(a).view(np.uint8).reshape(a.shape[0], -1)
    ib = np.ascontiguousarray(b).view(np.uint8).reshape(b.shape[0], -1)
    bad = np.argwhere(ia != ib)
    if bad.size == 0:
        return "equal"
    y, xb = bad[0]
    return f"{len(bad)} bytes differ, first at row {y} byte {xb}: {ia[y, xb]} vs {ib[y, xb]}"
