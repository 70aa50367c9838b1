"""The reference's own CUDA backend (IspPipeline(Backend::kCuda), built for
sm_100a from its sources into oracle/_ref/libisp_ref_cuda.so) against the B200
build on the same device frames: images and histograms byte for byte, frame
after frame (white balance state carried). A second witness beside the CPU
oracle; the statistics' auto-exposure fields are left out, since the
reference allows its own CUDA backend 1e-5 there (pipeline_test.cpp:224-231).
Skipped where the reference build is absent."""
from __future__ import annotations

import numpy as np
import pytest

import isp_b200
import oracle
from goldens import CASES, load_case
from isp_b200 import abi
from gpu_support import DeviceFrame

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.reference_cuda_available(), reason="reference CUDA build absent")]


def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("no CUDA device")
    return torch


def test_reference_cuda_backend_agrees():
    torch = torch_cuda()
    bad = []
    for name in CASES:
        case = load_case(name)
        ours = isp_b200.Pipeline(case.params)
        theirs = oracle.ReferenceCudaPipeline(case.params)
        for f, raw in enumerate(case.frame_raws()):
            a = DeviceFrame(raw, case.out_format, True)
            b = DeviceFrame(raw, case.out_format, True)
            a.run(ours, case.exposure)
            rv, ov = b.views()
            st = abi.StatsC(b.hist.data_ptr(), b.stats.data_ptr())
            theirs.process(rv, ov, st, abi.ExposureC(*case.exposure), 0)
            torch.cuda.synchronize()
            if not (torch.equal(a.out, b.out) and torch.equal(a.hist, b.hist)):
                bad.append((name, f))
        theirs.close()
        ours.close()
    assert not bad, bad[:10]
