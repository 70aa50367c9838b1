"""Oracle runs in worker processes, for the full-size GPU tests.

The pool is started with the spawn method (workers never inherit a CUDA
context): each job is one camera's frames through the C oracle, state
carried from frame to frame, returned as plain arrays.
"""
from __future__ import annotations

import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for _path in (ROOT, os.path.join(ROOT, "holoscan-zozo-modules_b200")):
    if _path not in sys.path:
        sys.path.insert(0, _path)


def camera_frames(job):
    """job = (key, params, raws, out_format, exposure): every raw frame of one
    camera in turn; returns (key, [(image, histogram, stats), ...], awb gains, valid)."""
    import oracle

    key, params, raws, fmt, exposure = job
    pipe = oracle.OraclePipeline(params)
    outs = []
    for raw in raws:
        r = pipe.process(raw, fmt, True, exposure)
        outs.append((r.image, r.histogram, r.stats))
    gains, valid = pipe.awb()
    return key, outs, gains, valid


def run_pool(jobs, workers: int = 0):
    """Runs camera_frames over `jobs` in a spawn pool; results in job order."""
    import multiprocessing as mp

    workers = workers or max(1, min(len(jobs), os.cpu_count() or 1, 16))
    with mp.get_context("spawn").Pool(workers) as pool:
        return pool.map(camera_frames, jobs)
