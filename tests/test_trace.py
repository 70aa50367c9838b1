"""Tracing: the library's host-side phases are NVTX ranges in the domain
"holoscan.isp" (frame submission, the statistics and tile pass launches, host
staging, batch build and replay, the serving loop, the converter and the
view), seen by any
tool that NVTX loads. The tool here is tests/nvtx_probe.c, an NVTX injection
library that records every range; each case runs in a child process so that
NVTX loads it at the process's first NVTX call."""
import json
import os
import subprocess
import sys
import textwrap

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA_INCLUDE = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("nvtx") / "nvtx_probe.so")
    subprocess.run(["gcc", "-O2", "-shared", "-fPIC", "-I", CUDA_INCLUDE, os.path.join(ROOT, "tests", "nvtx_probe.c"),
                    "-o", out, "-lpthread"], check=True)
    return out


_PRELUDE = """
import ctypes as C, json, os, sys
ROOT = {root!r}
for p in (ROOT, os.path.join(ROOT, "holoscan-zozo-modules_b200"), os.path.join(ROOT, "tests")):
    sys.path.insert(0, p)

def dump_ranges():
    p = C.CDLL(os.environ["NVTX_INJECTION64_PATH"])
    p.nvtx_probe_dump.restype = C.c_long
    buf = C.create_string_buffer(1 << 20)
    n = p.nvtx_probe_dump(buf, len(buf))
    lines = [l.split("\\t") for l in buf.value.decode().splitlines()] if n >= 0 else None
    print(json.dumps({{"lines": lines}}))
"""


def run_traced(probe_path, body, tmp_path, timeout=600):
    script = tmp_path / "traced.py"
    script.write_text(_PRELUDE.format(root=ROOT) + textwrap.dedent(body) + "\ndump_ranges()\n")
    env = dict(os.environ, NVTX_INJECTION64_PATH=probe_path)
    res = subprocess.run([sys.executable, str(script)], env=env, capture_output=True, text=True, timeout=timeout)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-4000:]
    lines = json.loads(res.stdout.strip().splitlines()[-1])["lines"]
    assert lines is not None, "the probe's record overflowed"
    return lines


def ranges_of(lines, domain="holoscan.isp"):
    """The domain's ranges as nested (name, children) trees per thread, in
    order; fails on a pop without a push or a range left open."""
    stacks, roots = {}, {}
    for kind, dom, thread, message in lines:
        if dom != domain:
            continue
        stack = stacks.setdefault(thread, [])
        if kind == "push":
            node = (message, [])
            (stack[-1][1] if stack else roots.setdefault(thread, [])).append(node)
            stack.append(node)
        else:
            assert stack, f"pop without a push on thread {thread}"
            stack.pop()
    for thread, stack in stacks.items():
        assert not stack, f"ranges left open on thread {thread}: {[n for n, _ in stack]}"
    return [node for thread in roots for node in roots[thread]]


def test_ranges_reach_an_injected_tool(probe, tmp_path):
    """Entry points whose first step is the range (the converter, the view)
    open and close it in the library's domain even when they refuse their
    arguments: no GPU is needed."""
    lines = run_traced(probe, """
        lib = C.CDLL(os.path.join(ROOT, "holoscan-zozo-modules_b200", "libisp_b200.so"))
        lib.cc_b200_convert.argtypes = [C.c_void_p] * 4
        assert lib.cc_b200_convert(None, None, None, None) != 0
        lib.isp_b200_view_compose.argtypes = [C.c_void_p, C.c_float, C.c_void_p, C.c_size_t, C.c_void_p,
                                              C.c_size_t, C.c_void_p]
        assert lib.isp_b200_view_compose(None, 0.0, None, 0, None, 0, None) != 0
    """, tmp_path)
    assert ranges_of(lines) == [("cc.convert", []), ("isp.view", [])]


@pytest.mark.gpu
def test_frame_phases_are_ranges(probe, tmp_path):
    """A frame with auto white balance is one isp.process range holding its
    statistics pass and tile pass launches; isp_b200_process_host wraps it in
    the upload and the download; a batch launch holds its build and its graph
    replay (or its direct launches)."""
    lines = run_traced(probe, """
        import numpy as np
        import torch
        import isp_b200
        from gpu_support import DeviceFrame
        from isp_b200 import abi, scene

        w, h = 320, 200
        params = abi.IspParams(black_level=64.0, white_balance=abi.GRAY_WORLD, demosaic=abi.MALVAR, sharpen=0.5,
                               ccm=scene.CCM, lens_shading=scene.lens_shading_grid(w, h))
        counts = scene.mosaic_counts(w, h, abi.GRBG, 64.0, 1023, 10, 7)
        data, pitch = scene.pack(counts, abi.RAW10, abi.raw_row_bytes(abi.RAW10, w))
        raw = abi.RawFrame(data, w, h, pitch, abi.RAW10, 10, abi.GRBG)
        stream = torch.cuda.Stream()
        with isp_b200.Pipeline(params) as pipe, isp_b200.Pipeline(params) as other:
            frames = [DeviceFrame(raw, abi.RGB16) for _ in range(2)]
            for f in frames:
                f.run(pipe, stream=stream.cuda_stream)
            torch.cuda.synchronize()
            pipe.process_host(raw, abi.RGB16)
            batch = isp_b200.Batch(4)
            for use_graph in (False, True):
                batch.clear()
                for f, cam in zip(frames, (pipe, other)):
                    r, o = f.views()
                    batch.add(cam, r, o, f.hist.data_ptr(), f.stats.data_ptr())
                batch.launch(stream.cuda_stream, use_graph)
            torch.cuda.synchronize()
            batch.close()
    """, tmp_path)
    trees = ranges_of(lines)
    frame = ("isp.process", [("isp.statistics_pass", []), ("isp.tile_pass", [])])
    host = ("isp.process_host", [("isp.upload", []), frame, ("isp.download", [])])
    direct = ("isp.batch.launch", [("isp.batch.build", []), ("isp.batch.enqueue", [])])
    replay = ("isp.batch.launch", [("isp.batch.build", []), ("isp.batch.replay", [])])
    assert trees == [frame, frame, host, direct, replay], json.dumps(trees)


@pytest.mark.gpu
def test_serving_loop_phases_are_ranges(probe, tmp_path):
    """The server's worker marks each admission, each batch it launches (the
    batch launch nested inside) and each batch it retires."""
    lines = run_traced(probe, """
        import numpy as np
        import isp_b200
        from isp_b200 import abi, scene

        w, h = 256, 128
        params = abi.IspParams(black_level=64.0, white_balance=abi.GRAY_WORLD, demosaic=abi.MALVAR, ccm=scene.CCM)
        server = isp_b200.Server(max_batch=4, max_inflight=2, queue_depth=3, slots_per_stream=2)
        sid = server.add_stream(params, w, h, abi.RAW10, 10, abi.GRBG, abi.RGB8)
        server.start()
        outs = []
        for k in range(3):
            counts = scene.mosaic_counts(w, h, abi.GRBG, 64.0, 1023, 10, 11 + k)
            data, pitch = scene.pack(counts, abi.RAW10)
            img = np.zeros((h, w, 3), np.uint8)
            outs.append(img)
            server.submit(sid, abi.RawFrame(data, w, h, pitch, abi.RAW10, 10, abi.GRBG), img)
        server.drain(60.0)
        assert server.stats()["completed"] == 3
        server.close()
    """, tmp_path)
    trees = ranges_of(lines)
    names = [n for n, _ in trees]
    assert names.count("isp.server.admit") == 3, names
    launches = [c for n, c in trees if n == "isp.server.launch"]
    assert launches and all(c and all(k == "isp.batch.launch" for k, _ in c) for c in launches), json.dumps(trees)
    assert names.count("isp.server.retire") == len(launches), names
