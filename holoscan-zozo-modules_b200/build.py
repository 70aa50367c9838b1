"""Builds libisp_b200.so in-tree: the sm_100a kernels and the C ABI.

    python holoscan-zozo-modules_b200/build.py [--verbose] [--checked]

--checked builds libisp_b200_checked.so instead: the ISP sources compiled with
ISP_CHECKED, every shared- and global-memory access of the ISP kernels checked
against the extent of the array it indexes (isp_checked.cuh), for the tests.

Every translation unit is compiled for sm_100a only, without fused
multiply-add contraction (--fmad=false, -ffp-contract=off): the kernels must
round every product and sum separately, as the holoscan::isp CPU backend does.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libisp_b200.so")
OBJ_CHECKED = os.path.join(HERE, "_build_checked")
LIB_CHECKED = os.path.join(HERE, "libisp_b200_checked.so")

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
          "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-DISP_B200_BUILD"]

SOURCES = ["isp_batch.cu", "isp_batch_global_lut.cu", "isp_batch_short.cu", "isp_batch_short_global_lut.cu",
           "isp_main_bilinear.cu", "isp_main_bilinear_sharpen.cu", "isp_main_malvar.cu", "isp_main_malvar_sharpen.cu",
           "isp_main_bilinear_short.cu", "isp_main_bilinear_sharpen_short.cu", "isp_main_malvar_short.cu",
           "isp_main_malvar_sharpen_short.cu",
           "isp_awb.cu", "isp_kernels.cu", "isp_capi.cu", "isp_batch_host.cu", "isp_noalloc.cu", "isp_server.cu", "isp_synth.cu", "isp_view.cu", "isp_params.cpp",
           # the colour converter (the step after the ISP)
           "cc/cc_direct_yuv.cu", "cc/cc_direct_rgb.cu", "cc/cc_direct_gray.cu", "cc/cc_resample.cu", "cc/cc_capi.cu",
           "cc/cc_plan.cpp"]


def _headers(folder: str) -> list:
    return [os.path.join(folder, f) for f in os.listdir(folder) if f.endswith((".cuh", ".hpp"))]


def _compile(src: str, verbose: bool, checked: bool = False) -> str:
    out = os.path.join(OBJ_CHECKED if checked else OBJ, os.path.splitext(src)[0].replace("/", "_") + ".o")
    path = os.path.join(CSRC, src)
    # A source depends on the headers of its own folder and of csrc/ (the
    # converter's folder includes the ISP's host helpers, not the reverse).
    folder = os.path.dirname(path)
    deps = [path] + _headers(CSRC) + (_headers(folder) if folder != CSRC else [])
    deps.append(os.path.join(ROOT, "include", "isp_b200.h"))
    if folder != CSRC:
        deps.append(os.path.join(ROOT, "include", "cc_b200.h"))
    if os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(d) for d in deps):
        return out
    # The checked build is for tests: its kernels are compiled with less
    # scheduling effort in ptxas (the checks make them large), not other
    # arithmetic (no contraction either way, --fmad=false).
    checked_flags = ["-DISP_CHECKED", "-Xptxas", "-O1"]
    cmd = [NVCC, *ARCH, *COMMON, *(checked_flags if checked else []), "-c", path, "-o", out]
    if src.endswith(".cpp"):
        cmd[1:1] = ["-x", "cu"]
    if verbose and src.endswith(".cu"):
        cmd += ["-Xptxas", "-v"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{res.stdout}\n{res.stderr}")
    if verbose:
        sys.stderr.write(res.stderr)
    return out


# The checked library holds the ISP alone (not the colour converter).
CHECKED_SOURCES = [s for s in SOURCES if not s.startswith("cc/")]


def _link(lib: str, objs: list) -> None:
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(lib) or os.path.getmtime(lib) < newest:
        cmd = [NVCC, *ARCH, "-shared", "-o", lib, *objs, "-Xcompiler", "-fPIC"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")


def build(verbose: bool = False, checked: bool = False) -> str:
    """Builds libisp_b200.so (or, with checked, libisp_b200_checked.so)."""
    os.makedirs(OBJ_CHECKED if checked else OBJ, exist_ok=True)
    sources = CHECKED_SOURCES if checked else SOURCES
    with cf.ThreadPoolExecutor(max_workers=len(sources)) as pool:
        objs = list(pool.map(lambda s: _compile(s, verbose, checked), sources))
    lib = LIB_CHECKED if checked else LIB
    _link(lib, objs)
    return lib


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--checked", action="store_true")
    args = ap.parse_args()
    print(build(args.verbose, args.checked))
