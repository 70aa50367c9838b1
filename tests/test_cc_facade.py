"""holoscan::color_convert's C++ interface of the B200 build (header-only over
the C ABI, holoscan-zozo-modules_b200/cpp/include/holoscan/color_convert/):
compiled with g++ and run. Names, sizes and letterbox geometry are the
reference's; unusable images and the VIC backend throw the reference's
exception types with its messages; and on a GPU, Converter's outputs equal
the C oracle's."""
import json
import os
import subprocess

import numpy as np
import pytest

from isp_b200 import cc
from oracle import cc as occ

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "holoscan-zozo-modules_b200")
CUDA = "/usr/local/cuda"


@pytest.fixture(scope="module")
def facade(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("ccfacade") / "cc_facade_check")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(PKG, "cpp", "include"),
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "cpp", "cc_facade_check.cpp"), "-L", PKG, "-lisp_b200",
           "-L", os.path.join(CUDA, "lib64"), "-lcudart", f"-Wl,-rpath,{PKG}", f"-Wl,-rpath,{CUDA}/lib64", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_host_checks(facade):
    out = subprocess.run([facade, "host"], check=True, capture_output=True, text=True, timeout=60).stdout
    c = {d["check"]: d for d in (json.loads(line) for line in out.splitlines() if line.startswith("{"))}
    assert c["names"] == {"check": "names", "nv12": "nv12", "rgb16": "rgb16", "parsed_uyvy": cc.UYVY,
                          "bt2020": "bt2020", "full": "full", "area": "area", "bad": 0, "auto": "auto"}
    assert (c["sizes"]["nv12_5x3"], c["sizes"]["i420_5x3"], c["sizes"]["nv16_5x3"]) == (27, 27, 33)
    assert c["sizes"]["yuyv_even"] == 1 and c["sizes"]["alpha"] == 1 and c["sizes"]["planar"] == 1
    assert c["letterbox"]["content"] == [0, 140, 640, 360] and c["letterbox"]["source"] == [0, 0, 1920, 1080]
    assert c["bad_crop"] == {"check": "bad_crop", "throws": "invalid_argument",
                             "what": "crop 20x10+90+0 is not inside the 100x100 source"}
    assert c["odd_yuyv"]["throws"] == "invalid_argument"
    assert c["odd_yuyv"]["what"] == "source image: yuyv needs an even width, not 3"
    assert c["host_images"]["what"] == "source image must be in CUDA device memory"
    assert c["vic_backend"]["throws"] == "invalid_argument" and "VPI" in c["vic_backend"]["what"]
    assert c["auto"]["chosen"] == "cuda"


@pytest.mark.gpu
def test_converter_on_gpu_matches_oracle(facade, tmp_path):
    path = str(tmp_path / "out.bin")
    subprocess.run([facade, "gpu", path], check=True, timeout=120)
    got = np.fromfile(path, np.uint8)
    rgb = occ.test_pattern(1920, 1080, 3)
    nv12 = occ.convert(rgb, cc.RGB8, 1920, 1080, cc.NV12, 1920, 1080, cc.params(cc.BT709, mode=cc.NEAREST), threads=8)
    box = occ.convert(nv12, cc.NV12, 1920, 1080, cc.RGB8, 640, 640,
                      cc.params(cc.BT709, letterbox=True, fill_rgb=(200, 30, 90)), threads=8)
    assert np.array_equal(got, np.concatenate([nv12, box]))
