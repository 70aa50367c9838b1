"""holoscan::isp's C++ interface of the B200 build (header-only over the C
ABI, holoscan-zozo-modules_b200/cpp/include/holoscan/isp/): compiled with
g++ and run. The settings checks throw the reference's exception types with
the reference's messages (checked against the reference's own validation,
built in oracle/_ref, where present); the CPU backend is refused; and on a
GPU, frames through IspPipeline equal the C oracle's on the same bytes."""
import json
import os
import subprocess

import numpy as np
import pytest

import oracle
from isp_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "holoscan-zozo-modules_b200")
CUDA = "/usr/local/cuda"


@pytest.fixture(scope="module")
def facade(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("facade") / "facade_check")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(PKG, "cpp", "include"),
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "cpp", "facade_check.cpp"), "-L", PKG, "-lisp_b200",
           "-L", os.path.join(CUDA, "lib64"), "-lcudart", f"-Wl,-rpath,{PKG}", f"-Wl,-rpath,{CUDA}/lib64", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def _checks(exe, *args):
    out = subprocess.run([exe, *args], check=True, capture_output=True, text=True, timeout=120).stdout
    return {d["check"]: d for d in (json.loads(line) for line in out.splitlines() if line.startswith("{"))}


def test_host_checks_throw_the_reference_exceptions(facade):
    c = _checks(facade, "host")
    assert c["valid_params"]["throws"] == "none"
    bad = {
        "bad_sharpen": abi.IspParams(sharpen=5.0),
        "bad_wb_gain": abi.IspParams(wb_gains=(0.0, 1.0, 1.0)),
        "bad_lut": abi.IspParams(tone_curve=abi.LUT, lut=np.array([0.5], np.float32)),
    }
    for name, params in bad.items():
        assert c[name]["throws"] == "invalid_argument", name
        if oracle.reference_available():
            assert c[name]["what"] == oracle.ref_validate_params(params), name
    for name in ("bad_grid", "bad_raw_width", "bad_bit_depth", "bad_params_before_cuda"):
        assert c[name]["throws"] == "invalid_argument", name
    assert c["bad_params_before_cuda"]["what"] == c["bad_sharpen"]["what"]
    assert c["cpu_backend"]["throws"] == "invalid_argument"


def test_host_tables_and_names(facade):
    c = _checks(facade, "host")
    lut = oracle.oracle_tone_lut(abi.IspParams(tone_curve=abi.GAMMA, gamma=2.4))
    t = c["tone_gamma"]
    assert t["size"] == lut.size == 4097
    assert np.float32(t["mid"]) == lut[lut.size // 2] and t["last"] == float(lut[-1]) and t["first"] == float(lut[0])
    assert t["sum"] == pytest.approx(float(lut.astype(np.float64).sum()), rel=0, abs=1e-9)
    assert c["row_bytes"] == {"check": "row_bytes", "u8": 3839, "u16": 7678,
                              "raw10": abi.raw_row_bytes(abi.RAW10, 3839), "raw12": abi.raw_row_bytes(abi.RAW12, 3839)}
    assert c["names"]["pattern"] == "GBRG" and c["names"]["parsed"] == abi.GRBG and c["names"]["wb"] == "white-patch"
    assert c["names"]["backend"] == 0 and c["names"]["unknown"] == 0
    assert c["channels"]["rgba8"] == 4 and c["channels"]["rgb16_bytes"] == 2 and c["channels"]["resolve_no_gpu"] == 1


def _raw10_frame(width, height, seed):
    """facade_check.cpp's frame: xorshift32 counts below 2^10."""
    s = seed
    counts = np.empty(width * height, np.uint16)
    for i in range(width * height):
        s ^= (s << 13) & 0xFFFFFFFF
        s ^= s >> 17
        s ^= (s << 5) & 0xFFFFFFFF
        counts[i] = s & 1023
    from isp_b200 import scene
    data, pitch = scene.pack(counts.reshape(height, width), abi.RAW10)
    return abi.RawFrame(data, width, height, pitch, abi.RAW10, 10, abi.GRBG)


@pytest.mark.gpu
def test_pipeline_frames_match_oracle(facade, tmp_path):
    out = tmp_path / "frames.bin"
    c = _checks(facade, "gpu", str(out))
    assert c["gpu"]["error"] == "no error"
    width, height = 200, 120
    grid = np.array([1.0 + (i % 7) * 0.125 for i in range(5 * 4 * 4)], np.float32)
    params = abi.IspParams(black_level=64.0, white_balance=abi.GRAY_WORLD, demosaic=abi.MALVAR, sharpen=0.5,
                           ccm=(1.6, -0.3, -0.3, -0.3, 1.6, -0.3, -0.3, -0.3, 1.6),
                           lens_shading=abi.LensShading(5, 4, 4, grid))
    ref = oracle.OraclePipeline(params)
    blob = out.read_bytes()
    image_bytes = width * height * 6
    frame_bytes = image_bytes + 4096 + 48
    assert len(blob) == 2 * frame_bytes
    for f in range(2):
        exp = ref.process(_raw10_frame(width, height, 12345 + f), abi.RGB16, True, (8_000_000, 1.5))
        part = blob[f * frame_bytes:(f + 1) * frame_bytes]
        assert part[:image_bytes] == exp.image.tobytes(), f"frame {f}: image"
        assert part[image_bytes:image_bytes + 4096] == exp.histogram.astype(np.uint32).tobytes(), f"frame {f}: histogram"
        assert part[image_bytes + 4096:] == exp.stats.astype(np.float32).tobytes(), f"frame {f}: statistics"


# ---- The operator's work without the SDK (holoscan/isp/isp_op_core.hpp) -------

@pytest.fixture(scope="module")
def op_core(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("opcore") / "op_core_check")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(PKG, "cpp", "include"),
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "cpp", "op_core_check.cpp"), "-L", PKG, "-lisp_b200",
           "-L", os.path.join(CUDA, "lib64"), "-lcudart", f"-Wl,-rpath,{PKG}", f"-Wl,-rpath,{CUDA}/lib64", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_operator_configuration_checks(op_core):
    c = _checks(op_core, "host")
    assert c["config_ok"]["error"] == ""
    assert c["config_max_size"]["error"] == "max_width and max_height must be 2..16384"
    assert c["config_bit_depth"]["error"] == "bit_depth must be 0 (from the image) or 1..16"
    assert c["config_packed_bits"]["error"] == "packed RAW10 and RAW12 samples have 10 and 12 bits"
    assert c["config_params"]["error"] == "sharpen must be 0..4"


def test_operator_describes_inputs_as_the_reference_does(op_core):
    c = _checks(op_core, "host")
    pad = c["u16_padded"]
    assert (pad["error"], pad["width"], pad["height"], pad["pitch"], pad["format"], pad["bits"], pad["pattern"],
            pad["span"], pad["contiguous"]) == ("", 64, 32, 160, abi.U16, 12, abi.GRBG, 160 * 31 + 128, 0)
    assert c["u16_contiguous"]["contiguous"] == 1 and c["u16_contiguous"]["span"] == 64 * 32 * 2
    assert c["mono_with_pattern"]["error"] == "" and c["mono_with_pattern"]["pattern"] == abi.BGGR
    assert c["unknown_bits"]["bits"] == 16  # the container's bits when the image does not say
    raw10 = c["raw10"]
    assert (raw10["error"], raw10["width"], raw10["format"], raw10["bits"], raw10["span"]) == (
        "", 80, abi.RAW10, 10, 112 * 31 + abi.raw_row_bytes(abi.RAW10, 80))
    errors = {
        "bad_encoding": "IspOp: unsupported raw encoding RGB8; use BAYER_RGGB, BAYER_BGGR, BAYER_GRBG, BAYER_GBRG, "
                        "MONO8 or MONO16",
        "mono_without_pattern": "IspOp: a MONO8 or MONO16 raw image needs the Bayer pattern in the configuration",
        "pattern_disagrees": "IspOp: the image's pattern GRBG disagrees with the configured BGGR",
        "element_vs_encoding": "IspOp: raw element type disagrees with its encoding",
        "strided_row": "IspOp: raw samples within a row must be packed",
        "overlap": "IspOp: raw rows overlap",
        "too_large": "IspOp: raw image 4000x32 is outside 2x2 to the configured 3840x2160",
        "misaligned": "IspOp: uint16 raw data must be aligned to 2 bytes",
        "raw10_short_rows": "IspOp: packed rows of 100 bytes cannot hold 81 samples",
        "elsewhere": "IspOp: raw images must be in host or CUDA memory",
    }
    for name, message in errors.items():
        assert c[name]["error"] == message, name


@pytest.mark.gpu
def test_operator_stages_host_frames_and_counts_waits_and_copies(op_core):
    g = _checks(op_core, "gpu")["gpu"]
    assert g["error"] == "no error" and g["same"] == 1
    # As the reference's operator test counts them (isp_op_test.cpp:220-232,
    # README's table): a pageable host frame waits for its producer and for
    # the staged copy, one copy; a pinned frame whose tensor cannot hold its
    # memory waits once for the copy; a device frame costs nothing.
    assert (g["pageable_waits"], g["pageable_copies"]) == (2, 1)
    assert (g["pinned_waits"], g["pinned_copies"]) == (1, 1)
    # A pinned frame whose tensor holds its memory until the stream passes
    # the copy (set_deallocation_stream): the hold on the operator's stream, no wait.
    assert (g["held_waits"], g["held_copies"], g["holds"], g["held_on_stream"]) == (0, 1, 1, 1)
    assert (g["device_waits"], g["device_copies"]) == (0, 0)
