"""TEST INFRASTRUCTURE ONLY: Python bindings of the CPU oracle.

`OraclePipeline` drives libisp_oracle.so, the C restatement of the
holoscan::isp CPU backend (oracle/isp_oracle.c). `ReferencePipeline` drives
oracle/_ref/libisp_ref.so, the reference's own CPU backend compiled unmodified
(oracle/Makefile), present only where the reference tree was available when
it was built. Both mirror IspPipeline(Backend::kCpu): host buffers in, host
buffers out, white balance state carried from frame to frame
(modules/isp/src/isp_pipeline.cpp:65-84).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use
this package, as the checker or the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from dataclasses import dataclass
from typing import Optional, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_PKG = os.path.join(os.path.dirname(_HERE), "holoscan-zozo-modules_b200")
if _PKG not in sys.path:
    sys.path.insert(0, _PKG)

from isp_b200 import abi  # noqa: E402  (types only)

ORACLE_SO = os.path.join(_HERE, "libisp_oracle.so")
REF_SO = os.path.join(_HERE, "_ref", "libisp_ref.so")

_oracle = None
_ref = None


def build_oracle() -> None:
    """Compiles libisp_oracle.so (and _ref where the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", _HERE, "all"], check=True)


def _lib_oracle():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            subprocess.run(["make", "-s", "-C", _HERE, "oracle"], check=True)
        lib = C.CDLL(ORACLE_SO)
        P = C.POINTER
        lib.oracle_raw_row_bytes.restype = C.c_size_t
        lib.oracle_raw_row_bytes.argtypes = [C.c_int32, C.c_int32]
        lib.oracle_validate_params.argtypes = [P(abi.ParamsC), C.c_char_p, C.c_size_t]
        lib.oracle_validate_raw.argtypes = [P(abi.RawViewC), P(abi.ParamsC), C.c_char_p, C.c_size_t]
        lib.oracle_tone_lut.restype = C.c_size_t
        lib.oracle_tone_lut.argtypes = [P(abi.ParamsC), C.c_void_p, C.c_size_t]
        lib.oracle_awb_init.argtypes = [P(abi.ParamsC), C.c_void_p]
        lib.oracle_awb_stats.argtypes = [P(abi.ParamsC), P(abi.RawViewC), C.c_void_p]
        lib.oracle_process.argtypes = [P(abi.ParamsC), P(abi.RawViewC), P(abi.RgbViewC), P(abi.StatsC),
                                       P(abi.ExposureC), C.c_void_p]
        lib.oracle_view_compose.argtypes = [P(abi.RawViewC), C.c_float, C.c_void_p, C.c_size_t, C.c_void_p,
                                            C.c_size_t]
        lib.oracle_view_compose.restype = None
        _oracle = lib
    return _oracle


def view_compose(raw: abi.RawFrame, black: float, rgb: np.ndarray) -> np.ndarray:
    """The demo's side-by-side view from the C oracle: [H, 2W, 3] uint8 from a
    raw frame and an [H, W, 3] RGB8 image."""
    rgb = np.ascontiguousarray(rgb, np.uint8)
    out = np.zeros((raw.height, 2 * raw.width, 3), np.uint8)
    rv = raw.view()
    _lib_oracle().oracle_view_compose(C.byref(rv), black, rgb.ctypes.data, rgb.strides[0], out.ctypes.data,
                                      out.strides[0])
    return out


def reference_available() -> bool:
    return os.path.exists(REF_SO)


REF_VIEW_SO = os.path.join(_HERE, "_ref", "libview_ref_cuda.so")
_ref_view = None


def reference_view_available() -> bool:
    return os.path.exists(REF_VIEW_SO)


def reference_view_compose(raw_ptr: int, raw_pitch: int, width: int, height: int, fmt: int, bit_depth: int,
                           black_level: float, rgb8_ptr: int, view_ptr: int, stream: int = 0) -> None:
    """The reference demo's view kernel (view_op.cu, built for sm_100a into
    oracle/_ref/libview_ref_cuda.so), launched as its operator launches it on
    device buffers: the raw frame at raw_pitch, a packed RGB8 image and a
    packed [H, 2W, 3] view. The checker of isp_b200_view_compose."""
    global _ref_view
    if _ref_view is None:
        lib = C.CDLL(REF_VIEW_SO)
        lib.ref_view_compose.argtypes = [C.c_void_p, C.c_size_t, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                         C.c_void_p, C.c_void_p, C.c_void_p]
        _ref_view = lib
    rc = _ref_view.ref_view_compose(raw_ptr, raw_pitch, width, height, fmt, bit_depth, black_level, rgb8_ptr,
                                    view_ptr, stream or None)
    if rc != 0:
        raise RuntimeError(f"reference view kernel launch failed: cudaError {rc}")


REF_CUDA_SO = os.path.join(_HERE, "_ref", "libisp_ref_cuda.so")
_ref_cuda = None


def reference_cuda_available() -> bool:
    return os.path.exists(REF_CUDA_SO)


class ReferenceCudaPipeline:
    """The reference's own CUDA backend (IspPipeline(Backend::kCuda), built
    for sm_100a into oracle/_ref/libisp_ref_cuda.so): device views, frames
    queued on a stream. The GPU bar of the benchmark, not a checker."""

    def __init__(self, params: abi.IspParams):
        global _ref_cuda
        if _ref_cuda is None:
            lib = C.CDLL(REF_CUDA_SO)
            P = C.POINTER
            lib.ref_cuda_pipeline_create.restype = C.c_void_p
            lib.ref_cuda_pipeline_create.argtypes = [P(abi.ParamsC)]
            lib.ref_cuda_pipeline_destroy.argtypes = [C.c_void_p]
            lib.ref_cuda_pipeline_process.argtypes = [C.c_void_p, P(abi.RawViewC), P(abi.RgbViewC), P(abi.StatsC),
                                                      P(abi.ExposureC), C.c_void_p]
            _ref_cuda = lib
        self.lib = _ref_cuda
        self.holder = params.to_c()
        self.handle = self.lib.ref_cuda_pipeline_create(self.holder.ref())
        if not self.handle:
            raise RuntimeError("the reference CUDA pipeline could not be created")

    def process(self, raw: abi.RawViewC, out: abi.RgbViewC, stats: abi.StatsC, exposure: abi.ExposureC,
                stream: int) -> None:
        if self.lib.ref_cuda_pipeline_process(self.handle, C.byref(raw), C.byref(out), C.byref(stats),
                                              C.byref(exposure), C.c_void_p(stream)) != 0:
            raise RuntimeError("the reference CUDA pipeline failed")

    def close(self) -> None:
        if self.handle:
            self.lib.ref_cuda_pipeline_destroy(self.handle)
            self.handle = None


def _lib_ref():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise RuntimeError(f"{REF_SO} is not built: the reference sources were not available")
        lib = C.CDLL(REF_SO)
        P = C.POINTER
        lib.ref_last_error.restype = C.c_char_p
        lib.ref_raw_row_bytes.restype = C.c_size_t
        lib.ref_raw_row_bytes.argtypes = [C.c_int32, C.c_int32]
        lib.ref_validate_params.argtypes = [P(abi.ParamsC)]
        lib.ref_validate_raw.argtypes = [P(abi.RawViewC), P(abi.ParamsC)]
        lib.ref_tone_lut.restype = C.c_size_t
        lib.ref_tone_lut.argtypes = [P(abi.ParamsC), C.c_void_p, C.c_size_t]
        lib.ref_pipeline_create.restype = C.c_void_p
        lib.ref_pipeline_create.argtypes = [P(abi.ParamsC)]
        lib.ref_pipeline_destroy.argtypes = [C.c_void_p]
        lib.ref_pipeline_reset.argtypes = [C.c_void_p]
        lib.ref_pipeline_awb.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        lib.ref_pipeline_process.argtypes = [C.c_void_p, P(abi.RawViewC), P(abi.RgbViewC), P(abi.StatsC),
                                             P(abi.ExposureC)]
        lib.ref_awb_stats.argtypes = [P(abi.ParamsC), P(abi.RawViewC), C.c_void_p, C.c_void_p, C.c_void_p]
        lib.ref_render_synthetic.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
        lib.ref_synthetic_params.argtypes = [C.c_void_p, C.c_int, P(abi.ParamsC), C.c_void_p, C.c_size_t]
        _ref = lib
    return _ref


class OracleAwb(C.Structure):
    _fields_ = [("gains", C.c_float * 3), ("valid", C.c_int32)]


class OracleAwbAccum(C.Structure):
    _fields_ = [("sum", C.c_uint64 * 3), ("quads", C.c_uint64), ("hist", (C.c_uint32 * 1024) * 3)]


@dataclass
class Result:
    """What a pipeline produced for one frame, in host memory."""

    image: np.ndarray       # [H, W, channels] of the output dtype
    histogram: Optional[np.ndarray]  # [4, 256] uint32
    stats: Optional[np.ndarray]      # [12] float32


def _out_buffers(raw: abi.RawFrame, fmt: int, with_stats: bool):
    ch = abi.output_channels(fmt)
    image = np.zeros((raw.height, raw.width, ch), dtype=abi.output_dtype(fmt))
    hist = np.zeros((abi.HISTOGRAM_CHANNELS, abi.HISTOGRAM_BINS), np.uint32) if with_stats else None
    stats = np.zeros(abi.STATS_SIZE, np.float32) if with_stats else None
    return image, hist, stats


def _views(image, hist, stats, fmt):
    rgb = abi.RgbViewC(image.ctypes.data, image.strides[0], fmt)
    st = abi.StatsC(hist.ctypes.data if hist is not None else None,
                    stats.ctypes.data if stats is not None else None)
    return rgb, st


class OraclePipeline:
    """The C oracle with IspPipeline(kCpu)'s state and call shape."""

    def __init__(self, params: abi.IspParams):
        self.lib = _lib_oracle()
        self.params = params
        self.holder = params.to_c()
        msg = C.create_string_buffer(256)
        if self.lib.oracle_validate_params(self.holder.ref(), msg, 256) != abi.OK:
            raise ValueError(msg.value.decode())
        self.state = OracleAwb()
        self.lib.oracle_awb_init(self.holder.ref(), C.byref(self.state))

    def reset(self) -> None:
        self.lib.oracle_awb_init(self.holder.ref(), C.byref(self.state))

    def awb(self) -> Tuple[np.ndarray, int]:
        return np.array(list(self.state.gains), np.float32), int(self.state.valid)

    def process(self, raw: abi.RawFrame, fmt: int, with_stats: bool = True,
                exposure: Tuple[int, float] = (0, 0.0)) -> Result:
        image, hist, stats = _out_buffers(raw, fmt, with_stats)
        rgb, st = _views(image, hist, stats, fmt)
        view = raw.view()
        exp = abi.ExposureC(exposure[0], exposure[1])
        status = self.lib.oracle_process(self.holder.ref(), C.byref(view), C.byref(rgb), C.byref(st),
                                         C.byref(exp), C.byref(self.state))
        if status != abi.OK:
            raise ValueError("oracle rejected the frame")
        return Result(image, hist, stats)


class ReferencePipeline:
    """The reference's own CPU backend (oracle/_ref) with the same interface."""

    def __init__(self, params: abi.IspParams):
        self.lib = _lib_ref()
        self.params = params
        self.holder = params.to_c()
        self.handle = self.lib.ref_pipeline_create(self.holder.ref())
        if not self.handle:
            raise ValueError(self.lib.ref_last_error().decode())

    def __del__(self):
        if getattr(self, "handle", None):
            self.lib.ref_pipeline_destroy(self.handle)
            self.handle = None

    def reset(self) -> None:
        self.lib.ref_pipeline_reset(self.handle)

    def awb(self) -> Tuple[np.ndarray, int]:
        gains = (C.c_float * 3)()
        valid = C.c_int32()
        self.lib.ref_pipeline_awb(self.handle, gains, C.byref(valid))
        return np.array(list(gains), np.float32), int(valid.value)

    def process(self, raw: abi.RawFrame, fmt: int, with_stats: bool = True,
                exposure: Tuple[int, float] = (0, 0.0)) -> Result:
        image, hist, stats = _out_buffers(raw, fmt, with_stats)
        rgb, st = _views(image, hist, stats, fmt)
        view = raw.view()
        exp = abi.ExposureC(exposure[0], exposure[1])
        status = self.lib.ref_pipeline_process(self.handle, C.byref(view), C.byref(rgb), C.byref(st),
                                               C.byref(exp))
        if status != abi.OK:
            raise ValueError(self.lib.ref_last_error().decode())
        return Result(image, hist, stats)


def oracle_tone_lut(params: abi.IspParams) -> np.ndarray:
    lib = _lib_oracle()
    h = params.to_c()
    n = lib.oracle_tone_lut(h.ref(), None, 0)
    out = np.zeros(n, np.float32)
    lib.oracle_tone_lut(h.ref(), out.ctypes.data, n)
    return out


def oracle_validate_params(params: abi.IspParams) -> Optional[str]:
    msg = C.create_string_buffer(256)
    h = params.to_c()
    return None if _lib_oracle().oracle_validate_params(h.ref(), msg, 256) == abi.OK else msg.value.decode()


def oracle_validate_raw(raw: abi.RawViewC, params: abi.IspParams) -> Optional[str]:
    msg = C.create_string_buffer(256)
    h = params.to_c()
    status = _lib_oracle().oracle_validate_raw(C.byref(raw), h.ref(), msg, 256)
    return None if status == abi.OK else msg.value.decode()


def oracle_awb_stats(params: abi.IspParams, raw: abi.RawFrame):
    acc = OracleAwbAccum()
    h = params.to_c()
    view = raw.view()
    _lib_oracle().oracle_awb_stats(h.ref(), C.byref(view), C.byref(acc))
    return (np.array(list(acc.sum), np.uint64), int(acc.quads),
            np.ctypeslib.as_array(acc.hist).reshape(3, 1024).copy())


# ---- The reference's synthetic camera (for golden fixtures) ----------------

class RefSyntheticConfig(C.Structure):
    """SyntheticRawConfig (modules/isp/include/holoscan/isp/synthetic_raw.hpp:40-59)."""

    _fields_ = [
        ("width", C.c_int32), ("height", C.c_int32), ("pattern", C.c_int32), ("format", C.c_int32),
        ("bit_depth", C.c_int32), ("black_levels", C.c_float * 4), ("wb_gains", C.c_float * 3),
        ("ccm", C.c_float * 9), ("vignetting", C.c_float), ("kind", C.c_int32), ("exposure", C.c_float),
        ("frame", C.c_uint32),
    ]


def ref_synthetic_config(width=640, height=480, pattern=abi.RGGB, fmt=abi.U16, bit_depth=12,
                         black_levels=(256.0,) * 4, wb_gains=(1.9, 1.0, 1.6),
                         ccm=(1.6, -0.4, -0.2, -0.3, 1.5, -0.2, -0.1, -0.5, 1.6), vignetting=0.0,
                         kind=0, exposure=1.0, frame=0) -> RefSyntheticConfig:
    c = RefSyntheticConfig()
    c.width, c.height, c.pattern, c.format, c.bit_depth = width, height, pattern, fmt, bit_depth
    for k in range(4):
        c.black_levels[k] = black_levels[k]
    for k in range(3):
        c.wb_gains[k] = wb_gains[k]
    for k in range(9):
        c.ccm[k] = ccm[k]
    c.vignetting, c.kind, c.exposure, c.frame = vignetting, kind, exposure, frame
    return c


def ref_render(config: RefSyntheticConfig) -> abi.RawFrame:
    """The reference's synthetic sensor, rows padded to 2 bytes (scene_support.hpp:38-45)."""
    lib = _lib_ref()
    pitch = abi.raw_row_bytes(config.format, config.width)
    pitch = (pitch + 1) & ~1
    data = np.zeros(pitch * config.height, np.uint8)
    if lib.ref_render_synthetic(C.byref(config), data.ctypes.data, pitch) != abi.OK:
        raise ValueError(lib.ref_last_error().decode())
    return abi.RawFrame(data, config.width, config.height, pitch, config.format, config.bit_depth,
                        config.pattern)


def ref_synthetic_params(config: RefSyntheticConfig, grid: int = 17) -> abi.IspParams:
    """synthetic_isp_params (modules/isp/src/synthetic_raw.cpp:102-133)."""
    lib = _lib_ref()
    c = abi.ParamsC()
    lsc = np.zeros(256 * 256 * 4, np.float32)
    if lib.ref_synthetic_params(C.byref(config), grid, C.byref(c), lsc.ctypes.data, lsc.size) != abi.OK:
        raise ValueError(lib.ref_last_error().decode())
    p = abi.IspParams()
    p.black_level = c.black_level
    p.channel_black_levels = list(c.channel_black_levels) if c.has_channel_black_levels else None
    p.white_level = c.white_level
    if c.has_lens_shading:
        p.lens_shading = abi.LensShading(c.lsc_width, c.lsc_height, c.lsc_channels,
                                         lsc[: c.lsc_gains_count].copy())
    p.white_balance = c.white_balance
    p.wb_gains = tuple(c.wb_gains)
    p.awb_smoothing = c.awb_smoothing
    p.white_patch_percentile = c.white_patch_percentile
    p.demosaic = c.demosaic
    p.ccm = tuple(c.ccm)
    p.tone_curve = c.tone_curve
    p.gamma = c.gamma
    p.sharpen = c.sharpen
    ae = c.auto_exposure
    p.auto_exposure = abi.AutoExposure(ae.target, ae.damping, ae.min_exposure_ns, ae.max_exposure_ns,
                                       ae.min_gain, ae.max_gain)
    return p


def ref_tone_lut(params: abi.IspParams) -> np.ndarray:
    lib = _lib_ref()
    h = params.to_c()
    n = lib.ref_tone_lut(h.ref(), None, 0)
    out = np.zeros(n, np.float32)
    lib.ref_tone_lut(h.ref(), out.ctypes.data, n)
    return out


def ref_awb_stats(params: abi.IspParams, raw: abi.RawFrame):
    lib = _lib_ref()
    h = params.to_c()
    view = raw.view()
    s = (C.c_uint64 * 3)()
    q = C.c_uint64()
    hist = np.zeros((3, 1024), np.uint32)
    if lib.ref_awb_stats(h.ref(), C.byref(view), s, C.byref(q), hist.ctypes.data) != abi.OK:
        raise ValueError(lib.ref_last_error().decode())
    return np.array(list(s), np.uint64), int(q.value), hist


def ref_validate_params(params: abi.IspParams) -> Optional[str]:
    lib = _lib_ref()
    h = params.to_c()
    return None if lib.ref_validate_params(h.ref()) == abi.OK else lib.ref_last_error().decode()


def ref_validate_raw(raw: abi.RawViewC, params: abi.IspParams) -> Optional[str]:
    lib = _lib_ref()
    h = params.to_c()
    return None if lib.ref_validate_raw(C.byref(raw), h.ref()) == abi.OK else lib.ref_last_error().decode()
