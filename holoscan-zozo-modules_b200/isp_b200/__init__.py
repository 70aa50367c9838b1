"""Python binding of libisp_b200.so, the B200 ISP's C ABI (include/isp_b200.h).

`Pipeline` is holoscan::isp::IspPipeline with the CUDA backend
(modules/isp/include/holoscan/isp/isp_pipeline.hpp:39-74): create from
IspParams, `process` frames held in device memory on a CUDA stream,
`process_host` frames held in host memory (the CPU backend's call shape),
`reset` the white balance estimate. Errors raise as the reference's façade
throws: ValueError for std::invalid_argument, RuntimeError for CUDA failures.

The library is the product's only compute path: if it is missing or fails to
load, every call raises; nothing falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Tuple

import numpy as np

from . import abi
from .abi import IspParams, RawFrame  # noqa: F401  (re-exported)

_HERE = os.path.dirname(os.path.abspath(__file__))
# ISP_B200_LIBRARY=checked selects the bounds-checked build of the ISP
# (libisp_b200_checked.so: every shared- and global-memory access of its
# kernels checked, refused accesses counted per pipeline).
CHECKED = os.environ.get("ISP_B200_LIBRARY", "") == "checked"
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libisp_b200_checked.so" if CHECKED else "libisp_b200.so")
# Pipelines the checked build refused accesses for, as (what, count, first
# address), recorded when they close.
VIOLATIONS = []

_lib = None


class IspError(RuntimeError):
    """A failed call of the C ABI; `status` is its isp_status."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class IspTimeout(IspError, TimeoutError):
    pass


class IspBusy(IspError):
    pass


def lib() -> C.CDLL:
    """The loaded C-ABI library; raises if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built: run holoscan-zozo-modules_b200/build.py")
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        L.isp_b200_abi_version.restype = C.c_int
        L.isp_b200_last_error.restype = C.c_char_p
        L.isp_b200_last_cuda_error.restype = C.c_int
        L.isp_b200_params_default.argtypes = [P(abi.ParamsC)]
        L.isp_b200_validate_params.argtypes = [P(abi.ParamsC)]
        L.isp_b200_validate_raw.argtypes = [P(abi.RawViewC), P(abi.ParamsC)]
        L.isp_b200_raw_row_bytes.restype = C.c_size_t
        L.isp_b200_raw_row_bytes.argtypes = [C.c_int32, C.c_int32]
        L.isp_b200_tone_lut.argtypes = [P(abi.ParamsC), C.c_void_p, C.c_size_t, P(C.c_size_t)]
        L.isp_b200_create.argtypes = [P(abi.ParamsC), P(C.c_void_p)]
        L.isp_b200_destroy.argtypes = [C.c_void_p]
        L.isp_b200_reset.argtypes = [C.c_void_p]
        L.isp_b200_awb_state.argtypes = [C.c_void_p, C.c_void_p, P(C.c_int32)]
        L.isp_b200_process.argtypes = [C.c_void_p, P(abi.RawViewC), P(abi.RgbViewC), P(abi.StatsC),
                                       P(abi.ExposureC), C.c_void_p]
        L.isp_b200_process_noalloc.argtypes = [P(abi.ParamsC), P(abi.RawViewC), P(abi.RgbViewC), P(abi.StatsC),
                                               P(abi.ExposureC), C.c_void_p]
        L.isp_b200_noalloc_status.argtypes = [C.c_void_p, P(C.c_int32)]
        L.isp_b200_device_status.argtypes = [C.c_void_p, P(C.c_int32)]
        L.isp_b200_set_kernel_events.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.isp_b200_check_bounded_wait.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
        L.isp_b200_checked_violations.argtypes = [C.c_void_p, P(C.c_uint32), P(C.c_uint64)]
        L.isp_b200_set_frame_overlap.argtypes = [C.c_void_p, C.c_int32]
        L.isp_b200_process_host.argtypes = [C.c_void_p, P(abi.RawViewC), P(abi.RgbViewC), P(abi.StatsC),
                                            P(abi.ExposureC)]
        L.isp_b200_batch_create.argtypes = [C.c_int32, P(C.c_void_p)]
        L.isp_b200_batch_destroy.argtypes = [C.c_void_p]
        L.isp_b200_batch_clear.argtypes = [C.c_void_p]
        L.isp_b200_batch_size.argtypes = [C.c_void_p]
        L.isp_b200_batch_add.argtypes = [C.c_void_p, C.c_void_p, P(abi.RawViewC), P(abi.RgbViewC), P(abi.StatsC),
                                         P(abi.ExposureC)]
        L.isp_b200_batch_launch.argtypes = [C.c_void_p, C.c_void_p, C.c_int32]
        L.isp_b200_batch_autotune.argtypes = [C.c_void_p, C.c_void_p]
        L.isp_b200_batch_set_tuning.argtypes = [C.c_void_p, C.c_void_p, C.c_int32]
        L.isp_b200_batch_info.argtypes = [C.c_void_p, P(abi.BatchInfoC)]
        L.isp_b200_batch_set_tile_rows.argtypes = [C.c_void_p, C.c_int32]
        L.isp_b200_set_tile_rows.argtypes = [C.c_void_p, C.c_int32]
        L.isp_b200_autotune.argtypes = [C.c_void_p, P(abi.RawViewC), P(abi.RgbViewC), P(abi.StatsC), P(abi.ExposureC),
                                        C.c_void_p, P(C.c_int32)]
        L.isp_b200_server_config_default.argtypes = [P(abi.ServerConfigC)]
        L.isp_b200_server_create.argtypes = [P(abi.ServerConfigC), P(C.c_void_p)]
        L.isp_b200_server_add_stream.argtypes = [C.c_void_p, P(abi.ParamsC), P(abi.ServerStreamC), P(C.c_int32)]
        L.isp_b200_server_start.argtypes = [C.c_void_p]
        L.isp_b200_server_submit.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.c_int64, P(C.c_uint64)]
        L.isp_b200_server_poll.argtypes = [C.c_void_p, P(abi.ServerResultC), C.c_int32, P(C.c_int32)]
        L.isp_b200_server_drain.argtypes = [C.c_void_p, C.c_int64]
        L.isp_b200_server_stats.argtypes = [C.c_void_p, P(abi.ServerStatsC)]
        L.isp_b200_server_reset_stats.argtypes = [C.c_void_p]
        L.isp_b200_server_submit_device.argtypes = L.isp_b200_server_submit.argtypes
        L.isp_b200_server_add_source.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_size_t, C.c_int32]
        L.isp_b200_server_run_poisson.argtypes = [C.c_void_p, P(C.c_double), C.c_double, C.c_uint64]
        L.isp_b200_server_run_closed.argtypes = [C.c_void_p, C.c_double]
        L.isp_b200_synth_default.argtypes = [P(abi.SynthC)]
        L.isp_b200_synth_default.restype = None
        L.isp_b200_synthetic_raw.argtypes = [P(abi.SynthC), C.c_uint64, C.c_void_p, C.c_size_t, C.c_void_p]
        L.isp_b200_server_destroy.argtypes = [C.c_void_p]
        L.isp_b200_view_compose.argtypes = [P(abi.RawViewC), C.c_float, C.c_void_p, C.c_size_t, C.c_void_p,
                                            C.c_size_t, C.c_void_p]
        if L.isp_b200_abi_version() != abi.ABI_VERSION:
            raise RuntimeError("libisp_b200.so ABI version mismatch")
        _lib = L
    return _lib


def check(status: int) -> None:
    if status == abi.OK:
        return
    message = lib().isp_b200_last_error().decode()
    if status == abi.EINVAL:
        raise ValueError(message)
    if status == abi.ETIMEOUT:
        raise IspTimeout(status, message)
    if status == abi.EBUSY:
        raise IspBusy(status, message)
    raise IspError(status, message)


def validate_params(params: IspParams) -> None:
    h = params.to_c()
    check(lib().isp_b200_validate_params(h.ref()))


def validate_raw(raw: abi.RawViewC, params: IspParams) -> None:
    h = params.to_c()
    check(lib().isp_b200_validate_raw(C.byref(raw), h.ref()))


def raw_row_bytes(fmt: int, width: int) -> int:
    return int(lib().isp_b200_raw_row_bytes(fmt, width))


def tone_lut(params: IspParams) -> np.ndarray:
    h = params.to_c()
    n = C.c_size_t()
    check(lib().isp_b200_tone_lut(h.ref(), None, 0, C.byref(n)))
    out = np.zeros(n.value, np.float32)
    check(lib().isp_b200_tone_lut(h.ref(), out.ctypes.data, out.size, C.byref(n)))
    return out


class Result:
    """One frame's outputs in host memory."""

    def __init__(self, image: np.ndarray, histogram: Optional[np.ndarray], stats: Optional[np.ndarray]):
        self.image = image
        self.histogram = histogram
        self.stats = stats


class Pipeline:
    """IspPipeline(Backend::kCuda, params) on the current CUDA device."""

    def __init__(self, params: IspParams):
        self.params = params
        self._holder = params.to_c()
        handle = C.c_void_p()
        check(lib().isp_b200_create(self._holder.ref(), C.byref(handle)))
        self.handle = handle

    def close(self) -> None:
        if getattr(self, "handle", None):
            if CHECKED:
                count, first = self.checked_violations()
                if count:
                    VIOLATIONS.append((repr(self.params)[:200], count, hex(first)))
            lib().isp_b200_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def checked_violations(self) -> Tuple[int, int]:
        """(count, first address) of the accesses the checked build refused on this camera's frames since
        the last call; raises ValueError (ISP_EINVAL) with the regular library, which checks nothing."""
        count = C.c_uint32()
        first = C.c_uint64()
        check(lib().isp_b200_checked_violations(self.handle, C.byref(count), C.byref(first)))
        return int(count.value), int(first.value)

    def reset(self) -> None:
        check(lib().isp_b200_reset(self.handle))

    def awb(self) -> Tuple[np.ndarray, int]:
        gains = (C.c_float * 3)()
        valid = C.c_int32()
        check(lib().isp_b200_awb_state(self.handle, gains, C.byref(valid)))
        return np.array(list(gains), np.float32), int(valid.value)

    def device_status(self) -> int:
        """1 if a kernel gave up a bounded wait on this camera's frames since the last call, else 0."""
        v = C.c_int32()
        check(lib().isp_b200_device_status(self.handle, C.byref(v)))
        return int(v.value)

    def set_tile_rows(self, tile_rows: int) -> None:
        """0 (default): the height autotune picked for the frame's shape, else 64; 64 or 32 force it."""
        check(lib().isp_b200_set_tile_rows(self.handle, tile_rows))

    def autotune(self, raw: abi.RawViewC, out: abi.RgbViewC, histogram_ptr: int = 0, stats_ptr: int = 0,
                 exposure: Tuple[int, float] = (0, 0.0), stream: int = 0) -> int:
        """Times both tile heights on this frame (device buffers), keeps the faster for its raw format and
        size, restores the white balance state; returns the chosen rows."""
        st = abi.StatsC(histogram_ptr or None, stats_ptr or None)
        exp = abi.ExposureC(exposure[0], exposure[1])
        rows = C.c_int32()
        check(lib().isp_b200_autotune(self.handle, C.byref(raw), C.byref(out), C.byref(st), C.byref(exp),
                                      stream or None, C.byref(rows)))
        return int(rows.value)

    def set_frame_overlap(self, enable: bool) -> None:
        """On (default): a frame queued right behind the previous one on the same stream starts its statistics
        pass while that frame's tile pass finishes."""
        check(lib().isp_b200_set_frame_overlap(self.handle, 1 if enable else 0))

    def check_bounded_wait(self, polls: int = 1024, stream: int = 0) -> None:
        """Queues a kernel whose bounded barrier wait runs out after `polls` polls and flags this camera
        as a pass that gave up a wait does (device_status then reads 1 once)."""
        check(lib().isp_b200_check_bounded_wait(self.handle, polls, stream or None))

    def set_kernel_events(self, before: int = 0, after: int = 0) -> None:
        """Events (cudaEvent_t handles) recorded around the fused tile kernel of every later frame."""
        check(lib().isp_b200_set_kernel_events(self.handle, before or None, after or None))

    def process(self, raw: abi.RawViewC, out: abi.RgbViewC, histogram_ptr: int = 0, stats_ptr: int = 0,
                exposure: Tuple[int, float] = (0, 0.0), stream: int = 0) -> None:
        """Queues one frame whose buffers are device pointers, on `stream` (a cudaStream_t)."""
        st = abi.StatsC(histogram_ptr or None, stats_ptr or None)
        exp = abi.ExposureC(exposure[0], exposure[1])
        check(lib().isp_b200_process(self.handle, C.byref(raw), C.byref(out), C.byref(st), C.byref(exp),
                                     stream or None))

    def process_host(self, raw: RawFrame, fmt: int, with_stats: bool = True,
                     exposure: Tuple[int, float] = (0, 0.0), out: Optional[np.ndarray] = None) -> Result:
        """One frame from host memory to host memory; returns when the outputs are there."""
        ch = abi.output_channels(fmt)
        image = out if out is not None else np.empty((raw.height, raw.width, ch), abi.output_dtype(fmt))
        hist = np.zeros((abi.HISTOGRAM_CHANNELS, abi.HISTOGRAM_BINS), np.uint32) if with_stats else None
        stats = np.zeros(abi.STATS_SIZE, np.float32) if with_stats else None
        view = raw.view()
        rgb = abi.RgbViewC(image.ctypes.data, image.strides[0], fmt)
        st = abi.StatsC(hist.ctypes.data if hist is not None else None,
                        stats.ctypes.data if stats is not None else None)
        exp = abi.ExposureC(exposure[0], exposure[1])
        check(lib().isp_b200_process_host(self.handle, C.byref(view), C.byref(rgb), C.byref(st), C.byref(exp)))
        return Result(image, hist, stats)


class Batch:
    """Frames of many cameras through one launch per pass (isp_b200_batch_*)."""

    def __init__(self, capacity: int):
        handle = C.c_void_p()
        check(lib().isp_b200_batch_create(capacity, C.byref(handle)))
        self.handle = handle
        self._keep = []

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib().isp_b200_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def clear(self) -> None:
        check(lib().isp_b200_batch_clear(self.handle))
        self._keep = []

    def __len__(self) -> int:
        return int(lib().isp_b200_batch_size(self.handle))

    def add(self, camera: "Pipeline", raw: abi.RawViewC, out: abi.RgbViewC, histogram_ptr: int = 0,
            stats_ptr: int = 0, exposure: Tuple[int, float] = (0, 0.0)) -> None:
        st = abi.StatsC(histogram_ptr or None, stats_ptr or None)
        exp = abi.ExposureC(exposure[0], exposure[1])
        check(lib().isp_b200_batch_add(self.handle, camera.handle, C.byref(raw), C.byref(out), C.byref(st),
                                       C.byref(exp)))
        self._keep.append(camera)

    def launch(self, stream: int = 0, use_graph: bool = False) -> None:
        check(lib().isp_b200_batch_launch(self.handle, stream or None, 1 if use_graph else 0))

    def autotune(self, stream: int = 0) -> None:
        check(lib().isp_b200_batch_autotune(self.handle, stream or None))

    def set_tuning(self, weights, ctas_per_sm: int = 0) -> None:
        w = (C.c_float * 4)(*weights)
        check(lib().isp_b200_batch_set_tuning(self.handle, w, ctas_per_sm))

    def set_tile_rows(self, tile_rows: int) -> None:
        """The tile pass's tile height for later launches: 64 or 32 rows."""
        check(lib().isp_b200_batch_set_tile_rows(self.handle, tile_rows))

    def info(self) -> dict:
        i = abi.BatchInfoC()
        check(lib().isp_b200_batch_info(self.handle, C.byref(i)))
        return {"frames": i.frames, "weights": list(i.weights), "ctas_per_sm": i.ctas_per_sm, "tuned": bool(i.tuned),
                "graph_replays": i.graph_replays, "graph_main_ctas": i.graph_main_ctas,
                "graph_awb_ctas": i.graph_awb_ctas, "tile_rows": i.tile_rows, "block_threads": i.block_threads}


class Server:
    """Many camera streams with continuous batching (isp_b200_server_*)."""

    def __init__(self, max_batch: int = 64, max_inflight: int = 2, queue_depth: int = 4, slots_per_stream: int = 2,
                 memory_budget: int = 8 << 30, use_graph: bool = False, per_frame: bool = False):
        cfg = abi.ServerConfigC()
        lib().isp_b200_server_config_default(C.byref(cfg))
        cfg.max_batch, cfg.max_inflight, cfg.queue_depth = max_batch, max_inflight, queue_depth
        cfg.slots_per_stream, cfg.memory_budget, cfg.use_graph = slots_per_stream, memory_budget, int(use_graph)
        cfg.per_frame = int(per_frame)
        handle = C.c_void_p()
        check(lib().isp_b200_server_create(C.byref(cfg), C.byref(handle)))
        self.handle = handle
        self._keep = []

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib().isp_b200_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_stream(self, params: IspParams, width: int, height: int, fmt: int, bit_depth: int, pattern: int,
                   out_format: int, with_histogram: bool = True, with_stats: bool = True,
                   copy_back: bool = False) -> int:
        h = params.to_c()
        shape = abi.ServerStreamC(width, height, fmt, bit_depth, pattern, out_format, int(with_histogram),
                                  int(with_stats), int(copy_back))
        sid = C.c_int32()
        check(lib().isp_b200_server_add_stream(self.handle, h.ref(), C.byref(shape), C.byref(sid)))
        return int(sid.value)

    def start(self) -> None:
        check(lib().isp_b200_server_start(self.handle))

    def submit(self, stream: int, raw: RawFrame, host_out: Optional[np.ndarray] = None,
               host_hist: Optional[np.ndarray] = None, host_stats: Optional[np.ndarray] = None,
               arrival_ns: int = 0) -> int:
        ticket = C.c_uint64()
        ptr = lambda a: a.ctypes.data if a is not None else None  # noqa: E731
        check(lib().isp_b200_server_submit(self.handle, stream, raw.data.ctypes.data, raw.pitch, ptr(host_out),
                                           ptr(host_hist), ptr(host_stats), arrival_ns, C.byref(ticket)))
        return int(ticket.value)

    def poll(self, capacity: int = 256):
        buf = (abi.ServerResultC * capacity)()
        n = C.c_int32()
        check(lib().isp_b200_server_poll(self.handle, buf, capacity, C.byref(n)))
        return [buf[i] for i in range(n.value)]

    def drain(self, timeout_s: float = 60.0) -> None:
        check(lib().isp_b200_server_drain(self.handle, int(timeout_s * 1e9)))

    def stats(self) -> dict:
        st = abi.ServerStatsC()
        check(lib().isp_b200_server_stats(self.handle, C.byref(st)))
        return {name: getattr(st, name) for name, _ in abi.ServerStatsC._fields_}

    def reset_stats(self) -> None:
        check(lib().isp_b200_server_reset_stats(self.handle))

    def submit_device(self, stream: int, device_raw: int, pitch: int, host_out: Optional[np.ndarray] = None,
                      host_hist: Optional[np.ndarray] = None, host_stats: Optional[np.ndarray] = None,
                      arrival_ns: int = 0) -> int:
        """A frame already in device memory (read in place until it completes)."""
        ticket = C.c_uint64()
        ptr = lambda a: a.ctypes.data if a is not None else None  # noqa: E731
        check(lib().isp_b200_server_submit_device(self.handle, stream, device_raw, pitch, ptr(host_out),
                                                  ptr(host_hist), ptr(host_stats), arrival_ns, C.byref(ticket)))
        return int(ticket.value)

    def add_source(self, stream: int, raw: RawFrame, on_device: bool = False) -> None:
        check(lib().isp_b200_server_add_source(self.handle, stream, raw.data.ctypes.data, raw.pitch, int(on_device)))

    def run_poisson(self, fps, seconds: float, seed: int = 1) -> None:
        arr = (C.c_double * len(fps))(*fps)
        check(lib().isp_b200_server_run_poisson(self.handle, arr, seconds, seed))

    def run_closed(self, seconds: float) -> None:
        check(lib().isp_b200_server_run_closed(self.handle, seconds))


def synthetic_raw(width: int, height: int, fmt: int, bit_depth: int, pattern: int, black: float, seed: int,
                  device_raw: int, pitch: int, stream: int = 0, gain: float = 0.5, read_noise: float = 3.0,
                  vignette_edge: float = 0.5) -> None:
    """Renders the seeded synthetic frame into device memory (isp_b200_synthetic_raw)."""
    cfg = abi.SynthC()
    lib().isp_b200_synth_default(C.byref(cfg))
    cfg.width, cfg.height, cfg.format, cfg.bit_depth, cfg.pattern = width, height, fmt, bit_depth, pattern
    cfg.black, cfg.gain, cfg.read_noise, cfg.vignette_edge = black, gain, read_noise, vignette_edge
    check(lib().isp_b200_synthetic_raw(C.byref(cfg), seed & 0xFFFFFFFFFFFFFFFF, device_raw, pitch, stream or None))


def process_noalloc(params: IspParams, raw: abi.RawViewC, out: abi.RgbViewC, histogram_ptr: int = 0,
                    stats_ptr: int = 0, exposure: Tuple[int, float] = (0, 0.0), stream: int = 0) -> None:
    """One frame (device buffers) without allocating memory: isp_b200_process_noalloc."""
    h = params.to_c()
    st = abi.StatsC(histogram_ptr or None, stats_ptr or None)
    exp = abi.ExposureC(exposure[0], exposure[1])
    check(lib().isp_b200_process_noalloc(h.ref(), C.byref(raw), C.byref(out), C.byref(st), C.byref(exp),
                                         stream or None))


def noalloc_status(stream: int = 0) -> int:
    """After `stream`'s work: 1 if a kernel of the last no-alloc frame gave up a bounded wait, else 0
    (isp_b200_noalloc_status; read and cleared, allocating nothing)."""
    v = C.c_int32()
    check(lib().isp_b200_noalloc_status(stream or None, C.byref(v)))
    return int(v.value)


def view_compose(raw: abi.RawViewC, black_level: float, rgb8_ptr: int, rgb8_pitch: int, view_ptr: int,
                 view_pitch: int, stream: int = 0) -> None:
    """The demo's side-by-side view (isp_b200_view_compose): device raw frame
    and RGB8 image in, double-width RGB8 image out, queued on `stream`."""
    check(lib().isp_b200_view_compose(C.byref(raw), black_level, C.c_void_p(rgb8_ptr), rgb8_pitch,
                                      C.c_void_p(view_ptr), view_pitch, C.c_void_p(stream)))


def params_default() -> abi.ParamsC:
    c = abi.ParamsC()
    lib().isp_b200_params_default(C.byref(c))
    return c
