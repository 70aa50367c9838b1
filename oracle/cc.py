"""TEST INFRASTRUCTURE ONLY: Python bindings of the colour converter's CPU
checkers.

`convert` drives libcc_oracle.so, the C restatement of the
holoscan::color_convert conversion (oracle/cc_oracle.c); `ref_convert`
drives oracle/_ref/libcc_ref.so, the reference's own reference_convert
compiled unmodified (oracle/Makefile), present only where the reference tree
was available when it was built. Both take and return packed host images
(numpy uint8 arrays, planes one after the other). `ref_cuda_convert` runs the
reference's own CUDA kernel (oracle/_ref/libcc_ref_cuda.so) on device
buffers, for the benchmark's GPU bar.

Only tests/ and bench.py's baseline legs may use this module.
"""
from __future__ import annotations

import concurrent.futures as cf
import ctypes as C
import os
import subprocess
import sys
from typing import Optional, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_PKG = os.path.join(os.path.dirname(_HERE), "holoscan-zozo-modules_b200")
if _PKG not in sys.path:
    sys.path.insert(0, _PKG)

from isp_b200.cc import CcImageC, CcMappingC, CcParamsC, HOST, DEVICE  # noqa: E402  (types only)

ORACLE_SO = os.path.join(_HERE, "libcc_oracle.so")
REF_SO = os.path.join(_HERE, "_ref", "libcc_ref.so")
REF_CUDA_SO = os.path.join(_HERE, "_ref", "libcc_ref_cuda.so")

_libs = {}


def _load(path: str, cuda: bool = False):
    if path in _libs:
        return _libs[path]
    if path == ORACLE_SO and not os.path.exists(path):
        subprocess.run(["make", "-s", "-C", _HERE, "oracle"], check=True)
    L = C.CDLL(path)
    P = C.POINTER
    prefix = "cc_oracle" if path == ORACLE_SO else "cc_ref"
    getattr(L, f"{prefix}_convert").argtypes = [P(CcImageC), P(CcImageC), P(CcParamsC), C.c_char_p, C.c_size_t]
    getattr(L, f"{prefix}_mapping").argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, P(CcParamsC),
                                                P(CcMappingC), C.c_char_p, C.c_size_t]
    if prefix == "cc_oracle":
        L.cc_oracle_convert_rows.argtypes = [P(CcImageC), P(CcImageC), P(CcParamsC), C.c_int, C.c_int, C.c_char_p,
                                             C.c_size_t]
        L.cc_oracle_packed_size.argtypes = [C.c_int, C.c_int, C.c_int]
        L.cc_oracle_packed_size.restype = C.c_size_t
        L.cc_oracle_test_pattern.argtypes = [C.c_void_p, C.c_size_t, C.c_int, C.c_int, C.c_uint32]
        L.cc_oracle_test_pattern.restype = None
    else:
        L.cc_ref_validate.argtypes = [P(CcImageC), P(CcImageC), P(CcParamsC), C.c_char_p, C.c_size_t]
        L.cc_ref_test_pattern.argtypes = [P(CcImageC), C.c_uint32, C.c_char_p, C.c_size_t]
        if cuda:
            L.cc_ref_cuda_convert.argtypes = [P(CcImageC), P(CcImageC), P(CcParamsC), C.c_void_p, C.c_char_p,
                                              C.c_size_t]
    _libs[path] = L
    return L


def have_ref() -> bool:
    return os.path.exists(REF_SO)


def have_ref_cuda() -> bool:
    return os.path.exists(REF_CUDA_SO)


# Plane layout of a packed image, restated here (pixel_format.hpp:58-138) so
# that the checkers need nothing from the product but its struct types.
_INFO = {0: (2, 1, 1, 1, 1), 1: (2, 1, 0, 1, 1), 2: (3, 1, 1, 1, 1), 3: (1, 1, 0, 1, 2), 4: (1, 1, 0, 1, 2),
         5: (1, 0, 0, 1, 3), 6: (1, 0, 0, 1, 3), 7: (1, 0, 0, 1, 4), 8: (1, 0, 0, 1, 4), 9: (1, 0, 0, 1, 1),
         10: (1, 0, 0, 2, 1), 11: (1, 0, 0, 2, 3)}  # planes, shift x, shift y, bytes per sample, channels


def planes_of(fmt: int, width: int, height: int):
    """[(row bytes, rows)] of each plane of a packed image."""
    planes, sx, sy, nbytes, channels = _INFO[fmt]
    out = [(width * channels * nbytes, height)]
    for _ in range(1, planes):
        cw = (width + (1 << sx) - 1) >> sx
        out.append((cw * (2 if planes == 2 else 1), (height + (1 << sy) - 1) >> sy))
    return out


def packed_size(fmt: int, width: int, height: int) -> int:
    return sum(rb * rows for rb, rows in planes_of(fmt, width, height))


def host_view(buf: np.ndarray, fmt: int, width: int, height: int, pitches=None, offsets=None,
              location: int = HOST) -> CcImageC:
    """A view of `buf` (uint8): packed, or with the given plane pitches and offsets."""
    v = CcImageC()
    v.format, v.width, v.height, v.location = fmt, width, height, location
    base = buf.ctypes.data
    off = 0
    for k, (rb, rows) in enumerate(planes_of(fmt, width, height)):
        pitch = rb if pitches is None else pitches[k]
        start = off if offsets is None else offsets[k]
        v.planes[k].data = base + start
        v.planes[k].pitch = pitch
        off += rb * rows
    return v


class OracleError(ValueError):
    pass


def _call(fn, *args) -> None:
    err = C.create_string_buffer(512)
    status = fn(*args, err, 512)
    if status != 0:
        raise OracleError(err.value.decode())


def convert(src: np.ndarray, src_fmt: int, sw: int, sh: int, dst_fmt: int, dw: int, dh: int, p: CcParamsC,
            threads: int = 1, src_view: Optional[CcImageC] = None) -> np.ndarray:
    """The C oracle's conversion of a packed host image; returns the packed result."""
    L = _load(ORACLE_SO)
    dst = np.zeros(packed_size(dst_fmt, dw, dh), np.uint8)
    sv = src_view if src_view is not None else host_view(src, src_fmt, sw, sh)
    dv = host_view(dst, dst_fmt, dw, dh)
    if threads <= 1:
        _call(L.cc_oracle_convert, C.byref(sv), C.byref(dv), C.byref(p))
        return dst
    # Destination block rows split across threads (ctypes releases the GIL).
    sy = _INFO[dst_fmt][2] if dst_fmt <= 4 else 0
    rows = (dh + (1 << sy) - 1) >> sy
    step = (rows + threads - 1) // threads
    with cf.ThreadPoolExecutor(threads) as pool:
        list(pool.map(lambda r0: _call(L.cc_oracle_convert_rows, C.byref(sv), C.byref(dv), C.byref(p), r0,
                                       min(rows, r0 + step)), range(0, rows, step)))
    return dst


def ref_convert(src: np.ndarray, src_fmt: int, sw: int, sh: int, dst_fmt: int, dw: int, dh: int,
                p: CcParamsC, src_view: Optional[CcImageC] = None) -> np.ndarray:
    """The reference's reference_convert (built from its sources) of a packed host image."""
    L = _load(REF_SO)
    dst = np.zeros(packed_size(dst_fmt, dw, dh), np.uint8)
    sv = src_view if src_view is not None else host_view(src, src_fmt, sw, sh)
    _call(L.cc_ref_convert, C.byref(sv), C.byref(host_view(dst, dst_fmt, dw, dh)), C.byref(p))
    return dst


def mapping(sw: int, sh: int, w: int, h: int, dst_fmt: int, p: CcParamsC, ref: bool = False):
    """((source rect), (content rect)) from the oracle, or from the reference."""
    L = _load(REF_SO if ref else ORACLE_SO)
    m = CcMappingC()
    _call(getattr(L, "cc_ref_mapping" if ref else "cc_oracle_mapping"), sw, sh, w, h, dst_fmt, C.byref(p),
          C.byref(m))
    return m.source.tuple(), m.content.tuple()


def ref_validate(src: CcImageC, dst: CcImageC, p: CcParamsC) -> Optional[str]:
    """The reference's validate_conversion message, or None when usable."""
    L = _load(REF_SO)
    err = C.create_string_buffer(512)
    status = L.cc_ref_validate(C.byref(src), C.byref(dst), C.byref(p), err, 512)
    return None if status == 0 else err.value.decode()


def test_pattern(width: int, height: int, frame: int) -> np.ndarray:
    """The synthetic camera's RGB8 frame from the oracle."""
    L = _load(ORACLE_SO)
    out = np.zeros(width * height * 3, np.uint8)
    L.cc_oracle_test_pattern(out.ctypes.data, width * 3, width, height, frame)
    return out


def ref_test_pattern(width: int, height: int, frame: int) -> np.ndarray:
    L = _load(REF_SO)
    out = np.zeros(width * height * 3, np.uint8)
    _call(L.cc_ref_test_pattern, C.byref(host_view(out, 5, width, height)), frame)
    return out


def ref_cuda_convert(src: CcImageC, dst: CcImageC, p: CcParamsC, stream: int = 0) -> None:
    """The reference's own CUDA kernel (Converter(kCuda)) on device images."""
    L = _load(REF_CUDA_SO, cuda=True)
    _call(L.cc_ref_cuda_convert, C.byref(src), C.byref(dst), C.byref(p), C.c_void_p(stream))


def noise(fmt: int, width: int, height: int, seed: int) -> np.ndarray:
    """Every byte of a packed image pseudo-random: the top byte of each step of
    the 32-bit linear congruential sequence x -> 1664525 x + 1013904223 from
    seed * 2654435761 + 1, so chroma differs inside blocks."""
    n = packed_size(fmt, width, height)
    a, c, mask = 1664525, 1013904223, 0xFFFFFFFF
    k = 4096
    first, x = [], (seed * 2654435761 + 1) & mask
    for _ in range(min(k, n)):
        x = (x * a + c) & mask
        first.append(x)
    out = np.empty(((n + k - 1) // k) * k, np.uint64)
    out[:len(first)] = first
    # k steps at once: x -> ak x + ck.
    ak, ck = 1, 0
    for _ in range(k):
        ak, ck = (ak * a) & mask, (ck * a + c) & mask
    block = np.array(first, np.uint64)
    for j in range(1, len(out) // k):
        block = (block * np.uint64(ak) + np.uint64(ck)) & np.uint64(mask)
        out[j * k:(j + 1) * k] = block
    return (out[:n] >> np.uint64(24)).astype(np.uint8)
