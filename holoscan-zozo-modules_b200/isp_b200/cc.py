"""Python face of the B200 colour converter (include/cc_b200.h), the step
after the ISP in a camera graph.

Mirrors holoscan::color_convert (modules/color-convert/include/holoscan/
color_convert/): `PixelFormat`-style constants, `ImageView` as `CcImageC`,
`ConversionParams` as `params(...)`, `compute_mapping`,
`validate_conversion`, `packed_size`/`plane_size`/`packed_view`, and
`Converter(...).convert(source, destination, params, stream)` for device
images. Errors raise as the reference's do: ValueError where it throws
std::invalid_argument, IspError where it throws std::runtime_error.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence, Tuple

from . import check, lib

NV12, NV16, I420, YUYV, UYVY, RGB8, BGR8, RGBA8, BGRA8, MONO8, MONO16, RGB16 = range(12)
ALL_FORMATS = tuple(range(12))
BT601, BT709, BT2020 = range(3)
LIMITED, FULL = range(2)
NEAREST, BILINEAR, AREA = range(3)
HOST, DEVICE = range(2)


class CcPlaneC(C.Structure):
    _fields_ = [("data", C.c_void_p), ("pitch", C.c_size_t)]


class CcImageC(C.Structure):
    _fields_ = [("format", C.c_int32), ("width", C.c_int32), ("height", C.c_int32), ("location", C.c_int32),
                ("planes", CcPlaneC * 3)]


class CcRectC(C.Structure):
    _fields_ = [("x", C.c_int32), ("y", C.c_int32), ("width", C.c_int32), ("height", C.c_int32)]

    def tuple(self) -> Tuple[int, int, int, int]:
        return (self.x, self.y, self.width, self.height)


class CcParamsC(C.Structure):
    _fields_ = [("matrix", C.c_int32), ("range", C.c_int32), ("mode", C.c_int32), ("has_crop", C.c_int32),
                ("crop", CcRectC), ("letterbox", C.c_int32), ("fill_rgb", C.c_uint8 * 3)]


class CcMappingC(C.Structure):
    _fields_ = [("source", CcRectC), ("content", CcRectC)]


class CcFormatInfoC(C.Structure):
    _fields_ = [("model", C.c_int32), ("planes", C.c_int32), ("chroma_shift_x", C.c_int32),
                ("chroma_shift_y", C.c_int32), ("bytes_per_sample", C.c_int32), ("channels", C.c_int32)]


_bound = False


def _cc():
    global _bound
    L = lib()
    if not _bound:
        P = C.POINTER
        L.cc_b200_params_default.argtypes = [P(CcParamsC)]
        L.cc_b200_params_default.restype = None
        L.cc_b200_format_info.argtypes = [C.c_int32, P(CcFormatInfoC)]
        L.cc_b200_plane_size.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int32, P(C.c_size_t), P(C.c_int32)]
        L.cc_b200_packed_size.argtypes = [C.c_int32, C.c_int32, C.c_int32]
        L.cc_b200_packed_size.restype = C.c_size_t
        L.cc_b200_packed_view.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, P(CcImageC)]
        for what in ("format", "matrix", "range", "resize_mode"):
            getattr(L, f"cc_b200_{what}_name").argtypes = [C.c_int32]
            getattr(L, f"cc_b200_{what}_name").restype = C.c_char_p
            getattr(L, f"cc_b200_parse_{what}").argtypes = [C.c_char_p]
            getattr(L, f"cc_b200_parse_{what}").restype = C.c_int32
        L.cc_b200_compute_mapping.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, P(CcParamsC),
                                              P(CcMappingC)]
        L.cc_b200_validate.argtypes = [P(CcImageC), P(CcImageC), P(CcParamsC)]
        L.cc_b200_convert.argtypes = [P(CcImageC), P(CcImageC), P(CcParamsC), C.c_void_p]
        L.cc_b200_test_pattern.argtypes = [P(CcImageC), C.c_uint32, C.c_void_p]
        _bound = True
    return L


def params(matrix: int = BT601, range: int = LIMITED, mode: int = BILINEAR,  # noqa: A002  (the reference's name)
           crop: Optional[Sequence[int]] = None, letterbox: bool = False,
           fill_rgb: Sequence[int] = (0, 0, 0)) -> CcParamsC:
    """ConversionParams (conversion.hpp:56-67); crop is (x, y, width, height)."""
    p = CcParamsC()
    _cc().cc_b200_params_default(C.byref(p))
    p.matrix, p.range, p.mode = matrix, range, mode
    if crop is not None:
        p.has_crop = 1
        p.crop = CcRectC(*crop)
    p.letterbox = 1 if letterbox else 0
    for i, v in enumerate(fill_rgb):
        p.fill_rgb[i] = v
    return p


def format_info(fmt: int) -> CcFormatInfoC:
    info = CcFormatInfoC()
    check(_cc().cc_b200_format_info(fmt, C.byref(info)))
    return info


def plane_size(fmt: int, width: int, height: int, plane: int) -> Tuple[int, int]:
    """(row bytes, rows) of one plane of a packed image."""
    rb, rows = C.c_size_t(), C.c_int32()
    check(_cc().cc_b200_plane_size(fmt, width, height, plane, C.byref(rb), C.byref(rows)))
    return rb.value, rows.value


def packed_size(fmt: int, width: int, height: int) -> int:
    return int(_cc().cc_b200_packed_size(fmt, width, height))


def packed_view(base: int, fmt: int, width: int, height: int, location: int = DEVICE) -> CcImageC:
    """A view of a packed image at `base`: planes one after the other, rows unpadded."""
    v = CcImageC()
    check(_cc().cc_b200_packed_view(C.c_void_p(base), fmt, width, height, location, C.byref(v)))
    return v


def format_name(fmt: int) -> str:
    return _cc().cc_b200_format_name(fmt).decode()


def parse_format(name: str) -> Optional[int]:
    v = _cc().cc_b200_parse_format(name.encode())
    return None if v < 0 else v


def matrix_name(m: int) -> str:
    return _cc().cc_b200_matrix_name(m).decode()


def parse_matrix(name: str) -> Optional[int]:
    v = _cc().cc_b200_parse_matrix(name.encode())
    return None if v < 0 else v


def range_name(r: int) -> str:
    return _cc().cc_b200_range_name(r).decode()


def parse_range(name: str) -> Optional[int]:
    v = _cc().cc_b200_parse_range(name.encode())
    return None if v < 0 else v


def resize_mode_name(m: int) -> str:
    return _cc().cc_b200_resize_mode_name(m).decode()


def parse_resize_mode(name: str) -> Optional[int]:
    v = _cc().cc_b200_parse_resize_mode(name.encode())
    return None if v < 0 else v


def compute_mapping(source_width: int, source_height: int, width: int, height: int, destination: int,
                    p: CcParamsC) -> Tuple[Tuple[int, int, int, int], Tuple[int, int, int, int]]:
    """(source rect, content rect), each (x, y, width, height)."""
    m = CcMappingC()
    check(_cc().cc_b200_compute_mapping(source_width, source_height, width, height, destination, C.byref(p),
                                        C.byref(m)))
    return m.source.tuple(), m.content.tuple()


def validate_conversion(source: CcImageC, destination: CcImageC, p: CcParamsC) -> None:
    check(_cc().cc_b200_validate(C.byref(source), C.byref(destination), C.byref(p)))


def test_pattern(rgb8: CcImageC, frame: int, stream: int = 0) -> None:
    """launch_test_pattern: the synthetic camera's frame into a device RGB8 view."""
    check(_cc().cc_b200_test_pattern(C.byref(rgb8), frame, C.c_void_p(stream)))


class Converter:
    """Converter(Backend::kCuda) (converter.hpp:43-80): stateless; convert()
    queues one kernel on `stream` after its earlier work and returns."""

    def __init__(self) -> None:
        _cc()

    def convert(self, source: CcImageC, destination: CcImageC, p: CcParamsC, stream: int = 0) -> None:
        check(_cc().cc_b200_convert(C.byref(source), C.byref(destination), C.byref(p), C.c_void_p(stream)))
