"""The C-ABI library without a GPU: it loads, exports every entry point that
include/isp_b200.h and include/cc_b200.h declare, and its host-side settings logic (defaults,
validation and messages, row sizes, tone tables) is the reference's
(modules/isp/src/isp_params.cpp:85-237), checked against the oracle and, where
it is built, the reference itself."""
import ctypes as C
import math
import os
import re

import numpy as np
import pytest

import isp_b200
import oracle
from goldens import CASES, load_case
from isp_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(header="isp_b200.h", prefix="isp_b200_"):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(" + prefix + r"\w+)\s*\(", text)))


@pytest.mark.parametrize("header,prefix,least", [("isp_b200.h", "isp_b200_", 12), ("cc_b200.h", "cc_b200_", 17)])
def test_library_exports_every_declared_symbol(header, prefix, least):
    lib = isp_b200.lib()
    names = declared_functions(header, prefix)
    assert len(names) >= least
    for name in names:
        assert hasattr(lib, name), f"{name} is declared in include/{header} but not exported"
    assert lib.isp_b200_abi_version() == abi.ABI_VERSION


def test_checked_library_exports_every_isp_symbol():
    """libisp_b200_checked.so (the bounds-checked build) is a drop-in for the ISP part of the library."""
    lib = C.CDLL(os.path.join(ROOT, "holoscan-zozo-modules_b200", "libisp_b200_checked.so"))
    for name in declared_functions():
        assert hasattr(lib, name), f"{name} is declared in include/isp_b200.h but not exported by the checked build"
    assert lib.isp_b200_abi_version() == abi.ABI_VERSION
    count, first = C.c_uint32(7), C.c_uint64(7)
    assert lib.isp_b200_checked_violations(None, C.byref(count), C.byref(first)) == abi.EINVAL


def test_defaults_are_the_reference_defaults():
    c = isp_b200.params_default()
    p = abi.IspParams().to_c().c
    for name, _ in abi.ParamsC._fields_:
        a, b = getattr(c, name), getattr(p, name)
        if name in ("lsc_gains", "lut"):
            continue
        if name == "auto_exposure":
            a, b = bytes(a), bytes(b)
        elif hasattr(a, "_length_"):
            a, b = list(a), list(b)
        assert a == b, name


def test_raw_row_bytes():
    # isp_params.cpp:184-197 and host/params_test.cpp:95-100.
    for fmt in (abi.U8, abi.U16, abi.RAW10, abi.RAW12):
        for w in (0, 1, 2, 3, 4, 5, 7, 67, 3840, 8192):
            assert isp_b200.raw_row_bytes(fmt, w) == abi.raw_row_bytes(fmt, w) == oracle._lib_oracle().oracle_raw_row_bytes(fmt, w)
    assert isp_b200.raw_row_bytes(abi.RAW10, 5) == 10 and isp_b200.raw_row_bytes(abi.RAW12, 3) == 6


def _bad_params():
    # The rejects of pipeline_test.cpp:706-721, and one per remaining check.
    cases = []
    def add(**kw):
        p = abi.IspParams()
        for k, v in kw.items():
            setattr(p, k, v)
        cases.append(p)
    add(black_level=-1.0)
    add(black_level=float("nan"))
    add(channel_black_levels=[0.0, 0.0, 70000.0, 0.0])
    add(white_level=-5.0)
    add(wb_gains=(1.0, 0.0, 1.0))
    add(wb_gains=(1.0, 65.0, 1.0))
    add(ccm=(1.0, 0, 0, 0, float("nan"), 0, 0, 0, 1.0))
    add(ccm=(17.0, 0, 0, 0, 1, 0, 0, 0, 1.0))
    add(awb_smoothing=0.0)
    add(white_patch_percentile=0.4)
    add(white_patch_percentile=1.0)
    add(sharpen=5.0)
    add(sharpen=-1.0)
    add(tone_curve=abi.LUT)
    add(tone_curve=abi.LUT, lut=np.array([0.5], np.float32))
    add(tone_curve=abi.LUT, lut=np.array([0.0, 1.5], np.float32))
    add(tone_curve=abi.GAMMA, gamma=0.05)
    add(lens_shading=abi.LensShading(2, 2, 1, np.ones(3, np.float32)))
    add(lens_shading=abi.LensShading(1, 2, 1, np.ones(2, np.float32)))
    add(lens_shading=abi.LensShading(2, 2, 3, np.ones(12, np.float32)))
    add(lens_shading=abi.LensShading(2, 2, 1, np.array([1, 1, 1, 17], np.float32)))
    add(auto_exposure=abi.AutoExposure(max_exposure_ns=1))
    add(auto_exposure=abi.AutoExposure(min_exposure_ns=0))
    add(auto_exposure=abi.AutoExposure(target=1.0))
    add(auto_exposure=abi.AutoExposure(damping=1.5))
    add(auto_exposure=abi.AutoExposure(min_gain=2.0, max_gain=1.0))
    return cases


@pytest.mark.parametrize("index", range(len(_bad_params())))
def test_rejected_params_same_message(index):
    p = _bad_params()[index]
    with pytest.raises(ValueError) as err:
        isp_b200.validate_params(p)
    assert oracle.oracle_validate_params(p) == str(err.value)
    if oracle.reference_available():
        assert oracle.ref_validate_params(p) == str(err.value)


def test_accepted_params():
    for name in CASES[:20]:
        isp_b200.validate_params(load_case(name).params)
    isp_b200.validate_params(abi.IspParams())


def test_rejected_raw_views_same_message():
    # pipeline_test.cpp:723-744 and host/params_test.cpp validation.
    buf = np.zeros(64, np.uint16)
    good = abi.RawViewC(buf.ctypes.data, 4, 4, 8, abi.U16, 12, abi.RGGB)
    isp_b200.validate_raw(good, abi.IspParams())
    tweaks = [
        dict(width=1), dict(pitch=6), dict(bit_depth=17), dict(format=abi.RAW10), dict(data=None),
        dict(bit_depth=0), dict(width=16385), dict(format=abi.U16, pitch=9), dict(data=buf.ctypes.data + 1),
    ]
    for t in tweaks:
        v = abi.RawViewC(good.data, good.width, good.height, good.pitch, good.format, good.bit_depth, good.pattern)
        for k, val in t.items():
            setattr(v, k, val)
        with pytest.raises(ValueError) as err:
            isp_b200.validate_raw(v, abi.IspParams())
        assert oracle.oracle_validate_raw(v, abi.IspParams()) == str(err.value), t
        if oracle.reference_available():
            assert oracle.ref_validate_raw(v, abi.IspParams()) == str(err.value), t
    for params in (abi.IspParams(black_level=5000.0), abi.IspParams(white_level=5000.0),
                   abi.IspParams(black_level=4095.0)):
        with pytest.raises(ValueError) as err:
            isp_b200.validate_raw(good, params)
        assert oracle.oracle_validate_raw(good, params) == str(err.value)


@pytest.mark.parametrize("curve,gamma", [(abi.SRGB, 2.2), (abi.GAMMA, 2.2), (abi.GAMMA, 0.45), (abi.GAMMA, 7.3),
                                         (abi.LINEAR, 2.2)])
def test_tone_tables_bit_exact(curve, gamma):
    p = abi.IspParams(tone_curve=curve, gamma=gamma)
    got = isp_b200.tone_lut(p)
    assert got.size == abi.TONE_LUT_SIZE and got[0] == 0.0 and got[-1] == 1.0
    assert np.all(np.diff(got) > 0)
    assert np.array_equal(got.view(np.uint32), oracle.oracle_tone_lut(p).view(np.uint32))
    if oracle.reference_available():
        assert np.array_equal(got.view(np.uint32), oracle.ref_tone_lut(p).view(np.uint32))
    if curve == abi.SRGB:
        # host/params_test.cpp:112-115: sRGB codes 18 % gray as about 0.46.
        assert abs(got[int(0.18 * (abi.TONE_LUT_SIZE - 1))] - 0.4613) < 2e-3


def test_user_table_verbatim():
    lut = np.array([0.0, 0.25, 1.0], np.float32)
    assert np.array_equal(isp_b200.tone_lut(abi.IspParams(tone_curve=abi.LUT, lut=lut)), lut)
