"""The golden cases: the reference's pipeline test settings, and their fixtures.

Each case restates one setting of modules/isp/tests/pipeline_test.cpp (the
`camera()`, `flat()` and ramp frames and the tweaks applied to
synthetic_isp_params). `build_case` renders them with the reference's own
synthetic camera (needs oracle/_ref, so only where the reference tree is);
`load_case` reads the committed fixture, which also holds the reference's
outputs for every frame (tests/golden/make_golden.py).
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

from isp_b200 import abi

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# SampleFormat list of pipeline_test.cpp:50-57: format, bits, black.
FORMATS = [
    (abi.U8, 8, 16.0),
    (abi.U16, 10, 64.0),
    (abi.U16, 12, 256.0),
    (abi.U16, 16, 4096.0),
    (abi.RAW10, 10, 64.0),
    (abi.RAW12, 12, 256.0),
]
FORMAT_NAMES = ["u8", "u16_10", "u16_12", "u16_16", "raw10", "raw12"]
PATTERNS = [abi.RGGB, abi.BGGR, abi.GRBG, abi.GBRG]
PATTERN_NAMES = ["RGGB", "BGGR", "GRBG", "GBRG"]


@dataclass
class Case:
    name: str
    params: abi.IspParams
    raws: List[abi.RawFrame]
    sequence: List[int]  # raw index of each frame, in order
    out_format: int
    with_stats: bool = True
    exposure: Tuple[int, float] = (0, 0.0)
    expected: Optional[List[Dict[str, np.ndarray]]] = None  # per frame, from the fixture

    def frame_raws(self) -> List[abi.RawFrame]:
        return [self.raws[i] for i in self.sequence]


# ---- Frames (need the reference's synthetic camera) ------------------------

def _camera(pattern, f, width=480, height=360, **kw):
    """camera() of pipeline_test.cpp:75-88."""
    import oracle

    fmt, bits, black = f
    step = black / 16.0
    cfg = oracle.ref_synthetic_config(width, height, pattern, fmt, bits,
                                      black_levels=(black, black + step, black + 2 * step, black + 3 * step),
                                      vignetting=0.4, frame=3)
    for key, value in kw.items():
        if key in ("wb_gains",):
            for k in range(3):
                cfg.wb_gains[k] = value[k]
        else:
            setattr(cfg, key, value)
    return cfg


def flat(width, height, r, g, b, pattern=abi.RGGB) -> abi.RawFrame:
    """flat() of pipeline_test.cpp:459-482: 16-bit samples, one value per colour."""
    cfa = [[0, 1, 1, 2], [2, 1, 1, 0], [1, 0, 2, 1], [1, 2, 0, 1]][pattern]  # colour per quad position
    values = np.array([r, g, b], np.uint16)
    y, x = np.mgrid[0:height, 0:width]
    img = values[np.array(cfa)[((y & 1) << 1) | (x & 1)]].astype("<u2")
    return abi.RawFrame(img.view(np.uint8).ravel().copy(), width, height, 2 * width, abi.U16, 16, pattern)


def ramp(width=256, height=4) -> abi.RawFrame:
    """The horizontal gray ramp of tone_curves (pipeline_test.cpp:519-532)."""
    img = np.tile((np.arange(width) * 257).astype("<u2"), (height, 1))
    return abi.RawFrame(img.view(np.uint8).ravel().copy(), width, height, 2 * width, abi.U16, 16, abi.RGGB)


def linear_params() -> abi.IspParams:
    """linear_params() of pipeline_test.cpp:484-489."""
    return abi.IspParams(tone_curve=abi.LINEAR, white_level=65535.0)


def _render(cfg) -> abi.RawFrame:
    import oracle

    return oracle.ref_render(cfg)


def _synth_params(cfg, grid=17) -> abi.IspParams:
    import oracle

    return oracle.ref_synthetic_params(cfg, grid)


# ---- The case list ---------------------------------------------------------

def _cuda_matches_cpu(name: str) -> Case:
    """cuda_matches_cpu (pipeline_test.cpp:164-235): two frames each."""
    method_name, _, kind = name.partition("_")
    method = abi.BILINEAR if method_name == "bilinear" else abi.MALVAR
    exposure = (10_000_000, 2.0)
    if kind == "plain":
        cfg = _camera(abi.RGGB, FORMATS[2], 200, 150)
        fmt = abi.RGB8
    elif kind == "sharpened":
        cfg = _camera(abi.GBRG, FORMATS[2], 200, 150)
        fmt = abi.RGBA8
    elif kind == "odd_size":
        cfg = _camera(abi.GRBG, FORMATS[4], 67, 35)
        fmt = abi.RGB16
    elif kind == "gray_world":
        cfg = _camera(abi.BGGR, FORMATS[5], 96, 72)  # 160x120 in the reference; smaller fixture
        fmt = abi.RGB32F
    else:
        cfg = _camera(abi.RGGB, FORMATS[0], 160, 120)
        fmt = abi.RGB8
    p = _synth_params(cfg, 9)
    p.demosaic = method
    if kind == "sharpened":
        p.sharpen = 1.5
    elif kind == "odd_size":
        p.sharpen = 0.5
    elif kind == "gray_world":
        p.white_balance = abi.GRAY_WORLD
        p.tone_curve = abi.GAMMA
    elif kind == "white_patch_lut":
        p.white_balance = abi.WHITE_PATCH
        p.tone_curve = abi.LUT
        p.lut = np.array([0.0, 0.6, 0.85, 1.0], np.float32)
        s = p.lens_shading
        four = np.repeat(np.asarray(s.gains, np.float32), 4).reshape(-1, 4)
        four = four * (np.float32(1.0) + np.float32(0.01) * np.arange(4, dtype=np.float32))
        p.lens_shading = abi.LensShading(s.width, s.height, 4, four.astype(np.float32).ravel())
    return Case(name, p, [_render(cfg)], [0, 0], fmt, True, exposure)


def _edge(name: str) -> Case:
    """edge_cases, tiny sizes (pipeline_test.cpp:637-661)."""
    _, size, pat = name.split("_")
    w, h = (int(v) for v in size.split("x"))
    pattern = PATTERN_NAMES.index(pat)
    p = linear_params()
    p.sharpen = 1.0
    return Case(name, p, [flat(w, h, 9000, 21000, 15000, pattern)], [0], abi.RGB8)


def _sweep(name: str) -> Case:
    """Every sample format x pattern x method on the chart (accuracy, pipeline_test.cpp:99-141)."""
    _, fname, pat, method_name = name.split("_", 3)
    f = FORMATS[FORMAT_NAMES.index(fname.replace("-", "_"))]
    cfg = _camera(PATTERN_NAMES.index(pat), f, 64, 40)
    p = _synth_params(cfg)
    p.demosaic = abi.BILINEAR if method_name == "bilinear" else abi.MALVAR
    return Case(name, p, [_render(cfg)], [0], abi.RGB8, True)


def _special(name: str) -> Case:
    if name == "statistics_flat":
        level = int(0.09 * 65535.0 + 0.5)
        p = linear_params()
        p.auto_exposure = abi.AutoExposure(target=0.18, damping=1.0, max_exposure_ns=20_000_000)
        return Case(name, p, [flat(64, 48, level, level, level)], [0, 0], abi.RGB8, True, (15_000_000, 1.0))
    if name == "statistics_chart":
        cfg = _camera(abi.BGGR, FORMATS[3], 123, 77)
        return Case(name, _synth_params(cfg), [_render(cfg)], [0], abi.RGB16)
    if name == "black_frame":
        cfg = _camera(abi.RGGB, FORMATS[2], 64, 48, exposure=1e-6)
        p = _synth_params(cfg)
        p.white_balance = abi.GRAY_WORLD
        return Case(name, p, [_render(cfg)], [0, 0], abi.RGB8)
    if name == "saturated":
        cfg = _camera(abi.RGGB, FORMATS[2], 160, 120, exposure=4.0)
        return Case(name, _synth_params(cfg), [_render(cfg)], [0], abi.RGB8)
    if name.startswith("padded_"):
        f = FORMATS[{"padded_u8": 0, "padded_u16": 2, "padded_raw12": 5}[name]]
        cfg = _camera(abi.GBRG, f, 75, 41)
        packed = _render(cfg)
        pitch = packed.pitch + 38
        data = np.full(pitch * cfg.height, 0xAB, np.uint8)
        for y in range(cfg.height):
            data[y * pitch: y * pitch + packed.pitch] = packed.data[y * packed.pitch: (y + 1) * packed.pitch]
        padded = abi.RawFrame(data, packed.width, packed.height, pitch, packed.format, packed.bit_depth,
                              packed.pattern)
        return Case(name, _synth_params(cfg, 5), [packed, padded], [0, 1], abi.RGB8)
    if name == "color_matrix":
        p = linear_params()
        p.ccm = (0.9, 0.2, -0.1, 0.05, 0.8, 0.15, -0.2, 0.1, 1.1)
        p.wb_gains = (1.25, 1.0, 0.8)
        return Case(name, p, [flat(32, 24, 20000, 30000, 40000, abi.GBRG)], [0], abi.RGB32F)
    if name.startswith("tone_"):
        curve = {"tone_srgb": abi.SRGB, "tone_gamma": abi.GAMMA, "tone_linear": abi.LINEAR, "tone_lut": abi.LUT}[name]
        p = linear_params()
        p.demosaic = abi.BILINEAR
        p.tone_curve = curve
        if curve == abi.LUT:
            p.lut = np.array([1.0, 0.0], np.float32)
        return Case(name, p, [ramp()], [0], abi.RGB32F)
    if name.startswith("awb_") and name != "awb_smoothing":
        _, mode, pat = name.split("_")
        kind = 1 if mode == "gray" else 0
        cfg = _camera(PATTERN_NAMES.index(pat), FORMATS[2], 160, 120, kind=kind, wb_gains=(2.1, 1.0, 1.45))
        p = _synth_params(cfg)
        p.white_balance = abi.GRAY_WORLD if mode == "gray" else abi.WHITE_PATCH
        p.wb_gains = (1.0, 1.0, 1.0)
        return Case(name, p, [_render(cfg)], [0], abi.RGB8)
    if name == "awb_smoothing":
        cfg1 = _camera(abi.RGGB, FORMATS[2], 160, 120, kind=1, wb_gains=(2.0, 1.0, 1.5))
        cfg2 = _camera(abi.RGGB, FORMATS[2], 160, 120, kind=1, wb_gains=(1.5, 1.0, 2.0))
        p = _synth_params(cfg2)
        p.white_balance = abi.GRAY_WORLD
        p.awb_smoothing = 0.25
        return Case(name, p, [_render(cfg1), _render(cfg2)], [0, 1, 1, 1, 1, 1], abi.RGB8)
    if name == "sequence_two_streams":
        raws = []
        cfg = None
        for f in range(8):
            cfg = _camera(abi.RGGB, FORMATS[2], 128, 72, frame=f,
                          wb_gains=(1.9 if f % 2 == 0 else 1.4, 1.0, 1.6 if f % 2 == 0 else 2.1))
            raws.append(_render(cfg))
        p = _synth_params(cfg, 9)
        p.white_balance = abi.GRAY_WORLD
        p.sharpen = 0.5
        return Case(name, p, raws, list(range(8)), abi.RGB8)
    if name == "white_patch_sharp_rgba":
        cfg = _camera(abi.BGGR, FORMATS[5], 130, 66)
        p = _synth_params(cfg)
        p.white_balance = abi.WHITE_PATCH
        p.white_patch_percentile = 0.995
        p.sharpen = 0.5
        return Case(name, p, [_render(cfg)], [0, 0, 0], abi.RGBA8, True, (5_000_000, 0.0))
    raise KeyError(name)


def _case_names() -> List[str]:
    names = []
    for m in ("bilinear", "malvar"):
        for kind in ("plain", "sharpened", "odd_size", "gray_world", "white_patch_lut"):
            names.append(f"{m}_{kind}")
    for w, h in ((2, 2), (3, 5), (33, 17), (5, 2)):
        for pat in PATTERN_NAMES:
            names.append(f"edge_{w}x{h}_{pat}")
    for fname in FORMAT_NAMES:
        for pat in PATTERN_NAMES:
            for m in ("bilinear", "malvar"):
                names.append(f"sweep_{fname.replace('_', '-')}_{pat}_{m}")
    names += ["statistics_flat", "statistics_chart", "black_frame", "saturated", "padded_u8", "padded_u16",
              "padded_raw12", "color_matrix", "tone_srgb", "tone_gamma", "tone_linear", "tone_lut"]
    for mode in ("gray", "white"):
        for pat in PATTERN_NAMES:
            names.append(f"awb_{mode}_{pat}")
    names += ["awb_smoothing", "sequence_two_streams", "white_patch_sharp_rgba"]
    return names


CASES = _case_names()


def build_case(name: str) -> Case:
    if name.startswith(("bilinear_", "malvar_")):
        return _cuda_matches_cpu(name)
    if name.startswith("edge_"):
        return _edge(name)
    if name.startswith("sweep_"):
        return _sweep(name)
    return _special(name)


def load_case(name: str) -> Case:
    """The committed fixture: inputs, settings and the reference's outputs."""
    z = np.load(os.path.join(GOLDEN_DIR, f"{name}.npz"))
    meta = json.loads(bytes(z["meta"]).decode())
    params = abi.IspParams.from_dict(meta["params"], z["lsc"] if "lsc" in z else None)
    raws = [abi.RawFrame(z[f"raw{i}"], r["width"], r["height"], r["pitch"], r["format"], r["bit_depth"],
                         r["pattern"]) for i, r in enumerate(meta["raws"])]
    expected = []
    for f in range(len(meta["sequence"])):
        e = {"image": z[f"image{f}"], "awb": z[f"awb{f}"]}
        if meta["with_stats"]:
            e["hist"] = z[f"hist{f}"]
            e["stats"] = z[f"stats{f}"]
        expected.append(e)
    return Case(name, params, raws, meta["sequence"], meta["out_format"], meta["with_stats"],
                tuple(meta["exposure"]), expected)
