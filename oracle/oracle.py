"""Oracle wrapper — TEST INFRASTRUCTURE ONLY.

ctypes binding of oracle/_ref/liblgcr_ref_*.so: the reference's own compute
code (MysteryDove/vapoursynth-LGCR src/{maps,kernels,recon,algos,bm}.cpp,
compiled unmodified by oracle/Makefile) driven by the restated Recon
orchestration in oracle/harness.cpp (lgcrCreate src/plugin.cpp:998-1158,
lgcrGetFrame src/plugin.cpp:177-721).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use
this module, and only as the checker or the timed CPU baseline.

Variants: "scalar" (the parity oracle, the reference's liblgcr_scalar.so
flags), "avx2" (the reference's liblgcr.so flags; the CPU baseline) and
"f64" (the scalar code with float mapped to double).
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(HERE, "_ref")
UNSET_INT = -(2 ** 31)

_VARIANTS = {"scalar": "liblgcr_ref_scalar.so", "avx2": "liblgcr_ref_avx2.so",
             "f64": "liblgcr_ref_f64.so"}


class Params(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_int), ("height", ctypes.c_int),
        ("kernel", ctypes.c_char_p), ("taps", ctypes.c_int), ("algo", ctypes.c_int),
        ("b", ctypes.c_double), ("c", ctypes.c_double),
        ("strength", ctypes.c_double), ("sigma", ctypes.c_double),
        ("sratio", ctypes.c_double), ("sdb", ctypes.c_double),
        ("stretch", ctypes.c_double), ("gsigma", ctypes.c_double),
        ("rescue", ctypes.c_double),
        ("ridge", ctypes.c_int), ("cedge", ctypes.c_int),
        ("ar", ctypes.c_double), ("reg", ctypes.c_double),
        ("loc", ctypes.c_char_p), ("sparse", ctypes.c_int),
        ("bp", ctypes.c_double), ("ms", ctypes.c_double), ("qgate", ctypes.c_double),
        ("bm", ctypes.c_int),
    ]


class Format(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in (
        "color_family", "sample_type", "bits_per_sample", "subsampling_w",
        "subsampling_h", "width", "height")]


class PlaneDesc(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("stride", ctypes.c_ssize_t),
                ("width", ctypes.c_int), ("height", ctypes.c_int)]


class FrameStats(ctypes.Structure):
    _fields_ = [("output_pixels", ctypes.c_uint64),
                ("sparse_active_pixels", ctypes.c_uint64),
                ("sparse_total_pixels", ctypes.c_uint64),
                ("active_output_pixels", ctypes.c_uint64),
                ("active_chroma_pixels", ctypes.c_uint64),
                ("sparse_active_ratio", ctypes.c_double),
                ("device_ms", ctypes.c_double)]


class Debug(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in (
        "jxx", "jxy", "jyy", "lc", "ms", "plain_u", "plain_v", "seed", "mask",
        "chroma_mask")] + [("active_output", ctypes.c_uint64),
                           ("active_chroma", ctypes.c_uint64),
                           ("has_workset", ctypes.c_int)]


INT_ARGS = ("width", "height", "taps", "algo", "ridge", "cedge", "sparse", "bm")
FLOAT_ARGS = ("b", "c", "strength", "sigma", "sratio", "sdb", "stretch", "gsigma",
              "rescue", "ar", "reg", "bp", "ms", "qgate")
STR_ARGS = ("kernel", "loc")


def make_params(**kwargs) -> Params:
    p = Params()
    for name in INT_ARGS:
        setattr(p, name, UNSET_INT)
    for name in FLOAT_ARGS:
        setattr(p, name, math.nan)
    for name in STR_ARGS:
        setattr(p, name, None)
    for key, value in kwargs.items():
        if value is None:
            continue
        if key in INT_ARGS:
            setattr(p, key, int(value))
        elif key in FLOAT_ARGS:
            setattr(p, key, float(value))
        elif key in STR_ARGS:
            setattr(p, key, value.encode())
        else:
            raise TypeError(f"Recon: unknown argument {key!r}")
    return p


def make_format(planes, bits=None) -> Format:
    y, u, _ = planes
    dt = np.asarray(y).dtype
    is_float = dt == np.float32
    if bits is None:
        bits = 32 if is_float else (8 if dt == np.uint8 else 16)
    h, w = y.shape
    ch, cw = u.shape
    ssw = {1: 0, 2: 1}.get(int(round(w / cw)), 2) if cw else 0
    ssh = {1: 0, 2: 1}.get(int(round(h / ch)), 2) if ch else 0
    return Format(3, 1 if is_float else 0, bits, ssw, ssh, w, h)


def _lib(variant: str):
    path = os.path.join(LIBDIR, _VARIANTS[variant])
    if not os.path.exists(path):
        raise FileNotFoundError(f"oracle library missing: {path} (run make -C oracle)")
    lib = ctypes.CDLL(path)
    lib.oracle_create.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(Format),
                                  ctypes.POINTER(ctypes.c_void_p), ctypes.c_char_p,
                                  ctypes.c_size_t]
    lib.oracle_create.restype = ctypes.c_int
    lib.oracle_destroy.argtypes = [ctypes.c_void_p]
    lib.oracle_frame.argtypes = [ctypes.c_void_p, ctypes.POINTER(PlaneDesc),
                                 ctypes.POINTER(PlaneDesc), ctypes.c_int, ctypes.c_int,
                                 ctypes.c_int, ctypes.POINTER(Debug),
                                 ctypes.POINTER(FrameStats)]
    lib.oracle_frame.restype = ctypes.c_int
    return lib


_LIBS: dict = {}


def library(variant: str = "scalar"):
    if variant not in _LIBS:
        _LIBS[variant] = _lib(variant)
    return _LIBS[variant]


def available(variant: str = "scalar") -> bool:
    return os.path.exists(os.path.join(LIBDIR, _VARIANTS[variant]))


class OracleError(Exception):
    pass


def _planes(arrays):
    arr = (PlaneDesc * 3)()
    for i, a in enumerate(arrays):
        arr[i].data = a.ctypes.data
        arr[i].stride = a.strides[0]
        arr[i].height, arr[i].width = a.shape
    return arr


class Recon:
    """Reference Recon over numpy planes (one filter instance)."""

    def __init__(self, fmt: Format, variant: str = "scalar", **kwargs):
        self.lib = library(variant)
        self.fmt = fmt
        self.params = make_params(**kwargs)
        handle = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        status = self.lib.oracle_create(ctypes.byref(self.params), ctypes.byref(fmt),
                                        ctypes.byref(handle), err, 512)
        if status != 0:
            raise OracleError(err.value.decode())
        self.handle = handle
        self.out_w = self.params.width if self.params.width != UNSET_INT else fmt.width
        self.out_h = self.params.height if self.params.height != UNSET_INT else fmt.height

    def __del__(self):
        if getattr(self, "handle", None):
            self.lib.oracle_destroy(self.handle)
            self.handle = None

    def frame(self, planes, chroma_location: int = -1, threads: int = 1,
              debug: bool = False, profile: bool = False):
        planes = [np.ascontiguousarray(p) for p in planes]
        dtype = planes[0].dtype
        outs = [np.zeros((self.out_h, self.out_w), dtype=dtype) for _ in range(3)]
        dbg = None
        bufs = {}
        if debug:
            sh, sw = planes[0].shape
            ch, cw = planes[1].shape
            dbg = Debug()
            for name, shape, dt in (("jxx", (sh, sw), np.float32), ("jxy", (sh, sw), np.float32),
                                    ("jyy", (sh, sw), np.float32), ("lc", (ch, cw), np.float32),
                                    ("ms", (ch, cw), np.float32),
                                    ("plain_u", (self.out_h, self.out_w), np.float32),
                                    ("plain_v", (self.out_h, self.out_w), np.float32),
                                    ("seed", (sh, sw), np.uint8), ("mask", (sh, sw), np.uint8),
                                    ("chroma_mask", (ch, cw), np.uint8)):
                bufs[name] = np.full(shape, np.nan if dt == np.float32 else 255, dtype=dt)
                setattr(dbg, name, bufs[name].ctypes.data)
        stats = FrameStats()
        status = self.lib.oracle_frame(self.handle, _planes(planes), _planes(outs),
                                       int(chroma_location), int(threads), int(profile),
                                       ctypes.byref(dbg) if dbg is not None else None,
                                       ctypes.byref(stats))
        if status != 0:
            raise OracleError(f"oracle_frame failed: {status}")
        if debug:
            bufs["active_output"] = dbg.active_output
            bufs["active_chroma"] = dbg.active_chroma
            bufs["has_workset"] = dbg.has_workset
            return outs, bufs, stats
        return outs, stats


def recon(planes, chroma_location: int = -1, variant: str = "scalar", bits=None, **kwargs):
    """One-shot reference Recon of one frame; returns (Y, U, V) outputs."""
    fmt = make_format(planes, bits)
    outs, _ = Recon(fmt, variant, **kwargs).frame(planes, chroma_location)
    return outs


def sharpen(planes, bits=None, variant: str = "scalar", **kwargs):
    """Reference Sharpen of one frame (sharpenCreate + sharpenGetFrame,
    src/plugin.cpp:14-111); returns the (Y, U, V) outputs. Raises
    OracleError with the reference's message on invalid arguments."""
    lib = library(variant)
    fn = lib.oracle_sharpen_frame
    fn.argtypes = [ctypes.POINTER(Format)] + [ctypes.c_double] * 5 + [
        ctypes.POINTER(PlaneDesc), ctypes.POINTER(PlaneDesc), ctypes.c_char_p, ctypes.c_size_t]
    fn.restype = ctypes.c_int
    planes = [np.ascontiguousarray(p) for p in planes]
    outs = [np.zeros_like(p) for p in planes]
    fmt = make_format(planes, bits)
    vals = [float(kwargs.pop(k, math.nan)) for k in ("alpha", "sigma", "sratio", "gspatial", "ar")]
    if kwargs:
        raise OracleError(f"unknown Sharpen arguments {sorted(kwargs)}")
    err = ctypes.create_string_buffer(512)
    if fn(ctypes.byref(fmt), *vals, _planes(planes), _planes(outs), err, 512) != 0:
        raise OracleError(err.value.decode())
    return outs


class TReconParams(ctypes.Structure):
    _fields_ = [("strength", ctypes.c_double), ("sigma", ctypes.c_double),
                ("sratio", ctypes.c_double), ("sdb", ctypes.c_double),
                ("gsigma", ctypes.c_double), ("stretch", ctypes.c_double),
                ("ar", ctypes.c_double), ("ridge", ctypes.c_int), ("sparse", ctypes.c_int),
                ("ms", ctypes.c_double), ("trad", ctypes.c_int), ("tsearch", ctypes.c_int),
                ("tsad", ctypes.c_double), ("bm", ctypes.c_int)]


TRECON_INT_ARGS = ("ridge", "sparse", "trad", "tsearch", "bm")


def trecon_params(**kwargs) -> TReconParams:
    p = TReconParams()
    for name, ctype in TReconParams._fields_:
        setattr(p, name, UNSET_INT if ctype is ctypes.c_int else math.nan)
    for key, value in kwargs.items():
        if key not in dict(TReconParams._fields_):
            raise OracleError(f"TRecon: unknown argument {key!r}")
        if value is not None:
            setattr(p, key, int(value) if key in TRECON_INT_ARGS else float(value))
    return p


def trecon(cur, nbrs, bits=None, num_frames=None, chroma_location: int = -1,
           variant: str = "scalar", **kwargs):
    """Reference TRecon of one frame (tReconCreate + tReconGetFrame,
    src/plugin.cpp:723-990): `cur` the frame's planes, `nbrs` the planes of
    its temporal neighbours in temporalFrameNumbers order. Returns the
    4:4:4 (Y, U, V) outputs."""
    lib = library(variant)
    fn = lib.oracle_trecon_frame
    fn.argtypes = [ctypes.POINTER(TReconParams), ctypes.POINTER(Format), ctypes.c_int,
                   ctypes.POINTER(PlaneDesc), ctypes.POINTER(PlaneDesc), ctypes.c_int,
                   ctypes.POINTER(PlaneDesc), ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t]
    fn.restype = ctypes.c_int
    cur = [np.ascontiguousarray(p) for p in cur]
    nbrs = [[np.ascontiguousarray(p) for p in f] for f in nbrs]
    h, w = cur[0].shape
    outs = [np.zeros((h, w), dtype=cur[0].dtype) for _ in range(3)]
    fmt = make_format(cur, bits)
    flat = (PlaneDesc * max(1, 3 * len(nbrs)))()
    for k, f in enumerate(nbrs):
        d = _planes(f)
        for q in range(3):
            flat[3 * k + q] = d[q]
    err = ctypes.create_string_buffer(512)
    params = trecon_params(**kwargs)
    if num_frames is None:
        num_frames = 1 + len(nbrs)
    if fn(ctypes.byref(params), ctypes.byref(fmt), int(num_frames), _planes(cur), flat,
          len(nbrs), _planes(outs), int(chroma_location), err, 512) != 0:
        raise OracleError(err.value.decode())
    return outs


def downsample(planes, bits=None, variant: str = "scalar", quality=None, kernel=None,
               strength=None, loc=None, color_family: int = 3, subsampling=(0, 0)):
    """Reference Downsample of one frame: the reference's own downsampleCreate
    and downsampleGetFrame (src/downsample.cpp:740-918), compiled unmodified
    and driven by oracle/ds_host.cpp. `planes` are the 4:4:4 source planes;
    returns (U, V, chroma_location) with U, V of (h/2, w/2) in the source's
    sample type. Raises OracleError with the reference's message on invalid
    arguments. `color_family` / `subsampling` override the source format, to
    check the create-time validation."""
    lib = library(variant)
    fn = lib.oracle_downsample_frame
    fn.argtypes = [ctypes.c_int] * 7 + [ctypes.POINTER(ctypes.c_void_p),
                                        ctypes.POINTER(ctypes.c_longlong), ctypes.c_int,
                                        ctypes.c_char_p, ctypes.c_double, ctypes.c_int,
                                        ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.POINTER(ctypes.c_int), ctypes.c_char_p, ctypes.c_int]
    fn.restype = ctypes.c_int
    planes = [np.ascontiguousarray(p) for p in planes]
    dt = planes[0].dtype
    is_float = dt == np.float32
    if bits is None:
        bits = 32 if is_float else (8 if dt == np.uint8 else 16)
    h, w = planes[0].shape
    ptrs = (ctypes.c_void_p * 3)(*[p.ctypes.data for p in planes])
    strides = (ctypes.c_longlong * 3)(*[p.strides[0] for p in planes])
    ou = np.zeros((h // 2, w // 2), dtype=dt)
    ov = np.zeros((h // 2, w // 2), dtype=dt)
    loc_out = ctypes.c_int(-1)
    err = ctypes.create_string_buffer(512)
    rc = fn(w, h, int(color_family), 1 if is_float else 0, int(bits), int(subsampling[0]),
            int(subsampling[1]), ptrs, strides, UNSET_INT if quality is None else int(quality),
            None if kernel is None else kernel.encode(),
            0.0 if strength is None else float(strength), 0 if strength is None else 1,
            None if loc is None else loc.encode(), ou.ctypes.data, ov.ctypes.data,
            ctypes.byref(loc_out), err, 512)
    if rc != 0:
        raise OracleError(err.value.decode())
    return ou, ov, loc_out.value
