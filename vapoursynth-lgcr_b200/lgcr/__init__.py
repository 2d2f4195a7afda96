"""B200-native LGCR Recon: Python mirror of the reference's `lgcr.Recon`.

The reference registers `Recon` with VapourSynth as
    clip:vnode; width,height,taps,algo,ridge,cedge,sparse,bm:int:opt;
    kernel,loc:data:opt; b,c,strength,sigma,sratio,sdb,stretch,gsigma,rescue,
    ar,reg,bp,ms,qgate:float:opt                      (src/plugin.cpp:1166-1171)
This module exposes the same arguments and error messages over the C ABI in
include/lgcr_b200.h (lgcr_recon_create / lgcr_recon_frame); frames are
numpy planes (host memory) or CUDA torch tensors (device memory).

The compute path is the CUDA library liblgcr_b200.so built in-tree; there is
no CPU fallback: without the library or a GPU, calls raise.
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# LGCR_B200_LIBRARY selects another build of the library (a different path)
LIBPATH = os.environ.get("LGCR_B200_LIBRARY") or os.path.join(HERE, "liblgcr_b200.so")
UNSET_INT = -(2 ** 31)

LGCR_OK = 0
LGCR_E_INVALID = 1
LGCR_MEM_HOST = 0
LGCR_MEM_DEVICE = 1

INT_ARGS = ("width", "height", "taps", "algo", "ridge", "cedge", "sparse", "bm")
FLOAT_ARGS = ("b", "c", "strength", "sigma", "sratio", "sdb", "stretch", "gsigma",
              "rescue", "ar", "reg", "bp", "ms", "qgate")
STR_ARGS = ("kernel", "loc")


class Error(Exception):
    """Raised where VapourSynth would raise vs.Error for Recon."""


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


class Plane(ctypes.Structure):
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


class BatchItem(ctypes.Structure):
    _fields_ = [("filter", ctypes.c_void_p), ("inp", Plane * 3), ("out", Plane * 3),
                ("chroma_location", ctypes.c_int)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("device_budget_bytes", ctypes.c_size_t), ("max_batch", ctypes.c_int),
                ("lanes", ctypes.c_int), ("queue_capacity", ctypes.c_int)]


class RequestInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("submit_ms", ctypes.c_double),
                ("start_ms", ctypes.c_double), ("done_ms", ctypes.c_double),
                ("batch_size", ctypes.c_int)]


# Every entry point declared in include/lgcr_b200.h.
EXPORTS = (
    "lgcr_params_init", "lgcr_recon_create", "lgcr_recon_destroy",
    "lgcr_recon_output_format", "lgcr_recon_frame", "lgcr_last_error",
    "lgcr_batch_create", "lgcr_batch_destroy", "lgcr_batch_run",
    "lgcr_batch_launch_count", "lgcr_autotune", "lgcr_batch_autotune",
    "lgcr_server_create", "lgcr_server_submit", "lgcr_server_wait", "lgcr_server_destroy",
    "lgcr_sharpen_params_init", "lgcr_sharpen_create", "lgcr_sharpen_frame",
    "lgcr_sharpen_destroy", "lgcr_trecon_params_init", "lgcr_trecon_create",
    "lgcr_trecon_neighbors", "lgcr_trecon_frame", "lgcr_trecon_destroy",
    "lgcr_downsample_params_init", "lgcr_downsample_create", "lgcr_downsample_destroy",
    "lgcr_downsample_chroma_location", "lgcr_downsample_frame",
)

_lib = None


def library():
    """Load liblgcr_b200.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise Error(f"liblgcr_b200.so is missing ({LIBPATH}); build it with "
                    "python vapoursynth-lgcr_b200/build.py")
    lib = ctypes.CDLL(LIBPATH)
    lib.lgcr_params_init.argtypes = [ctypes.POINTER(Params)]
    lib.lgcr_recon_create.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(Format),
                                      ctypes.POINTER(ctypes.c_void_p), ctypes.c_char_p,
                                      ctypes.c_size_t]
    lib.lgcr_recon_create.restype = ctypes.c_int
    lib.lgcr_recon_destroy.argtypes = [ctypes.c_void_p]
    lib.lgcr_recon_output_format.argtypes = [ctypes.c_void_p, ctypes.POINTER(Format)]
    lib.lgcr_recon_frame.argtypes = [ctypes.c_void_p, ctypes.POINTER(Plane),
                                     ctypes.POINTER(Plane), ctypes.c_int, ctypes.c_int,
                                     ctypes.c_void_p, ctypes.POINTER(FrameStats)]
    lib.lgcr_recon_frame.restype = ctypes.c_int
    lib.lgcr_last_error.restype = ctypes.c_char_p
    sigs = {
        "lgcr_batch_create": ([ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
        "lgcr_batch_destroy": ([ctypes.c_void_p], None),
        "lgcr_batch_run": ([ctypes.c_void_p, ctypes.POINTER(BatchItem), ctypes.c_int,
                            ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
        "lgcr_batch_launch_count": ([ctypes.c_void_p], ctypes.c_int),
        "lgcr_batch_set_profiling": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
        "lgcr_batch_stage_times": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                    ctypes.POINTER(ctypes.c_int), ctypes.c_int], ctypes.c_int),
        "lgcr_stage_count": ([], ctypes.c_int),
        "lgcr_stage_name": ([ctypes.c_int], ctypes.c_char_p),
        "lgcr_autotune": ([ctypes.POINTER(BatchItem), ctypes.c_int, ctypes.c_void_p,
                           ctypes.c_char_p, ctypes.c_size_t], ctypes.c_int),
        "lgcr_batch_autotune": ([ctypes.c_void_p, ctypes.POINTER(BatchItem), ctypes.c_int,
                                 ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t], ctypes.c_int),
        "lgcr_server_create": ([ctypes.POINTER(ServerConfig), ctypes.POINTER(ctypes.c_void_p)],
                               ctypes.c_int),
        "lgcr_server_submit": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(Plane),
                                ctypes.POINTER(Plane), ctypes.c_int], ctypes.c_int64),
        "lgcr_server_wait": ([ctypes.c_void_p, ctypes.c_int64, ctypes.c_int,
                              ctypes.POINTER(RequestInfo)], ctypes.c_int),
        "lgcr_server_destroy": ([ctypes.c_void_p], None),
    }
    for name, (args, res) in sigs.items():
        if hasattr(lib, name):
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
    _lib = lib
    return lib


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
            setattr(p, key, value.encode() if isinstance(value, str) else value)
        else:
            raise Error(f"Recon: argument {key!r} is not supported")
    return p


def video_format(width, height, bits=8, ssw=1, ssh=1, is_float=None) -> Format:
    """Format of a planar YUV clip (bits 32 = float)."""
    if is_float is None:
        is_float = bits == 32
    return Format(3, 1 if is_float else 0, 32 if is_float else bits, ssw, ssh, width, height)


def format_of(planes, bits=None) -> Format:
    """Format of a (Y, U, V) numpy/torch plane tuple."""
    y, u, _ = planes
    h, w = y.shape
    ch, cw = u.shape
    dt = str(getattr(y, "dtype", ""))
    is_float = "float32" in dt
    if bits is None:
        bits = 32 if is_float else (8 if "uint8" in dt else 16)
    ssw = 0 if cw == w else 1
    ssh = 0 if ch == h else 1
    return video_format(w, h, bits, ssw, ssh, is_float)


def _plane_desc(a) -> Plane:
    p = Plane()
    if a is None:
        return p
    if hasattr(a, "data_ptr"):           # torch tensor
        p.data = a.data_ptr()
        p.stride = a.stride(0) * a.element_size()
    else:
        p.data = a.ctypes.data
        p.stride = a.strides[0]
    p.height, p.width = a.shape
    return p


def planes_desc(arrays):
    arr = (Plane * 3)()
    for i, a in enumerate(arrays):
        arr[i] = _plane_desc(a)
    return arr


class Recon:
    """One Recon filter instance (lgcrCreate); call frame() per frame."""

    def __init__(self, fmt: Format, **kwargs):
        self.lib = library()
        self.fmt = fmt
        self.params = make_params(**kwargs)
        handle = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        status = self.lib.lgcr_recon_create(ctypes.byref(self.params), ctypes.byref(fmt),
                                            ctypes.byref(handle), err, 512)
        if status != LGCR_OK:
            raise Error(err.value.decode())
        self.handle = handle
        out = Format()
        self.lib.lgcr_recon_output_format(self.handle, ctypes.byref(out))
        self.out_w, self.out_h = out.width, out.height
        # the jinc kernel is the radial (2D) path
        self.radial = kwargs.get("kernel") == "jinc"

    def close(self):
        if getattr(self, "handle", None):
            self.lib.lgcr_recon_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def dtype(self):
        if self.fmt.sample_type == 1:
            return np.float32
        return np.uint8 if self.fmt.bits_per_sample == 8 else np.uint16

    def frame(self, planes, chroma_location: int = -1, out=None, stats: bool = False,
              stream=None, share_luma: bool = False):
        """Reconstruct one frame.

        numpy planes run through host memory (upload, run, download);
        CUDA tensors run in device memory on `stream` (a torch stream or
        raw handle) without waiting unless stats=True."""
        device = hasattr(planes[0], "data_ptr")
        if out is None:
            if device:
                import torch
                tdt = {np.uint8: torch.uint8, np.uint16: torch.uint16,
                       np.float32: torch.float32}[self.dtype]
                out = [torch.empty((self.out_h, self.out_w), dtype=tdt, device=planes[0].device)
                       for _ in range(3)]
            else:
                out = [np.empty((self.out_h, self.out_w), dtype=self.dtype) for _ in range(3)]
            if share_luma:
                out[0] = None
        else:
            out = list(out)
        if not device:
            planes = [np.ascontiguousarray(p) for p in planes]
        st = FrameStats()
        handle = None
        if stream is not None:
            handle = getattr(stream, "cuda_stream", stream)
        status = self.lib.lgcr_recon_frame(
            self.handle, planes_desc(planes), planes_desc(out), int(chroma_location),
            LGCR_MEM_DEVICE if device else LGCR_MEM_HOST, handle,
            ctypes.byref(st) if stats else None)
        if status != LGCR_OK:
            raise Error(self.lib.lgcr_last_error().decode())
        if stats:
            return out, st
        return out


class SharpenParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("alpha", "sigma", "sratio", "gspatial", "ar")]


SHARPEN_ARGS = ("alpha", "sigma", "sratio", "gspatial", "ar")


class Sharpen:
    """The reference's `lgcr.Sharpen` (sharpenCreate / sharpenGetFrame,
    src/plugin.cpp:14-111): a 5x5 gated bilateral unsharp mask; same format
    in and out. Arguments: alpha, sigma, sratio, gspatial, ar."""

    def __init__(self, fmt: Format, **kwargs):
        self.lib = library()
        lib = self.lib
        lib.lgcr_sharpen_create.argtypes = [ctypes.POINTER(SharpenParams), ctypes.POINTER(Format),
                                            ctypes.POINTER(ctypes.c_void_p), ctypes.c_char_p,
                                            ctypes.c_size_t]
        lib.lgcr_sharpen_frame.argtypes = [ctypes.c_void_p, ctypes.POINTER(Plane),
                                           ctypes.POINTER(Plane), ctypes.c_int, ctypes.c_void_p]
        lib.lgcr_sharpen_destroy.argtypes = [ctypes.c_void_p]
        params = SharpenParams(*([math.nan] * 5))
        for key, value in kwargs.items():
            if key not in SHARPEN_ARGS:
                raise Error(f"Sharpen: argument {key!r} is not supported")
            if value is not None:
                setattr(params, key, float(value))
        self.fmt = fmt
        handle = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        if lib.lgcr_sharpen_create(ctypes.byref(params), ctypes.byref(fmt), ctypes.byref(handle),
                                   err, 512) != LGCR_OK:
            raise Error(err.value.decode())
        self.handle = handle

    def close(self):
        if getattr(self, "handle", None):
            self.lib.lgcr_sharpen_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def frame(self, planes, out=None, stream=None):
        """Sharpen one frame (numpy planes through host memory, or CUDA
        tensors on `stream` without waiting)."""
        device = hasattr(planes[0], "data_ptr")
        if not device:
            planes = [np.ascontiguousarray(p) for p in planes]
        if out is None:
            if device:
                import torch
                out = [torch.empty_like(p) for p in planes]
            else:
                out = [np.empty_like(p) for p in planes]
        handle = getattr(stream, "cuda_stream", stream) if stream is not None else None
        status = self.lib.lgcr_sharpen_frame(self.handle, planes_desc(planes), planes_desc(out),
                                             LGCR_MEM_DEVICE if device else LGCR_MEM_HOST, handle)
        if status != LGCR_OK:
            raise Error(self.lib.lgcr_last_error().decode())
        return out


class TReconParams(ctypes.Structure):
    _fields_ = [("strength", ctypes.c_double), ("sigma", ctypes.c_double),
                ("sratio", ctypes.c_double), ("sdb", ctypes.c_double),
                ("gsigma", ctypes.c_double), ("stretch", ctypes.c_double),
                ("ar", ctypes.c_double), ("ridge", ctypes.c_int), ("sparse", ctypes.c_int),
                ("ms", ctypes.c_double), ("trad", ctypes.c_int), ("tsearch", ctypes.c_int),
                ("tsad", ctypes.c_double), ("bm", ctypes.c_int)]


TRECON_INT_ARGS = ("ridge", "sparse", "trad", "tsearch", "bm")


class TRecon:
    """The reference's `lgcr.TRecon` (tReconCreate / tReconGetFrame,
    src/plugin.cpp:723-990): motion-compensated temporal Recon of a clip of
    `num_frames` frames. frame(n, get) reconstructs frame n, fetching the
    planes of frame n and of its neighbours through get(i)."""

    def __init__(self, fmt: Format, num_frames: int, **kwargs):
        self.lib = library()
        lib = self.lib
        lib.lgcr_trecon_create.argtypes = [ctypes.POINTER(TReconParams), ctypes.POINTER(Format),
                                           ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                           ctypes.c_char_p, ctypes.c_size_t]
        lib.lgcr_trecon_frame.argtypes = [ctypes.c_void_p, ctypes.POINTER(Plane),
                                          ctypes.POINTER(Plane), ctypes.c_int,
                                          ctypes.POINTER(Plane), ctypes.c_int, ctypes.c_int,
                                          ctypes.c_void_p]
        lib.lgcr_trecon_neighbors.argtypes = [ctypes.c_void_p, ctypes.c_int,
                                              ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        lib.lgcr_trecon_destroy.argtypes = [ctypes.c_void_p]
        params = TReconParams()
        for name, ctype in TReconParams._fields_:
            setattr(params, name, UNSET_INT if ctype is ctypes.c_int else math.nan)
        for key, value in kwargs.items():
            if key not in dict(TReconParams._fields_):
                raise Error(f"TRecon: argument {key!r} is not supported")
            if value is not None:
                setattr(params, key, int(value) if key in TRECON_INT_ARGS else float(value))
        self.fmt = fmt
        handle = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        if lib.lgcr_trecon_create(ctypes.byref(params), ctypes.byref(fmt), int(num_frames),
                                  ctypes.byref(handle), err, 512) != LGCR_OK:
            raise Error(err.value.decode())
        self.handle = handle

    def close(self):
        if getattr(self, "handle", None):
            self.lib.lgcr_trecon_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def neighbors(self, n: int):
        buf = (ctypes.c_int * 16)()
        count = self.lib.lgcr_trecon_neighbors(self.handle, int(n), buf, 16)
        return list(buf[:count])

    def frame(self, n: int, get, chroma_location: int = -1, out=None, stream=None):
        """Reconstruct frame n; get(i) returns frame i's (Y, U, V) planes
        (numpy through host memory, or CUDA tensors on `stream`)."""
        cur = get(n)
        nbrs = [get(i) for i in self.neighbors(n)]
        device = hasattr(cur[0], "data_ptr")
        h, w = cur[0].shape
        if not device:
            cur = [np.ascontiguousarray(p) for p in cur]
            nbrs = [[np.ascontiguousarray(p) for p in f] for f in nbrs]
        if out is None:
            if device:
                import torch
                out = [torch.empty((h, w), dtype=cur[0].dtype, device=cur[0].device)
                       for _ in range(3)]
            else:
                out = [np.empty((h, w), dtype=cur[0].dtype) for _ in range(3)]
        flat = (Plane * max(1, 3 * len(nbrs)))()
        for k, f in enumerate(nbrs):
            for q in range(3):
                flat[3 * k + q] = _plane_desc(f[q])
        handle = getattr(stream, "cuda_stream", stream) if stream is not None else None
        status = self.lib.lgcr_trecon_frame(self.handle, planes_desc(cur), flat, len(nbrs),
                                            planes_desc(out), int(chroma_location),
                                            LGCR_MEM_DEVICE if device else LGCR_MEM_HOST, handle)
        if status != LGCR_OK:
            raise Error(self.lib.lgcr_last_error().decode())
        return out


def recon(planes, chroma_location: int = -1, bits=None, **kwargs):
    """One-shot Recon of a (Y, U, V) frame; returns the output planes."""
    return Recon(format_of(planes, bits), **kwargs).frame(planes, chroma_location)


class DownsampleParams(ctypes.Structure):
    _fields_ = [("quality", ctypes.c_int), ("kernel", ctypes.c_char_p),
                ("strength", ctypes.c_double), ("strength_set", ctypes.c_int),
                ("loc", ctypes.c_char_p)]


class Downsample:
    """The reference's `lgcr.Downsample` (downsampleCreate /
    downsampleGetFrame, src/downsample.cpp:740-918): 4:4:4 -> 4:2:0 with a
    luma-guided chroma correction. Arguments: quality (0..2), kernel
    ("spline36", "lanczos3", "binomial"), strength (0..1), loc ("left",
    "center", "topleft", "top", "bottomleft", "bottom"). `fmt` is the 4:4:4
    source format with its (even) width and height."""

    def __init__(self, fmt: Format, quality=None, kernel=None, strength=None, loc=None):
        self.lib = library()
        lib = self.lib
        lib.lgcr_downsample_create.argtypes = [ctypes.POINTER(DownsampleParams),
                                               ctypes.POINTER(Format),
                                               ctypes.POINTER(ctypes.c_void_p), ctypes.c_char_p,
                                               ctypes.c_size_t]
        lib.lgcr_downsample_frame.argtypes = [ctypes.c_void_p, ctypes.POINTER(Plane),
                                              ctypes.POINTER(Plane), ctypes.c_int, ctypes.c_void_p]
        lib.lgcr_downsample_destroy.argtypes = [ctypes.c_void_p]
        lib.lgcr_downsample_chroma_location.argtypes = [ctypes.c_void_p]
        params = DownsampleParams(UNSET_INT if quality is None else int(quality),
                                  None if kernel is None else kernel.encode(),
                                  0.0 if strength is None else float(strength),
                                  0 if strength is None else 1,
                                  None if loc is None else loc.encode())
        self.fmt = fmt
        handle = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        if lib.lgcr_downsample_create(ctypes.byref(params), ctypes.byref(fmt),
                                      ctypes.byref(handle), err, 512) != LGCR_OK:
            raise Error(err.value.decode())
        self.handle = handle
        self.chroma_location = lib.lgcr_downsample_chroma_location(handle)

    def close(self):
        if getattr(self, "handle", None):
            self.lib.lgcr_downsample_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def frame(self, planes, out=None, stream=None):
        """Downsample one frame: numpy planes through host memory, or CUDA
        tensors enqueued on `stream` without waiting. Returns (Y, U, V); Y is
        a copy of the source luma in `out[0]` (or the source plane itself
        when out[0] is None)."""
        device = hasattr(planes[0], "data_ptr")
        if not device:
            planes = [np.ascontiguousarray(p) for p in planes]
        h, w = planes[0].shape
        if out is None:
            if device:
                import torch
                out = [None] + [torch.empty((h // 2, w // 2), dtype=planes[0].dtype,
                                            device=planes[0].device) for _ in range(2)]
            else:
                out = [None] + [np.empty((h // 2, w // 2), dtype=planes[0].dtype)
                                for _ in range(2)]
        handle = getattr(stream, "cuda_stream", stream) if stream is not None else None
        status = self.lib.lgcr_downsample_frame(self.handle, planes_desc(planes), planes_desc(out),
                                                LGCR_MEM_DEVICE if device else LGCR_MEM_HOST,
                                                handle)
        if status != LGCR_OK:
            raise Error(self.lib.lgcr_last_error().decode())
        return [planes[0] if out[0] is None else out[0], out[1], out[2]]


class Server:
    """Continuous-batching request loop (lgcr_server_*): admission by a
    device-memory budget, up to `max_batch` frames per device batch, `lanes`
    batches in flight on separate streams."""

    def __init__(self, budget_bytes=8 << 30, max_batch=8, lanes=2, queue_capacity=256):
        self.lib = library()
        self.lib.lgcr_server_pause.argtypes = [ctypes.c_void_p, ctypes.c_int]
        cfg = ServerConfig(int(budget_bytes), int(max_batch), int(lanes), int(queue_capacity))
        handle = ctypes.c_void_p()
        status = self.lib.lgcr_server_create(ctypes.byref(cfg), ctypes.byref(handle))
        if status != LGCR_OK:
            raise Error(self.lib.lgcr_last_error().decode())
        self.handle = handle
        self._keep = {}

    def submit(self, recon: "Recon", planes, out, chroma_location: int = -1) -> int:
        """Queue one frame (host planes); returns a ticket, or a negative
        status (-LGCR_E_BUSY when the queue is full or the frame exceeds the
        budget)."""
        ins, outs = planes_desc(planes), planes_desc(out)
        ticket = self.lib.lgcr_server_submit(self.handle, recon.handle, ins, outs,
                                             int(chroma_location))
        if ticket >= 0:
            self._keep[ticket] = (planes, out)
        return ticket

    def wait(self, ticket: int, timeout_ms: int = -1):
        info = RequestInfo()
        status = self.lib.lgcr_server_wait(self.handle, int(ticket), int(timeout_ms),
                                           ctypes.byref(info))
        if status != 5:                 # LGCR_E_TIMEOUT keeps the request pending
            self._keep.pop(ticket, None)
        return status, info

    def pause(self, on: bool):
        self.lib.lgcr_server_pause(self.handle, 1 if on else 0)

    def close(self):
        if getattr(self, "handle", None):
            self.lib.lgcr_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
