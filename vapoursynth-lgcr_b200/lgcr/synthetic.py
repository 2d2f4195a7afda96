"""Seeded synthetic test frames: flat-shaded polygon "animation" scenes.

The generator follows the benchmark recipe of this Recon implementation:

* Luma: a flat-shaded base of 20-60 random polygons with uniform fills in
  [16, 235] (8-bit units), band-limited Gaussian noise (sigma 3 LSB at 8 bit,
  8 LSB at 10 bit, about 4 px correlation) and 1-px dark outlines on about
  30% of the polygon edges.
* Chroma: per polygon U, V = a_k * Y + b_k + N(0, 2), clipped to [16, 240],
  a_k ~ U(-0.6, 0.6), b_k ~ U(60, 190); full-resolution chroma is box
  averaged to the requested subsampling (2x2 for 4:2:0, 2x1 for 4:2:2).
* Depths: 8-bit codes as above; 10-bit scales to [64, 940] (chroma
  [64, 960]); 16-bit to [4096, 60160] (chroma [4096, 61440]); float gives
  Y in [0, 1] and chroma in [-0.5, 0.5].
* Options: `antialias` renders polygon coverage at 2x supersampling;
  `extra_noise` adds white noise (sigma 4 LSB luma, 3 LSB chroma, 8-bit
  units) before subsampling; `blur_chroma` low-passes full-resolution
  chroma (for 4:4:4 sources).

Frames are reproducible from (seed, geometry, format): seed = base + index.
"""
from __future__ import annotations

import dataclasses

import numpy as np

try:  # scipy is only used for the noise low-pass
    from scipy.ndimage import gaussian_filter as _gaussian_filter
except Exception:  # pragma: no cover
    _gaussian_filter = None


@dataclasses.dataclass(frozen=True)
class FrameFormat:
    """Planar YUV format: sample type, depth and log2 chroma subsampling."""
    bits: int = 8                 # 8..16, or 32 for float
    ssw: int = 1
    ssh: int = 1

    @property
    def is_float(self) -> bool:
        return self.bits == 32

    @property
    def dtype(self):
        if self.is_float:
            return np.float32
        return np.uint8 if self.bits == 8 else np.uint16

    @property
    def name(self) -> str:
        sub = {(1, 1): "420", (1, 0): "422", (0, 0): "444"}[(self.ssw, self.ssh)]
        return f"YUV{sub}" + ("PS" if self.is_float else f"P{self.bits}")


YUV420P8 = FrameFormat(8, 1, 1)
YUV420P10 = FrameFormat(10, 1, 1)
YUV420P16 = FrameFormat(16, 1, 1)
YUV420PS = FrameFormat(32, 1, 1)
YUV422P10 = FrameFormat(10, 1, 0)
YUV444PS = FrameFormat(32, 0, 0)


def _blur(a: np.ndarray, sigma: float) -> np.ndarray:
    if _gaussian_filter is not None:
        return _gaussian_filter(a, sigma, mode="wrap")
    # separable FFT fallback
    out = a
    for axis in (0, 1):
        n = a.shape[axis]
        f = np.fft.rfftfreq(n)
        g = np.exp(-2.0 * (np.pi * f * sigma) ** 2)
        shape = [1, 1]
        shape[axis] = g.size
        out = np.fft.irfft(np.fft.rfft(out, axis=axis) * g.reshape(shape), n=n, axis=axis)
    return out


def _polygon_fill(label: np.ndarray, verts: np.ndarray, value: int, scale: int) -> None:
    """Even-odd fill of a closed polygon (pixel centres) into `label`."""
    h, w = label.shape
    ys = verts[:, 1]
    y0 = max(0, int(np.floor(ys.min() - 0.5)))
    y1 = min(h, int(np.ceil(ys.max() + 0.5)) + 1)
    if y1 <= y0:
        return
    rows = np.arange(y0, y1)
    centres = (rows + 0.5) / scale
    toggle = np.zeros((y1 - y0, w + 1), dtype=np.int32)
    n = len(verts)
    for e in range(n):
        xa, ya = verts[e] / scale
        xb, yb = verts[(e + 1) % n] / scale
        if ya == yb:
            continue
        lo, hi = (ya, yb) if ya < yb else (yb, ya)
        sel = (centres >= lo) & (centres < hi)
        if not sel.any():
            continue
        yc = centres[sel]
        xc = xa + (yc - ya) * (xb - xa) / (yb - ya)
        col = np.clip(np.ceil(xc * scale - 0.5), 0, w).astype(np.int64)
        np.add.at(toggle, (np.nonzero(sel)[0], col), 1)
    inside = (np.cumsum(toggle[:, :w], axis=1) & 1).astype(bool)
    region = label[y0:y1]
    region[inside] = value


def _draw_segment(mask: np.ndarray, a: np.ndarray, b: np.ndarray) -> None:
    h, w = mask.shape
    length = float(np.hypot(*(b - a)))
    steps = max(2, int(length * 2))
    t = np.linspace(0.0, 1.0, steps)
    xs = np.floor(a[0] + (b[0] - a[0]) * t).astype(np.int64)
    ys = np.floor(a[1] + (b[1] - a[1]) * t).astype(np.int64)
    ok = (xs >= 0) & (xs < w) & (ys >= 0) & (ys < h)
    mask[ys[ok], xs[ok]] = True


def _scene(rng: np.random.Generator, w: int, h: int, scale: int):
    """Polygon label map (at `scale`x supersampling) + per-label shading."""
    npoly = int(rng.integers(20, 61))
    label = np.zeros((h * scale, w * scale), dtype=np.int16)
    outline = np.zeros((h, w), dtype=bool)
    fills = rng.uniform(16.0, 235.0, size=npoly + 1)
    slopes = rng.uniform(-0.6, 0.6, size=(npoly + 1, 2))
    offsets = rng.uniform(60.0, 190.0, size=(npoly + 1, 2))
    diag = float(np.hypot(w, h))
    for k in range(1, npoly + 1):
        nv = int(rng.integers(3, 9))
        cx, cy = rng.uniform(0, w), rng.uniform(0, h)
        radius = rng.uniform(0.03, 0.25) * diag
        ang = np.sort(rng.uniform(0, 2 * np.pi, size=nv))
        rad = radius * rng.uniform(0.4, 1.0, size=nv)
        verts = np.stack([cx + rad * np.cos(ang), cy + rad * np.sin(ang)], axis=1)
        _polygon_fill(label, verts * scale, k, scale)
        for e in range(nv):
            if rng.uniform() < 0.3:
                _draw_segment(outline, verts[e], verts[(e + 1) % nv])
    return label, outline, fills, slopes, offsets


def _box(a: np.ndarray, fy: int, fx: int) -> np.ndarray:
    if fy == 1 and fx == 1:
        return a
    h, w = a.shape
    hh, ww = h // fy, w // fx
    return a[: hh * fy, : ww * fx].reshape(hh, fy, ww, fx).mean(axis=(1, 3))


def make_frame(width: int, height: int, fmt: FrameFormat = YUV420P8, seed: int = 0,
               antialias: bool = False, extra_noise: bool = False,
               blur_chroma: bool = False):
    """Return (Y, U, V) numpy planes for one seeded synthetic frame."""
    rng = np.random.default_rng(seed)
    scale = 2 if antialias else 1
    label, outline, fills, slopes, offsets = _scene(rng, width, height, scale)
    luma8 = fills[label]
    if scale > 1:
        luma8 = _box(luma8, scale, scale)
    luma8 = luma8.copy()
    luma8[outline] = np.minimum(luma8[outline], 16.0 + 0.25 * (luma8[outline] - 16.0))

    if fmt.is_float:
        lo, hi, clo, chi, lsb = 0.0, 1.0, -0.5, 0.5, 1.0 / 219.0
    elif fmt.bits == 8:
        lo, hi, clo, chi, lsb = 16.0, 235.0, 16.0, 240.0, 1.0
    elif fmt.bits == 10:
        lo, hi, clo, chi, lsb = 64.0, 940.0, 64.0, 960.0, 876.0 / 219.0
    else:
        top = float((1 << fmt.bits) - 1)
        lo, hi = 16.0 / 255.0 * top, 235.0 / 255.0 * top
        clo, chi = 16.0 / 255.0 * top, 240.0 / 255.0 * top
        if fmt.bits == 16:
            lo, hi, clo, chi = 4096.0, 60160.0, 4096.0, 61440.0
        lsb = (hi - lo) / 219.0
    luma_sigma = 8.0 if fmt.bits == 10 else 3.0 * lsb

    # band-limited noise (about 4 px correlation), renormalised to sigma
    noise = _blur(rng.standard_normal((height, width)), 2.0)
    noise *= luma_sigma / max(noise.std(), 1e-12)
    y = lo + (luma8 - 16.0) * (hi - lo) / 219.0 + noise
    if extra_noise:
        y = y + rng.standard_normal((height, width)) * 4.0 * lsb

    # chroma from the shaded luma, per polygon
    lab = label if scale == 1 else label[::scale, ::scale]
    chroma = []
    for c in range(2):
        c8 = slopes[lab, c] * luma8 + offsets[lab, c] + rng.normal(0.0, 2.0, size=luma8.shape)
        c8 = np.clip(c8, 16.0, 240.0)
        ct = clo + (c8 - 16.0) * (chi - clo) / 224.0
        if extra_noise:
            ct = ct + rng.standard_normal(ct.shape) * 3.0 * (chi - clo) / 224.0
        if blur_chroma:
            ct = _blur(ct, 1.5)
        chroma.append(ct)

    fy, fx = 1 << fmt.ssh, 1 << fmt.ssw
    cw = (width + fx - 1) // fx
    ch = (height + fy - 1) // fy
    planes = [y]
    for ct in chroma:
        if fx > 1 or fy > 1:
            padded = np.pad(ct, ((0, ch * fy - height), (0, cw * fx - width)), mode="edge")
            ct = _box(padded, fy, fx)
        planes.append(ct)

    out = []
    for p in planes:
        if fmt.is_float:
            out.append(np.ascontiguousarray(p, dtype=np.float32))
        else:
            top = (1 << fmt.bits) - 1
            out.append(np.ascontiguousarray(np.clip(np.rint(p), 0, top)).astype(fmt.dtype))
    return tuple(out)


def make_frames(count: int, width: int, height: int, fmt: FrameFormat = YUV420P8,
                base_seed: int = 1000, **options):
    """`count` frames with seeds base_seed + index."""
    return [make_frame(width, height, fmt, base_seed + i, **options) for i in range(count)]


def edge_scene(width: int, height: int, fmt: FrameFormat = YUV420PS):
    """Small deterministic edge + diagonal + texture scene (vertical edge at
    the centre column, a diagonal, a low-amplitude sinusoid), box-subsampled.
    Used for known-answer tests."""
    yy, xx = np.mgrid[0:height, 0:width]
    edge = (xx >= width // 2).astype(np.float64)
    diagonal = (xx * height > yy * width).astype(np.float64)
    texture = 0.02 * np.sin(xx * 0.37) * np.cos(yy * 0.29)
    full = (0.17 + 0.31 * edge + 0.04 * diagonal + texture,
            -0.23 + 0.52 * edge + 0.3 * texture,
            0.29 - 0.57 * edge - 0.3 * texture)
    return from_float_planes(full, fmt)


def from_float_planes(full, fmt: FrameFormat):
    """Quantise normalised full-resolution planes (Y in [0,1], chroma centred
    on 0) to `fmt`, box-subsampling chroma."""
    y, u, v = (np.asarray(p, dtype=np.float64) for p in full)
    height, width = y.shape
    fy, fx = 1 << fmt.ssh, 1 << fmt.ssw
    cw = (width + fx - 1) // fx
    ch = (height + fy - 1) // fy
    planes = [y]
    for c in (u, v):
        if fx > 1 or fy > 1:
            c = _box(np.pad(c, ((0, ch * fy - height), (0, cw * fx - width)), mode="edge"), fy, fx)
        planes.append(c)
    if fmt.is_float:
        return tuple(np.ascontiguousarray(p, dtype=np.float32) for p in planes)
    top = float((1 << fmt.bits) - 1)
    out = [np.clip(np.rint(planes[0] * top), 0, top)]
    for c in planes[1:]:
        out.append(np.clip(np.rint((c + 0.5) * top), 0, top))
    return tuple(np.ascontiguousarray(p).astype(fmt.dtype) for p in out)
