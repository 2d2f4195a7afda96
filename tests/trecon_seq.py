"""Seeded synthetic clips with known motion for the TRecon tests: one 4:4:4
polygon scene, each frame a window of it displaced by that frame's motion,
chroma box-averaged to the clip's subsampling, light per-frame noise on the
samples."""
import numpy as np

from lgcr import synthetic as S


def make_clip(width, height, fmt, motions, seed=0, margin=16, noise=1.0):
    base_fmt = S.FrameFormat(fmt.bits, 0, 0)
    base = S.make_frame(width + 2 * margin, height + 2 * margin, base_fmt, seed=seed)
    rng = np.random.default_rng(seed + 1)
    frames = []
    for (mx, my) in motions:
        x0, y0 = margin + mx, margin + my
        planes = []
        for p, plane in enumerate(base):
            win = plane[y0:y0 + height, x0:x0 + width].astype(np.float64)
            if p and fmt.ssw:
                win = 0.5 * (win[:, 0::2] + win[:, 1::2])
            if p and fmt.ssh:
                win = 0.5 * (win[0::2, :] + win[1::2, :])
            if fmt.is_float:
                win = win + rng.normal(0.0, noise / 219.0, win.shape)
                planes.append(win.astype(np.float32))
            else:
                top = (1 << fmt.bits) - 1
                win = win + rng.normal(0.0, noise * (top / 255.0), win.shape)
                planes.append(np.clip(np.rint(win), 0, top).astype(fmt.dtype))
        frames.append(tuple(planes))
    return frames
