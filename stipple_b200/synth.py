"""Seeded synthetic inputs for the Riemersma workloads.

No public dataset is involved: every workload is generated from a seed.

* RGB8: per channel, the sum of three 2-D sinusoid gradients
  ``A_k * sin(2*pi*(fx*x + fy*y)/N + phi_k)`` with seeded amplitude, phase,
  frequency and orientation, centred on mid-grey, plus Gaussian noise of a
  given sigma; rounded and clamped to 0..255.
* RGBA8: the same RGB plus an alpha channel that is 0 on a seeded Bernoulli
  mask (about 20 % of pixels) and 255 elsewhere.
* Video: the gradient phase advances by a fixed number of pixels per frame
  (a translation) and each frame draws fresh noise.

8-bit samples map to the Q16 range as ``v * 257``, the factor an 8-bit decode
into ImageMagick's 16-bit quantum produces.
"""
from __future__ import annotations

import math

import numpy as np


def _waves(rng: np.random.Generator, channels: int):
    out = []
    for _ in range(channels):
        ch = []
        for _k in range(3):
            amp = rng.uniform(25.0, 55.0)
            phase = rng.uniform(0.0, 2.0 * math.pi)
            theta = rng.uniform(0.0, 2.0 * math.pi)
            cycles = rng.uniform(0.5, 3.0)
            ch.append((amp, phase, math.cos(theta) * cycles, math.sin(theta) * cycles))
        out.append(ch)
    return out


def gradient_rgb8(width: int, height: int, seed: int, sigma: float = 8.0,
                  shift: float = 0.0, noise_seed: int | None = None) -> np.ndarray:
    """(H, W, 3) uint8 gradient+noise image.  ``shift`` translates the gradients
    by that many pixels along x (used for video frames)."""
    rng = np.random.default_rng(seed)
    waves = _waves(rng, 3)
    n = float(max(width, height, 1))
    xs = (np.arange(width, dtype=np.float64) - shift)[None, :]
    ys = np.arange(height, dtype=np.float64)[:, None]
    nrng = np.random.default_rng(seed if noise_seed is None else noise_seed)
    img = np.empty((height, width, 3), np.uint8)
    for c in range(3):
        acc = np.full((height, width), 128.0)
        for amp, phase, fx, fy in waves[c]:
            acc += amp * np.sin(2.0 * math.pi * (fx * xs + fy * ys) / n + phase)
        if sigma > 0:
            acc += nrng.normal(0.0, sigma, size=(height, width))
        img[:, :, c] = np.clip(np.rint(acc), 0, 255).astype(np.uint8)
    return img


def alpha_mask(width: int, height: int, seed: int, transparent: float = 0.2) -> np.ndarray:
    rng = np.random.default_rng(seed ^ 0x5A5A5A5A)
    return np.where(rng.random((height, width)) < transparent, 0, 255).astype(np.uint8)


def gradient_rgba8(width: int, height: int, seed: int, sigma: float = 8.0,
                   transparent: float = 0.2) -> np.ndarray:
    rgb = gradient_rgb8(width, height, seed, sigma)
    a = alpha_mask(width, height, seed, transparent)
    return np.concatenate([rgb, a[:, :, None]], axis=2)


def video_frame(width: int, height: int, seed: int, frame: int, sigma: float = 6.0,
                px_per_frame: float = 2.0) -> np.ndarray:
    return gradient_rgb8(width, height, seed, sigma, shift=px_per_frame * frame,
                         noise_seed=seed * 100003 + frame + 1)


def video_clip_device(width: int, height: int, seed: int, frames: int, device="cuda",
                      sigma: float = 6.0, px_per_frame: float = 2.0):
    """The video clip of video_frame (same seeded gradients, translating
    px_per_frame pixels a frame), generated on the device as a torch uint8
    tensor (frames, H, W, 3).  The per-frame Gaussian noise is drawn from
    torch's generator seeded per frame, so the frames differ from
    video_frame's in the noise draw only; used where a long clip is needed
    fast (120 4K frames), parity tests use video_frame."""
    import torch
    rng = np.random.default_rng(seed)
    waves = _waves(rng, 3)
    n = float(max(width, height, 1))
    out = torch.empty((frames, height, width, 3), dtype=torch.uint8, device=device)
    ys = torch.arange(height, dtype=torch.float64, device=device)[:, None]
    gen = torch.Generator(device=device)
    for f in range(frames):
        xs = (torch.arange(width, dtype=torch.float64, device=device) - px_per_frame * f)[None, :]
        gen.manual_seed(seed * 100003 + f + 1)
        for c in range(3):
            acc = torch.full((height, width), 128.0, dtype=torch.float64, device=device)
            for amp, phase, fx, fy in waves[c]:
                acc += amp * torch.sin(2.0 * math.pi * (fx * xs + fy * ys) / n + phase)
            if sigma > 0:
                acc += sigma * torch.randn((height, width), dtype=torch.float64, device=device,
                                           generator=gen)
            out[f, :, :, c] = torch.clamp(torch.round(acc), 0, 255).to(torch.uint8)
    return out


def to_q16(img8: np.ndarray) -> np.ndarray:
    """uint8 (H, W, 3|4) -> float32 (H, W, 4) Q16 RGBA, opaque when no alpha."""
    h, w, c = img8.shape
    out = np.empty((h, w, 4), np.float32)
    out[:, :, :c] = img8.astype(np.float32) * np.float32(257.0)
    if c == 3:
        out[:, :, 3] = np.float32(65535.0)
    return out


def is_grayscale(img: np.ndarray) -> bool:
    """The reference's greyscale rule: every pixel has r == g == b."""
    return bool(np.all(img[..., 0] == img[..., 1]) and np.all(img[..., 1] == img[..., 2]))


def log_uniform_sizes(n: int, seed: int, lo: int = 1, hi: int = 4096):
    rng = np.random.default_rng(seed)
    ws = np.rint(np.exp(rng.uniform(math.log(lo), math.log(hi), n))).astype(int)
    hs = np.rint(np.exp(rng.uniform(math.log(lo), math.log(hi), n))).astype(int)
    return [(int(max(lo, w)), int(max(lo, h))) for w, h in zip(ws, hs)]


def mixed_batch_spec(n: int = 512, seed: int = 2024):
    """The mixed-size batch of uneven RGBA8 images: n - 4 sizes with W and H
    each log-uniform in 1..4096, plus the forced 1x1, 3x5, 17x13 and 4096x64
    strips.  Returns [(width, height, image_seed, colours)], colours drawn
    from {2, 4, 8, 16, 64, 256}; image k is gradient_rgba8(w, h, image_seed)
    (about 20 % transparent) and gets its own alpha-associated palette."""
    sizes = log_uniform_sizes(n - 4, seed=seed) + [(1, 1), (3, 5), (17, 13), (4096, 64)]
    rng = np.random.default_rng(5)
    return [(w, h, 1000 + k, int(rng.choice([2, 4, 8, 16, 64, 256])))
            for k, (w, h) in enumerate(sizes)]


# ---- decoder-format video frames --------------------------------------------
# Synthetic stand-ins for what a video decoder hands the block engine: the same
# gradient frames, widened to 16 bits with seeded low-order detail, or
# converted to planar 8-bit YCbCr (BT.601 limited range, rounded; 4:2:0 takes
# the rounded mean of each 2x2 chroma quad).

def rgb16_frame(img8: np.ndarray, seed: int) -> np.ndarray:
    """uint8 (H, W, C) -> uint16 (H, W, C): v * 257 plus seeded noise in
    [-96, 96], clipped; an alpha channel keeps its exact v * 257."""
    rng = np.random.default_rng(seed ^ 0x16161616)
    v = img8.astype(np.int32) * 257
    noise = rng.integers(-96, 97, v.shape, dtype=np.int32)
    if img8.shape[2] == 4:
        noise[:, :, 3] = 0
    return np.clip(v + noise, 0, 65535).astype(np.uint16)


def yuv444_frame(img8: np.ndarray) -> np.ndarray:
    """uint8 (H, W, >=3) RGB -> planar Y, Cb, Cr (3, H, W) uint8."""
    rgb = img8[:, :, :3].astype(np.float64)
    r, g, b = rgb[:, :, 0], rgb[:, :, 1], rgb[:, :, 2]
    y = 16 + (65.481 * r + 128.553 * g + 24.966 * b) / 255.0
    cb = 128 + (-37.797 * r - 74.203 * g + 112.0 * b) / 255.0
    cr = 128 + (112.0 * r - 93.786 * g - 18.214 * b) / 255.0
    return np.clip(np.rint(np.stack([y, cb, cr])), 0, 255).astype(np.uint8)


def yuv420_frame(img8: np.ndarray) -> np.ndarray:
    """uint8 (H, W, >=3) RGB, H and W even -> the packed 4:2:0 frame bytes:
    Y (H*W) then Cb and Cr (H/2 * W/2 each)."""
    p = yuv444_frame(img8).astype(np.int32)
    h, w = p.shape[1:]
    c = (p[1:, 0::2, 0::2] + p[1:, 0::2, 1::2] + p[1:, 1::2, 0::2] + p[1:, 1::2, 1::2] + 2) >> 2
    return np.concatenate([p[0].reshape(-1), c[0].reshape(-1), c[1].reshape(-1)]).astype(np.uint8)
