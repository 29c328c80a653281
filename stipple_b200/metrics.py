"""Tolerance metrics for the approximate engine.

* index mismatch: fraction of pixels whose palette index differs from a
  reference walk's;
* mean CIE dE76: mean Euclidean distance in CIE L*a*b* (sRGB, D65 white)
  between the two outputs' colours, over all pixels.
"""
from __future__ import annotations

import numpy as np

_M = np.array([[0.4124564, 0.3575761, 0.1804375],
               [0.2126729, 0.7151522, 0.0721750],
               [0.0193339, 0.1191920, 0.9503041]])
_WHITE = np.array([0.95047, 1.0, 1.08883])


def srgb_q16_to_lab(rgb: np.ndarray) -> np.ndarray:
    """(..., 3) Q16 sRGB (0..65535) -> (..., 3) L*a*b*."""
    c = np.clip(np.asarray(rgb, np.float64) / 65535.0, 0.0, 1.0)
    lin = np.where(c <= 0.04045, c / 12.92, ((c + 0.055) / 1.055) ** 2.4)
    xyz = lin @ _M.T / _WHITE
    eps, kappa = 216.0 / 24389.0, 24389.0 / 27.0
    f = np.where(xyz > eps, np.cbrt(xyz), (kappa * xyz + 16.0) / 116.0)
    L = 116.0 * f[..., 1] - 16.0
    a = 500.0 * (f[..., 0] - f[..., 1])
    b = 200.0 * (f[..., 1] - f[..., 2])
    return np.stack([L, a, b], axis=-1)


def index_mismatch(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.mean(np.asarray(a) != np.asarray(b)))


def mean_delta_e(palette: np.ndarray, idx_a: np.ndarray, idx_b: np.ndarray) -> float:
    lab = srgb_q16_to_lab(np.asarray(palette)[:, :3])
    da = lab[np.asarray(idx_a).reshape(-1)]
    db = lab[np.asarray(idx_b).reshape(-1)]
    return float(np.mean(np.linalg.norm(da - db, axis=1)))
