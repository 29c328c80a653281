"""Golden vectors generated from the reference's own CPU build (make_golden.py)."""
from __future__ import annotations

import glob
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def cases():
    """Yields (name, rgbaf float32 HxWx4, list of per-case dicts)."""
    for path in sorted(glob.glob(os.path.join(HERE, "*.npz"))):
        name = os.path.basename(path)[:-4]
        if name in ("curves", "frames"):
            continue
        z = np.load(path)
        if "rgba8" in z:
            rgbaf = z["rgba8"].astype(np.float32) * np.float32(257.0)
        else:
            rgbaf = z["rgbaf"]
        recs = []
        for i in range(int(z["ncases"])):
            pre = f"c{i}_"
            recs.append({k[len(pre):]: z[k] for k in z.files if k.startswith(pre)})
        yield name, rgbaf, recs


def curves():
    return np.load(os.path.join(HERE, "curves.npz"))


def frames():
    """Yields the fused-format block-walk cases of frames.npz as dicts."""
    z = np.load(os.path.join(HERE, "frames.npz"))
    for i in range(int(z["ncases"])):
        pre = f"c{i}_"
        yield {k[len(pre):]: z[k] for k in z.files if k.startswith(pre)}
