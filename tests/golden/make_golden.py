"""Generate the golden vectors in tests/golden/ from the reference itself.

Runs the reference's own CPU code (oracle/_ref/librdref.so: src/rd_octree.cpp
and src/rd_riemersma_cpu.cpp compiled unmodified by oracle/Makefile) on

* the reference's PNG test fixtures (tests/*.png of the reference tree,
  decoded with PIL the way an 8-bit decode into Q16 is scaled: v * 257, and
  16-bit samples as-is), and
* seeded synthetic images of the benchmark configurations, and
* seeded decoder-format video frames (rgb48 / rgba64 / planar 4:4:4 / RgbaF)
  through the block walk's fused gather and output (frames.npz),

and stores inputs and outputs as compressed .npz files.  The GPU tests and the
oracle tests compare against these files; the reference tree is not needed at
test time.  Re-run with:

    make -f oracle/Makefile && python tests/golden/make_golden.py [REF_DIR] [--frames-only]
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from pyoracle import RefLib  # noqa: E402
from stipple_b200 import synth  # noqa: E402

FIXTURES = ["t_1x1", "t_3x5", "t_17x13", "t_wide", "in_grad", "in_plasma", "in_shapes",
            "in_alpha", "in_gray_alpha", "noisy"]
COLORS = [2, 4, 16, 32, 64, 256]


def decode(path: str):
    """PNG -> (RgbaF Q16 float32 HxWx4, has_alpha)."""
    from PIL import Image
    im = Image.open(path)
    mode = im.mode
    if mode in ("I;16", "I;16B", "I;16L", "I"):
        a = np.asarray(im, dtype=np.uint32).astype(np.float32)
        out = np.empty(a.shape + (4,), np.float32)
        out[..., 0] = out[..., 1] = out[..., 2] = a
        out[..., 3] = 65535.0
        return out, False
    if mode == "P":
        im = im.convert("RGBA" if "transparency" in im.info else "RGB")
        mode = im.mode
    if mode == "L":
        g = np.asarray(im, np.float32) * np.float32(257.0)
        out = np.stack([g, g, g, np.full_like(g, 65535.0)], axis=-1)
        return out, False
    if mode == "LA":
        a = np.asarray(im, np.float32) * np.float32(257.0)
        out = np.stack([a[..., 0], a[..., 0], a[..., 0], a[..., 1]], axis=-1)
        return out, True
    if mode == "RGB":
        return synth.to_q16(np.asarray(im, np.uint8)), False
    if mode == "RGBA":
        return synth.to_q16(np.asarray(im, np.uint8)), True
    raise ValueError(f"unsupported PNG mode {mode}")


def reverse_index(out: np.ndarray, pal: np.ndarray, assoc: bool, src: np.ndarray):
    """Palette index of each output pixel (exact colour match), and the pixel
    indices that kept their source value instead (the block list's gap; their
    index entry is 0)."""
    h, w = out.shape[:2]
    flat = out.reshape(-1, 4)
    palf = pal.astype(np.float32)
    idx = np.zeros(h * w, np.uint8)
    found = np.zeros(h * w, bool)
    ch = 4 if assoc else 3
    for i in range(pal.shape[0]):
        m = np.all(flat[:, :ch] == palf[i, :ch], axis=1) & ~found
        idx[m] = i
        found |= m
    miss = ~found
    if np.any(miss):
        assert np.array_equal(flat[miss], src.reshape(-1, 4)[miss]), "unmatched output pixel"
    return idx.reshape(h, w), np.nonzero(miss)[0].astype(np.int64)


def run_case(ref: RefLib, rgbaf, colors, assoc, gray, blocks=(16, 512)):
    out, pal = ref.walk_seq(rgbaf, colors, assoc, gray)
    rec = {"colors": colors, "assoc": int(assoc), "gray": int(gray), "pal": pal,
           "seq": reverse_index(out, pal, assoc, rgbaf)[0]}
    nc, _ = ref.walk_seq(rgbaf, colors, assoc, gray, use_cache=False)
    rec["seq_nocache"] = reverse_index(nc, pal, assoc, rgbaf)[0]
    h, w = rgbaf.shape[:2]
    if w * h > 1:
        for b in blocks:
            bo, _ = ref.walk_blocks(rgbaf, colors, assoc, gray, b)
            rec[f"blk{b}"], rec[f"kept{b}"] = reverse_index(bo, pal, assoc, rgbaf)
    return rec


def save(name: str, rgbaf: np.ndarray, recs: list[dict]) -> None:
    # 8-bit sources are stored as bytes (v * 257 restores the Q16 floats exactly).
    if np.all(np.mod(rgbaf, 257.0) == 0.0):
        arrays = {"rgba8": (rgbaf / np.float32(257.0)).astype(np.uint8)}
    else:
        arrays = {"rgbaf": rgbaf}
    for i, r in enumerate(recs):
        for k, v in r.items():
            arrays[f"c{i}_{k}"] = np.asarray(v)
    arrays["ncases"] = np.asarray(len(recs))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)


def frames_golden(ref: RefLib) -> None:
    """RiemersmaBlocksCpu with gather_raw / raw_out on small seeded frames.
    Each case k stores: in (F, bytes) uint8, gather layout / channels (0 =
    RgbaF input), tree_src RgbaF, w, h, colors, assoc, block, and out_yuv /
    out_rgba64 (F, bytes) uint8."""
    arrays = {}
    cases = [  # (w, h, input, channels, alpha, assoc, colors, block)
        (32, 24, "u16", 4, True, False, 16, 32),
        (32, 24, "u16", 4, True, True, 64, 16),
        (37, 29, "u16", 3, False, False, 32, 16),
        (32, 24, "yuv", 0, False, False, 256, 64),
        (37, 29, "yuv", 0, False, False, 8, 512),
        (32, 24, "f32", 4, True, False, 16, 32),
        (1, 1, "u16", 4, True, False, 4, 16),
    ]
    for k, (w, h, kind, ch, alpha, assoc, colors, block) in enumerate(cases):
        fr8 = [synth.video_frame(w, h, 600 + k, f) for f in range(2)]
        if alpha:
            a = synth.alpha_mask(w, h, 600 + k)
            fr8 = [np.concatenate([f, a[:, :, None]], axis=2) for f in fr8]
        if kind == "u16":
            fr = [synth.rgb16_frame(f[:, :, :ch], 700 + k + i) for i, f in enumerate(fr8)]
            raw = np.stack([f.reshape(-1).view(np.uint8) for f in fr])
            layout = 4
            tree_src = np.zeros((h, w, 4), np.float32)
            tree_src[:, :, :ch] = fr[0].astype(np.float32)
            if ch == 3:
                tree_src[:, :, 3] = 65535.0
        elif kind == "yuv":
            fr = [synth.yuv444_frame(f) for f in fr8]
            raw = np.stack([f.reshape(-1) for f in fr])
            layout, ch = 3, 0
            tree_src = None  # widened by the reference-side gather of frame 0 below
        else:
            fr = [synth.to_q16(f) for f in fr8]
            raw = np.stack([f.reshape(-1).view(np.uint8) for f in fr])
            layout, ch = 0, 0
            tree_src = fr[0]
        if tree_src is None:
            # The palette's source image only: frame 0 widened by the oracle,
            # since the reference exposes no widening entry point.  Every
            # stored output is the reference's own.
            from pyoracle import Oracle
            tree_src = Oracle().widen_frame(444, raw[0], w, h)
        src = np.stack(fr).astype(np.float32) if layout == 0 else raw
        outs = {}
        for yuv in (True, False):
            rc, msg, out = ref.walk_blocks_raw(tree_src, src, layout, ch, w, h, yuv, colors,
                                               assoc, block)
            assert rc == 0, msg
            outs["out_yuv" if yuv else "out_rgba64"] = out
        rec = dict(inp=raw, layout=layout, channels=ch, tree_src=tree_src, w=w, h=h,
                   colors=colors, assoc=int(assoc), block=block, **outs)
        for key, v in rec.items():
            arrays[f"c{k}_{key}"] = np.asarray(v)
    arrays["ncases"] = np.asarray(len(cases))
    np.savez_compressed(os.path.join(HERE, "frames.npz"), **arrays)
    print("frames", len(cases))


def main(ref_dir: str) -> None:
    ref = RefLib()
    frames_golden(ref)
    if "--frames-only" in sys.argv:
        return
    # The reference's own fixtures.
    for fx in FIXTURES:
        rgbaf, alpha = decode(os.path.join(ref_dir, "tests", fx + ".png"))
        gray = bool(np.all(rgbaf[..., 0] == rgbaf[..., 1]) and np.all(rgbaf[..., 1] == rgbaf[..., 2]))
        cols = [16] if fx == "noisy" else COLORS
        recs = [run_case(ref, rgbaf, c, alpha, gray) for c in cols]
        save("fx_" + fx, rgbaf, recs)
        print(fx, rgbaf.shape, "alpha" if alpha else "", "gray" if gray else "", len(recs))
    # Configuration 1: 256x256 RGB8 gradient + noise (sigma 8), 16 colours.
    img = synth.gradient_rgb8(256, 256, seed=1)
    save("cfg1_256x256_16c", synth.to_q16(img), [run_case(ref, synth.to_q16(img), 16, False, False)])
    # Geometries with the block-list gap inside the image, and strips.
    for (w, h, c, seed, alpha) in [(256, 192, 64, 2, False), (64, 64, 256, 3, True),
                                   (640, 64, 16, 4, False), (37, 100, 8, 5, True)]:
        img = synth.gradient_rgba8(w, h, seed) if alpha else synth.gradient_rgb8(w, h, seed)
        q = synth.to_q16(img)
        save(f"syn_{w}x{h}_{c}c{'_a' if alpha else ''}", q,
             [run_case(ref, q, c, alpha, synth.is_grayscale(img), blocks=(16, 64, 4096))])
    # Curve lists (BuildCurveIndex) for a few geometries.
    curves = {}
    for w, h in [(1, 2), (3, 5), (17, 13), (64, 64), (256, 192), (100, 37), (8, 128)]:
        c, o = ref.block_order(w, h)
        curves[f"{w}x{h}_curve"] = c
        curves[f"{w}x{h}_owner"] = o
    for lv in range(1, 7):
        curves[f"seq_L{lv}"] = ref.curve_sequence(lv)
    np.savez_compressed(os.path.join(HERE, "curves.npz"), **curves)
    print("curves", len(curves))


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    main(args[0] if args else os.path.normpath(os.path.join(ROOT, "..", "reference")))
