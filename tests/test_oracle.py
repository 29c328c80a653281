"""Pins the oracle (oracle/oracle.c, the C restatement of the reference's CPU
path) against the reference's own CPU build and the golden vectors."""
from __future__ import annotations

import numpy as np
import pytest

import golden
from stipple_b200 import synth


def _colours(pal, idx, assoc):
    ch = 4 if assoc else 3
    return pal[idx.reshape(-1)][:, :ch]


@pytest.mark.parametrize("name,rgbaf,recs", list(golden.cases()), ids=lambda v: v if isinstance(v, str) else "")
def test_oracle_matches_golden(oracle, name, rgbaf, recs):
    h, w = rgbaf.shape[:2]
    for r in recs:
        colors, assoc, gray = int(r["colors"]), bool(r["assoc"]), bool(r["gray"])
        idx, out, pal = oracle.walk_seq(rgbaf, colors, assoc, gray)
        assert np.array_equal(pal, r["pal"]), (name, colors)
        assert np.array_equal(_colours(pal, idx, assoc), _colours(r["pal"], r["seq"], assoc)), (name, colors)
        idx, _, _ = oracle.walk_seq(rgbaf, colors, assoc, gray, use_cache=False)
        assert np.array_equal(_colours(pal, idx, assoc),
                              _colours(r["pal"], r["seq_nocache"], assoc)), (name, colors)
        for key in [k for k in r if k.startswith("blk")]:
            b = int(key[3:])
            bidx, bout, _ = oracle.walk_blocks(rgbaf, colors, assoc, gray, b)
            want = r[key]
            keep = np.ones(h * w, bool)
            keep[r[f"kept{b}"]] = False
            # pixels that kept their source value (the block list's gap)
            assert np.array_equal(bout.reshape(-1, 4)[~keep], rgbaf.reshape(-1, 4)[~keep])
            got = bidx.reshape(-1)[keep]
            assert np.array_equal(_colours(pal, got, assoc), _colours(r["pal"], want.reshape(-1)[keep], assoc)), (name, colors, b)


def test_curves_match_golden(oracle):
    z = golden.curves()
    for k in z.files:
        if k.endswith("_curve"):
            w, h = map(int, k[: -len("_curve")].split("x"))
            c, o = oracle.block_order(w, h)
            assert np.array_equal(c, z[k]) and np.array_equal(o, z[f"{w}x{h}_owner"])


def test_seq_order_is_recursion(oracle):
    """RiemersmaWalkCpu's order = the recursion's leaves + the resting cursor
    = the closed form over [0, 4^L) (the reference's recursion, dumped by
    BuildCurveSequence, holds the leaves)."""
    z = golden.curves()
    for lv in range(1, 7):
        seq = z[f"seq_L{lv}"]
        side = 1 << lv
        order = oracle.seq_order(side, side)
        xy = np.stack([order % side, order // side], axis=1)
        leaves = seq[:-1]
        assert np.array_equal(xy[:-1], leaves)
        assert tuple(xy[-1]) == (side - 1, 0)
        assert sorted(order.tolist()) == list(range(side * side))


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_oracle_matches_reference_build(oracle, reflib, seed):
    for (w, h) in [(64, 48), (17, 13), (100, 37), (128, 128)]:
        for colors in (2, 16, 256):
            for alpha in (False, True):
                img = synth.gradient_rgba8(w, h, seed) if alpha else synth.gradient_rgb8(w, h, seed)
                q = synth.to_q16(img)
                gray = synth.is_grayscale(img)
                t0 = oracle.build_tree(q, colors, alpha, gray)
                t1 = reflib.build_tree(q, colors, alpha, gray)
                assert np.array_equal(t0.palette, t1.palette)
                assert np.array_equal(t0.child, t1.child)
                assert np.array_equal(t0.color_number, t1.color_number)
                for diff in (1.0, 0.6):
                    _, out, _ = oracle.walk_seq(q, colors, alpha, gray, diffusion=diff)
                    rout, _ = reflib.walk_seq(q, colors, alpha, gray, diffusion=diff)
                    assert np.array_equal(out.view(np.uint32), rout.view(np.uint32))
                _, bout, _ = oracle.walk_blocks(q, colors, alpha, gray, 16 + seed * 9)
                rb, _ = reflib.walk_blocks(q, colors, alpha, gray, 16 + seed * 9)
                assert np.array_equal(bout.view(np.uint32), rb.view(np.uint32))


def test_float_inputs_not_multiples_of_257(oracle, reflib):
    """RgbaF inputs with arbitrary Q16 floats (e.g. from 16-bit sources)."""
    rng = np.random.default_rng(7)
    q = (rng.random((40, 56, 4)) * 65535.0).astype(np.float32)
    q[..., 3] = np.where(rng.random((40, 56)) < 0.3, q[..., 3], 65535.0)
    for alpha in (False, True):
        for colors in (8, 64):
            _, out, _ = oracle.walk_seq(q, colors, alpha, False)
            rout, _ = reflib.walk_seq(q, colors, alpha, False)
            assert np.array_equal(out.view(np.uint32), rout.view(np.uint32))


def test_blocks_refusals_match(oracle, reflib):
    q = synth.to_q16(synth.gradient_rgb8(32, 32, 1))
    with pytest.raises(ValueError):
        oracle.walk_blocks(q, 16, False, False, 15)
    with pytest.raises(ValueError):
        reflib.walk_blocks(q, 16, False, False, 15)
