"""The product's host palette builder against the oracle (and so the reference)."""
from __future__ import annotations

import numpy as np
import pytest

import golden
import stipple_b200 as sb
from stipple_b200 import synth


def _same_tree(t_prod: sb.Octree, t_orc) -> bool:
    child, parent, cn, nu = t_prod.nodes()
    return (np.array_equal(t_prod.colormap(), t_orc.palette) and np.array_equal(child, t_orc.child)
            and np.array_equal(parent, t_orc.parent) and np.array_equal(cn, t_orc.color_number)
            and np.array_equal(nu, t_orc.number_unique))


@pytest.mark.parametrize("seed", range(4))
def test_octree_matches_oracle(lib, oracle, seed):
    for (w, h) in [(1, 1), (3, 5), (17, 13), (64, 48), (100, 37), (256, 192)]:
        for colors in (2, 4, 8, 16, 64, 256):
            for alpha in (False, True):
                img = synth.gradient_rgba8(w, h, seed) if alpha else synth.gradient_rgb8(w, h, seed)
                if seed == 3:  # greyscale input: depth forced to 8
                    img[..., 1] = img[..., 0]
                    img[..., 2] = img[..., 0]
                gray = synth.is_grayscale(img)
                t = sb.Octree(img, colors, alpha, gray)
                assert t.grayscale == gray
                assert _same_tree(t, oracle.build_tree(synth.to_q16(img), colors, alpha, gray)), \
                    (w, h, colors, alpha)


def test_octree_on_golden_inputs(lib, oracle):
    for name, rgbaf, recs in golden.cases():
        for r in recs:
            colors, assoc, gray = int(r["colors"]), bool(r["assoc"]), bool(r["gray"])
            t = sb.Octree(rgbaf, colors, assoc, gray)
            assert np.array_equal(t.colormap(), r["pal"]), (name, colors)
            assert _same_tree(t, oracle.build_tree(rgbaf, colors, assoc, gray)), (name, colors)


def test_octree_large_reduction(lib, oracle):
    """A busy image that overflows MaxQNodes in the first classification loop."""
    rng = np.random.default_rng(3)
    img = rng.integers(0, 256, size=(600, 800, 3), dtype=np.uint8)
    t = sb.Octree(img, 256, False, False)
    assert _same_tree(t, oracle.build_tree(synth.to_q16(img), 256, False, False))
