"""Palette text files (rdb_palette_write_text / rdb_palette_read_text): the
writer's bytes against the reference's format (src/rd_im.cpp:1018-1028), the
reader's tree against the reference's own ColorTree::Build of the same strip
(src/rd_im.cpp:1325-1349, built from the reference's sources), and the
reader's refusals.  Host code only."""
from __future__ import annotations

import numpy as np
import pytest

from stipple_b200 import synth


@pytest.fixture(scope="module")
def sb(lib):
    import stipple_b200
    return stipple_b200


def _reference_text(colors):
    lines = [f"# rdither palette, {len(colors)} colours, Q16 (0..65535) and 8-bit hex",
             "# count\tr\tg\tb\ta\thex"]
    for i, (r, g, b, a) in enumerate(colors):
        hx = "".join(f"{int(v / 257.0 + 0.5):02X}" for v in (r, g, b))
        lines.append(f"{i}\t{r:.6f}\t{g:.6f}\t{b:.6f}\t{a:.6f}\t{hx}")
    return "\n".join(lines) + "\n"


def _strip(colors):
    """The reader's strip: r, g, b through float, sorted by (r, g, b, a)."""
    rows = [(float(np.float32(r)), float(np.float32(g)), float(np.float32(b)), float(a))
            for r, g, b, a in colors]
    rows.sort()
    return np.array(rows, np.float32).reshape(1, -1, 4)


@pytest.mark.parametrize("colors,alpha", [(16, False), (64, False), (256, False), (8, True)])
def test_write_then_read_matches_reference_tree(sb, reflib, tmp_path, colors, alpha):
    img = synth.gradient_rgba8(96, 64, colors) if alpha else synth.gradient_rgb8(96, 64, colors)
    pal = sb.Octree(img, colors, alpha).colormap()
    path = str(tmp_path / "pal.txt")
    sb.write_palette_text(pal, path)
    text = open(path).read()
    assert text == _reference_text(pal)
    tree, assoc = sb.read_palette_text(path, expect_colors=len(pal))
    assert assoc == bool(np.any(np.array([float(f"{a:.6f}") for a in pal[:, 3]]) != 65535.0))
    # What the reader hands the tree build is the file's numbers as printed.
    printed = [[float(x) for x in line.split("\t")[1:5]] for line in text.splitlines()[2:]]
    strip = _strip(printed)
    gray = bool(np.all(strip[..., 0] == strip[..., 1]) and np.all(strip[..., 1] == strip[..., 2]))
    want = reflib.build_tree(strip, len(pal), False, gray)
    assert tree.count == len(pal)
    assert np.array_equal(tree.colormap(), want.palette)


def test_reader_rules(sb, tmp_path):
    p = tmp_path / "a.text"
    # Comments and blank lines skipped; alpha read only when a sixth column
    # follows; rows in any order.
    p.write_text("# x\n\n1 30000 100 200\n0 10 20 30 1234.5 0A0B0C\n2 65535 0 0 FFFFFF\n")
    tree, assoc = sb.read_palette_text(str(p))
    assert tree.count == 3 and assoc
    p.write_text("0 10 20 30\n2 1 2 3\n")
    with pytest.raises(sb.RdbError, match="no row declares index 1"):
        sb.read_palette_text(str(p))
    p.write_text("0 10 20 30 70000 000000\n")
    with pytest.raises(sb.RdbError, match="alpha"):
        sb.read_palette_text(str(p))
    p.write_text("0 10 20\n")
    with pytest.raises(sb.RdbError, match="not a palette row"):
        sb.read_palette_text(str(p))
    p.write_text("0 10 20 30\n1 40 50 60\n")
    with pytest.raises(sb.RdbError, match="holds 2 colours"):
        sb.read_palette_text(str(p), expect_colors=3)
    p.write_text("0 10 20 30\n1 10 20 30\n")
    with pytest.raises(sb.RdbError, match="duplicate"):
        sb.read_palette_text(str(p))
    p.write_text("# nothing\n")
    with pytest.raises(sb.RdbError, match="no palette rows"):
        sb.read_palette_text(str(p))
    with pytest.raises(sb.RdbError, match="rdb_palette_read_png"):
        sb.read_palette_text(str(tmp_path / "pal.png"))
    with pytest.raises(sb.RdbError, match="rdb_palette_write_png"):
        sb.write_palette_text(np.zeros((2, 4)), str(tmp_path / "pal.png"))
