"""Palette image files in the PNG form (rdb_palette_write_png /
rdb_palette_read_png).  Host code only.

The writer's strip is decoded with PIL and checked against ImageMagick's
ScaleQuantumToChar of every entry (the PNG8 coder's narrowing,
src/rd_im.cpp:1047-1118).  The reader's tree is checked against the
reference's own ColorTree::Build (oracle/_ref) of the swatch that
ImAdoptPaletteFromColormap (src/rd_im.cpp:731-888) builds from the colours
PIL decodes: an indexed PNG's PLTE in order, else the distinct RGB values in
scan order -- across PNG colour types, bit depths, a tRNS chunk and Adam7
interlacing."""
from __future__ import annotations

import math

import numpy as np
import pytest

from stipple_b200 import synth

PIL = pytest.importorskip("PIL.Image")


@pytest.fixture(scope="module")
def sb(lib):
    import stipple_b200
    return stipple_b200


def _im_char(q: float) -> int:
    q = float(np.float32(q))
    if not q > 0.0:
        return 0
    if q / 257.0 >= 255.0:
        return 255
    return int(q / 257.0 + 0.5)


def _swatch(entries):
    """ImAdoptPaletteFromColormap's swatch: each colour an 8 x 8 square,
    ceil(sqrt(n)) squares per row, zeros elsewhere."""
    n = len(entries)
    block = max(1, int(math.ceil(math.sqrt(n))))
    rows = (n + block - 1) // block
    img = np.zeros((rows * 8, block * 8, 4), np.float32)
    for i, e in enumerate(entries):
        gx, gy = (i % block) * 8, (i // block) * 8
        img[gy:gy + 8, gx:gx + 8] = np.float32(e)
    gray = all(e[0] == e[1] == e[2] for e in entries)
    return img, gray


def _want_tree(reflib, entries):
    uniq = []
    for e in entries:
        if not any(u[:3] == e[:3] for u in uniq):
            uniq.append(e)
    img, gray = _swatch(uniq)
    return reflib.build_tree(img, len(uniq), False, gray), len(uniq)


@pytest.mark.parametrize("colors", [2, 16, 64, 256])
def test_writer_strip_is_im_narrowing(sb, tmp_path, colors):
    pal = sb.Octree(synth.gradient_rgb8(96, 64, colors), colors, False).colormap()
    path = str(tmp_path / "pal.png")
    sb.write_palette_png(pal, path)
    im = PIL.open(path)
    assert im.mode == "P" and im.size == (len(pal), 1)
    got = np.asarray(im.convert("RGB"))[0]
    want = np.array([[_im_char(v) for v in e[:3]] for e in pal], np.uint8)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("colors", [4, 16, 256])
def test_round_trip_matches_reference_tree(sb, reflib, tmp_path, colors):
    pal = sb.Octree(synth.gradient_rgb8(96, 64, colors + 1), colors, False).colormap()
    path = str(tmp_path / "pal.png")
    sb.write_palette_png(pal, path)
    tree = sb.read_palette_png(path)
    plte = np.asarray(PIL.open(path).convert("RGB"))[0].astype(np.float64) * 257.0
    entries = [(r, g, b, 65535.0) for r, g, b in plte]
    want, n = _want_tree(reflib, entries)
    assert tree.count == want.count
    assert np.array_equal(tree.colormap(), want.palette)
    # Importing the exported file again gives the same tree: the form is stable.
    path2 = str(tmp_path / "pal2.png")
    sb.write_palette_png(tree.colormap(), path2)
    assert np.array_equal(sb.read_palette_png(path2).colormap(), tree.colormap())


def _cases(rng):
    px8 = rng.integers(0, 256, (5, 7, 3), dtype=np.uint8)
    px8[1:3, 2:5] = px8[0, 0]  # repeated colours
    yield "rgb8", PIL.fromarray(px8, "RGB"), {}
    yield "rgb8_interlaced", PIL.fromarray(px8, "RGB"), {"interlace": 1}
    yield "rgba8", PIL.fromarray(np.dstack([px8, np.full((5, 7), 200, np.uint8)]), "RGBA"), {}
    yield "gray8", PIL.fromarray(px8[..., 0], "L"), {}
    yield "gray1", PIL.fromarray(px8[..., 0] > 128), {}
    g16 = rng.integers(0, 65536, (4, 6), dtype=np.uint16)
    yield "gray16", PIL.fromarray(g16.astype(np.int32), "I").convert("I;16"), {}
    p = PIL.fromarray(rng.integers(0, 5, (3, 9), dtype=np.uint8), "P")
    lut = rng.integers(0, 256, 15, dtype=np.uint8).tolist()
    p.putpalette(lut)
    yield "indexed", p, {}
    yield "indexed_trns", p, {"transparency": bytes([255, 128, 0, 255, 17])}


def _pil_entries(im):
    """The colours the reference's reader takes from a decoded image."""
    if im.mode == "P":
        lut = im.getpalette()
        n = len(lut) // 3
        trns = im.info.get("transparency")
        out = []
        for i in range(n):
            a = 65535.0
            if isinstance(trns, (bytes, bytearray)) and i < len(trns):
                a = trns[i] * 257.0
            out.append((lut[3 * i] * 257.0, lut[3 * i + 1] * 257.0, lut[3 * i + 2] * 257.0, a))
        return out
    if im.mode in ("I;16", "I"):
        v = np.asarray(im).astype(np.float64).reshape(-1)
        rgb = np.stack([v, v, v], 1)
    else:
        rgb = np.asarray(im.convert("RGB")).reshape(-1, 3).astype(np.float64) * 257.0
    out = []
    for r, g, b in rgb:
        if not any(e[:3] == (r, g, b) for e in out):
            out.append((r, g, b, 65535.0))
    return out


def test_reader_across_png_forms(sb, reflib, tmp_path):
    rng = np.random.default_rng(5)
    for name, im, kw in _cases(rng):
        path = str(tmp_path / f"{name}.png")
        im.save(path, **kw)
        back = PIL.open(path)
        back.load()
        entries = _pil_entries(back)
        want, n = _want_tree(reflib, entries)
        tree = sb.read_palette_png(path)
        assert tree.count == want.count, name
        assert np.array_equal(tree.colormap(), want.palette), name


def test_reader_refusals(sb, tmp_path):
    p = tmp_path / "x.png"
    PIL.fromarray(np.array([[[1, 2, 3], [4, 5, 6], [1, 2, 3]]], np.uint8), "RGB").save(p)
    assert sb.read_palette_png(str(p), expect_colors=2).count == 2
    with pytest.raises(sb.RdbError, match="holds 2 colours, not 3"):
        sb.read_palette_png(str(p), expect_colors=3)
    with pytest.raises(sb.RdbError, match="more than 1"):
        sb.read_palette_png(str(p), expect_colors=1)
    bad = tmp_path / "bad.png"
    bad.write_bytes(b"not a png at all")
    with pytest.raises(sb.RdbError, match="not a PNG"):
        sb.read_palette_png(str(bad))
    raw = bytearray(p.read_bytes())
    raw[40] ^= 0xFF  # inside a chunk: its CRC no longer matches
    bad.write_bytes(bytes(raw))
    with pytest.raises(sb.RdbError):
        sb.read_palette_png(str(bad))
    with pytest.raises(sb.RdbError, match="256"):
        sb.write_palette_png(np.zeros((300, 4)), str(tmp_path / "big.png"))


def test_dispatch_by_extension(sb, tmp_path):
    pal = sb.Octree(synth.gradient_rgb8(64, 64, 9), 8, False).colormap()
    sb.write_palette(pal, str(tmp_path / "a.txt"))
    sb.write_palette(pal, str(tmp_path / "a.png"))
    t_txt, _ = sb.read_palette(str(tmp_path / "a.txt"))
    t_png, assoc = sb.read_palette(str(tmp_path / "a.png"))
    assert not assoc and t_txt.count == t_png.count == len(pal)
