"""The device plan (rdb_plan_build) read back on the host: a numpy restatement
of the kernels' lookup -- descent through the live child table, then the
minimum over the stopping node's run of post-order slots, ties to the highest
slot -- must equal the oracle's descent + ClosestColor for every target."""
from __future__ import annotations

import ctypes as C
import struct

import numpy as np
import pytest

import stipple_b200 as sb
from stipple_b200 import synth

QS = 1.0 / 65535.0
START = 4.0 * ((65535.0 + 1.0) * (65535.0 + 1.0)) + 1.0


def parse(blob: bytes):
    hdr = struct.unpack("16i", blob[:64])
    count, assoc, nodes, fan, slots, smem, total, off_pal, off_child, off_range, off_seq, off_out, stride = hdr[:13]
    b = np.frombuffer(blob, np.uint8)
    pal = b[off_pal: off_pal + count * stride].view(np.float64).reshape(count, stride // 8)
    child = b[off_child: off_child + nodes * fan * 2].view(np.int16).reshape(nodes, fan)
    rng = b[off_range: off_range + nodes * 4].view(np.uint16).reshape(nodes, 2)
    seq = b[off_seq: off_seq + slots]
    return dict(count=count, assoc=bool(assoc), nodes=nodes, fan=fan, slots=slots, pal=pal,
                child=child, range=rng, seq=seq, smem=smem, total=total)


def byte(q):
    q = np.asarray(q, np.float32)
    t = np.trunc(np.float32(2.0) * q).astype(np.int64)
    return np.minimum(255, (t + 257) // 514)


def emulate(p, f):
    """f: (4,) float32 clamped target.  Returns the colour number."""
    bts = byte(f)
    node = 0
    for i in range(7, 0, -1):
        cid = ((bts[0] >> i) & 1) | (((bts[1] >> i) & 1) << 1) | (((bts[2] >> i) & 1) << 2)
        if p["assoc"]:
            cid |= ((bts[3] >> i) & 1) << 3
        c = int(p["child"][node, cid])
        if c < 0:
            break
        node = c
    start, n = (int(v) for v in p["range"][node])
    if n == 0:
        return 0
    t = f.astype(np.float64)
    if p["assoc"]:
        beta = QS * t[3]
        tr, tg, tb = beta * t[0], beta * t[1], beta * t[2]
    else:
        tr, tg, tb = t[0], t[1], t[2]
    cols = p["seq"][start: start + n].astype(np.int64)
    e = p["pal"][cols]
    x, y, z = e[:, 0] - tr, e[:, 1] - tg, e[:, 2] - tb
    d = x * x
    d = d + y * y
    d = d + z * z
    if p["assoc"]:
        w = e[:, 3] - t[3]
        d = d + w * w
    ok = d <= START
    if not np.any(ok):
        return 0
    m = d[ok].min()
    last = np.nonzero(ok & (d == m))[0][-1]
    return int(cols[last])


@pytest.mark.parametrize("alpha", [False, True])
@pytest.mark.parametrize("colors", [2, 16, 256])
def test_plan_lookup_equals_closest_color(lib, oracle, alpha, colors):
    from pyoracle import OrcTree
    rng = np.random.default_rng(colors * 3 + int(alpha))
    img = synth.gradient_rgba8(96, 80, colors) if alpha else synth.gradient_rgb8(96, 80, colors)
    q = synth.to_q16(img)
    raw = oracle.build_tree_raw(q, colors, alpha, False)
    try:
        tree = oracle._export(raw)
        blob = sb.plan_blob(tree.palette, tree.child, tree.color_number, tree.number_unique,
                            alpha, parent=tree.parent)
        p = parse(blob)
        assert p["count"] == tree.count and p["slots"] <= 256
        # Trees from the octree number colours in post-order: seq is the identity.
        assert np.array_equal(p["seq"], np.arange(p["slots"]))
        targets = [rng.random(4).astype(np.float32) * np.float32(65535.0) for _ in range(1500)]
        targets += [(tree.palette[rng.integers(tree.count)] + rng.normal(0, 900, 4)).clip(0, 65535).astype(np.float32)
                    for _ in range(1500)]
        for f in targets:
            if not alpha:
                f[3] = 65535.0
            want = oracle.lib.orc_tree_lookup(C.byref(raw), float(f[0]), float(f[1]), float(f[2]), float(f[3]))
            assert emulate(p, f) == want, f
    finally:
        oracle.lib.orc_tree_free(C.byref(raw))


def test_plan_refuses_large_palettes(lib):
    pal = np.zeros((257, 4))
    child = np.full((1, 16), -1, np.int32)
    with pytest.raises(sb.RdbError):
        sb.plan_blob(pal, child, np.zeros(1, np.uint32), np.ones(1, np.uint64), False)


def test_plan_general_tree_order(lib):
    """A hand-made tree whose colour numbers are not in post-order: the plan
    keeps the traversal order in `seq`, so ties still go to the last visited."""
    child = np.full((3, 16), -1, np.int32)
    child[0, 0] = 1
    child[0, 7] = 2
    nu = np.array([0, 5, 7], np.uint64)
    cn = np.array([0, 1, 0], np.uint32)  # post-order visits node 1 (colour 1) then node 2 (colour 0)
    pal = np.array([[100.0, 100.0, 100.0, 65535.0], [100.0, 100.0, 100.0, 65535.0]])
    p = parse(sb.plan_blob(pal, child, cn, nu, False, parent=np.array([0, 0, 0], np.int32)))
    assert list(p["seq"]) == [1, 0]
    f = np.array([100.0, 100.0, 100.0, 65535.0], np.float32)
    # Equal distances: the last in post-order (colour 0) wins.
    assert emulate(p, f) == 0
