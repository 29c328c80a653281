"""The request loop (rdb_server_*): a mixed stream of sizes, palettes, layouts
and engines submitted concurrently gives every request the same bytes as the
same request alone (its palette built by the host builder); admission keeps
within a tight budget; requests larger than the budget are refused at
submission.  Both palette paths: built by host threads (the default) and by
the device workers (device_palettes)."""
from __future__ import annotations

import threading

import numpy as np
import pytest

import stipple_b200 as sb
from stipple_b200 import synth

pytestmark = pytest.mark.gpu


def _mix(n, seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for k in range(n):
        w = int(np.exp(rng.uniform(np.log(8), np.log(700))))
        h = int(np.exp(rng.uniform(np.log(8), np.log(500))))
        alpha = bool(rng.random() < 0.4)
        img = synth.gradient_rgba8(w, h, 500 + k) if alpha else synth.gradient_rgb8(w, h, 500 + k)
        colors = int(rng.choice([2, 4, 8, 16, 64, 256]))
        engine = str(rng.choice(["seq", "seq", "seq", "blocks", "blocks", "jacobi"]))
        reqs.append((img, colors, engine, alpha))
    return reqs


def _alone(ctx, img, colors, engine, alpha):
    t = sb.Octree(img, colors, alpha)
    pid = ctx.palette_from_octree(t)
    try:
        return ctx.dither_host(engine, img, pid, rgba=True)
    finally:
        ctx.release_palette(pid)


@pytest.mark.parametrize("device_palettes", [False, True])
def test_mixed_stream_equals_each_request_alone(ctx, device_palettes):
    reqs = _mix(48, 3)
    srv = sb.Server(workers=3, max_batch=16, device_palettes=device_palettes)
    try:
        tickets = [None] * len(reqs)

        def submit(lo, hi):
            for k in range(lo, hi):
                img, colors, engine, alpha = reqs[k]
                tickets[k] = srv.submit(img, colors, engine, alpha=alpha, rgba=True)

        th = [threading.Thread(target=submit, args=(i * 16, (i + 1) * 16)) for i in range(3)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        results = [srv.wait(t) for t in tickets]
        st = srv.stats()
    finally:
        srv.close()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    assert st["batches"] < len(reqs)  # something was batched
    for k, (img, colors, engine, alpha) in enumerate(reqs):
        idx, rgba, info = results[k]
        want_idx, want_rgba = _alone(ctx, img, colors, engine, alpha)
        assert np.array_equal(idx, want_idx), (k, engine, img.shape)
        assert np.array_equal(rgba.view(np.uint32), want_rgba.view(np.uint32)), (k, engine)
        assert info["status"] == 0 and info["total_ms"] >= info["device_ms"]


@pytest.mark.parametrize("device_palettes", [False, True])
def test_admission_budget(ctx, device_palettes):
    reqs = _mix(12, 7)
    # Room for about two of the largest requests at once (rdb_request_bytes:
    # the bound the server admits by), so requests wait for each other and
    # idle workers release their cached buffers to let the next one in.
    need = [sb.Server.request_bytes(img, c, e, alpha=a, device_palettes=device_palettes)
            for img, c, e, a in reqs]
    budget = 2 * max(need) + (1 << 20)
    srv = sb.Server(workers=2, budget=budget, device_palettes=device_palettes)
    try:
        tickets = [srv.submit(img, c, e, alpha=a) for img, c, e, a in reqs]
        outs = [srv.wait(t)[0] for t in tickets]
        st = srv.stats()
        # Admitted bounds plus the contexts' kept buffers, never above it.
        assert st["peak_admitted_bytes"] <= budget
        assert st["completed"] == len(reqs) and st["failed"] == 0
        big = synth.gradient_rgb8(2048, 2048, 1)
        assert sb.Server.request_bytes(big, 16, "seq", device_palettes=device_palettes) > budget
        with pytest.raises(sb.RdbError):
            srv.submit(big, 16, "seq")
    finally:
        srv.close()
    for (img, c, e, a), idx in zip(reqs, outs):
        assert np.array_equal(idx, _alone(ctx, img, c, e, a)[0])


def test_many_geometries_and_small_alpha_batches(ctx):
    """More distinct image sizes than fit the workers' share of a small budget
    (visit orders are evicted between calls, never under the call that holds
    them), and batches of small alpha-associated images on the plain walk
    (its memo slabs are 32 MiB each, capped per launch): all complete, equal
    to each request alone."""
    rng = np.random.default_rng(11)
    reqs = []
    for k in range(160):
        w, h = int(rng.integers(8, 90)), int(rng.integers(8, 90))
        alpha = k % 2 == 0
        img = synth.gradient_rgba8(w, h, 900 + k) if alpha else synth.gradient_rgb8(w, h, 900 + k)
        reqs.append((img, int(rng.choice([4, 16, 64])), alpha))
    need = max(sb.Server.request_bytes(img, c, "seq", alpha=a) for img, c, a in reqs)
    budget = 8 * need
    srv = sb.Server(workers=2, budget=budget, max_batch=64)
    try:
        tickets = [srv.submit(img, c, "seq", alpha=a) for img, c, a in reqs]
        outs = [srv.wait(t)[0] for t in tickets]
        st = srv.stats()
    finally:
        srv.close()
    assert st["completed"] == len(reqs) and st["peak_admitted_bytes"] <= budget
    for (img, c, a), idx in zip(reqs, outs):
        assert np.array_equal(idx, _alone(ctx, img, c, "seq", a)[0])
