"""The numeric contract (include/rd_types.h of the reference) on the host side."""
from __future__ import annotations

import os
import subprocess

import numpy as np

from conftest import ROOT


def test_scale_char_exhaustive(oracle, tmp_path):
    """min(255, (trunc(2q)+257)/514) equals q/257.0f+0.5f truncated for every
    float in [0, 65535] -- the form the kernels use on the dependent chain."""
    exe = tmp_path / "numeric_check"
    src = os.path.join(ROOT, "tests", "numeric_check.cpp")
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-std=c++17",
                    "-I", os.path.join(ROOT, "stipple_b200", "csrc"), src,
                    os.path.join(ROOT, "oracle", "liboracle.so"),
                    f"-Wl,-rpath,{os.path.join(ROOT, 'oracle')}", "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("mismatches 0 checked 1199570691")


def test_error_weights(oracle, lib):
    import stipple_b200 as sb
    w = sb.error_weights()
    assert np.array_equal(w.view(np.uint64), oracle.error_weights().view(np.uint64))
    assert w[0] == 1.0 and abs(w[15] - 1.0 / 16.0) < 1e-15
    assert np.all(np.diff(w) < 0)


def test_error_weights_match_reference(oracle, reflib):
    assert np.array_equal(oracle.error_weights().view(np.uint64),
                          reflib.error_weights().view(np.uint64))


def test_inverse_filter(oracle, lib):
    import stipple_b200 as sb
    for taps in (1, 16, 96, 300):
        for diff in (1.0, 0.75):
            a = sb.inverse_filter(taps, diff)
            b = oracle.inverse_filter(taps, diff)
            assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


def test_block_gap_rule(oracle, lib):
    """The block list misses (2^L-1, 0), inside the image exactly when W is a
    power of two and W >= H (src/rd_riemersma_cpu.cpp:439-455)."""
    import stipple_b200 as sb
    geoms = [(256, 192), (512, 480), (1024, 768), (64, 64), (320, 240), (480, 512),
             (33, 17), (2, 1), (1, 2), (16, 3), (3, 16), (1920, 1080), (128, 128)]
    for w, h in geoms:
        _, owner = oracle.block_order(w, h)
        gaps = np.nonzero(owner < 0)[0]
        want = int(gaps[0]) if len(gaps) else -1
        assert len(gaps) <= 1
        assert sb.block_gap(w, h) == want, (w, h)
