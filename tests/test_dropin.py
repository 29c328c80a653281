"""The reference-facing C++ layer (stipple_b200/dropin), on the CPU: it exports
the seven engine symbols of the reference's rd_riemersma.h with the
reference's own signatures, registers "riemersma-b200" with the reference's
dither registry, and reports a missing device the way the reference's engines
do -- a message, never a silent success."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

from oracle import pyoracle
from stipple_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "stipple_b200", "lib", "librd_b200_dropin.so")

pytestmark = pytest.mark.skipif(not os.path.exists(LIB) or not pyoracle.dropin_available(),
                                reason="drop-in layer not built (reference headers absent)")

# include/rd_riemersma.h:214-217, :284, :288, :303-307, :310, :450-464, :480-481
EXPECTED = [
    "rd::CudaAvailable()",
    "rd::CudaMaxFrames(unsigned long, unsigned long, unsigned long)",
    "rd::CudaAllocPinned(unsigned long)",
    "rd::CudaFreePinned(void*)",
    "rd::ApproxInverseFilter(int, double)",
    "rd::RiemersmaWalkCuda(rd::Palette const&, rd::DitherParams const&, "
    "rd::ColorTree const&, unsigned long, unsigned long, rd::RgbaF*, int, "
    "std::__cxx11::basic_string<char, std::char_traits<char>, std::allocator<char> >*)",
    "rd::RiemersmaBlocksCuda(rd::Palette const&, rd::DitherParams const&, "
    "rd::ColorTree const&, unsigned long, unsigned long, rd::RgbaF*, rd::BlockOptions const&, "
    "std::__cxx11::basic_string<char, std::char_traits<char>, std::allocator<char> >*, "
    "unsigned short*, int, unsigned short const*)",
    "rd::RiemersmaApproxCuda(rd::Palette const&, rd::DitherParams const&, "
    "rd::ColorTree const&, unsigned long, unsigned long, rd::RgbaF*, rd::ApproxOptions const&, "
    "std::__cxx11::basic_string<char, std::char_traits<char>, std::allocator<char> >*)",
]


def _exports(path):
    out = subprocess.run(["nm", "-DC", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    return {line.split(" ", 2)[2] for line in out.splitlines() if line.count(" ") >= 2}


def test_exports_reference_signatures():
    names = _exports(LIB)
    for sym in EXPECTED:
        assert sym in names, sym


def test_inverse_filter_matches_c_abi():
    import stipple_b200 as sb
    d = pyoracle.DropinLib()
    for taps in (1, 16, 96):
        assert np.array_equal(d.inverse_filter(taps, 0.75), sb.inverse_filter(taps, 0.75))
    assert len(d.inverse_filter(0)) == 0  # the reference's range is 1..4096


def test_plugin_registered_and_reports_errors_without_device():
    d = pyoracle.DropinLib()
    if d.lib.dropin_available():
        pytest.skip("a device is present; the GPU tests cover this path")
    img = synth.to_q16(synth.gradient_rgb8(24, 16, 1))
    for eng in ("walk", "blocks", "approx", "plugin"):
        frames = img[None].copy()
        before = frames.copy()
        err, _ = d.run(eng, img, frames, 8)
        assert err, eng                                # never "" without output
        assert "not registered" not in err, eng        # the registry entry exists
        assert np.array_equal(frames, before), eng     # nothing half-written
    assert d.lib.dropin_max_frames(64, 64, 0) == 0


def test_refusals_match_reference():
    d = pyoracle.DropinLib()
    img = synth.to_q16(synth.gradient_rgb8(24, 16, 1))
    err, _ = d.run("blocks", img, img[None].copy(), 8, block=8)
    assert "block must be >= 16" in err
    err, _ = d.run("approx", img, img[None].copy(), 8, taps=0)
    assert "taps" in err
