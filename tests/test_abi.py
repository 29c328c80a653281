"""The C ABI: the library loads without a GPU and exports every symbol the
headers in include/ declare."""
from __future__ import annotations

import glob
import os
import re

from conftest import ROOT


def declared_symbols():
    syms = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b(rdb_[a-z0-9_]+)\s*\(", text):
            syms.add(m.group(1))
    return syms


def test_library_exports_every_declared_symbol(lib):
    syms = declared_symbols()
    assert len(syms) >= 25
    missing = [s for s in sorted(syms) if not hasattr(lib, s)]
    assert not missing, missing


def test_python_mirror_covers_the_abi(lib):
    import stipple_b200 as sb
    assert declared_symbols() <= set(sb.SIGNATURES)


def test_host_only_calls_work_without_device(lib):
    import stipple_b200 as sb
    assert sb.block_gap(256, 192) == 255
    assert sb.block_gap(1920, 1080) == -1
    w = sb.error_weights()
    assert w.shape == (16,)
    o = sb.options()
    assert o.block == 512 and o.use_cache == 1 and o.jacobi_taps == 96


def test_errors_are_reported(lib):
    import ctypes as C
    import numpy as np
    import pytest
    import stipple_b200 as sb
    with pytest.raises(sb.RdbError) as e:
        sb._check(lib.rdb_inverse_filter(0, 1.0, sb._ptr(np.zeros(4))))
    assert "taps" in str(e.value)
    h = C.c_void_p()
    assert lib.rdb_octree_build(None, 3, 1, 1, 0, 16, 0, 0, C.byref(h)) != 0
    assert b"null" in lib.rdb_last_error()
