"""TEST INFRASTRUCTURE ONLY: ctypes bindings for the CPU checkers.

``Oracle`` wraps liboracle.so (the C restatement in oracle.c).  ``RefLib``
wraps oracle/_ref/librdref.so (the reference's own CPU sources compiled
unmodified, see oracle/Makefile) and is present only where that library was
built.  Only tests, the smoke entry point and bench.py's CPU-baseline leg use
this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "librdref.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")


def build_oracle() -> None:
    """Compile liboracle.so (and oracle/_ref when the reference tree exists)."""
    subprocess.run(["make", "-s", "-f", os.path.join(HERE, "Makefile")], check=True)


class OrcNode(C.Structure):
    _fields_ = [
        ("child", C.c_int32 * 16),
        ("parent", C.c_int32),
        ("total_color", C.c_double * 4),
        ("quantize_error", C.c_double),
        ("number_unique", C.c_uint64),
        ("color_number", C.c_uint32),
        ("id", C.c_uint32),
        ("level", C.c_uint32),
    ]


class OrcTree(C.Structure):
    _fields_ = [
        ("nodes", C.POINTER(OrcNode)),
        ("node_count", C.c_size_t),
        ("node_cap", C.c_size_t),
        ("colormap", C.POINTER(C.c_double)),
        ("color_count", C.c_int),
        ("maximum_colors", C.c_int),
        ("depth", C.c_int),
        ("node_live_count", C.c_size_t),
        ("pruning_threshold", C.c_double),
        ("next_threshold", C.c_double),
        ("associate_alpha", C.c_int),
        ("root", C.c_int32),
    ]


class Tree:
    """Result of a palette build: the colormap and the node array."""

    def __init__(self, palette, child, parent, color_number, number_unique, depth, assoc):
        self.palette = palette  # (count, 4) float64
        self.child = child  # (nodes, 16) int32
        self.parent = parent  # (nodes,) int32
        self.color_number = color_number  # (nodes,) uint32
        self.number_unique = number_unique  # (nodes,) uint64
        self.depth = depth
        self.assoc = assoc

    @property
    def count(self) -> int:
        return int(self.palette.shape[0])


class Oracle:
    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build_oracle()
        lib = C.CDLL(path)
        self.lib = lib
        lib.orc_tree_build.argtypes = [C.POINTER(OrcTree), _f32p, C.c_size_t, C.c_size_t,
                                       C.c_int, C.c_int, C.c_int]
        lib.orc_tree_free.argtypes = [C.POINTER(OrcTree)]
        lib.orc_walk_seq.argtypes = [C.POINTER(OrcTree), _f64p, C.c_int, C.c_int, C.c_double,
                                     C.c_int, C.c_size_t, C.c_size_t, _f32p, _u8p]
        lib.orc_walk_blocks.argtypes = [C.POINTER(OrcTree), _f64p, C.c_int, C.c_int, C.c_double,
                                        C.c_int, C.c_size_t, C.c_size_t, _f32p, _u8p]
        lib.orc_walk_blocks.restype = C.c_int
        lib.orc_block_chosen.argtypes = [C.POINTER(OrcTree), _f64p, C.c_int, C.c_int, C.c_double,
                                         C.c_int, C.c_size_t, C.c_size_t, _f32p, _u8p]
        lib.orc_block_chosen.restype = C.c_int
        lib.orc_seq_order.argtypes = [C.c_size_t, C.c_size_t, _i32p]
        lib.orc_seq_order.restype = C.c_size_t
        lib.orc_block_order.argtypes = [C.c_size_t, C.c_size_t, _i32p, _i32p]
        lib.orc_block_order.restype = C.c_size_t
        lib.orc_hilbert_point.argtypes = [C.c_int64, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        lib.orc_curve_level.argtypes = [C.c_size_t, C.c_size_t]
        lib.orc_curve_level.restype = C.c_int
        lib.orc_scale_quantum_to_char.argtypes = [C.c_float]
        lib.orc_scale_quantum_to_char.restype = C.c_ubyte
        lib.orc_build_error_weights.argtypes = [_f64p]
        lib.orc_inverse_filter.argtypes = [C.c_int, C.c_double, _f64p]
        lib.orc_tree_lookup.argtypes = [C.POINTER(OrcTree), C.c_double, C.c_double, C.c_double,
                                        C.c_double]
        lib.orc_tree_lookup.restype = C.c_int
        lib.orc_widen_frame.argtypes = [C.c_int, C.c_void_p, C.c_size_t, C.c_size_t, _f32p]
        lib.orc_widen_frame.restype = C.c_int
        lib.orc_narrow_frame.argtypes = [C.c_int, _f32p, C.c_size_t, C.c_size_t, C.c_void_p]
        lib.orc_narrow_frame.restype = C.c_int

    # -- palette -------------------------------------------------------------
    def build_tree_raw(self, rgbaf: np.ndarray, max_colors: int, assoc: bool, gray: bool):
        h, w = rgbaf.shape[:2]
        t = OrcTree()
        px = np.ascontiguousarray(rgbaf, dtype=np.float32).reshape(-1)
        self.lib.orc_tree_build(C.byref(t), px, w, h, int(max_colors), int(assoc), int(gray))
        return t

    def build_tree(self, rgbaf: np.ndarray, max_colors: int, assoc: bool, gray: bool) -> Tree:
        t = self.build_tree_raw(rgbaf, max_colors, assoc, gray)
        try:
            return self._export(t)
        finally:
            self.lib.orc_tree_free(C.byref(t))

    def _export(self, t: OrcTree) -> Tree:
        n = t.node_count
        count = t.color_count
        cm = np.ctypeslib.as_array(t.colormap, shape=(count * 4,)).copy().reshape(count, 4) \
            if count else np.zeros((0, 4))
        child = np.empty((n, 16), np.int32)
        parent = np.empty(n, np.int32)
        cn = np.empty(n, np.uint32)
        nu = np.empty(n, np.uint64)
        arr = (OrcNode * n).from_address(C.addressof(t.nodes.contents))
        for i in range(n):
            child[i] = arr[i].child[:]
            parent[i] = arr[i].parent
            cn[i] = arr[i].color_number
            nu[i] = arr[i].number_unique
        return Tree(cm, child, parent, cn, nu, t.depth, bool(t.associate_alpha))

    # -- walks ---------------------------------------------------------------
    def lookups(self, rgbaf: np.ndarray, max_colors: int, assoc: bool, gray: bool,
                targets: np.ndarray) -> np.ndarray:
        """Builds the palette, then the reference lookup (descent + ClosestColor,
        src/rd_riemersma_cpu.cpp:82-92) of each clamped target row (r, g, b, a)."""
        t = self.build_tree_raw(rgbaf, max_colors, assoc, gray)
        try:
            out = np.empty(len(targets), np.int32)
            for i, (r, g, b, a) in enumerate(np.asarray(targets, np.float64)):
                out[i] = self.lib.orc_tree_lookup(C.byref(t), float(r), float(g), float(b), float(a))
            return out
        finally:
            self.lib.orc_tree_free(C.byref(t))

    def walk_seq(self, rgbaf: np.ndarray, max_colors: int, assoc: bool, gray: bool,
                 diffusion: float = 1.0, use_cache: bool = True):
        """Builds the palette, then the sequential walk.  Returns (idx, out, palette)."""
        h, w = rgbaf.shape[:2]
        t = self.build_tree_raw(rgbaf, max_colors, assoc, gray)
        try:
            count = t.color_count
            pal = np.ctypeslib.as_array(t.colormap, shape=(max(count, 1) * 4,)).copy()
            out = np.ascontiguousarray(rgbaf, dtype=np.float32).reshape(-1).copy()
            idx = np.zeros(w * h, np.uint8)
            self.lib.orc_walk_seq(C.byref(t), pal, count, int(assoc), float(diffusion),
                                  int(use_cache), w, h, out, idx)
            return idx.reshape(h, w), out.reshape(h, w, 4), pal.reshape(-1, 4)[:count]
        finally:
            self.lib.orc_tree_free(C.byref(t))

    def walk_blocks(self, rgbaf: np.ndarray, max_colors: int, assoc: bool, gray: bool,
                    block: int, diffusion: float = 1.0):
        h, w = rgbaf.shape[:2]
        t = self.build_tree_raw(rgbaf, max_colors, assoc, gray)
        try:
            count = t.color_count
            pal = np.ctypeslib.as_array(t.colormap, shape=(max(count, 1) * 4,)).copy()
            out = np.ascontiguousarray(rgbaf, dtype=np.float32).reshape(-1).copy()
            idx = np.zeros(w * h, np.uint8)
            rc = self.lib.orc_walk_blocks(C.byref(t), pal, count, int(assoc), float(diffusion),
                                          int(block), w, h, out, idx)
            if rc != 0:
                raise ValueError("blocks walk refused")
            return idx.reshape(h, w), out.reshape(h, w, 4), pal.reshape(-1, 4)[:count]
        finally:
            self.lib.orc_tree_free(C.byref(t))

    def block_chosen(self, rgbaf: np.ndarray, max_colors: int, assoc: bool, gray: bool,
                     block: int, diffusion: float = 1.0) -> np.ndarray:
        """The chosen index at every block-list position (list order)."""
        return self.block_chosen_with_tree(rgbaf, rgbaf, max_colors, assoc, gray, block, diffusion)

    def block_chosen_with_tree(self, tree_src: np.ndarray, rgbaf: np.ndarray, max_colors: int,
                               assoc: bool, gray: bool, block: int,
                               diffusion: float = 1.0) -> np.ndarray:
        """block_chosen of `rgbaf` with the tree built from `tree_src`."""
        h, w = rgbaf.shape[:2]
        t = self.build_tree_raw(tree_src, max_colors, assoc, gray)
        try:
            pal = np.ctypeslib.as_array(t.colormap, shape=(max(t.color_count, 1) * 4,)).copy()
            px = np.ascontiguousarray(rgbaf, dtype=np.float32).reshape(-1)
            out = np.zeros(w * h + 1, np.uint8)
            n = self.lib.orc_block_chosen(C.byref(t), pal, t.color_count, int(assoc),
                                          float(diffusion), int(block), w, h, px, out)
            if n < 0:
                raise ValueError("blocks walk refused")
            return out[:n]
        finally:
            self.lib.orc_tree_free(C.byref(t))

    # -- curve ----------------------------------------------------------------
    def seq_order(self, w: int, h: int) -> np.ndarray:
        out = np.empty(max(w * h, 1), np.int32)
        n = self.lib.orc_seq_order(w, h, out)
        return out[:n]

    # -- video frame formats ---------------------------------------------------
    def widen_frame(self, fmt: int, raw, w: int, h: int) -> np.ndarray:
        """orc_widen_frame: one frame of `fmt` bytes -> (h, w, 4) RgbaF."""
        buf = np.ascontiguousarray(np.frombuffer(np.ascontiguousarray(raw).tobytes(), np.uint8))
        out = np.empty(w * h * 4, np.float32)
        if self.lib.orc_widen_frame(int(fmt), buf.ctypes.data, w, h, out) != 0:
            raise ValueError(f"format {fmt} not widened")
        return out.reshape(h, w, 4)

    def narrow_frame(self, fmt: int, rgbaf: np.ndarray) -> np.ndarray:
        """orc_narrow_frame: (h, w, 4) RgbaF -> the frame's bytes as uint8."""
        h, w = rgbaf.shape[:2]
        src = np.ascontiguousarray(rgbaf, dtype=np.float32).reshape(-1)
        out = np.zeros(w * h * (8 if fmt == 8 else 3), np.uint8)
        if self.lib.orc_narrow_frame(int(fmt), src, w, h, out.ctypes.data) != 0:
            raise ValueError(f"format {fmt} not narrowed")
        return out

    def walk_blocks_raw(self, tree_src: np.ndarray, raw_frames: np.ndarray, in_fmt: int,
                        w: int, h: int, out_fmt: int, max_colors: int, assoc: bool,
                        block: int, diffusion: float = 1.0):
        """RiemersmaBlocksCpu's fused form restated: every frame (one row of
        `raw_frames`, uint8) is widened, block-walked with the tree built from
        `tree_src` (RgbaF) and narrowed to `out_fmt` (16 = RgbaF bytes).
        Returns (out (F, bytes) uint8, indices (F, h, w))."""
        t = self.build_tree_raw(tree_src, max_colors, assoc, False)
        try:
            count = t.color_count
            pal = np.ctypeslib.as_array(t.colormap, shape=(max(count, 1) * 4,)).copy()
            outs, idxs = [], []
            for f in range(raw_frames.shape[0]):
                px = self.widen_frame(in_fmt, raw_frames[f], w, h).reshape(-1).copy()
                idx = np.zeros(w * h, np.uint8)
                rc = self.lib.orc_walk_blocks(C.byref(t), pal, count, int(assoc),
                                              float(diffusion), int(block), w, h, px, idx)
                if rc != 0:
                    raise ValueError("blocks walk refused")
                px = px.reshape(h, w, 4)
                outs.append(px.view(np.uint8).reshape(-1) if out_fmt == 16
                            else self.narrow_frame(out_fmt, px))
                idxs.append(idx.reshape(h, w))
            return np.stack(outs), np.stack(idxs)
        finally:
            self.lib.orc_tree_free(C.byref(t))

    def block_order(self, w: int, h: int):
        out = np.empty(w * h + 1, np.int32)
        owner = np.empty(max(w * h, 1), np.int32)
        n = self.lib.orc_block_order(w, h, out, owner)
        return out[:n], owner[: w * h]

    def error_weights(self) -> np.ndarray:
        w = np.zeros(16, np.float64)
        self.lib.orc_build_error_weights(w)
        return w

    def inverse_filter(self, taps: int, diffusion: float = 1.0) -> np.ndarray:
        g = np.zeros(taps + 1, np.float64)
        self.lib.orc_inverse_filter(taps, diffusion, g)
        return g


class RefLib:
    """The reference's own CPU code (oracle/_ref).  Raises if not built."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        lib = C.CDLL(path)
        self.lib = lib
        lib.ref_tree_build.argtypes = [_f32p, C.c_size_t, C.c_size_t, C.c_int, C.c_int, C.c_int]
        lib.ref_tree_build.restype = C.c_void_p
        lib.ref_tree_free.argtypes = [C.c_void_p]
        lib.ref_tree_color_count.argtypes = [C.c_void_p]
        lib.ref_tree_depth.argtypes = [C.c_void_p]
        lib.ref_tree_node_count.argtypes = [C.c_void_p]
        lib.ref_tree_node_count.restype = C.c_size_t
        lib.ref_tree_colormap.argtypes = [C.c_void_p, _f64p]
        lib.ref_tree_nodes.argtypes = [C.c_void_p, _i32p, _i32p, _u32p, _u64p, _u32p]
        lib.ref_walk_seq.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_size_t, C.c_size_t, _f32p]
        lib.ref_walk_blocks.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_size_t, C.c_size_t,
                                        _f32p, C.c_int, C.c_char_p, C.c_size_t]
        lib.ref_walk_blocks.restype = C.c_int
        lib.ref_walk_blocks_raw.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_size_t,
                                            C.c_size_t, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                            C.c_void_p, C.c_size_t, C.c_int, C.c_int, C.c_char_p,
                                            C.c_size_t]
        lib.ref_walk_blocks_raw.restype = C.c_int
        lib.ref_hilbert_point.argtypes = [C.c_int64, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        lib.ref_curve_level.argtypes = [C.c_size_t, C.c_size_t]
        lib.ref_block_curve.argtypes = [C.c_size_t, C.c_size_t, _i32p, _i32p]
        lib.ref_block_curve.restype = C.c_size_t
        lib.ref_curve_sequence.argtypes = [C.c_int, _i32p]
        lib.ref_curve_sequence.restype = C.c_size_t
        lib.ref_curve_mismatches.argtypes = [C.c_int]
        lib.ref_curve_mismatches.restype = C.c_size_t
        lib.ref_error_weights.argtypes = [_f64p]
        lib.ref_scale_char.argtypes = [C.c_float]
        lib.ref_scale_char.restype = C.c_uint

    def build_tree(self, rgbaf: np.ndarray, max_colors: int, assoc: bool, gray: bool) -> Tree:
        h, w = rgbaf.shape[:2]
        px = np.ascontiguousarray(rgbaf, dtype=np.float32).reshape(-1)
        t = self.lib.ref_tree_build(px, w, h, int(max_colors), int(assoc), int(gray))
        try:
            return self._export(t, assoc)
        finally:
            self.lib.ref_tree_free(t)

    def _export(self, t, assoc) -> Tree:
        count = self.lib.ref_tree_color_count(t)
        cm = np.zeros(max(count, 1) * 4, np.float64)
        self.lib.ref_tree_colormap(t, cm)
        n = self.lib.ref_tree_node_count(t)
        child = np.zeros(n * 16, np.int32)
        parent = np.zeros(n, np.int32)
        cn = np.zeros(n, np.uint32)
        nu = np.zeros(n, np.uint64)
        lv = np.zeros(n, np.uint32)
        self.lib.ref_tree_nodes(t, child, parent, cn, nu, lv)
        return Tree(cm.reshape(-1, 4)[:count], child.reshape(n, 16), parent, cn, nu,
                    self.lib.ref_tree_depth(t), bool(assoc))

    def walk_seq(self, rgbaf: np.ndarray, max_colors: int, assoc: bool, gray: bool,
                 diffusion: float = 1.0, use_cache: bool = True):
        """Returns (out RgbaF, palette)."""
        h, w = rgbaf.shape[:2]
        px = np.ascontiguousarray(rgbaf, dtype=np.float32).reshape(-1)
        t = self.lib.ref_tree_build(px, w, h, int(max_colors), int(assoc), int(gray))
        try:
            count = self.lib.ref_tree_color_count(t)
            cm = np.zeros(max(count, 1) * 4, np.float64)
            self.lib.ref_tree_colormap(t, cm)
            out = px.copy()
            self.lib.ref_walk_seq(t, float(diffusion), int(use_cache), w, h, out)
            return out.reshape(h, w, 4), cm.reshape(-1, 4)[:count]
        finally:
            self.lib.ref_tree_free(t)

    def walk_blocks(self, rgbaf: np.ndarray, max_colors: int, assoc: bool, gray: bool,
                    block: int, diffusion: float = 1.0):
        h, w = rgbaf.shape[:2]
        px = np.ascontiguousarray(rgbaf, dtype=np.float32).reshape(-1)
        t = self.lib.ref_tree_build(px, w, h, int(max_colors), int(assoc), int(gray))
        try:
            count = self.lib.ref_tree_color_count(t)
            cm = np.zeros(max(count, 1) * 4, np.float64)
            self.lib.ref_tree_colormap(t, cm)
            out = px.copy()
            err = C.create_string_buffer(1024)
            rc = self.lib.ref_walk_blocks(t, float(diffusion), int(block), w, h, out, 1, err, 1024)
            if rc != 0:
                raise ValueError(err.value.decode())
            return out.reshape(h, w, 4), cm.reshape(-1, 4)[:count]
        finally:
            self.lib.ref_tree_free(t)

    def walk_seq_frame(self, tree_src: np.ndarray, frame: np.ndarray, max_colors: int,
                       assoc: bool, gray: bool, diffusion: float = 1.0,
                       use_cache: bool = True) -> np.ndarray:
        """RiemersmaWalkCpu of `frame` with the tree built from `tree_src`."""
        h, w = tree_src.shape[:2]
        src = np.ascontiguousarray(tree_src, dtype=np.float32).reshape(-1)
        t = self.lib.ref_tree_build(src, w, h, int(max_colors), int(assoc), int(gray))
        try:
            out = np.ascontiguousarray(frame, dtype=np.float32).reshape(-1).copy()
            self.lib.ref_walk_seq(t, float(diffusion), int(use_cache), w, h, out)
            return out.reshape(h, w, 4)
        finally:
            self.lib.ref_tree_free(t)

    def walk_blocks_frames(self, tree_src: np.ndarray, frames: np.ndarray, max_colors: int,
                           assoc: bool, gray: bool, block: int, diffusion: float = 1.0):
        """RiemersmaBlocksCpu over F frames in place ((F, H, W, 4) float32), the
        tree built from `tree_src`.  Returns (0, "") or (-1, refusal)."""
        h, w = tree_src.shape[:2]
        src = np.ascontiguousarray(tree_src, dtype=np.float32).reshape(-1)
        t = self.lib.ref_tree_build(src, w, h, int(max_colors), int(assoc), int(gray))
        try:
            flat = frames.reshape(-1)
            assert flat.base is frames or flat.base is frames.base or np.shares_memory(flat, frames)
            err = C.create_string_buffer(1024)
            rc = self.lib.ref_walk_blocks(t, float(diffusion), int(block), w, h, flat,
                                          frames.shape[0], err, 1024)
            return rc, err.value.decode()
        finally:
            self.lib.ref_tree_free(t)

    def walk_blocks_raw(self, tree_src: np.ndarray, in_frames, gather_layout: int,
                        gather_channels: int, w: int, h: int, out_yuv444: bool,
                        max_colors: int, assoc: bool, block: int, diffusion: float = 1.0):
        """RiemersmaBlocksCpu's fused output (and, with gather_layout 3 or 4,
        fused gather) over F frames, the tree built from `tree_src`.
        `in_frames`: (F, H, W, 4) float32 when gather_layout is 0, else (F,
        frame_bytes) uint8 of the decoder's bytes.  Returns (rc, message,
        out (F, bytes) uint8)."""
        src = np.ascontiguousarray(tree_src, dtype=np.float32).reshape(-1)
        t = self.lib.ref_tree_build(src, w, h, int(max_colors), int(assoc), 0)
        try:
            frames = in_frames.shape[0]
            out = np.zeros((frames, w * h * (3 if out_yuv444 else 8)), np.uint8)
            err = C.create_string_buffer(1024)
            if gather_layout == 0:
                rgba = np.ascontiguousarray(in_frames, dtype=np.float32)
                rc = self.lib.ref_walk_blocks_raw(t, float(diffusion), int(block), w, h,
                                                  rgba.ctypes.data, frames, out.ctypes.data,
                                                  int(out_yuv444), None, 0, 0, 0, err, 1024)
            else:
                raw = np.ascontiguousarray(in_frames, dtype=np.uint8)
                rc = self.lib.ref_walk_blocks_raw(t, float(diffusion), int(block), w, h, None,
                                                  frames, out.ctypes.data, int(out_yuv444),
                                                  raw.ctypes.data, raw.shape[1], int(gather_layout),
                                                  int(gather_channels), err, 1024)
            return rc, err.value.decode(), out
        finally:
            self.lib.ref_tree_free(t)

    def block_order(self, w: int, h: int):
        out = np.empty(w * h + 1, np.int32)
        owner = np.empty(max(w * h, 1), np.int32)
        n = self.lib.ref_block_curve(w, h, out, owner)
        return out[:n], owner[: w * h]

    def curve_sequence(self, level: int) -> np.ndarray:
        n = 1 << (2 * level)
        xy = np.zeros(2 * n, np.int32)
        self.lib.ref_curve_sequence(level, xy)
        return xy.reshape(n, 2)

    def error_weights(self) -> np.ndarray:
        w = np.zeros(16, np.float64)
        self.lib.ref_error_weights(w)
        return w


DROPIN_SO = os.path.join(HERE, "_ref", "librddropin.so")


class DropinLib:
    """The reference-facing C++ layer (stipple_b200/dropin) driven through
    oracle/dropin_shim.cpp with trees from the reference's ColorTree::Build.
    Test infrastructure: present only where the reference headers were."""

    ENGINES = {"walk": 0, "blocks": 1, "approx": 2, "plugin": 3}

    def __init__(self, path: str = DROPIN_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = lib = C.CDLL(path)
        lib.dropin_available.restype = C.c_int
        lib.dropin_max_frames.argtypes = [C.c_size_t, C.c_size_t, C.c_size_t]
        lib.dropin_max_frames.restype = C.c_int
        lib.dropin_inverse_filter.argtypes = [C.c_int, C.c_double,
                                              np.ctypeslib.ndpointer(np.float64)]
        lib.dropin_inverse_filter.restype = C.c_int
        lib.dropin_alloc_pinned.argtypes = [C.c_size_t]
        lib.dropin_alloc_pinned.restype = C.c_void_p
        lib.dropin_free_pinned.argtypes = [C.c_void_p]
        f32 = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
        lib.dropin_run.argtypes = [C.c_int, f32, C.c_size_t, C.c_size_t, C.c_int, C.c_int, C.c_int,
                                   f32, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                                   C.c_int, C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t]
        lib.dropin_run.restype = C.c_int
        lib.dropin_blocks_fused.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_int, C.c_int,
                                            C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                            C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                            C.c_char_p, C.c_size_t]
        lib.dropin_blocks_fused.restype = C.c_int

    def run(self, engine: str, tree_src: np.ndarray, frames: np.ndarray, colors: int,
            assoc: bool = False, gray: bool = False, diffusion: float = 1.0,
            use_cache: bool = True, block: int = 512, iterations: int = 20, taps: int = 96,
            slot: int = 0):
        """Dithers `frames` ((F, H, W, 4) float32, Q16) in place; returns
        (error or "", device name)."""
        h, w = tree_src.shape[:2]
        err = C.create_string_buffer(512)
        dev = C.create_string_buffer(256)
        src = np.ascontiguousarray(tree_src, np.float32)
        rc = self.lib.dropin_run(self.ENGINES[engine], src, w, h, colors, int(assoc), int(gray),
                                 frames, frames.shape[0], float(diffusion), int(use_cache), block,
                                 iterations, taps, slot, err, 512, dev, 256)
        return ("" if rc == 0 else err.value.decode()), dev.value.decode()

    def blocks_fused(self, tree_src: np.ndarray, frames: int, colors: int, assoc: bool = False,
                     block: int = 512, batch: np.ndarray | None = None, in_raw=None,
                     in_mode: int = 0, in_channels: int = 4, out_raw=None,
                     emit_yuv444: bool = False) -> str:
        """RiemersmaBlocksCuda with upload_u16 (when in_raw is given) and / or
        emit_u16 (when out_raw is given).  Returns the error or ""."""
        h, w = tree_src.shape[:2]
        err = C.create_string_buffer(512)
        src = np.ascontiguousarray(tree_src, np.float32)
        ptr = (lambda a: None if a is None else a.ctypes.data)
        rc = self.lib.dropin_blocks_fused(
            src.ctypes.data, w, h, colors, int(assoc), ptr(batch), frames, block,
            int(in_raw is not None), in_mode, in_channels, ptr(in_raw), int(out_raw is not None),
            int(emit_yuv444), ptr(out_raw), err, 512)
        return "" if rc == 0 else err.value.decode()

    def inverse_filter(self, taps: int, diffusion: float = 1.0) -> np.ndarray:
        out = np.zeros(taps + 1, np.float64)
        n = self.lib.dropin_inverse_filter(taps, diffusion, out)
        return out[:n]


def dropin_available() -> bool:
    return os.path.exists(DROPIN_SO)


def ref_available() -> bool:
    return os.path.exists(REF_SO)
