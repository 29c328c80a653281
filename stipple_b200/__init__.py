"""Riemersma dithering on B200 (sm_100a): Python mirror of the C ABI in include/rdb.h.

The engines live in ``stipple_b200/lib/librdb_b200.so`` (built by
``python -m stipple_b200.build``).  This module only binds that library with
ctypes for tests, the benchmark and scripting; it has no compute path of its
own and raises if the library is missing.

Engines (``ENGINE_*``) mirror the reference's entry points: ``SEQ`` is
RiemersmaWalkCpu/Cuda (bit-exact, memoised), ``BLOCKS`` is
RiemersmaBlocksCpu/Cuda (bit-exact with the host block walk), ``JACOBI`` is
RiemersmaApproxCuda (tolerance-held).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "librdb_b200.so")

RGB8, RGBA8, RGBAF32 = 3, 4, 16
ENGINE_SEQ, ENGINE_BLOCKS, ENGINE_JACOBI = 0, 1, 2
ENGINES = {"seq": ENGINE_SEQ, "blocks": ENGINE_BLOCKS, "jacobi": ENGINE_JACOBI}


class RdbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"rdb error {code}: {msg}")
        self.code = code


class KernelStats(C.Structure):
    """rdb_kernel_stats (include/rdb.h)."""
    _fields_ = [("walk_launches", C.c_int64), ("walk_ms", C.c_double),
                ("walk_positions", C.c_int64), ("passes", C.c_int64), ("launches", C.c_int64),
                ("seg_len", C.c_int64), ("chains", C.c_int64), ("block_threads", C.c_int),
                ("block_min_ctas", C.c_int), ("octree_ms", C.c_double * 4)]


class Options(C.Structure):
    _fields_ = [
        ("diffusion", C.c_double),
        ("use_cache", C.c_int),
        ("block", C.c_int),
        ("jacobi_iters", C.c_int),
        ("jacobi_taps", C.c_int),
        ("jacobi_fp64", C.c_int),
        ("cache_bits", C.c_int),
        ("seq_mode", C.c_int),
        ("seg_len", C.c_int),
        ("warm_len", C.c_int),
        ("max_passes", C.c_int),
        ("loop_mode", C.c_int),
        ("jacobi_form", C.c_int),
        ("seg_window", C.c_int),
        ("walk_form", C.c_int),
    ]


class ServerOptions(C.Structure):
    """rdb_server_options (include/rdb.h)."""
    _fields_ = [("device", C.c_int), ("memory_budget", C.c_size_t), ("workers", C.c_int),
                ("max_batch", C.c_int), ("host_threads", C.c_int), ("device_palettes", C.c_int)]


class Request(C.Structure):
    """rdb_request (include/rdb.h)."""
    _fields_ = [("pixels", C.c_void_p), ("row_stride", C.c_size_t), ("width", C.c_int),
                ("height", C.c_int), ("layout", C.c_int), ("colors", C.c_int),
                ("associate_alpha", C.c_int), ("engine", C.c_int), ("options", Options),
                ("indices", C.c_void_p), ("rgba_out", C.c_void_p)]


class RequestResult(C.Structure):
    _fields_ = [("status", C.c_int), ("queue_ms", C.c_double), ("admit_ms", C.c_double),
                ("device_ms", C.c_double), ("total_ms", C.c_double), ("batch_size", C.c_int)]


class ServerStats(C.Structure):
    _fields_ = [("completed", C.c_int64), ("failed", C.c_int64), ("pixels", C.c_int64),
                ("batches", C.c_int64), ("p50_ms", C.c_double), ("p99_ms", C.c_double),
                ("max_ms", C.c_double), ("mpx_per_s", C.c_double),
                ("peak_admitted_bytes", C.c_size_t), ("stage_p50_ms", C.c_double * 5),
                ("stage_p99_ms", C.c_double * 5), ("host_threads", C.c_int), ("workers", C.c_int)]


# Latency stages of a served request (RDB_STAGE_* in include/rdb.h).
SERVER_STAGES = ("build_wait", "build", "admit", "device", "total")


class LatencyTable(C.Structure):
    """rdb_latency_table (include/rdb.h): cycles per dependent operation."""
    _fields_ = [("dadd", C.c_double), ("dmul", C.c_double), ("f64_to_f32", C.c_double),
                ("f32_to_f64", C.c_double), ("f32_to_int", C.c_double),
                ("shared_load", C.c_double), ("global_load_l1", C.c_double),
                ("global_load_l2", C.c_double), ("int_op", C.c_double)]


class Job(C.Structure):
    _fields_ = [
        ("pixels", C.c_void_p),
        ("row_stride", C.c_size_t),
        ("width", C.c_int),
        ("height", C.c_int),
        ("layout", C.c_int),
        ("palette_id", C.c_int),
        ("indices", C.c_void_p),
        ("rgba_out", C.c_void_p),
    ]


HostJob = Job  # same layout: rdb_host_job

# Frame formats of rdb_dither_frames (include/rdb.h), beside RGB8 / RGBA8 /
# RGBAF32 = 3 / 4 / 16.
RGB8, RGBA8, RGBAF32 = 3, 4, 16
RGB16, RGBA16, YUV444P8, YUV420P8 = 6, 8, 444, 420


class Frames(C.Structure):
    _fields_ = [
        ("inp", C.c_void_p),
        ("in_frame_bytes", C.c_size_t),
        ("in_format", C.c_int),
        ("width", C.c_int),
        ("height", C.c_int),
        ("frames", C.c_int),
        ("palette_id", C.c_int),
        ("out_format", C.c_int),
        ("out", C.c_void_p),
        ("out_frame_bytes", C.c_size_t),
        ("indices", C.c_void_p),
    ]


class PaletteDesc(C.Structure):
    _fields_ = [
        ("count", C.c_int),
        ("associate_alpha", C.c_int),
        ("colors", C.c_void_p),
        ("search_colors", C.c_void_p),
        ("node_count", C.c_int),
        ("root", C.c_int),
        ("child", C.c_void_p),
        ("parent", C.c_void_p),
        ("color_number", C.c_void_p),
        ("number_unique", C.c_void_p),
    ]


# Every symbol include/rdb.h declares, with (restype, argtypes).
SIGNATURES = {
    "rdb_last_error": (C.c_char_p, []),
    "rdb_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "rdb_device_name": (C.c_int, [C.c_int, C.c_char_p, C.c_size_t]),
    "rdb_alloc_pinned": (C.c_void_p, [C.c_size_t]),
    "rdb_free_pinned": (None, [C.c_void_p]),
    "rdb_octree_build": (C.c_int, [C.c_void_p, C.c_int, C.c_size_t, C.c_size_t, C.c_size_t,
                                   C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "rdb_octree_color_count": (C.c_int, [C.c_void_p]),
    "rdb_octree_node_count": (C.c_int, [C.c_void_p]),
    "rdb_octree_depth": (C.c_int, [C.c_void_p]),
    "rdb_octree_colormap": (None, [C.c_void_p, C.c_void_p]),
    "rdb_octree_nodes": (None, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "rdb_octree_free": (None, [C.c_void_p]),
    "rdb_is_grayscale": (C.c_int, [C.c_void_p, C.c_int, C.c_size_t, C.c_size_t, C.c_size_t]),
    "rdb_palette_write_text": (C.c_int, [C.c_void_p, C.c_int, C.c_char_p]),
    "rdb_palette_read_text": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_void_p),
                                        C.POINTER(C.c_int)]),
    "rdb_context_create": (C.c_int, [C.c_int, C.c_size_t, C.POINTER(C.c_void_p)]),
    "rdb_context_destroy": (None, [C.c_void_p]),
    "rdb_context_bytes": (C.c_size_t, [C.c_void_p]),
    "rdb_context_last_passes": (C.c_int, [C.c_void_p]),
    "rdb_context_last_sweeps": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "rdb_server_create": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "rdb_server_submit": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_uint64)]),
    "rdb_request_bytes": (C.c_size_t, [C.c_void_p, C.c_int]),
    "rdb_server_wait": (C.c_int, [C.c_void_p, C.c_uint64, C.c_int, C.c_void_p]),
    "rdb_server_stats_get": (C.c_int, [C.c_void_p, C.c_void_p]),
    "rdb_server_stats_reset": (C.c_int, [C.c_void_p]),
    "rdb_probe_latency": (C.c_int, [C.c_int, C.c_void_p]),
    "rdb_context_dump_indices": (C.c_int, [C.c_void_p, C.c_char_p]),
    "rdb_octree_build_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_size_t, C.c_size_t,
                                          C.c_size_t, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                          C.POINTER(C.c_void_p), C.POINTER(C.c_int)]),
    "rdb_palette_write_png": (C.c_int, [C.c_void_p, C.c_int, C.c_char_p]),
    "rdb_palette_read_png": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_void_p)]),
    "rdb_server_destroy": (None, [C.c_void_p]),
    "rdb_max_frames": (C.c_int, [C.c_int, C.c_int, C.c_size_t, C.c_size_t, C.c_size_t]),
    "rdb_context_profile": (C.c_int, [C.c_void_p, C.c_int]),
    "rdb_context_stats": (C.c_int, [C.c_void_p, C.c_void_p]),
    "rdb_palette_create": (C.c_int, [C.c_void_p, C.POINTER(PaletteDesc), C.POINTER(C.c_int)]),
    "rdb_palette_from_octree": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]),
    "rdb_plan_build": (C.c_int, [C.POINTER(PaletteDesc), C.c_void_p, C.c_size_t,
                                 C.POINTER(C.c_size_t)]),
    "rdb_palette_destroy": (C.c_int, [C.c_void_p, C.c_int]),
    "rdb_palette_uniform": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]),
    "rdb_options_default": (None, [C.POINTER(Options)]),
    "rdb_dither": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(Job), C.c_int, C.POINTER(Options),
                             C.c_void_p]),
    "rdb_synchronize": (C.c_int, [C.c_void_p, C.c_void_p]),
    "rdb_dither_host": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(HostJob), C.c_int,
                                  C.POINTER(Options)]),
    "rdb_frame_bytes": (C.c_size_t, [C.c_int, C.c_int, C.c_int]),
    "rdb_dither_frames": (C.c_int, [C.c_void_p, C.POINTER(Frames), C.POINTER(Options), C.c_void_p]),
    "rdb_dither_frames_host": (C.c_int, [C.c_void_p, C.POINTER(Frames), C.POINTER(Options)]),
    "rdb_dither_seq_noalloc": (C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_int,
                                         C.c_int, C.c_int, C.c_void_p, C.c_double, C.c_int,
                                         C.c_void_p]),
    "rdb_error_weights": (None, [C.c_void_p]),
    "rdb_inverse_filter": (C.c_int, [C.c_int, C.c_double, C.c_void_p]),
    "rdb_block_gap": (C.c_int64, [C.c_int, C.c_int]),
}

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load librdb_b200.so; raises FileNotFoundError when it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with `python -m stipple_b200.build` "
            "(there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _check(rc: int) -> None:
    if rc != 0:
        raise RdbError(rc, load().rdb_last_error().decode())


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def options(**kw) -> Options:
    o = Options()
    load().rdb_options_default(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def layout_of(img: np.ndarray) -> int:
    if img.dtype == np.float32:
        if img.shape[-1] != 4:
            raise ValueError("float images must be RGBA (Q16 RgbaF)")
        return RGBAF32
    if img.dtype != np.uint8 or img.shape[-1] not in (3, 4):
        raise ValueError("uint8 images must be RGB or RGBA")
    return int(img.shape[-1])


class Octree:
    """Host palette build with ImageMagick octree semantics (rdb_octree_build)."""

    def __init__(self, img: np.ndarray | None, max_colors: int = 0,
                 associate_alpha: bool | None = None, grayscale: bool | None = None):
        lib = load()
        if img is None:  # filled by a reader (read_palette_text)
            self.handle = C.c_void_p()
            self.associate_alpha = False
            self.grayscale = False
            return
        img = np.ascontiguousarray(img)
        lay = layout_of(img)
        h, w = img.shape[:2]
        if associate_alpha is None:
            associate_alpha = lay == RGBA8
        if grayscale is None:
            grayscale = bool(lib.rdb_is_grayscale(_ptr(img), lay, w, h, 0))
        self.handle = C.c_void_p()
        _check(lib.rdb_octree_build(_ptr(img), lay, w, h, 0, int(max_colors),
                                    int(associate_alpha), int(grayscale), C.byref(self.handle)))
        self.associate_alpha = bool(associate_alpha)
        self.grayscale = bool(grayscale)

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.rdb_octree_free(self.handle)
            self.handle = None

    @property
    def count(self) -> int:
        return load().rdb_octree_color_count(self.handle)

    @property
    def depth(self) -> int:
        return load().rdb_octree_depth(self.handle)

    def colormap(self) -> np.ndarray:
        out = np.zeros((max(self.count, 1), 4), np.float64)
        load().rdb_octree_colormap(self.handle, _ptr(out))
        return out[: self.count]

    def nodes(self):
        n = load().rdb_octree_node_count(self.handle)
        child = np.zeros((n, 16), np.int32)
        parent = np.zeros(n, np.int32)
        cn = np.zeros(n, np.uint32)
        nu = np.zeros(n, np.uint64)
        load().rdb_octree_nodes(self.handle, _ptr(child), _ptr(parent), _ptr(cn), _ptr(nu))
        return child, parent, cn, nu


class Context:
    """A device context (rdb_context): resident palettes, orders, memo slabs."""

    def __init__(self, device: int = 0, budget: int = 0):
        lib = load()
        self.handle = C.c_void_p()
        _check(lib.rdb_context_create(device, budget, C.byref(self.handle)))
        self.device = device

    def close(self):
        if self.handle:
            load().rdb_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.rdb_context_destroy(self.handle)
            self.handle = None

    @property
    def bytes(self) -> int:
        return load().rdb_context_bytes(self.handle)

    @property
    def last_passes(self) -> int:
        """Passes the last segmented sequential walk took."""
        return load().rdb_context_last_passes(self.handle)

    @property
    def last_sweeps(self) -> tuple[int, bool]:
        """(sweeps, converged) of the last block-sweep approximation."""
        conv = C.c_int(0)
        n = load().rdb_context_last_sweeps(self.handle, C.byref(conv))
        return n, bool(conv.value)

    def dump_indices(self, prefix: str | None) -> None:
        """rdb_context_dump_indices: block walks write `<prefix>.idx.bin`."""
        _check(load().rdb_context_dump_indices(self.handle, (prefix or "").encode()))

    def profile(self, enable: bool = True) -> None:
        """Turns the walk-kernel counters on or off (and clears them)."""
        _check(load().rdb_context_profile(self.handle, int(enable)))

    def stats(self) -> dict:
        st = KernelStats()
        _check(load().rdb_context_stats(self.handle, C.byref(st)))
        return {f: getattr(st, f) for f, _ in KernelStats._fields_}

    # -- palettes ---------------------------------------------------------
    def octree_device(self, pixels: int, layout: int, width: int, height: int, max_colors: int,
                      associate_alpha: bool = False, grayscale: bool = False, row_stride: int = 0,
                      stream: int | None = None) -> tuple[Octree, int]:
        """rdb_octree_build_device: the palette build of an image in device
        memory (`pixels` a device pointer).  Returns the tree and how many rows
        the device classified."""
        t = Octree(None)
        rows = C.c_int(0)
        _check(load().rdb_octree_build_device(self.handle, pixels, layout, width, height, row_stride,
                                              int(max_colors), int(associate_alpha), int(grayscale),
                                              stream or None, C.byref(t.handle), C.byref(rows)))
        t.associate_alpha = bool(associate_alpha)
        t.grayscale = bool(grayscale)
        return t, rows.value

    def palette_from_octree(self, tree: Octree) -> int:
        pid = C.c_int()
        _check(load().rdb_palette_from_octree(self.handle, tree.handle, C.byref(pid)))
        return pid.value

    def palette(self, colors: np.ndarray, child: np.ndarray, color_number: np.ndarray,
                number_unique: np.ndarray, associate_alpha: bool,
                parent: np.ndarray | None = None, search_colors: np.ndarray | None = None,
                root: int = 0) -> int:
        d, keep = _desc(colors, child, color_number, number_unique, associate_alpha, parent,
                        search_colors, root)
        pid = C.c_int()
        _check(load().rdb_palette_create(self.handle, C.byref(d), C.byref(pid)))
        del keep
        return pid.value

    def palette_from_image(self, img: np.ndarray, max_colors: int, **kw) -> int:
        return self.palette_from_octree(Octree(img, max_colors, **kw))

    def release_palette(self, pid: int) -> None:
        _check(load().rdb_palette_destroy(self.handle, pid))

    def uniform_table(self, pid: int, alpha: bool = False) -> np.ndarray:
        """The palette's uniform-key table: 2^18 bytes (2^24 for a palette that
        associates alpha), 255 = not uniform."""
        out = np.empty(1 << (24 if alpha else 18), np.uint8)
        _check(load().rdb_palette_uniform(self.handle, pid, _ptr(out), out.nbytes))
        return out

    # -- dithering (host buffers) ----------------------------------------
    def dither_host(self, engine: str | int, images, palette_ids, rgba: bool = False,
                    **opts):
        """Dithers host images; returns a list of index maps (and RgbaF results)."""
        eng = ENGINES[engine] if isinstance(engine, str) else engine
        if isinstance(images, np.ndarray):
            images, palette_ids = [images], [palette_ids]
            single = True
        else:
            single = False
        n = len(images)
        jobs = (HostJob * n)()
        outs, rgbs, keep = [], [], []
        for i, (img, pid) in enumerate(zip(images, palette_ids)):
            img = np.ascontiguousarray(img)
            keep.append(img)
            h, w = img.shape[:2]
            idx = np.zeros((h, w), np.uint8)
            outs.append(idx)
            jobs[i].pixels = _ptr(img)
            jobs[i].row_stride = 0
            jobs[i].width = w
            jobs[i].height = h
            jobs[i].layout = layout_of(img)
            jobs[i].palette_id = pid
            jobs[i].indices = _ptr(idx)
            if rgba:
                r = np.zeros((h, w, 4), np.float32)
                rgbs.append(r)
                jobs[i].rgba_out = _ptr(r)
        o = options(**opts)
        _check(load().rdb_dither_host(self.handle, eng, jobs, n, C.byref(o)))
        if single:
            return (outs[0], rgbs[0]) if rgba else outs[0]
        return (outs, rgbs) if rgba else outs

    def dither_host_into(self, engine: str | int, img: np.ndarray, palette_id: int,
                         indices: np.ndarray, rgba_out: np.ndarray | None = None, **opts) -> None:
        """Host form for one image into caller-owned (e.g. pinned) buffers."""
        eng = ENGINES[engine] if isinstance(engine, str) else engine
        h, w = img.shape[:2]
        if indices.shape[:2] != (h, w) or indices.dtype != np.uint8 or not indices.flags.c_contiguous:
            raise ValueError("indices must be a contiguous uint8 HxW array")
        job = HostJob()
        job.pixels = _ptr(img)
        job.row_stride = img.strides[0]
        job.width = w
        job.height = h
        job.layout = layout_of(img)
        job.palette_id = palette_id
        job.indices = _ptr(indices)
        if rgba_out is not None:
            job.rgba_out = _ptr(rgba_out)
        o = options(**opts)
        _check(load().rdb_dither_host(self.handle, eng, C.byref(job), 1, C.byref(o)))

    def dither_frames_host(self, frames, in_format: int, width: int, height: int,
                           palette_id: int, out_format: int, indices: bool = False,
                           out=None, **opts):
        """Video frames through the blocks engine (rdb_dither_frames_host):
        `frames` holds F packed frames of `in_format` (any array whose bytes
        are F * frame_bytes(in_format)); returns the F output frames as a
        uint8 array (F, frame_bytes(out_format)) -- or fills `out` -- and,
        with indices=True, the (F, height, width) index maps."""
        buf = np.ascontiguousarray(frames)
        in_bytes = frame_bytes(in_format, width, height)
        out_bytes = frame_bytes(out_format, width, height)
        if in_bytes == 0 or out_bytes == 0 or buf.nbytes % in_bytes:
            raise ValueError("frames do not hold whole frames of the format")
        nf = buf.nbytes // in_bytes
        if out is None:
            out = np.zeros((nf, out_bytes), np.uint8)
        elif out.nbytes != nf * out_bytes or not out.flags.c_contiguous:
            raise ValueError("out must be contiguous and hold every output frame")
        f = Frames()
        f.inp = _ptr(buf)
        f.in_format = in_format
        f.width = width
        f.height = height
        f.frames = nf
        f.palette_id = palette_id
        f.out_format = out_format
        f.out = _ptr(out)
        idx = np.zeros((nf, height, width), np.uint8) if indices else None
        f.indices = _ptr(idx) if indices else 0
        o = options(**opts)
        _check(load().rdb_dither_frames_host(self.handle, C.byref(f), C.byref(o)))
        return (out, idx) if indices else out

    def dither_frames(self, inp: int, in_format: int, width: int, height: int, frames: int,
                      palette_id: int, out: int, out_format: int, indices: int = 0,
                      in_frame_bytes: int = 0, out_frame_bytes: int = 0,
                      stream: int | None = None, **opts) -> None:
        """Device-pointer form (rdb_dither_frames), asynchronous on `stream`."""
        f = Frames()
        f.inp = inp
        f.in_frame_bytes = in_frame_bytes
        f.in_format = in_format
        f.width = width
        f.height = height
        f.frames = frames
        f.palette_id = palette_id
        f.out_format = out_format
        f.out = out
        f.out_frame_bytes = out_frame_bytes
        f.indices = indices
        o = options(**opts)
        _check(load().rdb_dither_frames(self.handle, C.byref(f), C.byref(o), stream or None))

    # -- dithering (device buffers; torch tensors as plumbing) ------------
    def dither(self, engine: str | int, jobs: list[dict], stream: int | None = None,
               **opts) -> None:
        """Enqueue jobs whose buffers are device pointers: dicts with keys
        pixels, width, height, layout, palette_id, indices, optional rgba_out
        and row_stride.  `stream` is a cudaStream_t handle (e.g. a
        torch.cuda.Stream's ``cuda_stream``); None (or the null handle) means the
        context's own stream."""
        eng = ENGINES[engine] if isinstance(engine, str) else engine
        n = len(jobs)
        arr = (Job * n)()
        for i, j in enumerate(jobs):
            arr[i].pixels = j["pixels"]
            arr[i].row_stride = j.get("row_stride", 0)
            arr[i].width = j["width"]
            arr[i].height = j["height"]
            arr[i].layout = j["layout"]
            arr[i].palette_id = j["palette_id"]
            arr[i].indices = j["indices"]
            arr[i].rgba_out = j.get("rgba_out") or 0
        o = options(**opts)
        _check(load().rdb_dither(self.handle, eng, arr, n, C.byref(o), stream or None))

    def synchronize(self, stream: int | None = None) -> None:
        _check(load().rdb_synchronize(self.handle, stream or None))


def _desc(colors, child, color_number, number_unique, associate_alpha, parent=None,
          search_colors=None, root=0):
    colors = np.ascontiguousarray(colors, np.float64)
    child = np.ascontiguousarray(child, np.int32)
    cn = np.ascontiguousarray(color_number, np.uint32)
    nu = np.ascontiguousarray(number_unique, np.uint64)
    keep = [colors, child, cn, nu]
    d = PaletteDesc()
    d.count = colors.shape[0]
    d.associate_alpha = int(associate_alpha)
    d.colors = _ptr(colors)
    if search_colors is not None:
        sc = np.ascontiguousarray(search_colors, np.float64)
        keep.append(sc)
        d.search_colors = _ptr(sc)
    d.node_count = child.shape[0]
    d.root = root
    d.child = _ptr(child)
    if parent is not None:
        par = np.ascontiguousarray(parent, np.int32)
        keep.append(par)
        d.parent = _ptr(par)
    d.color_number = _ptr(cn)
    d.number_unique = _ptr(nu)
    return d, keep


def plan_blob(colors, child, color_number, number_unique, associate_alpha, parent=None,
              search_colors=None, root=0) -> bytes:
    """The device plan for a palette (rdb_plan_build), built on the host."""
    d, keep = _desc(colors, child, color_number, number_unique, associate_alpha, parent,
                    search_colors, root)
    size = C.c_size_t()
    _check(load().rdb_plan_build(C.byref(d), None, 0, C.byref(size)))
    buf = np.zeros(size.value, np.uint8)
    _check(load().rdb_plan_build(C.byref(d), _ptr(buf), size.value, C.byref(size)))
    del keep
    return buf.tobytes()


def probe_latency(device: int = 0) -> dict:
    """rdb_probe_latency: the measured dependent-latency table (cycles)."""
    t = LatencyTable()
    _check(load().rdb_probe_latency(device, C.byref(t)))
    return {f: getattr(t, f) for f, _ in LatencyTable._fields_}


def device_count() -> int:
    c = C.c_int()
    rc = load().rdb_device_count(C.byref(c))
    return c.value if rc == 0 else 0


def error_weights() -> np.ndarray:
    w = np.zeros(16, np.float64)
    load().rdb_error_weights(_ptr(w))
    return w


def inverse_filter(taps: int, diffusion: float = 1.0) -> np.ndarray:
    g = np.zeros(taps + 1, np.float64)
    _check(load().rdb_inverse_filter(taps, diffusion, _ptr(g)))
    return g


def write_palette_text(colors: np.ndarray, path: str) -> None:
    """rdither's palette text file (rdb_palette_write_text): `colors` is
    (count, 4) Q16 r, g, b, a."""
    c = np.ascontiguousarray(colors, np.float64).reshape(-1, 4)
    _check(load().rdb_palette_write_text(_ptr(c), c.shape[0], path.encode()))


def read_palette_text(path: str, expect_colors: int = 0) -> tuple[Octree, bool]:
    """Reads a palette text file (rdb_palette_read_text): the tree built from
    its colours, and whether the file's palette associates alpha."""
    t = Octree(None)
    assoc = C.c_int(0)
    _check(load().rdb_palette_read_text(path.encode(), int(expect_colors), C.byref(t.handle),
                                        C.byref(assoc)))
    return t, bool(assoc.value)


def write_palette_png(colors: np.ndarray, path: str) -> None:
    """rdither's palette image file as PNG (rdb_palette_write_png): a 1 x count
    indexed strip of the 8-bit colours."""
    c = np.ascontiguousarray(colors, np.float64).reshape(-1, 4)
    _check(load().rdb_palette_write_png(_ptr(c), c.shape[0], path.encode()))


def read_palette_png(path: str, expect_colors: int = 0) -> Octree:
    """Reads a palette image file (rdb_palette_read_png): the tree built from
    its colours."""
    t = Octree(None)
    _check(load().rdb_palette_read_png(path.encode(), int(expect_colors), C.byref(t.handle)))
    return t


def write_palette(colors: np.ndarray, path: str) -> None:
    """--palette-export: the text form for .txt / .text paths, else the PNG strip."""
    if path.endswith((".txt", ".text")):
        write_palette_text(colors, path)
    else:
        write_palette_png(colors, path)


def read_palette(path: str, expect_colors: int = 0) -> tuple[Octree, bool]:
    """--palette-from: the text form for .txt / .text paths, else a PNG (an image
    palette never associates alpha)."""
    if path.endswith((".txt", ".text")):
        return read_palette_text(path, expect_colors)
    return read_palette_png(path, expect_colors), False


def frame_bytes(fmt: int, width: int, height: int) -> int:
    """Bytes of one packed frame of `fmt` (0 when unknown or invalid)."""
    return int(load().rdb_frame_bytes(fmt, width, height))


def block_gap(width: int, height: int) -> int:
    return int(load().rdb_block_gap(width, height))


class Server:
    """The request loop (rdb_server_*): submit host images with a colour count
    and an engine from any thread; the server builds palettes on host
    threads, admits by device memory and batches on its device workers."""

    def __init__(self, device: int = 0, budget: int = 0, workers: int = 0, max_batch: int = 0,
                 host_threads: int = 0, device_palettes: bool = False):
        o = ServerOptions(device, budget, workers, max_batch, host_threads, int(device_palettes))
        self.handle = C.c_void_p()
        _check(load().rdb_server_create(C.byref(o), C.byref(self.handle)))
        self._live: dict[int, tuple] = {}

    @staticmethod
    def request_bytes(img: np.ndarray, colors: int, engine: str | int = "seq",
                      alpha: bool = False, rgba: bool = False, device_palettes: bool = False,
                      **opts) -> int:
        """Device bytes a server counts for this request while admitted
        (rdb_request_bytes)."""
        img, r, _, _ = Server._request(img, colors, engine, alpha, rgba, opts)
        return int(load().rdb_request_bytes(C.byref(r), int(device_palettes)))

    @staticmethod
    def _request(img, colors, engine, alpha, rgba, opts):
        # A crop of a larger image is submitted in place (its rows are
        # contiguous; the row stride says how far apart they are).
        if not (img.ndim == 3 and img.strides[2] == img.itemsize and
                img.strides[1] == img.shape[2] * img.itemsize and img.strides[0] > 0):
            img = np.ascontiguousarray(img)
        h, w = img.shape[:2]
        idx = np.empty((h, w), np.uint8)
        out = np.zeros((h, w, 4), np.float32) if rgba else None
        r = Request()
        r.pixels = img.__array_interface__["data"][0]
        r.row_stride = img.strides[0]
        r.width, r.height, r.layout = w, h, layout_of(img)
        r.colors = colors
        r.associate_alpha = int(alpha)
        r.engine = ENGINES[engine] if isinstance(engine, str) else engine
        r.options = options(**opts)
        r.indices = _ptr(idx)
        r.rgba_out = _ptr(out) if out is not None else None
        return img, r, idx, out

    def submit(self, img: np.ndarray, colors: int, engine: str | int = "seq",
               alpha: bool = False, rgba: bool = False, **opts) -> int:
        img, r, idx, out = Server._request(img, colors, engine, alpha, rgba, opts)
        t = C.c_uint64()
        _check(load().rdb_server_submit(self.handle, C.byref(r), C.byref(t)))
        self._live[t.value] = (img, idx, out, r)
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1):
        """(indices, rgba or None, timings dict) of one request."""
        res = RequestResult()
        rc = load().rdb_server_wait(self.handle, ticket, timeout_ms, C.byref(res))
        if rc == 6:  # RDB_E_TIMEOUT: still running, buffers stay alive
            raise TimeoutError(ticket)
        _, idx, out, _ = self._live.pop(ticket)
        _check(rc)
        return idx, out, {f: getattr(res, f) for f, _ in RequestResult._fields_}

    def stats(self) -> dict:
        st = ServerStats()
        _check(load().rdb_server_stats_get(self.handle, C.byref(st)))
        out = {f: getattr(st, f) for f, _ in ServerStats._fields_}
        out["stages"] = {name: {"p50_ms": st.stage_p50_ms[i], "p99_ms": st.stage_p99_ms[i]}
                         for i, name in enumerate(SERVER_STAGES)}
        del out["stage_p50_ms"], out["stage_p99_ms"]
        return out

    def reset_stats(self) -> None:
        _check(load().rdb_server_stats_reset(self.handle))

    def close(self) -> None:
        if self.handle:
            load().rdb_server_destroy(self.handle)
            self.handle = None
            self._live.clear()

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.rdb_server_destroy(self.handle)
            self.handle = None
