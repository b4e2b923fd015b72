"""Batched uneven 3D transforms (fftb_batch_* of include/fftb.h) and their sharding.

:class:`Batch` packs many 3D transforms of different (nx, ny, nz) into flat device
arrays and runs them either one transform after another (mode 0), in one
persistent launch (mode 1), in that launch replayed from a CUDA graph (mode 2), or as
one plain launch per (stage, line length) group (mode 3; mode 4 replays those from a
CUDA graph).

:func:`partition_lpt` splits a batch over GPUs for the multi-GPU form: the
transforms are independent, so each rank takes a subset (greedy longest-
processing-time on the algorithmic bytes of each transform) and runs it on its own
GPU with no collective on the data path.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _check, _dtype_code, _lib, _ptr, _stream_ptr

FORWARD, BACKWARD, ROUNDTRIP, POISSON = 0, 1, 2, 3
SEQUENTIAL, PERSISTENT, GRAPH, GROUPED, GROUPED_GRAPH = 0, 1, 2, 3, 4


def transform_bytes(shape, real_bytes=4) -> int:
    """Algorithmic bytes of one R2C + C2R round trip of a real shape (nx, ny, nz)."""
    nx, ny, nz = shape
    n = nx * ny * nz
    nc = nx * ny * (nz // 2 + 1)
    return 2 * (real_bytes * n + 2 * real_bytes * nc)


def partition_lpt(shapes, nranks: int):
    """Greedy longest-processing-time split of transform indices over nranks, balancing
    the algorithmic bytes.  Returns one sorted index list per rank."""
    order = sorted(range(len(shapes)), key=lambda i: -transform_bytes(shapes[i]))
    load = [0] * nranks
    parts = [[] for _ in range(nranks)]
    for i in order:
        r = min(range(nranks), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += transform_bytes(shapes[i])
    return [sorted(p) for p in parts]


def draw_shapes(count=512, seed=2, sizes=(32, 48, 64, 96, 128)):
    """The batched workload's shapes: each axis length drawn from `sizes` with
    numpy default_rng(seed) (non-cubic shapes allowed)."""
    rng = np.random.default_rng(seed)
    return [tuple(int(v) for v in rng.choice(sizes, size=3)) for _ in range(count)]


class Batch:
    def __init__(self, shapes, dtype="float32"):
        L = _lib.load()
        self.shapes = [tuple(int(v) for v in s) for s in shapes]
        self.dtype = _dtype_code(dtype)
        dims = (ctypes.c_longlong * (3 * len(self.shapes)))(*[v for s in self.shapes for v in s])
        h = ctypes.c_void_p()
        _check(L.fftb_batch_create(self.dtype, len(self.shapes), dims, ctypes.byref(h)), "fftb_batch_create")
        self._h = h
        n = len(self.shapes)
        ro = (ctypes.c_longlong * n)()
        so = (ctypes.c_longlong * n)()
        rt, st = ctypes.c_longlong(), ctypes.c_longlong()
        _check(L.fftb_batch_layout(h, ro, so, ctypes.byref(rt), ctypes.byref(st)), "fftb_batch_layout")
        self.real_offsets = list(ro)
        self.spectrum_offsets = list(so)
        self.real_total = rt.value
        self.spectrum_total = st.value
        self._work = None
        self.mode = GROUPED_GRAPH

    def __del__(self):
        h = getattr(self, "_h", None)
        try:
            if h is not None and h.value:
                _lib.load().fftb_batch_destroy(h)
        except Exception:
            pass
        self._h = None

    def set_work_area(self, tensor):
        self._work = tensor
        _check(_lib.load().fftb_batch_set_work_area(self._h, _ptr(tensor)), "set_work_area")

    def set_tuning(self, tiles_scale=1, ctas_per_sm=0):
        _check(_lib.load().fftb_batch_set_tuning(self._h, int(tiles_scale), int(ctas_per_sm)), "set_tuning")

    def apply_config(self, config) -> int:
        """Applies a tuned config's knobs; returns its execution mode."""
        from . import autotune as _at
        text = config if isinstance(config, str) else _at.to_text(config)
        m = ctypes.c_int()
        _check(_lib.load().fftb_batch_apply_config(self._h, text.encode(), ctypes.byref(m)), "apply_config")
        self.mode = m.value
        return m.value

    def autotune(self, op, cache_file, options=None, measured=None, sign=-1.0):
        """load_or_measure of the execution mode and tiling for op; the winner is applied
        and its mode becomes the default of :meth:`exec`.  Returns the selected config."""
        from . import autotune as _at
        opts = options or _at.autotune_options()
        opts.cache_file = str(cache_file)
        sel, mode = _at.autotune_batch(self, op, opts, measured, sign)
        self.mode = mode
        return sel

    def exec(self, op, inp, out, sign=-1.0, mode=None, stream=None):
        """mode: SEQUENTIAL, PERSISTENT, GRAPH, GROUPED or GROUPED_GRAPH; None takes the
        tuned mode (GROUPED_GRAPH if the batch was never tuned)."""
        if mode is None:
            mode = self.mode
        L = _lib.load()
        _check(L.fftb_batch_set_stream(self._h, _stream_ptr(stream)), "set_stream")
        _check(L.fftb_batch_exec(self._h, int(op), _ptr(inp), _ptr(out), float(sign), int(mode)), "fftb_batch_exec")

    def status(self, op) -> int:
        v = ctypes.c_int()
        _check(_lib.load().fftb_batch_status(self._h, int(op), ctypes.byref(v)), "fftb_batch_status")
        return v.value

    def set_wait_limit(self, polls: int = 0):
        """Polls a dependency wait of the persistent launch makes before the error flag
        (0: the default, about half a second)."""
        _check(_lib.load().fftb_batch_set_wait_limit(self._h, int(polls)), "fftb_batch_set_wait_limit")

    def describe(self, op, sign=-1.0) -> dict:
        vals = [ctypes.c_int() for _ in range(4)]
        _check(_lib.load().fftb_batch_describe(self._h, int(op), float(sign), *[ctypes.byref(v) for v in vals]),
               "fftb_batch_describe")
        return dict(zip(("passes", "items", "grid", "persistent"), [v.value for v in vals]))

    # ------------------------------------------------------------------ packing helpers
    def real_view(self, packed, i):
        nx, ny, nz = self.shapes[i]
        o = self.real_offsets[i]
        return packed[o:o + nx * ny * nz].view(nx, ny, nz)

    def spectrum_view(self, packed, i):
        nx, ny, nz = self.shapes[i]
        o = self.spectrum_offsets[i]
        return packed[o:o + nx * ny * (nz // 2 + 1)].view(nx, ny, nz // 2 + 1)

    def algorithmic_bytes(self) -> int:
        rb = 4 if self.dtype == 0 else 8
        return sum(transform_bytes(s, rb) for s in self.shapes)


def wait_selftest(polls: int = 1000) -> int:
    """Runs the persistent kernel on a work list whose dependency can never be met; its
    bounded wait must give up after `polls` polls and raise the error flag (returned, 1)."""
    v = ctypes.c_int()
    _check(_lib.load().fftb_batch_wait_selftest(int(polls), ctypes.byref(v)), "fftb_batch_wait_selftest")
    return v.value
