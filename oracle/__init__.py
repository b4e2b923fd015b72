"""FP64 CPU oracle for the single-GPU transform path (test infrastructure only).

This package is the checker for the CUDA library in ``fftm_b200``: only the
tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use
it.  The product never imports it.

It wraps ``oracle/fft_oracle.c`` (built to ``oracle/_build/liboracle.so`` by
``oracle.build.build()``), a double-precision restatement of the transforms that
fftm's ``ffts`` frontend performs through cuFFT: the ``ffts`` 2D/3D plans
(reference ``source/ffts.hpp:659-695``), the 4D pencil and slab pipelines
(``source/ffts.hpp:697-867``), the fftm 4D ``native_xzwy`` spectrum
(``source/fftm.hpp:2941-2961``), the Poisson multiply and the reference tests'
splitmix64 input generator (``source/tests/detail/fft_benchmark_common.h:201-257``).
Its header in ``fft_oracle.c`` lists how each part is pinned.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")

R2C, C2R, C2CF, C2CB = 1, 2, 3, 4          # source/fft_direction.h:9-15
PENCIL, SLAB, NATIVE_XZWY = 0, 1, 2        # 4D layouts

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build as _b
            _b.build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        lp = ctypes.POINTER(ctypes.c_long)
        c_l, c_u64, c_i = ctypes.c_long, ctypes.c_uint64, ctypes.c_int
        L.orc_exec.argtypes = [c_i, c_i, lp, lp, c_l, c_l, lp, c_l, c_l, c_l, dp, dp]
        L.orc_exec.restype = c_i
        L.orc_fill_random_3d.argtypes = [dp, c_l, c_l, c_l, c_l, c_l, c_l, c_u64, c_i]
        L.orc_fill_random_4d.argtypes = [dp, c_l, c_l, c_l, c_l, c_l, c_l, c_l, c_l, c_u64, c_i]
        for f in ("orc_ffts3d_forward", "orc_ffts3d_backward"):
            getattr(L, f).argtypes = [c_l, c_l, c_l, dp, dp]
            getattr(L, f).restype = c_i
        for f in ("orc_ffts2d_forward", "orc_ffts2d_backward"):
            getattr(L, f).argtypes = [c_l, c_l, dp, dp]
            getattr(L, f).restype = c_i
        for f in ("orc_ffts4d_forward", "orc_ffts4d_backward"):
            getattr(L, f).argtypes = [c_i, c_l, c_l, c_l, c_l, dp, dp]
            getattr(L, f).restype = c_i
        L.orc_poisson3d.argtypes = [c_l, c_l, c_l, ctypes.c_double, dp]
        L.orc_poisson4d.argtypes = [c_i, c_l, c_l, c_l, c_l, ctypes.c_double, dp]
        L.orc_splitmix64.argtypes = [c_u64]
        L.orc_splitmix64.restype = c_u64
        L.orc_set_threads.argtypes = [c_i]
        L.orc_get_max_threads.restype = c_i
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def max_threads() -> int:
    return int(lib().orc_get_max_threads())


def _dp(a: np.ndarray):
    assert a.dtype in (np.float64, np.complex128) and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _lp(v):
    if v is None:
        return None
    arr = (ctypes.c_long * len(v))(*[int(x) for x in v])
    return arr


def splitmix64(x: int) -> int:
    return int(lib().orc_splitmix64(ctypes.c_uint64(x & 0xFFFFFFFFFFFFFFFF)))


# ------------------------------------------------------------------ generators
def random_3d(nx, ny, nz, seed, single=True) -> np.ndarray:
    """fill_random_real_3d_functor over logical (x,y,z), stored [x][y][z]
    (reference source/tests/detail/fft_benchmark_common.h:219-237)."""
    a = np.empty((nx, ny, nz), np.float64)
    lib().orc_fill_random_3d(_dp(a), nx, ny, nz, ny * nz, nz, 1, ctypes.c_uint64(seed), int(single))
    return a


def random_4d(nx, ny, nz, nw, seed, layout=SLAB, single=True) -> np.ndarray:
    """fill_random_real_4d_functor over logical (x,y,z,w) (fft_benchmark_common.h:239-257).
    Stored [w][z][y][x] for the pencil layout, [x][y][z][w] otherwise."""
    if layout == PENCIL:
        a = np.empty((nw, nz, ny, nx), np.float64)
        sx, sy, sz, sw = 1, nx, nx * ny, nx * ny * nz
    else:
        a = np.empty((nx, ny, nz, nw), np.float64)
        sx, sy, sz, sw = ny * nz * nw, nz * nw, nw, 1
    lib().orc_fill_random_4d(_dp(a), nx, ny, nz, nw, sx, sy, sz, sw, ctypes.c_uint64(seed), int(single))
    return a


# ------------------------------------------------------------------ plans
def exec_plan(direction, n, inembed, istride, idist, onembed, ostride, odist, batch, inp, out_size):
    """One BaseFFT plan execution with cuFFT advanced-layout addressing
    (reference source/external_wrap/fft_wrap_many.h:137-186, :375-383).
    ``inp`` is float64 (real) or complex128; returns a flat output of ``out_size``
    elements (float64 for C2R, complex128 otherwise)."""
    rank = len(n)
    inp = np.ascontiguousarray(inp)
    if direction == C2R:
        out = np.zeros(out_size, np.float64)
    else:
        out = np.zeros(out_size, np.complex128)
    if direction in (C2R, C2CF, C2CB):
        inp = inp.astype(np.complex128, copy=True)
    else:
        inp = inp.astype(np.float64, copy=True)
    rc = lib().orc_exec(direction, rank, _lp(n), _lp(inembed), istride, idist, _lp(onembed), ostride, odist,
                        batch, _dp(inp), _dp(out))
    if rc != 0:
        raise RuntimeError(f"oracle exec failed: {rc}")
    return out


def ffts3d_forward(x: np.ndarray) -> np.ndarray:
    """ffts::forward 3D (source/ffts.hpp:356-361): real [x][y][z] -> [kx][ky][kz<nz/2+1]."""
    nx, ny, nz = x.shape
    x = np.ascontiguousarray(x, np.float64)
    out = np.zeros((nx, ny, nz // 2 + 1), np.complex128)
    assert lib().orc_ffts3d_forward(nx, ny, nz, _dp(x), _dp(out)) == 0
    return out


def ffts3d_backward(X: np.ndarray, nz: int) -> np.ndarray:
    """ffts::backward 3D (source/ffts.hpp:363-368), unnormalised."""
    nx, ny, _ = X.shape
    X = np.ascontiguousarray(X, np.complex128).copy()
    out = np.zeros((nx, ny, nz), np.float64)
    assert lib().orc_ffts3d_backward(nx, ny, nz, _dp(X), _dp(out)) == 0
    return out


def ffts2d_forward(x):
    nx, ny = x.shape
    x = np.ascontiguousarray(x, np.float64)
    out = np.zeros((nx, ny // 2 + 1), np.complex128)
    assert lib().orc_ffts2d_forward(nx, ny, _dp(x), _dp(out)) == 0
    return out


def ffts2d_backward(X, ny):
    nx = X.shape[0]
    X = np.ascontiguousarray(X, np.complex128).copy()
    out = np.zeros((nx, ny), np.float64)
    assert lib().orc_ffts2d_backward(nx, ny, _dp(X), _dp(out)) == 0
    return out


def spectrum_shape_4d(layout, nx, ny, nz, nw):
    nwh = nw // 2 + 1
    if layout == SLAB:
        return (nx, ny, nz, nwh)
    return (ny, nz, nwh, nx)


def ffts4d_forward(layout, x, dims):
    nx, ny, nz, nw = dims
    x = np.ascontiguousarray(x, np.float64)
    out = np.zeros(spectrum_shape_4d(layout, nx, ny, nz, nw), np.complex128)
    assert lib().orc_ffts4d_forward(layout, nx, ny, nz, nw, _dp(x), _dp(out)) == 0
    return out


def ffts4d_backward(layout, X, dims):
    nx, ny, nz, nw = dims
    X = np.ascontiguousarray(X, np.complex128).copy()
    shape = (nw, nz, ny, nx) if layout == PENCIL else (nx, ny, nz, nw)
    out = np.zeros(shape, np.float64)
    assert lib().orc_ffts4d_backward(layout, nx, ny, nz, nw, _dp(X), _dp(out)) == 0
    return out


def poisson3d(spec: np.ndarray, nz: int, sign: float = -1.0) -> np.ndarray:
    nx, ny, _ = spec.shape
    s = np.ascontiguousarray(spec, np.complex128).copy()
    lib().orc_poisson3d(nx, ny, nz, float(sign), _dp(s))
    return s


def poisson4d(layout, spec, dims, sign=-1.0):
    nx, ny, nz, nw = dims
    s = np.ascontiguousarray(spec, np.complex128).copy()
    lib().orc_poisson4d(layout, nx, ny, nz, nw, float(sign), _dp(s))
    return s


def poisson3d_solve(f: np.ndarray, sign: float = -1.0) -> np.ndarray:
    """R2C, multiply by sign/|k|^2 (k=0 -> 0), C2R, 1/N: the MPI-free Poisson
    pipeline of source/tests/test_3D_poisson.cu:229-244 (sign -1 solves lap u = f)."""
    nx, ny, nz = f.shape
    X = ffts3d_forward(f)
    X = poisson3d(X, nz, sign)
    return ffts3d_backward(X, nz) / float(nx * ny * nz)


def poisson4d_solve(layout, f, dims, sign=-1.0):
    nx, ny, nz, nw = dims
    X = ffts4d_forward(layout, f, dims)
    X = poisson4d(layout, X, dims, sign)
    return ffts4d_backward(layout, X, dims) / float(nx * ny * nz * nw)


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.complex128 if np.iscomplexobj(a) or np.iscomplexobj(b) else np.float64)
    b = np.asarray(b, a.dtype)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))
