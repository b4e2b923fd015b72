"""The reference's cuFFT-backed ``ffts`` path (cufft_ffts.cu), for parity tests and the
benchmark only: the exact cufftMakePlanMany64 plans of source/ffts.hpp:677-776 and
source/fftm.hpp:2941-2961 with auto-allocation off, the stage order and per-element
transposes of source/ffts.hpp:809-867, and the Poisson example's separate multiply and
1/N kernels.  Nothing in the fftb product loads this library.

    python -m cufft_ref.build        (from tests/; also run by __graft_entry__.build())
"""
from __future__ import annotations

import ctypes
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cufft_ffts.cu")
LIB = os.path.join(HERE, "_build", "libcufft_ffts.so")

PENCIL, SLAB, NATIVE_XZWY = 0, 1, 2
_LAYOUT = {"pencil": PENCIL, "slab": SLAB, "native_xzwy": NATIVE_XZWY}


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else (shutil.which("nvcc") or "nvcc")


def build() -> str:
    """Compiles the harness for sm_100a (when the source is newer than the library)."""
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    tmp = LIB + ".tmp"
    cmd = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-shared",
           "-Xcompiler", "-fPIC", "-o", tmp, SRC, "-lcufft"]
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise ImportError(f"{LIB} is missing (run `python -m cufft_ref.build` from tests/)")
        L = ctypes.CDLL(LIB)
        vp, ll, sz = ctypes.c_void_p, ctypes.c_longlong, ctypes.c_size_t
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ll, ll, ll, ll, ctypes.POINTER(vp),
                                 ctypes.POINTER(sz), ctypes.POINTER(sz)]
        L.ref_set_buffers.argtypes = [vp, vp, vp, vp]
        L.ref_set_stream.argtypes = [vp, vp]
        L.ref_forward.argtypes = [vp, vp, vp]
        L.ref_backward.argtypes = [vp, vp, vp]
        L.ref_poisson3d.argtypes = [vp, vp, vp, vp, ctypes.c_double]
        L.ref_scale.argtypes = [vp, vp, ll, ctypes.c_double]
        L.ref_destroy.argtypes = [vp]
        _lib = L
    return _lib


class RefFfts:
    """``fftm::ffts<cufft_wrap_many<T>>`` restated: init(dims) plans, forward, backward
    (unnormalised, destroys its input), and the Poisson example's solve (3D).  Buffers
    (the shared work area and the two 4D stage arrays) are torch tensors it owns."""

    def __init__(self, dtype, dims, layout="pencil", device=None):
        import torch
        self._torch = torch
        L = load()
        self.dims = tuple(int(d) for d in dims)
        self.dtype = dtype
        dt = 0 if dtype in ("float32", torch.float32) else 1
        nx, ny, nz = self.dims[:3]
        nw = self.dims[3] if len(self.dims) == 4 else 0
        h = ctypes.c_void_p()
        wb, sb = ctypes.c_size_t(), ctypes.c_size_t()
        lay = _LAYOUT[layout] if isinstance(layout, str) else int(layout)
        st = L.ref_create(dt, len(self.dims), lay, nx, ny, nz, nw, ctypes.byref(h), ctypes.byref(wb), ctypes.byref(sb))
        if st != 0:
            raise RuntimeError("cuFFT reference: " + L.ref_last_error().decode())
        self._h = h
        dev = device or torch.device("cuda", torch.cuda.current_device())
        self._work = torch.empty(max(1, wb.value), dtype=torch.uint8, device=dev)
        self._s0 = torch.empty(max(1, sb.value), dtype=torch.uint8, device=dev)
        self._s1 = torch.empty(max(1, sb.value), dtype=torch.uint8, device=dev)
        self.work_bytes, self.stage_bytes = wb.value, sb.value
        self._check(L.ref_set_buffers(h, self._work.data_ptr(), self._s0.data_ptr(), self._s1.data_ptr()))
        self.set_stream(torch.cuda.current_stream(dev))

    def _check(self, st):
        if st != 0:
            raise RuntimeError("cuFFT reference: " + load().ref_last_error().decode())

    def set_stream(self, stream):
        self._check(load().ref_set_stream(self._h, stream.cuda_stream))

    def forward(self, x, spec):
        self._check(load().ref_forward(self._h, x.data_ptr(), spec.data_ptr()))

    def backward(self, spec, y):
        self._check(load().ref_backward(self._h, spec.data_ptr(), y.data_ptr()))

    def backward_normalized(self, spec, y):
        """backward, then the callers' separate 1/N kernel."""
        self.backward(spec, y)
        self._check(load().ref_scale(self._h, y.data_ptr(), y.numel(), 1.0 / y.numel()))

    def poisson(self, rhs, spec, out, sign=-1.0):
        self._check(load().ref_poisson3d(self._h, rhs.data_ptr(), spec.data_ptr(), out.data_ptr(), float(sign)))

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                load().ref_destroy(self._h)
                self._h = None
        except Exception:
            pass
