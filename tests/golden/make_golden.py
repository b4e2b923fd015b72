"""Generates the golden fixtures in tests/golden/golden_small.npz.

The reference stores no golden vectors for its transform path (its tests pin
results analytically or by round trip).  These fixtures are produced by an
implementation independent of both the oracle and the CUDA library: numpy's
pocketfft in float64 (``numpy.fft.rfftn`` / ``fftn``), applied to inputs from
the reference tests' own splitmix64 generator
(source/tests/detail/fft_benchmark_common.h:201-257, restated here in plain
Python) and to numpy-seeded inputs.  Spectra are stored in the reference's
physical layouts: 3D [kx][ky][kz<nz/2+1] (source/ffts.hpp:680-686), 4D slab
[kx][ky][kz][kw<nw/2+1] and 4D pencil / native_xzwy [ky][kz][kw<nw/2+1][kx]
(source/ffts.hpp:126-150, source/fftm.hpp:2941-2961).

Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
M64 = (1 << 64) - 1


def splitmix64(x: int) -> int:
    x = (x + 0x9E3779B97F4A7C15) & M64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M64
    return x ^ (x >> 31)


def unit_random_f32(state: int) -> float:
    unit = float(splitmix64(state) >> 11) * (1.0 / 9007199254740992.0)
    u = np.float32(unit)
    return float(np.float32(np.float32(2.0) * u - np.float32(1.0)))


def random_3d(nx, ny, nz, seed):
    a = np.empty((nx, ny, nz))
    for x in range(nx):
        for y in range(ny):
            for z in range(nz):
                st = seed ^ ((x * 0xD6E8FEB86659FD93) & M64) ^ ((y * 0xA5A3564E27F886A5) & M64) ^ \
                    ((z * 0x9E3779B97F4A7C15) & M64)
                a[x, y, z] = unit_random_f32(st)
    return a


def random_4d(nx, ny, nz, nw, seed):
    a = np.empty((nx, ny, nz, nw))
    for x in range(nx):
        for y in range(ny):
            for z in range(nz):
                for w in range(nw):
                    st = seed ^ ((x * 0xD6E8FEB86659FD93) & M64) ^ ((y * 0xA5A3564E27F886A5) & M64) ^ \
                        ((z * 0x9E3779B97F4A7C15) & M64) ^ ((w * 0x94D049BB133111EB) & M64)
                    a[x, y, z, w] = unit_random_f32(st)
    return a


def main():
    out = {}
    seed = 0x1234ABCDEF987654  # source/tests/test_benchmark_ffts_3D.cu:69
    for shape in [(8, 8, 8), (6, 10, 12), (5, 7, 9), (16, 12, 10)]:
        x = random_3d(*shape, seed)
        key = "r3d_" + "x".join(map(str, shape))
        out[key + "_in"] = x
        out[key + "_spec"] = np.fft.rfftn(x)
    x = random_3d(4, 4, 4, seed)
    out["splitmix_first_values"] = x.ravel()[:8]
    # 4D: logical (x,y,z,w)
    dims = (6, 4, 8, 10)
    x = random_4d(*dims, 0xABCDEF0123456789)
    spec = np.fft.rfftn(x)                               # [kx][ky][kz][kw]
    out["r4d_in_xyzw"] = x
    out["r4d_spec_slab"] = spec
    out["r4d_spec_yzwx"] = np.ascontiguousarray(spec.transpose(1, 2, 3, 0))
    # 2D and batched 1D / C2C fixtures from numpy-seeded data
    rng = np.random.default_rng(0)
    x2 = rng.uniform(-1, 1, (12, 20))
    out["r2d_in"] = x2
    out["r2d_spec"] = np.fft.rfftn(x2)
    z = rng.normal(size=(3, 48)) + 1j * rng.normal(size=(3, 48))
    out["c1d_in"] = z
    out["c1d_fwd"] = np.fft.fft(z, axis=-1)
    out["c1d_inv"] = np.fft.ifft(z, axis=-1) * 48
    np.savez_compressed(os.path.join(HERE, "golden_small.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
