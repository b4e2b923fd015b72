"""Build recipe for the FP64 oracle (test infrastructure only).

Compiles ``oracle/fft_oracle.c`` with gcc into ``oracle/_build/liboracle.so``.

The reference itself is not compiled here: every header on its transform path
includes the SCFD submodule (reference ``source/ffts.hpp:15-17``), which is an
empty directory in the reference tree, and its FFT arithmetic is cuFFT, a closed
library.  ``oracle/_ref`` therefore stays empty.
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(force: bool = False) -> str:
    out_dir = os.path.join(HERE, "_build")
    os.makedirs(out_dir, exist_ok=True)
    src = os.path.join(HERE, "fft_oracle.c")
    out = os.path.join(out_dir, "liboracle.so")
    if not force and os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(src):
        return out
    cmd = ["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-Wall", "-o", out + ".tmp", src, "-lm"]
    subprocess.check_call(cmd)
    os.replace(out + ".tmp", out)
    return out


if __name__ == "__main__":
    print(build(force=True))
