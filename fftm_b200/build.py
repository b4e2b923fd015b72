"""Builds the fftb CUDA library in-tree for sm_100a.

``python -m fftm_b200.build`` compiles every ``.cu`` source under
``fftm_b200/csrc`` with nvcc (``-gencode arch=compute_100a,code=sm_100a``) into
objects under ``fftm_b200/_build`` and links ``fftm_b200/libfftb_b200.so``
(CUDA runtime linked statically, so the library does not depend on the runtime
version that other libraries in the process load).  The pass kernel is
instantiated in 8 parts per precision so the compiler runs in parallel.
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfftb_b200.so")
NPARTS = 8

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
              "--expt-relaxed-constexpr", f"-DFFTB_NPARTS={NPARTS}"]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else (shutil.which("nvcc") or "nvcc")


def _headers_digest() -> str:
    h = hashlib.sha256()
    for d in (CSRC, os.path.join(ROOT, "include")):
        for root, _, files in os.walk(d):
            for f in sorted(files):
                if f.endswith((".h", ".cuh", ".hpp")):
                    with open(os.path.join(root, f), "rb") as fh:
                        h.update(f.encode())
                        h.update(fh.read())
    return h.hexdigest()


def _jobs():
    jobs = []
    for f in sorted(os.listdir(CSRC)):
        if not f.endswith(".cu"):
            continue
        src = os.path.join(CSRC, f)
        if f == "fftb_pass_inst.cu":
            for real in ("float", "double"):
                for k in range(NPARTS):
                    obj = os.path.join(BUILD, f"pass_{real}_{k}.o")
                    jobs.append((src, obj, [f"-DFFTB_REAL={real}", f"-DFFTB_PART={k}"]))
        else:
            jobs.append((src, os.path.join(BUILD, f[:-3] + ".o"), []))
    return jobs


def _compile(job, digest):
    src, obj, extra = job
    stamp = obj + ".stamp"
    key = digest + "|" + " ".join(extra) + "|" + str(os.path.getmtime(src))
    if os.path.exists(obj) and os.path.exists(stamp) and open(stamp).read() == key:
        return obj, None
    cmd = [nvcc()] + ARCH + NVCC_FLAGS + extra + ["-c", src, "-o", obj]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        return obj, " ".join(cmd) + "\n" + p.stdout + p.stderr
    with open(stamp, "w") as fh:
        fh.write(key)
    return obj, None


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    digest = _headers_digest()
    jobs = _jobs()
    errors = []
    objs = []
    with cf.ThreadPoolExecutor(max_workers=max(2, os.cpu_count() or 2)) as ex:
        for obj, err in ex.map(lambda j: _compile(j, digest), jobs):
            objs.append(obj)
            if err:
                errors.append(err)
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        tmp = LIB + ".tmp"
        cmd = [nvcc()] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", tmp] + objs + ["-lcuda"]
        subprocess.check_call(cmd)
        os.replace(tmp, LIB)
    if verbose:
        print(LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True)
    sys.exit(0)
