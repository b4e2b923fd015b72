"""The C ABI from a plain C program (tests/c_abi_example.c): compiled with gcc against
include/fftb.h and linked to libfftb_b200.so, it solves a manufactured Poisson problem,
checks a round trip, runs a plan and an error path -- no Python or torch in between.
And the header-only C++ layer (include/fftb.hpp) from tests/cpp_api_example.cpp: plan
registry, ffts 3D / 4D, the reference's exception types, autotune cache, batches."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_c_program_uses_the_abi(tmp_path, torch_cuda):
    from fftm_b200 import build
    lib = build.build()
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    exe = tmp_path / "c_abi_example"
    cmd = ["gcc", "-O2", "-o", str(exe), os.path.join(ROOT, "tests", "c_abi_example.c"),
           "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(cuda, "include"),
           "-L" + os.path.dirname(lib), "-lfftb_b200", "-L" + os.path.join(cuda, "lib64"), "-lcudart", "-lm",
           "-Wl,-rpath," + os.path.dirname(lib) + ":" + os.path.join(cuda, "lib64")]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    p = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    print(p.stdout)
    assert p.returncode == 0, p.stdout + p.stderr
    assert p.stdout.strip().endswith("ok")


def test_cpp_program_uses_the_header_layer(tmp_path, torch_cuda):
    from fftm_b200 import build
    from test_abi import _build_cpp_example
    lib = build.build()
    exe = tmp_path / "cpp_api_example"
    _build_cpp_example(lib, exe)
    p = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=300)
    print(p.stdout)
    assert p.returncode == 0, p.stdout + p.stderr
    assert p.stdout.strip().endswith("ok")
    assert "FAIL" not in p.stdout
