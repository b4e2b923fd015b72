"""CPU tests of the C-ABI library: it loads, exports every symbol include/fftb.h
declares, and rejects invalid arguments before touching the GPU."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    from fftm_b200 import build
    build.build()
    from fftm_b200 import _lib
    return _lib.load()


def _declared():
    names = []
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            src = open(os.path.join(inc, f)).read()
            names += re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(fftb_\w+)\s*\(", src, re.M)
    return sorted(set(names))


def test_every_declared_symbol_is_exported(lib):
    names = _declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n


def test_python_binding_covers_header():
    from fftm_b200 import _lib
    assert set(_declared()) <= set(_lib.EXPORTS) | {"fftb_last_error_message"}


def test_version_and_status_strings(lib):
    from fftm_b200 import _lib
    assert re.match(r"\d+\.\d+\.\d+", lib.fftb_version().decode())
    assert _lib.status_string(0) == "success"
    assert "init" in _lib.status_string(-8)
    assert _lib.status_string(-1234) == "unknown status"


def test_library_digest_matches_the_sources(lib):
    from fftm_b200 import build
    assert lib.fftb_build_digest().decode() == build.source_digest()


def test_invalid_plan_arguments_rejected_without_gpu(lib):
    h = ctypes.c_void_p()
    ws = ctypes.c_size_t()
    n = (ctypes.c_longlong * 3)(8, 8, 8)
    # rank 0, rank 4, bad direction, bad dtype, batch 0: all FFTB_ERROR_INVALID_VALUE
    assert lib.fftb_plan_create(1, 0, 0, n, None, 1, 0, None, 1, 0, 1, ctypes.byref(h), ctypes.byref(ws)) == -1
    assert lib.fftb_plan_create(1, 0, 4, n, None, 1, 0, None, 1, 0, 1, ctypes.byref(h), ctypes.byref(ws)) == -1
    assert lib.fftb_plan_create(9, 0, 3, n, None, 1, 0, None, 1, 0, 1, ctypes.byref(h), ctypes.byref(ws)) == -1
    assert lib.fftb_plan_create(1, 7, 3, n, None, 1, 0, None, 1, 0, 1, ctypes.byref(h), ctypes.byref(ws)) == -1
    assert lib.fftb_plan_create(1, 0, 3, n, None, 1, 0, None, 1, 0, 0, ctypes.byref(h), ctypes.byref(ws)) == -1
    bad = (ctypes.c_longlong * 3)(8, 0, 8)
    assert lib.fftb_plan_create(1, 0, 3, bad, None, 1, 0, None, 1, 0, 1, ctypes.byref(h), ctypes.byref(ws)) == -1
    assert lib.fftb_exec(None, None, None) == -5
    assert lib.fftb_plan_destroy(None) == -5


def test_invalid_ffts_arguments_rejected_without_gpu(lib):
    h = ctypes.c_void_p()
    assert lib.fftb_ffts_create(0, 0, 8, 8, 0, 0, ctypes.byref(h)) == -1
    assert lib.fftb_ffts_create(3, 8, 8, 8, 0, 0, ctypes.byref(h)) == -1
    assert lib.fftb_ffts_create(0, 8, 8, 0, 8, 0, ctypes.byref(h)) == -1
    assert lib.fftb_ffts_forward(None, None, None) == -5
    assert lib.fftb_ffts_destroy(None) == -5


def test_python_frontend_logic_errors_without_gpu():
    import fftm_b200 as F
    f = F.ffts("float32")
    with pytest.raises(F.LogicError):
        f.dimension()
    assert not f.is_initialized()
    w = F.fft_wrap_many("float32")
    w.activate()
    with pytest.raises(F.LogicError):
        w.add_plan_1D(F.C2CF, "x", 8, 8, 1, 8, 8, 1, 8, 1)
    with pytest.raises(KeyError):
        w.exec("missing", None, None)


def test_library_has_no_cufft_dependency(lib):
    # the product path links no cuFFT (the oracle/baseline harness is the only cuFFT user)
    import subprocess
    from fftm_b200 import _lib
    out = subprocess.run(["ldd", _lib.LIB_PATH], capture_output=True, text=True).stdout
    assert "cufft" not in out


def _build_cpp_example(lib_path, exe):
    """Compiles tests/cpp_api_example.cpp against include/fftb.hpp and links it to the
    library (g++, C++17)."""
    import subprocess
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    libdir = os.path.dirname(lib_path)
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-o", str(exe),
           os.path.join(ROOT, "tests", "cpp_api_example.cpp"), "-I" + os.path.join(ROOT, "include"),
           "-I" + os.path.join(cuda, "include"), "-L" + libdir, "-lfftb_b200", "-L" + os.path.join(cuda, "lib64"),
           "-lcudart", "-Wl,-rpath," + libdir + ":" + os.path.join(cuda, "lib64")]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


def test_cpp_header_layer_host_checks(lib, tmp_path):
    # include/fftb.hpp compiles warning-free and its host-side logic (status -> exception
    # mapping, KEY=VALUE text, option flags) runs without a GPU
    import subprocess
    from fftm_b200 import _lib
    exe = tmp_path / "cpp_api_example"
    _build_cpp_example(_lib.LIB_PATH, exe)
    p = subprocess.run([str(exe), "--host-only"], capture_output=True, text=True, timeout=60)
    assert p.returncode == 0, p.stdout + p.stderr
    assert p.stdout.strip().endswith("ok")
    assert "FAIL" not in p.stdout
