"""CPU tests of the autotune cache (C++ in the library, no GPU needed): the KEY=VALUE
file grammar of the reference's cache (source/fftm_autotune.hpp:126-169), the atomic
tmp+rename write, and the identity / hardware validation rules
(source/fftm_autotune.hpp validate_match, source/detail/fftm_autotune_hardware.inc:
"v2:" signatures, strict device identity)."""
import os

import pytest

from fftm_b200 import FftbError


@pytest.fixture(scope="module")
def A():
    from fftm_b200 import build
    build.build()
    import fftm_b200.autotune as A
    return A


CACHE_IO, CACHE_MISMATCH = -11, -12

IDENT = {
    "FFTM_AUTOTUNE_SCHEMA": "2", "FFTM_AUTOTUNE_POLICY_VERSION": "fftb-1", "FFTM_AUTOTUNE_LIBRARY": "fftb",
    "FFTM_AUTOTUNE_DIM": "3", "FFTM_AUTOTUNE_NUM_GPUS": "1", "FFTM_AUTOTUNE_SIZE_3D": "256x256x256",
    "FFTB_AUTOTUNE_DTYPE": "float32",
    "FFTM_AUTOTUNE_HARDWARE_SIGNATURE": "v2:0123456789abcdef",
    "FFTM_AUTOTUNE_HARDWARE_SIGNATURE_STRICT": "v2:fedcba9876543210",
}


def _cache(**over):
    c = dict(IDENT)
    c.update({"FFTM_AUTOTUNE_SOURCE": "fftb-measured-v1", "FFTB_AUTOTUNE_STRATEGY": "fused",
              "FFTB_AUTOTUNE_PLANE_CLUSTER": "2"})
    c.update(over)
    return c


def test_save_load_roundtrip_is_atomic(A, tmp_path):
    p = tmp_path / "fftm_autotune.env"
    cfg = _cache(FFTB_AUTOTUNE_FAILED_x="value with = sign and spaces")
    A.save_key_value_file(p, cfg)
    assert not os.path.exists(str(p) + ".tmp")
    text = open(p).read()
    assert text.startswith("# ")
    assert "FFTM_AUTOTUNE_SCHEMA=2\n" in text
    assert A.load_key_value_file(p) == cfg
    # overwrite in place
    A.save_key_value_file(p, {"K": "v"})
    assert A.load_key_value_file(p) == {"K": "v"}


def test_load_accepts_comments_blank_lines_and_whitespace(A, tmp_path):
    p = tmp_path / "c.env"
    p.write_text("# FFTM C++ autotune cache\n\n  FFTM_AUTOTUNE_SCHEMA = 2 \n\t# x\nFFTM_AUTOTUNE_DIM=3\r\n")
    assert A.load_key_value_file(p) == {"FFTM_AUTOTUNE_SCHEMA": "2", "FFTM_AUTOTUNE_DIM": "3"}


@pytest.mark.parametrize("content", ["# only a comment\n\n", "", "FFTM_AUTOTUNE_DIM=3\nno equals sign\n",
                                     "=value\n"])
def test_load_rejects_malformed(A, tmp_path, content):
    p = tmp_path / "bad.env"
    p.write_text(content)
    with pytest.raises(FftbError) as e:
        A.load_key_value_file(p)
    assert e.value.status == CACHE_IO


def test_malformed_line_number_in_message(A, tmp_path):
    p = tmp_path / "bad.env"
    p.write_text("A=1\nB=2\nbroken\n")
    with pytest.raises(FftbError, match=r"bad\.env:3 is not KEY=VALUE"):
        A.load_key_value_file(p)


def test_load_missing_file_and_unwritable_path(A, tmp_path):
    with pytest.raises(FftbError) as e:
        A.load_key_value_file(tmp_path / "absent.env")
    assert e.value.status == CACHE_IO
    with pytest.raises(FftbError) as e:
        A.save_key_value_file(tmp_path / "no_such_dir" / "c.env", {"K": "v"})
    assert e.value.status == CACHE_IO
    assert not os.path.exists(tmp_path / "no_such_dir")


def test_validate_accepts_matching_cache(A):
    A.validate(_cache(), IDENT)
    # strict identity compares the strict signature too
    A.validate(_cache(), IDENT, A.autotune_options(strict_device_identity=True))


@pytest.mark.parametrize("key,value", [
    ("FFTM_AUTOTUNE_SIZE_3D", "128x128x128"), ("FFTM_AUTOTUNE_SCHEMA", "1"), ("FFTM_AUTOTUNE_DIM", "4"),
    ("FFTB_AUTOTUNE_DTYPE", "float64"), ("FFTM_AUTOTUNE_NUM_GPUS", "2"),
    ("FFTM_AUTOTUNE_POLICY_VERSION", "4"),
])
def test_validate_rejects_other_problem(A, key, value):
    with pytest.raises(FftbError, match=key) as e:
        A.validate(_cache(**{key: value}), IDENT)
    assert e.value.status == CACHE_MISMATCH
    # hardware validation off does not relax the problem identity
    with pytest.raises(FftbError):
        A.validate(_cache(**{key: value}), IDENT, A.autotune_options(validate_hardware=False))


def test_validate_rejects_unmeasured_fftb_cache(A):
    # an fftb cache must come from a measurement
    with pytest.raises(FftbError, match="not a measured"):
        A.validate(_cache(FFTM_AUTOTUNE_SOURCE="cpp-policy-cache-v4"), IDENT)


def _reference_policy_cache(**over):
    # what the reference's make_default_3d_policy_config writes for one rank
    # (source/fftm_autotune.hpp:595-605, :660-681) plus its hardware keys
    c = {"FFTM_AUTOTUNE_SCHEMA": "2", "FFTM_AUTOTUNE_POLICY_VERSION": "4", "FFTM_AUTOTUNE_LIBRARY": "fftm",
         "FFTM_AUTOTUNE_DIM": "3", "FFTM_AUTOTUNE_NUM_GPUS": "1", "FFTM_AUTOTUNE_SIZE_3D": "256x256x256",
         "FFTM_AUTOTUNE_SOURCE": "cpp-policy-cache-v4", "FFTM_AUTOTUNE_STRATEGY_3D": "slab-pencil",
         "FFTM_AUTOTUNE_GRID_3D": "1x1", "FFTM_AUTOTUNE_PENCIL_LAYOUT": "auto",
         "FFTM_AUTOTUNE_PENCIL_PIPELINE": "staged", "FFTM_AUTOTUNE_HARDWARE_SIGNATURE_VERSION": "2",
         "FFTM_AUTOTUNE_HARDWARE_SIGNATURE": IDENT["FFTM_AUTOTUNE_HARDWARE_SIGNATURE"],
         "FFTM_AUTOTUNE_HARDWARE_SIGNATURE_STRICT": IDENT["FFTM_AUTOTUNE_HARDWARE_SIGNATURE_STRICT"]}
    c.update(over)
    return c


def test_validate_accepts_single_gpu_cache_of_the_reference(A):
    A.validate(_reference_policy_cache(), IDENT)
    A.validate(_reference_policy_cache(FFTM_AUTOTUNE_STRATEGY_3D="pencil-slab"), IDENT,
               A.autotune_options(strict_device_identity=True))


@pytest.mark.parametrize("key,value", [("FFTM_AUTOTUNE_SIZE_3D", "128x128x128"), ("FFTM_AUTOTUNE_NUM_GPUS", "4"),
                                       ("FFTM_AUTOTUNE_SCHEMA", "1"), ("FFTM_AUTOTUNE_DIM", "4"),
                                       ("FFTM_AUTOTUNE_HARDWARE_SIGNATURE", "v2:1111111111111111")])
def test_validate_rejects_reference_cache_of_another_problem_or_machine(A, key, value):
    with pytest.raises(FftbError) as e:
        A.validate(_reference_policy_cache(**{key: value}), IDENT)
    assert e.value.status == CACHE_MISMATCH


def test_hardware_signature_follows_the_reference_hash(A):
    # 64-bit FNV-1a of the canonical string, "v2:" + 16 hex digits
    # (source/detail/fftm_autotune_hardware.inc:87-97)
    def fnv(s):
        h = 14695981039346656037
        for ch in s.encode():
            h = ((h ^ ch) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
        return f"{h:016x}"
    assert fnv("") == "cbf29ce484222325"
    canon = ("version=2;mpi_ranks=1;node_count=1;ranks_per_node=1;devices_per_node=1;mpi_library=unavailable;"
             "device_classes=backend_cuda:model_NVIDIA_B200:arch_10.0:memory_1:runtime_12090:driver_13000;"
             "transport=local;transport_env=affinity_default:ucx_tls_default")
    assert A.signature(canon) == "v2:" + fnv(canon)


def test_validate_hardware_signature(A):
    other = _cache(FFTM_AUTOTUNE_HARDWARE_SIGNATURE="v2:1111111111111111")
    with pytest.raises(FftbError, match="hardware signature"):
        A.validate(other, IDENT)
    A.validate(other, IDENT, A.autotune_options(validate_hardware=False))
    legacy = _cache(FFTM_AUTOTUNE_HARDWARE_SIGNATURE="mpi=1;device_total=1")
    with pytest.raises(FftbError, match="versioned"):
        A.validate(legacy, IDENT)
    strict = _cache(FFTM_AUTOTUNE_HARDWARE_SIGNATURE_STRICT="v2:2222222222222222")
    A.validate(strict, IDENT)  # compatible class, another device: accepted unless strict
    with pytest.raises(FftbError, match="strict"):
        A.validate(strict, IDENT, A.autotune_options(strict_device_identity=True))


def test_options_flags(A):
    assert A.autotune_options().flags() == A.CREATE_IF_MISSING
    o = A.autotune_options(create_if_missing=False, mismatch_policy="overwrite", validate_hardware=False,
                           strict_device_identity=True, force_measure=True)
    assert o.flags() == A.OVERWRITE_ON_MISMATCH | A.NO_HARDWARE_CHECK | A.STRICT_DEVICE | A.FORCE_MEASURE
    with pytest.raises(ValueError):
        A.autotune_options(mismatch_policy="ignore").flags()


def test_text_helpers(A):
    cfg = _cache()
    assert A.parse_text(A.to_text(cfg)) == cfg
    sel = A.selected_config(_cache(FFTB_AUTOTUNE_MEDIAN_MS_staged="1.5", **{"FFTB_AUTOTUNE_MEDIAN_MS_fused-cl2": "0.5"}),
                            "cache")
    assert sel.strategy == "fused" and sel.plane_cluster == 2
    assert sel.medians_ms() == {"staged": 1.5, "fused-cl2": 0.5}
