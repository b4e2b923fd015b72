"""GPU tests of the measured autotuner: load_or_measure for ffts problems and for
batches, the cache life cycle (measure -> file -> reuse -> mismatch error or
overwrite), and that the tuned choice is applied and computes the same transform as
the FP64 oracle."""
import os

import numpy as np
import pytest

import oracle as O
from fftm_b200 import FftbError

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def F(torch_cuda):
    from fftm_b200 import build
    build.build()
    import fftm_b200
    return fftm_b200


def test_hardware_keys(F):
    import fftm_b200.autotune as A
    hw = A.hardware_config(0)
    assert hw["FFTM_AUTOTUNE_HARDWARE_SIGNATURE"].startswith("v2:")
    assert hw["FFTM_AUTOTUNE_HARDWARE_SIGNATURE_STRICT"].startswith("v2:")
    assert hw["FFTM_AUTOTUNE_HARDWARE_SIGNATURE"] != hw["FFTM_AUTOTUNE_HARDWARE_SIGNATURE_STRICT"]
    assert hw["FFTM_AUTOTUNE_GPU_ARCHITECTURES"] == "10.0"
    assert A.hardware_config(0) == hw


def _token(v):
    # the reference's normalize_hardware_token (source/detail/fftm_autotune_hardware.inc:28-49)
    import re
    t = re.sub(r"[\x00\s;=,|]+", "_", v).strip("_")
    return t or "unknown"


def test_hardware_signature_is_the_reference_canonical_string(F, torch_cuda):
    # the single-rank canonical compatibility string of
    # source/detail/fftm_autotune_hardware.inc:285-310, rebuilt here from the device
    # properties and the environment, must be the one the library hashed
    torch = torch_cuda
    import fftm_b200.autotune as A
    hw = A.hardware_config(0)
    canon = hw["FFTB_AUTOTUNE_CANONICAL_COMPATIBILITY"]
    assert A.signature(canon) == hw["FFTM_AUTOTUNE_HARDWARE_SIGNATURE"]
    p = torch.cuda.get_device_properties(0)
    fields = dict(f.split("=", 1) for f in canon.split(";"))
    assert list(fields) == ["version", "mpi_ranks", "node_count", "ranks_per_node", "devices_per_node",
                            "mpi_library", "device_classes", "transport", "transport_env"]
    assert (fields["version"], fields["mpi_ranks"], fields["node_count"], fields["ranks_per_node"],
            fields["devices_per_node"], fields["mpi_library"], fields["transport"]) == \
        ("2", "1", "1", "1", "1", "unavailable", "local")
    cls = fields["device_classes"].split(":")
    assert cls[0] == "backend_cuda" and cls[1] == "model_" + _token(p.name) and cls[2] == f"arch_{p.major}.{p.minor}"
    assert cls[3] == f"memory_{p.total_memory}" and cls[4].startswith("runtime_") and cls[5].startswith("driver_")
    env = "affinity={}:ucx_tls={}:ucx_net_devices={}:mpi_pml={}:mpi_btl={}".format(
        *[_token(os.environ.get(k, "default")) for k in ("FFTM_MPI_RANK_AFFINITY_MODE", "UCX_TLS", "UCX_NET_DEVICES",
                                                         "OMPI_MCA_pml", "OMPI_MCA_btl")])
    assert fields["transport_env"] == _token(env)


def test_reference_written_single_gpu_cache_is_used(F, torch_cuda, tmp_path):
    # a cache as the reference's policy writes it for one rank on this machine: used as is
    # (nothing measured, the file untouched), its decomposition mapped onto the default
    # execution, and the transform still matches the oracle
    torch = torch_cuda
    import fftm_b200.autotune as A
    hw = A.hardware_config(0)
    ref = {"FFTM_AUTOTUNE_SCHEMA": "2", "FFTM_AUTOTUNE_POLICY_VERSION": "4", "FFTM_AUTOTUNE_LIBRARY": "fftm",
           "FFTM_AUTOTUNE_DIM": "3", "FFTM_AUTOTUNE_NUM_GPUS": "1", "FFTM_AUTOTUNE_SIZE_3D": "64x64x64",
           "FFTM_AUTOTUNE_SOURCE": "cpp-policy-cache-v4", "FFTM_AUTOTUNE_STRATEGY_3D": "slab-pencil",
           "FFTM_AUTOTUNE_GRID_3D": "1x1", "FFTM_AUTOTUNE_PENCIL_LAYOUT": "auto",
           "FFTM_AUTOTUNE_PENCIL_PIPELINE": "staged"}
    for k in ("FFTM_AUTOTUNE_HARDWARE_SIGNATURE_VERSION", "FFTM_AUTOTUNE_HARDWARE_SIGNATURE",
              "FFTM_AUTOTUNE_HARDWARE_SIGNATURE_STRICT"):
        ref[k] = hw[k]
    path = tmp_path / "fftm_autotune_3d.env"
    A.save_key_value_file(path, ref)
    mtime = os.path.getmtime(path)
    f = F.ffts("float32").init(64, 64, 64)
    sel = f.autotune(path, A.autotune_options(create_if_missing=False, strict_device_identity=True))
    assert sel.source == "cache" and os.path.getmtime(path) == mtime
    assert sel.strategy == "auto" and sel.config["FFTB_AUTOTUNE_REFERENCE_STRATEGY_3D"] == "slab-pencil"
    x = O.random_3d(64, 64, 64, 0x77, single=True)
    xin = torch.tensor(x, dtype=torch.float32, device="cuda")
    spec = torch.empty(f.spectrum_shape(), dtype=torch.complex64, device="cuda")
    f.forward(xin, spec)
    torch.cuda.synchronize()
    assert O.rel_l2(spec.cpu().numpy().astype(np.complex128), O.ffts3d_forward(x)) <= 2e-6


def test_ffts_cache_life_cycle(F, torch_cuda, tmp_path):
    torch = torch_cuda
    import fftm_b200.autotune as A
    path = tmp_path / "fftm_autotune_3d.env"
    opts = A.autotune_options(cache_file=str(path))
    m = A.measured_options(warmup=2, iterations=5)
    sel = A.load_or_measure_config("float32", (128, 128, 128), opts, m)
    assert sel.source == "measured" and os.path.exists(path)
    cfg = A.load_key_value_file(path)
    assert cfg == sel.config
    assert cfg["FFTM_AUTOTUNE_SCHEMA"] == "2" and cfg["FFTM_AUTOTUNE_SIZE_3D"] == "128x128x128"
    cands = cfg["FFTB_AUTOTUNE_CANDIDATES"].split(",")
    assert "staged" in cands and any(c.startswith("fused-cl") for c in cands)
    med = sel.medians_ms()
    assert set(med) == set(cands) and all(v > 0 for v in med.values())
    # the winner is the least median
    assert cfg["FFTM_AUTOTUNE_STRATEGY_3D"] == min(med, key=med.get)

    # second call: from the cache, nothing measured
    mtime = os.path.getmtime(path)
    again = A.load_or_measure_config("float32", (128, 128, 128), opts, m)
    assert again.source == "cache" and again.config == cfg and os.path.getmtime(path) == mtime

    # another size against this cache: error by default, re-measured with overwrite
    with pytest.raises(FftbError) as e:
        A.load_or_measure_config("float32", (64, 64, 64), opts, m)
    assert e.value.status == -12
    over = A.load_or_measure_config("float32", (64, 64, 64),
                                    A.autotune_options(cache_file=str(path), mismatch_policy="overwrite"), m)
    assert over.source == "measured" and A.load_key_value_file(path)["FFTM_AUTOTUNE_SIZE_3D"] == "64x64x64"

    # a missing cache without create_if_missing
    with pytest.raises(FftbError) as e:
        A.load_or_measure_config("float32", (64, 64, 64),
                                 A.autotune_options(cache_file=str(tmp_path / "none.env"), create_if_missing=False))
    assert e.value.status == -13


@pytest.mark.parametrize("dtype,dims,layout", [
    ("float32", (64, 48, 96), "pencil"), ("float64", (32, 24, 16), "pencil"), ("float32", (48, 40), "pencil"),
    ("float32", (16, 8, 8, 12), "native_xzwy"),
])
def test_ffts_autotune_applies_and_matches_oracle(F, torch_cuda, tmp_path, dtype, dims, layout):
    torch = torch_cuda
    f = F.ffts(dtype, strategy_4d=layout).init(*dims)
    sel = f.autotune(tmp_path / "t.env", measured=F.autotune.measured_options(warmup=1, iterations=3))
    strat, cl = f.strategy()
    assert strat == sel.strategy and (strat == "staged" or cl == sel.plane_cluster)
    rt = torch.float32 if dtype == "float32" else torch.float64
    ct = torch.complex64 if dtype == "float32" else torch.complex128
    rng = np.random.default_rng(11)
    x = rng.standard_normal(f.real_shape())
    X = torch.empty(f.spectrum_shape(), dtype=ct, device="cuda")
    f.forward(torch.tensor(x, dtype=rt, device="cuda"), X)
    got = X.cpu().numpy().astype(np.complex128)
    if len(dims) == 2:
        ref = np.fft.rfftn(x)
    elif len(dims) == 3:
        ref = O.ffts3d_forward(x)
    else:
        # native_xzwy spectrum [ky][kz][kw][kx] of the real [x][y][z][w] field
        ref = np.transpose(np.fft.rfftn(x), (1, 2, 3, 0))
    tol = 2e-6 if dtype == "float32" else 1e-12
    assert O.rel_l2(got, ref) <= tol


def test_every_strategy_agrees(F, torch_cuda):
    torch = torch_cuda
    f = F.ffts("float32").init(64, 128, 256)
    x = torch.randn(64, 128, 256, device="cuda")
    outs = {}
    for strat, cl in [("staged", 0), ("fused", 1), ("fused", 2), ("fused", 4), ("fused", 8)]:
        try:
            f.set_strategy(strat, cl)
        except FftbError as e:
            assert e.status == -2  # the size has no plane kernel with that cluster
            continue
        assert f.strategy() == (strat, cl)
        out = torch.empty_like(x)
        f.poisson(x, out, -1.0)
        outs[(strat, cl)] = out.double()
    assert len(outs) == 5
    base = outs[("staged", 0)]
    for k, v in outs.items():
        assert float(torch.linalg.norm(v - base) / torch.linalg.norm(base)) <= 2e-6, k
    f.set_strategy("auto")
    assert f.strategy()[0] == "fused"


def test_batch_autotune(F, torch_cuda, tmp_path):
    torch = torch_cuda
    import fftm_b200.batch as B
    shapes = B.draw_shapes(48, seed=2)
    b = B.Batch(shapes)
    path = tmp_path / "batch.env"
    sel = b.autotune(B.ROUNDTRIP, path, measured=F.autotune.measured_options(warmup=1, iterations=3))
    assert sel.source == "measured"
    cfg = F.autotune.load_key_value_file(path)
    assert cfg["FFTB_AUTOTUNE_BATCH_COUNT"] == "48" and cfg["FFTB_AUTOTUNE_BATCH_OP"] == "2"
    assert "sequential" in cfg["FFTB_AUTOTUNE_CANDIDATES"]
    assert b.mode == int(cfg["FFTB_AUTOTUNE_BATCH_MODE"])
    rng = np.random.default_rng(3)
    host = rng.uniform(-1, 1, b.real_total).astype(np.float32)
    x = torch.tensor(host, device="cuda")
    out = torch.zeros_like(x)
    b.exec(B.ROUNDTRIP, x, out)   # the tuned mode
    torch.cuda.synchronize()
    assert b.status(B.ROUNDTRIP) == 0
    assert float(torch.linalg.norm(out - x) / torch.linalg.norm(x)) <= 2e-6
    # a second batch with the same shapes reuses the cache; other shapes mismatch
    b2 = B.Batch(shapes)
    assert b2.autotune(B.ROUNDTRIP, path).source == "cache" and b2.mode == b.mode
    with pytest.raises(FftbError):
        B.Batch(shapes[:47]).autotune(B.ROUNDTRIP, path)
