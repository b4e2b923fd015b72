"""GPU tests of the batched uneven 3D transforms: every transform of a batch drawn
like the batched workload (axes from {32, 48, 64, 96, 128}, default_rng(2)) against
the FP64 oracle, the persistent and graph-replayed launches against the sequential
one, and the error flag of the bounded dependency waits."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
TOL = 2e-6


@pytest.fixture(scope="module")
def B(torch_cuda):
    from fftm_b200 import build
    build.build()
    import fftm_b200.batch as B
    return B


def _fill(torch, b, seed):
    rng = np.random.default_rng(seed)
    host = np.zeros(b.real_total, np.float32)
    for i, (nx, ny, nz) in enumerate(b.shapes):
        o = b.real_offsets[i]
        host[o:o + nx * ny * nz] = rng.uniform(-1, 1, nx * ny * nz)
    return torch.tensor(host, device="cuda"), host


@pytest.mark.parametrize("mode", [0, 1, 2, 3, 4])
def test_batch_forward_backward_vs_oracle(B, torch_cuda, mode):
    torch = torch_cuda
    shapes = B.draw_shapes(12, seed=2)
    b = B.Batch(shapes)
    x, host = _fill(torch, b, 5)
    spec = torch.zeros(b.spectrum_total, dtype=torch.complex64, device="cuda")
    b.exec(B.FORWARD, x, spec, mode=mode)
    torch.cuda.synchronize()
    assert b.status(B.FORWARD) == 0
    sp = spec.cpu().numpy().astype(np.complex128)
    for i, s in enumerate(shapes):
        o = b.real_offsets[i]
        xi = host[o:o + np.prod(s)].reshape(s).astype(np.float64)
        so = b.spectrum_offsets[i]
        got = sp[so:so + s[0] * s[1] * (s[2] // 2 + 1)].reshape(s[0], s[1], s[2] // 2 + 1)
        assert O.rel_l2(got, O.ffts3d_forward(xi)) <= TOL, (i, s)
    out = torch.zeros_like(x)
    b.exec(B.BACKWARD, spec, out, mode=mode)
    torch.cuda.synchronize()
    res = out.cpu().numpy().astype(np.float64)
    for i, s in enumerate(shapes):
        o = b.real_offsets[i]
        n = int(np.prod(s))
        assert O.rel_l2(res[o:o + n], host[o:o + n].astype(np.float64)) <= TOL, (i, s)


# lengths with and without the fused path's column and row tiles side by side in one stage
# (x, y: 32-128 column tiles, 8-40 the pass kernel; z: 64-256 row tiles, 16-96 the pass
# kernel), and spectra with fewer lines than one tile
EDGE_SHAPES = [(8, 12, 64), (12, 8, 128), (32, 20, 64), (64, 12, 128), (48, 16, 96), (96, 32, 40), (16, 16, 256),
               (128, 8, 32), (20, 48, 128), (40, 96, 16)]


@pytest.mark.parametrize("mode", [1, 2, 3, 4])
def test_batch_edge_shapes_vs_oracle(B, torch_cuda, mode):
    torch = torch_cuda
    b = B.Batch(EDGE_SHAPES)
    assert b.describe(B.ROUNDTRIP)["persistent"] == 1  # every length runs the one-launch forms
    x, host = _fill(torch, b, 9)
    spec = torch.zeros(b.spectrum_total, dtype=torch.complex64, device="cuda")
    b.exec(B.FORWARD, x, spec, mode=mode)
    torch.cuda.synchronize()
    assert b.status(B.FORWARD) == 0
    sp = spec.cpu().numpy().astype(np.complex128)
    for i, s in enumerate(EDGE_SHAPES):
        o = b.real_offsets[i]
        xi = host[o:o + np.prod(s)].reshape(s).astype(np.float64)
        so = b.spectrum_offsets[i]
        got = sp[so:so + s[0] * s[1] * (s[2] // 2 + 1)].reshape(s[0], s[1], s[2] // 2 + 1)
        assert O.rel_l2(got, O.ffts3d_forward(xi)) <= TOL, (i, s)
    out = torch.zeros_like(x)
    b.exec(B.ROUNDTRIP, x, out, mode=mode)
    torch.cuda.synchronize()
    res = out.cpu().numpy().astype(np.float64)
    for i, s in enumerate(EDGE_SHAPES):
        o = b.real_offsets[i]
        n = int(np.prod(s))
        assert O.rel_l2(res[o:o + n], host[o:o + n].astype(np.float64)) <= TOL, (i, s)
    po = torch.zeros_like(x)
    b.exec(B.POISSON, x, po, sign=-1.0, mode=mode)
    torch.cuda.synchronize()
    pr = po.cpu().numpy().astype(np.float64)
    for i, s in enumerate(EDGE_SHAPES):
        o = b.real_offsets[i]
        n = int(np.prod(s))
        ref = O.poisson3d_solve(host[o:o + n].reshape(s).astype(np.float64), -1.0)
        assert O.rel_l2(pr[o:o + n].reshape(s), ref) <= TOL, (i, s)


def test_batch_roundtrip_poisson_modes_agree(B, torch_cuda):
    torch = torch_cuda
    shapes = B.draw_shapes(40, seed=2)
    b = B.Batch(shapes)
    x, host = _fill(torch, b, 6)
    outs = {}
    for op in (B.ROUNDTRIP, B.POISSON):
        for mode in (0, 1, 2, 3, 4):
            out = torch.zeros_like(x)
            b.exec(op, x, out, sign=-1.0, mode=mode)
            b.exec(op, x, out, sign=-1.0, mode=mode)   # replay the same binding
            torch.cuda.synchronize()
            assert b.status(op) == 0
            outs[(op, mode)] = out.cpu().numpy()
        # the persistent and grouped modes run the same tiles (the fused path's column and
        # z-row tiles where a stage has them), so they agree bit for bit; the sequential mode
        # runs every stage on the pass kernel (half-length z FFTs, the Poisson multiply by a
        # division) and agrees with them to rounding
        for mode in (2, 3, 4):
            np.testing.assert_array_equal(outs[(op, 1)], outs[(op, mode)])
        d = O.rel_l2(outs[(op, 1)].astype(np.float64), outs[(op, 0)].astype(np.float64))
        assert d <= 1e-6, d
    for mode in (2, 4):
        rt = outs[(B.ROUNDTRIP, mode)].astype(np.float64)
        assert O.rel_l2(rt, host.astype(np.float64)) <= TOL
        po = outs[(B.POISSON, mode)].astype(np.float64)
        for i in (0, 7, 21, 39):
            s = shapes[i]
            o = b.real_offsets[i]
            n = int(np.prod(s))
            ref = O.poisson3d_solve(host[o:o + n].reshape(s).astype(np.float64), -1.0)
            assert O.rel_l2(po[o:o + n].reshape(s), ref) <= TOL


def test_batch_full_workload_512(B, torch_cuda):
    torch = torch_cuda
    shapes = B.draw_shapes(512, seed=2)
    b = B.Batch(shapes)
    d = b.describe(B.ROUNDTRIP)
    assert d["persistent"] == 1 and d["passes"] == 5 * 512
    x, host = _fill(torch, b, 7)
    out = torch.zeros_like(x)
    b.exec(B.ROUNDTRIP, x, out, mode=2)
    torch.cuda.synchronize()
    assert b.status(B.ROUNDTRIP) == 0
    assert float(torch.linalg.norm(out - x) / torch.linalg.norm(x)) <= TOL



def test_batch_full_workload_512_forward_spectra_vs_oracle(B, torch_cuda):
    # the benchmarked form (grouped launches replayed from a graph, mode 4) on the full
    # 512-shape workload: forward spectra of a sample of transforms of every length mix
    # against the FP64 oracle, and the round trip of all of them
    torch = torch_cuda
    shapes = B.draw_shapes(512, seed=2)
    b = B.Batch(shapes)
    x, host = _fill(torch, b, 9)
    spec = torch.zeros(b.spectrum_total, dtype=torch.complex64, device="cuda")
    b.exec(B.FORWARD, x, spec, mode=B.GROUPED_GRAPH)
    torch.cuda.synchronize()
    sp = spec.cpu().numpy()
    for i in list(range(0, 512, 37)) + [511]:
        s = shapes[i]
        o, so = b.real_offsets[i], b.spectrum_offsets[i]
        xi = host[o:o + int(np.prod(s))].reshape(s).astype(np.float64)
        got = sp[so:so + s[0] * s[1] * (s[2] // 2 + 1)].reshape(s[0], s[1], s[2] // 2 + 1)
        assert O.rel_l2(got.astype(np.complex128), O.ffts3d_forward(xi)) <= TOL, (i, s)
    out = torch.zeros_like(x)
    b.exec(B.ROUNDTRIP, x, out, mode=B.GROUPED_GRAPH)
    torch.cuda.synchronize()
    assert float(torch.linalg.norm(out - x) / torch.linalg.norm(x)) <= TOL


def test_bounded_dependency_wait_gives_up_and_flags(B, torch_cuda):
    # a wait on a producer that has no items (nothing ever counts it done) must run out of
    # polls, raise the error flag and return; the context stays usable afterwards
    torch = torch_cuda
    import time
    t0 = time.time()
    assert B.wait_selftest(2000) == 1
    assert time.time() - t0 < 30
    shapes = B.draw_shapes(6, seed=2)
    b = B.Batch(shapes)
    b.set_wait_limit(1 << 20)
    x, host = _fill(torch, b, 3)
    out = torch.zeros_like(x)
    b.exec(B.ROUNDTRIP, x, out, mode=B.PERSISTENT)
    torch.cuda.synchronize()
    assert b.status(B.ROUNDTRIP) == 0
    assert float(torch.linalg.norm(out - x) / torch.linalg.norm(x)) <= TOL
    b.set_wait_limit(0)


def test_batch_float64_runs_sequential_launches(B, torch_cuda):
    torch = torch_cuda
    shapes = [(16, 12, 10), (9, 8, 14), (32, 16, 8)]
    b = B.Batch(shapes, dtype="float64")
    assert b.describe(B.ROUNDTRIP)["persistent"] == 0
    x = torch.rand(b.real_total, dtype=torch.float64, device="cuda") * 2 - 1
    for mode in (B.SEQUENTIAL, B.GRAPH, B.GROUPED_GRAPH):   # float64 runs the plain launches in every mode
        out = torch.zeros_like(x)
        b.exec(B.ROUNDTRIP, x, out, mode=mode)
        torch.cuda.synchronize()
        for i, s in enumerate(shapes):
            o = b.real_offsets[i]
            n = int(np.prod(s))
            assert O.rel_l2(out[o:o + n].cpu().numpy(), x[o:o + n].cpu().numpy()) <= 1e-12


def test_tensor_core_form_needs_float32(B, torch_cuda):
    import fftm_b200 as F
    f = F.ffts("float64").init(64, 64, 64)
    with pytest.raises(F.FftbError) as e:
        f.set_strategy("fused_tc")
    assert e.value.status == -2
