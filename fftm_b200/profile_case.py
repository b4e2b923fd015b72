"""Runs one workload of the library a fixed number of times and nothing else, so that
a profiler (``ncu -k ... -s ... -c ...``) sees a short, predictable launch sequence.

  python -m fftm_b200.profile_case poisson3d --n 256 --reps 3      # fused 3D Poisson solve
  python -m fftm_b200.profile_case poisson3d --n 256 --cluster 4   # same, 4-CTA plane clusters
  python -m fftm_b200.profile_case staged3d --n 256 --reps 3       # same, one pass kernel per axis
  python -m fftm_b200.profile_case roundtrip4d --n 64 --reps 3     # 4D R2C + normalised C2R
  python -m fftm_b200.profile_case batch --count 512 --reps 2      # batched round trips

Inputs are seeded and created on the device; each rep is one solve / round trip.
The first line printed gives the library launches per rep (the -s / -c arithmetic).
Exits non-zero if a result is wrong: a round trip must return its input (relative L2
below 1e-5) and a Poisson solution must be finite and survive an identity filter round
trip; parity against the FP64 oracle is the tests' job.
"""
from __future__ import annotations

import argparse
import sys


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["poisson3d", "staged3d", "roundtrip4d", "batch"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--layout", default="native_xzwy")
    ap.add_argument("--count", type=int, default=512)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--mode", type=int, default=2, help="batch mode: 0 sequential, 1 persistent, 2 graph")
    ap.add_argument("--cluster", type=int, default=0,
                    help="poisson3d: CTAs per plane of the fused kernels (1, 2, 4, 8; 0 = the library's choice)")
    a = ap.parse_args(argv)

    import torch

    import fftm_b200 as F
    dev = torch.device("cuda", 0)
    gen = torch.Generator(device=dev).manual_seed(0)
    if a.case in ("poisson3d", "staged3d"):
        n = a.n
        f = F.ffts("float32").init(n, n, n)
        if a.case == "staged3d":
            f.set_strategy("staged")
        elif a.cluster:
            f.set_strategy("fused", a.cluster)
        x = torch.rand((n, n, n), device=dev, generator=gen) - 0.5
        x -= x.mean()
        y = torch.empty_like(x)
        print(f"launches per rep: {f.num_launches('poisson')} ({f.strategy()})", flush=True)
        for _ in range(a.reps):
            f.poisson(x, y, -1.0)
        z = torch.empty_like(x)
        f.filter(y, z, 1e30)                 # a round trip with G = 1
        torch.cuda.synchronize()
        ok = bool(torch.isfinite(y).all()) and float(torch.linalg.norm(z - y) / torch.linalg.norm(y)) < 1e-5
    elif a.case == "roundtrip4d":
        n = a.n
        f = F.ffts("float32", strategy_4d=a.layout).init(n, n, n, n)
        x = torch.randn(f.real_shape(), device=dev, generator=gen)
        s = torch.empty(f.spectrum_shape(), dtype=torch.complex64, device=dev)
        y = torch.empty_like(x)
        print(f"launches per rep: {f.num_launches('forward') + f.num_launches('backward')}", flush=True)
        for _ in range(a.reps):
            f.forward(x, s)
            f.backward(s, y, normalized=True)
        torch.cuda.synchronize()
        ok = float(torch.linalg.norm(y - x) / torch.linalg.norm(x)) < 1e-5
    else:
        import fftm_b200.batch as B
        b = B.Batch(B.draw_shapes(a.count, seed=2))
        x = torch.rand(b.real_total, device=dev, generator=gen) * 2 - 1
        y = torch.empty_like(x)
        d = b.describe(B.ROUNDTRIP)
        print(f"launches per rep: {1 if a.mode else d['passes']} ({d})", flush=True)
        for _ in range(a.reps):
            b.exec(B.ROUNDTRIP, x, y, mode=a.mode)
        torch.cuda.synchronize()
        ok = b.status(B.ROUNDTRIP) == 0 and float(torch.linalg.norm(y - x) / torch.linalg.norm(x)) < 1e-5
    print("ok" if ok else "WRONG RESULT", flush=True)
    return 0 if ok else 1


if __name__ == "__main__":
    sys.exit(main())
