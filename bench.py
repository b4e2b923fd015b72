#!/usr/bin/env python3
"""Benchmark of the single-GPU transform path: the 3D periodic Poisson solve at
256^3 float32 (R2C, multiply by -1/|k|^2 with k = 0 zeroed, C2R, 1/N).

One step = one R2C + C2R round trip over one 256^3 field (the fused Poisson
solve).  The metric is algorithmic HBM GB/s: bytes = 2 * (4 N + 8 N_c) per
round trip (N = 256^3 real points, N_c = 256*256*129 half-spectrum points), the
bytes a round trip must read and write once.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl fftb|reference]
  python bench.py --profile-case poisson3d|staged3d|roundtrip4d|batch [...]   (for ncu)

Device timing uses CUDA events on the launching stream.  Between timed steps a
1 GiB buffer (larger than the 126 MB L2) is overwritten outside the timed
window, so every step starts with a cold L2.  With N > 1 (torchrun), every rank
solves its own field (replicas; the single transform does not shard) and the
slowest rank's time is reported.  ``--impl reference`` times the CPU reference
arm: the reference's CUDA path cannot be built here (its SCFD submodule is
absent and its FFTs are cuFFT), so the arm runs the FP64 CPU restatement of
its algorithm (oracle/) on all host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "R2C+C2R ms & HBM GB/s at 256^3/64^4; TC/batched vs plain FP32 at err<=5e-6"
NX = NY = NZ = 256
N_REAL = NX * NY * NZ
N_CPLX = NX * NY * (NZ // 2 + 1)
BYTES_RT = 2 * (4 * N_REAL + 8 * N_CPLX)   # 269,484,032
FLOPS_RT = 2 * 5 * N_REAL * 24              # 5 N log2 N per transform, two transforms
WORKLOAD = "3D periodic Poisson solve 256^3 f32: R2C, x(-1/|k|^2) (k=0 -> 0), C2R, 1/N"
DATA = ("synthetic: f = sin x sin 2y cos 3z + 0.1*U[-1,1] (numpy default_rng(0)), mean removed, "
        "grid x_i = 2 pi i / 256")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="fftb", choices=["fftb", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--strategy", choices=["fused", "staged", "fused_tc"],
                    help="run the headline solve with this strategy instead of the autotuner's choice")
    # profiling mode: run one workload a fixed number of times and nothing else, so that a
    # profiler (ncu -k ... -s ... -c ...) sees a short, predictable launch sequence
    ap.add_argument("--profile-case", choices=["poisson3d", "staged3d", "roundtrip4d", "batch"])
    ap.add_argument("--n", type=int, default=256, help="profile case: grid size per axis")
    ap.add_argument("--layout", default="native_xzwy", help="profile case roundtrip4d: 4D layout")
    ap.add_argument("--count", type=int, default=512, help="profile case batch: transforms")
    ap.add_argument("--reps", type=int, default=3, help="profile case: solves / round trips")
    ap.add_argument("--mode", type=int, default=2, help="profile case batch: 0 sequential, 1 persistent, "
                                                        "2 persistent graph, 3 grouped, 4 grouped graph")
    ap.add_argument("--cluster", type=int, default=0,
                    help="profile case poisson3d: CTAs per plane (1, 2, 4, 8; 0 = the library's choice)")
    return ap.parse_args()


def profile_case(a) -> int:
    """Runs one workload `reps` times on seeded device inputs and nothing else.  The first
    line printed gives the library launches per rep (the ncu -s / -c arithmetic).  Exits
    non-zero if a result is wrong: a round trip must return its input (relative L2 below
    1e-5) and a Poisson solution must be finite and survive an identity filter round trip;
    parity against the FP64 oracle is the tests' job.

      python bench.py --profile-case poisson3d --n 256 --reps 3      # fused 3D Poisson solve
      python bench.py --profile-case poisson3d --n 256 --cluster 4   # 4-CTA plane clusters
      python bench.py --profile-case staged3d --n 256 --reps 3       # one pass kernel per axis
      python bench.py --profile-case roundtrip4d --n 64 --reps 3     # 4D R2C + normalised C2R
      python bench.py --profile-case batch --count 512 --reps 2      # batched round trips
    """
    import torch

    import fftm_b200 as F
    dev = torch.device("cuda", 0)
    gen = torch.Generator(device=dev).manual_seed(0)
    if a.profile_case in ("poisson3d", "staged3d"):
        n = a.n
        f = F.ffts("float32").init(n, n, n)
        if a.profile_case == "staged3d":
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
    elif a.profile_case == "roundtrip4d":
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
        print(f"launches per rep: {1 if a.mode in (1, 2) else d['passes']} ({d})", flush=True)
        for _ in range(a.reps):
            b.exec(B.ROUNDTRIP, x, y, mode=a.mode)
        torch.cuda.synchronize()
        ok = b.status(B.ROUNDTRIP) == 0 and float(torch.linalg.norm(y - x) / torch.linalg.norm(x)) < 1e-5
    print("ok" if ok else "WRONG RESULT", flush=True)
    return 0 if ok else 1


def make_rhs(dtype=np.float32):
    g = 2 * np.pi * np.arange(NX) / NX
    x = g[:, None, None]
    y = g[None, :, None]
    z = g[None, None, :]
    f = np.sin(x) * np.sin(2 * y) * np.cos(3 * z)
    rng = np.random.default_rng(0)
    f = f + 0.1 * rng.uniform(-1.0, 1.0, (NX, NY, NZ))
    f -= f.mean()
    return np.ascontiguousarray(f.astype(dtype))


# ---------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []          # (arrival time, csv line)
        self.window = (0.0, 0.0)

    def start(self):
        """Starts sampling and waits (up to 5 s) for the first sample, so that the
        sampler is live before the timed region begins."""
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < 5.0:
                time.sleep(0.01)
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def mark(self, t_begin, t_end):
        self.window = (t_begin, t_end)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        b, e = self.window
        inside = [ln for t, ln in self.lines if b <= t <= e + 0.05]
        if not inside and self.lines:
            after = [(t, ln) for t, ln in self.lines if t >= b]
            inside = [after[0][1]] if after else [self.lines[-1][1]]
        for ln in inside:
            p = [v.strip() for v in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm),
                "window_ms": round((e - b) * 1e3, 1)}


def measured_hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(kernel_name):
    """DRAM bytes per launch of a kernel from the committed ncu summary, or None."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(p) as fh:
            d = json.load(fh)
        v = d.get(kernel_name)
        return None if v is None else float(v["dram_bytes_per_launch"])
    except Exception:
        return None


# ---------------------------------------------------------------------- CPU legs
def scipy_fft_rates(f_host):
    """The same solve with scipy.fft on all host cores, float64 and float32 (a library
    baseline beside the oracle; FFTW, the reference's CPU library, is not installed)."""
    try:
        import scipy.fft as sf
    except Exception as exc:  # noqa: BLE001
        return {"unavailable": str(exc)[:120]}
    workers = os.cpu_count() or 1
    k = np.fft.fftfreq(NX, 1.0 / NX)
    kz = np.arange(NZ // 2 + 1)
    k2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + kz[None, None, :] ** 2
    with np.errstate(divide="ignore"):
        mult = np.where(k2 == 0, 0.0, -1.0 / k2)
    out = {"cores": workers}
    for name, dt in (("f64", np.float64), ("f32", np.float32)):
        x = f_host.astype(dt)
        m = mult.astype(dt)
        sf.irfftn(sf.rfftn(x, workers=workers) * m, s=x.shape, workers=workers)   # warm-up (plans)
        t0 = time.perf_counter()
        sf.irfftn(sf.rfftn(x, workers=workers) * m, s=x.shape, workers=workers)
        dt_s = time.perf_counter() - t0
        out[name] = {"seconds": dt_s, "value": BYTES_RT / dt_s / 1e9, "unit": "GB/s"}
    return out



def cpu_oracle_rate(f_host, sample_solves=1):
    """FP64 oracle Poisson solve on all host threads; returns (GB/s, seconds, threads, solution)."""
    import oracle as O
    threads = O.max_threads()
    O.set_threads(threads)
    f64 = f_host.astype(np.float64)
    t0 = time.perf_counter()
    sol = None
    for _ in range(sample_solves):
        sol = O.poisson3d_solve(f64, -1.0)
    dt = time.perf_counter() - t0
    return BYTES_RT * sample_solves / dt / 1e9, dt, threads, sol


def run_reference(args, rank):
    """CPU reference arm (rank 0 only).  Each step is a bounded sample: the full
    256^3 solve when K steps of it fit in about two minutes, otherwise a 128^3
    solve of the same field family (rate in the same unit, bytes of the sample)."""
    if rank != 0:
        return
    f = make_rhs(np.float32)
    import oracle as O
    threads = O.max_threads()
    O.set_threads(threads)
    f64 = f.astype(np.float64)
    t0 = time.perf_counter()
    O.poisson3d_solve(f64, -1.0)
    t_full = time.perf_counter() - t0
    if args.steps * t_full > 120.0:
        f64 = np.ascontiguousarray(f64[::2, ::2, ::2])
        sample = "128^3 FP64 Poisson solve per step (every other grid point of the 256^3 field)"
    else:
        sample = "full 256^3 FP64 Poisson solve per step"
    n = f64.shape[0]
    bytes_step = 2 * (4 * n ** 3 + 8 * n * n * (n // 2 + 1))
    for _ in range(max(0, min(args.warmup, 1))):
        O.poisson3d_solve(f64, -1.0)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.poisson3d_solve(f64, -1.0)
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    value = bytes_step * args.steps / tot / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": DATA, "config": {"workload": WORKLOAD, "n": [NX, NY, NZ], "bytes_per_step": BYTES_RT},
        "cpu_baseline": {"value": value, "unit": "GB/s", "cores": threads, "kind": "port",
                         "sample": sample + " (oracle/fft_oracle.c, OpenMP)"},
        "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": ("reference CUDA path not buildable here (SCFD submodule empty, cuFFT-only FFTs); "
                 "arm = FP64 CPU restatement of its transform path"),
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------- GPU arm
def main():
    args = parse()
    if args.profile_case:
        return profile_case(args)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return 0

    import torch
    from fftm_b200 import replicas
    torch.cuda.set_device(local)
    dist = replicas.init_group("nccl", device=torch.device("cuda", local))

    from fftm_b200 import build as _build
    if rank == 0 or world == 1:
        _build.build()
    if dist is not None:
        dist.barrier()
    import fftm_b200 as F

    dev = torch.device("cuda", local)
    f_host = make_rhs(np.float32)
    rhs = torch.from_numpy(f_host).to(dev)
    sol = torch.empty_like(rhs)
    ff = F.ffts("float32").init(NX, NY, NZ)
    work = torch.empty(ff.work_size // 8 + 1, dtype=torch.complex64, device=dev)
    ff.set_work_area(work)
    # execution strategy from the project autotuner (fresh cache per run: a measured sweep of
    # the fused plane-cluster sizes and the staged passes, least median of forward+backward)
    import tempfile
    if args.strategy:
        # a fixed strategy instead of the measured one (for ncu launch lists: under ncu the
        # profiled kernels run slower, which would bias the autotuner's choice)
        ff.set_strategy(args.strategy)
        tuned = None
    else:
        with tempfile.TemporaryDirectory() as td:
            tuned = ff.autotune(os.path.join(td, "fftm_autotune_3d.env"))
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.float32, device=dev)   # 1 GiB > L2
    stream = torch.cuda.current_stream()

    def step():
        ff.poisson(rhs, sol, -1.0)

    for _ in range(max(3, args.warmup)):
        flush.zero_()
        step()
    torch.cuda.synchronize()

    launches_per_step = ff.num_launches("poisson")
    ff.timing_enable(launches_per_step * args.steps + 8)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = ClockSampler(local)
    clocks.start()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    t_begin = time.time()
    for i in range(args.steps):
        flush.zero_()                # outside the timed window; also covers host enqueue time
        starts[i].record(stream)
        step()
        ends[i].record(stream)
    torch.cuda.synchronize()
    clocks.mark(t_begin, time.time())
    if dist is not None:
        dist.barrier()
    clk = clocks.stop()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = sum(step_ms)
    per_launch = ff.timing_read()
    ff.timing_enable(0)
    total_ms = replicas.max_over_ranks(dist, total_ms, dev)
    value = replicas.whole_job_rate(BYTES_RT, args.steps, world, total_ms) / 1e9

    # per-kernel roofline from the live per-launch events
    agg = {}
    for name, ms, by in per_launch:
        a = agg.setdefault(name, [0, 0.0, by])
        a[0] += 1
        a[1] += ms
    dom = max(agg.items(), key=lambda kv: kv[1][1])
    dom_name, (dom_n, dom_ms, dom_bytes) = dom
    peak, peak_kind = measured_hbm_peak()
    avg_ms = dom_ms / dom_n
    achieved = dom_bytes / (avg_ms * 1e-3) / 1e9
    traffic = ncu_traffic(dom_name)
    kernels = {k: {"launches": v[0], "avg_us": v[1] / v[0] * 1e3, "share": v[1] / max(1e-9, sum(x[1] for x in
                                                                                                agg.values())),
                   "alg_bytes": v[2], "gbs": v[2] / (v[1] / v[0] * 1e-3) / 1e9} for k, v in agg.items()}

    # end to end through the public API with host buffers (pinned), copies inside the timed region.
    # Every step copies its right-hand side host -> device, solves, and copies the solution
    # device -> host.  Two buffer sets and three streams (upload, solve, download) let step
    # i+1's upload (one copy engine) and step i-1's download (the other engine) run while step
    # i solves, as a serving loop would, so the step time approaches one PCIe transfer of the
    # field; the same loop with one stream (each copy after the previous step) is reported
    # beside it.
    h_in = torch.from_numpy(f_host).pin_memory()
    h_out = [torch.empty_like(h_in).pin_memory() for _ in range(2)]
    d_in = [torch.empty_like(rhs) for _ in range(2)]
    d_out = [torch.empty_like(rhs) for _ in range(2)]
    s_in, s_cmp, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    ev_in = [torch.cuda.Event() for _ in range(2)]        # upload of buffer set b done
    ev_solved = [torch.cuda.Event() for _ in range(2)]    # solve of set b done (d_in[b] free)
    ev_out = [torch.cuda.Event() for _ in range(2)]       # download of set b done (d_out[b] free)
    e2e_steps = max(3, min(args.steps, 20))

    def e2e_pipelined(nsteps):
        for i in range(nsteps):
            b = i % 2
            with torch.cuda.stream(s_in):
                if i >= 2:
                    s_in.wait_event(ev_solved[b])
                d_in[b].copy_(h_in, non_blocking=True)
                ev_in[b].record(s_in)
            with torch.cuda.stream(s_cmp):
                s_cmp.wait_event(ev_in[b])
                if i >= 2:
                    s_cmp.wait_event(ev_out[b])
                ff.poisson(d_in[b], d_out[b], -1.0, stream=s_cmp)
                ev_solved[b].record(s_cmp)
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev_solved[b])
                h_out[b].copy_(d_out[b], non_blocking=True)
                ev_out[b].record(s_out)

    def e2e_serial(nsteps):
        for _ in range(nsteps):
            d_in[0].copy_(h_in, non_blocking=True)
            ff.poisson(d_in[0], d_out[0], -1.0)
            h_out[0].copy_(d_out[0], non_blocking=True)

    e2e_pipelined(2)
    e2e_serial(2)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s_in)
    s_cmp.wait_event(e0)
    s_out.wait_event(e0)
    e2e_pipelined(e2e_steps)
    e1.record(s_out)   # after the last download, which follows every earlier copy and solve
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    e2e_ms = replicas.max_over_ranks(dist, e2e_ms, dev)
    e2e_val = replicas.whole_job_rate(BYTES_RT, e2e_steps, world, e2e_ms) / 1e9
    e0.record(stream)
    e2e_serial(e2e_steps)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_serial_ms = replicas.max_over_ranks(dist, e0.elapsed_time(e1), dev)
    e2e_ok = bool(torch.equal(h_out[1], h_out[0]))   # a pipelined step vs the last serial step

    # secondary size of the metric: 4D 64^4 native_xzwy R2C + C2R round trip (forward, then the
    # normalised inverse), input N(0,1) from default_rng(1), same flush / event protocol
    sec = None
    try:
        d4 = (64, 64, 64, 64)
        f4 = F.ffts("float32", strategy_4d="native_xzwy").init(*d4)
        w4 = torch.empty(f4.work_size // 8 + 1, dtype=torch.complex64, device=dev)
        f4.set_work_area(w4)
        x4 = torch.from_numpy(np.random.default_rng(1).standard_normal(d4).astype(np.float32)).to(dev)
        y4 = torch.empty_like(x4)
        s4 = torch.empty(f4.spectrum_shape(), dtype=torch.complex64, device=dev)

        def rt4():
            f4.forward(x4, s4)
            f4.backward(s4, y4, normalized=True)

        for _ in range(3):
            flush.zero_()
            rt4()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(20)]
        for a, b in ev:
            flush.zero_()
            a.record(stream)
            rt4()
            b.record(stream)
        torch.cuda.synchronize()
        ms4 = sum(a.elapsed_time(b) for a, b in ev) / len(ev)
        b4 = 2 * (4 * 64 ** 4 + 8 * 64 ** 3 * 33)
        err4 = float(torch.linalg.norm(y4 - x4) / torch.linalg.norm(x4))

        def cufft4():
            torch.fft.irfftn(torch.fft.rfftn(x4), s=d4)

        for _ in range(3):
            cufft4()
        torch.cuda.synchronize()
        cv = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(20)]
        for a, b in cv:
            flush.zero_()
            a.record(stream)
            cufft4()
            b.record(stream)
        torch.cuda.synchronize()
        cms4 = sum(a.elapsed_time(b) for a, b in cv) / len(cv)
        # the same round trip with the split-FP16 tensor-core column kernels, and the spectra
        # of both forms against cuFFT in FP64 on the same input
        ref64 = torch.fft.rfftn(x4.double()).permute(1, 2, 3, 0)
        err_plain = float(torch.linalg.norm(s4.to(torch.complex128) - ref64) / torch.linalg.norm(ref64))
        f4.set_strategy("fused_tc")
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(20)]
        for _ in range(3):
            flush.zero_()
            rt4()
        torch.cuda.synchronize()
        for a, b in ev:
            flush.zero_()
            a.record(stream)
            rt4()
            b.record(stream)
        torch.cuda.synchronize()
        ms4tc = sum(a.elapsed_time(b) for a, b in ev) / len(ev)
        f4.forward(x4, s4)
        err_tc = float(torch.linalg.norm(s4.to(torch.complex128) - ref64) / torch.linalg.norm(ref64))
        f4.backward(s4, y4, normalized=True)
        err4tc = float(torch.linalg.norm(y4 - x4) / torch.linalg.norm(x4))
        f4.set_strategy("fused")
        del ref64
        sec = {"workload": "4D 64^4 f32 native_xzwy R2C + normalised C2R round trip", "ms_per_step": ms4,
               "value": b4 / (ms4 * 1e-3) / 1e9, "unit": "GB/s", "bytes_per_step": b4,
               "launches_per_step": f4.num_launches("forward") + f4.num_launches("backward"),
               "round_trip_rel_l2": err4, "spectrum_rel_l2_vs_fp64_cufft": err_plain,
               "tensor_core_form": {"impl": "column kernels' first radix-16 stage as split-FP16 mma.sync "
                                            "m16n8k16 (head+tail operands, FP32 accumulate)",
                                    "ms_per_step": ms4tc, "value": b4 / (ms4tc * 1e-3) / 1e9,
                                    "speedup_vs_plain_fp32": ms4 / ms4tc,
                                    "spectrum_rel_l2_vs_fp64_cufft": err_tc, "round_trip_rel_l2": err4tc},
               "cufft_same_gpu": {"impl": "torch.fft rfftn + irfftn", "ms_per_step": cms4,
                                  "value": b4 / (cms4 * 1e-3) / 1e9}}
    except Exception as exc:  # noqa: BLE001
        sec = {"unavailable": str(exc)[:200]}

    def time_events(fn, n, flush_between=True):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
        for a, b in evs:
            if flush_between:
                flush.zero_()
            a.record(stream)
            fn()
            b.record(stream)
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in evs]

    # plain 256^3 round trip (forward, then normalised backward), U[-1,1] from default_rng(0)
    more = {}
    try:
        xr = torch.from_numpy(np.random.default_rng(0).uniform(-1, 1, (NX, NY, NZ)).astype(np.float32)).to(dev)
        yr = torch.empty_like(xr)
        sr = torch.empty(ff.spectrum_shape(), dtype=torch.complex64, device=dev)
        ms = time_events(lambda: (ff.forward(xr, sr), ff.backward(sr, yr, normalized=True)), 50)
        t = statistics.median(ms)
        more["roundtrip_256"] = {"workload": "3D 256^3 f32 R2C + normalised C2R, U[-1,1] default_rng(0)",
                                 "median_us": t * 1e3, "value": BYTES_RT / (t * 1e-3) / 1e9, "unit": "GB/s",
                                 "gflops": FLOPS_RT / (t * 1e-3) / 1e9,
                                 "round_trip_rel_l2": float(torch.linalg.norm(yr - xr) / torch.linalg.norm(xr))}
        del xr, yr, sr
    except Exception as exc:  # noqa: BLE001
        more["roundtrip_256"] = {"unavailable": str(exc)[:200]}
    # 64^3 round trip: fits in L2, latency bound, timed as CUDA-graph replays
    try:
        f64 = F.ffts("float32").init(64, 64, 64)
        w64 = torch.empty(max(1, f64.work_size // 8 + 1), dtype=torch.complex64, device=dev)
        f64.set_work_area(w64)
        x64 = torch.from_numpy(np.random.default_rng(0).uniform(-1, 1, (64, 64, 64)).astype(np.float32)).to(dev)
        y64 = torch.empty_like(x64)
        s64 = torch.empty(f64.spectrum_shape(), dtype=torch.complex64, device=dev)
        for _ in range(3):
            f64.forward(x64, s64)
            f64.backward(s64, y64, normalized=True)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            f64.forward(x64, s64)
            f64.backward(s64, y64, normalized=True)
        g.replay()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(200):
            g.replay()
        b.record(stream)
        torch.cuda.synchronize()
        t = a.elapsed_time(b) / 200
        b64 = 2 * (4 * 64 ** 3 + 8 * 64 * 64 * 33)
        more["roundtrip_64_graph"] = {"workload": "3D 64^3 f32 R2C + normalised C2R, CUDA-graph replay (L2 resident)",
                                      "us_per_round_trip": t * 1e3, "value": b64 / (t * 1e-3) / 1e9, "unit": "GB/s",
                                      "round_trip_rel_l2": float(torch.linalg.norm(y64 - x64) / torch.linalg.norm(x64))}
        del g
    except Exception as exc:  # noqa: BLE001
        more["roundtrip_64_graph"] = {"unavailable": str(exc)[:200]}
    # 4D 64^4 native_xzwy Poisson solve
    try:
        f4p = F.ffts("float32", strategy_4d="native_xzwy").init(64, 64, 64, 64)
        w4p = torch.empty(f4p.work_size // 8 + 1, dtype=torch.complex64, device=dev)
        f4p.set_work_area(w4p)
        x4p = torch.from_numpy(np.random.default_rng(1).standard_normal((64,) * 4).astype(np.float32)).to(dev)
        y4p = torch.empty_like(x4p)
        ms = time_events(lambda: f4p.poisson(x4p, y4p, -1.0), 30)
        t = statistics.median(ms)
        b4 = 2 * (4 * 64 ** 4 + 8 * 64 ** 3 * 33)
        more["poisson4d_64"] = {"workload": "4D 64^4 f32 native_xzwy Poisson solve, N(0,1) default_rng(1)",
                                "median_us": t * 1e3, "value": b4 / (t * 1e-3) / 1e9, "unit": "GB/s",
                                "launches": f4p.num_launches("poisson")}
        del x4p, y4p, w4p
    except Exception as exc:  # noqa: BLE001
        more["poisson4d_64"] = {"unavailable": str(exc)[:200]}
    # spectral derivative and gradient of the 256^3 field (the reference test's
    # derivative_spectra_functor pipeline); algorithmic bytes: one read of u, one write per
    # derivative
    try:
        xd = torch.from_numpy(np.random.default_rng(0).uniform(-1, 1, (NX, NY, NZ)).astype(np.float32)).to(dev)
        outs = [torch.empty_like(xd) for _ in range(3)]
        ms = time_events(lambda: ff.derivative(xd, outs[0], 1), 30)
        t = statistics.median(ms)
        more["derivative_256"] = {"workload": "du/dy of a 256^3 f32 field, U[-1,1] default_rng(0)",
                                  "median_us": t * 1e3, "value": 8 * NX * NY * NZ / (t * 1e-3) / 1e9, "unit": "GB/s"}
        ms = time_events(lambda: ff.gradient(xd, outs), 30)
        t = statistics.median(ms)
        more["gradient_256"] = {"workload": "(du/dx, du/dy, du/dz) of a 256^3 f32 field, U[-1,1] default_rng(0)",
                                "median_us": t * 1e3, "value": 16 * NX * NY * NZ / (t * 1e-3) / 1e9, "unit": "GB/s"}
        del xd, outs
    except Exception as exc:  # noqa: BLE001
        more["derivative_256"] = {"unavailable": str(exc)[:200]}

    # differentiable spectral pipeline at 128^3: u = sin x cos y cos z + 0.05 N(0,1)
    # (default_rng(4)), w = Poisson(C2R(G R2C(u))) with G = exp(-|k|^2 / (2 16^2)),
    # loss = 0.5 |w|^2, gradient through the adjoint kernels.  One step = forward + loss +
    # backward.  Composed: R2C, G multiply (torch), normalised C2R, Poisson solve, and their
    # adjoints: 4 round trips of algorithmic bytes (2 forward, 2 backward).  Fused: the
    # filter and Poisson multiply in one sandwich, forward and adjoint: 2 round trips.
    try:
        import fftm_b200.autograd as A
        n3 = (128, 128, 128)
        g1 = 2 * np.pi * np.arange(128) / 128
        u0 = (np.sin(g1)[:, None, None] * np.cos(g1)[None, :, None] * np.cos(g1)[None, None, :]
              + 0.05 * np.random.default_rng(4).standard_normal(n3)).astype(np.float32)
        f128 = F.ffts("float32").init(*n3)
        u = torch.from_numpy(u0).to(dev).requires_grad_(True)
        kx = torch.fft.fftfreq(128, 1.0 / 128, device=dev)
        kzz = torch.arange(65, device=dev, dtype=torch.float32)
        G = torch.exp(-(kx[:, None, None] ** 2 + kx[None, :, None] ** 2 + kzz[None, None, :] ** 2)
                      / (2 * 16.0 ** 2)).to(torch.complex64)

        def composed():
            u.grad = None
            w = A.poisson(A.c2r(A.r2c(u, f128) * G, f128, normalized=True), f128, -1.0)
            (0.5 * (w * w).sum()).backward()

        def fused():
            u.grad = None
            w = A.filter_poisson(u, f128, 16.0, -1.0)
            (0.5 * (w * w).sum()).backward()

        rt128 = 2 * (4 * 128 ** 3 + 8 * 128 * 128 * 65)
        tc = statistics.median(time_events(composed, 30))
        gc = u.grad.clone()
        tf = statistics.median(time_events(fused, 30))
        gfu = u.grad.clone()
        more["pipeline_128_grad"] = {
            "workload": "128^3 f32 loss 0.5|Poisson(C2R(G R2C(u)))|^2, G Gaussian sigma 16, forward + adjoint gradient",
            "composed": {"median_us": tc * 1e3, "value": 4 * rt128 / (tc * 1e-3) / 1e9, "unit": "GB/s",
                         "alg_bytes": 4 * rt128},
            "fused": {"median_us": tf * 1e3, "value": 2 * rt128 / (tf * 1e-3) / 1e9, "unit": "GB/s",
                      "alg_bytes": 2 * rt128},
            "grad_rel_l2_fused_vs_composed": float(torch.linalg.norm(gfu - gc) / torch.linalg.norm(gc))}
        del u, G, gc, gfu, f128
    except Exception as exc:  # noqa: BLE001
        more["pipeline_128_grad"] = {"unavailable": str(exc)[:200]}

    # batched uneven 3D transforms: 512 shapes with every axis drawn from {32, 48, 64, 96, 128}
    # (numpy default_rng(2)); one step = the R2C + normalised C2R round trip of every transform.
    # The execution mode and knobs come from the autotuner (fresh cache per run): the grouped
    # launches (one per stage and line length) or the single persistent launch, each replayed
    # from a CUDA graph; the persistent launch and 2560 sequential plain launches of the same
    # batch are timed beside it.  With N > 1 each rank runs its LPT share.
    bat = None
    try:
        import tempfile

        import fftm_b200.autotune as AT
        import fftm_b200.batch as B
        shapes = B.draw_shapes(512, seed=2)
        mine = [shapes[i] for i in replicas.shard(shapes, rank, world)]
        bt = B.Batch(mine)
        gen = torch.Generator(device=dev).manual_seed(2 + rank)
        bx = torch.rand(bt.real_total, device=dev, generator=gen) * 2 - 1
        by = torch.empty_like(bx)
        bbytes = bt.algorithmic_bytes()
        with tempfile.TemporaryDirectory() as td:
            sel = bt.autotune(B.ROUNDTRIP, os.path.join(td, "batch.env"),
                              measured=AT.measured_options(warmup=2, iterations=5))

        def time_batch(mode, n):
            for _ in range(2):
                bt.exec(B.ROUNDTRIP, bx, by, mode=mode)
            torch.cuda.synchronize()
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
            for a, b in evs:
                flush.zero_()
                a.record(stream)
                bt.exec(B.ROUNDTRIP, bx, by, mode=mode)
                b.record(stream)
            torch.cuda.synchronize()
            return sum(a.elapsed_time(b) for a, b in evs)

        if dist is not None:
            dist.barrier()
        tuned_ms = replicas.max_over_ranks(dist, time_batch(bt.mode, 10), dev) / 10
        berr = float(torch.linalg.norm(by - bx) / torch.linalg.norm(bx))
        seq_ms = replicas.max_over_ranks(dist, time_batch(B.SEQUENTIAL, 5), dev) / 5
        pers_ms = replicas.max_over_ranks(dist, time_batch(B.GRAPH, 10), dev) / 10
        pers_status = bt.status(B.ROUNDTRIP)
        total_bytes = sum(B.transform_bytes(s_) for s_ in shapes)
        bat = {"workload": "512 uneven 3D f32 R2C + normalised C2R round trips, axes from {32,48,64,96,128}, "
                           "numpy default_rng(2)",
               "ms_per_step": tuned_ms, "value": total_bytes / (tuned_ms * 1e-3) / 1e9, "unit": "GB/s",
               "bytes_per_step": total_bytes, "bytes_this_rank": bbytes,
               "tuned": {k: sel.config.get(k) for k in ("FFTM_AUTOTUNE_STRATEGY_3D", "FFTB_AUTOTUNE_BATCH_MODE",
                                                       "FFTB_AUTOTUNE_TILES_SCALE", "FFTB_AUTOTUNE_CTAS_PER_SM")},
               "candidates_median_ms": sel.medians_ms(),
               "mode": {0: "sequential", 1: "persistent", 2: "persistent, graph", 3: "grouped",
                        4: "grouped, graph"}[bt.mode],
               "graph_launches_per_step": 1 if bt.mode in (B.GRAPH, B.GROUPED_GRAPH) else None,
               "round_trip_rel_l2": berr,
               "persistent_single_launch": {"ms_per_step": pers_ms, "value": total_bytes / (pers_ms * 1e-3) / 1e9,
                                            "kernel_launches_per_step": 1, "wait_error_flag": pers_status},
               "sequential_plain_launches": {"ms_per_step": seq_ms,
                                             "value": total_bytes / (seq_ms * 1e-3) / 1e9,
                                             "launches_per_step": bt.describe(B.ROUNDTRIP)["passes"]}}
        del bx, by, bt
    except Exception as exc:  # noqa: BLE001
        bat = {"unavailable": str(exc)[:200]}

    # the same solve through cuFFT (torch.fft: R2C, multiply by -1/|k|^2, C2R with 1/N), the
    # library the reference's ffts wraps, timed with the same flush / event protocol
    cufft = None
    try:
        kx = torch.fft.fftfreq(NX, 1.0 / NX, device=dev)[:, None, None]
        ky = torch.fft.fftfreq(NY, 1.0 / NY, device=dev)[None, :, None]
        kz = torch.arange(NZ // 2 + 1, device=dev, dtype=torch.float32)[None, None, :]
        k2 = kx * kx + ky * ky + kz * kz
        mult = torch.where(k2 == 0, torch.zeros_like(k2), -1.0 / k2).to(torch.float32)

        def cufft_step():
            X = torch.fft.rfftn(rhs)
            X.mul_(mult)
            return torch.fft.irfftn(X, s=(NX, NY, NZ))

        for _ in range(3):
            flush.zero_()
            cufft_step()
        torch.cuda.synchronize()
        cs = [torch.cuda.Event(enable_timing=True) for _ in range(20)]
        ce = [torch.cuda.Event(enable_timing=True) for _ in range(20)]
        for i in range(20):
            flush.zero_()
            cs[i].record(stream)
            cufft_step()
            ce[i].record(stream)
        torch.cuda.synchronize()
        cms = sum(a.elapsed_time(b) for a, b in zip(cs, ce)) / 20
        cufft = {"impl": "torch.fft (cuFFT) rfftn, multiply, irfftn", "ms_per_step": cms,
                 "value": BYTES_RT / (cms * 1e-3) / 1e9, "unit": "GB/s"}
    except Exception as exc:  # noqa: BLE001
        cufft = {"unavailable": str(exc)[:200]}

    # the reference's own cuFFT ffts path (tests/cufft_ref: the exact cufftMakePlanMany64 plans
    # of source/ffts.hpp and source/fftm.hpp, auto-allocation off, its transposes and separate
    # multiply / 1/N kernels) on the same GPU, inputs and flush / event protocol
    refc = None
    try:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import cufft_ref
        cufft_ref.build()
        refc = {"impl": "reference ffts over cuFFT (cufftMakePlanMany64 plans of source/ffts.hpp:677-776, "
                        "source/fftm.hpp:2941-2961; separate Poisson multiply and 1/N kernels)"}
        r3 = cufft_ref.RefFfts("float32", (NX, NY, NZ))
        rspec = torch.empty(ff.spectrum_shape(), dtype=torch.complex64, device=dev)
        rsol = torch.empty_like(rhs)
        t = statistics.median(time_events(lambda: r3.poisson(rhs, rspec, rsol, -1.0), 30))
        refc["poisson_256"] = {"median_us": t * 1e3, "value": BYTES_RT / (t * 1e-3) / 1e9, "unit": "GB/s",
                               "fftb_speedup": t * 1e3 / statistics.median([x * 1e3 for x in step_ms]),
                               "rel_l2_vs_fftb": float(torch.linalg.norm(rsol - sol) / torch.linalg.norm(sol))}
        xr = torch.from_numpy(np.random.default_rng(0).uniform(-1, 1, (NX, NY, NZ)).astype(np.float32)).to(dev)
        yr = torch.empty_like(xr)
        t = statistics.median(time_events(lambda: (r3.forward(xr, rspec), r3.backward_normalized(rspec, yr)), 30))
        refc["roundtrip_256"] = {"median_us": t * 1e3, "value": BYTES_RT / (t * 1e-3) / 1e9, "unit": "GB/s",
                                 "round_trip_rel_l2": float(torch.linalg.norm(yr - xr) / torch.linalg.norm(xr))}
        if "median_us" in more.get("roundtrip_256", {}):
            refc["roundtrip_256"]["fftb_speedup"] = t * 1e3 / more["roundtrip_256"]["median_us"]
        del r3, rspec, rsol, xr, yr
        d4 = (64, 64, 64, 64)
        r4 = cufft_ref.RefFfts("float32", d4, "native_xzwy")
        x4r = torch.from_numpy(np.random.default_rng(1).standard_normal(d4).astype(np.float32)).to(dev)
        y4r = torch.empty_like(x4r)
        s4r = torch.empty((64, 64, 33, 64), dtype=torch.complex64, device=dev)
        t = statistics.median(time_events(lambda: (r4.forward(x4r, s4r), r4.backward_normalized(s4r, y4r)), 20))
        b4 = 2 * (4 * 64 ** 4 + 8 * 64 ** 3 * 33)
        refc["roundtrip4d_64_native"] = {"median_us": t * 1e3, "value": b4 / (t * 1e-3) / 1e9, "unit": "GB/s",
                                         "round_trip_rel_l2": float(torch.linalg.norm(y4r - x4r) /
                                                                    torch.linalg.norm(x4r)),
                                         "note": "the reference waits on the host after each transpose"}
        if sec and "ms_per_step" in sec:
            refc["roundtrip4d_64_native"]["fftb_speedup"] = t / sec["ms_per_step"]
        del r4, x4r, y4r, s4r
    except Exception as exc:  # noqa: BLE001
        refc = {"unavailable": str(exc)[:200]}

    # accuracy of the timed solution against the analytic solution of the smooth part is not
    # defined (the noise term has no closed form); the CPU leg checks it against the FP64 oracle.
    result = sol.detach().cpu().numpy()

    line = {
        "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "step_stats_us": {"mean": statistics.mean(step_ms) * 1e3, "median": statistics.median(step_ms) * 1e3,
                          "stdev": (statistics.stdev(step_ms) if len(step_ms) > 1 else 0.0) * 1e3,
                          "min": min(step_ms) * 1e3},
        "gflops": FLOPS_RT / (total_ms / args.steps * 1e-3) / 1e9,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": DATA,
        "config": {"workload": WORKLOAD, "n": [NX, NY, NZ], "bytes_per_step": BYTES_RT,
                   "strategy": tuned.config.get("FFTM_AUTOTUNE_STRATEGY_3D") if tuned else args.strategy,
                   "autotune_median_ms": tuned.medians_ms() if tuned else None,
                   "l2": "flushed between steps (1 GiB write outside the timed window)",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "gpu_launches": launches_per_step * args.steps,
        "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic},
        "kernels": kernels,
        "e2e": {"value": e2e_val, "unit": "GB/s", "h2d_bytes_per_step": int(rhs.numel() * 4),
                "d2h_bytes_per_step": int(sol.numel() * 4), "steps": e2e_steps,
                "ms_per_step": e2e_ms / e2e_steps,
                "pipelining": "two buffer sets, three streams: upload of step i+1 and download of step i-1 overlap the solve of step i",
                "serial_ms_per_step": e2e_serial_ms / e2e_steps,
                "serial_value": BYTES_RT * e2e_steps / (e2e_serial_ms * 1e-3) / 1e9,
                "solutions_identical": e2e_ok},
        "clocks": clk,
        "reference_cufft": refc,
        "cufft_same_gpu": cufft,
        "secondary": sec,
        "batched": bat,
        "more": more,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, secs, threads, ref = cpu_oracle_rate(f_host, 1)
        num = np.linalg.norm((result.astype(np.float64) - ref).ravel())
        line["cpu_baseline"] = {"value": rate, "unit": "GB/s", "cores": threads, "kind": "port",
                                "sample": "one full 256^3 FP64 Poisson solve (oracle/fft_oracle.c, OpenMP)",
                                "seconds": secs}
        line["accuracy"] = {"rel_l2_vs_fp64_oracle": float(num / np.linalg.norm(ref.ravel()))}
        line["cpu_scipy_fft"] = scipy_fft_rates(f_host)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
