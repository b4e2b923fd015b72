"""GPU tests of the ffts profiling options (the reference's ffts_init_options,
source/ffts.hpp:64-72, and its print-on-destroy, :199-208, :449-476): per-scope calls with
host and device times, the memory profile of the object's own allocations, the reports
printed when the object is destroyed, and profilers off when the keys are empty."""
import gc

import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def F(torch_cuda):
    from fftm_b200 import build
    build.build()
    import fftm_b200
    return fftm_b200


def test_profile_scopes_and_memory(F, torch_cuda):
    torch = torch_cuda
    opts = F.ffts_init_options("p", "m", False, False, False, False)
    f = F.ffts("float32").init(64, 64, 64, options=opts)
    x = torch.rand((64, 64, 64), device="cuda")
    spec = torch.empty(f.spectrum_shape(), dtype=torch.complex64, device="cuda")
    y = torch.empty_like(x)
    for _ in range(3):
        f.forward(x, spec)
    f.poisson(x, y, -1.0)
    torch.cuda.synchronize()
    rep = f.profile_report("summary")
    assert rep.startswith("Profile p:")
    line = [l for l in rep.splitlines() if "ffts::forward<3>:" in l][0]
    assert "calls=3" in line
    dev_total = float(line.split("device_ms(total/avg)=")[1].split("/")[0])
    assert dev_total > 0
    assert "ffts::init<3>: calls=1" in rep and "ffts::poisson<3>: calls=1" in rep
    assert "calls=5" in f.profile_report("totals")
    mem = f.profile_report("memory")
    assert f"ffts/shared_work_buffer: current(sum/max/avg)={f.work_size}/" in mem
    assert "Memory profile categories:" in mem and "device: current" in mem
    assert f"total: current(sum/max/avg)={f.work_size}/" in f.profile_report("memory_totals")


def test_reports_printed_on_destroy(F, torch_cuda, capfd):
    torch = torch_cuda
    f = F.ffts("float32").init(32, 32, 32, options=F.ffts_init_options())
    x = torch.rand((32, 32, 32), device="cuda")
    spec = torch.empty(f.spectrum_shape(), dtype=torch.complex64, device="cuda")
    f.forward(x, spec)
    torch.cuda.synchronize()
    capfd.readouterr()
    del f
    gc.collect()
    out = capfd.readouterr().out
    for head in ("Profile ffts_prof:", "Profile totals ffts_prof:", "Memory profile:", "Memory profile totals:"):
        assert head in out, out


def test_profilers_off(F, torch_cuda, capfd):
    torch = torch_cuda
    quiet = F.fftm_reporting_options().to_ffts_init_options()   # fftm's defaults: all off
    f = F.ffts("float32").init(32, 32, 32, options=quiet)
    x = torch.rand((32, 32, 32), device="cuda")
    spec = torch.empty(f.spectrum_shape(), dtype=torch.complex64, device="cuda")
    f.forward(x, spec)
    torch.cuda.synchronize()
    assert f.profile_report("summary") == "" and f.profile_report("memory") == ""
    capfd.readouterr()
    del f
    gc.collect()
    assert capfd.readouterr().out == ""
    p = F.profiling_reporting_options().to_ffts_init_options()
    assert (p.profiling_key, p.memory_profiling_key) == ("fftm_prof", "fftm_mem")
