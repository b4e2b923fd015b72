"""fftm_b200 -- B200-native (sm_100a) single-GPU transform path of fftm.

Python mirror of the reference's interfaces over the C ABI (include/fftb.h),
for tests, benchmarks and PyTorch users.  Device memory and streams come from
PyTorch; all transform work runs in ``libfftb_b200.so`` (hand-written CUDA).

* :class:`Plan` -- one plan with cuFFT advanced-layout parameters, the role of
  ``cufft::fft<T, D>`` (reference source/external_wrap/cufft_wrap.h:483-1282).
* :class:`fft_wrap_many` -- the named plan registry ``BaseFFT`` contract of
  ``ffts`` (source/external_wrap/fft_wrap_many.h:25-447).
* :class:`ffts` -- the single-GPU frontend (source/ffts.hpp:159-383): init /
  forward / backward for 2D, 3D and 4D, plus the fused Poisson solve.

Error behaviour follows the reference: API misuse raises :class:`LogicError`
(``std::logic_error``), library failures :class:`FftbError`
(``std::runtime_error``), unknown plan names ``KeyError`` (``std::out_of_range``).
"""
from __future__ import annotations

import ctypes

from . import _lib

R2C, C2R, C2CF, C2CB = 1, 2, 3, 4   # fftm::direction (source/fft_direction.h:9-15)
F32, F64 = 0, 1
PENCIL, SLAB, NATIVE_XZWY = 0, 1, 2

_STRATEGY = {"pencil": PENCIL, "pencil_pencil": PENCIL, "slab": SLAB, "slab_slab": SLAB,
             "native_xzwy": NATIVE_XZWY, PENCIL: PENCIL, SLAB: SLAB, NATIVE_XZWY: NATIVE_XZWY}


class FftbError(RuntimeError):
    """A failure inside the library (the reference throws std::runtime_error)."""

    def __init__(self, status: int, where: str = ""):
        self.status = status
        msg = _lib.status_string(status)
        detail = _lib.last_error_message()
        super().__init__(f"{where}: {msg}" + (f" ({detail})" if detail else ""))


class LogicError(RuntimeError):
    """API misuse (the reference throws std::logic_error)."""


_LOGIC = {-6, -7, -8}


def _check(st: int, where: str) -> None:
    if st != 0:
        if st in _LOGIC:
            raise LogicError(_lib.status_string(st))
        raise FftbError(st, where)


def _torch():
    import torch
    return torch


def _dtype_code(dtype) -> int:
    torch = _torch()
    if dtype in (torch.float32, torch.complex64, "float32", "f32", F32):
        return F32
    if dtype in (torch.float64, torch.complex128, "float64", "f64", F64):
        return F64
    raise ValueError(f"unsupported dtype {dtype}")


def _ptr(t) -> int:
    if t is None:
        return 0
    if not t.is_cuda:
        raise ValueError("fftb operates on CUDA tensors")
    return t.data_ptr()


def _stream_ptr(stream=None) -> int:
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def version() -> str:
    return _lib.load().fftb_version().decode()


def build_digest() -> str:
    """Digest of the sources the loaded library was compiled from (fftb_build_digest)."""
    return _lib.load().fftb_build_digest().decode()


# ====================================================================== plans
class Plan:
    """One transform plan (the role of cufft::fft<T, D>).

    Arguments have cuFFT advanced-layout meaning exactly as
    ``fft_wrap_many::add_plan_{1D,2D,3D}`` passes them; ``inembed``/``onembed``
    ``None`` selects the default layout (cufft_wrap.h:568-587)."""

    def __init__(self, direction, n, inembed=None, istride=1, idist=0, onembed=None, ostride=1, odist=0,
                 batch=1, dtype="float32"):
        L = _lib.load()
        self.direction = int(direction)
        self.dtype = _dtype_code(dtype)
        n = list(n)
        rank = len(n)
        arr = ctypes.c_longlong * 3
        nn = arr(*(n + [0] * (3 - rank)))
        ie = arr(*(list(inembed) + [0] * (3 - rank))) if inembed is not None else None
        oe = arr(*(list(onembed) + [0] * (3 - rank))) if onembed is not None else None
        h = ctypes.c_void_p()
        ws = ctypes.c_size_t()
        st = L.fftb_plan_create(self.direction, self.dtype, rank, nn, ie, istride, idist, oe, ostride, odist,
                                batch, ctypes.byref(h), ctypes.byref(ws))
        _check(st, "fftb_plan_create")
        self._h = h
        self.work_size = ws.value

    def __del__(self):
        h = getattr(self, "_h", None)
        try:
            if h is not None and h.value:
                _lib.load().fftb_plan_destroy(h)
        except Exception:
            pass
        self._h = None

    def set_stream(self, stream=None):
        _check(_lib.load().fftb_plan_set_stream(self._h, _stream_ptr(stream)), "set_stream")

    def set_work_area(self, tensor_or_ptr):
        ptr = tensor_or_ptr if isinstance(tensor_or_ptr, int) else _ptr(tensor_or_ptr)
        _check(_lib.load().fftb_plan_set_work_area(self._h, ptr), "set_work_area")

    def get_work_size(self) -> int:
        return self.work_size

    def exec(self, inp, out, stream=None):
        """Asynchronous execution on ``stream`` (torch's current stream by default)."""
        self.set_stream(stream)
        _check(_lib.load().fftb_exec(self._h, _ptr(inp), _ptr(out)), "exec")

    exec_no_sync = exec

    def exec_direction(self, direction, inp, out, stream=None):
        self.set_stream(stream)
        _check(_lib.load().fftb_exec_direction(self._h, int(direction), _ptr(inp), _ptr(out)), "exec_direction")

    def get_direction(self) -> int:
        return self.direction

    def descriptor(self) -> dict:
        L = _lib.load()
        d, dt, r = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        arr = ctypes.c_longlong * 3
        n, ie, oe = arr(), arr(), arr()
        vals = [ctypes.c_longlong() for _ in range(5)]
        _check(L.fftb_plan_describe(self._h, ctypes.byref(d), ctypes.byref(dt), ctypes.byref(r), n, ie,
                                    ctypes.byref(vals[0]), ctypes.byref(vals[1]), oe, ctypes.byref(vals[2]),
                                    ctypes.byref(vals[3]), ctypes.byref(vals[4])), "describe")
        rk = r.value
        return {"dir": d.value, "dtype": dt.value, "rank": rk, "n": list(n)[:rk], "inembed": list(ie)[:rk],
                "istride": vals[0].value, "idist": vals[1].value, "onembed": list(oe)[:rk],
                "ostride": vals[2].value, "odist": vals[3].value, "batch": vals[4].value}

    def num_launches(self) -> int:
        v = ctypes.c_int()
        _check(_lib.load().fftb_plan_num_launches(self._h, ctypes.byref(v)), "num_launches")
        return v.value


class fft_wrap_many:
    """Named plan registry with the ``BaseFFT`` contract of fftm::ffts
    (source/external_wrap/fft_wrap_many.h:25-447)."""

    def __init__(self, dtype="float32"):
        self.dtype = dtype
        self._plans: dict[str, Plan] = {}
        self._activated = False
        self._external = False
        self.work_area_size = 0

    def add_plan(self, direction, name, n, inembed, istride, idist, onembed, ostride, odist, batch):
        if self._activated:
            raise LogicError("fft_wrap_many::add_plan: cannot add new plans after activation.")
        self._plans[name] = Plan(direction, n, inembed, istride, idist, onembed, ostride, odist, batch, self.dtype)

    def add_plan_1D(self, direction, name, n, inembed, istride, idist, onembed, ostride, odist, batch):
        self.add_plan(direction, name, [n], [inembed], istride, idist, [onembed], ostride, odist, batch)

    def add_plan_1D_default(self, direction, name, n, batch):
        if self._activated:
            raise LogicError("fft_wrap_many::add_plan_1D_default: cannot add new plans after activation.")
        self._plans[name] = Plan(direction, [n], batch=batch, dtype=self.dtype)

    def add_plan_2D(self, direction, name, n0, n1, inembed0, inembed1, istride, idist, onembed0, onembed1, ostride,
                    odist, batch):
        self.add_plan(direction, name, [n0, n1], [inembed0, inembed1], istride, idist, [onembed0, onembed1],
                      ostride, odist, batch)

    def add_plan_3D(self, direction, name, n0, n1, n2, inembed0, inembed1, inembed2, istride, idist, onembed0,
                    onembed1, onembed2, ostride, odist, batch):
        self.add_plan(direction, name, [n0, n1, n2], [inembed0, inembed1, inembed2], istride, idist,
                      [onembed0, onembed1, onembed2], ostride, odist, batch)

    def activate_work_size(self) -> int:
        for p in self._plans.values():
            self.work_area_size = max(self.work_area_size, p.get_work_size())
        return self.work_area_size

    def activate(self):
        if self._activated:
            raise LogicError("fft_wrap_many::activate: cannot activate again.")
        self.activate_work_size()
        self._activated = True

    def set_external_work_area(self, ptr):
        if self._activated:
            raise LogicError("fft_wrap_many::set_external_work_area: cannot set external work_area with "
                             "activated local work_area.")
        for p in self._plans.values():
            p.set_work_area(ptr)
        self._external = True

    def get_work_size(self) -> int:
        return self.work_area_size

    def exec(self, name, inp, out, stream=None):
        self._plans[name].exec(inp, out, stream)   # KeyError = std::out_of_range

    exec_named_no_sync = exec

    def exec_raw_direction(self, name, direction, inp, out, stream=None):
        self._plans[name].exec_direction(direction, inp, out, stream)

    def release(self):
        self._plans.clear()


# ====================================================================== ffts
class ffts_init_options:
    """The reference's ffts_init_options (source/ffts.hpp:64-72), with its defaults: both
    profilers on (keys "ffts_prof" / "ffts_mem") and every report printed on destroy.  An
    empty key turns that profiler off."""

    def __init__(self, profiling_key="ffts_prof", memory_profiling_key="ffts_mem",
                 print_profile_summary_on_destroy=True, print_profile_totals_on_destroy=True,
                 print_memory_profile_on_destroy=True, print_memory_totals_on_destroy=True):
        self.profiling_key = profiling_key
        self.memory_profiling_key = memory_profiling_key
        self.print_profile_summary_on_destroy = print_profile_summary_on_destroy
        self.print_profile_totals_on_destroy = print_profile_totals_on_destroy
        self.print_memory_profile_on_destroy = print_memory_profile_on_destroy
        self.print_memory_totals_on_destroy = print_memory_totals_on_destroy

    def _c(self):
        o = _lib.InitOptions()
        o.profiling_key = (self.profiling_key or "").encode()
        o.memory_profiling_key = (self.memory_profiling_key or "").encode()
        o.print_profile_summary_on_destroy = int(bool(self.print_profile_summary_on_destroy))
        o.print_profile_totals_on_destroy = int(bool(self.print_profile_totals_on_destroy))
        o.print_memory_profile_on_destroy = int(bool(self.print_memory_profile_on_destroy))
        o.print_memory_totals_on_destroy = int(bool(self.print_memory_totals_on_destroy))
        return o


class fftm_reporting_options:
    """fftm's reporting options (source/fftm_options.hpp:220-241), defaults all off; the
    single-GPU path maps them onto ffts_init_options (to_ffts_init_options)."""

    def __init__(self, profiling_key="", memory_profiling_key="", verbose=False,
                 print_profile_summary_on_destroy=False, print_profile_totals_on_destroy=False,
                 print_memory_profile_on_destroy=False, print_memory_totals_on_destroy=False):
        self.profiling_key = profiling_key
        self.memory_profiling_key = memory_profiling_key
        self.verbose = verbose
        self.print_profile_summary_on_destroy = print_profile_summary_on_destroy
        self.print_profile_totals_on_destroy = print_profile_totals_on_destroy
        self.print_memory_profile_on_destroy = print_memory_profile_on_destroy
        self.print_memory_totals_on_destroy = print_memory_totals_on_destroy

    def to_ffts_init_options(self) -> ffts_init_options:
        return ffts_init_options(self.profiling_key, self.memory_profiling_key,
                                 self.print_profile_summary_on_destroy, self.print_profile_totals_on_destroy,
                                 self.print_memory_profile_on_destroy, self.print_memory_totals_on_destroy)


def profiling_reporting_options() -> fftm_reporting_options:
    """fftm's profiling preset (source/fftm_options.hpp:231-242): keys "fftm_prof" /
    "fftm_mem", every report printed on destroy."""
    return fftm_reporting_options("fftm_prof", "fftm_mem", False, True, True, True, True)


class ffts:
    """The single-GPU frontend (fftm::ffts, source/ffts.hpp:159-383).

    ``strategy_4d``: ``"pencil"`` (strategy_4d_pencil_pencil, real [w][z][y][x]),
    ``"slab"`` (strategy_4d_slab_slab, real [x][y][z][w]) or ``"native_xzwy"``
    (fftm's native slab spectrum [ky][kz][kw][kx])."""

    def __init__(self, dtype="float32", strategy_4d="pencil"):
        self.dtype = _dtype_code(dtype)
        self.strategy_4d = _STRATEGY[strategy_4d]
        self._h = None
        self._dims = None
        self._work = None

    def init(self, nx, ny, nz=None, nw=None, options=None):
        """``options``: an ``ffts_init_options`` (profiling keys and print-on-destroy flags);
        None keeps both profilers off (the C++ layer defaults to the reference's options,
        which print on destroy)."""
        if self._h is not None:
            raise LogicError("ffts::init can only be called once per instance.")
        L = _lib.load()
        h = ctypes.c_void_p()
        if options is None:
            _check(L.fftb_ffts_create(self.dtype, nx, ny, nz or 0, nw or 0, self.strategy_4d, ctypes.byref(h)),
                   "ffts::init")
        else:
            o = options._c()
            _check(L.fftb_ffts_create_ex(self.dtype, nx, ny, nz or 0, nw or 0, self.strategy_4d, ctypes.byref(o),
                                         ctypes.byref(h)), "ffts::init")
        self._h = h
        self._dims = tuple(d for d in (nx, ny, nz, nw) if d)
        ws = ctypes.c_size_t()
        _check(L.fftb_ffts_work_size(h, ctypes.byref(ws)), "work_size")
        self.work_size = ws.value
        return self

    def __del__(self):
        h = getattr(self, "_h", None)
        try:
            if h is not None and h.value:
                _lib.load().fftb_ffts_destroy(h)
        except Exception:
            pass
        self._h = None

    def is_initialized(self) -> bool:
        return self._h is not None

    def profile_report(self, which="summary") -> str:
        """The profilers' reports as text: "summary", "totals", "memory" or "memory_totals"
        (empty when that profiler is off)."""
        self._ensure()
        w = {"summary": 0, "totals": 1, "memory": 2, "memory_totals": 3}[which]
        L = _lib.load()
        need = ctypes.c_size_t()
        _check(L.fftb_ffts_profile_report(self._h, w, None, 0, ctypes.byref(need)), "profile_report")
        buf = ctypes.create_string_buffer(need.value)
        _check(L.fftb_ffts_profile_report(self._h, w, buf, need.value, ctypes.byref(need)), "profile_report")
        return buf.value.decode()

    def _ensure(self, dim=None):
        if self._h is None:
            raise LogicError("ffts: call init() before using the transform.")
        if dim is not None and len(self._dims) != dim:
            raise LogicError(f"ffts: initialized for {len(self._dims)}D but used as {dim}D.")

    def dimension(self) -> int:
        self._ensure()
        return len(self._dims)

    @property
    def dims(self):
        return self._dims

    def set_work_area(self, tensor):
        self._ensure()
        self._work = tensor
        _check(_lib.load().fftb_ffts_set_work_area(self._h, _ptr(tensor)), "set_work_area")

    def _bind(self, stream):
        _check(_lib.load().fftb_ffts_set_stream(self._h, _stream_ptr(stream)), "set_stream")

    def forward(self, real_in, complex_out, stream=None):
        self._ensure(real_in.dim() if real_in.dim() in (2, 3, 4) else None)
        self._bind(stream)
        _check(_lib.load().fftb_ffts_forward(self._h, _ptr(real_in), _ptr(complex_out)), "ffts::forward")

    def backward(self, complex_in, real_out, stream=None, normalized=False):
        """Unnormalised C2R; ``complex_in`` may be overwritten (as the reference's)."""
        self._ensure(real_out.dim() if real_out.dim() in (2, 3, 4) else None)
        self._bind(stream)
        fn = _lib.load().fftb_ffts_backward_normalized if normalized else _lib.load().fftb_ffts_backward
        _check(fn(self._h, _ptr(complex_in), _ptr(real_out)), "ffts::backward")

    def forward_adjoint(self, grad_spectrum, grad_real, stream=None):
        """Transpose of forward(): grad_real = C2R(W * grad_spectrum), W = 1/2 on interior
        half-axis bins.  grad_spectrum may be overwritten."""
        self._ensure()
        self._bind(stream)
        _check(_lib.load().fftb_ffts_forward_adjoint(self._h, _ptr(grad_spectrum), _ptr(grad_real)),
               "ffts::forward_adjoint")

    def backward_adjoint(self, grad_real, grad_spectrum, stream=None):
        """Transpose of the unnormalised backward(): grad_spectrum = W2 * R2C(grad_real)."""
        self._ensure()
        self._bind(stream)
        _check(_lib.load().fftb_ffts_backward_adjoint(self._h, _ptr(grad_real), _ptr(grad_spectrum)),
               "ffts::backward_adjoint")

    def poisson(self, rhs, solution, sign=-1.0, stream=None):
        """u = C2R(sign * R2C(f) / |k|^2) / N, k=0 -> 0, fused into the FFT passes."""
        self._ensure()
        self._bind(stream)
        _check(_lib.load().fftb_ffts_poisson(self._h, _ptr(rhs), _ptr(solution), float(sign)), "ffts::poisson")

    def filter(self, inp, out, sigma, poisson_sign=0.0, stream=None):
        self._ensure()
        self._bind(stream)
        _check(_lib.load().fftb_ffts_filter(self._h, _ptr(inp), _ptr(out), float(sigma), float(poisson_sign)),
               "ffts::filter")

    def spectrum_poisson(self, spectrum, sign=-1.0, scale=1.0, stream=None):
        self._ensure()
        self._bind(stream)
        _check(_lib.load().fftb_ffts_spectrum_poisson(self._h, _ptr(spectrum), float(sign), float(scale)),
               "spectrum_poisson")

    def spectrum_derivative(self, spec_in, spec_out, axis, scale=1.0, stream=None):
        """spec_out = i k_axis spec_in * scale (axis 0 = x, 1 = y, 2 = z, 3 = w)."""
        self._ensure()
        self._bind(stream)
        _check(_lib.load().fftb_ffts_spectrum_derivative(self._h, _ptr(spec_in), _ptr(spec_out), int(axis),
                                                         float(scale)), "spectrum_derivative")

    def gradient(self, u, outs, stream=None):
        """outs[a] = du/d(axis a) for every axis, from one forward transform."""
        self._ensure()
        self._bind(stream)
        if len(outs) != len(self._dims):
            raise ValueError(f"gradient needs {len(self._dims)} outputs")
        arr = (ctypes.c_void_p * len(outs))(*[_ptr(o) for o in outs])
        _check(_lib.load().fftb_ffts_gradient(self._h, _ptr(u), arr), "gradient")

    def spectrum_truncate(self, spectrum, rule="two_thirds", cutoff=0, stream=None):
        """Zero the modes outside |k_a| <= n_a / 3 ("two_thirds") or |k_a| <= cutoff ("box")."""
        self._ensure()
        self._bind(stream)
        code = {"two_thirds": 0, "box": 1}[rule]
        _check(_lib.load().fftb_ffts_spectrum_truncate(self._h, _ptr(spectrum), code, int(cutoff)),
               "spectrum_truncate")

    def derivative(self, u, out, axis, stream=None):
        """du/d(axis) of a periodic field on [0, 2 pi)^d (spectral, fused R2C / C2R)."""
        self._ensure()
        self._bind(stream)
        _check(_lib.load().fftb_ffts_derivative(self._h, _ptr(u), _ptr(out), int(axis)), "derivative")

    def num_launches(self, which="forward") -> int:
        self._ensure()
        code = {"forward": 0, "backward": 1, "poisson": 2, "filter": 3}[which]
        v = ctypes.c_int()
        _check(_lib.load().fftb_ffts_num_launches(self._h, code, ctypes.byref(v)), "num_launches")
        return v.value

    # ------------------------------------------------------------------ strategy / autotune
    def set_strategy(self, strategy="auto", plane_cluster=0):
        """"auto", "fused" (multi-axis kernels; plane_cluster 1, 2, 4 or 8 CTAs per 3D
        plane, 0 by occupancy), "fused_tc" (fused, with the column kernels' first radix-16
        stage on the tensor cores in split FP16) or "staged" (one pass kernel per axis)."""
        self._ensure()
        code = {"auto": 0, "fused": 1, "staged": 2, "fused_tc": 3}[strategy]
        _check(_lib.load().fftb_ffts_set_strategy(self._h, code, int(plane_cluster)), "set_strategy")

    def strategy(self):
        """(strategy in effect, plane cluster size)."""
        self._ensure()
        s, c = ctypes.c_int(), ctypes.c_int()
        _check(_lib.load().fftb_ffts_get_strategy(self._h, ctypes.byref(s), ctypes.byref(c)), "get_strategy")
        return {1: "fused", 2: "staged", 3: "fused_tc"}[s.value], c.value

    def apply_config(self, config):
        """Applies a tuned config (dict or KEY=VALUE text) to this object."""
        from . import autotune as _at
        self._ensure()
        text = config if isinstance(config, str) else _at.to_text(config)
        _check(_lib.load().fftb_ffts_apply_config(self._h, text.encode()), "apply_config")

    def autotune(self, cache_file, options=None, measured=None):
        """load_or_measure for this object's problem, then applies the winner; returns
        the selected config."""
        from . import autotune as _at
        self._ensure()
        opts = options or _at.autotune_options()
        opts.cache_file = str(cache_file)
        dt = "float32" if self.dtype == F32 else "float64"
        sel = _at.load_or_measure_config(dt, self._dims, opts, measured, strategy_4d=self.strategy_4d)
        self.apply_config(sel.config)
        return sel

    def timing_enable(self, max_launches=4096):
        """Per-launch device timing of later calls (profiling hook)."""
        self._ensure()
        _check(_lib.load().fftb_ffts_timing_enable(self._h, int(max_launches)), "timing_enable")

    def timing_read(self, cap=65536):
        """[(kernel name, ms, algorithmic bytes)] of the launches recorded since the last read."""
        self._ensure()
        ms = (ctypes.c_float * cap)()
        by = (ctypes.c_double * cap)()
        stride = 96
        names = ctypes.create_string_buffer(stride * cap)
        n = ctypes.c_int()
        _check(_lib.load().fftb_ffts_timing_read(self._h, ms, by, names, stride, cap, ctypes.byref(n)),
               "timing_read")
        raw = names.raw
        out = []
        for i in range(n.value):
            nm = raw[i * stride:(i + 1) * stride].split(b"\0", 1)[0].decode()
            out.append((nm, float(ms[i]), float(by[i])))
        return out

    # ------------------------------------------------------------------ helpers
    def real_shape(self):
        d = self._dims
        if len(d) == 4 and self.strategy_4d == PENCIL:
            nx, ny, nz, nw = d
            return (nw, nz, ny, nx)
        return tuple(d)

    def spectrum_shape(self):
        d = self._dims
        if len(d) == 2:
            return (d[0], d[1] // 2 + 1)
        if len(d) == 3:
            return (d[0], d[1], d[2] // 2 + 1)
        nx, ny, nz, nw = d
        if self.strategy_4d == SLAB:
            return (nx, ny, nz, nw // 2 + 1)
        return (ny, nz, nw // 2 + 1, nx)
