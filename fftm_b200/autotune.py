"""Measured autotuner with KEY=VALUE caches (the fftb_autotune_* entry points of
include/fftb.h), mirroring fftm's autotune surface:

* :class:`autotune_options` -- source/fftm_autotune.hpp:50-60 (cache_file,
  create_if_missing, mismatch_policy, validate_hardware, strict_device_identity)
* :class:`measured_options` -- source/fftm_autotune_measure.hpp:21-40 (warmup,
  iterations; the winner is the least median of the timed forward+backward pairs)
* :func:`load_key_value_file` / :func:`save_key_value_file` --
  source/fftm_autotune.hpp:126-169 (``#`` comments, ``KEY=VALUE`` lines, written to
  ``<path>.tmp`` and renamed into place)
* :func:`load_or_measure_config` -- ``load_or_measure_3d_config``,
  source/fftm_autotune_measure.hpp:432-520, for 2D, 3D and 4D ffts problems
* :class:`selected_config` -- ``selected_3d_config``, source/fftm_autotune.hpp:62-70

The parsing, validation, hardware signature and measurement run in the C++ library;
this module only marshals text.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

from . import FftbError, _check, _dtype_code, _lib

CREATE_IF_MISSING, OVERWRITE_ON_MISMATCH, NO_HARDWARE_CHECK, STRICT_DEVICE, FORCE_MEASURE = 1, 2, 4, 8, 16
_TEXT_CAP = 1 << 16


@dataclass
class autotune_options:
    cache_file: str = ""
    create_if_missing: bool = True
    mismatch_policy: str = "error"          # "error" | "overwrite"
    validate_hardware: bool = True
    strict_device_identity: bool = False
    force_measure: bool = False

    def flags(self) -> int:
        if self.mismatch_policy not in ("error", "overwrite"):
            raise ValueError(f"mismatch_policy must be 'error' or 'overwrite', not {self.mismatch_policy!r}")
        f = 0
        if self.create_if_missing:
            f |= CREATE_IF_MISSING
        if self.mismatch_policy == "overwrite":
            f |= OVERWRITE_ON_MISMATCH
        if not self.validate_hardware:
            f |= NO_HARDWARE_CHECK
        if self.strict_device_identity:
            f |= STRICT_DEVICE
        if self.force_measure:
            f |= FORCE_MEASURE
        return f


@dataclass
class measured_options:
    warmup: int = 2
    iterations: int = 5


@dataclass
class selected_config:
    config: dict = field(default_factory=dict)
    source: str = ""          # "cache" or "measured"

    @property
    def strategy(self) -> str:
        return self.config.get("FFTB_AUTOTUNE_STRATEGY", "")

    @property
    def plane_cluster(self) -> int:
        return int(self.config.get("FFTB_AUTOTUNE_PLANE_CLUSTER", "0"))

    def text(self) -> str:
        return to_text(self.config)

    def medians_ms(self) -> dict:
        p = "FFTB_AUTOTUNE_MEDIAN_MS_"
        return {k[len(p):]: float(v) for k, v in self.config.items() if k.startswith(p)}


def parse_text(text: str) -> dict:
    out = {}
    for line in text.splitlines():
        line = line.strip()
        if not line or line.startswith("#"):
            continue
        k, _, v = line.partition("=")
        out[k.strip()] = v.strip()
    return out


def to_text(config: dict) -> str:
    return "".join(f"{k}={v}\n" for k, v in sorted(config.items()))


def _text_call(fn, *args):
    buf = ctypes.create_string_buffer(_TEXT_CAP)
    need = ctypes.c_size_t()
    return buf, need, fn(*args, buf, _TEXT_CAP, ctypes.byref(need))


def load_key_value_file(path: str) -> dict:
    """Parses a cache file (errors: unreadable, empty, or a line without '=')."""
    buf, _, st = _text_call(_lib.load().fftb_autotune_load_file, str(path).encode())
    _check(st, "load_key_value_file")
    return parse_text(buf.value.decode())


def save_key_value_file(path: str, config: dict) -> None:
    _check(_lib.load().fftb_autotune_save_file(str(path).encode(), to_text(config).encode()),
           "save_key_value_file")


def validate(cache: dict, expected: dict, options: autotune_options | None = None) -> None:
    """Raises FftbError(FFTB_ERROR_CACHE_MISMATCH) if the cache does not match the
    expected identity / hardware keys."""
    opts = options or autotune_options()
    _check(_lib.load().fftb_autotune_validate(to_text(cache).encode(), to_text(expected).encode(), opts.flags()),
           "validate")


def hardware_config(device: int = 0) -> dict:
    buf, _, st = _text_call(_lib.load().fftb_autotune_hardware, int(device))
    _check(st, "hardware_config")
    return parse_text(buf.value.decode())


def signature(canonical: str) -> str:
    """"v2:" + 64-bit FNV-1a of a canonical hardware description (the reference's hash)."""
    buf, _, st = _text_call(_lib.load().fftb_autotune_signature, canonical.encode())
    _check(st, "signature")
    return buf.value.decode()


def load_or_measure_config(dtype, sizes, options: autotune_options, measured: measured_options | None = None,
                           strategy_4d="pencil") -> selected_config:
    """Uses the cache when it matches the problem and this GPU; otherwise measures the
    candidates (as the options allow) and writes the cache."""
    from . import _STRATEGY
    m = measured or measured_options()
    d = list(sizes) + [0] * (4 - len(sizes))
    frm = ctypes.c_int()
    buf, _, st = _text_call(
        lambda *a: _lib.load().fftb_autotune_ffts(
            _dtype_code(dtype), d[0], d[1], d[2], d[3], _STRATEGY[strategy_4d], str(options.cache_file).encode(),
            options.flags(), int(m.warmup), int(m.iterations), *a[:3], ctypes.byref(frm)))
    if st != 0:
        raise FftbError(st, "load_or_measure_config")
    return selected_config(parse_text(buf.value.decode()), "cache" if frm.value else "measured")


def autotune_batch(batch, op, options: autotune_options, measured: measured_options | None = None,
                   sign=-1.0):
    """Tunes a :class:`fftm_b200.batch.Batch` for one op; applies the winner's knobs and
    returns (selected_config, mode)."""
    m = measured or measured_options()
    frm, mode = ctypes.c_int(), ctypes.c_int()
    buf, _, st = _text_call(
        lambda *a: _lib.load().fftb_autotune_batch(
            batch._h, int(op), float(sign), str(options.cache_file).encode(), options.flags(), int(m.warmup),
            int(m.iterations), *a[:3], ctypes.byref(frm), ctypes.byref(mode)))
    if st != 0:
        raise FftbError(st, "autotune_batch")
    return selected_config(parse_text(buf.value.decode()), "cache" if frm.value else "measured"), mode.value
