"""The C oracle (``oracle/bloch_c.c``): ``simulate(case)`` with ``oracle.bloch.simulate``'s arguments and results,
threaded over spins — TEST INFRASTRUCTURE ONLY.

The same float64 algorithm as ``oracle/bloch.py`` (blochparty's core engine restated), for sequences of a million
segments and more, where the Python restatement's per-segment overhead dominates. Pinned against the reference's
golden fixtures and against ``oracle/bloch.py`` (``tests/test_oracle.py``). No gradients (use ``oracle.bloch``).
"""

from __future__ import annotations

import ctypes
import os

import numpy as np
import torch

from . import build as _build

_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        path = _build.LIB if _build.LIB.exists() else _build.build()
        _lib = ctypes.CDLL(str(path))
        P, I64 = ctypes.c_void_p, ctypes.c_int64
        _lib.bp_oracle_simulate.restype = ctypes.c_int
        _lib.bp_oracle_simulate.argtypes = [I64, P, P, P, P, P, P, P, ctypes.c_int, I64, P, P, P, P, P, P, P, P, P, P,
                                            ctypes.c_int, I64]
    return _lib


def _f64(t):
    return None if t is None else np.ascontiguousarray(t.detach().to(torch.float64).cpu().numpy())


def _u8(flags):
    return np.ascontiguousarray(np.asarray([bool(x) for x in flags], dtype=np.uint8))


def simulate(c, threads: int = 0, chunk: int = 0):
    """(signal (C, n_adc) complex128, m (N, 3) float64) of an ``oracle.bloch.Case``, with all host threads by
    default (``threads`` and ``chunk``, the samples per chunk, change only the speed)."""
    n = int(c.pd.shape[0])
    arrays = {k: _f64(getattr(c, k)) for k in ("pos", "pd", "t1", "t2", "db0", "b1", "dt", "rf", "grad", "adc_phase",
                                               "b0_offset")}
    coils = np.ascontiguousarray(torch.view_as_real(c.coils.to(torch.complex128).cpu().contiguous()).numpy())
    is_rf, adc, spoil = _u8(c.is_rf), _u8(c.adc), _u8(c.spoil)
    S, C, n_adc = int(arrays["dt"].shape[0]), int(coils.shape[1]), int(adc.sum())
    if c.m_init is None:
        m = np.zeros((n, 3))
        m[:, 2] = arrays["pd"]
    else:
        m = _f64(c.m_init).copy()
    sig = np.zeros((C, n_adc, 2))
    p = lambda a: None if a is None else a.ctypes.data
    code = lib().bp_oracle_simulate(n, p(arrays["pos"]), p(arrays["pd"]), p(arrays["t1"]), p(arrays["t2"]),
                                    p(arrays["db0"]), p(arrays["b1"]), p(coils), C, S, p(arrays["dt"]), p(arrays["rf"]),
                                    p(arrays["grad"]), p(arrays["adc_phase"]), p(arrays["b0_offset"]), p(is_rf),
                                    p(adc), p(spoil), p(m), p(sig), threads or (os.cpu_count() or 1), chunk)
    if code != 0:
        raise MemoryError("bp_oracle_simulate: out of memory")
    return torch.view_as_complex(torch.from_numpy(sig)), torch.from_numpy(m)
