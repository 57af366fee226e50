import math
import sys
import time
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built sm_100a library")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def tse_surrogates():
    """Networks for the six TSE pulses (3 slices x excitation / refocusing), trained on 2^20 samples each (600
    epochs of 4,096-sample steps, ~24 s per pulse) over |z_rel| <= 2.5: the slices are contiguous, so every spin
    of the 3-slice stack lies within 2.5 slice widths of every pulse's centre."""
    from blochparty_b200 import sequences, surrogate

    out, info = [], []
    for z0 in (-5e-3, 0.0, 5e-3):
        for flip, phase in ((90.0, 0.0), (180.0, 0.5 * math.pi)):
            w, dt, gz, _ = sequences.sinc_pulse(flip, 3e-3, 300, slice_thickness=5e-3,
                                                 slice_offset=z0, phase=phase)
            sg = surrogate.RFSurrogate(w, dt, gz, 5e-3, domain=(200.0, 0.3, 2.5))
            t = time.perf_counter()
            sg.train(epochs=600)
            info.append((flip, z0, time.perf_counter() - t, sg.validate()))
            out.append(sg)
    for flip, z0, sec, (mx, rms, cmx, crms) in info:
        print(f"\nsurrogate {flip:.0f} deg at {z0 * 1e3:+.0f} mm: trained in {sec:.1f} s, rotation max {mx:.1e} "
              f"rms {rms:.1e}, first-order terms max {cmx:.1e} rms {crms:.1e}")
    return out
