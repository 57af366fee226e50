"""Loading the golden fixtures of ``tests/golden`` (written by ``tests/golden/make_golden.py`` from the reference's
float64 core) as oracle cases and as phantom / sequence objects of this package."""

from pathlib import Path

import numpy as np
import torch

from blochparty_b200.types import Phantom, Sequence
from oracle.bloch import Case

GOLDEN = Path(__file__).resolve().parent / "golden"
F64 = torch.float64
NAMES = ("rand0", "rand1", "busy", "gre16", "sinc3d", "grad_rand", "grad_busy")


def load(name):
    z = np.load(GOLDEN / f"{name}.npz")
    t = lambda k: torch.from_numpy(z[k]).to(F64)
    opt = lambda k: t(k) if z[k].size else None
    coils = torch.complex(t("coils_re"), t("coils_im"))
    case = Case(t("pos"), t("pd"), t("t1"), t("t2"), t("db0"), opt("b1"), coils, t("dt"), t("rf"), t("grad"),
                t("adc_phase"), opt("b0_offset"), [bool(x) for x in z["is_rf"]], [bool(x) for x in z["adc"]],
                [bool(x) for x in z["spoil"]], opt("m_init"))
    sig = torch.complex(t("sig_re"), t("sig_im"))
    return case, sig, t("m"), z


def objects(case):
    """(Phantom, Sequence, coils, m_init) of this package for a golden case."""
    ph = Phantom(case.pos, case.pd, case.t1, case.t2, case.db0, b1=case.b1)
    seq = Sequence(case.dt, case.rf, case.grad, case.adc_phase, list(case.is_rf), list(case.adc), list(case.spoil),
                   b0_offset=case.b0_offset)
    return ph, seq, case.coils, case.m_init


def load_adjoint128():
    """The 128^2 flip-train golden (``make_golden.py adjoint128``): this package's builders make the case
    (``workloads.adjoint_2d_128``); the fixture holds the reference's target signal, loss and gradients, and float64
    sums of the inputs it was made from."""
    from blochparty_b200 import workloads

    z = np.load(GOLDEN / "adjoint128.npz")
    ph, seq, coils, flips, t1_target = workloads.adjoint_2d_128()
    sums = {"pos": ph.pos, "pd": ph.pd, "t1": ph.t1, "t2": ph.t2, "db0": ph.db0, "b1": ph.b1, "dt": seq.dt,
            "rf": seq.rf, "grad": seq.grad, "t1_target": t1_target, "coils_abs": coils.abs()}
    same = {k: float(v.double().sum()) == float(z[f"sum_{k}"]) for k, v in sums.items()}
    return z, (ph, seq, coils, flips, t1_target), same
