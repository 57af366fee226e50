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
