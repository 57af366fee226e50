"""Loading the golden fixtures of ``tests/golden`` (written by ``tests/golden/make_golden.py`` from the reference's
float64 core) as oracle cases and as phantom / sequence objects of this package."""

import math
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


PHYSICS = ("mt_sl", "mt_lor", "field_nl", "field_leading", "field_exact", "mt_field")


def load_physics(name):
    """A bound-pool / field-model golden (``make_golden.py physics``): (phantom, sequence, coils, m_init, scanner)
    of this package, the reference's (signal, m, m_bound) and the raw arrays."""
    from blochparty_b200 import physics

    z = np.load(GOLDEN / f"{name}.npz")
    t = lambda k: torch.from_numpy(z[k]).to(F64)
    opt = lambda k: t(k) if z[k].size else None
    bound = None
    if "pool_f" in z:
        bound = physics.BoundPool(t("pool_f"), t("pool_k"), t("pool_t1"), t("pool_t2"), t("pool_dw"),
                                  lineshape=str(z["pool_shape"]))
    ph = Phantom(t("pos"), t("pd"), t("t1"), t("t2"), t("db0"), b1=opt("b1"), bound=bound)
    seq = Sequence(t("dt"), t("rf"), t("grad"), t("adc_phase"), [bool(x) for x in z["is_rf"]],
                   [bool(x) for x in z["adc"]], [bool(x) for x in z["spoil"]], b0_offset=opt("b0_offset"),
                   bound_only=[bool(x) for x in z["bound_only"]] if z["bound_only"].size else None)
    scanner = None
    if "sc_r0" in z:
        b0 = float(z["sc_b0"])
        nl = physics.GradientNonlinearity(t("sc_alpha"), t("sc_beta"), float(z["sc_r0"]))
        scanner = physics.Scanner(None if math.isnan(b0) else b0, str(z["sc_conc"]) or None, nonlinearity=nl)
    coils = torch.complex(t("coils_re"), t("coils_im"))
    ref = (torch.complex(t("sig_re"), t("sig_im")), t("m"), opt("m_bound"))
    return (ph, seq, coils, opt("m_init"), scanner), ref, z
