"""What the b200 engine accepts, forward and with gradients, and its refusals in blochparty's wording.

The feature names and the message follow blochparty ``engines/capabilities.py:12-91`` (``FEATURES``, ``features``,
``check``) so that a caller switching engines sees the same ``NotImplementedError`` text pattern. The b200 engine
runs static spins with B1+, an initial magnetization and the scanner field model, forward and with gradients, and
forward also with the rate-model bound pool (magnetization transfer, bound-only RF); every other feature of the
reference's engines is refused here.
"""

from __future__ import annotations

FEATURES = {
    "b1": "B1+ (Phantom.b1)",
    "maps": "field maps (FieldMaps)",
    "bound": "a bound pool (Phantom.bound)",
    "generalized": "the generalized Bloch bound pool",
    "pools": "free exchanging pools (Phantom.pools)",
    "diffusion": "diffusion (Phantom.diffusion)",
    "motion": "motion (Phantom.motion)",
    "scanner": "the scanner field model (scanner=)",
    "bound_only": "bound-pool-only RF segments (Sequence.bound_only)",
    "m_init": "an initial magnetization (m_init)",
}
SUPPORTED = {
    "forward": frozenset({"b1", "m_init", "bound", "scanner", "bound_only"}),
    "gradients": frozenset({"b1", "m_init", "scanner"}),
}


def features(phantom, seq, m_init=None, scanner=None, maps=None) -> frozenset:
    """The ``FEATURES`` a case uses (read by attribute, so blochparty's own objects work too)."""
    bound = getattr(phantom, "bound", None)
    bound_only = getattr(seq, "bound_only", None)
    present = {
        "b1": getattr(phantom, "b1", None) is not None,
        "maps": maps is not None,
        "bound": bound is not None,
        "generalized": bound is not None and getattr(bound, "model", None) == "generalized",
        "pools": bool(getattr(phantom, "pools", None)),
        "diffusion": getattr(phantom, "diffusion", None) is not None,
        "motion": getattr(phantom, "motion", None) is not None,
        "scanner": scanner is not None,
        "bound_only": bound_only is not None and any(bound_only),
        "m_init": m_init is not None,
    }
    return frozenset(k for k, v in present.items() if v)


def unsupported(used: frozenset, grad: bool = False) -> list[str]:
    missing = set(used - SUPPORTED["forward"])
    if grad:
        missing |= used - SUPPORTED["gradients"]
    return sorted(missing)


def check(used: frozenset, grad: bool = False, engine: str = "b200") -> None:
    """Raise ``NotImplementedError`` if the engine does not run a case with features ``used``."""
    bad = unsupported(used, grad)
    if bad:
        what = "; ".join(FEATURES[k] for k in bad)
        kind = "gradients through" if grad else "simulating with"
        raise NotImplementedError(
            f"{engine} engine: {kind} {what} is not implemented; use blochparty.simulate (the core)")
