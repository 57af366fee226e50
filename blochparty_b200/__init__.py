"""B200-native rebuild of blochparty's plain-Bloch GPU simulation path (``bp.simulate(..., engine="gpu")``)."""

from .types import Phantom, Sequence, SimResult
