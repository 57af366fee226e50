"""B200-native rebuild of blochparty's plain-Bloch GPU simulation path (``bp.simulate(..., engine="gpu")``).

``simulate(phantom, seq, coils, ...)`` takes blochparty's ``Phantom`` / ``Sequence`` objects (or this package's
identical ``types``) and runs them on hand-written sm_100a CUDA kernels through the C ABI of
``libblochparty_b200.so`` (``include/blochparty_b200.h``). There is no CPU fallback.
"""

from .api import simulate
from .pulseq import read_pulseq
from .phantoms import birdcage_sensitivities, ellipse_phantom_2d, ellipsoid_phantom_3d, grid_positions, head_phantom_3d
from .sequences import SequenceBuilder, gre, sinc_pulse, tse_2d
from .types import Phantom, Sequence, SimResult

__all__ = ["simulate", "Phantom", "Sequence", "SimResult", "SequenceBuilder", "gre", "tse_2d", "sinc_pulse",
           "birdcage_sensitivities", "ellipse_phantom_2d", "ellipsoid_phantom_3d", "head_phantom_3d",
           "grid_positions", "read_pulseq"]
