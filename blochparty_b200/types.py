"""The simulation's inputs and outputs, field for field those of blochparty.

``Phantom`` (blochparty ``phantom.py:17-51``), ``Sequence`` (blochparty ``sequence.py:28-59``) and
``SimResult`` (blochparty ``result.py:10-15``) keep the reference's field names, shapes, units and
conventions, so code written against blochparty builds these objects unchanged, and objects built by
blochparty itself are accepted as they are (``simulate`` reads them by attribute only).

Units follow Pulseq, as in the reference: RF in Hz (gamma_bar * B1), gradients in Hz/m, times in s,
positions in m, off-resonance in Hz. A segment holds RF and gradients constant for ``dt``; an ADC
sample is taken at the end of its segment, before that segment's spoil.
"""

from __future__ import annotations

from dataclasses import dataclass, field, replace

import torch
from torch import Tensor


@dataclass
class Phantom:
    """Isochromats ("spins") with tissue properties (blochparty ``phantom.py:17-32``).

    ``bound``, ``pools``, ``diffusion``, ``restriction`` and ``motion`` exist so that a blochparty phantom
    maps one to one; the b200 engine refuses them with ``NotImplementedError`` (``capabilities``).
    """

    pos: Tensor  # (N, 3) [m]
    pd: Tensor  # (N,) proton density, the equilibrium magnetization
    t1: Tensor  # (N,) [s]
    t2: Tensor  # (N,) [s]
    db0: Tensor  # (N,) off-resonance [Hz]
    b1: Tensor | None = None  # (N,) relative transmit scale of every RF pulse; None = 1
    bound: object | None = None
    pools: tuple | None = None
    diffusion: Tensor | None = None
    restriction: object | None = None
    motion: object | None = None

    def __len__(self) -> int:
        return self.pd.shape[0]

    def to(self, dtype=None, device=None) -> Phantom:
        conv = lambda t: None if t is None else t.to(dtype=dtype, device=device)
        return replace(
            self,
            pos=conv(self.pos),
            pd=conv(self.pd),
            t1=conv(self.t1),
            t2=conv(self.t2),
            db0=conv(self.db0),
            b1=conv(self.b1),
            diffusion=conv(self.diffusion),
        )


@dataclass
class Sequence:
    """A flat list of piecewise-constant segments (blochparty ``sequence.py:28-48``).

    ``is_rf``, ``adc`` and ``spoil`` are per-segment booleans: an RF segment rotates about the effective
    field; ``adc`` samples the signal at the end of the segment; ``spoil`` zeroes the transverse
    magnetization at the end of the segment (after its sample).
    """

    dt: Tensor  # (S,) [s]
    rf: Tensor  # (S, 2) RF field (x, y) [Hz]
    grad: Tensor  # (S, 3) [Hz/m]
    adc_phase: Tensor  # (S,) receiver phase [rad], used where adc is True
    is_rf: list
    adc: list
    spoil: list
    meta: dict = field(default_factory=dict)
    b0_offset: Tensor | None = None  # (S,) uniform off-resonance [Hz] added to every spin; None = zeros
    rf_freq: Tensor | None = None  # (S,) RF carrier [Hz]: only the bound pool uses it (refused here)
    bound_only: list | None = None  # RF segments only a bound pool feels (refused here when any is set)

    def __len__(self) -> int:
        return self.dt.shape[0]

    @property
    def n_adc(self) -> int:
        return int(sum(bool(a) for a in self.adc))

    @property
    def duration(self) -> Tensor:
        return self.dt.sum()

    def to(self, dtype=None, device=None) -> Sequence:
        conv = lambda t: None if t is None else t.to(dtype=dtype, device=device)
        return replace(
            self,
            dt=conv(self.dt),
            rf=conv(self.rf),
            grad=conv(self.grad),
            adc_phase=conv(self.adc_phase),
            b0_offset=conv(self.b0_offset),
            rf_freq=conv(self.rf_freq),
        )


@dataclass
class SimResult:
    """What a simulation returns (blochparty ``result.py:10-15``): ``signal`` (C, n_adc) complex in ADC order,
    demodulated by each sample's receiver phase; ``m`` (N, 3) the magnetization after the last segment."""

    signal: Tensor
    m: Tensor
    m_bound: Tensor | None = None
    m_pools: Tensor | None = None
