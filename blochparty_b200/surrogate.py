"""Learned RF surrogate: a small network per shaped pulse, trained on the GPU, standing in for the pulse's
sub-stepped integration (``simulate(..., pulses="surrogate", surrogate=[...])``).

The reference has no learned part; its nearest mechanism is the exact per-spin map of a reused pulse
(blochparty ``engines/gpu/driver.py:112-164``, ``engines/gpu/cuda/pulse.cu.in:3-32``). Here each distinct pulse
waveform (dt, slice gradient G along z, RF samples) gets a 14 -> 64 -> 64 -> 64 -> 16 GELU network. Its inputs are
the spin's off-resonance in the slice gradient f = df + G (z - z0) and its B1 scale (the pulse depends on nothing
else), seen by the first layer with Fourier features of f. Its outputs are the unit quaternion (the Cayley-Klein
pair) of the pulse's rotation reduced by its free precession, R = Rz(wz/2) R~ Rz(wz/2), wz = -2 pi (G z + df) T,
and the pulse's first-order relaxation terms beyond the relax / rotate / relax splitting. The targets come from the
plain integrator (``bp_pulse_targets``: the per-step maps composed in float64); the network is trained by the
hand-written kernels ``bp_mlp_grad`` / ``bp_mlp_reduce`` / ``bp_adam``.

In a simulation, every occurrence of a trained pulse (the same dt and gradient, RF = trained waveform x exp(i phi0),
uniform b0_offset, no sample or spoil inside) is applied by ``bp_surrogate_pulse``: spins inside the training
domain (by default |df| <= 200 Hz, |b1 - 1| <= 0.3, |z_rel| <= 2; a network's own ``domain`` otherwise) take the
network's rotation between two half-pulse relaxations, with its first-order relaxation terms; the others take the
plain sub-stepped segments (the fallback; the plain simulation is the same call without the surrogate).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib, engine
from ._lib import ptr

F32, F64 = torch.float32, torch.float64
TWO_PI = 2.0 * math.pi
DOMAIN = (200.0, 0.3, 2.0)  # default training domain: |df| [Hz], |b1 - 1|, |z_rel| [slice widths]


def _fan_in_init(seed: int) -> torch.Tensor:
    """Flat initial parameters: weights N(0, 1/fan_in), biases 0 (seeded)."""
    g = torch.Generator().manual_seed(seed)
    parts = []
    for shape in ((64, 14), (64,), (64, 64), (64,), (64, 64), (64,), (16, 64), (16,)):
        if len(shape) == 2:
            parts.append(torch.randn(shape, generator=g, dtype=F64).reshape(-1) / math.sqrt(shape[1]))
        else:
            parts.append(torch.zeros(shape, dtype=F64))
    p = torch.cat(parts)
    p[-16] = 1.0  # output bias toward the identity rotation (1, 0, 0, 0) (then the 12 first-order terms: 0)
    return p.to(F32)


@dataclass
class TrainLog:
    steps: int = 0
    epochs: int = 0
    loss: list = field(default_factory=list)  # mean loss per epoch


class RFSurrogate:
    """The network of one shaped pulse: ``rf`` (K, 2) [Hz] on a raster ``dt`` [s] under the slice gradient ``gz``
    [Hz/m] (along z), slice ``thickness`` [m] centred at ``z0`` [m] (default: from the waveform's phase ramp), trained
    on ``domain`` = (|df| [Hz], |b1 - 1|, |z_rel| [slice widths]) bounds."""

    def __init__(self, rf, dt: float, gz: float, thickness: float, z0: float | None = None, device=None, seed=5,
                 domain=DOMAIN):
        self.rf = torch.as_tensor(np.asarray(rf, dtype=np.float64))
        self.dt, self.gz, self.thickness = float(dt), float(gz), float(thickness)
        self.K = self.rf.shape[0]
        self.T = self.K * self.dt
        self.z0 = self._centre() if z0 is None else float(z0)
        if device is None:
            device = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else "cpu"
        self.device = torch.device(device)
        self.params = _fan_in_init(seed).to(self.device)
        self.seed = seed
        self.vweight = 1.0  # the loss weight of the quaternion's vector part (set by train)
        # the loss weight of the first-order terms: their effect on the magnetization is about (r2 - r1) T times
        # their error (a few hundredths for T of a few ms), so they need far less precision than the rotation
        self.cweight = 0.01
        self.domain = tuple(float(d) for d in domain)
        if len(self.domain) != 3 or min(self.domain) <= 0:
            raise ValueError(f"domain must be three positive bounds (|df|, |b1 - 1|, |z_rel|), got {domain!r}")
        self.log = TrainLog()

    def _centre(self) -> float:
        """Slice centre from the waveform's linear phase ramp: RF ~ exp(-i 2 pi G z0 t) (least squares on the phase
        steps between samples of significant amplitude)."""
        z = self.rf[:, 0].numpy() + 1j * self.rf[:, 1].numpy()
        on = np.abs(z) > 1e-3 * np.abs(z).max()
        steps = np.angle(z[1:] * np.conj(z[:-1]))[on[1:] & on[:-1]]
        steps = steps[np.abs(steps) < 0.5 * np.pi]  # the sinc's sign flips are pi steps
        if steps.size == 0 or self.gz == 0:
            return 0.0
        f = -float(np.median(steps)) / (TWO_PI * self.dt)
        return f / self.gz

    # ---- targets and training ----
    def samples(self, n: int, seed: int) -> torch.Tensor:
        """n uniform samples (df [Hz], b1, z_rel) of the training domain, (n, 3) float32 on the device."""
        g = torch.Generator().manual_seed(seed)
        u = torch.rand(n, 3, generator=g, dtype=F64) * 2 - 1
        d = self.domain
        s = torch.stack([u[:, 0] * d[0], 1 + u[:, 1] * d[1], u[:, 2] * d[2]], -1)
        return s.to(F32).to(self.device).contiguous()

    def targets(self, samples: torch.Tensor, full: bool = False):
        """The network's targets (n, 16) for the samples from the plain integrator: the reduced rotation, dA~ / T
        and dC~ / T (and the whole rotations (n, 4) when ``full``)."""
        n = samples.shape[0]
        rf = self.rf.to(self.device).contiguous()
        tg = torch.empty(n, _lib.BP_MLP_OUTPUTS, dtype=F32, device=self.device)
        qfull = torch.empty(n, 4, dtype=F32, device=self.device) if full else None
        code = _lib.lib().bp_pulse_targets(ptr(rf), self.K, self.dt, self.gz, self.thickness, self.z0, ptr(samples),
                                           n, ptr(tg), ptr(qfull), _lib.stream_ptr())
        _lib.check(code, "bp_pulse_targets")
        return (tg, qfull) if full else tg

    @property
    def fmax(self) -> float:
        """The largest |f| = |df + G (z - z0)| [Hz] of the training domain: the scale of the input f^."""
        return self.domain[0] + abs(self.gz) * self.domain[2] * self.thickness

    def normalise(self, samples: torch.Tensor) -> torch.Tensor:
        """The network's inputs (n, 2) of samples (df, b1, z_rel): f^ = (df + G z_rel thickness) / F and
        b^ = (b1 - 1) / dom_b1 (float64 arithmetic, rounded once)."""
        s, d = samples.to(F64), self.domain
        f = (s[:, 0] + self.gz * self.thickness * s[:, 2]) / self.fmax
        return torch.stack([f, (s[:, 1] - 1) / d[1]], -1).to(F32).contiguous()

    def gradient(self, x: torch.Tensor, target: torch.Tensor, vweight: float = 1.0, cweight: float = 1.0):
        """(mean loss, gradient) of the batch through the training kernels (x normalised; ``vweight`` weights the
        quaternion's vector part in the loss, ``cweight`` the first-order terms)."""
        lib, n = _lib.lib(), x.shape[0]
        ctas = lib.bp_mlp_grad_ctas(n)
        gpart = torch.empty(ctas, _lib.BP_MLP_PARAMS, dtype=F32, device=self.device)
        lpart = torch.empty(ctas, dtype=F32, device=self.device)
        grad = torch.empty(_lib.BP_MLP_PARAMS, dtype=F32, device=self.device)
        loss = torch.empty(1, dtype=F32, device=self.device)
        st = _lib.stream_ptr()
        _lib.check(lib.bp_mlp_grad(ptr(self.params), ptr(x), ptr(target), n, vweight, cweight, ptr(gpart),
                                   ptr(lpart), st), "bp_mlp_grad")
        _lib.check(lib.bp_mlp_reduce(ptr(gpart), ptr(lpart), ctas, 1.0 / n, ptr(grad), ptr(loss), st), "bp_mlp_reduce")
        return loss, grad

    def train(self, n_samples: int = 1 << 20, epochs: int = 400, batch: int = 4096, lr: float = 4e-3,
              lr_min: float = 1e-6, seed: int | None = None) -> TrainLog:
        """Adam with a cosine learning-rate decay over ``epochs`` passes of ``n_samples`` plain-integrator targets
        (the defaults: 102,400 steps of 4,096 samples, about 16 s on one B200; the decay down to 1e-6 matters,
        since Adam's steps of about the learning rate per weight set the error floor).
        The loss weights the quaternion's vector part by 1 / s^2, s its largest magnitude among the targets (clipped
        to [1e-2, 1]): a small rotation (a 10-degree excitation) is then learned to a relative, not an absolute,
        precision."""
        lib, st = _lib.lib(), _lib.stream_ptr()
        seed = self.seed if seed is None else seed
        s = self.samples(n_samples, seed + 1)
        x, y = self.normalise(s), self.targets(s)
        vmax = float(torch.linalg.vector_norm(y[:, 1:4], dim=1).max())
        self.vweight = 1.0 / min(1.0, max(1e-2, vmax)) ** 2
        m = torch.zeros(_lib.BP_MLP_PARAMS, dtype=F32, device=self.device)
        v = torch.zeros_like(m)
        ctas = lib.bp_mlp_grad_ctas(batch)
        gpart = torch.empty(ctas, _lib.BP_MLP_PARAMS, dtype=F32, device=self.device)
        lpart = torch.empty(ctas, dtype=F32, device=self.device)
        grad = torch.empty_like(m)
        loss = torch.zeros(1, dtype=F32, device=self.device)
        steps_per_epoch = n_samples // batch
        total = epochs * steps_per_epoch
        g = torch.Generator(device="cpu").manual_seed(seed + 2)
        for ep in range(epochs):
            perm = torch.randperm(n_samples, generator=g).to(self.device)
            xs, ys = x[perm].contiguous(), y[perm].contiguous()
            acc = torch.zeros(1, dtype=F32, device=self.device)
            for b in range(steps_per_epoch):
                step = self.log.steps + 1
                frac = (ep * steps_per_epoch + b) / max(total - 1, 1)
                rate = lr_min + 0.5 * (lr - lr_min) * (1 + math.cos(math.pi * frac))
                xb, yb = xs[b * batch:(b + 1) * batch], ys[b * batch:(b + 1) * batch]
                _lib.check(lib.bp_mlp_grad(ptr(self.params), ptr(xb), ptr(yb), batch, self.vweight, self.cweight,
                                           ptr(gpart), ptr(lpart), st), "bp_mlp_grad")
                _lib.check(lib.bp_mlp_reduce(ptr(gpart), ptr(lpart), ctas, 1.0 / batch, ptr(grad), ptr(loss), st),
                           "bp_mlp_reduce")
                _lib.check(lib.bp_adam(ptr(self.params), ptr(grad), ptr(m), ptr(v), rate, 0.9, 0.999, 1e-8, step, st),
                           "bp_adam")
                acc += loss
                self.log.steps = step
            self.log.epochs += 1
            self.log.loss.append(float(acc) / steps_per_epoch)
        torch.cuda.synchronize(self.device)
        return self.log

    def wtiles(self) -> torch.Tensor:
        """W2 and W3 split into bfloat16 high / low tiles in the tensor cores' operand layout (``bp_mlp_wtiles``),
        made again whenever the parameters changed since the last call."""
        key = (self.log.steps, self.params.data_ptr())
        if getattr(self, "_wt_key", None) != key:
            self._wt = torch.empty(_lib.lib().bp_mlp_wtiles_bytes(), dtype=torch.uint8, device=self.device)
            _lib.check(_lib.lib().bp_mlp_wtiles(ptr(self.params), ptr(self._wt), _lib.stream_ptr()), "bp_mlp_wtiles")
            self._wt_key = key
        return self._wt

    def params_host(self) -> np.ndarray:
        """A float32 host copy of the parameters (the tensor-core inference passes the small ones by value), made
        again whenever the parameters changed since the last call."""
        key = (self.log.steps, self.params.data_ptr())
        if getattr(self, "_ph_key", None) != key:
            self._ph = np.ascontiguousarray(self.params.detach().float().cpu().numpy())
            self._ph_key = key
        return self._ph

    def predict(self, samples: torch.Tensor) -> torch.Tensor:
        """The network's outputs (n, 16) for samples (df, b1, z_rel)."""
        x = self.normalise(samples)
        y = torch.empty(x.shape[0], _lib.BP_MLP_OUTPUTS, dtype=F32, device=self.device)
        _lib.check(_lib.lib().bp_mlp_eval(ptr(self.params), ptr(x), x.shape[0], ptr(y), _lib.stream_ptr()),
                   "bp_mlp_eval")
        return y

    def validate(self, n: int = 1 << 16, seed: int = 99):
        """(largest, RMS) error of the network's reduced rotation against the plain integrator's (quaternion
        components; the rotation-matrix error is at most twice as large), then (largest, RMS) error of its
        first-order terms dA~ / T, dC~ / T, on fresh samples."""
        s = self.samples(n, seed)
        err = (self.predict(s) - self.targets(s)).abs()
        q, c = err[:, :4], err[:, 4:]
        return (float(q.max()), float(q.pow(2).mean().sqrt()), float(c.max()), float(c.pow(2).mean().sqrt()))

    # ---- matching occurrences in a sequence ----
    def phase_of(self, w: np.ndarray, tol: float = 1e-6):
        """phi0 if the complex RF samples ``w`` (K,) are the trained waveform times exp(i phi0), else None."""
        z = self.rf[:, 0].numpy() + 1j * self.rf[:, 1].numpy()
        c = np.vdot(z, w)
        phi0 = float(np.angle(c)) if c != 0 else 0.0
        if np.abs(w - z * np.exp(1j * phi0)).max() > tol * float(np.abs(z).max()):
            return None
        return phi0

    def clean_windows(self, dt, gz, other):
        """Prefix counts c (S + 1,) of segments that rule out this pulse (``other``: not RF, a sample, a spoil or an
        x / y gradient; or another dt or slice gradient ``gz``): [s, s + K) can be an occurrence only if
        c[s + K] == c[s]."""
        scale = max(abs(self.gz), 1.0)
        bad = other | (np.abs(dt - self.dt) > 1e-9 * self.dt) | (np.abs(gz - self.gz) > 1e-9 * scale)
        return np.concatenate([[0], np.cumsum(bad)])

    def match_at(self, s, dt, rf, grad, b0, is_rf, adc, spoil, tol: float = 1e-6):
        """phi0 if segments [s, s + K) are an occurrence of this pulse (the same dt and slice gradient, RF = trained
        waveform x exp(i phi0), uniform b0_offset, no sample or spoil), else None."""
        e = s + self.K
        if e > len(dt):
            return None
        other = ~is_rf[s:e] | adc[s:e] | spoil[s:e] | (np.abs(grad[s:e, :2]).max(1) > 1e-9 * max(abs(self.gz), 1.0))
        if self.clean_windows(dt[s:e], grad[s:e, 2], other)[-1] or np.abs(b0[s:e] - b0[s]).max() > 1e-9:
            return None
        return self.phase_of(rf[s:e, 0] + 1j * rf[s:e, 1], tol)


def pulse_pieces(rf, dt, gz, thickness, pieces: int = 1, device=None, seed=5, domain=DOMAIN):
    """Surrogates for a pulse cut into ``pieces`` consecutive equal parts (each a shorter shaped pulse with its own
    network; the relaxation is then split around every piece, which shrinks the splitting error ~pieces^2)."""
    rf = np.asarray(rf, dtype=np.float64)
    k = rf.shape[0]
    if k % pieces:
        raise ValueError(f"{k} steps do not split into {pieces} equal pieces")
    m = k // pieces
    return [RFSurrogate(rf[i * m:(i + 1) * m], dt, gz, thickness, device=device, seed=seed + 17 * i, domain=domain)
            for i in range(pieces)]


def find_occurrences(surrogates, inp, tol: float = 1e-6):
    """[(start, K, surrogate index, phi0, b0)] of every pulse occurrence (or piece) that one of ``surrogates`` stands
    in for: within every run of RF segments, from its start, the first surrogate that matches at the current
    position takes it and the scan continues after it; at a position no surrogate matches, the rest of the run is
    left to the plain integrator. Vectorised over positions: every run start at once, then every position just
    after a match, and so on (the per-segment conditions are prefix counts; the waveform test is one batched
    comparison per surrogate and level)."""
    d = lambda t: t.detach().to(F64).cpu().numpy()
    dt, rf, grad = d(inp.dt), d(inp.rf), d(inp.grad)
    S = len(dt)
    b0 = np.zeros(S) if inp.b0_offset is None else d(inp.b0_offset)
    is_rf, adc, spoil = (np.fromiter(f, dtype=bool, count=S) for f in (inp.is_rf, inp.adc, inp.spoil))
    w = rf[:, 0] + 1j * rf[:, 1]
    gxy = np.abs(grad[:, :2]).max(1)
    base = ~is_rf | adc | spoil
    clean = [sg.clean_windows(dt, grad[:, 2], base | (gxy > 1e-9 * max(abs(sg.gz), 1.0))) for sg in surrogates]
    # b0_offset steps: a window [s, e) is uniform when no step lies in (s, e)
    steps = np.concatenate([[0], np.cumsum(np.concatenate([[False], np.abs(np.diff(b0)) > 1e-9]))])
    occ = []
    cands = np.flatnonzero(is_rf & ~np.concatenate([[False], is_rf[:-1]]))
    while cands.size:
        taken = np.zeros(cands.size, dtype=bool)
        ends = []
        for i, sg in enumerate(surrogates):
            e = cands + sg.K
            ok = ~taken & (e <= S)
            ec = np.minimum(e, S)
            ok &= (clean[i][ec] == clean[i][cands]) & (steps[ec] == steps[np.minimum(cands + 1, S)])
            idx = np.flatnonzero(ok)
            if idx.size == 0:
                continue
            z = sg.rf[:, 0].numpy() + 1j * sg.rf[:, 1].numpy()
            W = w[cands[idx, None] + np.arange(sg.K)]
            c = W @ np.conj(z)
            phi = np.where(c != 0, np.angle(c), 0.0)
            good = np.abs(W - z[None, :] * np.exp(1j * phi)[:, None]).max(1) <= tol * np.abs(z).max()
            for j, ph in zip(idx[good].tolist(), phi[good].tolist()):
                s0 = int(cands[j])
                occ.append((s0, sg.K, i, ph, float(b0[s0])))
            taken[idx[good]] = True
            ends.append(e[idx[good]])
        cands = np.concatenate(ends) if ends else np.zeros(0, dtype=np.int64)
        cands = cands[cands < S]
    occ.sort()
    return occ


def forward_with_surrogate(inp, device, options):
    """``simulate(..., pulses="surrogate")``: signal (C, A) complex64 and m (N, 3) float32 on the CPU."""
    surrogates = options.get("surrogate")
    if surrogates is None:
        raise ValueError("pulses='surrogate' needs surrogate=[RFSurrogate, ...] (trained networks)")
    if isinstance(surrogates, RFSurrogate):
        surrogates = [surrogates]
    sig, m, _ = run_with_surrogates(inp, device, surrogates, options.get("surrogate_inference", "mma"))
    return sig, m


INFERENCE = ("mma", "fp32")


class SurrogateRun:
    """The occurrences of one packed case that ``surrogates`` stand in for, with the window plan around them."""

    def __init__(self, inp, pk, surrogates, inference: str = "mma"):
        if inference not in INFERENCE:
            raise ValueError(f"surrogate_inference must be one of {INFERENCE}, not {inference!r}")
        self.surrogates, self.inference = surrogates, inference
        self.occ = find_occurrences(surrogates, inp)
        self.spans = [(s, k) for s, k, *_ in self.occ]
        self.plan = engine.plan_replacing(pk, self.spans)

    def descriptors(self, counts=None):
        """The occurrences as ``BpSpan`` descriptors for ``bp_forward_spans`` (the networks' host parameters and
        weight tiles are made here and kept by the surrogates)."""
        arr = (_lib.BpSpan * max(1, len(self.occ)))()
        for i, (s, k, isg, phi0, b0) in enumerate(self.occ):
            sg = self.surrogates[isg]
            mma = self.inference == "mma"
            arr[i] = _lib.BpSpan(kind=_lib.BP_SPAN_NET_MMA if mma else _lib.BP_SPAN_NET_F32, seg0=s, k_steps=k,
                                 phase=phi0, b0off=b0,
                                 params=sg.params_host().ctypes.data if mma else ptr(sg.params),
                                 wtiles=ptr(sg.wtiles()) if mma else None, T=sg.T, gz=sg.gz, thickness=sg.thickness,
                                 z0=sg.z0, dom_df=sg.domain[0], dom_b1=sg.domain[1], dom_z=sg.domain[2],
                                 counts=ptr(counts))
        return arr

    def run(self, pk, state, raw, status, counts=None, events=None):
        """The forward with every occurrence through its network; counts (None or int32 [2]) += spins through the
        networks, through the fallback. One native call, or the launches one by one from Python when ``events``
        collects the forward launches' CUDA events."""
        if events is None:
            key = None if counts is None else counts.data_ptr()
            if getattr(self, "_desc_key", -1) != key:
                self._desc, self._desc_key = self.descriptors(counts), key
            engine.forward_spans(pk, state, self.plan, self._desc, raw, status)
            return
        lib, st = _lib.lib(), _lib.stream_ptr()

        def apply(i):
            s, k, isg, phi0, b0 = self.occ[i]
            sg = self.surrogates[isg]
            if self.inference == "mma":
                code = lib.bp_surrogate_pulse_mma(ptr(pk.spins), ptr(state), pk.n, sg.params_host().ctypes.data,
                                                  ptr(sg.wtiles()), ptr(pk.segs), s, k, sg.T, sg.gz, sg.thickness,
                                                  sg.z0, phi0, b0,
                                                  *sg.domain, ptr(counts), ptr(status), 0, st)
            else:
                code = lib.bp_surrogate_pulse(ptr(pk.spins), ptr(state), pk.n, ptr(sg.params), ptr(pk.segs), s, k,
                                              sg.T, sg.gz, sg.thickness, sg.z0, phi0, b0, *sg.domain, ptr(counts), st)
            _lib.check(code, "bp_surrogate_pulse")

        engine.forward_replacing(pk, state, self.spans, apply, raw, status, plan=self.plan, events=events)


def run_with_surrogates(inp, device, surrogates, inference: str = "mma"):
    """The forward with every matched pulse occurrence through its surrogate; returns (signal, m, counts).
    ``inference``: "mma" (layers 2 and 3 on the tensor cores, ``bp_surrogate_pulse_mma``) or "fp32" (the whole
    network on the CUDA cores, ``bp_surrogate_pulse``)."""
    pk = engine.pack(inp, device)
    plan = SurrogateRun(inp, pk, surrogates, inference)
    state = engine.initial_state(inp.pd, inp.m_init, device)
    raw = torch.zeros(max(pk.n_adc, 1), 2 * pk.n_coils, dtype=F64, device=device)
    status = torch.zeros(1, dtype=torch.int32, device=device)
    counts = torch.zeros(2, dtype=torch.int32, device=device)
    plan.run(pk, state, raw if pk.n_adc else None, status, counts)
    sig = engine.finish_signal(pk, raw)
    torch.cuda.synchronize(device)
    _lib.check_status(status, "bp_forward")
    return sig.cpu(), engine.final_m(state), counts.cpu().tolist()
