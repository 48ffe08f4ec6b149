"""Learned early stop: a 1-D conv + MLP network reads the early port
transient of a run and predicts its late-time ringing tail, so the run can
stop long before numberOfTimeSteps.

The reference always runs every step (js_fdtd/src/index.js:54-60) and turns
the full port traces into S11 (index.js:62-75, dft.js:17-38); this module is
the part with no counterpart there.

Model of the tail.  After the source pulse has left, the port voltage and
current of a linear, passive structure ring down as a sum of damped
sinusoids sum_m Re(c_m exp(s_m t)), s_m = -alpha_m + j 2 pi f_m.  The network
maps the first `n_in` steps (4x decimated, each channel scaled by its
largest magnitude) to the run's tail poles s_m (up to K_POLES of them).  At a
checkpoint the amplitudes c_m are fitted by least squares to the steps
[n_in, checkpoint) that were actually run, for the network's poles and for
matrix-pencil poles of those same steps; the best fit's residual energy is
the gate.  Below the threshold the run stops and its traces are completed
with the fitted tail; otherwise it keeps stepping (plain FDTD) to the next
checkpoint.

`EsNet` is the handle of the CUDA network (include/fdtd_b200.h, fdtd_es_*):
training, gradients and inference all run in the project's own kernels.
"""
from __future__ import annotations

import ctypes as C
import math
import multiprocessing as mp
import os
import threading
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass

import numpy as np
from threadpoolctl import threadpool_limits

from . import _native as N

ARCH = dict(in_channels=2, in_length=375, conv_layers=4, channels=64, kernel=5, stride=2, mlp_layers=2,
            mlp_width=256)
K_POLES = 6          # tail poles the network predicts
OUT_DIM = 2 * K_POLES  # per pole: (f - F_CENTER) / F_SCALE and log(alpha / ALPHA_UNIT), sorted by f
DECIM = 4            # input decimation
F_CENTER, F_SCALE = 2.5e9, 1.0e9
ALPHA_UNIT = 1.0e9   # decay rates in 1/ns


class EsNet:
    """The CUDA network.  Arrays are float32; inputs are (B, in_length, 2)."""

    def __init__(self, out_dim: int = OUT_DIM, max_batch: int = 512, device: int = 0, **arch):
        a = dict(ARCH, **arch)
        self.arch, self.out_dim, self.max_batch = a, out_dim, max_batch
        cfg = N.FdtdEsConfig(a["in_channels"], a["in_length"], a["conv_layers"], a["channels"], a["kernel"],
                             a["stride"], a["mlp_layers"], a["mlp_width"], out_dim, max_batch, device)
        h = C.c_void_p()
        N.check(N.lib().fdtd_es_create(C.byref(cfg), C.byref(h)))
        self._h = h
        n = C.c_long()
        N.check(N.lib().fdtd_es_param_count(self._h, C.byref(n)))
        self.n_params = n.value
        # targets are learned standardised: raw = out * out_sd + out_mu (FP32, outside the network)
        self.out_mu = np.zeros(out_dim, np.float32)
        self.out_sd = np.ones(out_dim, np.float32)

    def save(self, path: str) -> None:
        np.savez(path, params=self.params, out_mu=self.out_mu, out_sd=self.out_sd, out_dim=self.out_dim,
                 **{k: v for k, v in self.arch.items()})

    @classmethod
    def load(cls, path: str, max_batch: int = 512, device: int = 0) -> "EsNet":
        z = np.load(path)
        arch = {k: int(z[k]) for k in ARCH}
        net = cls(int(z["out_dim"]), max_batch=max_batch, device=device, **arch)
        net.params = z["params"]
        net.out_mu, net.out_sd = z["out_mu"].astype(np.float32), z["out_sd"].astype(np.float32)
        return net

    def init(self, seed: int = 0) -> None:
        N.check(N.lib().fdtd_es_init_params(self._h, int(seed)))

    @property
    def params(self) -> np.ndarray:
        out = np.zeros(self.n_params, np.float32)
        N.check(N.lib().fdtd_es_get_params(self._h, N.fptr(out), out.size))
        return out

    @params.setter
    def params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        N.check(N.lib().fdtd_es_set_params(self._h, N.fptr(p), p.size))

    def _x(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        if x.ndim != 3 or x.shape[1:] != (self.arch["in_length"], self.arch["in_channels"]):
            raise ValueError(f"inputs must be (B, {self.arch['in_length']}, {self.arch['in_channels']})")
        return x

    def forward(self, x) -> np.ndarray:
        x = self._x(x)
        y = np.zeros((x.shape[0], self.out_dim), np.float32)
        N.check(N.lib().fdtd_es_forward(self._h, N.fptr(x), x.shape[0], N.fptr(y)))
        return y

    def loss_grad(self, x, target, w=None, grad: bool = True):
        x = self._x(x)
        t = np.ascontiguousarray(target, dtype=np.float32)
        w = np.ascontiguousarray(np.ones(self.out_dim) if w is None else w, dtype=np.float32)
        loss = np.zeros(1, np.float32)
        g = np.zeros(self.n_params, np.float32) if grad else None
        N.check(N.lib().fdtd_es_loss_grad(self._h, N.fptr(x), N.fptr(t), N.fptr(w), x.shape[0], N.fptr(loss),
                                          N.fptr(g), self.n_params if grad else 0))
        return float(loss[0]), g

    def train(self, x, target, epochs: int, batch: int = 128, w=None, lr: float = 1e-3, beta1: float = 0.9,
              beta2: float = 0.999, eps: float = 1e-8, weight_decay: float = 0.0, seed: int = 0) -> np.ndarray:
        x = self._x(x)
        t = np.ascontiguousarray(target, dtype=np.float32)
        N.check(N.lib().fdtd_es_set_data(self._h, N.fptr(x), N.fptr(t), x.shape[0]))
        w = np.ascontiguousarray(np.ones(self.out_dim) if w is None else w, dtype=np.float32)
        losses = np.zeros(max(epochs, 1), np.float32)
        N.check(N.lib().fdtd_es_train(self._h, int(epochs), int(batch), N.fptr(w), lr, beta1, beta2, eps,
                                      weight_decay, int(seed), N.fptr(losses)))
        return losses[:epochs]

    def _members(self, engines):
        return (C.c_void_p * len(engines))(*[e._h.value for e in engines])

    def member_inputs(self, engines, decim: int = DECIM):
        arr = self._members(engines)
        scales = np.zeros(2 * len(engines), np.float32)
        x = np.zeros((len(engines), self.arch["in_length"], 2), np.float32)
        N.check(N.lib().fdtd_es_member_inputs(self._h, arr, len(engines), decim, N.fptr(scales), N.fptr(x)))
        return x, scales.reshape(-1, 2)

    def predict_members(self, engines, decim: int = DECIM):
        """Raw targets (standardisation undone) predicted from the engines'
        device traces, and the input scales of each engine."""
        arr = self._members(engines)
        scales = np.zeros(2 * len(engines), np.float32)
        y = np.zeros((len(engines), self.out_dim), np.float32)
        N.check(N.lib().fdtd_es_predict_members(self._h, arr, len(engines), decim, N.fptr(scales), N.fptr(y)))
        return y * self.out_sd + self.out_mu, scales.reshape(-1, 2)

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            N.lib().fdtd_es_free(h)
        self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Inputs, labels and the tail model (host side, FP64)
# ---------------------------------------------------------------------------
def inputs_from_traces(V, I, in_length: int = ARCH["in_length"], decim: int = DECIM):
    """Host restatement of the device input builder: means of `decim`
    consecutive steps, each channel divided by its largest magnitude."""
    n = in_length * decim
    out, scales = [], []
    for x in (V, I):
        d = np.asarray(x[:n], dtype=np.float64).reshape(in_length, decim).mean(axis=1).astype(np.float32)
        s = float(np.abs(d).max()) or 1.0
        out.append(d / np.float32(s))
        scales.append(s)
    return np.stack(out, axis=1), np.array(scales)


@dataclass
class Mode:
    """One damped mode: x(n) = Re(c exp(s (n - n0) dt)), s = -alpha + j 2 pi f."""
    f: float        # Hz
    alpha: float    # 1/s
    cV: complex
    cI: complex
    n0: int

    def s(self) -> complex:
        return complex(-self.alpha, 2 * math.pi * self.f)

    def eval(self, which: str, n, dt: float) -> np.ndarray:
        c = self.cV if which == "V" else self.cI
        t = (np.asarray(n, dtype=np.float64) - self.n0) * dt
        return (c * np.exp(self.s() * t)).real


def _pencil_orders(signals, orders) -> list:
    """Matrix-pencil poles (per sample) shared by several equally sampled
    signals, for each model order in `orders` (one SVD serves all)."""
    Ys = []
    for x in signals:
        L = len(x) // 3
        Ys.append(np.lib.stride_tricks.sliding_window_view(np.asarray(x, dtype=np.float64), L + 1))
    Y = np.concatenate(Ys, axis=0)
    _, _, Vh = np.linalg.svd(Y, full_matrices=False)
    out = []
    for M in orders:
        Vm = Vh[:M].conj().T
        out.append(np.linalg.eigvals(np.linalg.pinv(Vm[:-1]) @ Vm[1:]))
    return out


def _pencil(signals, M: int) -> np.ndarray:
    """Matrix-pencil poles (per sample) shared by several equally sampled signals."""
    return _pencil_orders(signals, (M,))[0]


def fit_modes(x, poles, n0: int, n_start: int, dt: float):
    """Least-squares complex amplitudes c_m of sum_m Re(c_m exp(s_m (n - n0) dt))
    on the samples x[n], n = n_start, n_start+1, ...; returns the amplitudes
    and the residual energy divided by the window energy."""
    x = np.asarray(x, dtype=np.float64)
    t = (np.arange(n_start, n_start + len(x)) - n0) * dt
    cols = []
    for s in poles:
        e = np.exp(s * t)
        cols += [e.real, -e.imag]                   # Re(c e) = Re(c) Re(e) - Im(c) Im(e)
    A = np.stack(cols, axis=1)
    sol, *_ = np.linalg.lstsq(A, x, rcond=None)
    r = x - A @ sol
    energy = float(np.dot(x, x)) or 1.0
    return [complex(sol[2 * q], sol[2 * q + 1]) for q in range(len(poles))], float(np.dot(r, r)) / energy


def fit_amplitudes(x, s: complex, n0: int, n_start: int, dt: float):
    """fit_modes with one pole."""
    c, r = fit_modes(x, [s], n0, n_start, dt)
    return c[0], r


def dominant_mode(V, I, n0: int, n1: int, dt: float, decim: int = DECIM, M: int = 4,
                  fmin: float = 0.3e9, fmax: float = 6e9) -> Mode:
    """The label of a run: the mode of largest V amplitude among the poles a
    joint matrix pencil finds in the (decimated) V and I samples of [n0, n1)."""
    sv = float(np.abs(V[n0:n1]).max()) or 1.0
    si = float(np.abs(I[n0:n1]).max()) or 1.0
    z = _pencil([np.asarray(V[n0:n1:decim]) / sv, np.asarray(I[n0:n1:decim]) / si], M)
    # every pole of the upper half plane (and real ones) takes part in the
    # amplitude fit, so the dominant mode's amplitude is not biased by the rest
    poles = [complex(np.log(zz)) / (decim * dt) for zz in z if zz.imag > 0 or abs(zz.imag) < 1e-12]
    if not poles:
        raise ValueError("no mode found")
    cV, _ = fit_modes(V[n0:n1], poles, n0, n0, dt)
    cI, _ = fit_modes(I[n0:n1], poles, n0, n0, dt)
    best = None
    for q, s in enumerate(poles):
        f, alpha = s.imag / (2 * math.pi), -s.real
        if not (fmin <= f <= fmax) or alpha <= 0:
            continue
        if best is None or abs(cV[q]) > abs(best.cV):
            best = Mode(float(f), float(alpha), cV[q], cI[q], n0)
    if best is None:
        raise ValueError("no decaying mode in the band")
    return best


def mode_to_target(m: Mode, scales) -> np.ndarray:
    sv, si = scales
    return np.array([(m.f - F_CENTER) / F_SCALE, math.log(m.alpha / ALPHA_UNIT),
                     m.cV.real / sv, m.cV.imag / sv, m.cI.real / si, m.cI.imag / si], np.float32)


def target_to_mode(y, scales, n0: int) -> Mode:
    sv, si = scales
    return Mode(float(y[0]) * F_SCALE + F_CENTER, math.exp(float(y[1])) * ALPHA_UNIT,
                complex(float(y[2]), float(y[3])) * sv, complex(float(y[4]), float(y[5])) * si, n0)


def refit(V, I, mode: Mode, n_stop: int, dt: float):
    """Amplitudes of `mode` refitted on the run's steps [mode.n0, n_stop);
    returns the updated mode and the larger residual-energy ratio of V and I."""
    s = mode.s()
    cV, rv = fit_amplitudes(V[mode.n0:n_stop], s, mode.n0, mode.n0, dt)
    cI, ri = fit_amplitudes(I[mode.n0:n_stop], s, mode.n0, mode.n0, dt)
    return Mode(mode.f, mode.alpha, cV, cI, mode.n0), max(rv, ri)


def extend(V, I, mode: Mode, n_stop: int, n_total: int, dt: float):
    """Traces of a stopped run: the steps run, then the mode's tail."""
    n = np.arange(n_stop, n_total)
    return (np.concatenate([np.asarray(V[:n_stop], np.float64), mode.eval("V", n, dt)]),
            np.concatenate([np.asarray(I[:n_stop], np.float64), mode.eval("I", n, dt)]))


# ---------------------------------------------------------------------------
# Transients from the batched solver
# ---------------------------------------------------------------------------
def _variant_problem(args):
    seed, steps, per_cell = (*args, False) if len(args) == 2 else args
    from .scenario import build_problem_from_scenario
    from .workloads import ifa_variant
    return build_problem_from_scenario(ifa_variant(seed, steps=steps), steps, per_cell=per_cell)


def variant_problems(seeds, steps: int, pool=None, per_cell: bool = False) -> list:
    """Problems of the inverted-F variant family (workloads.ifa_variant).
    per_cell=False carries the material grid only (about 0.7 MB): FP32-table
    and FP64 engines build their coefficients from it on the device.
    per_cell=True adds the 18 FP64 coefficient arrays built on the host
    (about 170 MB per variant).  A process
    pool must make this package importable in its workers first (an
    initializer that loads it), or the workers cannot run the jobs."""
    jobs = [(int(s), steps, per_cell) for s in seeds]
    return pool.map(_variant_problem, jobs) if pool is not None else [_variant_problem(j) for j in jobs]


def run_variants(problems, steps: int, precision: str = "f32-table", group: int = 128, device: int = 0,
                 tiling: dict | None = None, progress=None):
    """Runs the problems `steps` steps in batches of `group` (launch shape
    `tiling`, as Batch.tiling() returns it) and returns the port traces V, I
    (len(problems) x steps, FP64) and the device seconds of the stepping.
    `progress(msg)`, if given, is called after every batch."""
    from .backend import Batch, Engine
    V = np.zeros((len(problems), steps))
    I = np.zeros((len(problems), steps))
    device_s = 0.0
    for g0 in range(0, len(problems), group):
        engs = [Engine(p, precision, device=device) for p in problems[g0:g0 + group]]
        try:
            with Batch(engs) as b:
                if tiling:
                    b.set_shape(tiling)
                device_s += b.run_timed(steps) / 1e3
            for q, e in enumerate(engs):
                V[g0 + q] = e.voltages(steps)[0]
                I[g0 + q] = e.currents(steps)[0]
        finally:
            for e in engs:
                e.close()
        if progress:
            progress(f"{g0 + len(engs)} of {len(problems)} runs, {device_s:.1f} device s")
    return V, I, device_s




# ---------------------------------------------------------------------------
# Pole sets: what the network predicts and what stops a run
# ---------------------------------------------------------------------------
PAD_POLE = complex(-5.0e9, 2 * math.pi * 7.5e9)   # fills unused slots: fast decay, above the band


def window_poles_orders(V, I, n0: int, n1: int, dt: float, orders=(12,), decim: int = DECIM,
                        fmax: float = 8e9) -> list:
    """Decaying poles (upper half plane, f <= fmax) of joint matrix pencils of
    the given orders over the decimated V and I samples of [n0, n1)."""
    sv = float(np.abs(V[n0:n1]).max()) or 1.0
    si = float(np.abs(I[n0:n1]).max()) or 1.0
    sets = []
    for z in _pencil_orders([np.asarray(V[n0:n1:decim]) / sv, np.asarray(I[n0:n1:decim]) / si], orders):
        out = []
        for zz in z:
            if not (zz.imag > 0 or abs(zz.imag) < 1e-12) or zz == 0:
                continue
            s_ = complex(np.log(zz)) / (decim * dt)
            if s_.real < 0 and s_.imag / (2 * math.pi) <= fmax:
                out.append(s_)
        sets.append(out)
    return sets


def window_poles(V, I, n0: int, n1: int, dt: float, M: int = 12, decim: int = DECIM, fmax: float = 8e9) -> list:
    """window_poles_orders for one order."""
    return window_poles_orders(V, I, n0, n1, dt, (M,), decim, fmax)[0]


def poles_to_target(poles, k: int = K_POLES) -> np.ndarray:
    """Network target of a pole set: the k slowest-decaying poles sorted by
    frequency, unused slots filled with PAD_POLE."""
    ps = sorted(poles, key=lambda s_: s_.real, reverse=True)[:k]
    ps = sorted(ps, key=lambda s_: s_.imag) + [PAD_POLE] * (k - len(ps))
    y = []
    for s_ in ps:
        y += [(s_.imag / (2 * math.pi) - F_CENTER) / F_SCALE, math.log(-s_.real / ALPHA_UNIT)]
    return np.array(y, np.float32)


def target_to_poles(y) -> list:
    y = np.asarray(y, dtype=np.float64)
    return [complex(-math.exp(y[2 * q + 1]) * ALPHA_UNIT, 2 * math.pi * (y[2 * q] * F_SCALE + F_CENTER))
            for q in range(len(y) // 2)]


# The network's target: the run's two slowest-decaying resonances inside the
# S11 band.  These decay over thousands of steps and lie close together (a few
# hundred MHz apart), which is what a short window of the run's own samples
# cannot resolve; the faster poles are left to the pencils.
N_MODES = 2
MODE_DIM = 2 * N_MODES
MODE_BAND = (1.0e9, 4.0e9)


def band_modes(poles, k: int = N_MODES, band=MODE_BAND):
    """The k slowest-decaying poles with a frequency inside `band`, slowest
    first, or None when there are fewer."""
    inb = [s_ for s_ in poles if band[0] <= s_.imag / (2 * math.pi) <= band[1] and s_.real < 0]
    if len(inb) < k:
        return None
    return sorted(inb, key=lambda s_: s_.real, reverse=True)[:k]


def modes_to_target(modes) -> np.ndarray:
    y = []
    for s_ in modes:
        y += [(s_.imag / (2 * math.pi) - F_CENTER) / F_SCALE, math.log(-s_.real / ALPHA_UNIT)]
    return np.array(y, np.float32)


def target_to_modes(y) -> list:
    return target_to_poles(y)


def mode_label(V, I, n0: int, n1: int, dt: float, M: int = 12):
    """Network target of a run: band_modes of a matrix pencil of order M over
    [n0, n1) of its own traces, or None."""
    try:
        P = window_poles(V, I, n0, n1, dt, M=M)
    except (ValueError, np.linalg.LinAlgError):
        return None
    m = band_modes(P)
    return modes_to_target(m) if m else None


def vp_refine(V, I, poles, n0: int, n1: int, dt: float, decim: int = DECIM, max_nfev: int = 60) -> list:
    """Least-squares refinement of a pole set on the decimated V and I samples
    of [n0, n1) by variable projection: the poles are the unknowns, the
    complex amplitudes of each channel are solved for inside every residual
    evaluation (Golub and Pereyra's separable least squares), Levenberg-
    Marquardt from the given start.  Frequencies and log decay rates are the
    parameters, so the poles stay decaying.  Returns the start on failure."""
    from scipy.optimize import least_squares
    if not poles:
        return []
    sv = float(np.abs(V[n0:n1]).max()) or 1.0
    si = float(np.abs(I[n0:n1]).max()) or 1.0
    xs = (np.asarray(V[n0:n1:decim], np.float64) / sv, np.asarray(I[n0:n1:decim], np.float64) / si)
    t = np.arange(xs[0].size) * decim * dt

    def unpack(p):
        # log decay rates held to [-12, 6] (1/ns): a diverging step stays finite
        return [complex(-math.exp(min(max(p[2 * q + 1], -12.0), 6.0)) * ALPHA_UNIT, 2 * math.pi * p[2 * q] * F_SCALE)
                for q in range(len(p) // 2)]

    cache = {}

    def solve(p):
        """Basis, its QR factor, the amplitudes of both channels and the
        residual, for the parameter vector p (kept for the Jacobian)."""
        key = p.tobytes()
        if key not in cache:
            cache.clear()
            S = np.array(unpack(p))
            E = np.exp(np.outer(t, S))                     # n x K complex
            A = np.empty((t.size, 2 * S.size))
            A[:, 0::2] = E.real
            A[:, 1::2] = -E.imag                          # Re(c e) = Re(c) Re(e) - Im(c) Im(e)
            Q, Rm = np.linalg.qr(A)
            cs, rs = [], []
            for x in xs:
                qx = Q.T @ x
                cs.append(np.linalg.lstsq(Rm, qx, rcond=None)[0])   # a real pole leaves a zero column
                rs.append(x - Q @ qx)
            cache[key] = (S, E, Q, cs, np.concatenate(rs))
        return cache[key]

    def res(p):
        return solve(p)[4]

    def jac(p):
        # Kaufman's variable-projection Jacobian: -(I - Q Q^T) dA/dp c
        S, E, Q, cs, _ = solve(p)
        cols = []
        for q in range(S.size):
            ds = (2j * math.pi * F_SCALE, S[q].real)        # d s / d(freq param), d s / d(log decay)
            for d in ds:
                parts = []
                for c in cs:
                    amp = complex(c[2 * q], c[2 * q + 1])
                    v = (amp * E[:, q] * t * d).real
                    parts.append(-(v - Q @ (Q.T @ v)))
                cols.append(np.concatenate(parts))
        return np.stack(cols, axis=1)

    p0 = []
    for s_ in poles:
        p0 += [s_.imag / (2 * math.pi) / F_SCALE, math.log(max(-s_.real, 1e6) / ALPHA_UNIT)]
    if len(p0) > 2 * xs[0].size:
        return list(poles)
    try:
        r = least_squares(res, np.array(p0), jac=jac, method="lm", max_nfev=max_nfev * len(p0))
    except (ValueError, OverflowError, FloatingPointError, np.linalg.LinAlgError):
        return list(poles)
    return unpack(r.x) if np.all(np.isfinite(r.x)) else list(poles)


def vp_start(V, I, n1: int, dt: float, policy, modes=None, pencil12=None) -> list:
    """Start of the refinement at checkpoint n1: the given modes (the
    network's) plus the slowest poles of the run's own pencil (order 12 over
    [n_in, n1), `pencil12` when already computed) that lie more than 10% in
    frequency away from them, up to policy.vp_poles poles in all; without
    modes, the pencil's slowest policy.vp_poles poles."""
    if pencil12 is not None:
        P = pencil12
    else:
        try:
            P = window_poles(V, I, policy.n_in, n1, dt, M=12, decim=policy.decim)
        except (ValueError, np.linalg.LinAlgError):
            P = []
    start = list(modes or [])
    for s_ in sorted(P, key=lambda z: z.real, reverse=True):
        if len(start) >= policy.vp_poles:
            break
        if all(abs(s_.imag - m.imag) > 0.1 * abs(m.imag) for m in (modes or [])):
            start.append(s_)
    return start


def pole_tail(V, I, poles, n0: int, n_stop: int, n_total: int, dt: float):
    """Amplitudes of `poles` fitted on the steps [n0, n_stop) that were run;
    returns the traces over n_total steps (run steps, then the fitted tail)
    and the larger residual-energy ratio of V and I."""
    cV, rv = fit_modes(V[n0:n_stop], poles, n0, n0, dt)
    cI, ri = fit_modes(I[n0:n_stop], poles, n0, n0, dt)
    t = (np.arange(n_stop, n_total) - n0) * dt
    tv = np.zeros(t.size)
    ti = np.zeros(t.size)
    for c1, c2, s_ in zip(cV, cI, poles):
        e = np.exp(s_ * t)
        tv += (c1 * e).real
        ti += (c2 * e).real
    return (np.concatenate([np.asarray(V[:n_stop], np.float64), tv]),
            np.concatenate([np.asarray(I[:n_stop], np.float64), ti]), max(rv, ri))


# ---------------------------------------------------------------------------
# Stopping runs early
# ---------------------------------------------------------------------------
@dataclass
class StopPolicy:
    """n_in: steps the network reads.  checkpoints: steps at which a run may
    stop.  At a checkpoint each candidate pole set (the network's, and matrix
    pencils of the run's own samples since n_in, orders `pencil_orders`) is
    fitted to [n_in, checkpoint).  The run stops when the `agree_count`
    best-fitting candidates all have a residual-energy ratio of at most
    max_resid and their extrapolated |S11| agree within agree_db (largest
    difference over S11_FREQS); it then keeps the best-fitting tail.  At the
    last checkpoint it always stops, with the best-fitting tail.  Runs that do
    not stop keep stepping (plain FDTD) to the next checkpoint.  n_total: the
    step count the result stands in for.  (On 256 held-out inverted-F
    variants, seeds 10000..10255, this rule put 98% of the runs within 0.1 dB
    of the full FP64 S11, at a mean stop of 4557 steps; a residual gate
    alone at 1e-4 put 47-55% there.)"""
    n_in: int = 1500
    checkpoints: tuple = (2300, 3000, 4000, 5000)
    max_resid: float = 1e-3
    agree_db: float = 0.02
    agree_count: int = 3
    n_total: int = 7000
    pencil_orders: tuple = (8, 12, 16)
    decim: int = DECIM
    force_last: bool = True    # the last checkpoint always stops (else: plain FDTD to n_total)
    vp: bool = False           # a refined candidate (vp_refine from vp_start) may stop a run
    vp_poles: int = 6
    vp_decim: int = 16         # the refinement fits every 16th sample (modes below 8 GHz: 4.5x oversampled)
    vp_nfev: int = 10          # residual evaluations per parameter at most

    @classmethod
    def refined(cls, **kw) -> "StopPolicy":
        """The rule the learned stop uses: checkpoints at 2300, 3000, 4000,
        5000 and 6000 steps, a run that none of them stops finishes as plain
        FP32 FDTD, and at each
        checkpoint the refined candidate (started from the network's modes, or
        from the run's own pencil without the network) stops the run when it
        agrees with the best-fitting pencil candidate; otherwise the pencils'
        own agreement rule applies."""
        base = dict(checkpoints=(2300, 3000, 4000, 5000, 6000), force_last=False, vp=True)
        base.update(kw)
        return cls(**base)


def pencil_sets(V, I, n1: int, dt: float, policy: StopPolicy, orders=None) -> list:
    """The run's pencil pole sets over [n_in, n1), one per order (empty on failure)."""
    try:
        return window_poles_orders(V, I, policy.n_in, n1, dt, orders or policy.pencil_orders, policy.decim)
    except (ValueError, np.linalg.LinAlgError):
        return [[] for _ in (orders or policy.pencil_orders)]


def candidate_poles(V, I, n1: int, dt: float, policy: StopPolicy, net_poles=None, sets=None) -> list:
    out = [list(net_poles)] if net_poles else []
    if sets is None:
        sets = pencil_sets(V, I, n1, dt, policy)
    return out + [P for P in sets if P]


def tail_candidates(V, I, n1: int, dt: float, policy: StopPolicy, net_poles=None, sets=None) -> list:
    """(traces over n_total, residual, candidate index) of every candidate pole
    set fitted to [n_in, n1), lowest residual first."""
    out = []
    for q, P in enumerate(candidate_poles(V, I, n1, dt, policy, net_poles, sets)):
        try:
            v, i, r = pole_tail(V, I, P, policy.n_in, n1, policy.n_total, dt)
        except np.linalg.LinAlgError:
            continue
        if np.isfinite(r):
            out.append((v, i, r, q))
    return sorted(out, key=lambda c: c[2])


def best_tail(V, I, n1: int, dt: float, policy: StopPolicy, net_poles=None):
    """The candidate of tail_candidates with the lowest residual, or None."""
    c = tail_candidates(V, I, n1, dt, policy, net_poles)
    return c[0] if c else None


_BASIS: dict = {}
_BASIS_LOCK = threading.Lock()


def s11_db_host(V, I, dt: float, freqs=None, z0: float = 50.0) -> np.ndarray:
    """|S11| in dB on the host: the transform of dft.js:17-38 (X(f) = dt
    sum_n x[n] exp(-j w ((n + 1) dt + shift)), shift -dt/2 for the current)
    as a matrix product with a cached basis, then postproc.s11.  The stop
    rule compares candidate tails with it; reported S11 uses s11_db."""
    from . import postproc
    freqs = S11_FREQS if freqs is None else np.asarray(freqs, dtype=np.float64)
    n = len(V)
    key = (n, float(dt), freqs.size, float(freqs[0]), float(freqs[-1]))
    with _BASIS_LOCK:
        E = _BASIS.get(key)
        if E is None:
            w = 2 * math.pi * freqs
            E = np.exp(-1j * np.outer(w, (np.arange(n) + 1) * dt))
            _BASIS.clear()
            _BASIS[key] = E
    w = 2 * math.pi * freqs
    xv = dt * (E @ np.asarray(V, dtype=np.float64))
    xi = dt * (E @ np.asarray(I, dtype=np.float64)) * np.exp(1j * w * dt / 2)
    return postproc.s11((xv.real, xv.imag), (xi.real, xi.imag), z0)["mag_dB"]


def stop_fit(V, I, n1: int, dt: float, policy: StopPolicy, net_poles=None, last: bool = False, modes=None):
    """The tail (traces over n_total, residual, candidate index) a run stops
    with at checkpoint n1, or None to keep stepping (StopPolicy's rule).
    With policy.vp the refined candidate (index -1) is tried first: it stops
    the run when it and the best-fitting pencil candidate both pass the
    residual gate and their |S11| agree within agree_db; `modes` (the
    network's) start its refinement, else the run's own pencil does."""
    orders = tuple(policy.pencil_orders) + ((12,) if policy.vp and 12 not in policy.pencil_orders else ())
    sets = pencil_sets(V, I, n1, dt, policy, orders)      # one SVD serves every order
    cands = tail_candidates(V, I, n1, dt, policy, None if policy.vp else net_poles,
                            sets[:len(policy.pencil_orders)])
    if policy.vp and cands and cands[0][2] <= policy.max_resid:
        start = vp_start(V, I, n1, dt, policy, modes, sets[orders.index(12)])
        if start:
            P = vp_refine(V, I, start, policy.n_in, n1, dt, policy.vp_decim, policy.vp_nfev)
            try:
                v, i, r = pole_tail(V, I, P, policy.n_in, n1, policy.n_total, dt)
            except np.linalg.LinAlgError:
                r = float("inf")
            if np.isfinite(r) and r <= policy.max_resid:
                a = s11_db_host(v, i, dt)
                b = s11_db_host(cands[0][0], cands[0][1], dt)
                if np.abs(a - b).max() <= policy.agree_db:
                    return v, i, r, -1
    if not cands:
        return None
    ok = [c for c in cands if c[2] <= policy.max_resid][:policy.agree_count]
    if len(ok) == policy.agree_count:
        s = [s11_db_host(c[0], c[1], dt) for c in ok]
        if all(np.abs(s[0] - x).max() <= policy.agree_db for x in s[1:]):
            return ok[0]
    return cands[0] if last else None


def _warm_worker(i: int) -> int:
    return i


def _fit_job(job):
    V, I, cp, dt, policy, net_poles, last, modes = job
    return stop_fit(V, I, cp, dt, policy, net_poles, last, modes)


_FIT_POOL = None
_FIT_WORKERS = 1
# steps of one run of the step-ahead during a checkpoint's fits: a multiple of
# the far-field DFT's time block, short against the fits' duration
AHEAD_STEPS = 48
# longest wait for one checkpoint's fits in the pool (a fit takes about 60 ms)
FIT_TIMEOUT_S = 600.0


def start_fit_pool(workers: int | None = None) -> None:
    """Starts the process pool the refined rule's checkpoint fits run in (spawned,
    so it is safe after CUDA is initialised; kept for the life of the process).
    Without it the fits run in threads of this process."""
    global _FIT_POOL, _FIT_WORKERS
    if _FIT_POOL is not None:
        return
    import runpy
    _FIT_WORKERS = workers or min(16, os.cpu_count() or 1)
    boot = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_fit_worker.py")
    _FIT_POOL = mp.get_context("spawn").Pool(_FIT_WORKERS, initializer=runpy.run_path, initargs=(boot,))
    _FIT_POOL.map(_warm_worker, range(_FIT_WORKERS), chunksize=1)   # every worker imports its modules now


def stop_fit_pool(terminate: bool = False) -> None:
    """Ends the fit pool (the fits then run in threads again); terminate=True
    kills its workers instead of waiting for them."""
    global _FIT_POOL
    if _FIT_POOL is not None:
        pool, _FIT_POOL = _FIT_POOL, None
        if terminate:
            pool.terminate()
        else:
            pool.close()
        pool.join()


def run_with_early_stop(engines, net: EsNet | None, policy: StopPolicy, tiling: dict | None = None,
                        use_network: bool = True) -> list[dict]:
    """Advances FP32 engines of one batch through the checkpoints of `policy`
    and stops each run at the first checkpoint where the policy's rule
    (stop_fit) stops it; with policy.force_last the last checkpoint always
    stops, otherwise the runs left step on to n_total as plain FDTD.  With
    use_network the network's output (predicted on the device from the first
    n_in steps) takes part: a pole set competes with the pencils, or, for a
    network of the two in-band modes (MODE_DIM outputs), the modes start the
    refined candidate.  Returns per engine {"V", "I": traces over n_total
    steps, "stopped_at", "resid", "winner": "network", "refined", "pencil" or
    "full run"}."""
    from .backend import Batch
    out = [None] * len(engines)
    net_poles = [None] * len(engines)
    active = list(range(len(engines)))
    cps = list(policy.checkpoints)

    def batch_of(qs):
        bt = Batch([engines[q] for q in qs])
        if tiling:
            bt.set_shape(tiling)
        return bt

    b = batch_of(active)
    try:
        for n, cp in enumerate(cps):
            last = n == len(cps) - 1
            if b.step < cp:
                b.run(cp - b.step)
            if use_network and net is not None and n == 0:
                sub = [engines[q] for q in active]
                for g0 in range(0, len(sub), net.max_batch):
                    y, _ = net.predict_members(sub[g0:g0 + net.max_batch], policy.decim)
                    for k, q in enumerate(active[g0:g0 + net.max_batch]):
                        net_poles[q] = target_to_poles(y[k])
            modes_net = use_network and net is not None and net.out_dim == MODE_DIM
            traces = [(engines[q].voltages(cp)[0], engines[q].currents(cp)[0]) for q in active]
            # While the host fits this checkpoint, the GPU steps every active
            # run on towards the next one (the library call releases the GIL),
            # in short runs so that it stops soon after the fits return: the
            # runs that stop here are stepped for nothing, which costs less
            # than leaving the GPU idle during the fits, but only while the
            # fits last.
            ahead, err, fitted = None, [], threading.Event()
            if not last:
                def step_ahead(bt=b, target=cps[n + 1]):
                    try:
                        while not fitted.is_set() and bt.step < target:
                            bt.run(min(AHEAD_STEPS, target - bt.step))
                    except Exception as e:  # re-raised on this thread after the fits
                        err.append(e)
                ahead = threading.Thread(target=step_ahead)
                ahead.start()

            jobs = [(traces[k][0], traces[k][1], cp, engines[q].problem.grid.dt, policy,
                     net_poles[q] if use_network and not modes_net else None, last and policy.force_last,
                     net_poles[q] if modes_net else None) for k, q in enumerate(active)]
            try:
                pool = _FIT_POOL if policy.vp else None
                if pool is not None:
                    # the refinement's Levenberg-Marquardt loop is Python: worker
                    # processes (one BLAS thread each) run the fits side by side
                    # bounded: a worker that dies leaves map() waiting for good
                    try:
                        fits = pool.map_async(_fit_job, jobs, chunksize=max(1, len(jobs) // (4 * _FIT_WORKERS))
                                              ).get(timeout=FIT_TIMEOUT_S)
                    except mp.TimeoutError:
                        stop_fit_pool(terminate=True)
                        raise RuntimeError(f"the stop fits of checkpoint {cp} did not finish in {FIT_TIMEOUT_S:.0f} s; "
                                           "the fit pool was stopped") from None
                else:
                    # LAPACK-bound fits release the GIL: one thread per host core,
                    # each with a single BLAS thread
                    with threadpool_limits(limits=1), \
                            ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 1)) as ex:
                        fits = list(ex.map(lambda j: _fit_job(j), jobs))
            finally:
                fitted.set()
                if ahead is not None:
                    ahead.join()
            if err:
                raise err[0]
            rest = []
            for k, q in enumerate(active):
                got = fits[k]
                if got is not None:
                    v, i, r, w = got
                    win = ("refined" if w == -1 else
                           "network" if (use_network and not modes_net and net_poles[q] and w == 0) else "pencil")
                    out[q] = {"V": v, "I": i, "stopped_at": cp, "resid": r, "winner": win}
                else:                      # keeps stepping (at the last checkpoint: to n_total)
                    rest.append(q)
            if last or not rest:
                break
            if len(rest) != len(active):   # the rest step on from where the step-ahead left them
                b.close()
                b = batch_of(rest)
            active = rest
    finally:
        b.close()
    leftover = [q for q in range(len(engines)) if out[q] is None]
    if leftover:
        with Batch([engines[q] for q in leftover]) as b:
            b.run(policy.n_total - b.step)
        for q in leftover:
            e = engines[q]
            out[q] = {"V": e.voltages(policy.n_total)[0], "I": e.currents(policy.n_total)[0],
                      "stopped_at": policy.n_total, "resid": float("nan"), "winner": "full run"}
    return out


def s11_db(V, I, dt: float, freqs, z0: float = 50.0) -> np.ndarray:
    """|S11| in dB of one port from its traces (postproc.port_s11, GPU DFT)."""
    from . import postproc
    return postproc.port_s11(V, I, dt, freqs, z0)["mag_dB"]


S11_FREQS = np.linspace(1e9, 4e9, 301)
