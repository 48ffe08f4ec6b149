"""Learned early stop: a 1-D conv + MLP network reads the early port
transient of a run and predicts its late-time ringing tail, so the run can
stop long before numberOfTimeSteps.

The reference always runs every step (js_fdtd/src/index.js:54-60) and turns
the full port traces into S11 (index.js:62-75, dft.js:17-38); this module is
the part with no counterpart there.

Model of the tail.  After the source pulse has left, the port voltage and
current of a linear, passive structure ring down as a sum of damped
sinusoids; for the inverted-F family one mode dominates.  The network maps
the first `n_in` steps (4x decimated, each channel scaled by its largest
magnitude) to that mode's frequency and decay rate and to the complex
amplitudes of V and I at step `n_in`.  The tail of a run stopped at step
`n_stop` is x(n) = Re(c exp(s (n - n_in) dt)), s = -alpha + j 2 pi f, with
the amplitudes c refitted by least squares on the steps [n_in, n_stop) that
were actually run.  The residual energy of that fit is the gate: above the
threshold the run is not stopped and keeps stepping (plain FDTD).

`EsNet` is the handle of the CUDA network (include/fdtd_b200.h, fdtd_es_*):
training, gradients and inference all run in the project's own kernels.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _native as N

ARCH = dict(in_channels=2, in_length=375, conv_layers=4, channels=64, kernel=5, stride=2, mlp_layers=2,
            mlp_width=256)
OUT_DIM = 6          # f, log alpha, Re/Im c_V, Re/Im c_I
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


def _pencil(signals, M: int) -> np.ndarray:
    """Matrix-pencil poles (per sample) shared by several equally sampled signals."""
    Ys = []
    for x in signals:
        L = len(x) // 3
        Ys.append(np.lib.stride_tricks.sliding_window_view(np.asarray(x, dtype=np.float64), L + 1))
    Y = np.concatenate(Ys, axis=0)
    _, _, Vh = np.linalg.svd(Y, full_matrices=False)
    Vm = Vh[:M].conj().T
    return np.linalg.eigvals(np.linalg.pinv(Vm[:-1]) @ Vm[1:])


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
    seed, steps = args
    from .scenario import build_problem_from_scenario
    from .workloads import ifa_variant
    return build_problem_from_scenario(ifa_variant(seed, steps=steps), steps, per_cell=False)


def variant_problems(seeds, steps: int, pool=None) -> list:
    """Problems of the inverted-F variant family (workloads.ifa_variant).
    A process pool must make this package importable in its workers first
    (an initializer that loads it), or the workers cannot run the jobs."""
    jobs = [(int(s), steps) for s in seeds]
    return pool.map(_variant_problem, jobs) if pool is not None else [_variant_problem(j) for j in jobs]


def run_variants(problems, steps: int, precision: str = "f32-table", group: int = 128, device: int = 0,
                 tiling: dict | None = None):
    """Runs the problems `steps` steps in batches of `group` (launch shape
    `tiling`, as Batch.tiling() returns it) and returns the port traces V, I
    (len(problems) x steps, FP64) and the device seconds of the stepping."""
    from .backend import Batch, Engine
    V = np.zeros((len(problems), steps))
    I = np.zeros((len(problems), steps))
    device_s = 0.0
    for g0 in range(0, len(problems), group):
        engs = [Engine(p, precision, device=device) for p in problems[g0:g0 + group]]
        try:
            with Batch(engs) as b:
                if tiling:
                    b.set_tiling(tiling["chunk"], tiling["rows"], tiling["prefetch"], tiling["group"])
                device_s += b.run_timed(steps) / 1e3
            for q, e in enumerate(engs):
                V[g0 + q] = e.voltages(steps)[0]
                I[g0 + q] = e.currents(steps)[0]
        finally:
            for e in engs:
                e.close()
    return V, I, device_s


# ---------------------------------------------------------------------------
# Stopping runs early
# ---------------------------------------------------------------------------
@dataclass
class StopPolicy:
    """n_in: steps the network reads; n_check: steps run past n_in whose
    samples refit the amplitudes and measure the residual; max_resid: the
    residual-energy ratio above which a run is not stopped; n_total: the
    step count the result stands in for (numberOfTimeSteps)."""
    n_in: int = 1500
    n_check: int = 300
    max_resid: float = 0.03
    n_total: int = 7000
    decim: int = DECIM

    @property
    def n_stop(self) -> int:
        return self.n_in + self.n_check


def pencil_mode(V, I, n0: int, n1: int, dt: float, decim: int = DECIM) -> Mode:
    """The method without the network: the dominant mode estimated from the
    run's own samples [n0, n1) by the joint matrix pencil."""
    return dominant_mode(V, I, n0, n1, dt, decim=decim)


def decide(V, I, mode: Mode | None, policy: StopPolicy, dt: float):
    """Refits `mode` on [n_in, n_stop) and applies the residual-energy gate.
    Returns (accepted, refitted mode or None, residual)."""
    if mode is None or not (mode.alpha > 0 and math.isfinite(mode.f)):
        return False, None, float("inf")
    m, r = refit(V, I, mode, policy.n_stop, dt)
    return r <= policy.max_resid, m, r


def run_with_early_stop(engines, net: EsNet | None, policy: StopPolicy, tiling: dict | None = None,
                        use_network: bool = True) -> list[dict]:
    """Advances FP32 engines of one batch to policy.n_stop, predicts each run's
    tail mode (the network, or the pencil on the run's own samples when
    use_network is False), and stops the runs whose refit passes the gate;
    the others keep stepping to n_total (plain FDTD).  Returns per engine
    {"V", "I": traces over n_total steps (stopped runs extended with their
    tail), "stopped_at", "accepted", "resid", "mode"}."""
    from .backend import Batch
    with Batch(engines) as b:
        if tiling:
            b.set_tiling(tiling["chunk"], tiling["rows"], tiling["prefetch"], tiling["group"])
        b.run(policy.n_stop - b.step)
    modes = [None] * len(engines)
    if use_network:
        y, scales = net.predict_members(engines, policy.decim)
        modes = [target_to_mode(y[q], scales[q], policy.n_in) for q in range(len(engines))]
    out, rest = [], []
    for q, e in enumerate(engines):
        dt = e.problem.grid.dt
        V, I = e.voltages(policy.n_stop)[0], e.currents(policy.n_stop)[0]
        m = modes[q]
        if not use_network:
            try:
                m = pencil_mode(V, I, policy.n_in, policy.n_stop, dt, policy.decim)
            except (ValueError, np.linalg.LinAlgError):
                m = None
        ok, fit, r = decide(V, I, m, policy, dt)
        rec = {"accepted": ok, "resid": r, "mode": fit, "stopped_at": policy.n_stop}
        if ok:
            rec["V"], rec["I"] = extend(V, I, fit, policy.n_stop, policy.n_total, dt)
        else:
            rest.append(q)
        out.append(rec)
    if rest:
        with Batch([engines[q] for q in rest]) as b:
            if tiling:
                b.set_tiling(tiling["chunk"], tiling["rows"], tiling["prefetch"], tiling["group"])
            b.run(policy.n_total - b.step)
        for q in rest:
            e = engines[q]
            out[q]["V"], out[q]["I"] = e.voltages(policy.n_total)[0], e.currents(policy.n_total)[0]
            out[q]["stopped_at"] = policy.n_total
    return out


def s11_db(V, I, dt: float, freqs, z0: float = 50.0) -> np.ndarray:
    """|S11| in dB of one port from its traces (postproc.port_s11, GPU DFT)."""
    from . import postproc
    return postproc.port_s11(V, I, dt, freqs, z0)["mag_dB"]


S11_FREQS = np.linspace(1e9, 4e9, 301)
