"""CPU checks of the early-stop network's FP64 oracle and of the host-side
tail model (no GPU): BF16 rounding against torch's, the oracle's analytic
backward pass against finite differences, and mode fitting on synthetic
ringing with known parameters."""
import numpy as np
import pytest
import torch

import es_net_oracle as O
import oracle
from conftest import load_package

pkg = load_package()
from special_topics_b200 import earlystop as ES  # noqa: E402

SMALL = dict(in_channels=2, in_length=23, conv_layers=2, channels=4, kernel=5, stride=2, mlp_layers=1,
             mlp_width=8)


def test_bf16_round_matches_torch():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.standard_normal(20000) * 10.0 ** rng.integers(-30, 30, 20000),
                        [0.0, -0.0, 1.0, 1.00390625, 1.01171875, 3.4e38, -3.4e38, 1e-40, np.inf, -np.inf]])
    x = x.astype(np.float32)
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(O.bf16_round(x).view(np.uint32), ref.view(np.uint32))
    assert np.isnan(O.bf16_round(np.array([np.nan], np.float32)))[0]


def test_layer_table_and_param_count():
    Ls = O.layers(O.DEFAULT_ARCH, 6)
    assert [L["lout"] for L in Ls if L["conv"]] == [188, 94, 47, 24]
    assert O.param_count(O.DEFAULT_ARCH, 6) == (64 * 5 * 2 + 64) + 3 * (64 * 5 * 64 + 64) + (1536 * 256 + 256) \
        + (256 * 256 + 256) + (256 * 6 + 6)


@pytest.mark.parametrize("seed", [0, 1])
def test_oracle_backward_matches_finite_differences(seed):
    rng = np.random.default_rng(seed)
    n = O.param_count(SMALL, 3)
    p = rng.uniform(-0.5, 0.5, n)
    x = rng.standard_normal((5, SMALL["in_length"], 2))
    t = rng.standard_normal((5, 3))
    w = np.array([1.0, 0.5, 2.0])
    loss, g = O.loss_grad(SMALL, 3, p, x, t, w, bf16=False)
    assert abs(loss - O.loss(SMALL, 3, p, x, t, w, bf16=False)) < 1e-12
    idx = rng.choice(n, 60, replace=False)
    fd = O.finite_difference(SMALL, 3, p, x, t, w, idx)
    assert np.allclose(g[idx], fd, rtol=1e-5, atol=1e-8), np.abs(g[idx] - fd).max()


def test_inputs_from_traces_scales_each_channel():
    rng = np.random.default_rng(3)
    V, I = rng.standard_normal(1600), 0.01 * rng.standard_normal(1600)
    x, s = ES.inputs_from_traces(V, I)
    assert x.shape == (375, 2) and x.dtype == np.float32
    assert np.isclose(np.abs(x).max(axis=0), 1.0).all()
    assert np.isclose(s[0], np.abs(V[:1500].reshape(375, 4).mean(1)).max())


def _ringing(m, n, extra=None, dt=8.666e-13):
    V, I = m.eval("V", np.arange(n), dt), m.eval("I", np.arange(n), dt)
    if extra is not None:
        V = V + extra.eval("V", np.arange(n), dt)
        I = I + extra.eval("I", np.arange(n), dt)
    return V, I


def test_dominant_mode_recovers_a_damped_sinusoid():
    dt = 8.666e-13
    m0 = ES.Mode(2.17e9, 0.46e9, 0.011 - 0.004j, 1.5e-4 + 2e-5j, 1500)
    V, I = _ringing(m0, 7000, extra=ES.Mode(4.9e9, 2.5e9, 0.002, 3e-5, 1500))
    m = ES.dominant_mode(V, I, 1500, 7000, dt)
    assert abs(m.f - m0.f) < 1e3 and abs(m.alpha - m0.alpha) < 1e3
    assert abs(m.cV - m0.cV) < 1e-6 and abs(m.cI - m0.cI) < 1e-8
    y = ES.mode_to_target(m, (0.02, 3e-4))
    back = ES.target_to_mode(y, (0.02, 3e-4), 1500)
    assert abs(back.f - m.f) < 1e3 and abs(back.alpha / m.alpha - 1) < 1e-6


def test_refit_residual_separates_one_mode_from_two():
    dt = 8.666e-13
    m = ES.Mode(2.17e9, 0.46e9, 0.011, 1.5e-4, 1500)
    V, I = _ringing(m, 2000)
    guess = ES.Mode(m.f, m.alpha, 0j, 0j, 1500)
    got, r = ES.refit(V, I, guess, 2000, dt)
    assert r < 1e-20 and abs(got.cV - m.cV) < 1e-12
    V2, I2 = _ringing(m, 2000, extra=ES.Mode(3.1e9, 0.2e9, 0.008, 1e-4, 1500))
    _, r2 = ES.refit(V2, I2, guess, 2000, dt)
    assert r2 > 0.05
    Ve, _ = ES.extend(V, I, got, 1800, 7000, dt)
    full_V, _ = _ringing(m, 7000)
    assert len(Ve) == 7000 and np.allclose(Ve, full_V, atol=1e-12)


def test_pole_targets_round_trip_and_pad():
    poles = [complex(-0.4e9, 2 * np.pi * 2.1e9), complex(-2.0e9, 2 * np.pi * 6.6e9), complex(-0.2e9, 2 * np.pi * 0.7e9)]
    y = ES.poles_to_target(poles)
    assert y.shape == (ES.OUT_DIM,)
    back = ES.target_to_poles(y)
    got = sorted(back[:3], key=lambda s: s.imag)
    want = sorted(poles, key=lambda s: s.imag)
    for a, b in zip(got, want):
        assert abs(a - b) / abs(b) < 1e-6
    assert all(abs(p - ES.PAD_POLE) / abs(ES.PAD_POLE) < 1e-6 for p in back[3:])


def test_window_poles_and_tail_recover_two_modes():
    dt = 8.666e-13
    m1 = ES.Mode(2.09e9, 0.45e9, 0.011 - 0.004j, 1.5e-4 + 2e-5j, 1500)
    m2 = ES.Mode(2.61e9, 0.9e9, 0.004 + 0.002j, -4e-5 + 1e-5j, 1500)
    V, I = _ringing(m1, 7000, extra=m2)
    P = ES.window_poles(V, I, 1500, 3500, dt, M=4)
    assert len(P) == 2
    v, i, r = ES.pole_tail(V, I, P, 1500, 2300, 7000, dt)
    assert r < 1e-12
    assert np.allclose(v, V, atol=1e-9) and np.allclose(i, I, atol=1e-11)
    pol = ES.StopPolicy(pencil_orders=(4,))
    got = ES.best_tail(V, I, 2300, dt, pol)
    assert got is not None and got[2] < 1e-12


def test_stop_rule_needs_agreeing_candidates():
    dt = 8.666e-13
    m1 = ES.Mode(2.09e9, 0.45e9, 0.011 - 0.004j, 1.5e-4 + 2e-5j, 1500)
    m2 = ES.Mode(2.61e9, 0.9e9, 0.004 + 0.002j, -4e-5 + 1e-5j, 1500)
    V, I = _ringing(m1, 7000, extra=m2)
    # host S11 of the rule follows the reference's transform (oracle restatement)
    Vr, Vi = oracle.time_to_freq(V, dt, ES.S11_FREQS, 0.0)
    Ir, Ii = oracle.time_to_freq(I, dt, ES.S11_FREQS, -dt / 2)
    want = oracle.s11((Vr, Vi), (Ir, Ii), 50.0)["mag_dB"]
    assert np.allclose(ES.s11_db_host(V, I, dt), want, atol=1e-9)
    # three exact candidates agree: the run stops with an exact tail
    pol = ES.StopPolicy(pencil_orders=(4, 4, 4))
    got = ES.stop_fit(V, I, 2300, dt, pol)
    assert got is not None and got[2] < 1e-12
    # candidates that may not differ at all never agree: keep stepping, except at the last checkpoint
    strict = ES.StopPolicy(pencil_orders=(4, 4, 4), agree_db=-1.0)
    assert ES.stop_fit(V, I, 2300, dt, strict) is None
    assert ES.stop_fit(V, I, 2300, dt, strict, last=True) is not None
    # too few candidates pass the residual gate: keep stepping
    assert ES.stop_fit(V, I, 2300, dt, ES.StopPolicy(pencil_orders=(4,))) is None


def test_growth_onset_finds_late_growth():
    from special_topics_b200 import postproc
    n = np.arange(7000)
    decay = np.exp(-n / 800.0) * np.cos(0.1 * n)
    growth = 1e-6 * np.exp((n - 7000) / 300.0 + 12) * np.cos(2.5 * n)
    assert postproc.growth_onset(decay) == -1
    on = postproc.growth_onset(decay + growth)
    assert 4000 < on < 7000


def test_band_modes_label_round_trip():
    poles = [complex(-3e9, 0.0), complex(-0.4e9, 2 * np.pi * 1.9e9), complex(-2.5e9, 2 * np.pi * 2.1e9),
             complex(-0.3e9, 2 * np.pi * 5.2e9), complex(-5e9, 2 * np.pi * 0.5e9)]
    m = ES.band_modes(poles)
    assert m == [poles[1], poles[2]]                  # in 1-4 GHz, slowest first; 5.2 GHz and the real pole left out
    back = ES.target_to_modes(ES.modes_to_target(m))
    for a, b in zip(back, m):
        assert abs(a - b) / abs(b) < 1e-6
    assert ES.band_modes(poles[:2]) is None


def test_refinement_recovers_close_modes_from_a_rough_start():
    """Two resonances 180 MHz apart plus a fast one, seen only over steps
    1500-2300: the refinement from a start 2% off in frequency (30% in
    decay) finds the exact poles, and the refined candidate then stops the
    run under StopPolicy.refined() with the exact tail."""
    dt = 8.666e-13
    m1 = ES.Mode(2.09e9, 0.45e9, 0.011 - 0.004j, 1.5e-4 + 2e-5j, 1500)
    m2 = ES.Mode(2.27e9, 1.9e9, 0.006 + 0.002j, -6e-5 + 1e-5j, 1500)
    m3 = ES.Mode(5.1e9, 3.0e9, 0.003 + 0.001j, 2e-5 - 1e-5j, 1500)
    V, I = _ringing(m1, 7000, extra=m2)
    V = V + m3.eval("V", np.arange(7000), dt)
    I = I + m3.eval("I", np.arange(7000), dt)
    true = [m.s() for m in (m1, m2, m3)]
    start = [complex(s.real * 1.3, s.imag * 1.02) for s in true]
    got = ES.vp_refine(V, I, start, 1500, 2300, dt)
    for a, b in zip(sorted(got, key=lambda z: z.imag), true):
        assert abs(a - b) / abs(b) < 1e-6
    pol = ES.StopPolicy.refined(pencil_orders=(6, 6, 6), vp_poles=3)
    fit = ES.stop_fit(V, I, 2300, dt, pol, modes=[start[0], start[1]])
    assert fit is not None and fit[3] == -1 and fit[2] < 1e-10
    assert np.allclose(fit[0], V, atol=1e-9) and np.allclose(fit[1], I, atol=1e-11)


def test_fit_pool_gives_the_in_process_fits():
    """The refined rule's checkpoint fits in the spawned worker pool give what
    the same fits give in this process."""
    dt = 8.666e-13
    m1 = ES.Mode(2.09e9, 0.45e9, 0.011 - 0.004j, 1.5e-4 + 2e-5j, 1500)
    m2 = ES.Mode(2.27e9, 1.9e9, 0.006 + 0.002j, -6e-5 + 1e-5j, 1500)
    V, I = _ringing(m1, 7000, extra=m2)
    pol = ES.StopPolicy.refined(pencil_orders=(4, 4, 4), vp_poles=2)
    modes = [complex(m1.s().real * 1.2, m1.s().imag * 1.01), complex(m2.s().real * 0.8, m2.s().imag * 0.99)]
    jobs = [(V[:cp], I[:cp], cp, dt, pol, None, False, modes) for cp in (2300, 3000)]
    from threadpoolctl import threadpool_info
    ES.start_fit_pool(2)
    try:
        got = ES._FIT_POOL.map(ES._fit_job, jobs)
        # every worker's BLAS libraries (NumPy's and SciPy's) run one thread:
        # workers of one BLAS thread per core each slowed the fits 10-40x
        infos = [ES._FIT_POOL.apply_async(threadpool_info).get(timeout=60) for _ in range(4)]
    finally:
        ES.stop_fit_pool()
    for info in infos:
        blas = [d for d in info if d["user_api"] == "blas"]
        assert blas and all(d["num_threads"] == 1 for d in blas), blas
    for job, g in zip(jobs, got):
        want = ES._fit_job(job)
        assert (g is None) == (want is None)
        if want is not None:
            assert g[3] == want[3] and np.array_equal(g[0], want[0]) and g[2] == want[2]
