"""The early-stop network's CUDA kernels against its FP64 CPU oracle:
forward outputs, loss, and every parameter gradient (BF16 weights, FP32
accumulation on the GPU; the same BF16 weight values in FP64 on the CPU);
training reproducibility and progress; inputs built from device traces."""
import numpy as np
import pytest

import es_net_oracle as O
from conftest import load_package
from scenarios_small import small_scenario

pkg = load_package()
from special_topics_b200 import _native as N  # noqa: E402
from special_topics_b200 import earlystop as ES  # noqa: E402
from special_topics_b200.backend import Engine  # noqa: E402
from special_topics_b200.scenario import build_problem_from_scenario  # noqa: E402

pytestmark = pytest.mark.gpu

SMALL = dict(in_channels=2, in_length=23, conv_layers=2, channels=4, kernel=5, stride=2, mlp_layers=1, mlp_width=8)


def _layer_slices(arch, out_dim):
    for L in O.layers(arch, out_dim):
        for key in ("w", "b"):
            off, shape = L[key]
            yield f"{'conv' if L['conv'] else 'dense'}-{key}@{off}", slice(off, off + int(np.prod(shape)))


@pytest.mark.parametrize("arch,out_dim,B", [(O.DEFAULT_ARCH, 6, 8), (SMALL, 3, 5), (O.DEFAULT_ARCH, 6, 200)])
def test_forward_loss_and_gradients_match_oracle(arch, out_dim, B):
    rng = np.random.default_rng(7)
    with ES.EsNet(out_dim, max_batch=256, **arch) as net:
        assert net.n_params == O.param_count(arch, out_dim)
        net.init(3)
        p = net.params
        x = rng.standard_normal((B, arch["in_length"], 2)).astype(np.float32)
        t = rng.standard_normal((B, out_dim)).astype(np.float32)
        w = rng.uniform(0.5, 2.0, out_dim).astype(np.float32)
        y = net.forward(x)
        yo, _ = O.forward(arch, out_dim, p, x)
        assert np.abs(y - yo).max() <= 1e-4 * np.abs(yo).max() + 1e-6
        loss, g = net.loss_grad(x, t, w)
        lo, go = O.loss_grad(arch, out_dim, p, x, t, w)
        assert abs(loss - lo) <= 1e-4 * lo
        for name, sl in _layer_slices(arch, out_dim):
            scale = np.abs(go[sl]).max()
            assert np.abs(g[sl] - go[sl]).max() <= 2e-3 * scale + 1e-9, (name, np.abs(g[sl] - go[sl]).max(), scale)


def test_params_roundtrip_and_bf16_compute_copy():
    rng = np.random.default_rng(1)
    with ES.EsNet(3, max_batch=8, **SMALL) as net:
        p = rng.standard_normal(net.n_params).astype(np.float32)
        net.params = p
        assert np.array_equal(net.params, p)
        x = rng.standard_normal((4, SMALL["in_length"], 2)).astype(np.float32)
        # the forward pass sees the BF16 weights: the oracle with BF16 weights
        # agrees, the oracle with exact FP32 weights does not
        yo, _ = O.forward(SMALL, 3, p, x, bf16=True)
        ye, _ = O.forward(SMALL, 3, p, x, bf16=False)
        y = net.forward(x)
        assert np.abs(y - yo).max() < 1e-4 * np.abs(yo).max()
        assert np.abs(y - ye).max() > 10 * np.abs(y - yo).max()
        with pytest.raises(N.FdtdError):
            net.params = p[:-1]
        with pytest.raises(N.FdtdError):
            net.forward(np.zeros((9, SMALL["in_length"], 2), np.float32))


def _sinusoid_task(n, rng, L=64):
    """Inputs: damped sinusoids; targets: their frequency and decay."""
    f = rng.uniform(0.05, 0.2, n)
    a = rng.uniform(0.005, 0.05, n)
    t = np.arange(L)
    v = np.exp(-a[:, None] * t) * np.cos(2 * np.pi * f[:, None] * t)
    i = np.exp(-a[:, None] * t) * np.sin(2 * np.pi * f[:, None] * t)
    x = np.stack([v, i], axis=2).astype(np.float32)
    y = np.stack([(f - 0.125) / 0.05, (a - 0.0275) / 0.015], axis=1).astype(np.float32)
    return x, y


def test_training_reduces_loss_and_is_reproducible():
    rng = np.random.default_rng(5)
    arch = dict(in_channels=2, in_length=64, conv_layers=3, channels=16, kernel=5, stride=2, mlp_layers=2,
                mlp_width=64)
    x, y = _sinusoid_task(1024, rng)
    xt, yt = _sinusoid_task(256, rng)
    params = []
    for _ in range(2):
        with ES.EsNet(2, max_batch=256, **arch) as net:
            net.init(11)
            before, _ = net.loss_grad(xt, yt, grad=False)
            losses = net.train(x, y, epochs=40, batch=64, lr=2e-3, seed=4)
            after, _ = net.loss_grad(xt, yt, grad=False)
            params.append(net.params)
    assert losses[-1] < 0.05 * losses[0]
    assert after < 0.05 * before
    assert np.array_equal(params[0], params[1])


def test_inputs_from_member_traces_match_host_restatement():
    arch = dict(SMALL, in_length=15)
    scns = [small_scenario(1, "xp"), small_scenario(3, "zp", ncpml=(5, 4, 3, 3, 4, 5))]
    engs = [Engine(build_problem_from_scenario(s, 70), "f32-table") for s in scns]
    try:
        with ES.EsNet(3, max_batch=4, **arch) as net:
            net.init(2)
            with pytest.raises(N.FdtdError):
                net.member_inputs(engs)            # not enough steps yet
            for e in engs:
                e.run(70)
            x, s = net.member_inputs(engs)
            for b, e in enumerate(engs):
                xh, sh = ES.inputs_from_traces(e.voltages()[0], e.currents()[0], in_length=15)
                assert np.allclose(x[b], xh, rtol=1e-6, atol=1e-7)
                assert np.allclose(s[b], sh, rtol=1e-6)
            y, _ = net.predict_members(engs)
            assert np.array_equal(y, net.forward(x))
    finally:
        for e in engs:
            e.close()
