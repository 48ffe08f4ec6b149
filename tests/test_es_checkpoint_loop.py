"""The early-stop checkpoint loop's host logic (earlystop.run_with_early_stop) on the
CPU, with engines and batches faked: runs stop at the checkpoint where their
fit passes, the runs left are re-batched and stepped on, the step-ahead
during a checkpoint's fits ends soon after the fits return (in
AHEAD_STEPS pieces), traces are read only from steps an engine has reached,
and every result's trace up to its stop step is the run's own."""
import threading
import time
from types import SimpleNamespace

import numpy as np
import pytest

from conftest import load_package

pkg = load_package()
from special_topics_b200 import backend  # noqa: E402
from special_topics_b200 import earlystop as ES  # noqa: E402

N_TOTAL = 400
DT = 1e-11


class FakeEngine:
    def __init__(self, V, I):
        self.V, self.I, self.step = V, I, 0
        self.problem = SimpleNamespace(grid=SimpleNamespace(dt=DT))

    def voltages(self, n=None):
        n = self.step if n is None else n
        assert n <= self.step, f"trace of step {n} read at step {self.step}"
        return (self.V[:n].copy(),)

    def currents(self, n=None):
        n = self.step if n is None else n
        assert n <= self.step, f"trace of step {n} read at step {self.step}"
        return (self.I[:n].copy(),)


class FakeBatch:
    log = []
    lock = threading.Lock()

    def __init__(self, engines):
        assert len({e.step for e in engines}) == 1, "a batch's members are at one step"
        self.engines = engines

    @property
    def step(self):
        return self.engines[0].step

    def set_shape(self, shape):
        pass

    def run(self, count):
        assert count > 0 and self.step + count <= N_TOTAL
        time.sleep(2e-3 * count)            # the device's time for the steps
        with FakeBatch.lock:
            FakeBatch.log.append((self.step, count, len(self.engines)))
        for e in self.engines:
            e.step += count

    def close(self):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def _trace(seed, noisy):
    n = np.arange(N_TOTAL)
    rng = np.random.default_rng(seed)
    w1, w2 = 2 * np.pi * rng.uniform(1.5e9, 3.5e9) * DT, 2 * np.pi * rng.uniform(4.5e9, 6e9) * DT
    d1, d2 = rng.uniform(0.004, 0.01), rng.uniform(0.01, 0.02)
    V = np.exp(-d1 * n) * np.cos(w1 * n) + 0.5 * np.exp(-d2 * n) * np.sin(w2 * n)
    I = 0.02 * np.exp(-d1 * n) * np.sin(w1 * n + 0.3) + 0.01 * np.exp(-d2 * n) * np.cos(w2 * n)
    if noisy:
        V = V + 0.05 * rng.standard_normal(N_TOTAL)
        I = I + 0.001 * rng.standard_normal(N_TOTAL)
    return V, I


@pytest.fixture
def fake_batches(monkeypatch):
    monkeypatch.setattr(backend, "Batch", FakeBatch)
    FakeBatch.log = []
    return FakeBatch.log


def test_checkpoint_loop_stops_rebatches_and_cuts_the_step_ahead_short(fake_batches):
    noisy = [False, True, False, True, False]
    traces = [_trace(q, z) for q, z in enumerate(noisy)]
    engs = [FakeEngine(V, I) for V, I in traces]
    policy = ES.StopPolicy(n_in=40, checkpoints=(70, 250, 330), n_total=N_TOTAL, pencil_orders=(4, 6, 8),
                           decim=1, max_resid=1e-6, agree_db=1e9)
    res = ES.run_with_early_stop(engs, None, policy, {"chunk": 8, "rows": 4}, use_network=False)
    for q, r in enumerate(res):
        # clean traces fit at the first checkpoint; noisy ones only at the last (force_last)
        assert r["stopped_at"] == (330 if noisy[q] else 70), (q, r["stopped_at"])
        n = r["stopped_at"]
        assert r["V"].shape == (N_TOTAL,) and r["I"].shape == (N_TOTAL,)
        assert np.array_equal(r["V"][:n], traces[q][0][:n])
        assert np.array_equal(r["I"][:n], traces[q][1][:n])
    log = fake_batches
    # the step-ahead from checkpoint 70 ran one piece of AHEAD_STEPS on all five
    # runs, then the two runs left were re-batched and stepped on to 250
    ahead = [c for s, c, m in log if m == 5 and s >= 70]
    assert ahead and all(c <= ES.AHEAD_STEPS for c in ahead)
    assert sum(ahead) < 250 - 70
    assert any(m == 2 and s < 250 and s + c == 250 for s, c, m in log)
    assert max(e.step for e in engs) <= 330
    assert all(engs[q].step <= 70 + sum(ahead) for q in range(5) if not noisy[q])


def test_checkpoint_loop_without_stops_reaches_the_end_as_plain_runs(fake_batches):
    traces = [_trace(10 + q, True) for q in range(3)]
    engs = [FakeEngine(V, I) for V, I in traces]
    policy = ES.StopPolicy(n_in=40, checkpoints=(70, 250), n_total=N_TOTAL, pencil_orders=(4, 6, 8), decim=1,
                           max_resid=1e-6, agree_db=1e9, force_last=False)
    res = ES.run_with_early_stop(engs, None, policy, None, use_network=False)
    for q, r in enumerate(res):
        assert r["stopped_at"] == N_TOTAL and r["winner"] == "full run"
        assert np.array_equal(r["V"], traces[q][0]) and np.array_equal(r["I"], traces[q][1])
    assert all(e.step == N_TOTAL for e in engs)


class StuckPool:
    """A fit pool whose fits never return."""
    terminated = False

    def map_async(self, fn, jobs, chunksize=1):
        class Never:
            def get(self, timeout=None):
                import multiprocessing as mp
                raise mp.TimeoutError()
        return Never()

    def terminate(self):
        StuckPool.terminated = True

    def close(self):
        pass

    def join(self):
        pass


def test_stuck_fit_pool_ends_with_an_error_and_falls_back_to_threads(fake_batches, monkeypatch):
    monkeypatch.setattr(ES, "_FIT_POOL", StuckPool())
    engs = [FakeEngine(*_trace(q, False)) for q in range(2)]
    policy = ES.StopPolicy(n_in=40, checkpoints=(70, 250), n_total=N_TOTAL, pencil_orders=(4, 6, 8), decim=1,
                           max_resid=1e-6, agree_db=1e9, vp=True)
    with pytest.raises(RuntimeError, match="did not finish"):
        ES.run_with_early_stop(engs, None, policy, None, use_network=False)
    assert StuckPool.terminated and ES._FIT_POOL is None
    # the step-ahead started during the fits has ended with them
    assert all(e.step <= 70 + ES.AHEAD_STEPS for e in engs)


def test_fit_pool_and_threads_give_the_same_stops(fake_batches):
    """The refined rule's fits in the spawned pool (as the bench runs them)
    against the same fits in threads of this process."""
    noisy = [False, True, False]
    traces = [_trace(20 + q, z) for q, z in enumerate(noisy)]
    policy = ES.StopPolicy(n_in=40, checkpoints=(70, 250, 330), n_total=N_TOTAL, pencil_orders=(4, 6, 8),
                           decim=1, max_resid=1e-6, agree_db=1e9, vp=True, vp_decim=1)
    out = {}
    for name in ("threads", "pool"):
        if name == "pool":
            ES.start_fit_pool(2)
        try:
            engs = [FakeEngine(V, I) for V, I in traces]
            out[name] = ES.run_with_early_stop(engs, None, policy, None, use_network=False)
        finally:
            ES.stop_fit_pool()
    for a, b in zip(out["threads"], out["pool"]):
        assert a["stopped_at"] == b["stopped_at"] and a["winner"] == b["winner"]
        assert np.array_equal(a["V"], b["V"]) and np.array_equal(a["I"], b["I"])
