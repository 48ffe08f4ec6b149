"""Batched runs: members of uneven size advanced together give exactly what
each member gives when run on its own (same kernels, same arithmetic per
cell), for every launch shape, including the persistent tile-claiming grid."""
import numpy as np
import pytest

import oracle
from conftest import load_package, load_scenario
from scenarios_small import small_scenario

pkg = load_package()
from special_topics_b200 import _native as N  # noqa: E402
from special_topics_b200.backend import Batch, Engine  # noqa: E402
from special_topics_b200.scenario import FF_NAMES, build_problem_from_scenario  # noqa: E402

pytestmark = pytest.mark.gpu

STEPS = 70   # one 64-step graph replay plus 6 single steps


def _members(steps=STEPS):
    scns = [small_scenario(1, "xp"), small_scenario(2, "yn", ncpml=(3, 3, 5, 4, 6, 3)),
            small_scenario(3, "zp", ncpml=(5, 4, 3, 3, 4, 5)), load_scenario("ifa-fr4-substrate")]
    return [build_problem_from_scenario(s, steps) for s in scns]


def _state(eng):
    out = {"V": eng.voltages(), "I": eng.currents()}
    for f in ("Hx", "Hy", "Hz", "Ex", "Ey", "Ez"):
        out[f] = eng.field(f)
    ff = eng.farfield()
    for a in FF_NAMES:
        out[a] = ff[a]
    return out


def _assert_same(a, b, tag):
    for key in a:
        x, y = a[key], b[key]
        if isinstance(x, (list, tuple)):
            for q, (u, v) in enumerate(zip(x, y)):
                assert np.array_equal(u, v), f"{tag} {key}[{q}]"
        else:
            assert np.array_equal(x, y), f"{tag} {key}"


@pytest.fixture(scope="module", params=["f64", "f32-table"])
def solo(request):
    probs = _members()
    states = []
    for p in probs:
        with Engine(p, request.param) as eng:
            eng.run(STEPS)
            states.append(_state(eng))
    return request.param, states


@pytest.mark.parametrize("chunk,rows,pf,group,streams",
                         [(8, 4, 1, 0, 0), (3, 2, 2, 0, 0), (1, 8, 1, 1, 0), (5, 4, 1, 7, 0), (16, 2, 2, 3, 0),
                          (8, 4, 3, 0, 0), (4, 8, 4, 2, 0),
                          # member-kernel mode: 1 stream, fewer streams than members, more streams than members
                          (8, 4, 1, 0, 1), (3, 2, 2, 0, 3), (16, 4, 1, 0, 6), (8, 4, 3, 0, 2)])
def test_batch_matches_solo_runs(solo, chunk, rows, pf, group, streams):
    precision, states = solo
    if pf > 2 and precision != "f32-table":
        pytest.skip("shared-memory stages are a material-table form")
    engs = [Engine(p, precision) for p in _members()]
    try:
        with Batch(engs, chunk, rows, pf, group, streams) as b:
            assert b.tiling() == {"chunk": chunk, "rows": rows, "prefetch": pf, "group": group, "streams": streams,
                                  "width": 32, "per_launch": 0}
            b.run(STEPS)
            assert b.step == STEPS
        for q, e in enumerate(engs):
            assert e.step == STEPS
            assert e.status() == (0, -1)
            _assert_same(states[q], _state(e), f"member {q}")
    finally:
        for e in engs:
            e.close()


@pytest.mark.parametrize("chunk,rows,pf,width,per_launch",
                         [(8, 4, 1, 32, 1), (3, 2, 2, 32, 3), (64, 8, 1, 16, 22), (8, 4, 3, 32, 2),
                          (16, 16, 4, 16, 4), (5, 4, 1, 16, 3)])
def test_grouped_batch_matches_solo_runs(solo, chunk, rows, pf, width, per_launch):
    """Grouped mode: members' parameter blocks as kernel parameters, one
    member per launch up to all of them in one, launches side by side."""
    precision, states = solo
    if pf > 2 and precision != "f32-table":
        pytest.skip("shared-memory stages are a material-table form")
    engs = [Engine(p, precision) for p in _members()]
    try:
        with Batch(engs) as b:
            b.set_tiling(chunk, rows, pf, 0, 0, width, per_launch)
            assert b.tiling()["per_launch"] == per_launch
            b.run(STEPS)
            assert b.step == STEPS
        for q, e in enumerate(engs):
            assert e.step == STEPS
            assert e.status() == (0, -1)
            _assert_same(states[q], _state(e), f"member {q}")
    finally:
        for e in engs:
            e.close()


def test_grouped_mode_rejects_too_many_members_per_launch():
    engs = [Engine(p, "f32-table") for p in _members(8)[:2]]
    try:
        with Batch(engs) as b:
            with pytest.raises(N.FdtdError):
                b.set_tiling(8, 4, 1, 0, 0, 32, 23)
    finally:
        for e in engs:
            e.close()


def test_batch_fp64_matches_oracle():
    scn = small_scenario(5, "yn", ncpml=(3, 4, 5, 6, 3, 4))
    o = oracle.Oracle(scn, 40)
    o.step(40)
    probs = [build_problem_from_scenario(scn, 40), build_problem_from_scenario(small_scenario(6, "zp"), 40)]
    engs = [Engine(p, "f64") for p in probs]
    try:
        with Batch(engs, 4, 4, 1, 2) as b:
            b.run(25)
            b.run(15)    # a second run resumes from the members' step
        assert np.array_equal(engs[0].voltages()[0], o.get("V:0"))
        assert np.array_equal(engs[0].currents()[0], o.get("I:0"))
        assert np.array_equal(engs[0].field("Ez"), o.get("Ez"))
        # members keep running on their own after the batch is gone
        engs[1].run(0)
    finally:
        for e in engs:
            e.close()


def test_batch_and_solo_steps_interleave():
    probs = _members(40)
    ref = []
    for p in probs[:2]:
        with Engine(p, "f32-table") as e:
            e.run(40)
            ref.append(_state(e))
    engs = [Engine(p, "f32-table") for p in probs[:2]]
    try:
        engs[0].run(10)
        engs[1].run(10)
        with Batch(engs) as b:
            b.run(20)
        engs[0].run(10)
        engs[1].run(10)
        for q in range(2):
            _assert_same(ref[q], _state(engs[q]), f"member {q}")
    finally:
        for e in engs:
            e.close()


def test_batch_argument_errors():
    probs = _members(30)
    a = Engine(probs[0], "f32-table")
    b = Engine(probs[1], "f32-table")
    c = Engine(probs[2], "f64")
    try:
        with pytest.raises(N.FdtdError) as ei:
            Batch([a, c])
        assert ei.value.code == N.FDTD_ERR_BADARG
        with pytest.raises(N.FdtdError) as ei:
            Batch([a, a])
        assert ei.value.code == N.FDTD_ERR_BADARG
        with Batch([a, b]) as bt:
            with pytest.raises(N.FdtdError):
                bt.set_tiling(0, 4)
            with pytest.raises(N.FdtdError):
                bt.set_tiling(8, 3)
            a.run(5)
            with pytest.raises(N.FdtdError) as ei:
                bt.run(5)
            assert ei.value.code == N.FDTD_ERR_STATE
            b.run(5)
            with pytest.raises(N.FdtdError) as ei:
                bt.run(26)
            assert ei.value.code == N.FDTD_ERR_BADARG
            bt.run(25)
            assert a.step == b.step == 30
    finally:
        for e in (a, b, c):
            e.close()


def test_batch_watchdog_names_the_member():
    probs = _members(30)[:3]
    probs[1].voltage_sources[0].voltage_per_e_field[9] = np.nan
    engs = [Engine(p, "f32-table") for p in probs]
    try:
        with Batch(engs) as b:
            with pytest.raises(N.FdtdError) as ei:
                b.run(30)
            assert ei.value.code == N.FDTD_ERR_NONFINITE
            assert "member 1" in str(ei.value)
        assert engs[1].status() == (N.FDTD_ERR_NONFINITE, 9)
        assert engs[0].status() == (0, -1) and engs[2].status() == (0, -1)
    finally:
        for e in engs:
            e.close()


def test_batch_with_time_blocked_dft_matches_solo_runs():
    probs = [build_problem_from_scenario(s, 90, per_cell=False)
             for s in (small_scenario(1, "xp"), small_scenario(3, "zp", ncpml=(5, 4, 3, 3, 4, 5)))]
    solo = []
    for p in probs:
        with Engine(p, "f32-table", dft_block=16) as e:
            e.run(70)
            e.run(20)
            solo.append(_state(e))
    engs = [Engine(p, "f32-table", dft_block=16) for p in probs]
    try:
        with Batch(engs) as b:
            b.run(70)
            b.run(20)
        for q, e in enumerate(engs):
            _assert_same(solo[q], _state(e), f"member {q}")
    finally:
        for e in engs:
            e.close()


def test_batch_modes_alternate_within_one_run_sequence():
    """Tile-list, member-kernel and grouped runs of the same batch continue each other
    (the step counters and blocked-DFT state carry over between the modes)."""
    probs = [build_problem_from_scenario(s, 200, per_cell=False)
             for s in (small_scenario(1, "xp"), small_scenario(2, "yn", ncpml=(3, 3, 5, 4, 6, 3)),
                       small_scenario(3, "zp", ncpml=(5, 4, 3, 3, 4, 5)))]
    solo = []
    for p in probs:
        with Engine(p, "f32-table", dft_block=16) as e:
            e.run(200)
            solo.append(_state(e))
    engs = [Engine(p, "f32-table", dft_block=16) for p in probs]
    try:
        with Batch(engs) as b:
            b.run(30)                     # tile-list, no graph
            b.set_tiling(8, 4, 1, 0, 2)
            b.run(70)                     # member kernels: one graph replay + 6 steps
            b.set_tiling(16, 2, 1, 0, 0, 32, 2)
            b.run(64)                     # grouped launches, one graph replay
            b.set_tiling(32, 4, 1, 0, 3)
            b.run(36)
            assert b.step == 200
        for q, e in enumerate(engs):
            assert e.step == 200
            _assert_same(solo[q], _state(e), f"member {q}")
    finally:
        for e in engs:
            e.close()


def test_member_mode_watchdog_and_profile():
    probs = _members(140)[:3]
    probs[2].voltage_sources[0].voltage_per_e_field[100] = np.nan
    engs = [Engine(p, "f32-table") for p in probs]
    try:
        with Batch(engs, 8, 4, 1, 0, 2) as b:
            prof = b.profile_kernels(4)
            assert all(v > 0 for v in prof.values())
            with pytest.raises(N.FdtdError) as ei:
                b.run(128)
            assert ei.value.code == N.FDTD_ERR_NONFINITE
            assert "member 2" in str(ei.value)
            with pytest.raises(N.FdtdError):
                b.set_tiling(8, 4, 1, 0, 33)
        assert engs[2].status() == (N.FDTD_ERR_NONFINITE, 100)
        assert engs[0].status() == (0, -1)
    finally:
        for e in engs:
            e.close()


def test_early_stop_checkpoint_loop_keeps_each_runs_own_traces():
    """The checkpoint loop steps the batch to the next checkpoint while it
    fits the current one, and rebuilds the batch when runs stop: every run's
    traces up to its stop step are still those of the same run stepped alone."""
    from special_topics_b200 import earlystop as ES
    steps = 160
    probs = _members(steps)[:3]
    solo = []
    for p in probs:
        with Engine(p, "f32-table") as e:
            e.run(steps)
            solo.append((e.voltages()[0], e.currents()[0]))
    for policy in (ES.StopPolicy(n_in=40, checkpoints=(70, 100, 130), n_total=steps, pencil_orders=(4, 6, 8),
                                 decim=1, max_resid=1.0, agree_db=1e9),      # stops at the first fit
                   ES.StopPolicy(n_in=40, checkpoints=(70, 100, 130), n_total=steps, pencil_orders=(4, 6, 8),
                                 decim=1, agree_db=-1.0)):                    # stops at the last checkpoint
        engs = [Engine(p, "f32-table") for p in probs]
        try:
            res = ES.run_with_early_stop(engs, None, policy, {"chunk": 8, "rows": 4}, use_network=False)
        finally:
            for e in engs:
                e.close()
        for q, r in enumerate(res):
            # the strict rule never sees agreement: nothing stops before the last checkpoint
            assert r["stopped_at"] in ((70, 100, 130, steps) if policy.agree_db > 0 else (130, steps))
            assert r["V"].shape == (steps,) and r["I"].shape == (steps,)
            n = r["stopped_at"]
            assert np.array_equal(r["V"][:n], solo[q][0][:n])
            assert np.array_equal(r["I"][:n], solo[q][1][:n])


@pytest.mark.parametrize("chunk,rows,pf,group,streams", [(8, 4, 1, 0, 0), (5, 16, 2, 3, 0), (16, 2, 1, 0, 2)])
def test_batch_with_16_wide_blocks_matches_solo_runs(solo, chunk, rows, pf, group, streams):
    """16-wide blocks (a warp spans two rows) in the tile-list, persistent and
    member-kernel modes."""
    precision, states = solo
    engs = [Engine(p, precision) for p in _members()]
    try:
        with Batch(engs, chunk, rows, pf, group, streams) as b:
            b.set_tiling(chunk, rows, pf, group, streams, 16)
            assert b.tiling()["width"] == 16
            b.run(STEPS)
        for q, e in enumerate(engs):
            _assert_same(states[q], _state(e), f"member {q}")
    finally:
        for e in engs:
            e.close()
