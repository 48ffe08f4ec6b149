"""Parity at the step counts the workloads are run for, beyond the inverted-F
antennas of test_gpu_config0.py.

  scaling box, 2000 steps  the 128^3 vacuum box with 32 dielectric blocks and
                           a half-wave dipole (workloads.scaling_box, the
                           FP64/FP32 sweep's generator, scenario.js:73-131),
                           FP64 on the engine against the oracle (the
                           reference's Float64 loop, fdtdSolver.js:84-140):
                           port traces, all six fields and all far-field
                           accumulators bit-identical after 2000 steps; the
                           FP32 table path within 1e-3 of the largest |V| of
                           the oracle's trace, its x = max wall off so that it
                           computes what the oracle computes.
  batch, 7000 steps        four inverted-F variants on spread grids
                           (workloads.ifa_variant(seed, spread=True)), FP32
                           tables, stepped together at the bench's launch
                           shape for the batch: every member's traces, fields
                           and far-field accumulators bit-identical to the
                           same member run alone.
"""
import numpy as np
import pytest

import oracle
from conftest import load_package

pkg = load_package()
from special_topics_b200 import workloads  # noqa: E402
from special_topics_b200.backend import Batch, Engine  # noqa: E402
from special_topics_b200.scenario import FF_NAMES, build_problem_from_scenario  # noqa: E402

pytestmark = pytest.mark.gpu

FIELDS = ("Hx", "Hy", "Hz", "Ex", "Ey", "Ez")


@pytest.fixture(scope="module")
def box():
    steps = 2000
    scn = workloads.scaling_box((128, 128, 128), seed=1, steps=steps)
    o = oracle.Oracle(scn, steps)
    o.step(steps)
    return scn, steps, o


def test_scaling_box_fp64_bit_identical_after_2000_steps(box):
    scn, steps, o = box
    p = build_problem_from_scenario(scn, steps)
    with Engine(p, "f64") as eng:
        eng.run(steps)
        assert eng.step == steps and eng.status() == (0, -1)
        assert np.array_equal(eng.voltages()[0], o.get("V:0")), "V"
        assert np.array_equal(eng.currents()[0], o.get("I:0")), "I"
        for fld in FIELDS:
            assert np.array_equal(eng.field(fld), o.get(fld)), fld
        ff = eng.farfield()
        for a in FF_NAMES:
            for q in range(len(ff[a])):
                assert np.array_equal(ff[a][q], o.get(f"ff:{a}:{q}")), f"{a}[{q}]"


def test_scaling_box_fp32_table_within_tolerance_after_2000_steps(box):
    scn, steps, o = box
    p = build_problem_from_scenario(scn, steps, per_cell=False)
    with Engine(p, "f32-table", x_wall=False) as eng:
        eng.run(steps)
        assert eng.status() == (0, -1)
        v_ref = o.get("V:0")
        assert np.abs(eng.voltages()[0] - v_ref).max() <= 1e-3 * np.abs(v_ref).max()


def _state(eng):
    out = {"V": eng.voltages()[0], "I": eng.currents()[0]}
    for f in FIELDS:
        out[f] = eng.field(f)
    ff = eng.farfield()
    for a in FF_NAMES:
        for q in range(len(ff[a])):
            out[f"{a}[{q}]"] = ff[a][q]
    return out


def test_spread_batch_matches_solo_runs_after_7000_steps():
    steps = 7000
    probs = [build_problem_from_scenario(workloads.ifa_variant(s, steps=steps, spread=True), steps, per_cell=False)
             for s in (1, 5, 7, 12)]
    solo = []
    for p in probs:
        with Engine(p, "f32-table", dft_block=16) as eng:
            eng.run(steps)
            solo.append(_state(eng))
    engs = [Engine(p, "f32-table", dft_block=16) for p in probs]
    try:
        with Batch(engs) as b:
            b.set_shape({"chunk": 64, "rows": 16, "prefetch": 1, "group": 0, "width": 16})
            b.run(steps)
        for q, e in enumerate(engs):
            assert e.step == steps and e.status() == (0, -1)
            got = _state(e)
            for key, want in solo[q].items():
                assert np.array_equal(got[key], want), f"member {q} {key}"
    finally:
        for e in engs:
            e.close()
