"""Pins the FP64 CPU oracle to the reference's only Float64 output.

``tests/golden/ref_out_ifa_fr4_200.json`` is js_fdtd/results/out.json: the
200-step ``ifa-fr4-substrate`` run (V trace, S11 at 500 frequencies, xy/xz
directivity cuts at 2.0/5.0 GHz).  The reference's Ey(i=nx) bulk update reads
Ex(i=0) through an out-of-range Hz index while another worker rewrites it
(fdtd_kernels.ts:159-178 with fdtdWorker.js:22-30), so its output is a
run-dependent mix of two deterministic orders.  The oracle runs both orders;
the golden file must sit inside that bracket, and before the boundary
disturbance reaches the port (first 100 steps) it must match to round-off.
"""
import numpy as np
import pytest

import oracle
from conftest import load_scenario


@pytest.fixture(scope="module")
def runs():
    scn = load_scenario("ifa-fr4-substrate")
    return (oracle.run_pipeline(scn, steps=200, edge_read_old=False),
            oracle.run_pipeline(scn, steps=200, edge_read_old=True))


def test_grid_and_dt(runs, golden_out):
    o = runs[0]["oracle"]
    assert (o.nx, o.ny, o.nz) == (39, 136, 136)
    assert o.dt == golden_out["meta"]["dt"]          # bit-exact
    assert o.nsteps == golden_out["meta"]["numberOfTimeSteps"] == 200


def test_voltage_trace_early_steps_round_off(runs, golden_out):
    vg = np.array(golden_out["voltages"][0]["values"])
    v = runs[0]["V"][0]
    peak = np.abs(vg).max()
    assert np.abs(v[:100] - vg[:100]).max() <= 1e-13 * peak
    assert np.sum(v == vg) >= 60   # most early samples are bit-identical


def test_voltage_trace_inside_race_bracket(runs, golden_out):
    vg = np.array(golden_out["voltages"][0]["values"])
    v0, v1 = runs[0]["V"][0], runs[1]["V"][0]
    peak = np.abs(vg).max()
    spread = np.maximum.accumulate(np.abs(v0 - v1))
    assert np.all(np.abs(vg - v0) <= 2 * spread + 1e-13 * peak)
    assert np.abs(vg - v0).max() <= 1e-8 * peak


def test_s11_inside_race_bracket(runs, golden_out):
    sg = golden_out["sparams"][0]
    a, b = runs[0]["sparams"][0], runs[1]["sparams"][0]
    g = np.array(sg["magnitude_dB"])
    assert np.abs(g - a["mag_dB"]).max() <= np.abs(a["mag_dB"] - b["mag_dB"]).max() + 1e-12
    assert np.abs(g - a["mag_dB"]).max() < 1e-7
    gp = np.array(sg["phase_deg"])
    assert np.abs(gp - a["phase_deg"]).max() <= np.abs(a["phase_deg"] - b["phase_deg"]).max() + 1e-12


def test_farfield_cuts_inside_race_bracket(runs, golden_out):
    for ra, rb, g in zip(runs[0]["farfield"], runs[1]["farfield"], golden_out["farfield"]):
        assert ra["plane"] == g["plane"]
        for key in ("dataTheta_dB", "dataPhi_dB"):
            A, B, G = ra[key], rb[key], np.array(g[key])
            # an unrelated error would land inside the bracket about half the time or less
            inside = (G - A) * (G - B) <= 0
            assert inside.mean() >= 0.75, (g["plane"], g["freq_GHz"], key)
            assert np.abs(G - A).max() <= np.abs(A - B).max() + 1e-9
            assert np.abs(G - A).max() < 1e-4
