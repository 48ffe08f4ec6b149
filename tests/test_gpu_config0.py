"""Full-length FP64 parity on the inverted-F antennas, engine against the CPU oracle.

Two scenarios, each run for its whole 7000 steps on the engine (C ABI, FP64
drop-in) and on the oracle (the reference's Float64 loop,
js_fdtd/src/fdtdSolver.js:84-140):

  ifa-config0-0p5mm  the 0.5 mm inverted-F antenna: 39 x 136 x 136 cells, FR4
                     slab, 30 mm arm, stub 5 mm from the feed, 6 GHz Gaussian,
                     far field at 2.4 GHz
  ifa-matlab-7000    the reference's own scenario file, whose fields grow from
                     about step 4900 on (js_fdtd/scenarios/ifa-matlab-7000.json:3):
                     the run the late-time growth has to be reproduced on

Checked after the last step:
  - port voltage and current traces, all six fields and all 24 far-field
    accumulators: bit-identical;
  - S11 and Zin at 301 points in 1-4 GHz (postproc on the device DFT against
    the oracle's own transform and port-wave code, sparameters.js:23-101):
    complex S11 and Zin within 1e-10 relative, |S11| within 1e-9 dB;
  - radiated power and directivity at every far-field frequency on the xy
    and xz cuts (farfield.js:257-607): the device post-processing and the
    host restatement against the oracle's, within 1e-10 relative.
The FP32 material-table path on the 0.5 mm antenna (its default PEC wall at
i = nx, fdtd_ctx_set_x_wall) is held to |S11| within 0.1 dB, Zin within 1%
of its largest magnitude and directivity within 0.3 dB of the FP64 result.
"""
import numpy as np
import pytest

import oracle
from conftest import load_package, load_scenario

pkg = load_package()
from special_topics_b200 import postproc, workloads  # noqa: E402
from special_topics_b200.backend import Engine  # noqa: E402
from special_topics_b200.scenario import FF_NAMES, build_problem_from_scenario  # noqa: E402

pytestmark = pytest.mark.gpu

STEPS = 7000
S11_FREQS = np.linspace(1e9, 4e9, 301)
SCENARIOS = {
    "ifa-config0-0p5mm": lambda: workloads.ifa_config0(STEPS),
    "ifa-matlab-7000": lambda: load_scenario("ifa-matlab-7000"),
}


def _cut_directions():
    angles, th_xy, th_xz, ph_xz = oracle.xy_xz_angles()
    return np.concatenate([th_xy, th_xz]), np.concatenate([angles, ph_xz])


@pytest.fixture(scope="module", params=sorted(SCENARIOS))
def run(request):
    scn = SCENARIOS[request.param]()
    o = oracle.Oracle(scn, STEPS)
    o.step(STEPS)
    p = build_problem_from_scenario(scn, STEPS)
    th, ph = _cut_directions()
    with Engine(p, "f64") as eng:
        eng.run(STEPS)
        res = {"V": eng.voltages()[0], "I": eng.currents()[0], "ff": eng.farfield(),
               "fields": {f: eng.field(f) for f in ("Hx", "Hy", "Hz", "Ex", "Ey", "Ez")},
               "post": eng.farfield_post(th, ph), "status": eng.status(), "step": eng.step}
    return request.param, scn, p, o, res


def test_traces_fields_and_accumulators_bit_identical(run):
    name, scn, p, o, r = run
    assert r["step"] == STEPS and r["status"] == (0, -1)
    assert np.array_equal(r["V"], o.get("V:0")), "V"
    assert np.array_equal(r["I"], o.get("I:0")), "I"
    for fld, v in r["fields"].items():
        assert np.array_equal(v, o.get(fld)), fld
    for a in FF_NAMES:
        assert np.array_equal(r["ff"][a][0], o.get(f"ff:{a}:0")), a
        assert np.array_equal(r["ff"][a][1], o.get(f"ff:{a}:1")), a
    if name == "ifa-matlab-7000":
        # the late-time growth is part of what is reproduced
        v = np.abs(r["V"])
        assert v[-500:].max() > 10 * v[3000:3500].max()


def test_s11_and_zin_match_oracle_transform(run):
    name, scn, p, o, r = run
    dt = p.grid.dt
    port = postproc.port_s11(r["V"], r["I"], dt, S11_FREQS, 50.0)
    vf = oracle.time_to_freq(o.get("V:0"), o.dt, S11_FREQS, 0.0)
    jf = oracle.time_to_freq(o.get("I:0"), o.dt, S11_FREQS, -o.dt / 2)
    ref = oracle.s11(vf, jf, 50.0)
    s_got = port["re"] + 1j * port["im"]
    s_ref = ref["re"] + 1j * ref["im"]
    assert np.abs(s_got - s_ref).max() <= 1e-10 * np.abs(s_ref).max()
    assert np.abs(port["mag_dB"] - ref["mag_dB"]).max() <= 1e-9
    z_ref = (vf[0] + 1j * vf[1]) / (jf[0] + 1j * jf[1])
    assert np.abs(port["zin"] - z_ref).max() <= 1e-10 * np.abs(z_ref).max()


def test_radiated_power_and_directivity_match_oracle(run):
    name, scn, p, o, r = run
    th, ph = _cut_directions()
    radp_ref = o.radiated_power()
    dth_ref, dph_ref = o.directivity(radp_ref, th, ph)
    radp, dth, dph = r["post"]
    assert np.allclose(radp, radp_ref, rtol=1e-10, atol=0)
    # |D| sets the scale: once the late-time growth dominates the surface
    # currents the radiated power (and with it D) can come out negative
    scale = np.maximum(np.abs(dth_ref), np.abs(dph_ref)).max()
    assert np.abs(dth - dth_ref).max() <= 1e-10 * scale
    assert np.abs(dph - dph_ref).max() <= 1e-10 * scale
    radp_h = postproc.radiated_power(r["ff"], p.grid, p.farfield)
    dth_h, dph_h = postproc.directivity(r["ff"], p.grid, p.farfield, radp_h, th, ph)
    assert np.allclose(radp_h, radp_ref, rtol=1e-10, atol=0)
    assert np.abs(dth_h - dth_ref).max() <= 1e-10 * scale
    assert np.abs(dph_h - dph_ref).max() <= 1e-10 * scale


def test_fp32_table_within_targets_on_config0(run):
    name, scn, p64, o, r = run
    if name != "ifa-config0-0p5mm":
        pytest.skip("FP32 targets are stated on the 0.5 mm antenna")
    p32 = build_problem_from_scenario(scn, STEPS, per_cell=False)
    th, ph = _cut_directions()
    with Engine(p32, "f32-table") as eng:
        eng.run(STEPS)
        V, I = eng.voltages()[0], eng.currents()[0]
        radp, dth, dph = eng.farfield_post(th, ph)
    dt = p64.grid.dt
    s32 = postproc.port_s11(V, I, dt, S11_FREQS, 50.0)
    s64 = postproc.port_s11(r["V"], r["I"], dt, S11_FREQS, 50.0)
    assert np.abs(s32["mag_dB"] - s64["mag_dB"]).max() <= 0.1
    assert np.abs(s32["zin"] - s64["zin"]).max() <= 0.01 * np.abs(s64["zin"]).max()
    d64 = 10 * np.log10(r["post"][1] + r["post"][2])
    d32 = 10 * np.log10(dth + dph)
    assert np.abs(d32.max(axis=1) - d64.max(axis=1)).max() <= 0.3
    main = d64 >= d64.max(axis=1, keepdims=True) - 10.0
    assert np.abs(d32 - d64)[main].max() <= 0.3
