"""The engine's problem construction (numpy, special-topics_b200/scenario.py)
against the oracle's scalar restatement of the reference setup: every array
the time loop consumes must be bit-identical."""
import numpy as np
import pytest

import oracle
from conftest import load_package, load_scenario
from scenarios_small import small_scenario

pkg = load_package()
from special_topics_b200 import scenario as S  # noqa: E402

CASES = [("ifa-fr4-substrate", None)] + [(f"small-{d}", d) for d in ("xp", "yn", "zp", "xn")]


def _scn(case):
    name, d = case
    if d is None:
        return load_scenario(name), 50
    return small_scenario(seed=len(d) + ord(d[0]), direction=d), 40


@pytest.fixture(scope="module", params=CASES, ids=[c[0] for c in CASES])
def pair(request):
    scn, steps = _scn(request.param)
    return S.build_problem_from_scenario(scn, steps), oracle.Oracle(scn, steps)


def test_grid(pair):
    p, o = pair
    g = p.grid
    assert (g.nx, g.ny, g.nz) == (o.nx, o.ny, o.nz)
    assert g.dt == o.dt and g.min_x == o.min_x and g.max_z == o.max_z


def test_material_components(pair):
    p, o = pair
    for name in ("eps_r_x", "eps_r_y", "eps_r_z", "sigma_e_x", "sigma_e_y", "sigma_e_z",
                 "mu_r_x", "mu_r_y", "mu_r_z", "sigma_m_x", "sigma_m_y", "sigma_m_z"):
        assert np.array_equal(p.materials[name].ravel(), o.get(name)), name


def test_coefficients_bit_identical(pair):
    p, o = pair
    for name in S.COEFF_ORDER:
        assert np.array_equal(p.coeffs[name], o.get(name)), name


def test_cpml_profiles_and_cpsi(pair):
    p, o = pair
    for fid, f in enumerate(p.cpml):
        assert f is not None
        for q, arr in enumerate((f.b_e, f.a_e, f.b_m, f.a_m, f.kappa_e, f.kappa_m)):
            assert np.array_equal(arr, o.get(f"prof:{fid}:{q}")), (fid, q)
        for s in range(4):
            assert np.array_equal(f.cpsi[s], o.get(f"cpsi:{fid}:{s}")), (fid, s)


def test_sources_and_probes(pair):
    p, o = pair
    for n, vs in enumerate(p.voltage_sources):
        assert np.array_equal(vs.field_indices, o.get(f"vfi:{n}").astype(np.int32))
        assert np.array_equal(vs.coef, o.get(f"vcs:{n}"))
        assert np.array_equal(vs.voltage_per_e_field, o.get(f"vpe:{n}"))
    for n, sv in enumerate(p.sampled_voltages):
        assert np.array_equal(sv.field_indices, o.get(f"svfi:{n}").astype(np.int32))
        assert sv.Csvf == o.get(f"svcsvf:{n}")[0]


def test_current_probe_list_reproduces_oracle_sum(pair):
    """The ordered (component, index, weight) list summed like the kernel does
    gives the oracle's captured current bit for bit."""
    p, o = pair
    o.step(12)
    H = [o.get("Hx"), o.get("Hy"), o.get("Hz")]
    for n, si in enumerate(p.sampled_currents):
        sv = 0.0
        for c, i, w in zip(si.comp, si.idx, si.w):
            sv = sv + w * H[c][i]
        assert sv == o.get(f"I:{n}")[11]
