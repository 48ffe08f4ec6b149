"""GPU parity: the sm_100a engine against the FP64 CPU oracle, through the C ABI.

FP64 (the drop-in path): bit-identical fields, CPML Psi, port traces and far-
field accumulators.  FP32 paths: port voltage within 1e-3 of its peak (the
reference's own GPU-vs-CPU bar, js_fdtd/test/validate_cuda.js:115-135) and
far-field accumulators within 1e-3 relative to their largest magnitude.
"""
import ctypes

import numpy as np
import pytest

import oracle
from conftest import load_package, load_scenario
from scenarios_small import small_scenario

pkg = load_package()
from special_topics_b200 import _native as N  # noqa: E402
from special_topics_b200 import postproc  # noqa: E402
from special_topics_b200.backend import B200Backend, Engine  # noqa: E402
from special_topics_b200.scenario import FF_NAMES, build_problem_from_scenario  # noqa: E402

pytestmark = pytest.mark.gpu

CASES = {
    "ifa-fr4-substrate": lambda: (load_scenario("ifa-fr4-substrate"), 200),
    "small-xp": lambda: (small_scenario(1, "xp"), 60),
    "small-yn": lambda: (small_scenario(2, "yn", ncpml=(3, 3, 5, 4, 6, 3)), 60),
    "small-zp": lambda: (small_scenario(3, "zp", ncpml=(5, 4, 3, 3, 4, 5)), 60),
}


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request):
    scn, steps = CASES[request.param]()
    o = oracle.Oracle(scn, steps)
    o.step(steps)
    return request.param, scn, steps, o


def _psi_sizes(p, fid):
    f = p.cpml[fid]
    return [c.size for c in f.cpsi]


def test_fp64_bit_identical(case):
    name, scn, steps, o = case
    p = build_problem_from_scenario(scn, steps)
    with Engine(p, "f64") as eng:
        eng.run(steps)
        assert eng.step == steps
        for q in range(o.n_sv):
            assert np.array_equal(eng.voltages()[q], o.get(f"V:{q}")), f"V{q}"
        for q in range(o.n_si):
            assert np.array_equal(eng.currents()[q], o.get(f"I:{q}")), f"I{q}"
        for fld in ("Hx", "Hy", "Hz", "Ex", "Ey", "Ez"):
            assert np.array_equal(eng.field(fld), o.get(fld)), fld
        for fid in range(6):
            for s, n in enumerate(_psi_sizes(p, fid)):
                assert np.array_equal(eng.psi(fid, s, n), o.get(f"psi:{fid}:{s}")), (fid, s)
        ff = eng.farfield()
        for a in FF_NAMES:
            assert np.array_equal(ff[a][0], o.get(f"ff:{a}:0")), a
            assert np.array_equal(ff[a][1], o.get(f"ff:{a}:1")), a
        assert eng.status() == (0, -1)


@pytest.mark.parametrize("precision", ["f32", "f32-table"])
def test_fp32_paths_within_tolerance(case, precision):
    """FP32 arithmetic on the reference's loop: the x = max wall is set to the
    reference's reads, as the oracle has it (the FP32 default wall differs
    from the oracle by design, which the small boxes' Huygens surfaces inside
    the CPML see within these steps)."""
    name, scn, steps, o = case
    p = build_problem_from_scenario(scn, steps)
    with Engine(p, precision, x_wall=False) as eng:
        eng.run(steps)
        v, vo = eng.voltages()[0], o.get("V:0")
        peak = np.abs(vo).max()
        assert np.abs(v - vo).max() <= 1e-3 * peak, np.abs(v - vo).max() / peak
        i, io = eng.currents()[0], o.get("I:0")
        assert np.abs(i - io).max() <= 1e-3 * np.abs(io).max()
        ff = eng.farfield()
        for a in FF_NAMES:
            ref = o.get(f"ff:{a}:0") + 1j * o.get(f"ff:{a}:1")
            got = ff[a][0] + 1j * ff[a][1]
            scale = max(np.abs(ref).max(), 1e-300)
            assert np.abs(got - ref).max() <= 2e-3 * scale, (a, np.abs(got - ref).max() / scale)


def test_device_dft_matches_oracle_transform():
    rng = np.random.default_rng(5)
    x = rng.standard_normal(3000)
    f = np.linspace(1e8, 1e10, 301)
    dt = 5.77e-13
    for shift in (0.0, -dt / 2):
        re, im = postproc.time_to_freq(x, dt, f, shift)
        ore, oim = oracle.time_to_freq(x, dt, f, shift)
        scale = np.abs(ore + 1j * oim).max()
        assert np.abs((re - ore) + 1j * (im - oim)).max() <= 1e-12 * scale


def test_golden_s11_and_cuts_through_engine(golden_out):
    """The whole CLI pipeline (index.js:63-134) with the engine's traces: S11 and
    the directivity cuts agree with the reference's out.json."""
    scn = load_scenario("ifa-fr4-substrate")
    p = build_problem_from_scenario(scn, 200)
    with Engine(p, "f64") as eng:
        eng.run(200)
        V, I = eng.voltages()[0], eng.currents()[0]
        acc = eng.farfield()
    vg = np.array(golden_out["voltages"][0]["values"])
    assert np.abs(V - vg).max() <= 1e-8 * np.abs(vg).max()
    freqs = postproc.dft_frequencies(p.dft)
    s = postproc.port_s11(V, I, p.grid.dt, freqs, 50.0)
    sg = golden_out["sparams"][0]
    assert np.abs(s["mag_dB"] - np.array(sg["magnitude_dB"])).max() < 1e-6
    cuts = postproc.farfield_cuts(acc, p.grid, p.farfield)
    for c, g in zip(cuts, golden_out["farfield"]):
        assert c["plane"] == g["plane"]
        assert np.abs(c["dataTheta_dB"] - np.array(g["dataTheta_dB"])).max() < 1e-3
        assert np.abs(c["dataPhi_dB"] - np.array(g["dataPhi_dB"])).max() < 1e-3


def test_backend_contract_snapshots():
    scn = small_scenario(4, "xp")
    p = build_problem_from_scenario(scn, 55)
    b = B200Backend("f64")
    assert b.is_available()
    snaps = list(b.run(p, batch_size=20))
    assert [s["step"] for s in snaps] == [20, 40, 55]
    assert all(s["total"] == 55 and s["backend"] == "b200" for s in snaps)
    assert snaps[-1]["voltage"] == b.engine.voltages()[0][54]
    b.engine.close()


def test_watchdog_reports_nonfinite_port_sample():
    scn = small_scenario(6, "xp")
    p = build_problem_from_scenario(scn, 30)
    p.voltage_sources[0].voltage_per_e_field[7] = np.nan
    with Engine(p, "f64") as eng:
        with pytest.raises(N.FdtdError) as ei:
            eng.run(30)
        assert ei.value.code == N.FDTD_ERR_NONFINITE
        assert eng.status() == (N.FDTD_ERR_NONFINITE, 7)


def test_legacy_global_api_fp32():
    """The reference's fdtd_cuda.h call sequence (cudaBackend.js:183-289) on the legacy entry points."""
    scn = small_scenario(7, "xp")
    steps = 50
    p = build_problem_from_scenario(scn, steps)
    o = oracle.Oracle(scn, steps)
    o.step(steps)
    L, g = N.lib(), p.grid
    dims = N.FdtdDims(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, g.dt, steps)
    N.check(L.fdtd_init(ctypes.byref(dims)))
    try:
        from special_topics_b200.scenario import COEFF_ORDER
        for w, nm in enumerate(COEFF_ORDER):
            a = p.coeffs[nm].astype(np.float32)
            N.check(L.fdtd_upload_coeff(w, N.fptr(a), a.size))
        for fid, f in enumerate(p.cpml):
            pr = [x.astype(np.float32) for x in (f.b_e, f.a_e, f.b_m, f.a_m)]
            cp = [c.astype(np.float32) for c in f.cpsi]
            N.check(L.fdtd_upload_cpml(fid, f.nc, *[N.fptr(x) for x in pr], N.fptr(cp[0]), cp[0].size,
                                       N.fptr(cp[1]), cp[1].size, N.fptr(cp[2]), cp[2].size, N.fptr(cp[3]),
                                       cp[3].size, f.m_start, f.e_start, fid % 2))
        vs = p.voltage_sources[0]
        cs, wv = vs.coef.astype(np.float32), vs.voltage_per_e_field.astype(np.float32)
        N.check(L.fdtd_upload_vsource(vs.axis, N.iptr(vs.field_indices), N.fptr(cs), cs.size, N.fptr(wv), wv.size))
        sv = p.sampled_voltages[0]
        N.check(L.fdtd_upload_svoltage(sv.axis, N.iptr(sv.field_indices), sv.field_indices.size, sv.Csvf))
        si = p.sampled_currents[0]
        lists = []
        for c in range(3):
            m = si.comp == c
            lists += [np.ascontiguousarray(si.idx[m]), np.ascontiguousarray(si.w[m].astype(np.float32))]
        N.check(L.fdtd_upload_scurrent(N.iptr(lists[0]), N.fptr(lists[1]), lists[0].size,
                                       N.iptr(lists[2]), N.fptr(lists[3]), lists[2].size,
                                       N.iptr(lists[4]), N.fptr(lists[5]), lists[4].size))
        vout = np.zeros(steps, np.float32)
        iout = np.zeros(steps, np.float32)
        for ts in range(0, steps, 25):
            N.check(L.fdtd_run_batch(ts, 25, N.fptr(vout[ts:]), N.fptr(iout[ts:])))
        vo = o.get("V:0")
        assert np.abs(vout - vo).max() <= 1e-3 * np.abs(vo).max()
        io = o.get("I:0")
        assert np.abs(iout - io).max() <= 1e-3 * np.abs(io).max()
        ez = np.zeros(p.grid.shapes["Ez"], np.float32).ravel()
        N.check(L.fdtd_read_field(5, N.fptr(ez), ez.size))
        assert np.abs(ez - o.get("Ez")).max() <= 1e-3 * np.abs(o.get("Ez")).max()
    finally:
        L.fdtd_destroy()


@pytest.mark.parametrize("name", ["small-xp", "small-zp", "ifa-fr4-substrate"])
def test_device_material_tables_match_host_tables(name):
    """fdtd_ctx_build_material (GPU) gives every cell the same FP64 coefficient
    triple as the numpy construction from the reference's per-cell arrays."""
    scn, steps = CASES[name]()
    p = build_problem_from_scenario(scn, steps)
    q = build_problem_from_scenario(scn, steps, per_cell=False)
    from special_topics_b200.tables import COMPONENTS, build_tables
    host = build_tables(p)
    with Engine(q, "f32-table") as eng:
        for comp in COMPONENTS:
            ids, tab = eng.material(comp)
            hids, htab = host[comp]
            assert np.array_equal(tab[ids], htab[hids]), comp


def test_device_tables_run_matches_host_tables_run():
    scn, steps = CASES["small-yn"]()
    p = build_problem_from_scenario(scn, steps)
    q = build_problem_from_scenario(scn, steps, per_cell=False)
    with Engine(p, "f32-table", host_tables=True) as a, Engine(q, "f32-table") as b:
        a.run(steps)
        b.run(steps)
        assert np.array_equal(a.voltages()[0], b.voltages()[0])
        assert np.array_equal(a.field("Ez"), b.field("Ez"))


@pytest.mark.parametrize("chunk,rows,pf,width", [(1, 1, 1, 32), (3, 2, 2, 32), (7, 8, 1, 32), (64, 4, 2, 32),
                                                 (2, 4, 2, 32),
                                                 # 16-wide blocks: a warp spans two rows
                                                 (4, 2, 1, 16), (5, 16, 2, 16), (1, 8, 1, 16)])
def test_launch_shape_does_not_change_fp64_results(chunk, rows, pf, width):
    from special_topics_b200 import autotune
    scn, steps = CASES["small-zp"]()
    o = oracle.Oracle(scn, steps)
    o.step(steps)
    p = build_problem_from_scenario(scn, steps)
    with Engine(p, "f64") as eng:
        autotune.set_tiling(eng, min(chunk, p.grid.nx + 1), rows, pf, width)
        eng.run(steps)
        assert np.array_equal(eng.voltages()[0], o.get("V:0"))
        for fld in ("Hx", "Ey", "Ez"):
            assert np.array_equal(eng.field(fld), o.get(fld)), fld


def test_autotuner_picks_a_measured_shape(tmp_path, monkeypatch):
    from special_topics_b200 import autotune
    monkeypatch.setattr(autotune, "CACHE", str(tmp_path / "tiling.json"))
    scn, _ = CASES["small-xp"]()
    p = build_problem_from_scenario(scn, 1500)
    res = autotune.tune(p, "f32-table", steps_per_candidate=8)
    assert {"chunk", "rows", "ms_per_step"} <= set(res)
    assert res["ms_per_step"] == min(r["ms_per_step"] for r in res["table"])


@pytest.mark.parametrize("name", ["ifa-fr4-substrate", "small-yn"])
def test_device_farfield_post_matches_host(name):
    """Radiated power and directivity on the device against postproc's FP64
    host restatement of farfield.js:257-607, on the same accumulators."""
    scn, steps = CASES[name]()
    p = build_problem_from_scenario(scn, steps)
    with Engine(p, "f64") as eng:
        eng.run(steps)
        acc = eng.farfield()
        radp_h = postproc.radiated_power(acc, p.grid, p.farfield)
        th = np.radians(np.arange(0, 181, 7.0))
        ph = np.radians(np.arange(0, 360, 11.0))
        T, P = [a.ravel() for a in np.meshgrid(th, ph, indexing="ij")]
        dth_h, dph_h = postproc.directivity(acc, p.grid, p.farfield, radp_h, T, P)
        radp, dth, dph = eng.farfield_post(T, P)
        assert np.allclose(radp, radp_h, rtol=1e-10, atol=0)
        for d, h in ((dth, dth_h), (dph, dph_h)):
            assert np.abs(d - h).max() <= 1e-9 * np.abs(h).max()


def test_kahan_fp32_accumulators_track_fp64_ones():
    scn, steps = CASES["small-xp"]()
    p = build_problem_from_scenario(scn, steps, per_cell=False)
    with Engine(p, "f32-table") as a, Engine(p, "f32-table", dft_accumulator="kahan-f32") as b:
        a.run(steps)
        b.run(steps)
        fa, fb = a.farfield(), b.farfield()
        for name in FF_NAMES:
            for q in range(2):
                scale = np.abs(fa[name][q]).max() + 1e-30
                assert np.abs(fa[name][q] - fb[name][q]).max() <= 1e-5 * scale, name
        ra, _, _ = a.farfield_post(np.zeros(1), np.zeros(1))
        rb, _, _ = b.farfield_post(np.zeros(1), np.zeros(1))
        assert np.allclose(ra, rb, rtol=1e-4)
    with Engine(build_problem_from_scenario(scn, steps), "f64") as c:
        with pytest.raises(N.FdtdError):
            N.check(N.lib().fdtd_ctx_set_dft_accumulator(c._h, 1))


@pytest.mark.parametrize("chunk,rows,pf,width", [(5, 2, 3, 32), (16, 8, 4, 32), (1, 4, 4, 32), (64, 2, 3, 32),
                                                 (3, 8, 2, 32), (8, 4, 1, 16), (6, 16, 3, 16), (16, 2, 4, 16)])
def test_shared_memory_stages_give_identical_table_results(chunk, rows, pf, width):
    """Prefetch depths 3 and 4 stage the interior planes through shared
    memory; material-table results are bit-identical to the depth-1 form,
    also with 16-wide blocks."""
    from special_topics_b200 import autotune
    scn, steps = CASES["ifa-fr4-substrate"]()
    p = build_problem_from_scenario(scn, steps, per_cell=False)
    with Engine(p, "f32-table") as a, Engine(p, "f32-table") as b:
        autotune.set_tiling(a, 8, 4, 1)
        autotune.set_tiling(b, min(chunk, p.grid.nx + 1), rows, pf, width)
        a.run(steps)
        b.run(steps)
        assert np.array_equal(a.voltages()[0], b.voltages()[0])
        for fld in ("Hx", "Hy", "Hz", "Ex", "Ey", "Ez"):
            assert np.array_equal(a.field(fld), b.field(fld)), fld
    with Engine(build_problem_from_scenario(scn, steps), "f64") as c:
        with pytest.raises(N.FdtdError):
            autotune.set_tiling(c, 8, 4, 3)


@pytest.mark.parametrize("case_name,steps", [("ifa-fr4-substrate", 120), ("small-yn", 60), ("box-64", 80)])
@pytest.mark.parametrize("chunk,rows", [(8, 4), (1, 2), (5, 8), (64, 1), (16, 4)])
def test_bulk_staged_form_gives_identical_table_results(case_name, steps, chunk, rows):
    """Prefetch mode 5 stages each warp's interior rows through shared memory
    with bulk copies on an mbarrier ring; the results are bit-identical to
    the depth-1 register form, for every chunk and block height, including
    warps cut short at the k end and chunks shorter than the ring."""
    from special_topics_b200 import autotune, workloads
    if case_name == "box-64":
        scn = workloads.scaling_box((64, 64, 64), seed=3, steps=steps)
    elif case_name == "small-yn":
        scn = small_scenario(2, "yn", ncpml=(3, 3, 5, 4, 6, 3), steps=steps)
    else:
        scn = load_scenario(case_name)
    p = build_problem_from_scenario(scn, steps, per_cell=False)
    with Engine(p, "f32-table") as a, Engine(p, "f32-table") as b:
        autotune.set_tiling(a, 8, 4, 1)
        autotune.set_tiling(b, min(chunk, p.grid.nx + 1), rows, 5)
        a.run(steps)
        b.run(steps)
        assert b.status() == (0, -1)
        assert np.array_equal(a.voltages()[0], b.voltages()[0])
        for fld in ("Hx", "Hy", "Hz", "Ex", "Ey", "Ez"):
            assert np.array_equal(a.field(fld), b.field(fld)), fld
        fa, fb = a.farfield(), b.farfield()
        for k in FF_NAMES:
            assert np.array_equal(fa[k][0], fb[k][0]), k
    with Engine(p, "f32-table") as c:
        autotune.set_tiling(c, 8, 4, 5, 16)
        with pytest.raises(N.FdtdError):
            c.run(2)


@pytest.mark.parametrize("precision", ["f64", "f32-table"])
def test_state_checkpoint_resumes_bit_identically(precision):
    scn, steps = CASES["small-zp"]()
    p = build_problem_from_scenario(scn, steps, per_cell=(precision == "f64"))
    with Engine(p, precision) as a, Engine(p, precision) as b:
        a.run(25)
        state = a.save_state()
        a.run(steps - 25)
        b.load_state(state)
        assert b.step == 25
        b.run(steps - 25)
        assert np.array_equal(a.voltages()[0], b.voltages()[0])
        assert np.array_equal(a.currents()[0], b.currents()[0])
        for fld in ("Hx", "Ez"):
            assert np.array_equal(a.field(fld), b.field(fld))
        fa, fb = a.farfield(), b.farfield()
        assert all(np.array_equal(fa[k][0], fb[k][0]) for k in FF_NAMES)
    other = build_problem_from_scenario(small_scenario(1, "xp"), steps, per_cell=(precision == "f64"))
    with Engine(other, precision) as c:
        with pytest.raises(N.FdtdError):
            c.load_state(state)
    # same shape and probe set, other physics: a different dt, then another
    # permittivity in one material
    import copy
    for change in ("dt", "eps"):
        scn2 = copy.deepcopy(scn)
        if change == "dt":
            scn2["courantFactor"] = 0.8
        else:
            scn2["materialTypes"][3]["eps_r"] += 0.5       # the block that fills the box
        p2 = build_problem_from_scenario(scn2, steps, per_cell=(precision == "f64"))
        assert (p2.grid.nx, p2.grid.ny, p2.grid.nz) == (p.grid.nx, p.grid.ny, p.grid.nz)
        with Engine(p2, precision) as c:
            with pytest.raises(N.FdtdError) as ei:
                c.load_state(state)
            assert ei.value.code == N.FDTD_ERR_BADARG
            assert "other data" in str(ei.value), change


@pytest.mark.parametrize("acc", ["f64", "kahan-f32"])
def test_time_blocked_dft_matches_per_step(acc):
    """Surface samples buffered for 16 steps and accumulated at once give the
    per-step accumulators to FP32 rounding, across graph replays, partial
    blocks at run ends and a checkpoint/restore in the middle of a block."""
    scn = small_scenario(2, "yn", ncpml=(3, 3, 5, 4, 6, 3), steps=200, nff=3)
    p = build_problem_from_scenario(scn, 200, per_cell=False)
    with Engine(p, "f32-table", dft_accumulator=acc) as a, \
            Engine(p, "f32-table", dft_accumulator=acc, dft_block=16) as b:
        for n in (23, 64, 41, 5):
            a.run(n)
            b.run(n)
        state = b.save_state()
        fa, fb = a.farfield(), b.farfield()
        for name in FF_NAMES:
            for q in range(2):
                scale = np.abs(fa[name][q]).max() + 1e-30
                assert np.abs(fa[name][q] - fb[name][q]).max() <= 1e-5 * scale, name
        assert np.array_equal(a.voltages()[0], b.voltages()[0])
        a.run(67)
        with Engine(p, "f32-table", dft_accumulator=acc, dft_block=16) as c:
            c.load_state(state)
            c.run(67)
            fa, fc = a.farfield(), c.farfield()
            for name in FF_NAMES:
                scale = np.abs(fa[name][0]).max() + 1e-30
                assert np.abs(fa[name][0] - fc[name][0]).max() <= 1e-5 * scale, name
    with Engine(build_problem_from_scenario(scn, 200), "f64") as d:
        with pytest.raises(N.FdtdError):
            N.check(N.lib().fdtd_ctx_set_dft_block(d._h, 16))


def test_block_width_validation():
    from special_topics_b200 import autotune
    scn, steps = CASES["small-xp"]()
    p = build_problem_from_scenario(scn, steps, per_cell=False)
    with Engine(p, "f32-table") as e:
        with pytest.raises(N.FdtdError):
            N.check(N.lib().fdtd_ctx_set_block_width(e._h, 8))
        autotune.set_tiling(e, 4, 1, 1, 16)       # 16 threads: not a whole warp, refused at the run
        with pytest.raises(N.FdtdError) as ei:
            e.run(2)
        assert ei.value.code == N.FDTD_ERR_BADARG
        autotune.set_tiling(e, 4, 16, 1, 32)      # 512 threads: above the launch bounds
        with pytest.raises(N.FdtdError):
            e.run(2)
        autotune.set_tiling(e, 4, 16, 1, 16)
        e.run(2)
        w = ctypes.c_int()
        N.check(N.lib().fdtd_ctx_get_block_width(e._h, ctypes.byref(w)))
        assert w.value == 16


def test_whole_run_graphs_match_any_split_of_the_run():
    """A run replays CUDA graphs of its whole length (graphs of at most the
    handle's cap of steps plus one of the remainder, cached by step count);
    one run of 8100 steps (past the 8000-step cap of a 5-launch step) gives
    the same as the same steps in uneven pieces."""
    scn = small_scenario(7, "zp", steps=8100)
    p = build_problem_from_scenario(scn, 8100, per_cell=False)
    with Engine(p, "f32-table", dft_block=16) as a, Engine(p, "f32-table", dft_block=16) as b:
        a.run(8100)
        for n in (5, 64, 1, 1000, 3030, 5, 3995):
            b.run(n)
        assert a.step == b.step == 8100
        assert np.array_equal(a.voltages()[0], b.voltages()[0])
        assert np.array_equal(a.currents()[0], b.currents()[0])
        assert np.array_equal(a.field("Ez"), b.field("Ez"))
        fa, fb = a.farfield(), b.farfield()
        for k in FF_NAMES:
            assert np.abs(fa[k][0] - fb[k][0]).max() <= 1e-5 * (np.abs(fa[k][0]).max() + 1e-30), k
