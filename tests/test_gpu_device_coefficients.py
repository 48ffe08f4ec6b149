"""FP64 problems whose 18 per-cell coefficient arrays, CPML kappa division,
CPsi and source cells are built on the device (fdtd_ctx_build_material,
fdtd_ctx_upload_cpml without CPsi, fdtd_ctx_override_material) step exactly
like the same problems built by the numpy restatement and uploaded from the
host: every field, Psi slot, port trace and far-field accumulator is
bit-identical."""
import ctypes as C

import numpy as np
import pytest

from conftest import load_package, load_scenario
from scenarios_small import small_scenario

pkg = load_package()
from special_topics_b200 import _native as N  # noqa: E402
from special_topics_b200.backend import Engine  # noqa: E402
from special_topics_b200.scenario import FF_NAMES, build_problem_from_scenario  # noqa: E402
from special_topics_b200.workloads import ifa_variant  # noqa: E402

pytestmark = pytest.mark.gpu

STEPS = 70


def _state(eng):
    out = {"V": eng.voltages(), "I": eng.currents()}
    for f in ("Hx", "Hy", "Hz", "Ex", "Ey", "Ez"):
        out[f] = eng.field(f)
    ff = eng.farfield()
    for a in FF_NAMES:
        out[a] = ff[a]
    return out


def _same(a, b, tag):
    for key in a:
        x, y = a[key], b[key]
        if isinstance(x, (list, tuple)):
            for q, (u, v) in enumerate(zip(x, y)):
                assert np.array_equal(u, v), f"{tag}: {key}[{q}] differs"
        else:
            assert np.array_equal(x, y), f"{tag}: {key} differs"


@pytest.mark.parametrize("name,scn", [
    ("small xp", small_scenario(1, "xp")),
    ("small yn, uneven CPML", small_scenario(2, "yn", ncpml=(3, 3, 5, 4, 6, 3))),
    ("small zp, uneven CPML", small_scenario(3, "zp", ncpml=(5, 4, 3, 3, 4, 5))),
    ("ifa-fr4-substrate", load_scenario("ifa-fr4-substrate")),
    ("inverted-F variant 7", ifa_variant(7, steps=STEPS)),
])
def test_device_built_fp64_matches_host_built(name, scn):
    host = build_problem_from_scenario(scn, STEPS, per_cell=True)
    dev = build_problem_from_scenario(scn, STEPS, per_cell=False)
    assert host.coeffs and not dev.coeffs
    with Engine(host, "f64") as a, Engine(dev, "f64") as b:
        a.run(STEPS)
        b.run(STEPS)
        _same(_state(a), _state(b), name)
        # the Psi arrays themselves (CPsi and kappa division enter only through them and the fields)
        for fid, face in enumerate(host.cpml):
            if face is None:
                continue
            for s in range(4):
                n = face.cpsi[s].size
                assert np.array_equal(a.psi(fid, s, n), b.psi(fid, s, n)), f"{name}: psi {fid}.{s}"


def test_device_build_argument_errors():
    scn = small_scenario(4, "xp")
    p = build_problem_from_scenario(scn, 30, per_cell=False)
    L, g = N.lib(), p.grid
    # per-cell FP32 problems take host arrays, not a device build
    cfg = N.FdtdConfig(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, g.dt, g.numberOfTimeSteps, N.PREC_F32, 0)
    h = C.c_void_p()
    N.check(L.fdtd_create(C.byref(cfg), C.byref(h)))
    try:
        mat = np.ascontiguousarray(p.meta["material_grid"], dtype=np.uint8).ravel()
        props = np.ascontiguousarray(p.meta["material_props"], dtype=np.float64)
        rc = L.fdtd_ctx_build_material(h, mat.ctypes.data_as(C.POINTER(C.c_ubyte)), mat.size, props.shape[0],
                                       N.dptr(props.reshape(-1)), 0, None, None)
        assert rc == N.FDTD_ERR_STATE
    finally:
        L.fdtd_free(h)
    # a face's band is divided by kappa once: uploading the face again is refused
    with Engine(p, "f64") as e:
        f = next(q for q, face in enumerate(p.cpml) if face is not None)
        face = p.cpml[f]
        prof = [np.ascontiguousarray(x, dtype=np.float64)
                for x in (face.b_e, face.a_e, face.b_m, face.a_m, face.kappa_e, face.kappa_m)]
        with pytest.raises(N.FdtdError) as ei:
            N.check(N.lib().fdtd_ctx_upload_cpml(e._h, f, face.nc, *[N.dptr(x) for x in prof],
                                                 None, 0, None, 0, None, 0, None, 0, face.m_start, face.e_start))
        assert ei.value.code == N.FDTD_ERR_STATE
