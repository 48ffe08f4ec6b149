"""ctypes front end of the FP64 CPU oracle (test infrastructure only).

The C file ``fdtd_oracle.c`` restates the reference's Float64 CPU path; this
module turns a scenario (the reference's JSON schema, js_fdtd/src/scenario.js)
into the C description, drives the time loop and reproduces the CLI's
post-loop outputs (js_fdtd/src/index.js:63-134): the S11 sweep and the xy/xz
directivity cuts.  Only tests, the smoke check and the CPU-baseline leg of the
benchmark use it; the shipped engine never imports it.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from typing import Any

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

# scenario.js:32-40
DEFAULTS = {
    "courantFactor": 0.9,
    "numberOfCellsPerWavelength": 20,
    "numberOfTimeSteps": 4000,
    "cell": {"dx": 0.262e-3, "dy": 0.4e-3, "dz": 0.4e-3},
    "dft": {"maxFreq": 10e9, "step": 20e6},
    "farfield": {"frequencies": [], "number_of_cells_from_outer_boundary": 13},
}
FACES = ("xn", "xp", "yn", "yp", "zn", "zp")
WAVE_KINDS = ("gaussian", "derivative_gaussian", "sinusoidal", "unit_step", "cosine_modulated_gaussian")
FF_NAMES = ("cjyxp", "cjzxp", "cjyxn", "cjzxn", "cjxyp", "cjzyp", "cjxyn", "cjzyn",
            "cjxzp", "cjyzp", "cjxzn", "cjyzn", "cmyxp", "cmzxp", "cmyxn", "cmzxn",
            "cmxyp", "cmzyp", "cmxyn", "cmzyn", "cmxzp", "cmyzp", "cmxzn", "cmyzn")


class _Scn(C.Structure):
    _fields_ = [
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double), ("courant", C.c_double),
        ("nsteps", C.c_int),
        ("is_cpml", C.c_int * 6), ("air", C.c_int * 6), ("ncpml", C.c_int * 6),
        ("cpml_order", C.c_double), ("sigma_factor", C.c_double), ("kappa_max", C.c_double),
        ("alpha_min", C.c_double), ("alpha_max", C.c_double),
        ("n_mat", C.c_int), ("mat", C.POINTER(C.c_double)),
        ("n_brick", C.c_int), ("brick", C.POINTER(C.c_double)),
        ("n_sphere", C.c_int), ("sphere", C.POINTER(C.c_double)),
        ("n_wave", C.c_int), ("wave", C.POINTER(C.c_double)),
        ("n_vs", C.c_int), ("vs", C.POINTER(C.c_double)),
        ("n_sv", C.c_int), ("sv", C.POINTER(C.c_double)),
        ("n_si", C.c_int), ("si", C.POINTER(C.c_double)),
        ("n_ff", C.c_int), ("ff_freq", C.POINTER(C.c_double)),
        ("nc_ff", C.c_int),
    ]


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, no GPU needed)."""
    src = os.path.join(HERE, "fdtd_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        L.ofd_create.restype = C.c_void_p
        L.ofd_create.argtypes = [C.POINTER(_Scn)]
        L.ofd_step.restype = C.c_int
        L.ofd_step.argtypes = [C.c_void_p, C.c_int]
        L.ofd_meta.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.ofd_get.restype = C.c_long
        L.ofd_get.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_double), C.c_long]
        L.ofd_set.restype = C.c_long
        L.ofd_set.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_double), C.c_long]
        L.ofd_destroy.argtypes = [C.c_void_p]
        L.ofd_set_threads.argtypes = [C.c_int]
        L.ofd_max_threads.restype = C.c_int
        L.ofd_set_edge_read.argtypes = [C.c_int]
        dp = C.POINTER(C.c_double)
        L.ofd_time_to_freq.argtypes = [dp, C.c_int, C.c_double, dp, C.c_int, C.c_double, dp, dp]
        L.ofd_s11.argtypes = [dp, dp, dp, dp, C.c_int, C.c_double, dp, dp, dp, dp]
        L.ofd_radiated_power.argtypes = [C.c_void_p, dp]
        L.ofd_directivity.argtypes = [C.c_void_p, dp, dp, dp, C.c_int, dp, dp]
        _lib = L
    return _lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _axis_sign(direction: str):
    return "xyz".index(direction[0]), (-1.0 if direction[1] == "n" else 1.0)


def scenario_params(scn: dict, steps: int | None = None) -> dict[str, Any]:
    """Resolve a scenario dict into flat numeric tables (scenario.js:73-131 defaults)."""
    cell = dict(DEFAULTS["cell"], **(scn.get("cell") or {}))
    nsteps = int(steps or scn.get("numberOfTimeSteps") or DEFAULTS["numberOfTimeSteps"])
    ncpw = scn.get("numberOfCellsPerWavelength", DEFAULTS["numberOfCellsPerWavelength"])
    b = scn["boundary"]
    mats = np.array([[m["eps_r"], m.get("mu_r", 0), m["sigma_e"], m.get("sigma_m", 0)]
                     for m in scn["materialTypes"]], dtype=np.float64).reshape(-1, 4)
    bricks = np.array([[x["min_x"], x["min_y"], x["min_z"], x["max_x"], x["max_y"], x["max_z"],
                        x["material_type"]] for x in scn.get("bricks", [])], dtype=np.float64).reshape(-1, 7)
    spheres = np.array([[s["center_x"], s["center_y"], s["center_z"], s["radius"], s["material_type"]]
                        for s in (scn.get("spheres") or [])], dtype=np.float64).reshape(-1, 5)
    waves, wave_index = [], {}
    wf = scn.get("waveforms") or {}
    for kind_id, kind in enumerate(WAVE_KINDS):
        for n, w in enumerate(wf.get(kind, []) or []):
            wave_index[(kind, n + 1)] = len(waves)
            if kind in ("gaussian", "derivative_gaussian"):
                nc = w["number_of_cells_per_wavelength"]
                waves.append([kind_id, ncpw if nc == 0 else nc, 0, 0])
            elif kind == "sinusoidal":
                waves.append([kind_id, w["frequency"], 0, 0])
            elif kind == "unit_step":
                waves.append([kind_id, w["start_time_step"], 0, 0])
            else:
                waves.append([kind_id, w["bandwidth"], w["modulation_frequency"], 0])
    vs = []
    for v in scn.get("voltageSources", []) or []:
        ax, sg = _axis_sign(v["direction"])
        vs.append([v["min_x"], v["min_y"], v["min_z"], v["max_x"], v["max_y"], v["max_z"], ax, sg,
                   v["resistance"], v["magnitude"], wave_index[(v["waveform_type"], v["waveform_index"])]])

    def box(lst):
        out = []
        for p in lst or []:
            ax, sg = _axis_sign(p["direction"])
            out.append([p["min_x"], p["min_y"], p["min_z"], p["max_x"], p["max_y"], p["max_z"], ax, sg])
        return np.array(out, dtype=np.float64).reshape(-1, 8)

    ffp = dict(DEFAULTS["farfield"], **(scn.get("farfield") or {}))
    dft = dict(DEFAULTS["dft"], **(scn.get("dft") or {}))
    return {
        "dx": cell["dx"], "dy": cell["dy"], "dz": cell["dz"],
        "courant": scn.get("courantFactor", DEFAULTS["courantFactor"]), "nsteps": nsteps,
        "is_cpml": [int(b[f"type_{f}"] == "cpml") for f in FACES],
        "air": [int(b[f"air_buffer_{f}"]) for f in FACES],
        "ncpml": [int(b.get(f"cpml_cells_{f}", 0)) for f in FACES],
        "cpml": [b.get("cpml_order", 3), b.get("cpml_sigma_factor", 1.3), b.get("cpml_kappa_max", 7),
                 b.get("cpml_alpha_min", 0), b.get("cpml_alpha_max", 0.05)],
        "mat": mats, "brick": bricks, "sphere": spheres,
        "wave": np.array(waves, dtype=np.float64).reshape(-1, 4),
        "vs": np.array(vs, dtype=np.float64).reshape(-1, 11),
        "sv": box(scn.get("sampledVoltages")), "si": box(scn.get("sampledCurrents")),
        "ff_freq": np.array(ffp.get("frequencies") or [], dtype=np.float64),
        "nc_ff": int(ffp.get("number_of_cells_from_outer_boundary", 13)),
        "dft": dft, "ports": scn.get("ports") or [],
    }


class Oracle:
    """One FP64 reference simulation (setup + time loop + post-processing)."""

    def __init__(self, scn: dict, steps: int | None = None, threads: int | None = None,
                 edge_read_old: bool = False):
        """``edge_read_old`` selects which Ex(i=0) values the Ey(i=nx) bulk update
        reads through its out-of-range Hz neighbour (fdtd_oracle.c header)."""
        L = lib()
        self.edge_read_old = bool(edge_read_old)
        if threads:
            L.ofd_set_threads(int(threads))
        p = scenario_params(scn, steps)
        self.params = p
        keep = {k: np.ascontiguousarray(p[k], dtype=np.float64)
                for k in ("mat", "brick", "sphere", "wave", "vs", "sv", "si", "ff_freq")}
        self._keep = keep
        s = _Scn()
        s.dx, s.dy, s.dz, s.courant = p["dx"], p["dy"], p["dz"], p["courant"]
        s.nsteps = p["nsteps"]
        for i in range(6):
            s.is_cpml[i], s.air[i], s.ncpml[i] = p["is_cpml"][i], p["air"][i], p["ncpml"][i]
        s.cpml_order, s.sigma_factor, s.kappa_max, s.alpha_min, s.alpha_max = [float(x) for x in p["cpml"]]
        for key, n in (("mat", "n_mat"), ("brick", "n_brick"), ("sphere", "n_sphere"), ("wave", "n_wave"),
                       ("vs", "n_vs"), ("sv", "n_sv"), ("si", "n_si")):
            setattr(s, n, keep[key].shape[0])
            setattr(s, key, _dptr(keep[key]))
        s.n_ff = keep["ff_freq"].shape[0]
        s.ff_freq = _dptr(keep["ff_freq"])
        s.nc_ff = p["nc_ff"]
        self._h = L.ofd_create(C.byref(s))
        ints = (C.c_int * 15)()
        dbl = (C.c_double * 10)()
        L.ofd_meta(self._h, ints, dbl)
        (self.nx, self.ny, self.nz, self.nsteps, _, self.nfreq, self.li, self.lj, self.lk,
         self.ui, self.uj, self.uk, self.n_vs, self.n_sv, self.n_si) = list(ints)
        (self.dx, self.dy, self.dz, self.dt, self.min_x, self.min_y, self.min_z,
         self.max_x, self.max_y, self.max_z) = list(dbl)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.ofd_destroy(h)
            self._h = None

    @property
    def ts(self) -> int:
        ints = (C.c_int * 15)()
        dbl = (C.c_double * 10)()
        lib().ofd_meta(self._h, ints, dbl)
        return ints[4]

    def step(self, count: int) -> int:
        lib().ofd_set_edge_read(int(self.edge_read_old))
        return lib().ofd_step(self._h, int(count))

    def get(self, name: str) -> np.ndarray:
        n = lib().ofd_get(self._h, name.encode(), None, 0)
        if n < 0:
            raise KeyError(name)
        out = np.empty(n, dtype=np.float64)
        lib().ofd_get(self._h, name.encode(), _dptr(out), n)
        return out

    def set(self, name: str, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        if lib().ofd_set(self._h, name.encode(), _dptr(v), v.size) != v.size:
            raise KeyError(name)

    def farfield(self) -> dict[str, tuple[np.ndarray, np.ndarray]]:
        return {n: (self.get(f"ff:{n}:0"), self.get(f"ff:{n}:1")) for n in FF_NAMES}

    # -- post-processing ------------------------------------------------------
    def radiated_power(self) -> np.ndarray:
        out = np.zeros(self.nfreq)
        lib().ofd_radiated_power(self._h, _dptr(out))
        return out

    def directivity(self, radp: np.ndarray, theta: np.ndarray, phi: np.ndarray):
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        radp = np.ascontiguousarray(radp, dtype=np.float64)
        dth = np.zeros((self.nfreq, theta.size))
        dph = np.zeros((self.nfreq, theta.size))
        lib().ofd_directivity(self._h, _dptr(radp), _dptr(theta), _dptr(phi), theta.size, _dptr(dth), _dptr(dph))
        return dth, dph


def time_to_freq(x: np.ndarray, dt: float, freqs: np.ndarray, shift: float):
    x = np.ascontiguousarray(x, dtype=np.float64)
    f = np.ascontiguousarray(freqs, dtype=np.float64)
    re = np.zeros(f.size)
    im = np.zeros(f.size)
    lib().ofd_time_to_freq(_dptr(x), x.size, dt, _dptr(f), f.size, shift, _dptr(re), _dptr(im))
    return re, im


def s11(V: tuple, I: tuple, Z: float):
    M = V[0].size
    outs = [np.zeros(M) for _ in range(4)]
    args = [np.ascontiguousarray(a, dtype=np.float64) for a in (V[0], V[1], I[0], I[1])]
    lib().ofd_s11(*[_dptr(a) for a in args], M, float(Z), *[_dptr(o) for o in outs])
    return {"re": outs[0], "im": outs[1], "mag_dB": outs[2], "phase_deg": outs[3]}


def dft_freqs(dft: dict) -> np.ndarray:
    """index.js:64-67."""
    n = int(math.floor(dft["maxFreq"] / dft["step"]))
    return np.array([(i + 1) * dft["step"] for i in range(n)], dtype=np.float64)


def xy_xz_angles():
    """index.js:77-91: 360 one-degree angles; xy cut at theta=90 deg, xz cut folded."""
    angles = np.array([i * math.pi / 180 for i in range(360)], dtype=np.float64)
    th_xy = np.full(360, math.pi / 2)
    ph_xz = np.array([math.pi if a > math.pi else 0.0 for a in angles])
    th_xz = np.array([2 * math.pi - a if a > math.pi else a for a in angles])
    return angles, th_xy, th_xz, ph_xz


def to_db(x: np.ndarray) -> np.ndarray:
    return np.array([10 * math.log10(max(v, 1e-10)) for v in x])


def run_pipeline(scn: dict, steps: int | None = None, threads: int | None = None,
                 edge_read_old: bool = False) -> dict[str, Any]:
    """Whole CLI run (index.js:25-134) on the oracle: time loop, S11, far-field cuts."""
    o = Oracle(scn, steps, threads, edge_read_old)
    o.step(o.nsteps)
    p = o.params
    freqs = dft_freqs(p["dft"])
    V = [o.get(f"V:{n}") for n in range(o.n_sv)]
    I = [o.get(f"I:{n}") for n in range(o.n_si)]
    res: dict[str, Any] = {"dt": o.dt, "V": V, "I": I, "freqs": freqs, "oracle": o}
    sp = []
    for port in p["ports"]:
        if not port.get("is_source_port"):
            continue
        vf = time_to_freq(V[port["sampled_voltage_index"] - 1], o.dt, freqs, 0.0)
        jf = time_to_freq(I[port["sampled_current_index"] - 1], o.dt, freqs, -o.dt / 2)
        Z = port["impedance"] if isinstance(port["impedance"], (int, float)) else port["impedance"]["re"]
        sp.append(s11(vf, jf, Z))
    res["sparams"] = sp
    ff = []
    if o.nfreq > 0:
        radp = o.radiated_power()
        angles, th_xy, th_xz, ph_xz = xy_xz_angles()
        dth_xy, dph_xy = o.directivity(radp, th_xy, angles)
        dth_xz, dph_xz = o.directivity(radp, th_xz, ph_xz)
        for f in range(o.nfreq):
            ff.append({"plane": "xy", "dataTheta_dB": to_db(dth_xy[f]), "dataPhi_dB": to_db(dph_xy[f])})
            ff.append({"plane": "xz", "dataTheta_dB": to_db(dth_xz[f]), "dataPhi_dB": to_db(dph_xz[f])})
        res["radiated_power"] = radp
    res["farfield"] = ff
    return res
