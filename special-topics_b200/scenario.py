"""Problem construction: scenario JSON -> arrays the engine consumes.

Mirrors js_fdtd/src/scenario.js:73-131 (buildProblemFromScenario) and the
setup modules it calls, vectorised with numpy but with the reference's
expression order in every elementwise formula, so the FP64 arrays are
bit-identical to the reference's:

  grid            js_fdtd/src/grid.js:16-187, 228-243
  materials       js_fdtd/src/materials.js:21-332
  coefficients    js_fdtd/src/coefficients.js:22-116, 136-207
  CPML            js_fdtd/src/cpml.js:25-448
  waveforms       js_fdtd/src/sources.js:16-145
  samplers        js_fdtd/src/sampling.js:81-136
  far field box   js_fdtd/src/farfield.js:28-78

Transcendentals (exp/pow/sqrt) of the 1-D profiles and waveforms use the
``math`` module one value at a time; everything per cell is + - * /.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Any

import numpy as np

EPS0 = 8.854187817e-12
MU0 = 4 * math.pi * 1e-7
C0 = 2.99792458e8
ETA0 = 376.73031346177066

DEFAULTS = {  # scenario.js:32-40
    "courantFactor": 0.9,
    "numberOfCellsPerWavelength": 20,
    "numberOfTimeSteps": 4000,
    "cell": {"dx": 0.262e-3, "dy": 0.4e-3, "dz": 0.4e-3},
    "dft": {"maxFreq": 10e9, "step": 20e6},
    "farfield": {"frequencies": [], "number_of_cells_from_outer_boundary": 13},
}
FACES = ("xn", "xp", "yn", "yp", "zn", "zp")
# coefficient ids (js_fdtd/src/backends/cuda/cudaBackend.js:53-60)
COEFF_ORDER = ("Cexe", "Cexhz", "Cexhy", "Ceye", "Ceyhx", "Ceyhz", "Ceze", "Cezhy", "Cezhx",
               "Chxh", "Chxey", "Chxez", "Chyh", "Chyez", "Chyex", "Chzh", "Chzex", "Chzey")
FF_NAMES = ("cjyxp", "cjzxp", "cjyxn", "cjzxn", "cjxyp", "cjzyp", "cjxyn", "cjzyn",
            "cjxzp", "cjyzp", "cjxzn", "cjyzn", "cmyxp", "cmzxp", "cmyxn", "cmzxn",
            "cmxyp", "cmzyp", "cmxyn", "cmzyn", "cmxzp", "cmyzp", "cmxzn", "cmyzn")


def js_round(x: float) -> int:
    """Math.round: nearest integer, ties toward +infinity."""
    f = math.floor(x)
    return int(f + 1) if x - f >= 0.5 else int(f)


@dataclass
class Grid:
    dx: float
    dy: float
    dz: float
    dt: float
    nx: int
    ny: int
    nz: int
    min_x: float
    min_y: float
    min_z: float
    max_x: float
    max_y: float
    max_z: float
    numberOfTimeSteps: int

    @property
    def shapes(self) -> dict[str, tuple[int, int, int]]:
        nx, ny, nz = self.nx, self.ny, self.nz
        return {"Hx": (nx + 1, ny, nz), "Hy": (nx, ny + 1, nz), "Hz": (nx, ny, nz + 1),
                "Ex": (nx, ny + 1, nz + 1), "Ey": (nx + 1, ny, nz + 1), "Ez": (nx + 1, ny + 1, nz)}

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz


@dataclass
class CpmlFace:
    face: str
    nc: int
    b_e: np.ndarray
    a_e: np.ndarray
    b_m: np.ndarray
    a_m: np.ndarray
    kappa_e: np.ndarray
    kappa_m: np.ndarray
    cpsi: list            # 4 flat arrays, slots as cpml.js (x: hyx hzx eyx ezx, ...)
    m_start: int
    e_start: int


@dataclass
class VoltageSource:
    axis: int
    field_indices: np.ndarray   # int32, createLinearIndexList order
    coef: np.ndarray            # Cexs / Ceys / Cezs
    voltage_per_e_field: np.ndarray
    resistance_per_component: float
    box: tuple                  # 1-based is, js, ks, ie, je, ke
    override: np.ndarray        # (cells, 3): the gap cells' self and curl coefficients


@dataclass
class VoltageProbe:
    axis: int
    field_indices: np.ndarray
    Csvf: float
    label: str = ""


@dataclass
class CurrentProbe:
    comp: np.ndarray            # 0=Hx 1=Hy 2=Hz, in summation order
    idx: np.ndarray
    w: np.ndarray               # +-d with the probe's sign folded in
    label: str = ""


@dataclass
class FarFieldBox:
    frequencies: np.ndarray
    li: int
    lj: int
    lk: int
    ui: int
    uj: int
    uk: int

    @property
    def nFreq(self) -> int:
        return int(self.frequencies.size)


@dataclass
class Problem:
    grid: Grid
    coeffs: dict[str, np.ndarray]            # 18 FP64 arrays, flat, reference layout
    materials: dict[str, np.ndarray]         # eps_r_x ... sigma_m_z (flat)
    cpml: list                                # CpmlFace per present face (index = face id) or None
    voltage_sources: list
    sampled_voltages: list
    sampled_currents: list
    farfield: FarFieldBox | None
    ports: list
    dft: dict
    meta: dict = field(default_factory=dict)


# ---------------------------------------------------------------------------
# grid.js:16-187
# ---------------------------------------------------------------------------
def build_grid(dx, dy, dz, boundary, bricks, spheres, courant, nsteps) -> Grid:
    mn = [math.inf] * 3
    mx = [-math.inf] * 3
    for s in spheres:
        c = (s["center_x"], s["center_y"], s["center_z"])
        for a in range(3):
            mn[a] = min(mn[a], c[a] - s["radius"])
            mx[a] = max(mx[a], c[a] + s["radius"])
    for b in bricks:
        lo = (b["min_x"], b["min_y"], b["min_z"])
        hi = (b["max_x"], b["max_y"], b["max_z"])
        for a in range(3):
            mn[a] = min(mn[a], lo[a])
            mx[a] = max(mx[a], hi[a])
    d = (dx, dy, dz)
    for a, ax in enumerate("xyz"):
        mn[a] -= d[a] * boundary[f"air_buffer_{ax}n"]
        mx[a] += d[a] * boundary[f"air_buffer_{ax}p"]
    for a, ax in enumerate("xyz"):
        if boundary[f"type_{ax}n"] == "cpml" and boundary.get(f"cpml_cells_{ax}n", 0) > 0:
            mn[a] -= d[a] * boundary[f"cpml_cells_{ax}n"]
        if boundary[f"type_{ax}p"] == "cpml" and boundary.get(f"cpml_cells_{ax}p", 0) > 0:
            mx[a] += d[a] * boundary[f"cpml_cells_{ax}p"]
    n = [js_round((mx[a] - mn[a]) / d[a]) for a in range(3)]
    dt = courant / (C0 * math.sqrt(1 / (dx * dx) + 1 / (dy * dy) + 1 / (dz * dz)))
    return Grid(dx, dy, dz, dt, n[0], n[1], n[2], mn[0], mn[1], mn[2],
                mn[0] + n[0] * dx, mn[1] + n[1] * dy, mn[2] + n[2] * dz, nsteps)


def create_linear_index_list(i_s, i_e, j_s, j_e, k_s, k_e, d2, d3) -> np.ndarray:
    """grid.js:228-243: 1-based inclusive box -> flat 0-based indices, k outer, j, i inner."""
    ii = np.arange(i_s, i_e + 1, dtype=np.int64)
    jj = np.arange(j_s, j_e + 1, dtype=np.int64)
    kk = np.arange(k_s, k_e + 1, dtype=np.int64)
    K, J, I = np.meshgrid(kk, jj, ii, indexing="ij")
    return ((I - 1) * d2 * d3 + (J - 1) * d3 + (K - 1)).ravel().astype(np.int32)


# ---------------------------------------------------------------------------
# materials.js:21-332
# ---------------------------------------------------------------------------
def build_material_grid(g: Grid, bricks, spheres) -> np.ndarray:
    nx, ny, nz = g.nx, g.ny, g.nz
    mat = np.ones((nx, ny, nz), dtype=np.uint8)
    if spheres:
        cx = (np.arange(nx) + 0.5) * g.dx + g.min_x
        cy = (np.arange(ny) + 0.5) * g.dy + g.min_y
        cz = (np.arange(nz) + 0.5) * g.dz + g.min_z
        for s in spheres:
            ddx = (cx - s["center_x"])[:, None, None]
            ddy = (cy - s["center_y"])[None, :, None]
            ddz = (cz - s["center_z"])[None, None, :]
            inside = ddx * ddx + ddy * ddy + ddz * ddz <= s["radius"] * s["radius"]
            mat[inside] = s["material_type"] % 256
    for b in bricks:
        lo = [js_round((b["min_x"] - g.min_x) / g.dx), js_round((b["min_y"] - g.min_y) / g.dy),
              js_round((b["min_z"] - g.min_z) / g.dz)]
        hi = [js_round((b["max_x"] - g.min_x) / g.dx), js_round((b["max_y"] - g.min_y) / g.dy),
              js_round((b["max_z"] - g.min_z) / g.dz)]
        sl = tuple(slice(max(lo[a], 0), max(min(hi[a], n), 0)) for a, n in enumerate((nx, ny, nz)))
        mat[sl] = b["material_type"] % 256
    return mat


def compute_material_components(mat: np.ndarray, material_types, g: Grid) -> dict[str, np.ndarray]:
    nx, ny, nz = g.nx, g.ny, g.nz
    nmt = len(material_types)
    t_eps = np.zeros(nmt + 1)
    t_mu = np.zeros(nmt + 1)
    t_se = np.zeros(nmt + 1)
    t_sm = np.zeros(nmt + 1)
    for m, mt in enumerate(material_types):
        t_eps[m + 1] = mt["eps_r"]
        mu = mt.get("mu_r", 0) or 0
        t_mu[m + 1] = mu if (mu == mu and mu != 0) else 1e-20
        t_se[m + 1] = mt["sigma_e"]
        sm = mt.get("sigma_m", 0) or 0
        t_sm[m + 1] = sm if (sm == sm and sm != 0) else 1e-20
    if mat.max() > nmt:
        raise ValueError(f"brick material_type {int(mat.max())} exceeds the {nmt} material types")
    out = {}
    # eps_r_x / sigma_e_x: (nx, ny+1, nz+1), interior j in [1,ny), k in [1,nz)
    eps = np.ones((nx, ny + 1, nz + 1))
    sig = np.zeros((nx, ny + 1, nz + 1))
    m1, m2, m3, m4 = mat[:, 1:, 1:], mat[:, :-1, 1:], mat[:, 1:, :-1], mat[:, :-1, :-1]
    eps[:, 1:ny, 1:nz] = 0.25 * (t_eps[m1] + t_eps[m2] + t_eps[m3] + t_eps[m4])
    sig[:, 1:ny, 1:nz] = 0.25 * (t_se[m1] + t_se[m2] + t_se[m3] + t_se[m4])
    out["eps_r_x"], out["sigma_e_x"] = eps, sig
    # eps_r_y: (nx+1, ny, nz+1), i in [1,nx), k in [1,nz)
    eps = np.ones((nx + 1, ny, nz + 1))
    sig = np.zeros((nx + 1, ny, nz + 1))
    m1, m2, m3, m4 = mat[1:, :, 1:], mat[:-1, :, 1:], mat[1:, :, :-1], mat[:-1, :, :-1]
    eps[1:nx, :, 1:nz] = 0.25 * (t_eps[m1] + t_eps[m2] + t_eps[m3] + t_eps[m4])
    sig[1:nx, :, 1:nz] = 0.25 * (t_se[m1] + t_se[m2] + t_se[m3] + t_se[m4])
    out["eps_r_y"], out["sigma_e_y"] = eps, sig
    # eps_r_z: (nx+1, ny+1, nz), i in [1,nx), j in [1,ny)
    eps = np.ones((nx + 1, ny + 1, nz))
    sig = np.zeros((nx + 1, ny + 1, nz))
    m1, m2, m3, m4 = mat[1:, 1:, :], mat[:-1, 1:, :], mat[1:, :-1, :], mat[:-1, :-1, :]
    eps[1:nx, 1:ny, :] = 0.25 * (t_eps[m1] + t_eps[m2] + t_eps[m3] + t_eps[m4])
    sig[1:nx, 1:ny, :] = 0.25 * (t_se[m1] + t_se[m2] + t_se[m3] + t_se[m4])
    out["eps_r_z"], out["sigma_e_z"] = eps, sig
    del m1, m2, m3, m4

    def harm(a, b):
        return 2 * a * b / (a + b)

    mu = np.ones((nx + 1, ny, nz))
    sm = np.full((nx + 1, ny, nz), 0.0)
    mu[1:nx] = harm(t_mu[mat[1:]], t_mu[mat[:-1]])
    sm[1:nx] = harm(t_sm[mat[1:]], t_sm[mat[:-1]])
    out["mu_r_x"], out["sigma_m_x"] = mu, sm
    mu = np.ones((nx, ny + 1, nz))
    sm = np.zeros((nx, ny + 1, nz))
    mu[:, 1:ny] = harm(t_mu[mat[:, 1:]], t_mu[mat[:, :-1]])
    sm[:, 1:ny] = harm(t_sm[mat[:, 1:]], t_sm[mat[:, :-1]])
    out["mu_r_y"], out["sigma_m_y"] = mu, sm
    mu = np.ones((nx, ny, nz + 1))
    sm = np.zeros((nx, ny, nz + 1))
    mu[:, :, 1:nz] = harm(t_mu[mat[:, :, 1:]], t_mu[mat[:, :, :-1]])
    sm[:, :, 1:nz] = harm(t_sm[mat[:, :, 1:]], t_sm[mat[:, :, :-1]])
    out["mu_r_z"], out["sigma_m_z"] = mu, sm
    return out


def material_props(material_types) -> np.ndarray:
    """(types+1) x 4 table eps_r, mu_r, sigma_e, sigma_m by 1-based type id; row 0 stays
    zero and mu_r / sigma_m of 0 become 1e-20 (materials.js:90-101)."""
    t = np.zeros((len(material_types) + 1, 4))
    for m, mt in enumerate(material_types):
        mu = mt.get("mu_r", 0) or 0
        sm = mt.get("sigma_m", 0) or 0
        t[m + 1] = (mt["eps_r"], mu if (mu == mu and mu != 0) else 1e-20, mt["sigma_e"],
                    sm if (sm == sm and sm != 0) else 1e-20)
    return t


def pec_plate_boxes(bricks, material_types, g: Grid) -> list:
    """materials.js:253-332 as an ordered list of (component 0=Ex 1=Ey 2=Ez,
    i0, i1, j0, j1, k0, k1 inclusive, sigma) boxes; later boxes overwrite earlier."""
    nx, ny, nz = g.nx, g.ny, g.nz
    ext = {0: (nx, ny + 1, nz + 1), 1: (nx + 1, ny, nz + 1), 2: (nx + 1, ny + 1, nz)}
    out = []

    def add(comp, ri, rj, rk, sigma):
        lo_hi = []
        for (a, b), n in zip((ri, rj, rk), ext[comp]):
            a, b = max(a, 0), min(b, n)      # [a, b) clipped like the reference's bounds checks
            if a >= b:
                return
            lo_hi += [a, b - 1]
        out.append((comp, *lo_hi, sigma))

    for b in bricks:
        sigma_pec = material_types[b["material_type"] - 1]["sigma_e"]
        if sigma_pec == 0:
            continue
        blx = js_round((b["min_x"] - g.min_x) / g.dx) + 1
        bly = js_round((b["min_y"] - g.min_y) / g.dy) + 1
        blz = js_round((b["min_z"] - g.min_z) / g.dz) + 1
        bux = js_round((b["max_x"] - g.min_x) / g.dx) + 1
        buy = js_round((b["max_y"] - g.min_y) / g.dy) + 1
        buz = js_round((b["max_z"] - g.min_z) / g.dz) + 1
        if blx == bux and 0 <= blx - 1 < nx + 1:
            i = blx - 1
            add(1, (i, i + 1), (bly - 1, buy - 1), (blz - 1, buz), sigma_pec)
            add(2, (i, i + 1), (bly - 1, buy), (blz - 1, buz - 1), sigma_pec)
        if bly == buy and 0 <= bly - 1 < ny + 1:
            j = bly - 1
            add(0, (blx - 1, bux - 1), (j, j + 1), (blz - 1, buz), sigma_pec)
            add(2, (blx - 1, bux), (j, j + 1), (blz - 1, buz - 1), sigma_pec)
        if blz == buz and 0 <= blz - 1 < nz + 1:
            k = blz - 1
            add(0, (blx - 1, bux - 1), (bly - 1, buy), (k, k + 1), sigma_pec)
            add(1, (blx - 1, bux), (bly - 1, buy - 1), (k, k + 1), sigma_pec)
    return out


def apply_pec_plates(bricks, material_types, mc, g: Grid) -> None:
    """materials.js:253-332 (zero-thickness conducting bricks)."""
    arrs = (mc["sigma_e_x"], mc["sigma_e_y"], mc["sigma_e_z"])
    for comp, i0, i1, j0, j1, k0, k1, sigma in pec_plate_boxes(bricks, material_types, g):
        arrs[comp][i0:i1 + 1, j0:j1 + 1, k0:k1 + 1] = sigma


def e_values_at(axis: int, fi: np.ndarray, mat: np.ndarray, props: np.ndarray, plates: list, g: Grid):
    """(eps_r, sigma_e) of E component `axis` at flat indices fi, exactly as
    computeMaterialComponents + applyPECPlates would leave them."""
    nx, ny, nz = g.nx, g.ny, g.nz
    shape = {0: (nx, ny + 1, nz + 1), 1: (nx + 1, ny, nz + 1), 2: (nx + 1, ny + 1, nz)}[axis]
    i, j, k = np.unravel_index(np.asarray(fi, dtype=np.int64), shape)
    e = np.ones(i.size)
    s = np.zeros(i.size)
    if axis == 0:
        inside = (j >= 1) & (j < ny) & (k >= 1) & (k < nz)
        nb = ((0, 0, 0), (0, -1, 0), (0, 0, -1), (0, -1, -1))
    elif axis == 1:
        inside = (i >= 1) & (i < nx) & (k >= 1) & (k < nz)
        nb = ((0, 0, 0), (-1, 0, 0), (0, 0, -1), (-1, 0, -1))
    else:
        inside = (i >= 1) & (i < nx) & (j >= 1) & (j < ny)
        nb = ((0, 0, 0), (-1, 0, 0), (0, -1, 0), (-1, -1, 0))
    q = np.nonzero(inside)[0]
    m = [mat[i[q] + a, j[q] + b, k[q] + c] for a, b, c in nb]
    e[q] = 0.25 * (props[m[0], 0] + props[m[1], 0] + props[m[2], 0] + props[m[3], 0])
    s[q] = 0.25 * (props[m[0], 2] + props[m[1], 2] + props[m[2], 2] + props[m[3], 2])
    for comp, i0, i1, j0, j1, k0, k1, sigma in plates:
        if comp == axis:
            s[(i >= i0) & (i <= i1) & (j >= j0) & (j <= j1) & (k >= k0) & (k <= k1)] = sigma
    return e, s


# ---------------------------------------------------------------------------
# coefficients.js:22-116
# ---------------------------------------------------------------------------
def compute_general_coefficients(mc, g: Grid) -> dict[str, np.ndarray]:
    dt = g.dt
    two_dt_dy, two_dt_dz, two_dt_dx = 2 * dt / g.dy, 2 * dt / g.dz, 2 * dt / g.dx
    c = {}
    for comp, (e, s, n1, v1, n2, v2) in {
        "x": ("eps_r_x", "sigma_e_x", "Cexhz", two_dt_dy, "Cexhy", -two_dt_dz),
        "y": ("eps_r_y", "sigma_e_y", "Ceyhx", two_dt_dz, "Ceyhz", -two_dt_dx),
        "z": ("eps_r_z", "sigma_e_z", "Cezhy", two_dt_dx, "Cezhx", -two_dt_dy),
    }.items():
        a = 2 * mc[e] * EPS0
        b = dt * mc[s]
        denom = a + b
        c[f"Ce{comp}e"] = (a - b) / denom
        c[n1] = v1 / denom
        c[n2] = v2 / denom
    for comp, (m, s, n1, v1, n2, v2) in {
        "x": ("mu_r_x", "sigma_m_x", "Chxez", -two_dt_dy, "Chxey", two_dt_dz),
        "y": ("mu_r_y", "sigma_m_y", "Chyex", -two_dt_dz, "Chyez", two_dt_dx),
        "z": ("mu_r_z", "sigma_m_z", "Chzey", -two_dt_dx, "Chzex", two_dt_dy),
    }.items():
        a = 2 * mc[m] * MU0
        b = dt * mc[s]
        denom = a + b
        c[f"Ch{comp}h"] = (a - b) / denom
        c[n1] = v1 / denom
        c[n2] = v2 / denom
    return c


# ---------------------------------------------------------------------------
# cpml.js:25-448
# ---------------------------------------------------------------------------
def _cpml_1d(nc, cell, dt, p, sigma_ratio, kappa_max, alpha_min, alpha_max, ascending):
    sigma_max = sigma_ratio * (p + 1) / (150 * math.pi * cell)
    out = {k: np.zeros(nc) for k in ("b_e", "a_e", "b_m", "a_m", "kappa_e", "kappa_m")}
    for ci in range(nc):
        rho_e = (ci + 1 - 0.75) / nc if ascending else (nc - ci - 0.75) / nc
        rho_m = (ci + 1 - 0.25) / nc if ascending else (nc - ci - 0.25) / nc
        se = sigma_max * math.pow(rho_e, p)
        sm = (MU0 / EPS0) * sigma_max * math.pow(rho_m, p)
        ke = 1 + (kappa_max - 1) * math.pow(rho_e, p)
        km = 1 + (kappa_max - 1) * math.pow(rho_m, p)
        ae = alpha_min + (alpha_max - alpha_min) * (1 - rho_e)
        am = (MU0 / EPS0) * (alpha_min + (alpha_max - alpha_min) * (1 - rho_m))
        be = math.exp(-(dt / EPS0) * (se / ke + ae))
        bm = math.exp(-(dt / MU0) * (sm / km + am))
        out["b_e"][ci] = be
        out["a_e"][ci] = (1 / cell) * (be - 1) * se / (ke * (se + ke * ae))
        out["b_m"][ci] = bm
        out["a_m"][ci] = (1 / cell) * (bm - 1) * sm / (km * (sm + km * am))
        out["kappa_e"][ci] = ke
        out["kappa_m"][ci] = km
    return out


# per axis: (H coefficient of slot 0, H of slot 1, E of slot 2, E of slot 3); slot arrays
# index the band along the axis, so the CPsi of slot s is a slice of that coefficient.
_FACE_COEFS = {0: ("Chyez", "Chzey", "Ceyhz", "Cezhy"),
               1: ("Chxez", "Chzex", "Cezhx", "Cexhz"),
               2: ("Chxey", "Chyex", "Cexhy", "Ceyhx")}
_COEF_COMP = {"Chyez": "Hy", "Chzey": "Hz", "Ceyhz": "Ey", "Cezhy": "Ez",
              "Chxez": "Hx", "Chzex": "Hz", "Cezhx": "Ez", "Cexhz": "Ex",
              "Chxey": "Hx", "Chyex": "Hy", "Cexhy": "Ex", "Ceyhx": "Ey"}


def init_cpml(boundary, coeffs3d: dict[str, np.ndarray] | None, g: Grid) -> list:
    """Returns one CpmlFace per face id (None when that face is not a CPML);
    divides the affected 3-D coefficient arrays by kappa in place.  Without
    per-cell coefficients (material-table problems) only the 1-D profiles are
    made; CPsi is then None."""
    faces = [None] * 6
    p = boundary["cpml_order"]
    for fid, name in enumerate(FACES):
        if boundary[f"type_{name}"] != "cpml":
            continue
        nc = int(boundary[f"cpml_cells_{name}"])
        axis, ascending = fid // 2, fid % 2 == 1
        n_axis = (g.nx, g.ny, g.nz)[axis]
        cell = (g.dx, g.dy, g.dz)[axis]
        prof = _cpml_1d(nc, cell, g.dt, p, boundary["cpml_sigma_factor"], boundary["cpml_kappa_max"],
                        boundary["cpml_alpha_min"], boundary["cpml_alpha_max"], ascending)
        m_start = n_axis - nc if ascending else 0
        e_start = n_axis - nc if ascending else 1
        names = _FACE_COEFS[axis]
        if coeffs3d is None:
            faces[fid] = CpmlFace(name, nc, prof["b_e"], prof["a_e"], prof["b_m"], prof["a_m"],
                                  prof["kappa_e"], prof["kappa_m"], None, m_start, e_start)
            continue
        cpsi = []
        for s, nm in enumerate(names):
            arr = coeffs3d[nm]
            st = m_start if s < 2 else e_start
            sl = [slice(None)] * 3
            sl[axis] = slice(st, st + nc)
            cpsi.append(np.ascontiguousarray(arr[tuple(sl)] * cell).ravel())
        for s, nm in enumerate(names):
            arr = coeffs3d[nm]
            st = m_start if s < 2 else e_start
            kap = prof["kappa_m"] if s < 2 else prof["kappa_e"]
            shape = [1, 1, 1]
            shape[axis] = nc
            sl = [slice(None)] * 3
            sl[axis] = slice(st, st + nc)
            arr[tuple(sl)] /= kap.reshape(shape)
        faces[fid] = CpmlFace(name, nc, prof["b_e"], prof["a_e"], prof["b_m"], prof["a_m"],
                              prof["kappa_e"], prof["kappa_m"], cpsi, m_start, e_start)
    return faces


# ---------------------------------------------------------------------------
# sources.js:16-145 and coefficients.js:158-207
# ---------------------------------------------------------------------------
def init_waveforms(waveforms: dict, nsteps: int, dt: float, ncpw: int, cells) -> dict:
    max_cell = max(cells)
    out: dict[str, list] = {}
    t = [(n + 0.5) * dt for n in range(nsteps)]
    for kind, lst in (waveforms or {}).items():
        out[kind] = []
        for w in lst or []:
            wf = np.zeros(nsteps)
            if kind in ("gaussian", "derivative_gaussian"):
                nc = ncpw if w["number_of_cells_per_wavelength"] == 0 else w["number_of_cells_per_wavelength"]
                tau = (nc * max_cell) / (2 * C0)
                t0 = 4.5 * tau
                if kind == "gaussian":
                    for n in range(nsteps):
                        arg = (t[n] - t0) / tau
                        wf[n] = math.exp(-arg * arg)
                else:
                    scale = -math.sqrt(2 * math.e) / tau
                    for n in range(nsteps):
                        d2 = t[n] - t0
                        arg = d2 / tau
                        wf[n] = scale * d2 * math.exp(-arg * arg)
            elif kind == "sinusoidal":
                for n in range(nsteps):
                    wf[n] = math.sin(2 * math.pi * w["frequency"] * t[n])
            elif kind == "unit_step":
                wf[:] = 1.0
                wf[:max(int(w["start_time_step"]) - 1, 0)] = 0.0
            elif kind == "cosine_modulated_gaussian":
                tau = 0.966 / w["bandwidth"]
                t0 = 4.5 * tau
                for n in range(nsteps):
                    d2 = t[n] - t0
                    arg = d2 / tau
                    wf[n] = math.cos(2 * math.pi * w["modulation_frequency"] * d2) * math.exp(-arg * arg)
            else:
                raise ValueError(f"unknown waveform type {kind!r}")
            out[kind].append(wf)
    return out


def _box(el, g: Grid):
    return (js_round((el["min_x"] - g.min_x) / g.dx) + 1, js_round((el["min_y"] - g.min_y) / g.dy) + 1,
            js_round((el["min_z"] - g.min_z) / g.dz) + 1, js_round((el["max_x"] - g.min_x) / g.dx) + 1,
            js_round((el["max_y"] - g.min_y) / g.dy) + 1, js_round((el["max_z"] - g.min_z) / g.dz) + 1)


def init_voltage_sources(sources, waves, eps_sig_at, coeffs3d, g: Grid) -> list:
    out = []
    dt, dx, dy, dz = g.dt, g.dx, g.dy, g.dz
    nx, ny, nz = g.nx, g.ny, g.nz
    for vs in sources or []:
        i_s, j_s, k_s, i_e, j_e, k_e = _box(vs, g)
        axis = "xyz".index(vs["direction"][0])
        if axis == 0:
            n_fields = i_e - i_s
            r_fac = (1 + j_e - j_s) * (1 + k_e - k_s) / (i_e - i_s)
        elif axis == 1:
            n_fields = j_e - j_s
            r_fac = (1 + i_e - i_s) * (1 + k_e - k_s) / (j_e - j_s)
        else:
            n_fields = k_e - k_s
            r_fac = (1 + i_e - i_s) * (1 + j_e - j_s) / (k_e - k_s)
        v_sign = -1 if vs["direction"][1] == "n" else 1
        v_mag = v_sign * vs["magnitude"] / n_fields
        rpc = r_fac * vs["resistance"]
        base = waves[vs["waveform_type"]][vs["waveform_index"] - 1]
        vpe = v_mag * base
        R = rpc if rpc != 0 else 1e-20
        if axis == 0:
            fi = create_linear_index_list(i_s, i_e - 1, j_s, j_e, k_s, k_e, ny + 1, nz + 1)
            a_term = (dt * dx) / (R * dy * dz)
            ce, c1, c2 = "Cexe", "Cexhz", "Cexhy"
            v1, v2, vs_num = (2 * dt / dy), -(2 * dt / dz), -(2 * dt / (R * dy * dz))
        elif axis == 1:
            fi = create_linear_index_list(i_s, i_e, j_s, j_e - 1, k_s, k_e, ny, nz + 1)
            a_term = (dt * dy) / (R * dz * dx)
            ce, c1, c2 = "Ceye", "Ceyhx", "Ceyhz"
            v1, v2, vs_num = (2 * dt / dz), -(2 * dt / dx), -(2 * dt / (R * dz * dx))
        else:
            fi = create_linear_index_list(i_s, i_e, j_s, j_e, k_s, k_e - 1, ny + 1, nz)
            a_term = (dt * dz) / (R * dx * dy)
            ce, c1, c2 = "Ceze", "Cezhy", "Cezhx"
            v1, v2, vs_num = (2 * dt / dx), -(2 * dt / dy), -(2 * dt / (R * dx * dy))
        e, s = eps_sig_at(axis, fi)
        denom = 2 * EPS0 * e + dt * s + a_term
        trip = np.stack([(2 * EPS0 * e - dt * s - a_term) / denom, v1 / denom, v2 / denom], axis=1)
        if coeffs3d is not None:
            coeffs3d[ce].ravel()[fi] = trip[:, 0]
            coeffs3d[c1].ravel()[fi] = trip[:, 1]
            coeffs3d[c2].ravel()[fi] = trip[:, 2]
        cs = vs_num / denom
        out.append(VoltageSource(axis, fi, cs, vpe, rpc, (i_s, j_s, k_s, i_e, j_e, k_e), trip))
    return out


# ---------------------------------------------------------------------------
# sampling.js:81-136, 204-245
# ---------------------------------------------------------------------------
def init_sampled_voltages(probes, g: Grid) -> list:
    out = []
    ny, nz = g.ny, g.nz
    for obs in probes or []:
        i_s, j_s, k_s, i_e, j_e, k_e = _box(obs, g)
        axis = "xyz".index(obs["direction"][0])
        if axis == 0:
            fi = create_linear_index_list(i_s, i_e - 1, j_s, j_e, k_s, k_e, ny + 1, nz + 1)
            csvf = -g.dx / ((j_e - j_s + 1) * (k_e - k_s + 1))
        elif axis == 1:
            fi = create_linear_index_list(i_s, i_e, j_s, j_e - 1, k_s, k_e, ny, nz + 1)
            csvf = -g.dy / ((k_e - k_s + 1) * (i_e - i_s + 1))
        else:
            fi = create_linear_index_list(i_s, i_e, j_s, j_e, k_s, k_e - 1, ny + 1, nz)
            csvf = -g.dz / ((i_e - i_s + 1) * (j_e - j_s + 1))
        if obs["direction"][1] == "n":
            csvf *= -1
        out.append(VoltageProbe(axis, fi, csvf, obs.get("label", "")))
    return out


def init_sampled_currents(probes, g: Grid) -> list:
    """The Ampere loop of captureSampledCurrents as one ordered (component, index, weight) list."""
    out = []
    ny, nz, nyp1, nzp1 = g.ny, g.nz, g.ny + 1, g.nz + 1
    hx = lambda i, j, k: i * ny * nz + j * nz + k      # noqa: E731
    hy = lambda i, j, k: i * nyp1 * nz + j * nz + k    # noqa: E731
    hz = lambda i, j, k: i * ny * nzp1 + j * nzp1 + k  # noqa: E731
    for obs in probes or []:
        i_s, j_s, k_s, i_e, j_e, k_e = _box(obs, g)
        I, J, K, IE, JE, KE = i_s - 1, j_s - 1, k_s - 1, i_e - 1, j_e - 1, k_e - 1
        sg = -1.0 if obs["direction"][1] == "n" else 1.0
        terms = []
        a = obs["direction"][0]
        if a == "x":
            ix = IE - 1
            terms += [(1, hy(ix, j, K - 1), g.dy) for j in range(J, JE)]
            terms += [(2, hz(ix, JE - 1, k), g.dz) for k in range(K, KE)]
            terms += [(1, hy(ix, j, KE - 1), -g.dy) for j in range(J, JE)]
            terms += [(2, hz(ix, J - 1, k), -g.dz) for k in range(K, KE)]
        elif a == "y":
            jx = JE - 1
            terms += [(2, hz(I - 1, jx, k), g.dz) for k in range(K, KE)]
            terms += [(0, hx(i, jx, KE - 1), g.dx) for i in range(I, IE)]
            terms += [(2, hz(IE, jx, k), -g.dz) for k in range(K, KE)]
            terms += [(0, hx(i, jx, K - 1), -g.dx) for i in range(I, IE)]
        else:
            kx = KE - 1
            terms += [(0, hx(i, J - 1, kx), g.dx) for i in range(I, IE)]
            terms += [(1, hy(IE, j, kx), g.dy) for j in range(J, JE)]
            terms += [(0, hx(i, JE, kx), -g.dx) for i in range(I, IE)]
            terms += [(1, hy(I - 1, j, kx), -g.dy) for j in range(J, JE)]
        if not terms:
            raise ValueError("current probe loop is empty")
        comp = np.array([t[0] for t in terms], dtype=np.int32)
        idx = np.array([t[1] for t in terms], dtype=np.int32)
        w = np.array([sg * t[2] for t in terms], dtype=np.float64)
        out.append(CurrentProbe(comp, idx, w, obs.get("label", "")))
    return out


# ---------------------------------------------------------------------------
# scenario.js:73-131
# ---------------------------------------------------------------------------
def build_problem_from_scenario(scn: dict, steps: int | None = None, per_cell: bool = True) -> Problem:
    """scenario.js:73-131.  per_cell=False skips the 18 per-cell coefficient
    arrays and the CPsi slices (a material-table problem needs neither)."""
    courant = scn.get("courantFactor", DEFAULTS["courantFactor"])
    ncpw = scn.get("numberOfCellsPerWavelength", DEFAULTS["numberOfCellsPerWavelength"])
    nsteps = int(steps or scn.get("numberOfTimeSteps") or DEFAULTS["numberOfTimeSteps"])
    cell = dict(DEFAULTS["cell"], **(scn.get("cell") or {}))
    dx, dy, dz = cell["dx"], cell["dy"], cell["dz"]
    boundary = scn["boundary"]
    mtypes = scn["materialTypes"]
    bricks = scn.get("bricks") or []
    spheres = scn.get("spheres") or []
    if scn.get("sampledElectricFields") or scn.get("sampledMagneticFields"):
        raise ValueError("point field probes are not supported by this engine")
    g = build_grid(dx, dy, dz, boundary, bricks, spheres, courant, nsteps)
    mat = build_material_grid(g, bricks, spheres)
    props = material_props(mtypes)
    plates = pec_plate_boxes(bricks, mtypes, g)
    if per_cell:
        mc = compute_material_components(mat, mtypes, g)
        apply_pec_plates(bricks, mtypes, mc, g)
        coeffs = compute_general_coefficients(mc, g)

        def eps_sig_at(axis, fi):
            c = "xyz"[axis]
            return mc[f"eps_r_{c}"].ravel()[fi], mc[f"sigma_e_{c}"].ravel()[fi]
    else:
        if int(mat.max()) >= props.shape[0]:
            raise ValueError("brick material_type exceeds the material types")
        mc, coeffs = {}, None

        def eps_sig_at(axis, fi):
            return e_values_at(axis, fi, mat, props, plates, g)
    faces = init_cpml(boundary, coeffs, g)
    waves = init_waveforms(scn.get("waveforms") or {}, nsteps, g.dt, ncpw, [dx, dy, dz])
    vsrc = init_voltage_sources(scn.get("voltageSources"), waves, eps_sig_at, coeffs, g)
    sv = init_sampled_voltages(scn.get("sampledVoltages"), g)
    si = init_sampled_currents(scn.get("sampledCurrents"), g)
    ffp = dict(DEFAULTS["farfield"], **(scn.get("farfield") or {}))
    freqs = np.array(ffp.get("frequencies") or [], dtype=np.float64)
    ff = None
    if freqs.size:
        nc = int(ffp["number_of_cells_from_outer_boundary"])
        ff = FarFieldBox(freqs, nc + 1, nc + 1, nc + 1, g.nx - nc + 1, g.ny - nc + 1, g.nz - nc + 1)
    return Problem(
        grid=g,
        coeffs={k: v.ravel() for k, v in coeffs.items()} if coeffs is not None else {},
        materials=mc,
        cpml=faces,
        voltage_sources=vsrc,
        sampled_voltages=sv,
        sampled_currents=si,
        farfield=ff,
        ports=scn.get("ports") or [],
        dft=dict(DEFAULTS["dft"], **(scn.get("dft") or {})),
        meta={"name": scn.get("name"), "description": scn.get("description"), "material_grid": mat,
              "material_props": props, "plates": plates},
    )
