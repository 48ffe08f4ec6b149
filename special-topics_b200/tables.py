"""Material-table form of a problem, for the FP32 fast path.

The reference stores 18 per-cell FP64 coefficient arrays (coefficients.js:22-116).
Every coefficient triple of a component is a function of the (eps_r, sigma_e)
or (mu_r, sigma_m) pair averaged at that component's location
(materials.js:87-238), except (a) the CPML kappa division, which depends only
on the position along one axis (cpml.js:212-243), and (b) the lumped-source
cells, whose triples are overridden (coefficients.js:158-207).  So each
component gets one uint8 id per cell into a table of distinct triples computed
without kappa; the kernel applies 1/kappa from 1-D profiles, and source cells
get rows of their own.  This turns 9 coefficient reads per half-step and cell
into 3 one-byte reads.
"""
from __future__ import annotations

import numpy as np

from .scenario import EPS0, MU0, Problem

MAX_ROWS = 256
# API component order of fdtd_ctx_upload_material: Ex Ey Ez Hx Hy Hz
COMPONENTS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
_PAIR = {"Ex": ("eps_r_x", "sigma_e_x"), "Ey": ("eps_r_y", "sigma_e_y"), "Ez": ("eps_r_z", "sigma_e_z"),
         "Hx": ("mu_r_x", "sigma_m_x"), "Hy": ("mu_r_y", "sigma_m_y"), "Hz": ("mu_r_z", "sigma_m_z")}
# coefficient names (self, curl1, curl2) per component, the kernel's curl order
CURLS = {"Ex": ("Cexe", "Cexhz", "Cexhy"), "Ey": ("Ceye", "Ceyhx", "Ceyhz"), "Ez": ("Ceze", "Cezhy", "Cezhx"),
         "Hx": ("Chxh", "Chxey", "Chxez"), "Hy": ("Chyh", "Chyez", "Chyex"), "Hz": ("Chzh", "Chzex", "Chzey")}


def _codes(a: np.ndarray):
    """(sorted distinct values, index of each element) for an array with few distinct values."""
    flat = a.ravel()
    step = max(1, flat.size // 200_000)
    vals = np.unique(flat[::step])
    idx = np.clip(np.searchsorted(vals, flat), 0, vals.size - 1)
    if not np.array_equal(vals[idx], flat):
        vals = np.unique(flat)
        idx = np.searchsorted(vals, flat)
    return vals, idx


def _rows(comp: str, e: np.ndarray, s: np.ndarray, dt: float, d: tuple) -> np.ndarray:
    """Coefficient triples for value pairs, as computeGeneralCoefficients evaluates them."""
    dx, dy, dz = d
    tdx, tdy, tdz = 2 * dt / dx, 2 * dt / dy, 2 * dt / dz
    scale = EPS0 if comp[0] == "E" else MU0
    a = 2 * e * scale
    b = dt * s
    denom = a + b
    num1, num2 = {"Ex": (tdy, -tdz), "Ey": (tdz, -tdx), "Ez": (tdx, -tdy),
                  "Hx": (tdz, -tdy), "Hy": (tdx, -tdz), "Hz": (tdy, -tdx)}[comp]
    return np.stack([(a - b) / denom, num1 / denom, num2 / denom], axis=1)


def build_tables(p: Problem) -> dict[str, tuple[np.ndarray, np.ndarray]]:
    """Returns {component: (uint8 ids flat, rows x 3 FP64 table)} in reference index order."""
    g = p.grid
    d = (g.dx, g.dy, g.dz)
    out = {}
    bands = []
    for f in p.cpml:
        if f is not None:
            bands.append((f.face, f.m_start, f.e_start, f.nc))
    for comp in COMPONENTS:
        e_name, s_name = _PAIR[comp]
        ev, ei = _codes(p.materials[e_name])
        sv, si = _codes(p.materials[s_name])
        key = ei.astype(np.int64) * sv.size + si
        present = np.zeros(ev.size * sv.size, dtype=bool)
        present[key] = True
        keys = np.nonzero(present)[0]
        remap = np.full(present.size, -1, dtype=np.int64)
        remap[keys] = np.arange(keys.size)
        ids = remap[key]
        table = _rows(comp, ev[keys // sv.size], sv[keys % sv.size], g.dt, d)
        # lumped-source cells carry their own coefficients
        for vs in p.voltage_sources:
            if "xyz"[vs.axis] != comp[1] or comp[0] != "E":
                continue
            check_source_outside_cpml(vs, p)
            uniq, inv = np.unique(vs.override, axis=0, return_inverse=True)
            ids[vs.field_indices] = table.shape[0] + inv.ravel()
            table = np.concatenate([table, uniq], axis=0)
        if table.shape[0] > MAX_ROWS:
            raise ValueError(f"{comp}: {table.shape[0]} distinct coefficient rows exceed {MAX_ROWS}")
        out[comp] = (ids.astype(np.uint8), np.ascontiguousarray(table))
    return out


def check_source_outside_cpml(vs, p: Problem) -> None:
    """Source rows carry no kappa, so a source cell must not sit in a CPML band."""
    g = p.grid
    i_s, j_s, k_s, i_e, j_e, k_e = vs.box
    lo = (i_s - 1, j_s - 1, k_s - 1)
    hi = (i_e - 1, j_e - 1, k_e - 1)
    for f in p.cpml:
        if f is None:
            continue
        axis = "xyz".index(f.face[0])
        for start in (f.m_start, f.e_start):
            if not (hi[axis] < start or lo[axis] >= start + f.nc):
                raise ValueError(f"voltage source overlaps the {f.face} CPML band")
    del g
