"""Scenario generators for the benchmark workloads, in the reference's JSON
schema (js_fdtd/scenarios/*.json, read by scenario.py like scenario.js reads it).

  ifa_config0()      inverted-F antenna on 0.5 mm cubic cells: FR4 slab (eps_r 4.4,
                     1.5 mm = 3 cells), partial PEC ground plane, zero-thickness PEC
                     trace with a 30 mm arm and a shorting stub 5 mm from the feed,
                     50-ohm lumped Gaussian source to 6 GHz (100 cells per
                     wavelength), 8-cell CPML, Courant 0.9, far field at 2.4 GHz;
                     the grid comes out 39 x 136 x 136 like the reference's IFA.
  ifa_config2()      the same antenna on 0.25 mm cells (78 x 272 x 272: air and
                     CPML cell counts doubled), 64 far-field frequencies in 1-4 GHz.
  scaling_box(n)     vacuum box of n = (nx, ny, nz) cells (CPML included) holding
                     32 seeded dielectric blocks (eps_r U[1,10], edges U[4,32]
                     cells) and a PEC half-wave dipole with a 50-ohm gap source,
                     1 mm cells, 8-cell CPML.
  ifa_variant(seed)  one member of the batched sweep: arm U[20,35] mm, stub-to-feed
                     U[2,8] mm, substrate eps_r U[2.2,6.15], thickness U[0.8,3.2] mm;
                     spread=True pads it with air to grid extents drawn from
                     32x96x96 .. 64x200x200.

All inputs are synthetic; nothing here is data from the reference.
"""
from __future__ import annotations

import numpy as np

MM = 1e-3


def _boundary(ncpml: int, air: int) -> dict:
    """CPML of `ncpml` cells on every face; ncpml = 0 gives PEC walls."""
    b = {}
    for f in ("xn", "xp", "yn", "yp", "zn", "zp"):
        b[f"type_{f}"] = "cpml" if ncpml > 0 else "pec"
        b[f"air_buffer_{f}"] = air
        b[f"cpml_cells_{f}"] = ncpml
    b.update({"cpml_order": 3, "cpml_sigma_factor": 1.3, "cpml_kappa_max": 7,
              "cpml_alpha_min": 0, "cpml_alpha_max": 0.05})
    return b


def _brick(lo, hi, t):
    return {"min_x": lo[0], "min_y": lo[1], "min_z": lo[2], "max_x": hi[0], "max_y": hi[1], "max_z": hi[2],
            "material_type": t}


def _ifa(cell: float, h: float, eps_r: float, arm: float, stub: float, board=(50 * MM, 50 * MM),
         ground_len: float = 20 * MM, width: float = 2 * MM, air: int = 10, ncpml: int = 8,
         ncpw: int = 100, steps: int = 7000, freqs=(2.4e9,), name: str = "ifa") -> dict:
    """Inverted-F antenna on a substrate of thickness h (x), board in (y, z).

    Ground plane: x = -h plane for y in [0, ground_len].  Feed: strip on x = 0
    along y from the board edge (y = 0) to the arm; the source spans the slab
    at y = 0 under it.  Arm: strip along z at y in [ground_len + 2w, ...].
    Shorting stub: strip on x = 0 from the arm down to the ground edge plus a
    via through the slab at y = ground_len, `stub` away from the feed.
    """
    Ly, Lz = board
    w = width
    zf = round(0.3 * Lz / cell) * cell          # feed strip z start
    ya = ground_len + 2 * w                      # arm y start
    zs = zf + round(stub / cell) * cell          # stub z start
    bricks = [
        _brick((-h, 0, 0), (0, Ly, Lz), 3),                          # substrate
        _brick((-h, 0, 0), (-h, ground_len, Lz), 2),                 # ground plane
        _brick((0, 0, zf), (0, ya + w, zf + w), 2),                  # feed line
        _brick((0, ya, zf), (0, ya + w, zf + arm), 2),               # arm
        _brick((0, ground_len, zs), (0, ya + w, zs + w), 2),         # stub (top)
        _brick((-h, ground_len, zs), (0, ground_len, zs + w), 2),    # stub via through the slab
    ]
    src = {"min_x": -h, "min_y": 0, "min_z": zf, "max_x": 0, "max_y": 0, "max_z": zf + w,
           "direction": "xp", "resistance": 50, "magnitude": 1, "waveform_type": "gaussian", "waveform_index": 1}
    vprobe = {k: src[k] for k in ("min_x", "min_y", "min_z", "max_x", "max_y", "max_z", "direction")}
    mid = round(-h / 2 / cell) * cell
    iprobe = {"min_x": mid, "min_y": 0, "min_z": zf, "max_x": mid, "max_y": cell, "max_z": zf + w,
              "direction": "xp"}
    return {
        "name": name, "numberOfTimeSteps": steps, "courantFactor": 0.9, "numberOfCellsPerWavelength": 20,
        "cell": {"dx": cell, "dy": cell, "dz": cell}, "boundary": _boundary(ncpml, air),
        "materialTypes": [{"eps_r": 1, "mu_r": 1, "sigma_e": 0, "sigma_m": 0},
                          {"eps_r": 1, "mu_r": 1, "sigma_e": 1e10, "sigma_m": 0},
                          {"eps_r": eps_r, "mu_r": 1, "sigma_e": 0, "sigma_m": 0}],
        "bricks": bricks, "spheres": [],
        "waveforms": {"gaussian": [{"number_of_cells_per_wavelength": ncpw}]},
        "voltageSources": [src], "sampledVoltages": [vprobe], "sampledCurrents": [iprobe],
        "ports": [{"sampled_voltage_index": 1, "sampled_current_index": 1, "impedance": 50,
                   "is_source_port": True}],
        "farfield": {"frequencies": list(freqs), "number_of_cells_from_outer_boundary": 13},
        "dft": {"maxFreq": 10e9, "step": 20e6},
    }


def ifa_config0(steps: int = 7000) -> dict:
    return _ifa(0.5 * MM, 1.5 * MM, 4.4, 30 * MM, 5 * MM, steps=steps, name="ifa-config0-0p5mm")


def ifa_config2(steps: int = 20000) -> dict:
    s = _ifa(0.25 * MM, 1.5 * MM, 4.4, 30 * MM, 5 * MM, air=20, ncpml=16, ncpw=200, steps=steps,
             freqs=tuple(np.linspace(1e9, 4e9, 64)), name="ifa-config2-0p25mm")
    s["farfield"]["number_of_cells_from_outer_boundary"] = 26
    return s


VARIANT_SPAN = ((32, 64), (96, 200), (96, 200))   # grid extents of the batched sweep, cells
SPREAD_MIN_AIR = 6                                 # air cells per face of a spread variant, at least


def ifa_variant(seed: int, steps: int = 7000, spread: bool = False) -> dict:
    """A batched-sweep member on 0.5 mm cells with 8-cell CPML.  The antenna
    alone (10 air cells per face) gives grids of 39x117x107 .. 42x146x136.
    spread=True keeps the same antenna and draws the grid's extent along each
    axis uniformly from VARIANT_SPAN (a second random stream of the seed;
    never below the antenna plus SPREAD_MIN_AIR air cells per face), padding
    with air: the members then span 32x96x96 .. 64x200x200 as far as the
    antennas fit."""
    rng = np.random.default_rng(seed)
    arm = rng.uniform(20, 35) * MM
    stub = rng.uniform(2, 8) * MM
    eps = rng.uniform(2.2, 6.15)
    h = rng.uniform(0.8, 3.2) * MM
    cell = 0.5 * MM
    hc = max(1, round(h / cell)) * cell
    board = (round((arm + 20 * MM) / cell) * cell, round((arm + 15 * MM) / cell) * cell)
    scn = _ifa(cell, hc, eps, round(arm / cell) * cell, stub, board=board, steps=steps, ncpw=60,
               name=f"ifa-variant-{seed}")
    if spread:
        ncpml = scn["boundary"]["cpml_cells_xn"]
        body = (round(hc / cell), round(board[0] / cell), round(board[1] / cell))   # the bricks' extent, cells
        grng = np.random.default_rng([seed, 1])
        for ax, n0, (lo, hi) in zip("xyz", body, VARIANT_SPAN):
            least = n0 + 2 * (ncpml + SPREAD_MIN_AIR)
            n = max(int(grng.integers(lo, hi + 1)), least)
            air = n - n0 - 2 * ncpml
            scn["boundary"][f"air_buffer_{ax}n"] = air // 2
            scn["boundary"][f"air_buffer_{ax}p"] = air - air // 2
        scn["name"] = f"ifa-variant-spread-{seed}"
    return scn


def scaling_box(n=(128, 128, 128), seed: int = 1, cell: float = 1 * MM, ncpml: int = 8, air: int = 4,
                steps: int = 2000, nblocks: int = 32, freqs=(1.0e9, 2.0e9)) -> dict:
    """Vacuum box of exactly n cells (CPML and air buffer included)."""
    off = ncpml + air
    inner = [a - 2 * off for a in n]
    if min(inner) < 40:
        raise ValueError("box too small for the dipole and blocks")
    rng = np.random.default_rng(seed)
    mats = [{"eps_r": 1, "mu_r": 1, "sigma_e": 0, "sigma_m": 0},
            {"eps_r": 1, "mu_r": 1, "sigma_e": 1e10, "sigma_m": 0}]
    bricks = [_brick((0, 0, 0), [a * cell for a in inner], 1)]      # the vacuum box sets the extent
    for b in range(nblocks):
        edge = rng.integers(4, 33, 3)
        lo = [int(rng.integers(0, inner[a] - edge[a])) for a in range(3)]
        mats.append({"eps_r": float(rng.uniform(1, 10)), "mu_r": 1, "sigma_e": 0, "sigma_m": 0})
        bricks.append(_brick([lo[a] * cell for a in range(3)], [(lo[a] + edge[a]) * cell for a in range(3)],
                             len(mats)))
    # PEC half-wave dipole along z: two strips on the x = xc plane, one cell wide, one-cell gap
    ic, jc, kc = (inner[0] // 2, inner[1] // 2, inner[2] // 2)
    half = int(0.2 * inner[2])
    xc, yc, zg = ic * cell, jc * cell, kc * cell
    bricks.append(_brick((xc, yc, zg - half * cell), (xc, yc + cell, zg), 2))
    bricks.append(_brick((xc, yc, zg + cell), (xc, yc + cell, zg + (half + 1) * cell), 2))
    src = {"min_x": xc, "min_y": yc, "min_z": zg, "max_x": xc, "max_y": yc + cell, "max_z": zg + cell,
           "direction": "zp", "resistance": 50, "magnitude": 1, "waveform_type": "gaussian", "waveform_index": 1}
    vprobe = {k: src[k] for k in ("min_x", "min_y", "min_z", "max_x", "max_y", "max_z", "direction")}
    iprobe = {"min_x": xc, "min_y": yc, "min_z": zg, "max_x": xc + cell, "max_y": yc + 2 * cell,
              "max_z": zg + cell, "direction": "zp"}
    return {
        "name": f"scaling-box-{n[0]}x{n[1]}x{n[2]}-seed{seed}", "numberOfTimeSteps": steps,
        "courantFactor": 0.9, "numberOfCellsPerWavelength": 20,
        "cell": {"dx": cell, "dy": cell, "dz": cell}, "boundary": _boundary(ncpml, air),
        "materialTypes": mats, "bricks": bricks, "spheres": [],
        "waveforms": {"gaussian": [{"number_of_cells_per_wavelength": 20}]},
        "voltageSources": [src], "sampledVoltages": [vprobe], "sampledCurrents": [iprobe],
        "ports": [{"sampled_voltage_index": 1, "sampled_current_index": 1, "impedance": 50,
                   "is_source_port": True}],
        "farfield": {"frequencies": list(freqs), "number_of_cells_from_outer_boundary": 10},
        "dft": {"maxFreq": 6e9, "step": 20e6},
    }
