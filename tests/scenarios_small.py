"""Small seeded scenarios in the reference's JSON schema, for parity tests that
the CPU oracle finishes in seconds.  Each exercises zero-thickness PEC plates,
dielectric bricks, a lumped source, a voltage and a current probe and the
far-field box, with uneven CPML widths per face."""
import numpy as np


def _brick(x0, y0, z0, x1, y1, z1, t):
    return {"min_x": x0, "min_y": y0, "min_z": z0, "max_x": x1, "max_y": y1, "max_z": z1, "material_type": t}


def small_scenario(seed: int = 0, direction: str = "xp", ncpml=(4, 5, 3, 6, 4, 3), steps: int = 60,
                   nff: int = 2) -> dict:
    rng = np.random.default_rng(seed)
    d = 1e-3
    bricks = [_brick(0, 0, 0, 8 * d, 10 * d, 12 * d, 4)]          # dielectric block defines the box
    for _ in range(3):
        lo = rng.integers(0, 6, 3)
        hi = lo + rng.integers(1, 5, 3)
        bricks.append(_brick(lo[0] * d, lo[1] * d, lo[2] * d, hi[0] * d, hi[1] * d, hi[2] * d,
                             int(rng.integers(3, 6))))
    # PEC plates: one zero-thickness in each axis
    bricks.append(_brick(2 * d, 1 * d, 2 * d, 2 * d, 7 * d, 9 * d, 2))
    bricks.append(_brick(1 * d, 3 * d, 1 * d, 6 * d, 3 * d, 8 * d, 2))
    bricks.append(_brick(3 * d, 2 * d, 5 * d, 7 * d, 8 * d, 5 * d, 2))
    axis = "xyz".index(direction[0])
    lo = [4 * d, 5 * d, 6 * d]
    hi = list(lo)
    hi[axis] += 2 * d
    other = [a for a in range(3) if a != axis]
    hi[other[0]] += 1 * d
    src = {"min_x": lo[0], "min_y": lo[1], "min_z": lo[2], "max_x": hi[0], "max_y": hi[1], "max_z": hi[2],
           "direction": direction, "resistance": 50, "magnitude": 1, "waveform_type": "gaussian",
           "waveform_index": 1}
    vprobe = dict(src)
    for k in ("resistance", "magnitude", "waveform_type", "waveform_index"):
        vprobe.pop(k)
    iprobe = {"min_x": lo[0], "min_y": lo[1], "min_z": lo[2], "max_x": hi[0], "max_y": hi[1], "max_z": hi[2],
              "direction": direction}
    mid = (lo[axis] + hi[axis]) / 2
    for key in ("min_", "max_"):
        iprobe[key + "xyz"[axis]] = mid
    names = ("xn", "xp", "yn", "yp", "zn", "zp")
    boundary = {}
    for n, c in zip(names, ncpml):
        boundary[f"type_{n}"] = "cpml"
        boundary[f"air_buffer_{n}"] = 3
        boundary[f"cpml_cells_{n}"] = c
    boundary.update({"cpml_order": 3, "cpml_sigma_factor": 1.3, "cpml_kappa_max": 7,
                     "cpml_alpha_min": 0, "cpml_alpha_max": 0.05})
    return {
        "name": f"small-{seed}-{direction}", "numberOfTimeSteps": steps, "courantFactor": 0.9,
        "numberOfCellsPerWavelength": 20, "cell": {"dx": d, "dy": d, "dz": d},
        "boundary": boundary,
        "materialTypes": [{"eps_r": 1, "mu_r": 1, "sigma_e": 0, "sigma_m": 0},
                          {"eps_r": 1, "mu_r": 1, "sigma_e": 1e10, "sigma_m": 0},
                          {"eps_r": 2.2, "mu_r": 1, "sigma_e": 0, "sigma_m": 0},
                          {"eps_r": 4.4, "mu_r": 1, "sigma_e": 0.01, "sigma_m": 0},
                          {"eps_r": 3.0, "mu_r": 2.0, "sigma_e": 0, "sigma_m": 0}],
        "bricks": bricks,
        "waveforms": {"gaussian": [{"number_of_cells_per_wavelength": 12}]},
        "voltageSources": [src], "sampledVoltages": [vprobe], "sampledCurrents": [iprobe],
        "ports": [{"sampled_voltage_index": 1, "sampled_current_index": 1, "impedance": 50, "is_source_port": True}],
        "farfield": {"frequencies": [5e9, 9e9][:nff], "number_of_cells_from_outer_boundary": 3},
        "dft": {"maxFreq": 20e9, "step": 1e9},
    }
