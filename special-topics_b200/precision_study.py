"""Precision study: FP32 fields against the FP64 path on the refined
inverted-F antenna (0.25 mm cells, far field at 64 frequencies in 1-4 GHz).

  python special-topics_b200/precision_study.py [--steps 20000] [--out metrics.json]

FP32 runs are made with FP64 far-field accumulators and with Kahan-compensated
FP32 ones.  All runs use the same problem.  The FP64 run is the drop-in path, bit
identical to the CPU oracle (tests/test_gpu_parity.py), so its results stand
in for the oracle's at this size.  Reported per FP32 variant:
  - S11: max |dB difference| over 301 points in 1-4 GHz
  - Zin: max relative complex difference over the same points
  - directivity: on a 2-degree theta/phi grid at each of the 64 frequencies,
    the difference of peak directivity (dBi), the difference at the FP64 peak
    direction, and the largest difference over directions within 10 dB of the
    peak (elsewhere the pattern's nulls make dB differences meaningless)
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import sys
import time

import numpy as np


def _package():
    name = "special_topics_b200"
    if name in sys.modules:
        return sys.modules[name]
    d = os.path.dirname(os.path.abspath(__file__))
    spec = importlib.util.spec_from_file_location(name, os.path.join(d, "__init__.py"), submodule_search_locations=[d])
    m = importlib.util.module_from_spec(spec)
    sys.modules[name] = m
    spec.loader.exec_module(m)
    return m


def grid_2deg():
    th = np.radians(np.arange(0, 181, 2.0))
    ph = np.radians(np.arange(0, 360, 2.0))
    T, P = np.meshgrid(th, ph, indexing="ij")
    return T.ravel(), P.ravel()


def run_one(problem, precision: str, steps: int, device: int = 0, acc: str = "f64", block: int = 0) -> dict:
    from special_topics_b200 import postproc
    from special_topics_b200.backend import Engine
    freqs = np.linspace(1e9, 4e9, 301)
    t0 = time.perf_counter()
    with Engine(problem, precision, device=device, dft_accumulator=acc, dft_block=block) as eng:
        ms = eng.run_timed(steps)
        V, I = eng.voltages()[0], eng.currents()[0]
        port = postproc.port_s11(V, I, problem.grid.dt, freqs, 50.0)
        T, P = grid_2deg()
        radp, dth, dph = eng.farfield_post(T, P)
    return {"device_ms": ms, "wall_s": time.perf_counter() - t0, "s11_db": port["mag_dB"], "zin": port["zin"],
            "radp": radp, "d": dth + dph, "growth_onset_step": postproc.growth_onset(V)}


def compare(ref: dict, other: dict) -> dict:
    to_db = lambda x: 10 * np.log10(np.maximum(x, 1e-30))
    zr = ref["zin"][0] + 1j * ref["zin"][1] if isinstance(ref["zin"], tuple) else np.asarray(ref["zin"])
    zo = other["zin"][0] + 1j * other["zin"][1] if isinstance(other["zin"], tuple) else np.asarray(other["zin"])
    dref, doth = to_db(ref["d"]), to_db(other["d"])
    peak_err = np.abs(dref.max(axis=1) - doth.max(axis=1))
    at_peak = np.abs(np.take_along_axis(doth - dref, dref.argmax(axis=1)[:, None], axis=1)[:, 0])
    main = dref >= dref.max(axis=1, keepdims=True) - 10.0
    lobe_err = np.array([np.abs(doth[f][main[f]] - dref[f][main[f]]).max() for f in range(dref.shape[0])])
    freqs = np.linspace(1e9, 4e9, dref.shape[0])
    per_f = {"freq_GHz": (freqs / 1e9).round(4).tolist(),
             "peak_directivity_abs_dB": peak_err.round(4).tolist(),
             "radp_rel": np.abs(other["radp"] / ref["radp"] - 1).round(5).tolist(),
             "radp_fp64": ref["radp"].tolist()}
    return {"per_frequency": per_f,
            "s11_max_abs_dB": float(np.abs(other["s11_db"] - ref["s11_db"]).max()),
            "zin_max_rel": float(np.abs(zo - zr).max() / np.abs(zr).max()),
            "radp_max_rel": float(np.abs(other["radp"] / ref["radp"] - 1).max()),
            "peak_directivity_max_abs_dB": float(peak_err.max()),
            "directivity_at_fp64_peak_max_abs_dB": float(at_peak.max()),
            "directivity_within_10dB_of_peak_max_abs_dB": float(lobe_err.max()),
            "peak_directivity_dBi_range": [float(dref.max(axis=1).min()), float(dref.max(axis=1).max())]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    _package()
    from special_topics_b200 import workloads
    from special_topics_b200.scenario import build_problem_from_scenario
    scn = workloads.ifa_config2(steps=args.steps)
    p64 = build_problem_from_scenario(scn, args.steps)
    g = p64.grid
    ref = run_one(p64, "f64", args.steps)
    out = {"workload": scn["name"], "grid": [g.nx, g.ny, g.nz], "steps": args.steps,
           "far_field_freqs": int(p64.farfield.nFreq), "directions": int(grid_2deg()[0].size),
           "f64": {"device_ms": ref["device_ms"], "growth_onset_step": ref["growth_onset_step"]}}
    p32 = build_problem_from_scenario(scn, args.steps, per_cell=False)
    for name, acc, block in (("f32-table, FP64 accumulators", "f64", 0),
                             ("f32-table, Kahan FP32 accumulators", "kahan-f32", 0),
                             ("f32-table, FP64 accumulators, DFT blocked by 16 steps", "f64", 16)):
        r32 = run_one(p32, "f32-table", args.steps, acc=acc, block=block)
        out[name] = dict(compare(ref, r32), device_ms=r32["device_ms"], growth_onset_step=r32["growth_onset_step"])
    # FP32 fields with the reference's per-cell coefficient arrays
    r32 = run_one(p64, "f32", args.steps)
    out["f32 per-cell, FP64 accumulators"] = dict(compare(ref, r32), device_ms=r32["device_ms"],
                                                  growth_onset_step=r32["growth_onset_step"])
    text = json.dumps(out, indent=1)
    print(text, flush=True)
    if args.out:
        with open(args.out, "w") as f:
            f.write(text)


if __name__ == "__main__":
    main()
