"""Benchmark of the FDTD time-step loop on B200 (one JSON line on rank 0).

Workload: the plain-method scaling box (vacuum, 32 seeded dielectric blocks,
PEC half-wave dipole with a 50-ohm gap source, 8-cell CPML, far-field DFT at
two frequencies), 512 x 512 x 640 cells by default, FP32 fields with
material-table coefficients.  One step = one full FDTD time step of that grid
(H half-step + magnetic CPML, port current, E half-step + electric CPML +
source, port voltage, running far-field DFT).  The metric is Gcell-updates/s
= cells x steps / device time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With N > 1 (under torchrun) every rank advances its own independent problem
(seed = 1 + rank; the instances share nothing), the time is the max over ranks
and the value is the whole-job aggregate.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "Gcell-updates/s & time-to-S11 at 0.1 dB: FP32/learned vs FP64 plain, 1 B200"
FALLBACK_HBM_GBS = 6650.0
NOMINAL_HBM_GBS = 8000.0   # nominal B200 HBM3e bandwidth (DGX figure)


def _package():
    name = "special_topics_b200"
    if name in sys.modules:
        return sys.modules[name]
    d = os.path.join(ROOT, "special-topics_b200")
    spec = importlib.util.spec_from_file_location(name, os.path.join(d, "__init__.py"), submodule_search_locations=[d])
    m = importlib.util.module_from_spec(spec)
    sys.modules[name] = m
    spec.loader.exec_module(m)
    return m


def hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def algorithmic_bytes(p, precision: str) -> dict:
    """Compulsory DRAM bytes of one H and one E launch: each own-field value read
    and written once, each other-field value read once, the per-cell coefficient
    data read once (3 one-byte ids, or 3 FP64 arrays), each Psi element read and
    written once (plus its CPsi for the per-cell layout)."""
    sh = p.grid.shapes
    nH = sum(int(np.prod(sh[c])) for c in ("Hx", "Hy", "Hz"))
    nE = sum(int(np.prod(sh[c])) for c in ("Ex", "Ey", "Ez"))
    psi_m = psi_e = 0
    for f in p.cpml:
        if f is None:
            continue
        n = _psi_sizes(p, f)
        psi_m += n[0] + n[1]
        psi_e += n[2] + n[3]
    # bytes per component value: field word, coefficient data, Psi traffic per Psi element
    w, coef, psi_w = {"f32-table": (4, 1, 8), "f32": (4, 12, 12), "f64": (8, 24, 24)}[precision]
    return {"h": nH * (2 * w + coef) + nE * w + psi_m * psi_w,
            "e": nE * (2 * w + coef) + nH * w + psi_e * psi_w}


def _psi_sizes(p, f):
    g = p.grid
    nx, ny, nz, nc = g.nx, g.ny, g.nz, f.nc
    a = "xyz".index(f.face[0])
    if a == 0:
        return [nc * (ny + 1) * nz, nc * ny * (nz + 1), nc * ny * (nz + 1), nc * (ny + 1) * nz]
    if a == 1:
        return [(nx + 1) * nc * nz, nx * nc * (nz + 1), (nx + 1) * nc * nz, nx * nc * (nz + 1)]
    return [(nx + 1) * ny * nc, nx * (ny + 1) * nc, nx * (ny + 1) * nc, (nx + 1) * ny * nc]


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=10)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        rows = [r.split(",") for r in (getattr(self, "out", "") or "").strip().splitlines() if r.strip()]
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def ncu_traffic(workload: str):
    """dram bytes per launch of the dominant kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", f"traffic_{workload}.txt")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


def _host_ram_ok(n, factor: float = 1.5) -> bool:
    """Whether the host can hold the oracle's FP64 fields and 18 per-cell
    coefficient arrays of an n-cell box (with `factor` headroom)."""
    need = 8 * 26 * int(np.prod(n))
    try:
        avail = next(int(l.split()[1]) * 1024 for l in open("/proc/meminfo") if l.startswith("MemAvailable"))
    except (OSError, StopIteration, ValueError):
        return False
    return avail > factor * need


def cpu_oracle_rate(n=(256, 256, 256), budget_s: float = 15.0, steps: int | None = None, warm: int = 5,
                    max_steps: int = 390, one_thread: bool = True) -> dict:
    """The CPU oracle (C restatement of the reference's FP64 loop, OpenMP over
    all host cores) on a bounded sample of the scaling-box workload: `steps`
    steps, or as many as fit `budget_s` (at most max_steps), after `warm`."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    _package()
    from special_topics_b200 import workloads
    total = warm + (steps or max_steps) + 3
    scn = workloads.scaling_box(n, seed=1, steps=total)
    threads = os.cpu_count() or 1
    t = time.perf_counter()
    o = oracle.Oracle(scn, total, threads=threads)
    setup_s = time.perf_counter() - t
    o.step(max(0, warm - 3))
    t = time.perf_counter()
    o.step(3)
    per = (time.perf_counter() - t) / 3
    k = steps or int(max(1, min(max_steps, budget_s / max(per, 1e-6))))
    t = time.perf_counter()
    o.step(k)
    dt = time.perf_counter() - t
    cells = o.nx * o.ny * o.nz
    del o
    one = None
    if one_thread:
        # the same sample on one thread, a few steps
        o1 = oracle.Oracle(scn, total, threads=1)
        o1.step(1)
        t = time.perf_counter()
        o1.step(2)
        one = cells * 2 / (time.perf_counter() - t) / 1e9
        del o1
    cpu = ""
    try:
        cpu = next(l.split(":", 1)[1].strip() for l in open("/proc/cpuinfo") if l.startswith("model name"))
    except (OSError, StopIteration):
        pass
    return {"value": cells * k / dt / 1e9, "unit": "Gcell-updates/s", "cores": threads, "kind": "port",
            "sample": f"scaling box {n[0]}x{n[1]}x{n[2]} ({cells} cells), {k} FP64 steps timed after {warm} warm-up steps",
            "ms_per_step": dt / k * 1e3, "setup_s": setup_s,
            "one_thread_value": one, "cpu_model": cpu}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=8)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--grid", default="512x512x640")
    ap.add_argument("--ncpml", type=int, default=8, help="CPML cells per face of the scaling box (0: PEC walls)")
    ap.add_argument("--precision", default="f32-table", choices=["f32-table", "f32", "f64"])
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 side measurement")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU oracle baseline")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end pass (profiling runs)")
    ap.add_argument("--no-tune", action="store_true", help="keep the default launch shape")
    ap.add_argument("--tiling", default=None, help="fixed launch shape chunk,rows,prefetch[,width] (skips the tuner)")
    ap.add_argument("--tune-steps", type=int, default=16, help="steps timed per autotuner candidate")
    ap.add_argument("--dft-block", type=int, default=16,
                    help="FP32 legs: time-blocked far-field DFT, steps per block (0: accumulate every step)")
    ap.add_argument("--batch-members", type=int, default=128, help="inverted-F variants in the batched sweep (0: skip)")
    ap.add_argument("--batch-steps", type=int, default=1000, help="timed steps of the batched sweep")
    ap.add_argument("--batch-tiling", default=None,
                    help="fixed batch shape chunk,rows,prefetch,group[,streams[,width[,per_launch]]] (skips the tuner)")
    ap.add_argument("--ttS11-members", dest="ttS11_members", type=int, default=64,
                    help="held-out variants of the time-to-S11 leg (0: skip)")
    ap.add_argument("--no-sweep", action="store_true", help="skip the 128^3..512x512x640 FP32/FP64 sweep")
    ap.add_argument("--no-config0", action="store_true", help="skip the 0.5 mm inverted-F antenna leg")
    ap.add_argument("--cpu-sweep", action="store_true",
                    help="only time the CPU oracle for 50 steps at each sweep size (long; needs about 40 GB RAM)")
    args = ap.parse_args()
    n = tuple(int(x) for x in args.grid.split("x"))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    workload = f"scaling-box-{args.grid}"
    # bytes one half-step kernel streams per cell (fields, coefficients or ids)
    half_step_bytes = int(np.prod(n)) * {"f32-table": 40, "f32": 72, "f64": 144}[args.precision]
    l2 = ("inputs larger than L2 (fields and ids >> 126 MB), no flush needed" if half_step_bytes > 4 * L2_BYTES else
          f"working set about {half_step_bytes / 2**20:.0f} MB per half-step against the 126 MB L2: partly "
          "L2-resident, not an HBM figure")
    config = {"workload": workload, "grid": list(n), "cells": int(np.prod(n)), "ncpml": args.ncpml,
              "far_field_freqs": 2, "l2": l2,
              "parallelism": f"{args.gpus} independent problem(s), one per GPU"}

    if args.cpu_sweep:
        if rank == 0:
            print(json.dumps({"cpu_sweep": [cpu_oracle_rate(g, steps=50, warm=2) for g in SWEEP_GRIDS]}), flush=True)
        return

    if args.impl == "reference":
        if rank != 0:
            return
        # the reference's FP64 CPU loop (the oracle) on this same grid when the
        # host holds its per-cell arrays, else on a 256^3 sample of the workload
        grid = n if _host_ram_ok(n) else (256, 256, 256)
        base = cpu_oracle_rate(grid, budget_s=20.0, max_steps=max(1, args.steps))
        line = {"metric": METRIC, "value": base["value"], "unit": "Gcell-updates/s", "impl": "reference",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": dict(config) if grid == n else dict(config, workload=f"scaling-box-{grid[0]}x{grid[1]}x{grid[2]}",
                                                                grid=list(grid), cells=int(np.prod(grid))),
                "cpu_baseline": base,
                "e2e": {"value": base["value"], "unit": "Gcell-updates/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    pkg = _package()
    from special_topics_b200 import workloads
    from special_topics_b200.backend import Engine
    from special_topics_b200.scenario import build_problem_from_scenario

    # batched-sweep members are built on host processes started before any GPU work
    # the sweep's members; with N ranks each takes its share (sharding.partition
    # on cells x steps, the same on every rank, so nothing is exchanged)
    variants = None
    if args.batch_members > 0:
        import multiprocessing as mp
        from special_topics_b200 import autotune as _at
        from special_topics_b200 import sharding
        vsteps = 2 * args.warmup + args.batch_steps + 16 + _at.batch_steps_needed(args.tune_steps)
        seeds = list(range(args.batch_members))
        if world > 1:
            seeds = [seeds[q] for q in sharding.partition(sharding.variant_costs(seeds, 7000, True), world)[rank]]
        with mp.get_context("spawn").Pool(max(1, min(16, (os.cpu_count() or 1) // world))) as pool:
            variants = variant_problems(seeds, max(7000, vsteps), pool, spread=True)

    K, W, P = args.steps, args.warmup, 16
    dft_block = args.dft_block if args.precision != "f64" else 0   # FP64 keeps the reference's per-step sums
    scn = workloads.scaling_box(n, seed=1 + rank, steps=K + W + P, ncpml=args.ncpml)
    t0 = time.perf_counter()
    prob = build_problem_from_scenario(scn, K + W + P, per_cell=(args.precision != "f32-table"))
    setup_s = time.perf_counter() - t0
    cells = prob.grid.cells

    # --- launch shape from the autotuner (timed on a scratch copy of the problem)
    from special_topics_b200 import autotune
    tuning = None
    if args.tiling:
        v = [int(x) for x in args.tiling.split(",")]
        tuning = {"chunk": v[0], "rows": v[1], "prefetch": v[2], "width": v[3] if len(v) > 3 else 32,
                  "ms_per_step": None}
    elif not args.no_tune:
        scratch = build_problem_from_scenario(workloads.scaling_box(n, seed=1 + rank, steps=3000, ncpml=args.ncpml), 3000,
                                              per_cell=(args.precision != "f32-table"))
        tuning = autotune.tune(scratch, args.precision, device=local, steps_per_candidate=args.tune_steps)
        del scratch

    # --- end to end through the C ABI with host buffers: upload + K steps + readback
    barrier()
    e2e = None
    t0 = time.perf_counter()
    if not args.no_e2e:
        eng = Engine(prob, args.precision, device=local, dft_block=dft_block)
        t_up = time.perf_counter()
        if tuning:
            autotune.set_tiling(eng, tuning["chunk"], tuning["rows"], tuning.get("prefetch", 1), tuning.get("width", 32))
        h2d = _uploaded_bytes(prob, args.precision)
        eng.run(K)
        t_run = time.perf_counter()
        V, I = eng.voltages(K), eng.currents(K)
        ff = eng.farfield()
        e2e_s = time.perf_counter() - t0
        e2e_parts = {"create_and_upload_s": t_up - t0, "run_s": t_run - t_up, "readback_s": e2e_s - (t_run - t0)}
        d2h = sum(v.nbytes for v in V + I) + sum(a[0].nbytes + a[1].nbytes for a in ff.values())
        eng.close()
        e2e_s = max_over_ranks(e2e_s)
        e2e = {"value": world * cells * K / e2e_s / 1e9, "unit": "Gcell-updates/s",
               "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": d2h / K,
               "note": "one step's share of a whole run through the C ABI: uploads from host buffers, "
                       "K steps, readback of port traces and far-field accumulators",
               "parts_rank0": e2e_parts}

    # --- device-timed run
    eng = Engine(prob, args.precision, device=local, dft_block=dft_block)
    if tuning:
        autotune.set_tiling(eng, tuning["chunk"], tuning["rows"], tuning.get("prefetch", 1), tuning.get("width", 32))
    eng.run(W)
    barrier()
    with ClockSampler(local) as clk:
        ms = eng.run_timed(K)
    barrier()
    ms = max_over_ranks(ms)
    kern = eng.profile_kernels(P)
    eng.close()
    value = world * cells * K / (ms / 1e3) / 1e9
    byts = algorithmic_bytes(prob, args.precision)
    dom = "e" if kern["e"] >= kern["h"] else "h"
    peak, peak_kind = hbm_peak()
    achieved = byts[dom] / (kern[dom] / 1e3) / 1e9
    traffic = ncu_traffic(workload)
    line = {
        "metric": METRIC, "value": value, "unit": "Gcell-updates/s", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if args.precision != "f64" else "f64",
        "data": "synthetic (seeded scaling-box scenario in the reference's JSON schema)",
        "config": config,
        "setup": {"precision": args.precision, "time_steps_in_problem": K + W + P,
                  "far_field_dft": f"time-blocked, {dft_block} steps per block" if dft_block else "every step",
                  "x_wall": "Ey, Ez at i = nx held at zero (FP32 default)" if args.precision != "f64"
                            else "the reference's reads at i = nx"},
        "roofline": {"bound": "hbm", "kernel": f"k_step_{dom}", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                     "frac_of_nominal_8TBs": achieved / NOMINAL_HBM_GBS,
                     "algorithmic_bytes_per_launch": byts[dom], "launch_ms": kern[dom],
                     "traffic": traffic},
        "kernel_ms": kern,
        "tiling": {k: tuning.get(k, 32 if k == "width" else None) for k in ("chunk", "rows", "prefetch", "width", "ms_per_step")}
                  if tuning else "default",
        "clocks": clk.summary(),
        "gpu_launches": (5 if dft_block else 4) * K,   # H, mid, E, epilogue (+ the DFT flush)
        "e2e": e2e,
        "setup_s": setup_s,
    }
    if variants is not None:
        if variants:
            bs = batched_side(variants, K=args.batch_steps, W=args.warmup, tune_steps=args.tune_steps,
                              dft_block=args.dft_block,
                              device=local, barrier=barrier, fixed=args.batch_tiling)
        else:                       # a rank with no members still takes the same collective steps
            bs = None
            barrier()
            barrier()
        if world > 1:
            # whole-sweep rate: all ranks' cells over the slowest rank's time
            ms = max_over_ranks(bs["ms_per_step"] * args.batch_steps if bs else 0.0)
            tot = _sum_over_ranks(float(bs["cells"] if bs else 0), dist, local)
            if bs:
                bs = dict(bs, value=tot * args.batch_steps / (ms / 1e3) / 1e9, cells=int(tot),
                          ms_per_step=ms / args.batch_steps, members=args.batch_members,
                          scaling="strong: the members are split over the ranks")
        if rank == 0 and bs:
            line["batched"] = bs
    if rank == 0 and world == 1 and not args.no_config0:
        try:
            line["config0"] = config0_side(device=local)
        except Exception as e:  # a side leg must not hide the main number
            line["config0"] = {"error": str(e)}
    if rank == 0 and world == 1 and not args.no_sweep:
        try:
            t64 = None
            if not args.no_fp64:
                line["fp64_plain"] = fp64_side(pkg)
                t64 = line["fp64_plain"]["tiling"]
            line["scaling_sweep"] = scaling_sweep_side(tuning, t64, device=local, dft_block=dft_block)
        except Exception as e:
            line["scaling_sweep"] = {"error": str(e)}
    if rank == 0 and world == 1 and args.ttS11_members > 0:
        try:
            line["time_to_s11"] = time_to_s11_side(args.ttS11_members, device=local, dft_block=args.dft_block)
        except Exception as e:  # this leg must not hide the main number
            line["time_to_s11"] = {"error": str(e)}
    if rank == 0 and world == 1 and not args.no_fp64 and "fp64_plain" not in line:
        line["fp64_plain"] = fp64_side(pkg)
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            line["cpu_baseline"] = cpu_oracle_rate()
        except Exception as e:  # the baseline must not hide the GPU number
            line["cpu_baseline"] = {"error": str(e)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def _uploaded_bytes(p, precision: str) -> int:
    b = 0
    if precision == "f32-table":
        b += p.meta["material_grid"].nbytes
    else:
        b += sum(a.nbytes for a in p.coeffs.values())
    for f in p.cpml:
        if f is not None:
            b += 6 * f.nc * 8 + (sum(c.nbytes for c in f.cpsi) if f.cpsi is not None else 0)
    for vs in p.voltage_sources:
        b += vs.field_indices.nbytes + vs.coef.nbytes + vs.voltage_per_e_field.nbytes
    return b


def _variant_problem(args):
    seed, steps, spread = args
    pkg = _package()
    from special_topics_b200 import workloads
    from special_topics_b200.scenario import build_problem_from_scenario
    return build_problem_from_scenario(workloads.ifa_variant(seed, steps=steps, spread=spread), steps,
                                      per_cell=False)


def variant_problems(seeds, steps: int, pool=None, spread: bool = False) -> list:
    """Inverted-F variants of the given seeds (workloads.ifa_variant): the
    batched sweep's members with spread=True (grids spanning 32x96x96 ..
    64x200x200), the time-to-S11 runs without."""
    _package()    # results unpickle into the package's classes
    jobs = [(int(s), steps, spread) for s in seeds]
    if pool is None:
        return [_variant_problem(j) for j in jobs]
    return pool.map(_variant_problem, jobs)


def _sum_over_ranks(x: float, dist, local: int) -> float:
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def _best_by_mode(table: list) -> dict:
    """Fastest tuned step time (ms) of the tile-list and member-kernel modes."""
    out = {}
    for name, pick in (("tile_list", lambda r: r.get("streams", 0) == 0 and r.get("per_launch", 0) == 0),
                       ("grouped", lambda r: r.get("streams", 0) == 0 and r.get("per_launch", 0) > 0),
                       ("member_kernels", lambda r: r.get("streams", 0) > 0)):
        rows = [r for r in table if pick(r)]
        if rows:
            b = min(rows, key=lambda r: r["ms_per_step"])
            out[name] = {k: b[k] for k in ("ms_per_step", "chunk", "rows", "prefetch", "group", "streams", "width",
                                           "per_launch") if k in b}
    return out


def batched_side(problems, K: int = 1000, W: int = 8, tune_steps: int = 16, device: int = 0,
                 barrier=lambda: None, fixed: str | None = None, dft_block: int = 0) -> dict:
    """The batched sweep (FP32 fields, material tables): every member advanced
    either by one set of four launches per step for the whole batch (tile-list
    mode) or by its own four kernels per step on worker streams inside one
    graph (member-kernel mode); mode and launch shape from the batch
    autotuner."""
    from special_topics_b200 import autotune
    from special_topics_b200.backend import Batch, Engine
    t0 = time.perf_counter()
    engs = [Engine(p, "f32-table", device=device, dft_block=dft_block) for p in problems]
    create_s = time.perf_counter() - t0
    try:
        with Batch(engs) as b:
            if fixed:
                v = [int(x) for x in fixed.split(",")]
                b.set_tiling(v[0], v[1], v[2], v[3], v[4] if len(v) > 4 else 0, v[5] if len(v) > 5 else 32,
                             v[6] if len(v) > 6 else 0)
                tuning = {"ms_per_step": None}
            else:
                tuning = autotune.tune_batch(b, steps_per_candidate=tune_steps)
            b.run(W)
            barrier()
            with ClockSampler(device) as clk:
                ms = b.run_timed(K)
            barrier()
            kern = b.profile_kernels(8)
            cells = b.cells
            tiling = b.tiling()
    finally:
        for e in engs:
            e.close()
    byts = {"h": 0, "e": 0}
    for p in problems:
        a = algorithmic_bytes(p, "f32-table")
        byts["h"] += a["h"]
        byts["e"] += a["e"]
    dom = "e" if kern["e"] >= kern["h"] else "h"
    peak, peak_kind = hbm_peak()
    if tiling.get("streams", 0) > 0:
        # member-kernel mode: the members' launches overlap on the worker
        # streams, so a launch timed alone says little; the roofline is the
        # whole step's H and E algorithmic bytes over the measured step time
        # (mid-step and epilogue time included, so conservative)
        roof_kernel = f"k_step_h + k_step_e of every member on {tiling['streams']} streams (whole step)"
        roof_bytes, roof_ms = byts["h"] + byts["e"], ms / K
    elif tiling.get("per_launch", 0) > 0:
        ngroups = -(-len(problems) // tiling["per_launch"])
        roof_kernel = (f"k_batch_group ({dom.upper()}): {ngroups} launches of {tiling['per_launch']} members "
                       "side by side, timed together")
        roof_bytes, roof_ms = byts[dom], kern[dom]
    else:
        roof_kernel = f"k_batch_half ({dom.upper()})"
        roof_bytes, roof_ms = byts[dom], kern[dom]
    ach = roof_bytes / (roof_ms / 1e3) / 1e9
    dims = [(p.grid.nx, p.grid.ny, p.grid.nz) for p in problems]
    span = np.array(dims)
    return {"workload": f"ifa-variants-{len(problems)} (grids drawn from 32x96x96 .. 64x200x200)",
            "members": len(problems), "cells": cells,
            "grid_span_per_axis": [[int(a), int(b)] for a, b in zip(span.min(0), span.max(0))],
            "far_field_dft": f"time-blocked, {dft_block} steps per block" if dft_block else "every step",
            "grid_min": list(min(dims, key=lambda d: d[0] * d[1] * d[2])),
            "grid_max": list(max(dims, key=lambda d: d[0] * d[1] * d[2])),
            "value": cells * K / (ms / 1e3) / 1e9, "unit": "Gcell-updates/s", "steps": K, "warmup": W,
            "ms_per_step": ms / K,
            "gpu_launches": K * ((5 if dft_block else 4) * len(problems) if tiling.get("streams", 0) else
                                 (3 if dft_block else 2) + 2 * (-(-len(problems) // tiling["per_launch"])
                                                                if tiling.get("per_launch", 0) else 1)),
            "kernel_ms": kern,
            "tiling": tiling, "tuning_ms_per_step": tuning["ms_per_step"],
            "tuning_best_ms_by_mode": _best_by_mode(tuning.get("table", [])),
            "roofline": {"bound": "hbm", "kernel": roof_kernel, "achieved": ach, "peak": peak,
                         "unit": "GB/s", "frac": ach / peak, "peak_kind": peak_kind,
                         "frac_of_nominal_8TBs": ach / NOMINAL_HBM_GBS,
                         "algorithmic_bytes": roof_bytes, "time_ms": roof_ms},
            "clocks": clk.summary(), "engine_create_s": create_s}


WEIGHTS = os.path.join(ROOT, "special-topics_b200", "weights", "es_ifa_variants.npz")


def time_to_s11_side(count: int, device: int = 0, dft_block: int = 0) -> dict:
    """Time-to-S11 on inverted-F variants that neither training (seeds 1000..)
    nor the choice of the stop rule's thresholds (seeds 10000..10255) saw
    (seeds 20000..): plain FP64 batched runs of all 7000 steps, plain FP32
    runs of all 7000 steps, and FP32 runs stopped early: StopPolicy.refined()
    with the refinement started from the trained network's modes ("learned"),
    the same rule started from the run's own pencil ("no_network"), and the
    pencils' agreement rule alone ("pencil_rule", StopPolicy.refined(vp=False)).
    Each time runs from the first step launch to S11 on the host (301 points,
    1-4 GHz), the stop rule's fits and inference included, engine set-up and
    the start of the fit pool excluded."""
    import multiprocessing as mp
    from special_topics_b200 import earlystop as ES
    from special_topics_b200.backend import Batch, Engine
    if not os.path.exists(WEIGHTS):
        return {"unavailable": "no trained weights in special-topics_b200/weights"}
    seeds = list(range(20000, 20000 + count))
    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        probs = variant_problems(seeds, 7000, pool)
    # the FP64 engines build their per-cell coefficients on the device from the
    # same material grids (bit-identical to the host-built arrays)
    probs64 = probs
    freqs = ES.S11_FREQS
    policy = ES.StopPolicy.refined()
    # the batch tuner's shape for the inverted-F variants: one x chunk per column, 16-wide blocks
    tiling = {"chunk": 64, "rows": 16, "prefetch": 1, "group": 0, "width": 16}
    net = ES.EsNet.load(WEIGHTS, max_batch=max(count, 1), device=device)
    # the refined rule's checkpoint fits run in a spawned process pool, started
    # (and its workers' imports done) before any timing
    ES.start_fit_pool()
    out = {"workload": f"ifa-variants-{count} (seeds {seeds[0]}..{seeds[-1]})", "steps": policy.n_total,
           "fit_workers": ES._FIT_WORKERS}
    engs = [Engine(p, "f64", device=device) for p in probs64]
    try:
        t0 = time.perf_counter()
        with Batch(engs) as b:
            b.set_shape(tiling)            # every method runs the same launch shape
            b.run(policy.n_total)
        ref = [ES.s11_db(e.voltages()[0], e.currents()[0], e.problem.grid.dt, freqs) for e in engs]
        out["plain_f64_s"] = time.perf_counter() - t0
    finally:
        for e in engs:
            e.close()
    engs = [Engine(p, "f32-table", device=device, dft_block=dft_block) for p in probs]
    try:
        t0 = time.perf_counter()
        with Batch(engs) as b:
            b.set_shape(tiling)
            b.run(policy.n_total)
        s11 = [ES.s11_db(e.voltages()[0], e.currents()[0], e.problem.grid.dt, freqs) for e in engs]
        t = time.perf_counter() - t0
    finally:
        for e in engs:
            e.close()
    err = np.array([np.abs(a - b).max() for a, b in zip(s11, ref)])
    out["plain_f32"] = {"time_s": t, "within_0p1_dB": float(np.mean(err <= 0.1)),
                        "max_err_dB_median": float(np.median(err)), "max_err_dB_worst": float(err.max())}
    for name, use, pol in (("learned", True, policy), ("no_network", False, policy),
                           ("pencil_rule", False, ES.StopPolicy.refined(vp=False))):
        engs = [Engine(p, "f32-table", device=device, dft_block=dft_block) for p in probs]
        try:
            t0 = time.perf_counter()
            res = ES.run_with_early_stop(engs, net, pol, tiling, use_network=use)
            s11 = [ES.s11_db(r["V"], r["I"], e.problem.grid.dt, freqs) for r, e in zip(res, engs)]
            t = time.perf_counter() - t0
        finally:
            for e in engs:
                e.close()
        err = np.array([np.abs(a - b).max() for a, b in zip(s11, ref)])
        winners = [r["winner"] for r in res]
        out[name] = {"time_s": t, "within_0p1_dB": float(np.mean(err <= 0.1)),
                     "mean_stop_step": float(np.mean([r["stopped_at"] for r in res])),
                     "max_err_dB_median": float(np.median(err)), "max_err_dB_worst": float(err.max()),
                     "winners": {w: winners.count(w) for w in sorted(set(winners))}}
    net.close()
    ES.stop_fit_pool()
    out["ratio_plain_f64_over_learned"] = out["plain_f64_s"] / out["learned"]["time_s"]
    out["ratio_plain_f64_over_no_network"] = out["plain_f64_s"] / out["no_network"]["time_s"]
    out["ratio_plain_f64_over_plain_f32"] = out["plain_f64_s"] / out["plain_f32"]["time_s"]
    out["ratio_plain_f64_over_pencil_rule"] = out["plain_f64_s"] / out["pencil_rule"]["time_s"]
    return out


SWEEP_GRIDS = ((128, 128, 128), (256, 256, 256), (384, 384, 384), (512, 512, 640))
L2_BYTES = 126 * 2**20


def _leg(p, precision: str, K: int, W: int, tiling: dict | None, device: int = 0, dft_block: int = 0) -> dict:
    """One device-timed run: K steps after W warm-up steps, Gcell/s and the
    dominant step kernel against the HBM roofline."""
    from special_topics_b200 import autotune
    from special_topics_b200.backend import Engine
    with Engine(p, precision, device=device, dft_block=dft_block) as eng:
        if tiling:
            autotune.set_tiling(eng, tiling["chunk"], tiling["rows"], tiling.get("prefetch", 1), tiling.get("width", 32))
        eng.run(W)
        ms = eng.run_timed(K)
        kern = eng.profile_kernels(8)
    byts = algorithmic_bytes(p, precision)
    peak, peak_kind = hbm_peak()
    dom = "e" if kern["e"] >= kern["h"] else "h"
    ach = byts[dom] / (kern[dom] / 1e3) / 1e9
    return {"precision": precision, "value": p.grid.cells * K / (ms / 1e3) / 1e9, "unit": "Gcell-updates/s",
            "steps": K, "ms_per_step": ms / K, "kernel_ms": kern,
            "roofline": {"kernel": f"k_step_{dom}", "achieved": ach, "peak": peak, "peak_kind": peak_kind,
                         "frac": ach / peak, "algorithmic_bytes_per_launch": byts[dom]}}


def scaling_sweep_side(tiling32: dict | None, tiling64: dict | None, device: int = 0, dft_block: int = 0,
                       grids=SWEEP_GRIDS) -> list:
    """The scaling boxes (128^3, 256^3, 384^3, 512x512x640; 32 dielectric
    blocks and a dipole) at every size in FP32 material tables and FP64 (per-cell
    coefficients built on the device, bit-identical to the host-built ones).
    About 2 G cell-updates are timed per leg (at least 20 steps).  Grids whose
    FP32 working set fits the 126 MB L2 are marked L2-resident: their rate is
    not an HBM figure."""
    from special_topics_b200 import workloads
    from special_topics_b200.scenario import build_problem_from_scenario
    out = []
    for n in grids:
        cells = n[0] * n[1] * n[2]
        K = int(min(1000, max(20, 2e9 // cells)))
        W = 68                      # the 64-step graph is captured and warmed before the timed steps
        p = build_problem_from_scenario(workloads.scaling_box(n, seed=1, steps=K + W + 8), K + W + 8, per_cell=False)
        for prec, tiling in (("f32-table", tiling32), ("f64", tiling64)):
            leg = _leg(p, prec, K, W, tiling, device, dft_block if prec != "f64" else 0)
            work = algorithmic_bytes(p, prec)
            leg.update({"grid": list(n), "cells": cells,
                        "l2_resident": bool(work["e"] < L2_BYTES),
                        "tiling": {k: tiling.get(k) for k in ("chunk", "rows", "prefetch", "width")} if tiling else "default"})
            out.append(leg)
        del p
    return out


def config0_side(device: int = 0, oracle_steps: int = 1000) -> dict:
    """The FP64 parity scenario: the 0.5 mm inverted-F antenna (39 x 136
    x 136, 7000 steps, far field at 2.4 GHz).  Device-timed FP64 (the drop-in)
    and FP32-table runs of the whole 7000 steps; time-to-S11 (301 points,
    1-4 GHz) from the first step launch to S11 on the host for each; the CPU
    oracle on the box's cores for `oracle_steps` steps of the same scenario
    (extrapolated to 7000, stated), whose traces must equal the FP64 run's
    first steps bit for bit."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from special_topics_b200 import earlystop as ES
    from special_topics_b200 import workloads
    from special_topics_b200.backend import Engine
    from special_topics_b200.scenario import build_problem_from_scenario
    steps = 7000
    scn = workloads.ifa_config0(steps)
    p64 = build_problem_from_scenario(scn, steps)
    p32 = build_problem_from_scenario(scn, steps, per_cell=False)
    cells = p64.grid.cells
    out = {"workload": scn["name"], "grid": [p64.grid.nx, p64.grid.ny, p64.grid.nz], "cells": cells, "steps": steps,
           "l2_resident": True}
    s11 = {}
    for name, prob, prec in (("f64", p64, "f64"), ("f32_table", p32, "f32-table")):
        with Engine(prob, prec, device=device) as eng:
            start = eng.save_state()        # step 0
            eng.run(64)                     # captures and warms the step graph
            eng.load_state(start)           # back to step 0: the timed run is the whole run
            t0 = time.perf_counter()
            ms = eng.run_timed(steps)
            V, I = eng.voltages()[0], eng.currents()[0]
            s11[name] = ES.s11_db(V, I, prob.grid.dt, ES.S11_FREQS)
            tt = time.perf_counter() - t0
            if name == "f64":
                v64 = V
        out[name] = {"value": cells * steps / (ms / 1e3) / 1e9, "unit": "Gcell-updates/s", "device_ms": ms,
                     "time_to_s11_s": tt}
    out["f32_table"]["s11_max_abs_dB_vs_f64"] = float(np.abs(s11["f32_table"] - s11["f64"]).max())
    out["time_to_s11_ratio_f64_over_f32_table"] = out["f64"]["time_to_s11_s"] / out["f32_table"]["time_to_s11_s"]
    threads = os.cpu_count() or 1
    o = oracle.Oracle(scn, steps, threads=threads)
    t0 = time.perf_counter()
    o.step(oracle_steps)
    dt = time.perf_counter() - t0
    same = bool(np.array_equal(o.get("V:0")[:oracle_steps], v64[:oracle_steps]))
    del o
    out["cpu_oracle"] = {"value": cells * oracle_steps / dt / 1e9, "unit": "Gcell-updates/s", "cores": threads,
                         "kind": "port", "steps_timed": oracle_steps, "s_per_7000_steps_extrapolated": dt * steps / oracle_steps,
                         "v_trace_bit_identical_to_gpu_f64": same}
    out["time_to_s11_ratio_cpu_oracle_over_f64"] = out["cpu_oracle"]["s_per_7000_steps_extrapolated"] / out["f64"]["time_to_s11_s"]
    return out


def fp64_side(pkg, n=(256, 256, 256), K: int = 300, W: int = 8) -> dict:
    """The FP64 drop-in path (reference coefficient layout) on a 256^3 box."""
    from special_topics_b200 import workloads
    from special_topics_b200.backend import Engine
    from special_topics_b200.scenario import build_problem_from_scenario
    from special_topics_b200 import autotune
    p = build_problem_from_scenario(workloads.scaling_box(n, seed=1, steps=1000), 1000)
    tuning = autotune.tune(p, "f64", steps_per_candidate=8)
    eng = Engine(p, "f64")
    autotune.set_tiling(eng, tuning["chunk"], tuning["rows"], tuning.get("prefetch", 1), tuning.get("width", 32))
    eng.run(W)
    ms = eng.run_timed(K)
    kern = eng.profile_kernels(8)
    eng.close()
    byts = algorithmic_bytes(p, "f64")
    peak, _ = hbm_peak()
    dom = "e" if kern["e"] >= kern["h"] else "h"
    ach = byts[dom] / (kern[dom] / 1e3) / 1e9
    return {"workload": f"scaling-box-{n[0]}x{n[1]}x{n[2]}", "value": p.grid.cells * K / (ms / 1e3) / 1e9,
            "unit": "Gcell-updates/s", "ms_per_step": ms / K, "tiling": {k: tuning[k] for k in ("chunk", "rows", "prefetch")},
            "roofline": {"kernel": f"k_step_{dom}", "achieved": ach, "peak": peak, "frac": ach / peak}}


if __name__ == "__main__":
    main()
