"""Launch-shape autotuner for the step kernels.

Every launch shape computes the same values.  For a problem, the tuner times
the candidate shapes (x planes per thread x thread rows per block) on a
scratch copy of the problem, so the caller's engine state is untouched, and
keeps the fastest.  Results are cached per (precision, nx, ny, nz) in a JSON
file next to the built library.
"""
from __future__ import annotations

import ctypes as C
import json
import os

from . import _native as N

CACHE = os.path.join(N.BUILD_DIR, "tiling_cache.json")
CHUNKS = (1, 2, 4, 8, 16, 32, 64)
ROWS = (2, 4, 8)
PREFETCH = (1, 2)
TABLE_PREFETCH = (1, 2, 3, 4)   # 3, 4: shared-memory stages, material-table problems only


def prefetch_depths(precision: str) -> tuple:
    return TABLE_PREFETCH if precision == "f32-table" else PREFETCH


def _key(problem, precision: str) -> str:
    g = problem.grid
    return f"{precision}:{g.nx}x{g.ny}x{g.nz}"


def _load() -> dict:
    try:
        with open(CACHE) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def get_tiling(engine) -> tuple[int, int]:
    a, b = C.c_int(), C.c_int()
    N.check(N.lib().fdtd_ctx_get_tiling(engine._h, C.byref(a), C.byref(b)))
    return a.value, b.value


def set_tiling(engine, chunk: int, rows: int, prefetch: int = 1, width: int = 32) -> None:
    N.check(N.lib().fdtd_ctx_set_tiling(engine._h, int(chunk), int(rows)))
    N.check(N.lib().fdtd_ctx_set_prefetch(engine._h, int(prefetch)))
    N.check(N.lib().fdtd_ctx_set_block_width(engine._h, int(width)))


# 16-wide blocks (a warp spans two rows) are tried at the best 32-wide
# (chunk, prefetch) with these row counts
NARROW_ROWS = (2, 4, 8, 16)


def tune(problem, precision: str, device: int = 0, steps_per_candidate: int = 64, use_cache: bool = True) -> dict:
    """Returns {"chunk", "rows", "ms_per_step", "table"} for the problem's grid."""
    from .backend import Engine
    key = _key(problem, precision)
    cache = _load()
    if use_cache and key in cache:
        return cache[key]
    depths = prefetch_depths(precision)
    need = 2 * steps_per_candidate * (len(CHUNKS) * len(ROWS) * len(depths) + len(NARROW_ROWS)) + 8
    if problem.grid.numberOfTimeSteps < need:
        raise ValueError(f"the scratch problem needs at least {need} time steps for tuning")
    nx = problem.grid.nx
    table = []
    with Engine(problem, precision, device=device) as eng:
        eng.run(4)
        for chunk in CHUNKS:
            if chunk > nx + 1:
                continue
            for rows in ROWS:
                for pf in depths:
                    set_tiling(eng, chunk, rows, pf)
                    eng.run_timed(steps_per_candidate)          # capture and warm the graph
                    ms = eng.run_timed(steps_per_candidate) / steps_per_candidate
                    table.append({"chunk": chunk, "rows": rows, "prefetch": pf, "width": 32, "ms_per_step": ms})
        best = min(table, key=lambda r: r["ms_per_step"])
        for rows in NARROW_ROWS:
            set_tiling(eng, best["chunk"], rows, best["prefetch"], 16)
            eng.run_timed(steps_per_candidate)
            ms = eng.run_timed(steps_per_candidate) / steps_per_candidate
            table.append({"chunk": best["chunk"], "rows": rows, "prefetch": best["prefetch"], "width": 16,
                          "ms_per_step": ms})
    best = min(table, key=lambda r: r["ms_per_step"])
    out = {"chunk": best["chunk"], "rows": best["rows"], "prefetch": best["prefetch"], "width": best["width"],
           "ms_per_step": best["ms_per_step"], "table": table}
    cache[key] = out
    os.makedirs(os.path.dirname(CACHE), exist_ok=True)
    with open(CACHE, "w") as f:
        json.dump(cache, f, indent=1)
    return out


BATCH_CHUNKS = (2, 4, 8, 16, 32, 64)   # 64 is cut to the members' depth: one x chunk per column
BATCH_GROUPS = (0, 1, 2, 4, 8, 16)
# member-kernel mode: worker stream counts and member launch shapes tried
BATCH_STREAMS = (2, 3, 4, 6, 8, 16)
MEMBER_SHAPES = ((32, 4, 1), (16, 4, 1), (32, 8, 1), (64, 4, 1))
MEMBER_STEPS = 64   # member-kernel trials time whole graphs of this many steps
# grouped mode: members per launch, then launch shapes (rows, width, prefetch) at the best count
PER_LAUNCH = (8, 11, 16, 22)
GROUPED_SHAPES = ((2, 32), (4, 32), (8, 32), (8, 16), (16, 16))   # at most 256 threads a block


def batch_key(batch) -> str:
    """Grid class of a batch: precision, member count and the member grid
    extents rounded up to multiples of 16 cells."""
    dims = sorted(tuple(-(-d // 16) * 16 for d in (e.problem.grid.nx, e.problem.grid.ny, e.problem.grid.nz))
                  for e in batch.engines)
    lo, hi = dims[0], dims[-1]
    return f"batch:{batch.engines[0].precision}:{len(dims)}:{lo[0]}x{lo[1]}x{lo[2]}-{hi[0]}x{hi[1]}x{hi[2]}"


def batch_steps_needed(steps_per_candidate: int, precision: str = "f32-table") -> int:
    tile_mode = 2 * steps_per_candidate * (len(BATCH_CHUNKS) * len(ROWS) * len(prefetch_depths(precision))
                                           + len(BATCH_GROUPS))
    member_mode = 2 * MEMBER_STEPS * (len(BATCH_STREAMS) + len(MEMBER_SHAPES))
    grouped = 2 * steps_per_candidate * (len(PER_LAUNCH) + len(GROUPED_SHAPES) * len(prefetch_depths(precision)))
    return tile_mode + 2 * steps_per_candidate * len(NARROW_ROWS) + member_mode + grouped


def tune_batch(batch, steps_per_candidate: int = 16, use_cache: bool = True) -> dict:
    """Tunes a batch's launch shape on the batch itself (every shape computes
    the same values, so tuning only advances the members by
    batch_steps_needed(steps_per_candidate) steps).  Tile-list mode: x planes
    per thread, block rows and prefetch depth with one block per tile, then
    the tile group of the persistent grid.  Grouped mode: the members per
    launch at the best tile-list shape, then block shapes and prefetch depths
    at the best count.  Member-kernel mode: the worker
    stream count at the first member shape, then the member shapes at the best
    count (whole graphs of MEMBER_STEPS steps, since a member-mode step is
    many launches).  Sets and returns the fastest."""
    key = batch_key(batch)
    cache = _load()
    if use_cache and key in cache:
        r = cache[key]
        batch.set_tiling(r["chunk"], r["rows"], r["prefetch"], r["group"], r.get("streams", 0), r.get("width", 32),
                         r.get("per_launch", 0))
        return r
    max_x = max(e.problem.grid.nx for e in batch.engines) + 1
    table = []

    def trial(chunk, rows, pf, group, streams=0, steps=steps_per_candidate, width=32, per_launch=0):
        batch.set_tiling(chunk, rows, pf, group, streams, width, per_launch)
        batch.run_timed(steps)              # capture and warm the graph
        ms = batch.run_timed(steps) / steps
        table.append({"chunk": chunk, "rows": rows, "prefetch": pf, "group": group, "streams": streams,
                      "width": width, "per_launch": per_launch, "ms_per_step": ms})

    for chunk in BATCH_CHUNKS:
        for rows in ROWS:
            for pf in prefetch_depths(batch.engines[0].precision):
                trial(min(chunk, max_x), rows, pf, 0)
    best = min(table, key=lambda r: r["ms_per_step"])
    for rows in NARROW_ROWS:
        trial(best["chunk"], rows, best["prefetch"], 0, width=16)
    best = min(table, key=lambda r: r["ms_per_step"])
    for group in BATCH_GROUPS[1:]:
        trial(best["chunk"], best["rows"], best["prefetch"], group, width=best["width"])
    tl = min(table, key=lambda r: r["ms_per_step"])
    for per in PER_LAUNCH:
        trial(tl["chunk"], tl["rows"], tl["prefetch"], 0, width=tl["width"], per_launch=per)
    p_best = min((r for r in table if r["per_launch"] > 0), key=lambda r: r["ms_per_step"])["per_launch"]
    for rw, wd in GROUPED_SHAPES:
        for pf in prefetch_depths(batch.engines[0].precision):
            trial(max_x, rw, pf, 0, width=wd, per_launch=p_best)
    ch, rw, pf = MEMBER_SHAPES[0]
    for streams in BATCH_STREAMS:
        trial(min(ch, max_x), rw, pf, 0, streams, MEMBER_STEPS)
    s_best = min((r for r in table if r["streams"] > 0), key=lambda r: r["ms_per_step"])["streams"]
    for ch, rw, pf in MEMBER_SHAPES[1:]:
        trial(min(ch, max_x), rw, pf, 0, s_best, MEMBER_STEPS)
    best = min(table, key=lambda r: r["ms_per_step"])
    out = dict(best, table=table)
    batch.set_tiling(best["chunk"], best["rows"], best["prefetch"], best["group"], best["streams"], best["width"],
                     best["per_launch"])
    cache[key] = out
    os.makedirs(os.path.dirname(CACHE), exist_ok=True)
    with open(CACHE, "w") as f:
        json.dump(cache, f, indent=1)
    return out


def apply(engine, precision: str, device: int = 0, scratch_problem=None) -> dict:
    """Tunes (on scratch_problem, or the engine's own problem rebuilt with enough
    steps by the caller) and sets the best shape on `engine`."""
    res = tune(scratch_problem or engine.problem, precision, device)
    set_tiling(engine, res["chunk"], res["rows"], res.get("prefetch", 1), res.get("width", 32))
    return res
