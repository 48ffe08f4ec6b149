"""Sweep sharding over ranks: the greedy partition, and the host protocol of
a multi-rank sweep run as world_size-2 gloo ranks on the CPU (each rank
derives its share from the same costs; gathering the shares recovers every
problem exactly once)."""
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as tmp

from conftest import load_package

pkg = load_package()
from special_topics_b200 import sharding  # noqa: E402


def test_partition_covers_every_problem_once_and_balances():
    rng = np.random.default_rng(0)
    costs = rng.integers(500_000, 800_000, 128).tolist()
    for world in (1, 2, 3, 8):
        parts = sharding.partition(costs, world)
        flat = sorted(q for p in parts for q in p)
        assert flat == list(range(128))
        assert sharding.imbalance(costs, parts) < 1.02
    assert sharding.partition([5, 4, 3], 5)[3:] == [[], []]
    with pytest.raises(ValueError):
        sharding.partition([1], 0)


def test_variant_costs_follow_the_grids():
    c = sharding.variant_costs([0, 9], 7000)
    assert c[0] == 38 * 135 * 125 * 7000 and c[1] == 41 * 142 * 132 * 7000
    c = sharding.variant_costs([0], 7000, spread=True)
    assert c[0] == 49 * 189 * 200 * 7000


def test_spread_variants_span_the_sweep_range_with_the_same_antennas():
    """The batched sweep's members (spread=True) keep each seed's antenna and
    fill grids drawn from 32x96x96 .. 64x200x200: extents inside that range,
    its x ends reached, every face at least SPREAD_MIN_AIR air cells."""
    from special_topics_b200 import workloads as W
    from special_topics_b200.scenario import DEFAULTS, build_grid
    dims = []
    for seed in range(128):
        a, b = W.ifa_variant(seed), W.ifa_variant(seed, spread=True)
        assert a["bricks"] == b["bricks"] and a["voltageSources"] == b["voltageSources"]
        assert a["materialTypes"] == b["materialTypes"]
        bd = b["boundary"]
        assert min(bd[f"air_buffer_{f}"] for f in ("xn", "xp", "yn", "yp", "zn", "zp")) >= W.SPREAD_MIN_AIR
        cell = dict(DEFAULTS["cell"], **b["cell"])
        g = build_grid(cell["dx"], cell["dy"], cell["dz"], bd, b["bricks"], [], 0.9, 10)
        dims.append((g.nx, g.ny, g.nz))
    d = np.array(dims)
    for ax, (lo, hi) in enumerate(W.VARIANT_SPAN):
        assert d[:, ax].min() >= lo and d[:, ax].max() <= hi
    assert d[:, 0].min() == 32 and d[:, 0].max() == 64
    assert d[:, 1].max() >= 195 and d[:, 2].max() >= 195


def _rank(rank, world, port, seeds, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        costs = sharding.variant_costs(seeds, 100)
        mine = [seeds[q] for q in sharding.partition(costs, world)[rank]]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        if rank == 0:
            out.put(gathered)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_a_sweep_without_exchanging_the_assignment():
    seeds = list(range(12))
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, seeds, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(s for part in got for s in part) == seeds
    assert all(part for part in got)
