"""Every launch shape the tuners try is one the library accepts: blocks 16
or 32 wide made of whole warps and at most 256 threads (check_block in
csrc/fdtd_b200.cu, the step kernels' launch bounds), x planes per thread in
1..1024, members per grouped launch at most kGroupMembers (csrc/fdtd_batch.cuh),
prefetch depths the precision has.  A shape outside these is refused with
FDTD_ERR_BADARG and would end a tuning run on the GPU."""
import os
import re

from conftest import ROOT, load_package

pkg = load_package()
from special_topics_b200 import autotune as T  # noqa: E402

CSRC = os.path.join(ROOT, "special-topics_b200", "csrc")


def _block_ok(width, rows):
    t = width * rows
    return width in (16, 32) and t <= 256 and t % 32 == 0


def _group_members():
    with open(os.path.join(CSRC, "fdtd_batch.cuh")) as f:
        return int(re.search(r"constexpr int kGroupMembers = (\d+);", f.read()).group(1))


def test_single_grid_tuner_shapes_are_accepted():
    for rows in T.ROWS:
        assert _block_ok(32, rows), rows
    for rows in T.NARROW_ROWS:
        assert _block_ok(16, rows), rows
    assert all(1 <= c <= 1024 for c in T.CHUNKS)
    assert set(T.PREFETCH) <= set(T.TABLE_PREFETCH)
    assert T.prefetch_depths("f64") == T.PREFETCH and T.prefetch_depths("f32-table") == T.TABLE_PREFETCH


def test_batch_tuner_shapes_are_accepted():
    for rows in T.ROWS:
        assert _block_ok(32, rows)
    for rows in T.NARROW_ROWS:
        assert _block_ok(16, rows)
    for rows, width in T.GROUPED_SHAPES:
        assert _block_ok(width, rows), (rows, width)
    for chunk, rows, pf in T.MEMBER_SHAPES:
        assert _block_ok(32, rows) and 1 <= chunk <= 1024 and pf in T.PREFETCH
    assert all(1 <= c <= 1024 for c in T.BATCH_CHUNKS)
    assert all(g >= 0 for g in T.BATCH_GROUPS) and T.BATCH_GROUPS[0] == 0
    assert all(s > 0 for s in T.BATCH_STREAMS)
    assert all(0 < p <= _group_members() for p in T.PER_LAUNCH)


def test_block_rule_matches_the_library():
    """The rule above is the library's: its check_block text states the same limits."""
    with open(os.path.join(CSRC, "fdtd_b200.cu")) as f:
        src = f.read()
    body = re.search(r"int check_block\(int w, int rows\) \{(.*?)\n\}", src, re.S).group(1)
    assert "w != 16 && w != 32" in body and "t > 256" in body and "t % 32 != 0" in body
