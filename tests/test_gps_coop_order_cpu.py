"""Draw order of the GPS scatter kernel's cooperative phase, restated on the CPU.

In the reference (scatter_utils.cuh:140-183) the warp walks its larger Gaussians in lane order;
point j (counted after the first kSequentialFragments) of Gaussian `src` is drawn by lane j % 32 from
that lane's own PCG2D stream, one step per point, in (src, j) order. `gps_scatter_kernel`
(csrc/accumulate_gps.cu) evaluates whole rows of 32 points as they are drawn and parks the partial
last row of each Gaussian (drawn in the same order) in a per-warp buffer of kItemsPerWarp items,
evaluated 32 items at a time across Gaussians. These tests run both schedules lane by lane and check that every point gets
the same (lane, draw number), that buffer positions stay in bounds, and that each point is evaluated
exactly once.
"""
import random

import pytest

SEQ = 4
ITEMS = 128


def reference_order(counts: list[int]) -> dict:
    """(src, j) -> (lane, k): lane's k-th cooperative draw, as the reference walks it."""
    draws = [0] * 32
    out = {}
    for src in range(32):
        n = counts[src]
        if n <= SEQ:
            continue
        iterations = (n - SEQ + 31) // 32
        for it in range(iterations):
            for lane in range(32):
                fi = it * 32 + lane + SEQ
                if fi >= n:
                    continue
                out[(src, fi - SEQ)] = (lane, draws[lane])
                draws[lane] += 1
    return out


def buffered_order(counts: list[int]) -> tuple[dict, int]:
    """The kernel's schedule: whole rows of 32 points drawn and evaluated at once, the partial last row
    drawn in order and parked; returns (src, j) -> (lane, k) and the number of buffer flushes."""
    draws = [0] * 32
    buf = [None] * ITEMS
    out, evaluated = {}, set()
    fill = flushes = 0

    def record(key, drawn):
        assert key not in evaluated
        evaluated.add(key)
        out[key] = drawn

    def flush(n):
        nonlocal flushes
        flushes += 1
        for base in range(0, n, 32):
            for lane in range(32):
                b = base + lane
                if b < n:
                    record(*buf[b])

    for src in range(32):
        if counts[src] <= SEQ:
            continue
        n_items = counts[src] - SEQ
        full = n_items & ~31
        for lane in range(32):
            for j in range(lane, full, 32):
                record((src, j), (lane, draws[lane]))
                draws[lane] += 1
        rest = n_items - full
        if rest == 0:
            continue
        if fill + rest > ITEMS:
            flush(fill)
            fill = 0
        for lane in range(rest):
            assert 0 <= fill + lane < ITEMS and (full + lane) % 32 == lane
            buf[fill + lane] = ((src, full + lane), (lane, draws[lane]))
            draws[lane] += 1
        fill += rest
    if fill:
        flush(fill)
    return out, flushes


@pytest.mark.parametrize("seed", range(20))
def test_buffered_schedule_draws_like_the_reference(seed):
    rng = random.Random(seed)
    kind = seed % 4
    if kind == 0:
        counts = [rng.randint(0, 40) for _ in range(32)]
    elif kind == 1:
        counts = [rng.choice([0, 3, 5, 37, 132, 133, 300]) for _ in range(32)]
    elif kind == 2:
        counts = [rng.randint(0, 2000) if rng.random() < 0.2 else rng.randint(0, 8) for _ in range(32)]
    else:
        counts = [ITEMS + SEQ + rng.choice([-1, 0, 1, 31, 32, 33]) for _ in range(32)]
    want = reference_order(counts)
    got, _ = buffered_order(counts)
    assert got == want


def test_buffered_schedule_fills_the_lanes():
    counts = [10] * 32  # 6 cooperative points each: 32 iterations in the reference, 6 here
    _, flushes = buffered_order(counts)
    assert flushes == 2  # 192 items in buffers of 128 (126 when the next 6 do not fit, then 66)
