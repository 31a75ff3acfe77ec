"""Index arithmetic of the stochastic-transparency row walker, restated on the CPU.

A queued Gaussian's AABB (width w, height h) is cut into chunks of 2^r rows, r = log2 of
max(1, min(32, 2048 / w)) (`log_chunk_rows`, csrc/accumulate_st.cu); in a chunk, lane l walks
segment l >> r of row r0 + (l & (2^r - 1)), the row's span split into 2^(5 - r) equal parts
(`walk_chunk`, `walk_rows`). Each lane steps two pixels at a time and writes pixel xs + i only when
i < len. These tests run that arithmetic lane by lane for many widths, heights and spans and check
that every span pixel of every row is written exactly once and that no write leaves the row's span.
"""
import random

import pytest

CHUNK_PIXELS = 2048


def log_chunk_rows(w: int) -> int:
    rows = max(1, min(32, CHUNK_PIXELS // max(w, 1)))
    return rows.bit_length() - 1


def lane_segment(xs: int, length: int, seg: int, log_segs: int) -> tuple[int, int]:
    """walk_rows: the part of the span [xs, xs + length) that segment `seg` of 2^log_segs walks."""
    if log_segs > 0:
        part = (length + (1 << log_segs) - 1) >> log_segs
        skip = min(seg * part, length)
        xs += skip
        length = min(length - skip, part)
    return xs, length


def walk_queued(w: int, h: int, spans: list[tuple[int, int]]) -> dict[tuple[int, int], int]:
    """Pixels (row, x) written, with their counts, over all chunks of one queued Gaussian."""
    log_rpc = log_chunk_rows(w)
    assert 0 <= log_rpc <= 5
    chunks = (h + (1 << log_rpc) - 1) >> log_rpc
    written: dict[tuple[int, int], int] = {}
    for c in range(chunks):
        r0 = c << log_rpc
        assert r0 < h
        steps = 0
        lanes = []
        for lane in range(32):
            r = r0 + (lane & ((1 << log_rpc) - 1))
            valid = r < h
            xs, length = 0, 0
            if valid:
                xs, length = lane_segment(*spans[r], lane >> log_rpc, 5 - log_rpc)
            lanes.append((r, xs, length))
            steps = max(steps, length)
        for i in range(0, steps, 2):  # two pixels per step, written only inside the segment
            for r, xs, length in lanes:
                for x in (i, i + 1):
                    if x < length:
                        key = (r, xs + x)
                        written[key] = written.get(key, 0) + 1
    return written


@pytest.mark.parametrize("seed", range(12))
def test_queued_chunks_cover_each_span_pixel_once(seed):
    rng = random.Random(seed)
    for _ in range(40):
        w = rng.choice([1, 2, 31, 32, 33, 63, 64, 65, 100, 2047, 2048, 2049, 5000, rng.randint(1, 8000)])
        h = rng.choice([1, 2, 3, 31, 32, 33, rng.randint(1, 300)])
        spans = []
        for _ in range(h):
            if rng.random() < 0.1:
                spans.append((0, 0))  # a row with no span pixel
                continue
            length = rng.randint(1, w)
            xs = rng.randint(0, w - length)
            spans.append((xs, length))
        written = walk_queued(w, h, spans)
        want = {(r, x) for r, (xs, length) in enumerate(spans) for x in range(xs, xs + length)}
        assert set(written) == want
        assert all(n == 1 for n in written.values())


@pytest.mark.parametrize("w", [1, 7, 32, 64, 65, 128, 2048, 4096, 100_000])
def test_chunk_rows_and_segments(w):
    r = log_chunk_rows(w)
    rows = 1 << r
    cap = max(1, min(32, CHUNK_PIXELS // w))
    assert rows <= cap < 2 * rows  # the largest power of two within the cap
    # every lane of a chunk has a (row, segment) of its own
    pairs = {(lane & (rows - 1), lane >> r) for lane in range(32)}
    assert len(pairs) == 32 and max(s for _, s in pairs) == (32 >> r) - 1


@pytest.mark.parametrize("length", [0, 1, 2, 31, 32, 33, 1000])
@pytest.mark.parametrize("log_segs", [0, 1, 3, 5])
def test_segments_partition_a_span(length, log_segs):
    xs = 17
    covered = []
    for seg in range(1 << log_segs):
        s, n = lane_segment(xs, length, seg, log_segs)
        assert n >= 0 and (n == 0 or xs <= s and s + n <= xs + length)
        covered.extend(range(s, s + n))
    assert covered == list(range(xs, xs + length))


# ---- the scatter kernel's level 1 (st_scatter_kernel) ----

NO_ROWS_KEY = (1 << 26) - 1


def level1_owner_slots(heights: list[int], widths: list[int]) -> list[tuple[int, int]]:
    """st_scatter_kernel's level 1 for one warp: lane l's Gaussian has heights[l] AABB rows (0: culled,
    queued or empty) of about widths[l] pixels. The Gaussians are sorted by (width, lane), those without
    rows last; their rows are laid end to end in that order and each Gaussian with rows is stored at
    its rank; a row finds its slot as `prev + popc(row starts up to it)` over 32-row batches. Returns,
    per row, (slot read, lane the slot was written by)."""
    keys = [((min(w, NO_ROWS_KEY - 1) if h > 0 else NO_ROWS_KEY) << 5) | lane
            for lane, (h, w) in enumerate(zip(heights, widths))]
    order = sorted(range(32), key=lambda lane: keys[lane])  # position i: the lane of the i-th smallest key
    rank = {lane: i for i, lane in enumerate(order)}
    incl, first_sorted = 0, []
    for lane in order:
        first_sorted.append(incl)
        incl += heights[lane]
    row_first = [first_sorted[rank[lane]] for lane in range(32)]
    slots = {rank[lane]: lane for lane in range(32) if heights[lane] > 0}
    total = incl
    out, prev = [], -1
    for base in range(0, total, 32):
        bits = 0
        for lane in range(32):
            rel = row_first[lane] - base
            if heights[lane] > 0 and 0 <= rel < 32:
                bits |= 1 << rel
        for lane in range(32):
            r = base + lane
            owner = prev + bin(bits & ((1 << (lane + 1)) - 1)).count("1")
            if r < total:
                out.append((owner, slots[owner]))
        prev += bin(bits).count("1")
    return out


@pytest.mark.parametrize("seed", range(20))
def test_level1_rows_find_their_own_gaussian(seed):
    """Every row reads the constants of the Gaussian it belongs to, also with Gaussians without rows
    among them (sorted last, so the ranks of the Gaussians with rows are 0, 1, ... in row order), and
    the rows come in order of the Gaussians' widths."""
    rng = random.Random(seed)
    heights = [0 if rng.random() < 0.4 else rng.randint(1, rng.choice([3, 40, 200])) for _ in range(32)]
    widths = [rng.randint(1, rng.choice([4, 64, 3000])) for _ in range(32)]
    order = sorted((lane for lane in range(32) if heights[lane] > 0), key=lambda lane: (widths[lane], lane))
    want = [lane for lane in order for _ in range(heights[lane])]
    got = [lane for _, lane in level1_owner_slots(heights, widths)]
    assert got == want
