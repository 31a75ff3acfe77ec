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


# ---- the scatter kernel's pixel-pair stream (st_scatter_kernel, consume_pairs) ----

STREAM_ROWS = 64
STREAM_WORDS = 128
STREAM_MAX_PAIRS = 64


def run_pair_stream(batches: list[list[tuple[int, int]]]):
    """Restates one warp's pair stream: `batches` holds, per batch of (at most) 32 rows, each lane's row
    span (xs, length). Returns the pixels written per (row id, x), the ids given to the published rows,
    the rows walked lane by lane, and the largest number of live ring rows and bitmap words seen."""
    ring: dict[int, tuple] = {}
    bitmap = [0] * STREAM_WORDS
    rows_head = pairs_head = window = rows_before = 0
    written: dict[tuple[int, int], int] = {}
    long_rows = []
    max_live_rows = max_words = 0

    def consume(end):
        nonlocal rows_before
        starts = bitmap[(window >> 5) & (STREAM_WORDS - 1)]
        for lane in range(32):
            q = window + lane
            owner = rows_before + bin(starts & ((1 << (lane + 1)) - 1)).count("1") - 1
            if q >= end:
                continue
            row_id, xs, length, start = ring[owner & (STREAM_ROWS - 1)]
            assert row_id == owner, "a live ring entry was overwritten"
            j2 = 2 * (q - start)
            assert 0 <= j2 < length
            for x in (xs + j2, xs + j2 + 1):
                if x < xs + length:
                    written[(row_id, x)] = written.get((row_id, x), 0) + 1
        rows_before += bin(starts).count("1")

    row_id_of = {}
    for b, batch in enumerate(batches):
        assert len(batch) <= 32
        pairs = [(length + 1) // 2 if length <= 2 * STREAM_MAX_PAIRS else 0 for _, length in batch]
        incl = rank = 0
        for lane, ((xs, length), p) in enumerate(zip(batch, pairs)):
            incl += p
            if p:
                start = pairs_head + incl - p
                rid = rows_head + rank
                ring[rid & (STREAM_ROWS - 1)] = (rid, xs, length, start)
                row_id_of[(b, lane)] = rid
                word = (start >> 5) & (STREAM_WORDS - 1)
                assert not bitmap[word] >> (start & 31) & 1
                bitmap[word] |= 1 << (start & 31)
                rank += 1
            elif length > 2 * STREAM_MAX_PAIRS:
                long_rows.append((b, lane))
        rows_head += rank
        pairs_head += incl
        max_live_rows = max(max_live_rows, rows_head - rows_before)
        max_words = max(max_words, (pairs_head + 31) // 32 - window // 32)
        while pairs_head - window >= 32:
            word = (window >> 5) & (STREAM_WORDS - 1)
            consume(pairs_head)
            window += 32
            bitmap[word] = 0
    if pairs_head > window:
        consume(pairs_head)
    return written, row_id_of, long_rows, max_live_rows, max_words


@pytest.mark.parametrize("seed", range(16))
def test_pair_stream_writes_each_span_pixel_once(seed):
    rng = random.Random(seed)
    batches = []
    for _ in range(rng.randint(1, 40)):
        n = 32 if rng.random() < 0.8 else rng.randint(1, 32)
        kind = rng.random()
        batch = []
        for _ in range(n):
            if rng.random() < 0.15:
                batch.append((0, 0))  # an empty span
            elif kind < 0.1:
                batch.append((rng.randint(0, 100), rng.randint(100, 300)))  # long rows, some walked by lanes
            elif kind < 0.2:
                batch.append((rng.randint(0, 100), 2 * STREAM_MAX_PAIRS))  # the longest streamed rows
            else:
                batch.append((rng.randint(0, 2000), rng.randint(1, 9)))
        batches.append(batch)
    written, ids, long_rows, live, words = run_pair_stream(batches)
    want = {}
    for b, batch in enumerate(batches):
        for lane, (xs, length) in enumerate(batch):
            if (b, lane) in ids:
                for x in range(xs, xs + length):
                    want[(ids[(b, lane)], x)] = 1
            elif length > 0:
                assert length > 2 * STREAM_MAX_PAIRS and (b, lane) in long_rows
    assert written == want
    assert live <= STREAM_ROWS and words <= STREAM_WORDS


def test_pair_stream_capacity_bounds():
    """Worst cases for the rings: a batch of 32 one-pair rows after 31 pending one-pair rows, and a
    batch of 32 rows of the most pairs the stream takes."""
    batches = [[(0, 1)] * 31, [(0, 2)] * 32, [(0, 2 * STREAM_MAX_PAIRS)] * 32, [(0, 1)] * 32]
    _, _, _, live, words = run_pair_stream(batches)
    assert live <= STREAM_ROWS and words <= STREAM_WORDS
    assert live == 63


def level1_owner_slots(heights: list[int]) -> list[tuple[int, int]]:
    """st_scatter_kernel's level 1 for one warp: lane l's Gaussian has heights[l] AABB rows (0: culled,
    queued or empty). Rows are laid end to end in lane order; each Gaussian with rows is stored at slot
    popc(lanes with rows below it); a row finds its slot as `prev + popc(row starts up to it)` over
    32-row batches. Returns, per row, (slot read, lane the slot was written by)."""
    with_rows = [h > 0 for h in heights]
    incl, row_first, slots = 0, [], {}
    for lane, h in enumerate(heights):
        row_first.append(incl)
        incl += h
        if with_rows[lane]:
            slots[sum(with_rows[:lane])] = lane
    total = incl
    out, prev = [], -1
    for base in range(0, total, 32):
        bits = 0
        for lane in range(32):
            rel = row_first[lane] - base
            if with_rows[lane] and 0 <= rel < 32:
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
    between them (a lane-indexed store would hand those rows another Gaussian's or an unwritten slot)."""
    rng = random.Random(seed)
    heights = [0 if rng.random() < 0.4 else rng.randint(1, rng.choice([3, 40, 200])) for _ in range(32)]
    want = [lane for lane, h in enumerate(heights) for _ in range(h)]
    got = [lane for _, lane in level1_owner_slots(heights)]
    assert got == want
