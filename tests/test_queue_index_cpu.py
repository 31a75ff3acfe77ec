"""Index arithmetic of the large-Gaussian queue consumers, restated on the CPU.

`queue_entry_of_chunk` (csrc/sgs_internal.h) finds the entry that owns chunk c with a 32-ary search
by the whole warp; `gps_queue_kernel` (csrc/accumulate_gps.cu) claims 8 chunks per atomic and reloads
the entry only when a chunk lies past it. These tests run the same steps lane by lane in Python on
random and edge-case queues and check that every chunk maps to its owner (the last entry whose first
chunk is <= c), that every index a lane reads is in bounds, and that the claims draw every point of
every entry exactly once.
"""
import random

import pytest

CHUNK_POINTS = 256
CHUNKS_PER_CLAIM = 8


def entry_of_chunk(first: list[int], n: int, c: int, reads: list[int] | None = None) -> int:
    """The device search step by step: 32 lanes, lane 0 never reads, lanes past `hi` read nothing."""
    lo, hi = 0, n
    while hi - lo > 1:
        step = (hi - lo + 31) >> 5
        le = []
        for lane in range(32):
            idx = lo + lane * step
            if lane == 0:
                le.append(True)
                continue
            ok = idx < hi
            if ok:
                assert 0 <= idx < n
                if reads is not None:
                    reads.append(idx)
                ok = first[idx] <= c
            le.append(ok)
        k = max(i for i, v in enumerate(le) if v)
        # the lanes that pass form a prefix (first[] is nondecreasing)
        assert all(le[: k + 1]) and not any(le[k + 1:])
        lo += k * step
        hi = min(hi, lo + step)
    return lo


def owner(first: list[int], c: int) -> int:
    return max(e for e, f in enumerate(first) if f <= c)


def make_queue(counts: list[int]) -> tuple[list[int], int]:
    first, total = [], 0
    for n in counts:
        first.append(total)
        total += (n + CHUNK_POINTS - 1) // CHUNK_POINTS
    return first, total


@pytest.mark.parametrize("n_entries", [1, 2, 31, 32, 33, 1000, 1025, 40_000])
def test_search_finds_the_owner(n_entries):
    rng = random.Random(n_entries)
    counts = [rng.choice([513, 600, 1024, 5000, 70_000]) for _ in range(n_entries)]
    first, n_chunks = make_queue(counts)
    probes = {0, n_chunks - 1} | {rng.randrange(n_chunks) for _ in range(200)} | set(first[:50]) | set(first[-50:])
    for c in probes:
        reads: list[int] = []
        assert entry_of_chunk(first, n_entries, c, reads) == owner(first, c)
        # 32-ary: rounds of at most 31 reads each, ceil(log32(n)) rounds
        rounds, span = 0, n_entries
        while span > 1:
            span = (span + 31) >> 5
            rounds += 1
        assert len(reads) <= 31 * rounds


def test_search_with_repeated_first_chunks():
    # nondecreasing with runs (entries that own no chunk would repeat a first chunk)
    first = [0, 0, 3, 3, 3, 7, 7, 8, 20, 20]
    for c in range(25):
        want = max(e for e, f in enumerate(first) if f <= c)
        assert entry_of_chunk(first, len(first), c) == want


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_claims_draw_every_point_once(seed):
    rng = random.Random(seed)
    counts = [rng.choice([513, 777, 2048, 2049, 9000, 33_333]) for _ in range(300)]
    first, n_chunks = make_queue(counts)
    drawn = [set() for _ in counts]
    cursor = 0
    warps = 7
    finished = [False] * warps
    while not all(finished):
        for w in range(warps):  # any interleaving of the warps' claims gives the same set
            if finished[w]:
                continue
            c0, cursor = cursor, cursor + CHUNKS_PER_CLAIM
            if c0 >= n_chunks:
                finished[w] = True
                continue
            entry_first = entry_end = 0
            e = n_points = -1
            for c in range(c0, min(c0 + CHUNKS_PER_CLAIM, n_chunks)):
                if c >= entry_end:
                    e = entry_of_chunk(first, len(first), c)
                    n_points = counts[e]
                    entry_first = first[e]
                    entry_end = entry_first + (n_points + CHUNK_POINTS - 1) // CHUNK_POINTS
                assert e == owner(first, c)
                first_point = (c - entry_first) * CHUNK_POINTS
                for lane in range(32):
                    for k in range(lane, CHUNK_POINTS, 32):
                        point = first_point + k
                        if point >= n_points:
                            break
                        assert point not in drawn[e]
                        drawn[e].add(point)
    assert all(len(d) == n for d, n in zip(drawn, counts))
    # the cursor overshoots the last chunk by less than one claim per warp
    assert cursor - n_chunks < warps * CHUNKS_PER_CLAIM + CHUNKS_PER_CLAIM
