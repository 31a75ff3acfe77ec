"""Index arithmetic of the large-Gaussian queue consumers, restated on the CPU.

`queue_entry_of_chunk` (csrc/sgs_internal.h) finds the entry that owns chunk c with a 32-ary search
by the whole warp; `gps_queue_kernel` (csrc/accumulate_gps.cu) claims 8 chunks per atomic and reloads
the entry only when a chunk lies past it. These tests run the same steps lane by lane in Python on
random and edge-case queues and check that every chunk maps to its owner (the last entry whose first
chunk is <= c), that every index a lane reads is in bounds, and that the claims draw every point of
every entry exactly once. An entry whose chunks would pass 32-bit chunk indices is marked unused by its
producer (csrc/accumulate_gps.cu, accumulate_st.cu, backward_st.cu); the last test restates that
marking and the consumers' search for the last used entry.
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


UNUSED = 0xFFFFFFFF
MAX_QUEUE_CHUNKS = 0xFFFFFFFF - (1 << 24)


def reserve(chunks_per_entry: list[int], capacity: int, start_chunk: int = 0):
    """The producers' reservations in arrival order (entry index and first chunk from one 64-bit word):
    an entry whose chunks would pass MAX_QUEUE_CHUNKS is marked unused (first chunk UNUSED, no points)
    and its Gaussian scattered instead. Returns the queue's first-chunk array, point counts and the
    entries kept."""
    first, count, kept = [], [], []
    total = start_chunk
    for e, ch in enumerate(chunks_per_entry):
        if e >= capacity:
            total += ch
            continue
        if total + ch <= MAX_QUEUE_CHUNKS:
            first.append(total)
            count.append(ch * CHUNK_POINTS)
            kept.append(e)
        else:
            first.append(UNUSED)
            count.append(0)
        total += ch
    return first, count, kept


@pytest.mark.parametrize("seed", range(6))
def test_marked_entries_are_the_last_ones_and_the_consumer_ends_at_the_last_used(seed):
    """With the chunk counter near the 32-bit limit (a first entry that starts late stands in for the
    chunks of earlier entries), the marked entries form the queue's tail, the consumer's last used entry
    is found by the same search (marked entries start past every chunk), and every chunk below the
    consumer's total maps to a used entry."""
    rng = random.Random(seed)
    chunks = [rng.choice([3, 4, 1800, 7201, 16200]) for _ in range(400)]
    # entry 0 starts at chunk 0; let the later ones start close to the limit
    big = MAX_QUEUE_CHUNKS - sum(chunks[1:200])
    chunks[0] = big
    first, count, kept = reserve(chunks, capacity=300)
    n_entries = min(len(chunks), 300)
    assert first[0] == 0
    marked = [e for e in range(n_entries) if first[e] == UNUSED]
    assert marked and marked == list(range(marked[0], n_entries))
    last = n_entries - 1
    if first[last] == UNUSED:
        last = entry_of_chunk(first, n_entries, UNUSED - 1)
    assert last == max(kept)
    n_chunks = first[last] + (count[last] + CHUNK_POINTS - 1) // CHUNK_POINTS
    assert n_chunks <= MAX_QUEUE_CHUNKS
    for c in {0, n_chunks - 1, first[last], big - 1, big} | {rng.randrange(n_chunks) for _ in range(100)}:
        if c >= n_chunks:
            continue
        e = entry_of_chunk(first, n_entries, c)
        assert first[e] != UNUSED and first[e] <= c < first[e] + count[e] // CHUNK_POINTS
