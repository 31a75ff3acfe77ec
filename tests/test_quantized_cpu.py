"""The quantised Gaussian layout (sgs_quantize, csrc/quantize.cu), restated on the CPU.

Record of one Gaussian, four 32-bit words:
  w0  position relative to its chunk's box: x in bits 21-31 (11 bits), y in bits 11-20 (10 bits),
      z in bits 0-10 (11 bits), each round((p - lo) / extent * (2^bits - 1)), 0 for a zero extent
  w1  rotation, smallest three: bits 30-31 the index of the largest |component| of the normalised
      quaternion (r, i, j, k), made positive; the other three in order, 10 bits each from bit 20 down,
      round((c * sqrt(2) + 1) / 2 * 1022), so that 0 is exact
  w2  log-scales x (bits 0-15) and y (bits 16-31) as IEEE half
  w3  log-scale z (bits 0-15) and the opacity logit (bits 16-31) as IEEE half
A chunk is 256 consecutive Gaussians; its table entry holds (lo.x, lo.y, lo.z, 0) and
(extent.x, extent.y, extent.z, 0). The SH coefficients become IEEE half.

`encode` below does the kernel's arithmetic with the same float32 operations (round to nearest, no
fused multiply-add), so the GPU test compares records bit for bit; this file checks the format's
error bounds and corner cases.
"""
import numpy as np
import pytest

CHUNK = 256
BITS = (11, 10, 11)
F32 = np.float32


def chunk_table(means: np.ndarray) -> np.ndarray:
    n = means.shape[0]
    n_chunks = (n + CHUNK - 1) // CHUNK
    table = np.zeros((n_chunks, 2, 4), dtype=F32)
    for c in range(n_chunks):
        m = means[c * CHUNK:(c + 1) * CHUNK]
        lo, hi = m.min(axis=0), m.max(axis=0)
        table[c, 0, :3] = lo
        table[c, 1, :3] = (hi - lo).astype(F32)
    return table


def encode(means, scales, rotations, opacities):
    """(N, 4) uint32 records and the chunk table, as the encoder computes them."""
    means = means.astype(F32)
    n = means.shape[0]
    table = chunk_table(means)
    lo = table[np.arange(n) // CHUNK, 0, :3]
    ext = table[np.arange(n) // CHUNK, 1, :3]
    w0 = np.zeros(n, dtype=np.uint32)
    shift = (21, 11, 0)
    for a in range(3):
        top = F32((1 << BITS[a]) - 1)
        with np.errstate(divide="ignore", invalid="ignore"):
            t = np.where(ext[:, a] > 0, (means[:, a] - lo[:, a]) / ext[:, a], F32(0)).astype(F32)
        q = np.clip(np.rint((t * top).astype(F32)), 0, top).astype(np.uint32)
        w0 |= q << np.uint32(shift[a])
    r = rotations.astype(F32)
    sq = ((r[:, 0] * r[:, 0] + r[:, 1] * r[:, 1]).astype(F32) + r[:, 2] * r[:, 2]).astype(F32)
    sq = (sq + r[:, 3] * r[:, 3]).astype(F32)
    norm = np.sqrt(sq).astype(F32)
    with np.errstate(divide="ignore", invalid="ignore"):
        u = np.where(norm[:, None] > 0, r / norm[:, None], np.array([1, 0, 0, 0], F32)).astype(F32)
    big = np.argmax(np.abs(u), axis=1)
    sign = np.where(u[np.arange(n), big] < 0, F32(-1), F32(1))
    w1 = (big.astype(np.uint32) << np.uint32(30))
    others = np.array([[j for j in range(4) if j != b] for b in range(4)])[big]
    for o in range(3):
        c = (u[np.arange(n), others[:, o]] * sign).astype(F32)
        v = ((c * F32(np.sqrt(2.0)) + F32(1)) * F32(0.5)).astype(F32)
        q = np.clip(np.rint((v * F32(1022)).astype(F32)), 0, 1022).astype(np.uint32)
        w1 |= q << np.uint32(20 - 10 * o)
    h = lambda x: x.astype(np.float16).view(np.uint16).astype(np.uint32)
    s = scales.astype(F32)
    w2 = h(s[:, 0]) | (h(s[:, 1]) << np.uint32(16))
    w3 = h(s[:, 2]) | (h(opacities.reshape(-1).astype(F32)) << np.uint32(16))
    return np.stack([w0, w1, w2, w3], axis=1), table


def decode(records, table):
    n = records.shape[0]
    lo = table[np.arange(n) // CHUNK, 0, :3].astype(np.float64)
    ext = table[np.arange(n) // CHUNK, 1, :3].astype(np.float64)
    w0, w1, w2, w3 = (records[:, i] for i in range(4))
    q = np.stack([(w0 >> 21) & 2047, (w0 >> 11) & 1023, w0 & 2047], axis=1).astype(np.float64)
    means = lo + q / np.array([2047.0, 1023.0, 2047.0]) * ext
    big = (w1 >> 30).astype(np.int64)
    rest = np.stack([(w1 >> 20) & 1023, (w1 >> 10) & 1023, w1 & 1023], axis=1).astype(np.float64)
    rest = (rest / 1022.0 * 2.0 - 1.0) / np.sqrt(2.0)
    largest = np.sqrt(np.maximum(0.0, 1.0 - (rest ** 2).sum(axis=1)))
    quat = np.zeros((n, 4))
    others = np.array([[j for j in range(4) if j != b] for b in range(4)])[big]
    quat[np.arange(n), big] = largest
    for o in range(3):
        quat[np.arange(n), others[:, o]] = rest[:, o]
    f16 = lambda x: (x & 0xFFFF).astype(np.uint16).view(np.float16).astype(np.float64)
    scales = np.stack([f16(w2), f16(w2 >> 16), f16(w3)], axis=1)
    opac = f16(w3 >> 16)
    return means, scales, quat, opac


@pytest.fixture(scope="module")
def model():
    rng = np.random.default_rng(0)
    n = 3000
    means = rng.normal(size=(n, 3)).astype(F32)
    means = means[np.argsort(means[:, 0])]  # spatially coherent chunks, as Morton order gives
    scales = rng.normal(-4.0, 0.5, size=(n, 3)).astype(F32)
    rot = rng.normal(size=(n, 4)).astype(F32)
    opac = rng.normal(0, 1.5, size=n).astype(F32)
    return means, scales, rot, opac


def test_round_trip_error_bounds(model):
    means, scales, rot, opac = model
    rec, table = encode(means, scales, rot, opac)
    m, s, q, o = decode(rec, table)
    ext = table[np.arange(len(means)) // CHUNK, 1, :3]
    assert (np.abs(m - means) <= ext / np.array([2047.0, 1023.0, 2047.0]) * 0.5 + 1e-6).all()
    assert np.abs(s - scales).max() <= 2.0 ** -8  # half precision at |log-scale| < 8
    assert np.abs(o - opac).max() <= 2.0 ** -7
    u = rot / np.linalg.norm(rot, axis=1, keepdims=True)
    # the same rotation: q or -q, within the 10-bit steps of the three stored components
    dot = np.abs((q * u).sum(axis=1))
    assert dot.min() > 1.0 - 1e-5


def test_degenerate_inputs():
    means = np.zeros((5, 3), F32)
    rec, table = encode(means, np.zeros((5, 3), F32), np.zeros((5, 4), F32), np.zeros(5, F32))
    m, s, q, o = decode(rec, table)
    assert (m == 0).all() and (table[:, 1] == 0).all()
    assert np.allclose(q, [[1, 0, 0, 0]] * 5)  # a zero quaternion encodes the identity


def test_chunks_of_256():
    means = np.arange(600 * 3, dtype=F32).reshape(600, 3)
    table = chunk_table(means)
    assert table.shape == (3, 2, 4)
    assert (table[2, 0, :3] == means[512]).all() and (table[2, 1, :3] == means[599] - means[512]).all()
