"""The red.min.u64 throughput probe (sgs_probe_atomic_min) leaves exactly the minima its documented
slot and value sequence implies, so the rate it measures is for the work it claims."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

M32 = np.uint64(0xFFFFFFFF)


def lowbias32(x: np.ndarray) -> np.ndarray:
    x = x.astype(np.uint64) & M32
    x ^= x >> np.uint64(16)
    x = (x * np.uint64(0x7FEB352D)) & M32
    x ^= x >> np.uint64(15)
    x = (x * np.uint64(0x846CA68B)) & M32
    x ^= x >> np.uint64(16)
    return x


def expected(n_slots: int, ops: int, blocks: int, pattern: int, seed: int) -> np.ndarray:
    t = np.arange(blocks * 256, dtype=np.uint64)
    base = lowbias32(t ^ np.uint64(seed))
    out = np.full(n_slots, np.iinfo(np.uint64).max, dtype=np.uint64)
    for i in range(ops):
        h = lowbias32(base + np.uint64((i * 0x9E3779B9) & 0xFFFFFFFF))
        slot = (h if pattern == 0 else base * np.uint64(2048) + np.uint64(i)) & np.uint64(n_slots - 1)
        np.minimum.at(out, slot.astype(np.int64), (h << np.uint64(32)) | t)
    return out


@pytest.mark.parametrize("pattern", [0, 1])
def test_probe_minima_match_the_documented_sequence(pattern, cuda_device):
    from StochasticGSCudaBackend import _C

    n_slots, ops, blocks, seed = 4096, 24, 3, 12345
    slots = torch.full((n_slots,), -1, dtype=torch.int64, device=cuda_device)
    issued = _C.probe_atomic_min(slots, ops, blocks, pattern, seed)
    assert issued == blocks * 256 * ops
    got = slots.cpu().numpy().view(np.uint64)
    np.testing.assert_array_equal(got, expected(n_slots, ops, blocks, pattern, seed))


def test_probe_rejects_bad_arguments(cuda_device):
    from StochasticGSCudaBackend import _C

    with pytest.raises(RuntimeError, match="power of two"):
        _C.probe_atomic_min(torch.zeros(1000, dtype=torch.int64, device=cuda_device), 4, 1)
    with pytest.raises(RuntimeError, match="pattern"):
        _C.probe_atomic_min(torch.zeros(1024, dtype=torch.int64, device=cuda_device), 4, 1, pattern=2)
