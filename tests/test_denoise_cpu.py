"""Host logic of the learned resolve without a GPU: weight packing layouts and the ABI sizes.

The packed layouts are what csrc/denoise.cu's shared-memory descriptors read, so they are checked
element by element against their definitions: forward B[tap][ci / 8][co][ci % 8] = W[co][ci][dy][dx]
and data-gradient B[tap][co / 8][ci][co % 8] = W[co][ci][2 - dy][2 - dx].
"""
import numpy as np
import torch

from StochasticGSCudaBackend import _abi
from StochasticGSCudaBackend import denoise as dn


def test_forward_packing_layout():
    w = torch.randn(32, 7, 3, 3)
    p = dn.pack_forward(w, 16, 32).float().view(9, 2, 32, 8).numpy()
    wb = w.to(torch.bfloat16).float().numpy()
    for tap in range(9):
        dy, dx = divmod(tap, 3)
        for ci in range(16):
            for co in range(32):
                want = wb[co, ci, dy, dx] if ci < 7 else 0.0
                assert p[tap, ci // 8, co, ci % 8] == want


def test_dgrad_packing_layout():
    w = torch.randn(3, 32, 3, 3)
    p = dn.pack_dgrad(w, 32, 16).float().view(9, 2, 32, 8).numpy()
    wb = w.to(torch.bfloat16).float().numpy()
    for tap in range(9):
        dy, dx = divmod(tap, 3)
        for co in range(16):
            for ci in range(32):
                want = wb[co, ci, 2 - dy, 2 - dx] if co < 3 else 0.0
                assert p[tap, co // 8, ci, co % 8] == want


def test_wgrad_unpacking_inverts_the_kernel_layout():
    g = torch.randn(9, 16, 32)
    out = dn.unpack_wgrad(g, 5)
    assert out.shape == (3, 32, 3, 3)
    for tap in range(9):
        dy, dx = divmod(tap, 3)
        assert torch.equal(out[:, :, dy, dx], g[tap, :3, :])


def test_sizes_agree_with_the_library():
    lib = _abi.load()
    total = sum(dn.pack_forward(torch.zeros(co, ci, 3, 3), si, so).numel() * 2
                for (ci, co), si, so in zip(dn.LAYERS, dn.STAGED_IN, dn.STAGED_OUT))
    assert lib.sgs_denoise_weights_size() == total
    for (ci, co), abi_in, so in zip(dn.LAYERS, dn.ABI_IN, dn.STAGED_OUT):
        assert lib.sgs_conv3x3_weights_size(abi_in, so) == 9 * (16 if abi_in == 8 else abi_in) * so * 2
    assert lib.sgs_denoise_scratch_size(2, 10, 12) == 2 * 2 * 10 * 12 * 32 * 2
    assert lib.sgs_denoise_scratch_size(0, 10, 12) == 0


def test_invalid_layer_shapes_are_rejected_before_any_launch():
    lib = _abi.load()
    fake = 0x10000
    args = _abi.Conv3x3Args(fake, fake, fake, fake, None, None, 1, 16, 16, 16, 16, _abi.SGS_CONV_RELU)
    assert lib.sgs_conv3x3(args, None) == _abi.SGS_ERROR_INVALID_ARGUMENT
    assert "unsupported" in _abi.last_error(lib)
    args = _abi.Conv3x3Args(fake, fake, fake, fake, None, None, 1, 0, 16, 32, 32, _abi.SGS_CONV_RELU)
    assert lib.sgs_conv3x3(args, None) == _abi.SGS_ERROR_INVALID_ARGUMENT
    args = _abi.Conv3x3Args(fake, fake, fake, None, None, None, 1, 16, 16, 32, 32, _abi.SGS_CONV_MASK)
    assert lib.sgs_conv3x3(args, None) == _abi.SGS_ERROR_INVALID_ARGUMENT  # mask missing
    assert lib.sgs_conv3x3_wgrad(fake, 16, fake, 16, 1, 8, 8, fake, fake, None) == _abi.SGS_ERROR_INVALID_ARGUMENT
    assert lib.sgs_denoise(fake, 1, 8, 8, fake, fake, fake, 10, fake, None) == _abi.SGS_ERROR_WORKSPACE


def test_untrained_parameters_make_the_last_layer_zero():
    params = dn.init_params(seed=0, device="cpu")
    assert len(params) == 12
    assert all(p.shape == (co, ci, 3, 3) for p, (ci, co) in zip(params[0::2], dn.LAYERS))
    assert not params[10].any() and not params[11].any()
    assert np.isclose(float(params[0].std()), (2 / 63) ** 0.5, rtol=0.2)
