"""The learned resolve's tensor-core kernels against a plain PyTorch FP32 reference (GPU).

Every layer kernel (csrc/denoise.cu through the C ABI) is compared with torch's FP32 conv2d on the
same BF16-rounded operands: forward with bias + ReLU, the final layer with the residual, data
gradients with the ReLU mask, weight and bias gradients, the whole network's forward and backward,
and the feature kernel against features computed in torch from the same renders. Image sizes are
ragged (not multiples of the 8 x 16 tile) and batched. Tolerances: outputs are stored as BF16
(relative rounding 2^-8), so |got - ref| <= 1e-2 |ref| + 2e-3 max |ref|; FP32 gradients summed over
pixels agree to 2e-3 of their largest magnitude.
"""
import numpy as np
import pytest
import torch
import torch.nn.functional as F

import sgs_scenes
from StochasticGSCudaBackend import Settings, _C, _abi
from StochasticGSCudaBackend import denoise as dn

pytestmark = pytest.mark.gpu

SHAPES = [(1, 16, 8), (2, 37, 29), (1, 133, 70)]


def bf(x: torch.Tensor) -> torch.Tensor:
    return x.to(torch.bfloat16).float()


def nchw(x):
    return x.permute(0, 3, 1, 2)


def nhwc(x):
    return x.permute(0, 2, 3, 1)


def assert_close(got, ref, rel=1e-2, floor=2e-3):
    got = got.float().cpu()
    ref = ref.float().cpu()
    tol = rel * ref.abs() + floor * ref.abs().max().clamp_min(1e-6)
    bad = (got - ref).abs() > tol
    assert not bad.any(), f"{int(bad.sum())} of {bad.numel()} differ; max err {(got - ref).abs().max():.4g}"


def _rand(shape, gen, scale=1.0, dtype=torch.bfloat16):
    return (torch.randn(shape, generator=gen) * scale).to(dtype).cuda()


@pytest.mark.parametrize("shape", SHAPES)
def test_forward_layers(shape, cuda_device):
    b, h, w = shape
    g = torch.Generator().manual_seed(1)
    feats = _rand((b, h, w, 8), g, dtype=torch.float16)
    x32 = _rand((b, h, w, 32), g).relu()
    w1 = torch.randn((32, 8, 3, 3), generator=g) * 0.2
    w2 = torch.randn((32, 32, 3, 3), generator=g) * 0.1
    w6 = torch.randn((3, 32, 3, 3), generator=g) * 0.1
    b1, b2, b6 = (torch.randn(n, generator=g) * 0.1 for n in (32, 32, 3))

    got = dn.conv3x3(feats, dn.pack_forward(w1.cuda(), 16, 32), b1.cuda(), 8, 32, _abi.SGS_CONV_RELU)
    ref = nhwc(F.conv2d(nchw(bf(feats.float().cpu())), bf(w1), b1, padding=1)).relu()
    assert_close(got, ref)

    got = dn.conv3x3(x32, dn.pack_forward(w2.cuda(), 32, 32), b2.cuda(), 32, 32, _abi.SGS_CONV_RELU)
    ref = nhwc(F.conv2d(nchw(x32.float().cpu()), bf(w2), b2, padding=1)).relu()
    assert_close(got, ref)

    bias16 = torch.zeros(16)
    bias16[:3] = b6
    got = dn.conv3x3(x32, dn.pack_forward(w6.cuda(), 32, 16), bias16.cuda(), 32, 16, _abi.SGS_CONV_FINAL,
                     residual=feats)
    ref = nhwc(F.conv2d(nchw(x32.float().cpu()), bf(w6), b6, padding=1)) + feats.float().cpu()[..., :3]
    assert got.dtype == torch.float32 and got.shape == (b, h, w, 3)
    assert_close(got, ref, rel=1e-4, floor=1e-4)
    dn.status()


@pytest.mark.parametrize("shape", SHAPES)
def test_data_gradient_layers(shape, cuda_device):
    b, h, w = shape
    g = torch.Generator().manual_seed(2)
    gz = _rand((b, h, w, 32), g)
    mask = _rand((b, h, w, 32), g).relu()
    w2 = torch.randn((32, 32, 3, 3), generator=g) * 0.1
    got = dn.conv3x3(gz, dn.pack_dgrad(w2.cuda(), 32, 32), None, 32, 32, _abi.SGS_CONV_MASK, mask=mask)
    ref = torch.nn.grad.conv2d_input((b, 32, h, w), bf(w2), nchw(gz.float().cpu()), padding=1)
    ref = nhwc(ref) * (mask.float().cpu() > 0)
    assert_close(got, ref)

    w6 = torch.randn((3, 32, 3, 3), generator=g) * 0.1
    gz16 = torch.zeros((b, h, w, 16), dtype=torch.bfloat16, device="cuda")
    gz16[..., :3] = _rand((b, h, w, 3), g)
    got = dn.conv3x3(gz16, dn.pack_dgrad(w6.cuda(), 32, 16), None, 16, 32, _abi.SGS_CONV_MASK, mask=mask)
    ref = torch.nn.grad.conv2d_input((b, 32, h, w), bf(w6), nchw(gz16[..., :3].float().cpu()), padding=1)
    ref = nhwc(ref) * (mask.float().cpu() > 0)
    assert_close(got, ref)
    dn.status()


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("cin,cout", [(8, 32), (32, 32), (32, 16)])
def test_weight_gradient(shape, cin, cout, cuda_device):
    b, h, w = shape
    g = torch.Generator().manual_seed(3 + cin + cout)
    x = _rand((b, h, w, cin), g, dtype=torch.float16 if cin == 8 else torch.bfloat16)
    gz = _rand((b, h, w, cout), g)
    gw, gb = dn.conv3x3_wgrad(x, cin, gz, cout)
    staged_in = 16 if cin == 8 else cin
    gw = gw.view(3, 3, cout, staged_in).permute(2, 3, 0, 1)[:, :cin].cpu()
    ref_w = torch.nn.grad.conv2d_weight(nchw(bf(x.float()).cpu()), (cout, cin, 3, 3), nchw(gz.float().cpu()),
                                        padding=1)
    ref_b = gz.float().cpu().sum((0, 1, 2))
    scale = ref_w.abs().max()
    assert (gw - ref_w).abs().max() <= 2e-3 * scale, float((gw - ref_w).abs().max() / scale)
    assert (gb.cpu() - ref_b).abs().max() <= 2e-3 * ref_b.abs().max()
    dn.status()


def _torch_network(feats, params):
    """FP32 torch reference of the denoiser with BF16 rounding where the kernels round."""
    x = nchw(bf(feats.float()))[:, :7]
    for l in range(5):
        x = bf(F.conv2d(x, bf(params[2 * l]), params[2 * l + 1], padding=1).relu())
    out = F.conv2d(x, bf(params[10]), params[11], padding=1)
    return nhwc(out) + feats.float()[..., :3]


def test_network_forward_backward(cuda_device):
    g = torch.Generator().manual_seed(4)
    params = dn.init_params(seed=7, device="cpu")
    params[10] = torch.randn(params[10].shape, generator=g) * 0.05
    params = [p.cuda().requires_grad_(True) for p in params]
    b, h, w = 2, 45, 38
    feats = (torch.rand((b, h, w, 8), generator=g)).half().cuda()
    target = torch.rand((b, h, w, 3), generator=g).cuda()

    out = dn.denoise_train(feats, params)
    loss = ((out - target) ** 2).mean()
    loss.backward()
    got = [p.grad.detach().cpu() for p in params]

    ref_params = [p.detach().cpu().requires_grad_(True) for p in params]
    ref_out = _torch_network(feats.cpu(), ref_params)
    assert_close(out.detach(), ref_out.detach(), rel=1e-2, floor=5e-3)
    ((ref_out - target.cpu()) ** 2).mean().backward()
    for i, (a, r) in enumerate(zip(got, [p.grad for p in ref_params])):
        rel = (a - r).norm() / r.norm().clamp_min(1e-12)
        assert rel < 3e-2, f"parameter {i}: relative L2 error {rel:.4f}"

    # inference (one sgs_denoise call) runs the same kernels on the same packed weights
    model = dn.Denoiser([p.detach() for p in params])
    assert torch.equal(model(feats), out.detach())
    dn.status()


def test_untrained_denoiser_returns_the_mean(cuda_device):
    feats = torch.rand((1, 20, 20, 8)).half().cuda()
    out = dn.Denoiser(seed=0)(feats)
    assert torch.equal(out, feats[..., :3].float())


def test_features_match_torch(cuda_device):
    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=3000, log_scale_mean=-3.0), seed=3)
    cam = sgs_scenes.pinhole((0.0, 0.0, -4.0), 61, 47, 60.0)
    tensors = tuple(t.cuda() for t in scene.tensors())
    settings = Settings(cam.w2c.cuda(), cam.position.cuda(), cam.width, cam.height, cam.focal_x, cam.focal_y,
                        cam.center_x, cam.center_y, cam.near_plane, cam.far_plane, False, 1, False, False, False)
    n, first, scale = 5, 321, 0.25
    feats = dn.render_features(tensors, settings, n, first, scale).float().cpu()

    e = torch.empty(0)
    kb = (torch.empty((0, 61 * 47, 2), dtype=torch.int32, device="cuda"), torch.empty((0, 61 * 47, 4), device="cuda"))
    images, alphas, depths, winners = [], [], [], []
    for s in range(n):
        _C.set_frame_index(first + s)
        outs, ws, layout = _C.render_with_workspace(*tensors, *settings.as_tuple(),
                                                    torch.empty(0, dtype=torch.uint8, device="cuda"), *kb, e, e, e, e,
                                                    torch.eye(4, device="cuda"), 0)
        images.append(outs[0].cpu())
        depths.append(outs[1].cpu())
        alphas.append(outs[2].cpu())
        winners.append(_C.workspace_views(ws, layout, 61 * 47, False)["framebuffer"].cpu() & 0xFFFFFFFF)
    img = torch.stack(images)
    lum = img @ torch.tensor([0.2126, 0.7152, 0.0722])
    mean = img.mean(0)
    mlum = mean @ torch.tensor([0.2126, 0.7152, 0.0722])
    se = ((lum ** 2).mean(0) - mlum ** 2).clamp_min(0).div(n).sqrt()
    w = torch.stack(winners).view(n, 47, 61)
    change = (w[1:] != w[:-1]).float().sum(0) / (n - 1)
    ref = torch.cat([mean, torch.stack(alphas).mean(0), torch.stack(depths).mean(0) * scale, se[..., None],
                     change[..., None], torch.zeros(47, 61, 1)], -1)
    assert feats.shape == (47, 61, 8)
    assert (feats - ref).abs().max() < 2e-3 * max(1.0, float(ref.abs().max())), float((feats - ref).abs().max())
    assert change.max() > 0  # the scene is noisy enough that winners change


def test_captured_features_equal_eager(cuda_device):
    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=4000, log_scale_mean=-3.0), seed=8)
    cams = [sgs_scenes.pinhole((0.5, 0.2, -4.0), 64, 40, 60.0), sgs_scenes.pinhole((-1.0, 0.0, -3.5), 64, 40, 60.0)]
    tensors = tuple(t.cuda() for t in scene.tensors())

    def settings(cam):
        return Settings(cam.w2c.cuda(), cam.position.cuda(), cam.width, cam.height, cam.focal_x, cam.focal_y,
                        cam.center_x, cam.center_y, cam.near_plane, cam.far_plane, False, 1, False, False, False)

    sampler = dn.CapturedFeatures(tensors, settings(cams[0]), 0.5).capture()
    for i, cam in enumerate(cams):
        sampler.set_pose(cam.w2c.cuda(), cam.position.cuda())
        got = sampler.run(9, first_frame=50 + 100 * i, checkpoints=(1, 4, 9))
        want = dn.render_features(tensors, settings(cam), 9, 50 + 100 * i, 0.5, checkpoints=(1, 4, 9))
        for k in (1, 4, 9):
            assert torch.equal(got[k], want[k]), (i, k)
