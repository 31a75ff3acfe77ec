"""The quantised Gaussian layout on the GPU (sgs_quantize, quantized= on the render calls).

The encoder's records, chunk table and half SH equal the float32 restatement of tests/test_quantized_cpu.py
bit for bit. Renders from the layout are not bit-identical to the float32 path (the positions, rotations,
scales, opacities and SH are rounded), so they are checked statistically: with the same frame indices
almost every winner agrees, and the converged images agree to a high PSNR, in every mode.
"""
import numpy as np
import pytest
import torch

import sgs_scenes
from StochasticGSCudaBackend import _C
from test_quantized_cpu import encode

pytestmark = pytest.mark.gpu


def _args(scene, cam, flags, hist, mode, kb=None, v2pv=None, reuse=False):
    ss = flags["ss"]
    n_fb = cam.width * cam.height * ss * ss
    if kb is None:
        kb = (torch.empty((0, n_fb, 2), dtype=torch.int32, device="cuda"), torch.empty((0, n_fb, 4), device="cuda"))
    return (*scene.tensors(), cam.w2c.cuda(), cam.position.cuda(), cam.width, cam.height, cam.focal_x, cam.focal_y,
            cam.center_x, cam.center_y, cam.near_plane, cam.far_plane, flags["aa"], ss, flags["gps"], flags["hybrid"],
            reuse, torch.empty(0, dtype=torch.uint8, device="cuda"), *kb, *hist,
            v2pv if v2pv is not None else torch.eye(4, device="cuda"), mode)


def test_encoder_matches_the_restatement(cuda_device):
    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=5_000), seed=11)
    q = _C.quantize(*(t.cuda() for t in scene.tensors()))
    rec, table = encode(*(t.numpy() for t in scene.tensors()[:4]))
    assert np.array_equal(q.records.cpu().numpy().view(np.uint32), rec)
    assert np.array_equal(q.chunks.cpu().numpy().reshape(-1, 2, 4), table)
    assert np.array_equal(q.sh_half.cpu().numpy(), scene.sh_coefficients.numpy().astype(np.float16))
    assert q.records.numel() * 4 == 16 * 5_000


def psnr(a, b):
    mse = float(((a.clamp(0, 1) - b.clamp(0, 1)) ** 2).mean())
    return 10.0 * np.log10(1.0 / max(mse, 1e-20))


def test_quantised_renders_agree_with_float32(cuda_device):
    """The plain stochastic-transparency workload (100k Gaussians at 640x480): with the same thresholds per
    sample at least 97 % of the winners agree (a winner flips where the rounded alpha crosses its threshold
    or a rounded depth reorders two fragments), and the 64-sample averages agree to more than 40 dB."""
    scene = sgs_scenes.make_scene(sgs_scenes.SCENES["st_100k"], seed=0).to("cuda")
    q = _C.quantize(*scene.tensors())
    cam = sgs_scenes.front_camera(640, 480)
    flags = dict(aa=False, ss=1, gps=False, hybrid=False)
    e = torch.empty(0)
    agree = []
    for f in (3, 40):
        _C.set_frame_index(f)
        _, ws, lay = _C.render_with_workspace(*_args(scene, cam, flags, (e, e, e, e), 0))
        fb32 = _C.workspace_views(ws, lay, 640 * 480, False)["framebuffer"].clone()
        _C.set_frame_index(f)
        _, ws, lay = _C.render_with_workspace(*_args(scene, cam, flags, (e, e, e, e), 0), quantized=q)
        fbq = _C.workspace_views(ws, lay, 640 * 480, False)["framebuffer"]
        agree.append(float(((fb32 & 0xFFFFFFFF) == (fbq & 0xFFFFFFFF)).float().mean()))
    assert min(agree) > 0.97, agree
    _C.set_frame_index(100)
    a = _C.render_samples(64, *_args(scene, cam, flags, (e, e, e, e), 0))
    _C.set_frame_index(100)
    b = _C.render_samples(64, *_args(scene, cam, flags, (e, e, e, e), 0), quantized=q)
    assert psnr(a[0], b[0]) > 40.0 and psnr(a[2], b[2]) > 40.0, (psnr(a[0], b[0]), psnr(a[2], b[2]))


MODES = [
    # flags, spatial reuse, Reproject between two views
    (dict(aa=False, ss=2, gps=True, hybrid=True), True, True),
    (dict(aa=True, ss=1, gps=False, hybrid=True), False, True),
    (dict(aa=False, ss=1, gps=True, hybrid=False), False, False),
]


@pytest.mark.parametrize("flags,reuse,reproject", MODES)
def test_quantised_layout_in_every_mode(flags, reuse, reproject, cuda_device):
    """GPS, hybrid scheduling, spatial reuse and Reproject read the layout too: 16 samples (the first of a
    second view in Reproject) agree with the float32 path to more than 30 dB, and one render_samples call
    equals the loop of render calls bit for bit."""
    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=40_000, log_scale_mean=-3.0, log_scale_std=1.0), 6).to("cuda")
    q = _C.quantize(*scene.tensors())
    cams = sgs_scenes.orbit_cameras(16, 4.0, 160, 120, step_deg=3.0)
    ss = flags["ss"]
    n_fb = 160 * 120 * ss * ss
    e = torch.empty(0)

    def run(quant, loop):
        k = _C.k_buffer_size if reuse else 0
        kb = (torch.full((k, n_fb, 2), -1, dtype=torch.int32, device="cuda"), torch.zeros((k, n_fb, 4), device="cuda"))
        extra = {} if quant is None else {"quantized": quant}
        _C.set_frame_index(500)
        h = _C.render_samples(4, *_args(scene, cams[0], flags, (e, e, e, e), 0, kb, reuse=reuse), **extra)
        cam, mode, v2pv = cams[0], 1, None
        if reproject:
            cam, mode = cams[1], 2
            v2pv = (cams[0].w2c.double() @ torch.linalg.inv(cams[1].w2c.double())).float().cuda()
        if loop:
            for i in range(12):
                h = _C.render(*_args(scene, cam, flags, h, mode if i == 0 else 1, kb, v2pv, reuse), **extra)
            return h
        return _C.render_samples(12, *_args(scene, cam, flags, h, mode, kb, v2pv, reuse), **extra)

    a = run(None, False)
    b = run(q, False)
    c = run(q, True)
    assert all(torch.isfinite(t).all() for t in b)
    assert psnr(a[0], b[0]) > 30.0, psnr(a[0], b[0])
    assert all(torch.equal(x, y) for x, y in zip(b, c))


def test_quantised_layout_is_rejected_by_the_backward(cuda_device):
    from StochasticGSCudaBackend import _abi

    lib = _abi.load()
    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=100), seed=1).to("cuda")
    q = _C.quantize(*scene.tensors())
    assert lib.sgs_backward_workspace_size(100) > 0
    g = _abi.Gaussians(*(t.data_ptr() for t in scene.tensors()), 100, 16, None, *(t.data_ptr() for t in q))
    import ctypes

    cam = sgs_scenes.front_camera(32, 24)
    c = _abi.Camera(cam.w2c.cuda().data_ptr(), cam.position.cuda().data_ptr(), 32, 24, cam.focal_x, cam.focal_y,
                    16.0, 12.0, 0.2, 100.0)
    s = _abi.SettingsC(0, 1, 0, 0, 0, 0, None, None, 0, 0)
    st = lib.sgs_backward_finish(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s), None, None, None, None, None,
                                 None, None)
    assert st == _abi.SGS_ERROR_INVALID_ARGUMENT and "quantised" in _abi.last_error(lib)
