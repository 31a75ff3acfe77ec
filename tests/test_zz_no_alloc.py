"""sgs_render_no_alloc: the render for callers that cannot allocate device memory while they render.

It is called here through the C ABI, with inputs and outputs the test owns, and compared bit for bit
with sgs_render (through `_C.render`) on two calls in a row: a Reset frame, then a Static frame that
merges it. The no-alloc path keeps all its scratch in a fixed array of the library, so the second
call also shows that the previous call's leftovers there do not leak into the result. A second pair
renders Gaussian point splatting with hybrid scheduling after those stochastic-transparency calls:
that path keeps its work queue (entry keys, geometry, counts, cursors) in the same array, so it shows
that one call's queue contents cannot leak into the next. The test sets the frame index itself, so
it gives the same result alone in a fresh process or after others.
"""
import ctypes

import pytest
import torch

import sgs_scenes
from StochasticGSCudaBackend import _abi, _C

pytestmark = pytest.mark.gpu

W, H = 320, 240


def _structs(scene, cam, mode, history, outputs, dev, gps=0, hybrid=0):
    g = _abi.Gaussians(scene.means.data_ptr(), scene.scales.data_ptr(), scene.rotations.data_ptr(),
                       scene.opacities.data_ptr(), scene.sh_coefficients.data_ptr(), scene.means.shape[0],
                       scene.sh_coefficients.shape[1])
    c = _abi.Camera(cam["w2c"].data_ptr(), cam["pos"].data_ptr(), W, H, cam["fx"], cam["fy"], W / 2, H / 2, 0.2,
                    10000.0)
    s = _abi.SettingsC(0, 1, gps, hybrid, 0, mode, None, None, 0, 0)
    h = _abi.HistoryC(*(t.data_ptr() if mode else None for t in history), None, None)
    o = _abi.Outputs(*(t.data_ptr() for t in outputs))
    return g, c, s, h, o


def _no_alloc_call(lib, scene, cam, mode, history, dev, frame, gps=0, hybrid=0):
    outputs = (torch.empty((H, W, 3), device=dev), torch.empty((H, W, 1), device=dev),
               torch.empty((H, W, 1), device=dev), torch.empty((H, W, 1), device=dev))
    g, c, s, h, o = _structs(scene, cam, mode, history, outputs, dev, gps, hybrid)
    _C.set_frame_index(frame)
    st = lib.sgs_render_no_alloc(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s), ctypes.byref(h), ctypes.byref(o),
                                 ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    assert st == _abi.SGS_OK, _abi.last_error(lib)
    return outputs


def test_no_alloc_matches_workspace_render_on_two_calls(cuda_device):
    lib = _abi.load()
    dev = cuda_device
    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=50_000, log_scale_mean=-3.0, log_scale_std=0.7), seed=21)
    scene = scene.to(dev)
    camera = sgs_scenes.front_camera(W, H)
    cam = {"w2c": camera.w2c.to(dev), "pos": camera.position.to(dev), "fx": camera.focal_x, "fy": camera.focal_y}
    e = torch.empty(0)
    kb = (torch.empty((0, W * H, 2), dtype=torch.int32, device=dev), torch.empty((0, W * H, 4), device=dev))
    blue = torch.empty(0, dtype=torch.uint8, device=dev)

    def workspace_render(mode, history, frame, gps=False, hybrid=False):
        _C.set_frame_index(frame)
        return _C.render(*scene.tensors(), cam["w2c"], cam["pos"], W, H, cam["fx"], cam["fy"], W / 2, H / 2, 0.2,
                         10000.0, False, 1, gps, hybrid, False, blue, *kb, *history, torch.eye(4, device=dev), mode)

    empty_hist = (e, e, e, e)
    a1 = _no_alloc_call(lib, scene, cam, 0, empty_hist, dev, frame=40)
    b1 = workspace_render(0, empty_hist, 40)
    a2 = _no_alloc_call(lib, scene, cam, 1, a1, dev, frame=41)
    b2 = workspace_render(1, b1, 41)
    # Gaussian point splatting with hybrid scheduling after the stochastic-transparency calls: its
    # work queue lives in the same array as their framebuffers and queue
    a3 = _no_alloc_call(lib, scene, cam, 0, empty_hist, dev, frame=42, gps=1, hybrid=1)
    b3 = workspace_render(0, empty_hist, 42, gps=True, hybrid=True)
    a4 = _no_alloc_call(lib, scene, cam, 1, a3, dev, frame=43, gps=1, hybrid=1)
    b4 = workspace_render(1, b3, 43, gps=True, hybrid=True)
    torch.cuda.synchronize(dev)
    assert float(b1[2].sum()) > 0 and float(b3[2].sum()) > 0
    for step, (got, want) in enumerate(((a1, b1), (a2, b2), (a3, b3), (a4, b4))):
        for name, x, y in zip(("image", "depth", "alpha", "weight_mass"), got, want):
            assert torch.equal(x, y), f"call {step + 1}: {name} differs"


def test_no_alloc_rejects_renders_beyond_its_scratch(cuda_device):
    lib = _abi.load()
    dev = cuda_device
    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=64), seed=1).to(dev)
    camera = sgs_scenes.front_camera(3840, 2160)
    cam = {"w2c": camera.w2c.to(dev), "pos": camera.position.to(dev), "fx": camera.focal_x, "fy": camera.focal_y}
    outputs = tuple(torch.empty(1, device=dev) for _ in range(4))
    g, c, s, h, o = _structs(scene, cam, 0, (None,) * 4, outputs, dev)
    c.width, c.height = 3840, 2160
    st = lib.sgs_render_no_alloc(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s), ctypes.byref(h), ctypes.byref(o),
                                 None)
    assert st == _abi.SGS_ERROR_WORKSPACE
    assert "scratch" in _abi.last_error(lib)
