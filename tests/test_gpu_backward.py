"""The B200 backward pass: unbiased gradient estimates of the expected image (GPU).

The estimator (csrc/backward_st.cu) averaged over many samples must agree with the exact gradient of
the expected image computed in double precision by the CPU restatement (oracle: expected_image),
which tests/test_backward_oracle_cpu.py pins to central finite differences. The samples are split
into independent batches: every parameter's mean estimate must lie within 6 standard errors of the
exact value, and the relative L2 error of each parameter group must be small.
"""
import numpy as np
import pytest
import torch

import sgs_scenes
from oracle import cpu
from StochasticGSCudaBackend import Settings
from StochasticGSCudaBackend.autograd import render_samples

pytestmark = pytest.mark.gpu

KEYS = ("means", "scales", "rotations", "opacities", "sh_coefficients")
W, H = 48, 36


def _problem(ss=1, sh_bases=16, n=120):
    spec = sgs_scenes.SceneSpec(n=n, log_scale_mean=-2.3, log_scale_std=0.4, opacity_logit_std=1.0,
                                sh_bases=sh_bases)
    scene = sgs_scenes.make_scene(spec, seed=5, morton=False)
    cam = sgs_scenes.pinhole((0.3, -0.2, -4.0), W, H, 60.0)
    rng = np.random.default_rng(0)
    gi = rng.normal(size=(H, W, 3))
    ga = rng.normal(size=(H, W, 1))
    gd = rng.normal(size=(H, W, 1)) * 0.1
    return scene, cam, gi, ga, gd


def _settings(cam, ss):
    return Settings(cam.w2c.cuda(), cam.position.cuda(), W, H, cam.focal_x, cam.focal_y, cam.center_x, cam.center_y,
                    cam.near_plane, cam.far_plane, False, ss, False, False, False)


@pytest.mark.parametrize("ss,hybrid,store,aa", [(1, False, True, False), (2, False, False, False),
                                                 (1, True, True, False), (1, False, True, True),
                                                 (2, False, False, True)])
def test_estimator_matches_exact_gradient(ss, hybrid, store, aa, cuda_device):
    """Also with proper antialiasing (aa): the opacity scaled by sqrt(det / det dilated) and the smaller
    dilation, through both the per-fragment terms and the projection backward."""
    scene, cam, gi, ga, gd = _problem(ss)
    sc = {k: t.numpy() for k, t in zip(KEYS, scene.tensors())}
    cd = dict(width=W, height=H, focal_x=cam.focal_x, focal_y=cam.focal_y, center_x=cam.center_x,
              center_y=cam.center_y, near_plane=cam.near_plane, far_plane=cam.far_plane, w2c=cam.w2c.numpy(),
              position=cam.position.numpy())
    exact = cpu.expected_image(sc, cd, ss=ss, g_image=gi, g_alpha=ga, g_depth=gd, grad=True, aa=aa)["grad"]
    settings = _settings(cam, ss)._replace(hybrid_scheduling=hybrid, proper_antialiasing=aa)
    gi_t = torch.tensor(gi, dtype=torch.float32, device="cuda")
    ga_t = torch.tensor(ga, dtype=torch.float32, device="cuda")
    gd_t = torch.tensor(gd, dtype=torch.float32, device="cuda")
    batches, per_batch = 16, 512
    est = {k: [] for k in KEYS}
    for bi in range(batches):
        params = [t.cuda().requires_grad_(True) for t in scene.tensors()]
        image, depth, alpha = render_samples(*params, settings, n_samples=per_batch, first_frame=1000 + bi * per_batch,
                                             store_winners=store)
        loss = (image * gi_t).sum() + (alpha * ga_t).sum() + (depth * gd_t).sum()
        loss.backward()
        for k, p in zip(KEYS, params):
            est[k].append(p.grad.detach().cpu().numpy().astype(np.float64))
    for k in KEYS:
        e = np.stack(est[k])
        mean = e.mean(0)
        se = e.std(0, ddof=1) / np.sqrt(batches)
        ex = exact[k]
        rel = np.linalg.norm(mean - ex) / np.linalg.norm(ex)
        z = np.abs(mean - ex) / np.maximum(se, 1e-6 * np.abs(ex).max())
        assert rel < 0.06, f"{k}: relative L2 error {rel:.4f}"
        assert np.percentile(z, 99.5) < 6.0, f"{k}: z-scores {np.sort(z.ravel())[-5:]}"


@pytest.mark.parametrize("ss,hybrid,store,aa", [(1, False, True, False), (2, True, False, False),
                                                 (1, True, True, True)])
def test_gps_estimator_matches_exact_gradient(ss, hybrid, store, aa, cuda_device):
    """Gaussian point splatting (scatter and hybrid scheduling): the estimator with each fragment's alpha
    replaced by the probability that the Gaussian puts a point into the (sub)pixel, averaged over the
    render's own GPS samples, against the exact gradient of the GPS expected image (the count law of
    the render's draw, the pixel integrals by an order-8 rule; the kernels use order 3 and a table of
    the law). 128 Gaussians: the render's draw repeats the random streams of a partial last warp's
    padding lanes, which the model does not follow (tests/test_backward_oracle_cpu.py)."""
    scene, cam, gi, ga, gd = _problem(ss, n=128)
    sc = {k: t.numpy() for k, t in zip(KEYS, scene.tensors())}
    cd = dict(width=W, height=H, focal_x=cam.focal_x, focal_y=cam.focal_y, center_x=cam.center_x,
              center_y=cam.center_y, near_plane=cam.near_plane, far_plane=cam.far_plane, w2c=cam.w2c.numpy(),
              position=cam.position.numpy())
    exact = cpu.expected_image(sc, cd, ss=ss, g_image=gi, g_alpha=ga, g_depth=gd, grad=True, aa=aa, gps=True,
                               quad=8)["grad"]
    settings = _settings(cam, ss)._replace(use_gps=True, hybrid_scheduling=hybrid, proper_antialiasing=aa)
    gi_t = torch.tensor(gi, dtype=torch.float32, device="cuda")
    ga_t = torch.tensor(ga, dtype=torch.float32, device="cuda")
    gd_t = torch.tensor(gd, dtype=torch.float32, device="cuda")
    batches, per_batch = 16, 512
    est = {k: [] for k in KEYS}
    for bi in range(batches):
        params = [t.cuda().requires_grad_(True) for t in scene.tensors()]
        image, depth, alpha = render_samples(*params, settings, n_samples=per_batch, first_frame=7000 + bi * per_batch,
                                             store_winners=store)
        loss = (image * gi_t).sum() + (alpha * ga_t).sum() + (depth * gd_t).sum()
        loss.backward()
        for k, p in zip(KEYS, params):
            est[k].append(p.grad.detach().cpu().numpy().astype(np.float64))
    for k in KEYS:
        e = np.stack(est[k])
        mean = e.mean(0)
        se = e.std(0, ddof=1) / np.sqrt(batches)
        ex = exact[k]
        rel = np.linalg.norm(mean - ex) / np.linalg.norm(ex)
        z = np.abs(mean - ex) / np.maximum(se, 1e-6 * np.abs(ex).max())
        assert rel < 0.06, f"{k}: relative L2 error {rel:.4f}"
        assert np.percentile(z, 99.5) < 6.0, f"{k}: z-scores {np.sort(z.ravel())[-5:]}"


def test_gps_count_law_table_matches_the_oracle(cuda_device):
    """The table the GPS backward builds per call (sgs_gps_count_law: P(N = n) and dP/dlambda of the
    render's point count, 1025 rows over log2(lambda) in [-10, 3], N >= 31 in the last term) against
    the oracle's law at every 16th row."""
    import ctypes

    from StochasticGSCudaBackend import _abi

    lib = _abi.load()
    n_bytes = lib.sgs_gps_count_law_size()
    assert n_bytes == 1025 * 32 * 8
    buf = torch.empty(n_bytes // 4, dtype=torch.float32, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.sgs_gps_count_law(ctypes.c_void_p(buf.data_ptr()), stream) == _abi.SGS_OK
    table = buf.view(1025, 32, 2).cpu().numpy().astype(np.float64)
    for r in list(range(0, 1025, 16)) + [1024]:
        P, dP = cpu.gps_count_law(2.0 ** (-10.0 + 13.0 * r / 1024.0))
        want, dwant = np.zeros(32), np.zeros(32)
        k = min(31, len(P))
        want[:k], dwant[:k] = P[:k], dP[:k]
        want[31], dwant[31] = 1.0 - want[:31].sum(), -dwant[:31].sum()
        assert np.abs(table[r, :, 0] - want).max() < 2e-6, r
        assert np.abs(table[r, :, 1] - dwant).max() < 1e-4 * max(1.0, np.abs(dwant).max()), r


def test_backward_rejects_unsupported_modes(cuda_device):
    """Spatial reuse is not differentiated; GPS gradients come from the fused walk only (the per-sample
    sgs_backward_accumulate rejects GPS settings)."""
    import ctypes

    from StochasticGSCudaBackend import _abi
    from StochasticGSCudaBackend.autograd import _structs

    scene, cam, *_ = _problem()
    params = [t.cuda().requires_grad_(True) for t in scene.tensors()]
    with pytest.raises(RuntimeError, match="spatial reuse"):
        render_samples(*params, _settings(cam, 1)._replace(spatial_reuse=True), n_samples=2)
    lib = _abi.load()
    tensors = tuple(t.detach().contiguous() for t in params)
    g, c, s = _structs(*tensors, _settings(cam, 1)._replace(use_gps=True))
    bw = torch.empty(lib.sgs_backward_workspace_size(tensors[0].shape[0]) // 4 + 4, device="cuda")
    grad = torch.zeros((H, W, 3), device="cuda")
    ws = torch.zeros(1 << 20, dtype=torch.uint8, device="cuda")
    st = lib.sgs_backward_accumulate(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s), ctypes.c_void_p(ws.data_ptr()),
                                     ctypes.c_void_p(grad.data_ptr()), None, None, ctypes.c_float(1.0), 1,
                                     ctypes.c_void_p(bw.data_ptr()), None)
    assert st == _abi.SGS_ERROR_INVALID_ARGUMENT
    assert "fused walk" in _abi.last_error(lib)


def _big_problem(ss=1):
    """Footprints of several thousand (sub)pixels, wide and narrow: the fused walk queues them and walks
    their rows in chunks and lane segments."""
    spec = sgs_scenes.SceneSpec(n=60, log_scale_mean=-1.2, log_scale_std=0.5, opacity_logit_std=1.0)
    scene = sgs_scenes.make_scene(spec, seed=8, morton=False)
    g = torch.Generator().manual_seed(9)
    scales = scene.scales.clone()
    scales[:20, 1] -= 2.5  # flat, wide footprints
    scene = sgs_scenes.Scene(scene.means, scales, scene.rotations, scene.opacities, scene.sh_coefficients)
    cam = sgs_scenes.pinhole((0.3, -0.2, -4.0), W, H, 60.0)
    rng = np.random.default_rng(1)
    return scene, cam, rng.normal(size=(H, W, 3)), rng.normal(size=(H, W, 1)), rng.normal(size=(H, W, 1)) * 0.1


@pytest.mark.parametrize("ss,n_samples,big", [(1, 6, False), (3, 5, False), (2, 16, False), (2, 7, True),
                                              (3, 4, True)])
def test_fused_walk_equals_one_walk_per_sample(ss, n_samples, big, cuda_device):
    """sgs_backward_sample_terms + sgs_backward_accumulate_samples (one walk for all samples, large
    footprints through the row-chunk queue) give the gradients of sgs_backward_accumulate called once
    per sample, up to float summation order."""
    import ctypes

    from StochasticGSCudaBackend import _abi
    from StochasticGSCudaBackend.autograd import _render_one, _structs

    lib = _abi.load()
    scene, cam, gi, ga, gd = _big_problem(ss) if big else _problem(ss)
    settings = _settings(cam, ss)
    tensors = tuple(t.cuda().contiguous() for t in scene.tensors())
    g, c, s = _structs(*tensors, settings)
    grads = [torch.tensor(a, dtype=torch.float32, device="cuda").contiguous() for a in (gi, ga, gd)]
    gp = [ctypes.c_void_p(t.data_ptr()) for t in grads]
    e = torch.empty(0)
    hist, workspaces = (e, e, e, e), []
    for k in range(n_samples):
        hist, ws, _ = _render_one(tensors, settings, hist, 0 if k == 0 else 1, 300 + k)
        workspaces.append(ws)
    weight = ctypes.c_float(1.0 / n_samples)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    nbytes = lib.sgs_backward_workspace_size(tensors[0].shape[0])

    def finish(bw):
        outs = [torch.empty_like(t) for t in tensors]
        assert lib.sgs_backward_finish(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s), ctypes.c_void_p(bw.data_ptr()),
                                       *(ctypes.c_void_p(t.data_ptr()) for t in outs), stream) == _abi.SGS_OK
        return [t.cpu().numpy() for t in outs]

    bw_a = torch.empty(nbytes // 4 + 4, device="cuda")
    for k, ws in enumerate(workspaces):
        assert lib.sgs_backward_accumulate(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s), ctypes.c_void_p(ws.data_ptr()),
                                           *gp, weight, int(k == 0), ctypes.c_void_p(bw_a.data_ptr()),
                                           stream) == _abi.SGS_OK
    per_sample = finish(bw_a)

    bw_b = torch.empty(nbytes // 4 + 4, device="cuda")
    scratch = torch.empty(lib.sgs_backward_samples_scratch_size(ctypes.byref(c), ctypes.byref(s), n_samples),
                          dtype=torch.uint8, device="cuda")
    for k, ws in enumerate(workspaces):
        assert lib.sgs_backward_sample_terms(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s),
                                             ctypes.c_void_p(ws.data_ptr()), *gp, weight, k, n_samples,
                                             ctypes.c_void_p(scratch.data_ptr()), stream) == _abi.SGS_OK
    assert lib.sgs_backward_accumulate_samples(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s), *gp, weight,
                                               n_samples, 1, ctypes.c_void_p(scratch.data_ptr()),
                                               ctypes.c_void_p(bw_b.data_ptr()), stream) == _abi.SGS_OK
    fused = finish(bw_b)
    for k, a, b in zip(KEYS, per_sample, fused):
        scale = np.abs(a).max()
        assert scale > 0, k
        np.testing.assert_allclose(b, a, rtol=2e-3, atol=2e-5 * scale, err_msg=k)


def test_fused_walk_rejects_bad_sample_counts(cuda_device):
    import ctypes

    from StochasticGSCudaBackend import _abi
    from StochasticGSCudaBackend.autograd import _structs

    lib = _abi.load()
    scene, cam, *_ = _problem()
    settings = _settings(cam, 1)
    tensors = tuple(t.cuda().contiguous() for t in scene.tensors())
    g, c, s = _structs(*tensors, settings)
    assert lib.sgs_backward_samples_scratch_size(ctypes.byref(c), ctypes.byref(s), 0) == 0
    assert lib.sgs_backward_samples_scratch_size(ctypes.byref(c), ctypes.byref(s), 1025) == 0
    gi = torch.zeros((H, W, 3), device="cuda")
    scratch = torch.empty(1 << 20, dtype=torch.uint8, device="cuda")
    bw = torch.empty(lib.sgs_backward_workspace_size(tensors[0].shape[0]) // 4 + 4, device="cuda")
    st = lib.sgs_backward_accumulate_samples(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s),
                                             ctypes.c_void_p(gi.data_ptr()), None, None, ctypes.c_float(1.0), 0, 1,
                                             ctypes.c_void_p(scratch.data_ptr()), ctypes.c_void_p(bw.data_ptr()), None)
    assert st == _abi.SGS_ERROR_INVALID_ARGUMENT
    st = lib.sgs_backward_sample_terms(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s),
                                       ctypes.c_void_p(scratch.data_ptr()), ctypes.c_void_p(gi.data_ptr()), None, None,
                                       ctypes.c_float(1.0), 4, 4, ctypes.c_void_p(scratch.data_ptr()), None)
    assert st == _abi.SGS_ERROR_INVALID_ARGUMENT


@pytest.mark.parametrize("ss,n_samples,big", [(1, 6, False), (2, 5, True), (3, 4, True)])
def test_framebuffer_walk_equals_one_walk_per_sample(ss, n_samples, big, cuda_device):
    """sgs_backward_accumulate_framebuffers on the framebuffers of one sgs_render_samples call gives
    the gradients of sgs_backward_accumulate called once per sample (one render call each), up to
    float summation order."""
    import ctypes

    from StochasticGSCudaBackend import _abi, _C
    from StochasticGSCudaBackend.autograd import _render_all, _render_one, _structs

    lib = _abi.load()
    scene, cam, gi, ga, gd = _big_problem(ss) if big else _problem(ss)
    settings = _settings(cam, ss)
    tensors = tuple(t.cuda().contiguous() for t in scene.tensors())
    g, c, s = _structs(*tensors, settings)
    grads = [torch.tensor(a, dtype=torch.float32, device="cuda").contiguous() for a in (gi, ga, gd)]
    gp = [ctypes.c_void_p(t.data_ptr()) for t in grads]
    e = torch.empty(0)
    hist, workspaces = (e, e, e, e), []
    for k in range(n_samples):
        hist, ws, _ = _render_one(tensors, settings, hist, 0 if k == 0 else 1, 700 + k)
        workspaces.append(ws)
    outs, ws_all, layout = _render_all(tensors, settings, n_samples, 700)
    for a, b in zip(outs, hist):
        assert torch.equal(a, b)
    weight = ctypes.c_float(1.0 / n_samples)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    nbytes = lib.sgs_backward_workspace_size(tensors[0].shape[0])

    def finish(bw):
        res = [torch.empty_like(t) for t in tensors]
        assert lib.sgs_backward_finish(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s), ctypes.c_void_p(bw.data_ptr()),
                                       *(ctypes.c_void_p(t.data_ptr()) for t in res), stream) == _abi.SGS_OK
        return [t.cpu().numpy() for t in res]

    bw_a = torch.empty(nbytes // 4 + 4, device="cuda")
    for k, ws in enumerate(workspaces):
        assert lib.sgs_backward_accumulate(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s), ctypes.c_void_p(ws.data_ptr()),
                                           *gp, weight, int(k == 0), ctypes.c_void_p(bw_a.data_ptr()),
                                           stream) == _abi.SGS_OK
    per_sample = finish(bw_a)
    bw_b = torch.empty(nbytes // 4 + 4, device="cuda")
    scratch = torch.empty(lib.sgs_backward_samples_scratch_size(ctypes.byref(c), ctypes.byref(s), n_samples),
                          dtype=torch.uint8, device="cuda")
    assert lib.sgs_backward_accumulate_framebuffers(
        ctypes.byref(g), ctypes.byref(c), ctypes.byref(s), ctypes.c_void_p(ws_all.data_ptr() + layout.framebuffer),
        n_samples, *gp, weight, 1, ctypes.c_void_p(scratch.data_ptr()), ctypes.c_void_p(bw_b.data_ptr()),
        stream) == _abi.SGS_OK
    fused = finish(bw_b)
    for k, a, b in zip(KEYS, per_sample, fused):
        scale = np.abs(a).max()
        assert scale > 0, k
        np.testing.assert_allclose(b, a, rtol=2e-3, atol=2e-5 * scale, err_msg=k)
