"""Caller-side helpers on the CPU: camera-path files, views and PNG output (sgs_viewer)."""
import json

import numpy as np
import torch

import sgs_scenes


def _viewer():
    import sgs_viewer  # imports the library binding, which needs the built .so (no GPU call)

    return sgs_viewer


def test_camera_path_round_trip_and_intrinsics(tmp_path):
    v = _viewer()
    cams = sgs_scenes.orbit_cameras(5, 4.0, 640, 360)
    views = [v.View.from_camera(c, frame_idx=10 + i) for i, c in enumerate(cams)]
    path = tmp_path / "path.json"
    v.save_camera_path(path, views)
    frames = json.loads(path.read_text())
    assert [f["id"] for f in frames] == [10, 11, 12, 13, 14]
    assert set(frames[0]) == {"rotation", "position", "fx", "fy", "width", "height", "id"}
    # the dataset camera: every frame keeps the given intrinsics
    back = v.load_camera_path(path, camera=views[0])
    for a, b in zip(views, back):
        np.testing.assert_allclose(a.c2w, b.c2w, atol=1e-12)
        assert (b.width, b.height, b.focal_x) == (views[0].width, views[0].height, views[0].focal_x)
    # own intrinsics: focal lengths scaled to the requested size, principal point at the centre
    scaled = v.load_camera_path(path, width=1280, height=720)
    assert scaled[0].focal_x == views[0].focal_x * 2 and scaled[0].focal_y == views[0].focal_y * 2
    assert (scaled[0].center_x, scaled[0].center_y) == (640.0, 360.0)


def test_view_pose_matches_the_scene_camera():
    v = _viewer()
    cam = sgs_scenes.pinhole((1.0, -2.0, -4.0), 320, 240, 50.0, target=(0.2, 0.1, 0.0))
    view = v.View.from_camera(cam)
    w2c, pos, c2w = view.pose("cpu")
    np.testing.assert_allclose(w2c.numpy(), cam.w2c.numpy(), atol=1e-6)
    np.testing.assert_allclose(pos.numpy(), cam.position.numpy(), atol=1e-6)
    np.testing.assert_allclose((c2w @ w2c).numpy(), np.eye(4), atol=1e-6)


def test_png_round_trip(tmp_path):
    v = _viewer()
    rng = np.random.default_rng(0)
    img = rng.random((7, 11, 3)).astype(np.float32)
    img[0, 0] = (-1.0, 2.0, 0.5)  # clamped
    v.write_png(tmp_path / "a.png", torch.from_numpy(img))
    back = v.read_png(tmp_path / "a.png")
    want = (np.clip(img, 0, 1) * 255 + 0.5).astype(np.uint8)
    assert back.shape == (7, 11, 3) and (back == want).all()
    v.write_png(tmp_path / "b.png", torch.from_numpy(img).permute(2, 0, 1))  # CHW accepted
    assert (v.read_png(tmp_path / "b.png") == want).all()
