"""3DGS .ply loading (sgs_model, the restatement of Model.py:22-79) on the CPU."""
import numpy as np
import pytest
import torch

import sgs_model
import sgs_scenes


@pytest.mark.parametrize("bases", [1, 4, 16])
def test_ply_round_trip_without_reordering(tmp_path, bases):
    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=257, sh_bases=bases), seed=3, morton=False)
    sgs_model.save_ply(tmp_path / "m.ply", scene)
    back = sgs_model.load_ply(tmp_path / "m.ply", device="cpu", morton=False)
    for a, b in zip(scene.tensors(), back.tensors()):
        assert a.shape == b.shape and torch.equal(a, b)


def test_ply_rest_coefficients_are_channel_major(tmp_path):
    """f_rest_i holds basis 1 + i % (B - 1) of channel i // (B - 1) (Model.py:76-77)."""
    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=3, sh_bases=4), seed=4, morton=False)
    sgs_model.save_ply(tmp_path / "m.ply", scene)
    v = sgs_model.read_ply_vertices(tmp_path / "m.ply")
    sh = scene.sh_coefficients.numpy()
    for i in range(9):
        np.testing.assert_array_equal(v[f"f_rest_{i}"], sh[:, 1 + i % 3, i // 3])
    np.testing.assert_array_equal(v["f_dc_1"], sh[:, 0, 1])


def test_ply_load_orders_along_the_morton_curve(tmp_path):
    scene = sgs_scenes.make_scene(sgs_scenes.SceneSpec(n=1000), seed=5, morton=False)
    sgs_model.save_ply(tmp_path / "m.ply", scene)
    back = sgs_model.load_ply(tmp_path / "m.ply", device="cpu")
    codes = sgs_scenes.morton_codes(back.means)
    assert (codes[1:] >= codes[:-1]).all()
    order = torch.argsort(sgs_scenes.morton_codes(scene.means), stable=True)
    for a, b in zip(scene.tensors(), back.tensors()):
        assert torch.equal(a[order], b)


def test_ply_ascii_and_big_endian(tmp_path):
    names = ["x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0", "scale_1", "scale_2",
             "rot_0", "rot_1", "rot_2", "rot_3"]
    rows = np.arange(2 * len(names), dtype=np.float32).reshape(2, len(names)) / 7.0
    head = "element vertex 2\n" + "".join(f"property float {n}\n" for n in names) + "end_header\n"
    (tmp_path / "a.ply").write_text("ply\nformat ascii 1.0\ncomment test\n" + head +
                                    "\n".join(" ".join(repr(float(x)) for x in r) for r in rows) + "\n")
    (tmp_path / "b.ply").write_bytes(("ply\nformat binary_big_endian 1.0\n" + head).encode() +
                                     rows.astype(">f4").tobytes())
    for name in ("a.ply", "b.ply"):
        s = sgs_model.load_ply(tmp_path / name, device="cpu", morton=False)
        np.testing.assert_allclose(s.means.numpy(), rows[:, :3], rtol=1e-6)
        np.testing.assert_allclose(s.rotations.numpy(), rows[:, 10:14], rtol=1e-6)
        assert s.sh_coefficients.shape == (2, 1, 3)


def test_ply_rejects_what_it_cannot_read(tmp_path):
    (tmp_path / "x.ply").write_bytes(b"ply\nformat binary_little_endian 1.0\nelement face 1\n"
                                     b"property list uchar int vertex_indices\nend_header\n")
    with pytest.raises(ValueError):
        sgs_model.load_ply(tmp_path / "x.ply", device="cpu")
    (tmp_path / "y.txt").write_bytes(b"not a ply\n")
    with pytest.raises(ValueError):
        sgs_model.load_ply(tmp_path / "y.txt", device="cpu")
