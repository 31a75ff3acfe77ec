"""Seeded synthetic Gaussian scenes and pinhole cameras for the render path.

The reference renders pretrained 3DGS `.ply` models (Model.py:22-79) whose datasets are not available
here; these generators stand in for them with the shapes, layouts and value distributions of the
named workloads. Layouts follow Model.py exactly: fp32 `means (N,3)`, log `scales (N,3)`,
`rotations (N,4)` as (r, i, j, k), logit `opacities (N,)`, `sh_coefficients (N,B,3)`, optionally in
Morton order (Model.py:32-34). Cameras follow the reference's OpenCV convention (x right, y down,
z forward; StochasticGSCudaBackend/render.py:15-16): `w2c` is a 4x4 row-major world-to-view matrix.

Everything is drawn on the CPU with `torch.Generator().manual_seed(seed)` in a fixed order (means,
log-scales, quaternions, opacity logits, SH DC, SH rest), so a seed names one scene on any machine.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import torch


@dataclass(frozen=True)
class SceneSpec:
    """Distribution of a synthetic scene."""

    n: int
    means: str = "normal"  # "normal": N(0, means_scale^2); "uniform": U[-means_scale, means_scale]
    means_scale: float = 1.0
    log_scale_mean: float = -4.0
    log_scale_std: float = 0.5
    opacity_logit_std: float = 1.5
    sh_bases: int = 16
    sh_dc_std: float = 0.5
    sh_rest_std: float = 0.05


# workload families: plain ST at 640x480, GPS hybrid at 1280x720 ss 2, the 6M-Gaussian batched
# scene (headline 1920x1080), and the 500k-Gaussian differentiable-training scene
SCENES = {
    "st_100k": SceneSpec(n=100_000),
    "gps_1m": SceneSpec(n=1_000_000, log_scale_mean=-3.0, log_scale_std=1.0),
    "batch_6m": SceneSpec(n=6_000_000, means="uniform", means_scale=10.0, log_scale_mean=-4.5, log_scale_std=0.8,
                          opacity_logit_std=2.0),
    "train_500k": SceneSpec(n=500_000, log_scale_mean=-3.5, log_scale_std=0.7),
}


@dataclass
class Scene:
    means: torch.Tensor
    scales: torch.Tensor
    rotations: torch.Tensor
    opacities: torch.Tensor
    sh_coefficients: torch.Tensor

    def tensors(self) -> tuple[torch.Tensor, ...]:
        return self.means, self.scales, self.rotations, self.opacities, self.sh_coefficients

    def to(self, device) -> "Scene":
        return Scene(*(t.to(device) for t in self.tensors()))

    def nbytes(self) -> int:
        return sum(t.numel() * t.element_size() for t in self.tensors())


def make_scene(spec: SceneSpec, seed: int = 0, morton: bool = True) -> Scene:
    g = torch.Generator().manual_seed(seed)
    n = spec.n
    if spec.means == "uniform":
        means = (torch.rand((n, 3), generator=g) * 2.0 - 1.0) * spec.means_scale
    else:
        means = torch.randn((n, 3), generator=g) * spec.means_scale
    scales = torch.randn((n, 3), generator=g) * spec.log_scale_std + spec.log_scale_mean
    rotations = torch.randn((n, 4), generator=g)
    rotations = rotations / rotations.norm(dim=1, keepdim=True).clamp_min(1e-12)
    opacities = torch.randn((n,), generator=g) * spec.opacity_logit_std
    sh = torch.empty((n, spec.sh_bases, 3))
    sh[:, 0, :] = torch.randn((n, 3), generator=g) * spec.sh_dc_std
    if spec.sh_bases > 1:
        sh[:, 1:, :] = torch.randn((n, spec.sh_bases - 1, 3), generator=g) * spec.sh_rest_std
    scene = Scene(means.float(), scales.float(), rotations.float(), opacities.float(), sh.float())
    if morton:
        order = torch.argsort(morton_codes(scene.means), stable=True)
        scene = Scene(*(t[order].contiguous() for t in scene.tensors()))
    return scene


def _spread_bits_10(v: torch.Tensor) -> torch.Tensor:
    v = v & 0x3FF
    v = (v | (v << 16)) & 0x030000FF
    v = (v | (v << 8)) & 0x0300F00F
    v = (v | (v << 4)) & 0x030C30C3
    v = (v | (v << 2)) & 0x09249249
    return v


def morton_codes(means: torch.Tensor) -> torch.Tensor:
    """30-bit Morton codes of the means quantised to 10 bits per axis over their bounding box."""
    lo = means.min(dim=0).values
    hi = means.max(dim=0).values
    q = ((means - lo) / (hi - lo).clamp_min(1e-12) * 1023.0).clamp(0, 1023).to(torch.int64)
    return _spread_bits_10(q[:, 0]) | (_spread_bits_10(q[:, 1]) << 1) | (_spread_bits_10(q[:, 2]) << 2)


@dataclass
class Camera:
    w2c: torch.Tensor  # (4, 4) float32, row-major world -> view
    position: torch.Tensor  # (3,) float32
    width: int
    height: int
    focal_x: float
    focal_y: float
    center_x: float
    center_y: float
    near_plane: float = 0.2
    far_plane: float = 10000.0

    def to(self, device) -> "Camera":
        return Camera(self.w2c.to(device), self.position.to(device), self.width, self.height, self.focal_x,
                      self.focal_y, self.center_x, self.center_y, self.near_plane, self.far_plane)

    @property
    def c2w(self) -> torch.Tensor:
        return torch.linalg.inv(self.w2c.double()).float()


def look_at(position, target=(0.0, 0.0, 0.0), down=(0.0, 1.0, 0.0)) -> torch.Tensor:
    """OpenCV world-to-view matrix: rows are the camera's x (right), y (down) and z (forward) axes."""
    c = torch.tensor(position, dtype=torch.float64)
    f = torch.tensor(target, dtype=torch.float64) - c
    f = f / f.norm()
    d = torch.tensor(down, dtype=torch.float64)
    d = d - (d @ f) * f
    d = d / d.norm()
    r = torch.linalg.cross(d, f)
    rot = torch.stack([r, d, f])
    w2c = torch.eye(4, dtype=torch.float64)
    w2c[:3, :3] = rot
    w2c[:3, 3] = -rot @ c
    return w2c.float()


def pinhole(position, width: int, height: int, fov_y_deg: float = 60.0, target=(0.0, 0.0, 0.0),
            near_plane: float = 0.2, far_plane: float = 10000.0) -> Camera:
    fy = height / (2.0 * math.tan(math.radians(fov_y_deg) / 2.0))
    return Camera(look_at(position, target), torch.tensor(position, dtype=torch.float32), width, height, fy, fy,
                  width / 2.0, height / 2.0, near_plane, far_plane)


def orbit_cameras(n_views: int, radius: float, width: int, height: int, fov_y_deg: float = 60.0,
                  step_deg: float | None = None) -> list[Camera]:
    """Views on the equator (y = 0) around the origin, all looking at it."""
    step = math.radians(step_deg if step_deg is not None else 360.0 / n_views)
    cams = []
    for i in range(n_views):
        a = i * step
        cams.append(pinhole((radius * math.sin(a), 0.0, -radius * math.cos(a)), width, height, fov_y_deg))
    return cams


def front_camera(width: int = 640, height: int = 480, distance: float = 4.0, fov_y_deg: float = 60.0) -> Camera:
    """Camera at (0, 0, -distance) looking at the origin: w2c = [I | (0, 0, distance)]."""
    return pinhole((0.0, 0.0, -distance), width, height, fov_y_deg)


def synthetic_blue_noise(seed: int = 0) -> torch.Tensor:
    """A uint8 (64, 128, 128) volume with the layout of the STBN scalar volume (a hashed stand-in:
    NVIDIA's texture is not redistributable and there is no network). Deterministic on any machine:
    byte i is the top byte of a 32-bit integer hash of (i, seed)."""
    x = torch.arange(64 * 128 * 128, dtype=torch.int64) ^ (seed * 0x9E3779B9)
    m = 0xFFFFFFFF
    x = x & m
    x = x ^ (x >> 16)
    x = (x * 0x7FEB352D) & m
    x = x ^ (x >> 15)
    x = (x * 0x846CA68B) & m
    x = x ^ (x >> 16)
    return (x >> 24).to(torch.uint8).view(64, 128, 128)
