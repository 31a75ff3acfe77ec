"""Loads and stores 3D Gaussian splatting models in the .ply layout the reference's model reads.

`load_ply(path)` restates StochasticGSModel.build (Model.py:22-79) without plyfile (absent here): the
vertex element's x, y, z (means), scale_0..2 (log-scales), rot_0..3 (quaternions, r i j k),
opacity (logit), f_dc_0..2 and f_rest_* (SH coefficients, the rest stored channel-major: all bases
of red, then green, then blue, Model.py:72-77), as fp32 tensors in the layouts `render()` takes,
reordered along a Morton curve of the means (Model.py:32-34) so that neighbouring Gaussians sit in
neighbouring warps. The Morton code is this package's (`sgs_scenes.morton_codes`, 10 bits per axis
over the bounding box); the reference's comes from NeRFICG's CudaUtils, which is not available, and
only the order of the Gaussians depends on it.

`save_ply(path, scene)` writes the same layout (binary little endian), for tests and for exporting
synthetic scenes.

The parser reads `binary_little_endian`, `binary_big_endian` and `ascii` files whose first element
is the vertex element with scalar properties (float, double and the integer types); later elements
are ignored.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import torch

import sgs_scenes

_TYPES = {
    "char": "i1", "int8": "i1", "uchar": "u1", "uint8": "u1", "short": "i2", "int16": "i2", "ushort": "u2",
    "uint16": "u2", "int": "i4", "int32": "i4", "uint": "u4", "uint32": "u4", "float": "f4", "float32": "f4",
    "double": "f8", "float64": "f8",
}


def _read_header(f):
    if f.readline().strip() != b"ply":
        raise ValueError("not a PLY file")
    fmt, elements = None, []
    while True:
        line = f.readline()
        if not line:
            raise ValueError("PLY header without end_header")
        words = line.decode("ascii", "replace").split()
        if not words or words[0] in ("comment", "obj_info"):
            continue
        if words[0] == "format":
            fmt = words[1]
        elif words[0] == "element":
            elements.append((words[1], int(words[2]), []))
        elif words[0] == "property":
            if words[1] == "list":
                raise ValueError(f"list property {words[-1]} of element {elements[-1][0]} is not supported")
            if words[1] not in _TYPES:
                raise ValueError(f"unknown PLY property type {words[1]}")
            elements[-1][2].append((words[2], _TYPES[words[1]]))
        elif words[0] == "end_header":
            break
    if fmt not in ("binary_little_endian", "binary_big_endian", "ascii"):
        raise ValueError(f"unsupported PLY format {fmt}")
    if not elements or elements[0][0] != "vertex":
        raise ValueError("the first PLY element must be the vertex element")
    return fmt, elements[0]


def read_ply_vertices(path) -> dict[str, np.ndarray]:
    """The vertex element's properties as arrays, by name."""
    with open(path, "rb") as f:
        fmt, (_, count, props) = _read_header(f)
        if fmt == "ascii":
            rows = np.loadtxt(f, dtype=np.float64, max_rows=count, ndmin=2)
            return {name: rows[:, i].astype(np.dtype(t)) for i, (name, t) in enumerate(props)}
        order = "<" if fmt == "binary_little_endian" else ">"
        dtype = np.dtype([(name, order + t) for name, t in props])
        data = np.frombuffer(f.read(dtype.itemsize * count), dtype=dtype, count=count)
        return {name: data[name] for name, _ in props}


def load_ply(path, device="cuda", morton: bool = True) -> sgs_scenes.Scene:
    """A 3DGS .ply as the five fp32 tensors of `render()` on `device` (Model.py:22-79)."""
    v = read_ply_vertices(path)
    col = lambda names: np.stack([np.asarray(v[n], dtype=np.float32) for n in names], axis=1)
    means = torch.from_numpy(col(("x", "y", "z")))
    scales = torch.from_numpy(col(("scale_0", "scale_1", "scale_2")))
    rotations = torch.from_numpy(col(("rot_0", "rot_1", "rot_2", "rot_3")))
    opacities = torch.from_numpy(np.asarray(v["opacity"], dtype=np.float32).copy())
    n_rest = len([name for name in v if name.startswith("f_rest_")])
    if n_rest % 3 != 0 or (n_rest // 3 + 1) not in (1, 4, 9, 16):
        raise ValueError(f"{n_rest} f_rest_ properties do not form degree 0-3 SH")
    bases = n_rest // 3 + 1
    sh = torch.empty((means.shape[0], bases, 3), dtype=torch.float32)
    sh[:, 0, :] = torch.from_numpy(col(("f_dc_0", "f_dc_1", "f_dc_2")))
    if bases > 1:
        rest = torch.from_numpy(col([f"f_rest_{i}" for i in range(n_rest)]))
        sh[:, 1:, :] = rest.reshape(-1, 3, bases - 1).permute(0, 2, 1)
    scene = sgs_scenes.Scene(means, scales, rotations, opacities, sh)
    if morton:
        order = torch.argsort(sgs_scenes.morton_codes(means), stable=True)
        scene = sgs_scenes.Scene(*(t[order].contiguous() for t in scene.tensors()))
    return scene.to(device)


def save_ply(path, scene: sgs_scenes.Scene) -> None:
    """Writes a scene in the 3DGS .ply layout (binary little endian, normals zero)."""
    means, scales, rotations, opacities, sh = (t.detach().float().cpu().numpy() for t in scene.tensors())
    n, bases = means.shape[0], sh.shape[1]
    names = ["x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2"]
    names += [f"f_rest_{i}" for i in range(3 * (bases - 1))]
    names += ["opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"]
    rest = sh[:, 1:, :].transpose(0, 2, 1).reshape(n, -1)  # channel-major, as Model.py:76-77 reads it
    cols = np.concatenate([means, np.zeros((n, 3), np.float32), sh[:, 0, :], rest, opacities.reshape(n, 1), scales,
                           rotations], axis=1).astype("<f4")
    header = "ply\nformat binary_little_endian 1.0\nelement vertex %d\n" % n
    header += "".join(f"property float {name}\n" for name in names) + "end_header\n"
    Path(path).write_bytes(header.encode("ascii") + np.ascontiguousarray(cols).tobytes())
