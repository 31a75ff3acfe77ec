"""Builds and wraps the C++ CPU restatement of the render path (oracle/sgs_oracle.cpp). TEST INFRASTRUCTURE.

`build()` compiles oracle/_cpu/libsgs_oracle.so with g++ (OpenMP, -ffp-contract=off so that only the
fused multiply-adds written out in the source are fused). The wrappers take and return numpy arrays.
"""
from __future__ import annotations

import ctypes
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
SOURCE = ORACLE_DIR / "sgs_oracle.cpp"
LIB = ORACLE_DIR / "_cpu" / "libsgs_oracle.so"
CXXFLAGS = ["-O3", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared"]


def build(force: bool = False) -> Path:
    if not force and LIB.is_file() and LIB.stat().st_mtime >= SOURCE.stat().st_mtime:
        return LIB
    LIB.parent.mkdir(exist_ok=True)
    tmp = LIB.with_suffix(".tmp.so")
    # the system g++ (the image's $CXX wrapper lacks OpenMP)
    cmd = [shutil.which("g++") or "g++", *CXXFLAGS, str(SOURCE), "-o", str(tmp)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{res.stderr}")
    os.replace(tmp, LIB)
    return LIB


class Stats(ctypes.Structure):
    _fields_ = [("fragments", ctypes.c_uint64), ("accepted", ctypes.c_uint64), ("binned", ctypes.c_uint64)]


_lib = None
_P = ctypes.c_void_p


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        l = ctypes.CDLL(str(build()))
        f, u, i = ctypes.c_float, ctypes.c_uint32, ctypes.c_int
        l.oracle_project.argtypes = [_P, _P, _P, _P, u, _P, u, u, f, f, f, f, f, f, i, i, _P]
        l.oracle_accumulate.argtypes = [_P, _P, _P, _P, u, _P, u, u, f, f, f, f, f, f, i, i, i, i, _P, u, u, u, i, _P,
                                        ctypes.POINTER(Stats)]
        l.oracle_sample_resolve.argtypes = [_P, _P, _P, _P, _P, u, u, _P, _P, u, u, f, f, f, f, f, f, i, i, i, _P, _P, _P,
                                            _P, _P, _P, _P, _P, i, i, _P, _P, _P, _P, _P, _P]
        l.oracle_fragment_alpha.argtypes = [_P, _P, _P, _P, u, _P, u, u, f, f, f, f, f, f, i, i, u, u,
                                            ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double)]
        _lib = l
    return _lib


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _cam(cam: dict):
    return (cam["width"], cam["height"], cam["focal_x"], cam["focal_y"], cam["center_x"], cam["center_y"],
            cam["near_plane"], cam["far_plane"])


def project(scene: dict, cam: dict, aa: bool = False, ss: int = 1) -> np.ndarray:
    m, s, r, o = (_f32(scene[k]) for k in ("means", "scales", "rotations", "opacities"))
    n = m.shape[0]
    out = np.zeros((n, 18), dtype=np.float32)
    w2c = _f32(cam["w2c"])
    lib().oracle_project(_p(m), _p(s), _p(r), _p(o), n, _p(w2c), *_cam(cam), int(aa), int(ss), _p(out))
    return out


def accumulate(scene: dict, cam: dict, flags: dict, frame_idx: int, blue_noise=None, max_fragments: int = 0,
               max_binned: int = 0, threads: int = 0, return_stats: bool = False):
    """Winner framebuffer (int64, P_fb) of one sample-frame; optional fragment statistics."""
    m, s, r, o = (_f32(scene[k]) for k in ("means", "scales", "rotations", "opacities"))
    n = m.shape[0]
    ss = max(1, int(flags["ss"]))
    fb = np.empty(cam["width"] * cam["height"] * ss * ss, dtype=np.uint64)
    bn = None if blue_noise is None else np.ascontiguousarray(np.asarray(blue_noise, dtype=np.uint8))
    st = Stats()
    lib().oracle_accumulate(_p(m), _p(s), _p(r), _p(o), n, _p(_f32(cam["w2c"])), *_cam(cam), int(flags["aa"]), ss,
                            int(flags["gps"]), int(flags["hybrid"]), _p(bn), int(frame_idx) & 0xFFFFFFFF,
                            int(max_fragments), int(max_binned), int(threads), _p(fb), ctypes.byref(st))
    fb = fb.view(np.int64)
    if return_stats:
        return fb, {"fragments": st.fragments, "accepted": st.accepted, "binned": st.binned}
    return fb


def sample_resolve(scene: dict, cam: dict, flags: dict, fb: np.ndarray, *, spatial_reuse: bool = False,
                   k_buffer=None, history=None, v2pv=None, temporal_mode: int = 0, threads: int = 0) -> dict:
    """samples, reuse weights, outputs and the updated k-buffer for a winner framebuffer."""
    m, s, r, o, sh = (_f32(scene[k]) for k in ("means", "scales", "rotations", "opacities", "sh_coefficients"))
    n, bases = m.shape[0], sh.shape[1]
    ss = max(1, int(flags["ss"]))
    W, H = cam["width"], cam["height"]
    n_fb, n_px = W * H * ss * ss, W * H
    samples = np.zeros((n_fb, 4), dtype=np.float32)
    reuse = np.zeros((n_fb, 4), dtype=np.float32) if spatial_reuse else None
    if spatial_reuse:
        kp = np.array(k_buffer[0], dtype=np.int32, copy=True) if k_buffer is not None else np.full((4, n_fb, 2), -1, np.int32)
        ko = np.array(k_buffer[1], dtype=np.float32, copy=True) if k_buffer is not None else np.full((4, n_fb, 4), 0.5, np.float32)
    else:
        kp = ko = None
    hist = [None] * 4 if history is None or temporal_mode == 0 else [_f32(h) for h in history]
    v = _f32(v2pv if v2pv is not None else np.eye(4))
    image = np.zeros((H, W, 3), np.float32)
    depth = np.zeros((H, W, 1), np.float32)
    alpha = np.zeros((H, W, 1), np.float32)
    wm = np.zeros((H, W, 1), np.float32)
    fbu = np.ascontiguousarray(fb.astype(np.int64)).view(np.uint64)
    lib().oracle_sample_resolve(_p(m), _p(s), _p(r), _p(o), _p(sh), n, bases, _p(_f32(cam["w2c"])),
                                _p(_f32(cam["position"])), *_cam(cam), int(flags["aa"]), ss, int(spatial_reuse),
                                _p(fbu), _p(kp), _p(ko), *(_p(h) for h in hist), _p(v), int(temporal_mode),
                                int(threads), _p(samples), _p(reuse), _p(image), _p(depth), _p(alpha), _p(wm))
    return {"samples": samples, "reuse": reuse, "image": image, "depth": depth, "alpha": alpha, "weight_mass": wm,
            "k_buffer": (kp, ko) if spatial_reuse else None}


def fragment_alpha(scene: dict, cam: dict, g: int, px: int, py: int, aa: bool = False, ss: int = 1):
    m, s, r, o = (_f32(scene[k]) for k in ("means", "scales", "rotations", "opacities"))
    af, ad = ctypes.c_float(), ctypes.c_double()
    active = lib().oracle_fragment_alpha(_p(m), _p(s), _p(r), _p(o), int(g), _p(_f32(cam["w2c"])), *_cam(cam),
                                         int(aa), int(ss), int(px), int(py), ctypes.byref(af), ctypes.byref(ad))
    return bool(active), af.value, ad.value


def st_uniform(frame: int, g: int, x: int, y: int) -> float:
    """The reference's white-noise threshold (math_utils.h:113-122), exact."""
    M = 0xFFFFFFFF
    seed = (g ^ (frame * 1973) ^ (x * 9277) ^ (y * 2699)) & M
    state = (seed * 747796405 + 2891336453) & M
    word = (((state >> ((state >> 28) + 4)) ^ state) * 277803737) & M
    h = ((word >> 22) ^ word) & M
    bits = 0x3F800000 | (h >> 9)
    return float(np.array([bits], dtype=np.uint32).view(np.float32)[0]) - 1.0


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def expected_image(scene: dict, cam: dict, ss: int = 1, base: dict | None = None, g_image=None, g_alpha=None,
                   g_depth=None, grad: bool = False, aa: bool = False, gps: bool = False, quad: int = 8,
                   max_fragments: int = 0) -> dict:
    """Expected image of one stochastic-transparency sample (double precision) and, with `grad`, the
    gradient of sum(g_image * image + g_alpha * alpha + g_depth * depth) w.r.t. every parameter.
    The fragment support and key order are frozen at `base` (single precision; default: `scene`).
    `aa`: proper antialiasing (smaller dilation, opacity scaled by sqrt(det / det dilated)).
    `gps`: Gaussian point splatting instead, each fragment's alpha replaced by the probability that
    the Gaussian puts a point into the (sub)pixel, its pixel integrals by an order-`quad`
    Gauss-Legendre rule per axis, and the point count capped at `max_fragments` as the render caps it
    (0: the render's default cap, < 0: no cap)."""
    l = lib()
    P, u, d, i = _P, ctypes.c_uint32, ctypes.c_double, ctypes.c_int
    args = [P, P, P, P, P, u, u, P, P, u, u, d, d, d, d, d, d, i, i, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P]
    if not hasattr(l.oracle_expected_image, "_typed"):
        l.oracle_expected_image.argtypes = args
        l.oracle_expected_image._typed = True
        l.oracle_expected_image_gps.argtypes = args + [i, i]
    base = scene if base is None else base
    m, s, r, o, sh = (_f64(scene[k]) for k in ("means", "scales", "rotations", "opacities", "sh_coefficients"))
    bm, bs, br, bo = (_f32(base[k]) for k in ("means", "scales", "rotations", "opacities"))
    n, bases = m.shape[0], sh.shape[1]
    W, H = cam["width"], cam["height"]
    image = np.zeros((H, W, 3))
    alpha = np.zeros((H, W, 1))
    depth = np.zeros((H, W, 1))
    loss = ctypes.c_double(0.0)
    gi = None if g_image is None else _f64(g_image)
    ga = None if g_alpha is None else _f64(g_alpha)
    gd = None if g_depth is None else _f64(g_depth)
    out = {}
    if grad:
        out = {"means": np.zeros_like(m), "scales": np.zeros_like(s), "rotations": np.zeros_like(r),
               "opacities": np.zeros_like(o), "sh_coefficients": np.zeros_like(sh)}
    w2c = _f64(np.asarray(cam["w2c"])[:3].reshape(-1))
    call = (_p(m), _p(s), _p(r), _p(o), _p(sh), n, bases, _p(w2c), _p(_f64(cam["position"])), W, H, cam["focal_x"],
            cam["focal_y"], cam["center_x"], cam["center_y"], cam["near_plane"], cam["far_plane"], int(ss), int(aa),
            _p(bm), _p(bs), _p(br), _p(bo), _p(gi), _p(ga), _p(gd), _p(image), _p(alpha), _p(depth),
            ctypes.byref(loss),
            *(_p(out[k]) if grad else None for k in ("means", "scales", "rotations", "opacities", "sh_coefficients")))
    if gps:
        l.oracle_expected_image_gps(*call, int(quad), int(max_fragments))
    else:
        l.oracle_expected_image(*call)
    return {"image": image, "alpha": alpha, "depth": depth, "loss": loss.value, "grad": out if grad else None}


def gps_count_law(lam: float, cap: int = 4096) -> tuple[np.ndarray, np.ndarray]:
    """Law of the GPS point count at importance `lam` (the Cornish-Fisher draw of the render, exact up
    to its rounding): (P(N = n), dP(N = n) / dlam) for n = 0, 1, ..."""
    l = lib()
    if not hasattr(l.oracle_gps_count_law, "_typed"):
        l.oracle_gps_count_law.argtypes = [ctypes.c_double, _P, _P, ctypes.c_int]
        l.oracle_gps_count_law.restype = ctypes.c_int
        l.oracle_gps_count_law._typed = True
    P = np.zeros(cap)
    dP = np.zeros(cap)
    k = l.oracle_gps_count_law(float(lam), _p(P), _p(dP), cap)
    return P[:min(k, cap)], dP[:min(k, cap)]
