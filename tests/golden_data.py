"""Loader of the golden fixtures in tests/golden/ (outputs of the reference CUDA backend).

tests/golden/make_golden.py produced them on a B200 from the reference's own kernels; the scene
inputs are stored beside them so that no RNG is involved when they are read back.
"""
from __future__ import annotations

import json
from functools import lru_cache
from pathlib import Path

import numpy as np

GOLDEN_DIR = Path(__file__).resolve().parent / "golden"


@lru_cache(maxsize=None)
def manifest() -> dict:
    return json.loads((GOLDEN_DIR / "manifest.json").read_text())


@lru_cache(maxsize=None)
def scene(name: str) -> dict[str, np.ndarray]:
    with np.load(GOLDEN_DIR / f"scene_{name}.npz") as z:
        return {k: z[k] for k in z.files}


def case(name: str) -> dict[str, np.ndarray]:
    with np.load(GOLDEN_DIR / f"case_{name}.npz") as z:
        return {k: z[k] for k in z.files}


def sequence(name: str) -> dict[str, np.ndarray]:
    with np.load(GOLDEN_DIR / f"seq_{name}.npz") as z:
        return {k: z[k] for k in z.files}


def blue_noise() -> np.ndarray:
    import sgs_scenes

    return sgs_scenes.synthetic_blue_noise(0).numpy()


SCENE_KEYS = ("means", "scales", "rotations", "opacities", "sh_coefficients")
