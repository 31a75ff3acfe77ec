"""Index arithmetic of the tiled resolve (tile_resolve_kernel, csrc/sample_resolve.cu), restated on the CPU.

A block resolves a 32 x 8 tile of image pixels. It stages the tile's framebuffer subpixels with a halo
(one subpixel with spatial reuse, ss subpixels for Reproject's 3 x 3 moment windows) and, for Reproject,
the box-filtered colours of the tile's pixels and a one-pixel ring clamped to the image. These tests
check, for many image sizes and supersampling factors, that every subpixel the resolve reads lies in
the staged rectangle, that in the fused pass each framebuffer subpixel's sample is written by exactly one
tile, and that the staged bytes match the layout the launcher sizes.
"""
import math
import random

import pytest

TILE_W, TILE_H = 32, 8
RING_W, RING_H = TILE_W + 2, TILE_H + 2
HIST_FLOATS = 5
MIN_HIST_BYTES = 24 << 10
MAX_TILE_BYTES = 200 << 10


def tile_layout(ss: int, reuse: bool, reproject: bool) -> dict:
    halo = ss if reproject else (1 if reuse else 0)
    sw, sh = TILE_W * ss + 2 * halo, TILE_H * ss + 2 * halo
    n = sw * sh
    off = n * 16 + (n * 16 if reuse else 0)
    hist_cap = 0
    if reproject:
        off = max(off, MIN_HIST_BYTES)
        hist_cap = off // (HIST_FLOATS * 4)
        off += RING_W * RING_H * 12
    return dict(halo=halo, sw=sw, sh=sh, bytes=off, hist_cap=hist_cap)


def reads_of_tile(tx0, ty0, width, height, ss, reuse, reproject):
    """Framebuffer subpixels the tile's threads read (box filter, reuse neighbours, moment ring)."""
    fbw, fbh = width * ss, height * ss
    reads = set()
    for t in range(TILE_W * TILE_H):
        x, y = tx0 + t % TILE_W, ty0 + t // TILE_W
        px, py = min(x, width - 1), min(y, height - 1)
        for sy in range(ss):
            for sx in range(ss):
                fx, fy = px * ss + sx, py * ss + sy
                reads.add((fx, fy))
                if reuse:
                    if fx > 0:
                        reads.add((fx - 1, fy))
                    if fx < fbw - 1:
                        reads.add((fx + 1, fy))
                    if fy > 0:
                        reads.add((fx, fy - 1))
                    if fy < fbh - 1:
                        reads.add((fx, fy + 1))
    if reproject:
        for j in range(RING_W * RING_H):
            qx = min(max(tx0 - 1 + j % RING_W, 0), width - 1)
            qy = min(max(ty0 - 1 + j // RING_W, 0), height - 1)
            for sy in range(ss):
                for sx in range(ss):
                    reads.add((qx * ss + sx, qy * ss + sy))
    return reads


@pytest.mark.parametrize("seed", range(6))
def test_reads_stay_inside_the_staged_rectangle(seed):
    rng = random.Random(seed)
    for _ in range(6):
        width, height = rng.randint(1, 80), rng.randint(1, 30)
        ss = rng.randint(1, 3)
        reuse, reproject = rng.random() < 0.6, rng.random() < 0.6
        if not (reuse or reproject):
            reuse = True
        L = tile_layout(ss, reuse, reproject)
        for ty0 in range(0, height, TILE_H):
            for tx0 in range(0, width, TILE_W):
                ox, oy = tx0 * ss - L["halo"], ty0 * ss - L["halo"]
                for fx, fy in reads_of_tile(tx0, ty0, width, height, ss, reuse, reproject):
                    assert 0 <= fx < width * ss and 0 <= fy < height * ss
                    assert 0 <= fx - ox < L["sw"] and 0 <= fy - oy < L["sh"], (fx, fy, tx0, ty0, ss)


@pytest.mark.parametrize("width,height,ss", [(1, 1, 1), (33, 9, 1), (64, 16, 2), (70, 17, 3), (31, 7, 2)])
def test_fused_pass_writes_each_sample_once(width, height, ss):
    written = {}
    for ty0 in range(0, height, TILE_H):
        for tx0 in range(0, width, TILE_W):
            L = tile_layout(ss, False, True)
            ox, oy = tx0 * ss - L["halo"], ty0 * ss - L["halo"]
            for i in range(L["sw"] * L["sh"]):
                fx, fy = ox + i % L["sw"], oy + i // L["sw"]
                inside = 0 <= fx < width * ss and 0 <= fy < height * ss
                own = inside and tx0 * ss <= fx < (tx0 + TILE_W) * ss and ty0 * ss <= fy < (ty0 + TILE_H) * ss
                if own:
                    written[(fx, fy)] = written.get((fx, fy), 0) + 1
    assert len(written) == width * height * ss * ss and set(written.values()) == {1}


def test_layout_sizes():
    # supersampling 2 with spatial reuse and Reproject stays below the 48 KB static limit
    assert tile_layout(2, True, True)["bytes"] < 48 << 10
    assert tile_layout(4, True, True)["bytes"] <= MAX_TILE_BYTES
    assert tile_layout(5, True, True)["bytes"] > MAX_TILE_BYTES  # read from global memory instead
    for ss in range(1, 5):
        for reuse in (False, True):
            assert tile_layout(ss, reuse, True)["hist_cap"] >= 1228


def test_history_taps_stay_inside_the_image():
    """A pixel uses its history only when its reprojection lies at least 2 pixels inside the image: the
    4 x 4 Catmull-Rom taps from floor(p - 0.5) - 1 then stay in [0, W - 1]."""
    rng = random.Random(3)
    for _ in range(20000):
        width = rng.randint(4, 4000)
        ppx = rng.uniform(2.0, width - 2.0)
        hx = int(math.floor(ppx - 0.5)) - 1
        assert 0 <= hx and hx + 3 <= width - 1
