"""Seeded synthetic porous media in the reference's mask conventions.

A mask is one byte per node, x fastest (n = i + LX*(j + LY*k)), with 1 for
solid and 0 for fluid: the convention of the reference's .raw volumes
(src/lbio.c:542-559) and of the device rule solid iff byte == 1
(src/lattice.c:2314).  Writers for the reference's file formats (24-bit BMP
with black = solid, raw bytes) live in lbx.formats.
"""
from __future__ import annotations

import numpy as np


def sphere_pack(LX: int, LY: int, LZ: int, radius: int, porosity: float,
                seed: int, periodic: bool = True) -> np.ndarray:
    """Overlapping spheres with uniform random centres, added until the
    fluid fraction is <= porosity.  Periodic wrap on every axis."""
    rng = np.random.default_rng(seed)
    sol = np.zeros((LZ, LY, LX), dtype=np.uint8)
    N = LX * LY * LZ
    target_solid = int(np.ceil((1.0 - porosity) * N))
    r = int(radius)
    off = np.arange(-r, r + 1)
    dz, dy, dx = np.meshgrid(off, off, off, indexing="ij")
    ball = (dx * dx + dy * dy + dz * dz) <= r * r
    bz, by, bx = dz[ball], dy[ball], dx[ball]
    nsolid = 0
    while nsolid < target_solid:
        cx, cy, cz = rng.integers(0, LX), rng.integers(0, LY), rng.integers(0, LZ)
        xs, ys, zs = cx + bx, cy + by, cz + bz
        if periodic:
            xs %= LX; ys %= LY; zs %= LZ
        else:
            keep = (xs >= 0) & (xs < LX) & (ys >= 0) & (ys < LY) & (zs >= 0) & (zs < LZ)
            xs, ys, zs = xs[keep], ys[keep], zs[keep]
        before = sol[zs, ys, xs]
        nsolid += int(np.count_nonzero(before == 0))
        sol[zs, ys, xs] = 1
    return sol.reshape(-1)


def disc_pack(LX: int, LY: int, radius: int, porosity: float, seed: int,
              keep_x_fluid: bool = True, wrap_y: bool = True,
              max_tries: int = 200000) -> np.ndarray:
    """Non-overlapping discs placed by rejection until the fluid fraction is
    <= porosity (or no further disc fits).  Wrapped in y, clipped in x; with
    keep_x_fluid the columns x = 0 and x = LX-1 stay fluid."""
    rng = np.random.default_rng(seed)
    sol = np.zeros((LY, LX), dtype=np.uint8)
    r = int(radius)
    centres = []
    target_solid = (1.0 - porosity) * LX * LY
    jj, ii = np.mgrid[0:LY, 0:LX]
    tries = 0
    while np.count_nonzero(sol) < target_solid and tries < max_tries:
        tries += 1
        cx, cy = rng.uniform(0, LX), rng.uniform(0, LY)
        ok = True
        for (px, py) in centres:
            ddx = cx - px
            ddy = cy - py
            if wrap_y:
                ddy = (ddy + LY / 2) % LY - LY / 2
            if ddx * ddx + ddy * ddy < (2 * r) ** 2:
                ok = False
                break
        if not ok:
            continue
        centres.append((cx, cy))
        ddx = ii - cx
        ddy = jj - cy
        if wrap_y:
            ddy = (ddy + LY / 2) % LY - LY / 2
        sol[(ddx * ddx + ddy * ddy) <= r * r] = 1
        if keep_x_fluid:
            sol[:, 0] = 0
            sol[:, LX - 1] = 0
    return sol.reshape(-1)


def transpose_2d(mask: np.ndarray, LX: int, LY: int) -> np.ndarray:
    """Swap the axes of a 2D mask (n = i + LX*j) -> (n' = j + LY*i)."""
    return np.ascontiguousarray(mask.reshape(LY, LX).T).reshape(-1)


def porosity(mask: np.ndarray) -> float:
    return float(np.count_nonzero(mask != 1)) / mask.size
