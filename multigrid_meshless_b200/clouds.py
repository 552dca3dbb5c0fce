"""Seeded synthetic point clouds standing in for the reference's Gmsh meshes.

The reference reads Gmsh v2 files (mesh_functions.h:172-476) and leaves each
level in this state: boundary nodes first (indices < num_boundary_nodes), no
corner nodes (they are deleted, mesh_functions.h:434-473), raw boundary normals
that correct_normal_directions later flips outward and normalises
(mesh_functions.h:478-527).  These generators produce exactly that state from a
counter-based splitmix64 stream, so every cloud is reproducible from
(kind, size, seed) alone and no mesh file is needed.

Kinds
  cavity2d(m)      unit square, m x m Cartesian nodes, interior jittered by
                   U(-0.25h, 0.25h) per coordinate, boundary nodes evenly spaced
                   on the edges, the 4 corners removed.
  annulus2d(h)     r in [0.5, 1], jittered polar rings of roughly uniform
                   density; the two boundary rings evenly spaced in theta.
  cube3d(m)        unit cube, m^3 nodes, interior jittered by U(-0.25h, 0.25h),
                   face nodes evenly spaced, edge and corner nodes removed
                   (Gmsh line/point elements are corner-tagged, mesh_functions.h:396-413).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def _splitmix64(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = x + _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def uniform(seed: int, stream: int, n: int) -> np.ndarray:
    """n doubles in [0, 1) from counter (seed, stream, 0..n-1)."""
    with np.errstate(over="ignore"):
        base = _splitmix64(np.uint64(seed) * np.uint64(0xD1B54A32D192ED03) + np.uint64(stream))
        ctr = base + np.arange(n, dtype=np.uint64) * _GOLDEN
    return (_splitmix64(ctr) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


@dataclass
class Cloud:
    """One multigrid level's nodes in the reference's post-read state."""
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    nx: np.ndarray
    ny: np.ndarray
    nz: np.ndarray
    btag: np.ndarray            # uint8, 1 on boundary nodes
    nb: int                     # boundary nodes occupy indices [0, nb)
    dim: int
    h: float                    # nominal spacing (used as the reference's d_avg seed)
    kind: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.x.shape[0])


def cavity2d(m: int, seed: int = 1) -> Cloud:
    if m < 3:
        raise ValueError("cavity2d needs m >= 3")
    h = 1.0 / (m - 1)
    t = np.arange(1, m - 1, dtype=np.float64) * h
    one = np.ones(m - 2)
    zero = np.zeros(m - 2)
    # edges without corners, walked counter-clockwise: bottom, right, top, left
    bx = np.concatenate([t, one, t[::-1], zero])
    by = np.concatenate([zero, t, one, t[::-1]])
    bnx = np.concatenate([zero, one, zero, -one])
    bny = np.concatenate([-one, zero, one, zero])
    ii, jj = np.meshgrid(np.arange(1, m - 1), np.arange(1, m - 1), indexing="xy")
    ii = ii.ravel().astype(np.float64)
    jj = jj.ravel().astype(np.float64)
    ni = ii.shape[0]
    jx = (uniform(seed, 0, ni) - 0.5) * 0.5 * h
    jy = (uniform(seed, 1, ni) - 0.5) * 0.5 * h
    x = np.concatenate([bx, ii * h + jx])
    y = np.concatenate([by, jj * h + jy])
    nb = bx.shape[0]
    n = x.shape[0]
    btag = np.zeros(n, np.uint8)
    btag[:nb] = 1
    nx = np.zeros(n); ny = np.zeros(n)
    nx[:nb] = bnx; ny[:nb] = bny
    return Cloud(x, y, np.zeros(n), nx, ny, np.zeros(n), btag, nb, 2, h, "cavity2d", {"m": m, "seed": seed})


def annulus2d(h: float, seed: int = 1, r_in: float = 0.5, r_out: float = 1.0) -> Cloud:
    nr = max(2, int(round((r_out - r_in) / h)))
    dr = (r_out - r_in) / nr
    xs, ys, nxs, nys, bt = [], [], [], [], []
    inner = []
    for ring in range(nr + 1):
        r = r_in + ring * dr
        nt = max(8, int(round(2.0 * math.pi * r / h)))
        dth = 2.0 * math.pi / nt
        th = (np.arange(nt) + 0.5 * (ring % 2)) * dth
        if ring == 0 or ring == nr:
            sgn = -1.0 if ring == 0 else 1.0
            # evaluate r*cos/sin so that |r - r_wall| < 1e-9 holds (init_TC.c:37 test)
            xs.append(r * np.cos(th)); ys.append(r * np.sin(th))
            nxs.append(sgn * np.cos(th)); nys.append(sgn * np.sin(th))
            bt.append(np.ones(nt, np.uint8))
        else:
            inner.append((ring, r, nt, dth, th))
    # interior rings, jittered in r and theta
    ix, iy = [], []
    for (ring, r, nt, dth, th) in inner:
        jr = (uniform(seed, 2 * ring, nt) - 0.5) * 0.5 * dr
        jt = (uniform(seed, 2 * ring + 1, nt) - 0.5) * 0.5 * dth
        rr = r + jr
        tt = th + jt
        ix.append(rr * np.cos(tt)); iy.append(rr * np.sin(tt))
    bx = np.concatenate(xs); by = np.concatenate(ys)
    nb = bx.shape[0]
    x = np.concatenate([bx] + ix); y = np.concatenate([by] + iy)
    n = x.shape[0]
    btag = np.zeros(n, np.uint8); btag[:nb] = 1
    nx = np.zeros(n); ny = np.zeros(n)
    nx[:nb] = np.concatenate(nxs); ny[:nb] = np.concatenate(nys)
    return Cloud(x, y, np.zeros(n), nx, ny, np.zeros(n), btag, nb, 2, h, "annulus2d",
                 {"h": h, "seed": seed, "r_in": r_in, "r_out": r_out})


def cube3d(m: int, seed: int = 1) -> Cloud:
    if m < 3:
        raise ValueError("cube3d needs m >= 3")
    h = 1.0 / (m - 1)
    g = np.arange(m)
    I, J, K = np.meshgrid(g, g, g, indexing="ij")
    I = I.ravel(); J = J.ravel(); K = K.ravel()
    onb = (I == 0).astype(int) + (I == m - 1) + (J == 0) + (J == m - 1) + (K == 0) + (K == m - 1)
    face = onb == 1
    inside = onb == 0
    fi, fj, fk = I[face], J[face], K[face]
    fx = fi * h; fy = fj * h; fz = fk * h
    fnx = np.where(fi == 0, -1.0, np.where(fi == m - 1, 1.0, 0.0))
    fny = np.where(fj == 0, -1.0, np.where(fj == m - 1, 1.0, 0.0))
    fnz = np.where(fk == 0, -1.0, np.where(fk == m - 1, 1.0, 0.0))
    ci, cj, ck = I[inside], J[inside], K[inside]
    ni = ci.shape[0]
    x = np.concatenate([fx, ci * h + (uniform(seed, 0, ni) - 0.5) * 0.5 * h])
    y = np.concatenate([fy, cj * h + (uniform(seed, 1, ni) - 0.5) * 0.5 * h])
    z = np.concatenate([fz, ck * h + (uniform(seed, 2, ni) - 0.5) * 0.5 * h])
    nb = fx.shape[0]
    n = x.shape[0]
    btag = np.zeros(n, np.uint8); btag[:nb] = 1
    nx = np.zeros(n); ny = np.zeros(n); nz = np.zeros(n)
    nx[:nb] = fnx; ny[:nb] = fny; nz[:nb] = fnz
    return Cloud(x, y, z, nx, ny, nz, btag, nb, 3, h, "cube3d", {"m": m, "seed": seed})


def cavity_hierarchy(m: int, levels: int, seed: int = 1) -> list[Cloud]:
    """Fine level m x m, each coarser level with half the spacing count."""
    out = []
    for l in range(levels):
        out.append(cavity2d(m, seed + l))
        m = max(3, (m + 1) // 2) if l == 0 and m % 2 == 1 else max(3, m // 2)
    return out


def annulus_hierarchy(h: float, levels: int, seed: int = 1) -> list[Cloud]:
    """Fine spacing h, each coarser level at twice the spacing (4x fewer nodes)."""
    return [annulus2d(h * (2 ** l), seed + l) for l in range(levels)]


def annulus_h_for_nodes(n_target: int, r_in: float = 0.5, r_out: float = 1.0) -> float:
    return math.sqrt(math.pi * (r_out * r_out - r_in * r_in) / n_target)


def cube_hierarchy(m: int, levels: int, seed: int = 1) -> list[Cloud]:
    out = []
    for l in range(levels):
        out.append(cube3d(m, seed + l))
        m = max(3, m // 2)
    return out
