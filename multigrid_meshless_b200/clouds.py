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
  shell3d(h)       spherical shell r in [0.5, 1]: interior nodes by rejection
                   of a jittered Cartesian lattice of spacing h (uniform
                   density), boundary nodes on both spheres by a Fibonacci
                   lattice of matching spacing.
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


def _fibonacci_sphere(count: int, r: float):
    i = np.arange(count, dtype=np.float64) + 0.5
    zc = 1.0 - 2.0 * i / count
    rho = np.sqrt(np.maximum(0.0, 1.0 - zc * zc))
    th = math.pi * (3.0 - math.sqrt(5.0)) * i
    return rho * np.cos(th), rho * np.sin(th), zc


def shell3d(h: float, seed: int = 1, r_in: float = 0.5, r_out: float = 1.0) -> Cloud:
    """Shell r in [r_in, r_out]; nodes at spacing about h.  Interior: lattice
    points of spacing h jittered by U(-0.25h, 0.25h), kept when their radius
    lies in [r_in + 0.5h, r_out - 0.5h].  Boundary: Fibonacci points on each
    sphere, one per h^2 of area, normals pointing out of the fluid."""
    m = int(math.ceil(2.0 * r_out / h)) + 1
    g = (np.arange(m, dtype=np.float64) - 0.5 * (m - 1)) * h
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    X = X.ravel(); Y = Y.ravel(); Z = Z.ravel()
    nt = X.shape[0]
    X = X + (uniform(seed, 0, nt) - 0.5) * 0.5 * h
    Y = Y + (uniform(seed, 1, nt) - 0.5) * 0.5 * h
    Z = Z + (uniform(seed, 2, nt) - 0.5) * 0.5 * h
    R = np.sqrt(X * X + Y * Y + Z * Z)
    keep = (R >= r_in + 0.5 * h) & (R <= r_out - 0.5 * h)
    ix, iy, iz = X[keep], Y[keep], Z[keep]
    bxs, bys, bzs, nxs, nys, nzs = [], [], [], [], [], []
    for r, sgn in ((r_in, -1.0), (r_out, 1.0)):
        cnt = max(12, int(round(4.0 * math.pi * r * r / (h * h))))
        ux, uy, uz = _fibonacci_sphere(cnt, r)
        bxs.append(r * ux); bys.append(r * uy); bzs.append(r * uz)
        nxs.append(sgn * ux); nys.append(sgn * uy); nzs.append(sgn * uz)
    bx = np.concatenate(bxs); by = np.concatenate(bys); bz = np.concatenate(bzs)
    nb = bx.shape[0]
    x = np.concatenate([bx, ix]); y = np.concatenate([by, iy]); z = np.concatenate([bz, iz])
    n = x.shape[0]
    btag = np.zeros(n, np.uint8); btag[:nb] = 1
    nx = np.zeros(n); ny = np.zeros(n); nz = np.zeros(n)
    nx[:nb] = np.concatenate(nxs); ny[:nb] = np.concatenate(nys); nz[:nb] = np.concatenate(nzs)
    return Cloud(x, y, z, nx, ny, nz, btag, nb, 3, h, "shell3d", {"h": h, "seed": seed, "r_in": r_in, "r_out": r_out})


def shell_h_for_nodes(n_target: int, r_in: float = 0.5, r_out: float = 1.0) -> float:
    """Spacing giving about n_target interior plus boundary nodes."""
    vol = 4.0 / 3.0 * math.pi * (r_out ** 3 - r_in ** 3)
    return (vol / n_target) ** (1.0 / 3.0)


def shell_hierarchy(h: float, levels: int, seed: int = 1) -> list[Cloud]:
    """Fine spacing h, each coarser level at twice the spacing (8x fewer nodes)."""
    return [shell3d(h * (2 ** l), seed + l) for l in range(levels)]


def shell_stencil_sizes(c: Cloud, k_interior: int, k_boundary: int, band: float = 1.5):
    """Per-node stencil size: k_boundary for boundary nodes and nodes within
    band*h of either sphere, k_interior elsewhere."""
    r = np.sqrt(c.x * c.x + c.y * c.y + c.z * c.z)
    near = (r - c.meta["r_in"] < band * c.h) | (c.meta["r_out"] - r < band * c.h) | (c.btag != 0)
    return np.where(near, k_boundary, k_interior).astype(np.int32)


def gaussian_fields(c: Cloud, count: int, seed: int = 1, bumps: int = 8, wmin: float = 0.1, wmax: float = 0.3):
    """count smooth fields [count][n], each a sum of `bumps` Gaussians with
    amplitude N(0,1), width U(wmin, wmax) and centres uniform in the shell."""
    out = np.zeros((count, c.n))
    r_in, r_out = c.meta.get("r_in", 0.0), c.meta.get("r_out", 1.0)
    for f in range(count):
        u = uniform(seed, 1000 + f, 16 * bumps)
        k = 0
        for b in range(bumps):
            # amplitude N(0,1) by Box-Muller
            a = math.sqrt(-2.0 * math.log(max(u[k], 1e-300))) * math.cos(2.0 * math.pi * u[k + 1]); k += 2
            w = wmin + (wmax - wmin) * u[k]; k += 1
            # centre: uniform in the shell (radius by inverse CDF, direction uniform)
            rr = (r_in ** 3 + u[k] * (r_out ** 3 - r_in ** 3)) ** (1.0 / 3.0); k += 1
            cz = 1.0 - 2.0 * u[k]; k += 1
            ph = 2.0 * math.pi * u[k]; k += 1
            s = math.sqrt(max(0.0, 1.0 - cz * cz))
            cx, cy, cz = rr * s * math.cos(ph), rr * s * math.sin(ph), rr * cz
            d2 = (c.x - cx) ** 2 + (c.y - cy) ** 2 + (c.z - cz) ** 2
            out[f] += a * np.exp(-d2 / (w * w))
    return out
