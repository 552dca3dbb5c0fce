"""Synthetic Gmsh 2.2 ASCII meshes for the mesh-reader tests.

Nodes are numbered as Gmsh numbers them: geometric points first, then the
nodes on curves, then on surfaces, then inside -- the order the reference's
reader relies on when it drops the first num_corners nodes
(mesh_functions.h:434-473).  Element lines carry two tags ("2 <physical>
<geometric>"), as Gmsh writes them.  Coordinates are written with 17
significant digits so that they read back bit for bit.
"""
from __future__ import annotations

import numpy as np


def write_msh(path, nodes, elements):
    """nodes: (N, 3) array; elements: list of (type, geometric_tag, [1-based node ids])."""
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%d\n" % len(nodes))
        for i, (x, y, z) in enumerate(nodes):
            f.write("%d %r %r %r\n" % (i + 1, float(x), float(y), float(z)))
        f.write("$EndNodes\n$Elements\n%d\n" % len(elements))
        for e, (t, tag, ids) in enumerate(elements):
            f.write("%d %d 2 0 %d %s\n" % (e + 1, t, tag, " ".join(str(int(v)) for v in ids)))
        f.write("$EndElements\n")


def square2d(path, m, seed=0, jitter=0.25):
    """Unit square, m nodes per edge: 4 corner points (type 15), boundary
    lines (type 1), jittered interior, Delaunay triangles (type 2)."""
    from scipy.spatial import Delaunay
    rng = np.random.default_rng(seed)
    h = 1.0 / (m - 1)
    t = np.arange(1, m - 1) * h
    corners = [(0.0, 0.0), (1.0, 0.0), (1.0, 1.0), (0.0, 1.0)]
    edges = [[(v, 0.0) for v in t], [(1.0, v) for v in t], [(v, 1.0) for v in t[::-1]], [(0.0, v) for v in t[::-1]]]
    g = np.arange(1, m - 1) * h
    X, Y = np.meshgrid(g, g, indexing="ij")
    inner = np.stack([X.ravel(), Y.ravel()], 1) + rng.uniform(-jitter * h, jitter * h, (X.size, 2))
    pts = [np.array(corners)] + [np.array(e) for e in edges] + [inner]
    xy = np.concatenate(pts)
    nodes = np.concatenate([xy, np.zeros((len(xy), 1))], 1)
    els = [(15, c + 1, [c + 1]) for c in range(4)]
    start = 4
    for ei, e in enumerate(edges):
        ids = [ei + 1] + list(range(start + 1, start + len(e) + 1)) + [(ei + 1) % 4 + 1]
        start += len(e)
        els += [(1, ei + 1, [ids[q], ids[q + 1]]) for q in range(len(ids) - 1)]
    tri = Delaunay(xy).simplices
    els += [(2, 1, list(s + 1)) for s in tri]
    write_msh(path, nodes, els)
    return len(nodes)


def annulus2d(path, h, seed=0, r_in=0.5, r_out=1.0):
    """Annulus: one point per circle (its first node, type 15), closed line
    loops (type 1) on both circles, jittered interior, triangles."""
    from scipy.spatial import Delaunay
    rng = np.random.default_rng(seed)
    nin, nout = int(round(2 * np.pi * r_in / h)), int(round(2 * np.pi * r_out / h))
    ci = [(r_in * np.cos(a), r_in * np.sin(a)) for a in 2 * np.pi * np.arange(nin) / nin]
    co = [(r_out * np.cos(a), r_out * np.sin(a)) for a in 2 * np.pi * np.arange(nout) / nout]
    g = np.arange(-r_out, r_out + h / 2, h)
    X, Y = np.meshgrid(g, g, indexing="ij")
    p = np.stack([X.ravel(), Y.ravel()], 1) + rng.uniform(-0.25 * h, 0.25 * h, (X.size, 2))
    r = np.hypot(p[:, 0], p[:, 1])
    inner = p[(r > r_in + 0.5 * h) & (r < r_out - 0.5 * h)]
    xy = np.concatenate([np.array([ci[0], co[0]]), np.array(ci[1:]), np.array(co[1:]), inner])
    nodes = np.concatenate([xy, np.zeros((len(xy), 1))], 1)
    els = [(15, 1, [1]), (15, 2, [2])]
    loop_in = [1] + list(range(3, 3 + nin - 1))
    loop_out = [2] + list(range(3 + nin - 1, 3 + nin - 1 + nout - 1))
    for tag, loop in ((1, loop_in), (2, loop_out)):
        els += [(1, tag, [loop[q], loop[(q + 1) % len(loop)]]) for q in range(len(loop))]
    tri = Delaunay(xy).simplices
    els += [(2, 3, list(s + 1)) for s in tri]
    write_msh(path, nodes, els)
    return len(nodes)


def cube3d(path, m, seed=0, quads_on_top=True):
    """Unit cube, m nodes per edge: 8 corner points (type 15), 12 edges of
    2-node lines (type 1: the reference tags both ends as corners in 3D),
    boundary faces as triangles (type 2; quads, type 3, on z = 1), jittered
    interior, no volume elements."""
    rng = np.random.default_rng(seed)
    h = 1.0 / (m - 1)
    idx = {}
    nodes = []

    def add(key, p):
        if key not in idx:
            idx[key] = len(nodes) + 1
            nodes.append(p)
        return idx[key]

    def coord(i):
        return i * h

    cube_corners = [(i, j, k) for k in (0, m - 1) for j in (0, m - 1) for i in (0, m - 1)]
    els = []
    for c, (i, j, k) in enumerate(cube_corners):
        els.append((15, c + 1, [add((i, j, k), (coord(i), coord(j), coord(k)))]))
    # edges: along each axis, the 4 lines with the other two indices on the box
    for ax in range(3):
        for a in (0, m - 1):
            for b in (0, m - 1):
                ids = []
                for t in range(m):
                    key = [0, 0, 0]
                    key[ax] = t
                    o = [d for d in range(3) if d != ax]
                    key[o[0]], key[o[1]] = a, b
                    key = tuple(key)
                    ids.append(add(key, tuple(coord(v) for v in key)))
                els += [(1, 10 + ax, [ids[q], ids[q + 1]]) for q in range(m - 1)]
    # faces
    for ax in range(3):
        for side in (0, m - 1):
            grid = np.zeros((m, m), dtype=int)
            o = [d for d in range(3) if d != ax]
            for u in range(m):
                for v in range(m):
                    key = [0, 0, 0]
                    key[ax] = side
                    key[o[0]], key[o[1]] = u, v
                    key = tuple(key)
                    grid[u, v] = add(key, tuple(coord(q) for q in key))
            quads = quads_on_top and ax == 2 and side == m - 1
            for u in range(m - 1):
                for v in range(m - 1):
                    a, b, c, d = grid[u, v], grid[u + 1, v], grid[u + 1, v + 1], grid[u, v + 1]
                    if quads:
                        els.append((3, 20 + ax, [a, b, c, d]))
                    else:
                        els.append((2, 20 + ax, [a, b, c]))
                        els.append((2, 20 + ax, [a, c, d]))
    for i in range(1, m - 1):
        for j in range(1, m - 1):
            for k in range(1, m - 1):
                p = np.array([coord(i), coord(j), coord(k)]) + rng.uniform(-0.25 * h, 0.25 * h, 3)
                add((i, j, k), tuple(p))
    write_msh(path, np.array(nodes), els)
    return len(nodes)
