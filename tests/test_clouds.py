"""Synthetic clouds are in the state the reference's mesh reader leaves:
boundary nodes first, no corner nodes, seeded and reproducible."""
import numpy as np

from multigrid_meshless_b200 import clouds


def test_cavity_counts_and_layout():
    c = clouds.cavity2d(128, seed=1)
    assert c.n == 128 * 128 - 4 and c.nb == 4 * 126
    assert np.all(c.btag[:c.nb] == 1) and np.all(c.btag[c.nb:] == 0)
    assert np.allclose(np.hypot(c.nx[:c.nb], c.ny[:c.nb]), 1.0)
    h = 1 / 127
    ix = c.x[c.nb:] / h
    assert np.all(np.abs(ix - np.round(ix)) <= 0.25 + 1e-9)
    top = np.abs(c.y - 1.0) < 1e-9
    assert top.sum() == 126 and np.all(c.btag[top] == 1)


def test_reproducible():
    a = clouds.cavity2d(32, seed=5)
    b = clouds.cavity2d(32, seed=5)
    c = clouds.cavity2d(32, seed=6)
    assert np.array_equal(a.x, b.x) and not np.array_equal(a.x, c.x)


def test_annulus_walls():
    c = clouds.annulus2d(0.02, seed=3)
    r = np.hypot(c.x, c.y)
    assert np.all(r >= 0.5 - 1e-12) and np.all(r <= 1 + 1e-12)
    inner = np.abs(r - 0.5) < 1e-9
    outer = np.abs(r - 1.0) < 1e-9
    assert inner.sum() + outer.sum() == c.nb
    assert np.all(c.btag[:c.nb] == 1)
    # outward normals: inner wall points to the centre
    assert np.all(c.nx[inner] * c.x[inner] + c.ny[inner] * c.y[inner] < 0)


def test_annulus_million_node_spacing():
    h = clouds.annulus_h_for_nodes(1_000_000)
    assert 1.4e-3 < h < 1.7e-3


def test_cube_has_no_edge_nodes():
    c = clouds.cube3d(6, seed=2)
    assert c.n == 6 ** 3 - 8 - 12 * 4
    onb = ((np.abs(c.x) < 1e-12) | (np.abs(c.x - 1) < 1e-12)).astype(int) + \
          ((np.abs(c.y) < 1e-12) | (np.abs(c.y - 1) < 1e-12)) + ((np.abs(c.z) < 1e-12) | (np.abs(c.z - 1) < 1e-12))
    assert np.all(onb[:c.nb] == 1)
