"""CPU checks of the C ABI: the library loads, exports every entry point that
include/mgm.h declares, and rejects bad input on the host before touching a
GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from multigrid_meshless_b200 import _lib, api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"MGM_API\s+[\w\s\*]*?\b(mgm_\w+)\s*\(", txt))
    return names


def reference_surface_symbols():
    txt = open(os.path.join(ROOT, "include", "mgm_reference.h")).read()
    return set(re.findall(r"MGM_API\s+(?:extern\s+)?[\w\s\*]*?\b([A-Za-z_]\w*)\s*[\(;]", txt))


def test_reference_surface_exported():
    """Every function of the reference's call surface (and the `parameters`
    global) that include/mgm_reference.h declares is exported."""
    names = reference_surface_symbols()
    for must in ("find_cloud_index", "create_derivative_matrices", "fractional_step_explicit",
                 "multiply_sparse_matrix_vector_gpu", "copyin_essentials_to_gpu", "parameters"):
        assert must in names
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [nm for nm in sorted(names) if not hasattr(lib, nm)]
    assert not missing, missing


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "mgm_knn_cloud" in names and "mgm_step" in names and "mgm_solve_poisson" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [nm for nm in sorted(declared_symbols()) if not hasattr(lib, nm)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    assert declared_symbols() <= set(_lib.SIGNATURES)


def test_knn_rejects_too_few_interior_nodes():
    """The reference recurses forever when fewer than k-1 interior nodes exist
    (kdtree_functions.h:99-105); the ABI returns MGM_ERR_ARG instead."""
    n = 10
    x = np.linspace(0, 1, n); y = np.zeros(n); z = np.zeros(n)
    bt = np.ones(n, np.uint8); bt[-2:] = 0
    with pytest.raises(_lib.MgmError) as e:
        api.knn_cloud(x, y, z, bt, 8, 5, 2)
    assert e.value.code == _lib.MGM_ERR_ARG


def test_bfs_rejects_out_of_range_index():
    cl = np.array([[0, 1], [1, 7]], np.int32)
    with pytest.raises(_lib.MgmError) as e:
        api.bfs_order(cl)
    assert e.value.code == _lib.MGM_ERR_ARG


def test_spmv_rejects_bad_index():
    with pytest.raises(_lib.MgmError):
        api.spmv(np.ones((3, 2)), np.array([[0, 1], [1, 2], [2, 3]], np.int32), np.ones(3))


@pytest.mark.parametrize("name", ["mgm_use_half_operator", "mgm_set_compatible_rhs", "mgm_use_tiled", "mgm_use_graphs",
                                  "mgm_use_compact"])
def test_solver_switches_reject_null_context(name):
    """The V-cycle switches check their context on the host: a null context
    is MGM_ERR_ARG with a message, before any CUDA call."""
    L = _lib.load()
    rc = getattr(L, name)(None, 1)
    assert rc == _lib.MGM_ERR_ARG
    assert b"null context" in L.mgm_last_error()


def test_reference_compatible_rhs_switch_without_context():
    """Before copyin_essentials_to_gpu there is no context: the legacy switch
    only records the setting (no CUDA call, no exit)."""
    L = _lib.load()
    L.mgm_reference_set_compatible_rhs(1)
    L.mgm_reference_set_compatible_rhs(0)
