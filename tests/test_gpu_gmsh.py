"""The Gmsh reader on the GPU through the C ABI (mgm_mesh_read:
read_PointStructure, mesh_functions.h:172-476) against the restatement
(itself pinned to the reference's reader in tests/test_gmsh_oracle.py), bit
for bit; and level hierarchies read from Gmsh files running end to end:
through the Python mirror, and through the reference's own call sequence
(read_flow_parameters, read_grid_filenames, read_complete_mesh_data,
fractional_step_explicit) in a C program linked against libmgm.so."""
import os
import subprocess

import numpy as np
import pytest

import meshgen
import multigrid_meshless_b200 as mgm
from multigrid_meshless_b200 import api
from multigrid_meshless_b200.clouds import Cloud
from oracle import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "multigrid_meshless_b200")
KEYS = ("x", "y", "z", "nx", "ny", "nz")


def _cases(d):
    out = []
    p = os.path.join(d, "sq.msh"); meshgen.square2d(p, 31, seed=4); out.append((p, 2))
    p = os.path.join(d, "an.msh"); meshgen.annulus2d(p, 0.05, seed=5); out.append((p, 2))
    p = os.path.join(d, "cu.msh"); meshgen.cube3d(p, 9, seed=6); out.append((p, 3))
    p = os.path.join(d, "cq.msh"); meshgen.cube3d(p, 6, seed=7, quads_on_top=False); out.append((p, 3))
    return out


def _cloud(r, dim):
    return Cloud(r["x"], r["y"], r["z"], r["nx"], r["ny"], r["nz"], r["btag"], r["nb"], dim, r["d_avg"])


def test_reader_bit_exact(require_gpu, tmp_path):
    for path, dim in _cases(str(tmp_path)):
        got = api.read_gmsh(path, dim)
        want = O.read_mesh(path, dim)
        for k in KEYS:
            assert np.array_equal(getattr(got, k), want[k]), (path, k)
        assert np.array_equal(got.btag, want["btag"]) and np.array_equal(got.meta["corner"], want["corner"])
        assert got.nb == want["nb"] and got.meta["num_elem"] == want["num_elem"]
        assert got.meta["d_avg"] == want["d_avg"]
        assert np.any(got.nx != 0)


def test_reader_rejects_bad_files(require_gpu, tmp_path):
    with pytest.raises(Exception, match="unable to open"):
        api.read_gmsh(str(tmp_path / "missing.msh"), 2)
    p = tmp_path / "trunc.msh"
    p.write_text("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n5\n1 0 0 0\n2 1 0 0\n")
    with pytest.raises(Exception, match="truncated"):
        api.read_gmsh(str(p), 2)
    p.write_text("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n2\n1 0 0 0\n2 1 0 0\n$EndNodes\n"
                 "$Elements\n1\n1 1 2 0 1 1 7\n$EndElements\n")
    with pytest.raises(Exception, match="out of range"):
        api.read_gmsh(str(p), 2)


def _square_levels(d, sizes):
    paths = []
    for l, m in enumerate(sizes):
        p = os.path.join(d, f"sq{l}.msh")
        meshgen.square2d(p, m, seed=10 + l)
        paths.append(p)
    return paths


def test_gmsh_hierarchy_reference_step(require_gpu, tmp_path):
    """Three square levels read from Gmsh files: set-up and two
    reference-semantics fractional steps bit for bit against the oracle run on
    the restatement's reading of the same files."""
    paths = _square_levels(str(tmp_path), (33, 17, 9))
    k, poly = 20, 3
    mg = api.Multigrid([api.read_gmsh(p, 2) for p in paths], [k] * 3, [poly] * 3, reference_transfer=True)
    try:
        P = O.orc_pipeline([_cloud(O.read_mesh(p, 2), 2) for p in paths], [k] * 3, [poly] * 3, crpow=True)
        levels = O.levels_from_device(mg)
        for l, L in enumerate(P):
            for nm in ("cloud", "x", "y", "nx", "ny", "btag"):
                assert np.array_equal(getattr(levels[l], nm), getattr(L, nm)), (l, nm)
            for nm in ("Dx", "Dy", "lap", "lapP"):
                assert np.array_equal(getattr(levels[l], nm), getattr(L, nm)), (l, nm)
        mg.set_flow(Re=100.0, courant=0.5, omega=1.2, num_relax=3, num_vcycles=2)
        S = O.OracleSolver(levels, 100.0, 0.5, 1.2, 3, 2, jacobi=True)
        mg.apply_bc(mgm.BC_LID)
        O.lid_bc(levels[0], S.f)
        for s in range(2):
            mg.step(mgm.MODE_REFERENCE)
            S.step()
            for nm in ("u", "v"):
                assert np.array_equal(mg.get_field(nm), S.f[nm]), (s, nm)
            assert np.array_equal(mg.get_field("p"), S.p[0]), (s, "p")
        # and the convergent FP32-in-FP64 step runs on the same hierarchy
        mg.set_solver(rel_tol=1e-8, max_iters=80)
        mg.step(mgm.MODE_FP32_IR)
        assert mg.last_solve()[1] < 1e-8
    finally:
        mg.close()


FLOW = [("dimension", 2), ("poly_degree", 3), ("phs_degree", 3), ("cloud_size_multiplier", 2), ("test", 0),
        ("courant_number", 0.5), ("steady_state_tolerance", 1e-6), ("poisson_solver_tolerance", 1e-6),
        ("omega", 1.2), ("num_vcycles", 2), ("num_relax", 3), ("num_time_steps", 2), ("write_interval", 100),
        ("neumann_flag_boundary", 1), ("dt", 0.0), ("iter_momentum", 1), ("iter_timple", 1), ("Re", 100.0),
        ("facRe", 1.0), ("facdt", 1.0)]


def test_reference_main_on_gmsh_files(require_gpu, tmp_path):
    """mg_NS_solver.c's own sequence on Gmsh files (relative names, as the
    reference's 50-character mesh_filename needs) through libmgm.so."""
    d = str(tmp_path)
    exe = os.path.join(d, "legacy_driver")
    subprocess.run(["gcc", "-O2", "-std=c11", "-I", os.path.join(ROOT, "include"), "-o", exe,
                    os.path.join(ROOT, "tests", "legacy_driver.c"), "-L", PKG, "-lmgm", f"-Wl,-rpath,{PKG}", "-lm"],
                   check=True)
    paths = _square_levels(d, (29, 15, 8))
    with open(os.path.join(d, "flow.csv"), "w") as f:
        for nm, v in FLOW:
            f.write(f"{nm},{v}\n")
    with open(os.path.join(d, "grid.csv"), "w") as f:
        f.write(f"num_levels,{len(paths)}\n")
        for p in paths:
            f.write(os.path.basename(p) + "\n")
    os.makedirs(os.path.join(d, "out"))
    r = subprocess.run([exe, "--gmsh", "flow.csv", "grid.csv", "out"], cwd=d, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("Reading mesh data for level") == 3

    def rd(name, dtype, shape=None):
        a = np.fromfile(os.path.join(d, "out", name), dtype=dtype)
        return a.reshape(shape) if shape else a

    k = 20
    P = O.orc_pipeline([_cloud(O.read_mesh(p, 2), 2) for p in paths], [k] * 3, [3] * 3, crpow=True)
    for l, L in enumerate(P):
        n = L.n
        assert np.array_equal(rd(f"l{l}_cloud", np.int32, (n, k)), L.cloud), (l, "cloud")
        for nm in ("x", "y", "nx", "ny"):
            assert np.array_equal(rd(f"l{l}_{nm}", np.float64), getattr(L, nm)), (l, nm)
        for nm in ("Dx", "Dy", "lap", "lapP"):
            assert np.array_equal(rd(f"l{l}_{nm}", np.float64, (n, k)), getattr(L, nm)), (l, nm)
    S = O.OracleSolver(P, 100.0, 0.5, 1.2, 3, 2, jacobi=True)
    assert S.dt == rd("dt", np.float64)[0]
    O.lid_bc(P[0], S.f)
    for s in range(2):
        S.step()
    assert np.array_equal(rd("u", np.float64), S.f["u"])
    assert np.array_equal(rd("v", np.float64), S.f["v"])
    assert np.array_equal(rd("p", np.float64), S.p[0])


def test_gmsh_cube_hierarchy_setup(require_gpu, tmp_path):
    """Two 3D levels read from Gmsh cube meshes (triangle and quad faces; edge
    lines make their nodes corners, which the reader drops): clouds, order,
    normals and every operator bit for bit against the oracle pipeline on the
    restatement's reading, and a convergent FP32-in-FP64 step on top."""
    paths = []
    for l, m in enumerate((10, 6)):
        p = os.path.join(str(tmp_path), f"cu{l}.msh")
        meshgen.cube3d(p, m, seed=30 + l, quads_on_top=(l == 0))
        paths.append(p)
    k, poly = 30, 2
    mg = api.Multigrid([api.read_gmsh(p, 3) for p in paths], [k] * 2, [poly] * 2, reference_transfer=True)
    try:
        P = O.orc_pipeline([_cloud(O.read_mesh(p, 3), 3) for p in paths], [k] * 2, [poly] * 2, crpow=True)
        levels = O.levels_from_device(mg)
        for l, L in enumerate(P):
            for nm in ("cloud", "x", "y", "z", "nx", "ny", "nz", "btag"):
                assert np.array_equal(getattr(levels[l], nm), getattr(L, nm)), (l, nm)
            for nm in ("Dx", "Dy", "Dz", "lap", "lapP"):
                assert np.array_equal(getattr(levels[l], nm), getattr(L, nm)), (l, nm)
        mg.set_flow(Re=400.0, courant=0.3)
        mg.set_solver(rel_tol=1e-8, max_iters=80)
        mg.apply_bc(mgm.BC_LID)
        mg.step(mgm.MODE_FP32_IR)
        assert mg.last_solve()[1] < 1e-8
    finally:
        mg.close()
