"""The reference's own main program, unmodified but for the include swap, on
libmgm.so.

oracle/build_reference_main.sh (run by `make -C oracle REF=<tree>` where the
reference tree exists; the binaries travel in oracle/_ref/main/) compiles
mg_NS_solver.c twice per variant: alone with the reference's headers (CPU),
and with `#include "header_files/timple_solver.h"` (or
fractional_step_solver.h) replaced by `#include "mgm_reference.h"` and linked
against libmgm.so.  Both run here in a directory holding
flow_parameters.csv, grid_filenames.csv and synthetic Gmsh meshes of an
annulus (init/init_TC.c's geometry):

* test_derivatives (general_functions.h:44-192, parameters.test = 1): the
  printed RMS errors of Dx, Dy and lap on every level equal the reference
  build's printed values;
* Convergence.csv and Solution.csv (mg_NS_solver.c:66-90) equal, number for
  number, the restatement's run of the same program -- the reader, the
  set-up, init_TC.c's conditions and the time loop in the library's
  data-parallel sweep order -- formatted as the main formats them;
* free_PointStructure / free_field end the program cleanly (the reference
  build's own versions crash there, after the work is done).

Reference: mg_NS_solver.c:17-103, structures.h:174-226.
"""
import os
import subprocess

import numpy as np
import pytest

import meshgen
from multigrid_meshless_b200.clouds import Cloud
from oracle import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MAIN = os.path.join(ROOT, "oracle", "_ref", "main")

# flow_parameters.csv in the positional order read_flow_parameters reads
# (mesh_functions.h:37-100); names are not parsed
FLOW = [("domain_dimensions", 2), ("poly_deg", 3), ("phs_deg", 3), ("cloud_size_multiplier", 2),
        ("test_derivative", 1), ("courant_number", 0.5), ("steady_tolerance", 1e-30),
        ("poisson_solver_tolerance", 1e-8), ("sor_parameter", 1.0), ("num_vcycles", 3), ("num_relax", 2),
        ("num_time_steps", 3), ("write_interval", 100), ("neumann_flag_boundary", 1), ("time_step", 0.1),
        ("iter_momentum", 2), ("iter_timple", 2), ("Re", 100.0), ("facRe", 1.0), ("facdt", 1.0)]
K, POLY, RE, COURANT, OMEGA, NRELAX, NCYC, STEPS = 20, 3, 100.0, 0.5, 1.0, 2, 3, 3


def _built(variant):
    return all(os.path.exists(os.path.join(MAIN, f"{variant}_{kind}")) for kind in ("ref", "mgm"))


def _case(d):
    """Two annulus levels as Gmsh files and the two csv inputs, in d."""
    names = []
    for l, h in enumerate((0.05, 0.1)):
        nm = f"an{l}.msh"
        meshgen.annulus2d(os.path.join(d, nm), h, seed=40 + l)
        names.append(nm)
    with open(os.path.join(d, "flow_parameters.csv"), "w") as f:
        for nm, v in FLOW:
            f.write(f"{nm},{v}\n")
    with open(os.path.join(d, "grid_filenames.csv"), "w") as f:
        f.write(f"num_levels,{len(names)}\n")
        for nm in names:
            f.write(nm + "\n")
    return names


def _run(exe, d, reference_build=False):
    """Runs a main in d.  The reference build's own free_PointStructure
    (structures.h:174-209) frees rows that were never allocated and crashes
    after the program's work is done; for that build a SIGSEGV after the
    final timing line is accepted.  The library's build must exit 0."""
    # line-buffered stdout (coreutils stdbuf), so that a crash at exit loses no output
    r = subprocess.run(["stdbuf", "-oL", exe], cwd=d, capture_output=True, text=True, timeout=600)
    done = "Time for execution (total)" in r.stdout
    ok = r.returncode == 0 or (reference_build and r.returncode == -11 and done)
    assert ok and done, (r.returncode, r.stdout[-3000:] + r.stderr[-3000:])
    return r.stdout


def _derivative_lines(out):
    lines = out.splitlines()
    return [lines[i + 1].split() for i, ln in enumerate(lines) if ln.startswith("L2 error in f")]


def _restated(d, names, variant):
    """The restatement's run of the main: reader, set-up (poly 3 on every
    level here), init_TC.c's conditions, STEPS time steps in the library's
    sweep order.  Returns (steady errors, x, y, z, u, v, w, pressure column)."""
    P = O.orc_pipeline([Cloud(r["x"], r["y"], r["z"], r["nx"], r["ny"], r["nz"], r["btag"], r["nb"], 2, r["d_avg"])
                        for r in (O.read_mesh(os.path.join(d, nm), 2) for nm in names)],
                       [K, K], [POLY, POLY], crpow=True)
    if variant == "timple":
        S = O.TimpleSolver(P, RE, COURANT, OMEGA, NRELAX, NCYC, 2, 2, 1.0, 1.0, jacobi=True)
    else:
        S = O.OracleSolver(P, RE, COURANT, OMEGA, NRELAX, NCYC, jacobi=True)
    O.tc_bc(P[0], S.f)
    errs = []
    for _ in range(STEPS):
        e = S.step()
        errs.append(e if variant == "timple" else e[0])
    L0 = P[0]
    pres = S.p_old if variant == "timple" else np.zeros(L0.n)  # the main prints p_old
    return errs, L0.x, L0.y, L0.z, S.f["u"], S.f["v"], S.f["w"], pres


@pytest.mark.parametrize("variant", ["timple", "fs"])
def test_unmodified_main_on_libmgm(require_gpu, tmp_path, variant):
    if not _built(variant):
        pytest.skip("oracle/_ref/main not built (needs the reference tree at build time)")
    runs = {}
    for kind in ("ref", "mgm"):
        d = tmp_path / kind
        d.mkdir()
        names = _case(str(d))
        out = _run(os.path.join(MAIN, f"{variant}_{kind}"), str(d), reference_build=(kind == "ref"))
        runs[kind] = (str(d), names, out)
    # the derivative self-test: printed RMS errors equal the reference build's
    dref, dmgm = _derivative_lines(runs["ref"][2]), _derivative_lines(runs["mgm"][2])
    assert len(dmgm) == 2 and dmgm == dref, (dmgm, dref)
    # the time loop's files against the restatement of the same program
    d, names, _ = runs["mgm"]
    errs, x, y, z, u, v, w, pres = _restated(d, names, variant)
    conv = np.loadtxt(os.path.join(d, "Convergence.csv"), delimiter=",", ndmin=2)
    assert conv.shape == (STEPS, 2)
    assert np.array_equal(conv[:, 0], np.arange(STEPS))
    want = np.array([float("%e" % e) for e in errs])
    assert np.allclose(conv[:, 1], want, rtol=2e-6, atol=0, equal_nan=True), (conv[:, 1], want)
    sol = np.loadtxt(os.path.join(d, "Solution.csv"), delimiter=",")
    cols = np.stack([x, y, z, u, v, w, pres], 1)
    want = np.vectorize(lambda t: float("%f" % t))(cols)
    assert sol.shape == want.shape
    assert np.array_equal(sol, want, equal_nan=True)
    assert np.isfinite(sol).all()
