"""A C program written against the reference's call surface
(include/mgm_reference.h: find_cloud_index, rcm_reordering_with_boundarynodes,
create_derivative_matrices, copyin_*_to_gpu, fractional_step_explicit, ...)
runs on the GPU through libmgm.so and reproduces the oracle.

The driver (tests/legacy_driver.c) is compiled here with gcc against the
in-tree library; its outputs are compared bit for bit with the oracle
restatement (correctly-rounded-power build for the weights; same sweep order
for the fractional step)."""
import os
import struct
import subprocess

import numpy as np
import pytest

from multigrid_meshless_b200 import clouds
from oracle import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "multigrid_meshless_b200")


def _compile(tmp):
    exe = os.path.join(tmp, "legacy_driver")
    subprocess.run(["gcc", "-O2", "-std=c11", "-I", os.path.join(ROOT, "include"), "-o", exe,
                    os.path.join(ROOT, "tests", "legacy_driver.c"), "-L", PKG, "-lmgm", f"-Wl,-rpath,{PKG}", "-lm"],
                   check=True)
    return exe


def _write_input(path, cl, poly, mult, nsteps, nv, nr, mode, Re, courant, omega):
    with open(path, "wb") as f:
        f.write(struct.pack("9i", len(cl), cl[0].dim, 3, poly, mult, nsteps, nv, nr, mode))
        f.write(struct.pack("3d", Re, courant, omega))
        for c in cl:
            f.write(struct.pack("2i", c.n, c.nb))
            for a in (c.x, c.y, c.z, c.nx, c.ny, c.nz):
                f.write(np.ascontiguousarray(a, np.float64).tobytes())
            f.write(np.ascontiguousarray(c.btag, np.uint8).tobytes())


def _read(out, name, dtype, shape=None):
    a = np.fromfile(os.path.join(out, name), dtype=dtype)
    return a.reshape(shape) if shape else a


def test_reference_call_surface_end_to_end(require_gpu, tmp_path):
    exe = _compile(str(tmp_path))
    cl = clouds.cavity_hierarchy(36, 2, seed=13)
    k, poly = 20, 3
    inp = str(tmp_path / "in.bin")
    out = str(tmp_path / "out")
    os.makedirs(out)
    _write_input(inp, cl, poly, 2, 2, 2, 3, 0, 100.0, 0.5, 1.2)
    r = subprocess.run([exe, inp, out], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("Mass residual") == 2

    P = O.orc_pipeline(cl, [k, k], [poly, poly], crpow=True)
    levels = []
    for l, L in enumerate(P):
        n = L.n
        assert np.array_equal(_read(out, f"l{l}_cloud", np.int32, (n, k)), L.cloud)
        for nm in ("x", "y", "nx", "ny"):
            assert np.array_equal(_read(out, f"l{l}_{nm}", np.float64), getattr(L, nm)), nm
        assert np.array_equal(_read(out, f"l{l}_btag", np.uint8), L.btag)
        assert _read(out, f"l{l}_d_avg", np.float64)[0] == L.d_avg
        assert np.array_equal(_read(out, f"l{l}_rpts", np.int32), L.rpts)
        assert np.array_equal(_read(out, f"l{l}_ppts", np.int32), L.ppts)
        for nm in ("Dx", "Dy", "lap", "lapP"):
            assert np.array_equal(_read(out, f"l{l}_{nm}", np.float64, (n, k)), getattr(L, nm)), nm
        if l > 0:
            assert np.array_equal(_read(out, f"l{l}_restr", np.float64, (n, k)), L.restr)
        if l < len(P) - 1:
            assert np.array_equal(_read(out, f"l{l}_prol", np.float64, (n, k)), L.prol)

    # two fractional steps in the reference's semantics (sweeps in Jacobi order)
    S = O.OracleSolver(P, 100.0, 0.5, 1.2, 3, 2, jacobi=True)
    assert S.dt == _read(out, "dt", np.float64)[0]
    O.lid_bc(P[0], S.f)
    errs = _read(out, "errs", np.float64)
    for s in range(2):
        e, _ = S.step()
        assert abs(errs[s] - e) <= 1e-12 * abs(e)
    assert np.array_equal(_read(out, "u", np.float64), S.f["u"])
    assert np.array_equal(_read(out, "v", np.float64), S.f["v"])
    assert np.array_equal(_read(out, "p", np.float64), S.p[0])


def test_reference_call_surface_timple(require_gpu, tmp_path):
    """The reference main's default loop, time_implicit_solver, called by name
    from C through libmgm.so (reference-semantics multigrid on p'), against
    the TIMPLE restatement in the same data-parallel sweep order.  The coarse
    annulus holds node pairs one gap apart across the channel (squared
    distance 0.25 (1 - 2^-53), whose power 1.5 lies 2^-107 from a rounding
    midpoint), so the set-up comparison also covers the near-midpoint
    rounding of the power helpers."""
    exe = _compile(str(tmp_path))
    cl = clouds.annulus_hierarchy(0.06, 2, seed=3)
    k, poly = 20, 3
    inp = str(tmp_path / "in.bin")
    out = str(tmp_path / "out")
    os.makedirs(out)
    _write_input(inp, cl, poly, 2, 3, 3, 2, 0, 100.0, 0.5, 1.0)
    r = subprocess.run([exe, inp, out, "timple"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    P = O.orc_pipeline(cl, [k, k], [poly, poly], crpow=True)
    levels = []
    for l, L in enumerate(P):
        n = L.n
        assert np.array_equal(_read(out, f"l{l}_cloud", np.int32, (n, k)), L.cloud), (l, "cloud")
        for nm in ("x", "y", "nx", "ny"):
            assert np.array_equal(_read(out, f"l{l}_{nm}", np.float64), getattr(L, nm)), (l, nm)
        ops = {nm: _read(out, f"l{l}_{nm}", np.float64, (n, k)) for nm in ("Dx", "Dy", "lap", "lapP")}
        for nm, v in ops.items():
            assert np.array_equal(v, getattr(L, nm)), (l, nm)
        restr = _read(out, f"l{l}_restr", np.float64, (n, k)) if l > 0 else None
        prol = _read(out, f"l{l}_prol", np.float64, (n, k)) if l < len(P) - 1 else None
        for nm, got, want in (("restr", restr, L.restr), ("prol", prol, L.prol)):
            if got is not None:
                assert np.array_equal(got, want), (l, nm)
        levels.append(O.Level(n, L.nb, k, 2, poly, L.x, L.y, L.z, L.nx, L.ny, L.nz, L.btag, L.cloud, L.d_avg,
                              ops["Dx"], ops["Dy"], None, ops["lap"], ops["lapP"], L.rpts, L.ppts, restr, prol))
    S = O.TimpleSolver(levels, 100.0, 0.5, 1.0, 2, 3, 2, 2, 1.0, 1.0, jacobi=True)
    assert S.dt == _read(out, "dt", np.float64)[0]
    O.tc_bc(levels[0], S.f)
    errs = _read(out, "errs", np.float64)
    for s in range(3):
        e = S.step()
        assert abs(errs[s] - e) <= 1e-12 * abs(e)
    for nm in ("u_new", "v_new"):
        assert np.array_equal(_read(out, nm, np.float64), S.f[nm]), nm
    assert np.array_equal(_read(out, "p_old", np.float64), S.p_old)


def test_reference_routines_one_by_one(require_gpu, tmp_path):
    """A C program that builds the operators with create_full_gradx/grady/
    laplacian_matrix + create_laplacian_for_Poisson and runs each step through
    calculate_intermediate_velocity ... update_velocity with the multigrid
    written out (relaxation, calculate_residuals, restrict_residuals,
    prolongate_corrections per level) gets the bits of create_derivative_matrices
    + fractional_step_explicit; and its matrixInverse_Gauss_Jordan matches the
    restatement."""
    exe = _compile(str(tmp_path))
    cl = clouds.cavity_hierarchy(40, 3, seed=21)
    k = 20
    inp = str(tmp_path / "in.bin")
    _write_input(inp, cl, 3, 2, 2, 2, 3, 0, 100.0, 0.5, 1.2)
    outs = {}
    for mode in ("default", "routines"):
        out = str(tmp_path / mode)
        os.makedirs(out)
        args = [exe, inp, out] + ([mode] if mode == "routines" else [])
        r = subprocess.run(args, capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr
        outs[mode] = out
    for l, c in enumerate(cl):
        for nm in ("Dx", "Dy", "lap", "lapP"):
            a = _read(outs["default"], f"l{l}_{nm}", np.float64)
            b = _read(outs["routines"], f"l{l}_{nm}", np.float64)
            assert np.array_equal(a, b), (l, nm)
    for nm in ("u", "v", "p"):
        a, b = _read(outs["default"], nm, np.float64), _read(outs["routines"], nm, np.float64)
        assert np.array_equal(a, b), nm
        assert np.abs(a).max() > 0
    A = np.array([[0, 2, 1, 0, 3], [2, 0, 4, 1, 0], [1, 4, 0, 2, 1], [0, 1, 2, 5, 1], [3, 0, 1, 1, 6]], np.float64)
    want = np.zeros(25)
    O.lib().orc_gauss_jordan(5, np.ascontiguousarray(A), want)
    assert np.array_equal(_read(outs["routines"], "gj_inverse", np.float64), want)
