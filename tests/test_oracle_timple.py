"""The TIMPLE restatement (oracle/mgm_oracle.c, orc_timple_*) against the
reference's own time_implicit_solver (timple_solver.h:40-410, compiled from
the reference tree into oracle/_ref/libref_timple.so), bit for bit, on the
configuration the reference main runs it with: the Taylor-Couette annulus
(init_TC.c).  The restatement runs the reference's in-place sweep order here;
its data-parallel order is what the GPU path is compared with."""
import numpy as np
import pytest

from multigrid_meshless_b200 import clouds
from oracle import oracle as O

pytestmark = pytest.mark.skipif(not O.ref_available(timple=True), reason="reference TIMPLE build absent")

FIELDS = ("u_new", "v_new", "u", "v", "u_old", "v_old", "dpdn", "source")


@pytest.mark.parametrize("iters", [(2, 2, 1.0, 1.0), (3, 4, 1.3, 2.0)])
def test_timple_steps_bit_exact(iters):
    it_timple, it_mom, facRe, facdt = iters
    cl = clouds.annulus_hierarchy(0.06, 2, seed=3)
    ks, polys = [20, 20], [3, 3]
    R = O.ref_lib(timple=True)
    levels = O.ref_pipeline(cl, ks, polys, timple=True)
    Re, courant, omega, nrelax, nvc = 100.0, 0.5, 1.0, 2, 3
    R.ref_set_flow(courant, Re, omega, nvc, nrelax)
    R.ref_fields_alloc()
    R.ref_bc(1)
    dt = R.ref_dt()
    R.ref_timple_params(it_timple, it_mom, facRe, facdt)
    S = O.TimpleSolver(levels, Re, courant, omega, nrelax, nvc, it_timple, it_mom, facRe, facdt, jacobi=False, dt=dt)
    O.tc_bc(levels[0], S.f)
    n = levels[0].n
    got = np.zeros(n)
    for step in range(3):
        e_ref = R.ref_timple_step()
        e = S.step()
        assert e == e_ref, (step, e, e_ref)
        for nm in FIELDS:
            R.ref_field_get(0, O.FIELD[nm], got)
            want = S.f[nm] if nm in S.f else S.source[0]
            assert np.array_equal(got, want), (step, nm)
        R.ref_field_get(0, O.FIELD["p_old"], got)
        assert np.array_equal(got, S.p_old), (step, "p_old")
        for l in range(2):
            pl = np.zeros(levels[l].n)
            R.ref_field_get(l, O.FIELD["pprime"], pl)
            assert np.array_equal(pl, S.p[l]), (step, "pprime", l)
    assert np.all(np.isfinite(S.p_old)) and np.abs(S.f["u_new"]).max() > 0
