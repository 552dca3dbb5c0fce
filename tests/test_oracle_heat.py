"""The heat-conduction program's restatement (mgm_oracle.c: orc_heat_*) against
the reference's own routines (heat_conduction.h:24-113 and
init/init_heat_conduction.c:14-67, compiled from the reference tree into
oracle/_ref/libref_heat.so), driven as mg_heat_conduction.c:47-77 drives them:
level pressures and the steady-state error after every time step, bit for bit,
in the C build's in-place sweep order."""
import numpy as np
import pytest

from multigrid_meshless_b200 import clouds
from oracle import oracle as O

pytestmark = pytest.mark.skipif(not O.ref_available(heat=True), reason="reference build not present")


@pytest.mark.parametrize("m,nl,k,poly,wave,omega,nrelax,nv", [(32, 3, 20, 3, 1, 1.0, 3, 2), (24, 2, 30, 4, 2, 1.2, 2, 3)])
def test_heat_restatement_matches_reference(m, nl, k, poly, wave, omega, nrelax, nv):
    cl = clouds.cavity_hierarchy(m, nl, seed=7)
    P = O.ref_pipeline(cl, [k] * nl, [poly] * nl, heat=True)
    R = O.ref_lib(heat=True)
    R.ref_set_flow(0.5, 100.0, omega, nv, nrelax)
    R.ref_fields_alloc()
    R.ref_heat_init(wave)
    S = O.HeatSolver(P, omega, nrelax, nv, wave=wave, jacobi=False)
    assert np.array_equal(S.source[0], _get(R, 0, "source", P[0].n))
    for step in range(3):
        e_ref = R.ref_heat_step(wave)
        e = S.step()
        assert e == e_ref, (step, e, e_ref)
        for l, L in enumerate(P):
            assert np.array_equal(S.p[l], _get(R, l, "p", L.n)), (step, l)
            assert np.array_equal(S.source[l], _get(R, l, "source", L.n)), (step, l, "source")
    assert np.abs(S.p[0]).max() > 0
    # the Dirichlet rows of set_boundary_rhs
    L0 = P[0]
    dirichlet = (L0.btag > 0) & (L0.x == 0)
    assert dirichlet.any()
    lap0 = S.lapP0.reshape(L0.n, L0.k)
    assert np.all(lap0[dirichlet, 0] == 1) and np.all(lap0[dirichlet, 1:] == 0)


def _get(R, l, name, n):
    out = np.zeros(n)
    R.ref_field_get(l, O.FIELD[name], out)
    return out
