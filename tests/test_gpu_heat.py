"""The heat-conduction program on the GPU through the C ABI (mgm_heat_init /
mgm_heat_step) against its restatement run in the same data-parallel sweep
order on the device-built operators (the restatement is pinned to the
reference's own routines in tests/test_oracle_heat.py): every level's p and
source after each time step bit for bit, the steady-state error to 1e-12."""
import numpy as np
import pytest

from multigrid_meshless_b200 import api, clouds
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m,nl,k,poly,wave,omega,nrelax,nv", [(40, 3, 20, 3, 1, 1.0, 3, 2), (33, 2, 30, 4, 2, 1.2, 2, 3)])
def test_heat_program_bit_exact(require_gpu, m, nl, k, poly, wave, omega, nrelax, nv):
    cl = clouds.cavity_hierarchy(m, nl, seed=9)
    mg = api.Multigrid(cl, [k] * nl, [poly] * nl, reference_transfer=True)
    try:
        levels = O.levels_from_device(mg)
        mg.set_flow(Re=100.0, courant=0.5, omega=omega, num_relax=nrelax, num_vcycles=nv)
        mg.heat_init(wave)
        S = O.HeatSolver(levels, omega, nrelax, nv, wave=wave, jacobi=True)
        S.boundary_rhs()
        assert np.array_equal(mg.get_field("source"), S.source[0])
        lap_dev = mg.operators(0)["lapP"]
        assert np.array_equal(lap_dev, S.lapP0.reshape(lap_dev.shape))
        for step in range(3):
            e = mg.heat_step()
            e_o = S.step()
            assert abs(e - e_o) <= 1e-12 * abs(e_o), (step, e, e_o)
            for l in range(nl):
                assert np.array_equal(mg.get_field("p", l), S.p[l]), (step, l)
                assert np.array_equal(mg.get_field("source", l), S.source[l]), (step, l, "source")
        assert np.abs(S.p[0]).max() > 0
    finally:
        mg.close()


def test_heat_needs_init(require_gpu):
    cl = clouds.cavity_hierarchy(24, 2, seed=1)
    mg = api.Multigrid(cl, [20, 20], [3, 3], reference_transfer=True)
    try:
        with pytest.raises(Exception, match="mgm_heat_init first"):
            mg.heat_step()
    finally:
        mg.close()
