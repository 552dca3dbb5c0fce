"""Output and restart through the C ABI: Solution.csv in the reference main's
format, and checkpoints from which a run continues bit for bit (fractional
step in reference semantics and in FP32-in-FP64 mode, TIMPLE, the
heat-conduction program), rejected by a context of other levels."""
import numpy as np
import pytest

import multigrid_meshless_b200 as mgm
from multigrid_meshless_b200 import api, clouds

pytestmark = pytest.mark.gpu


def _cavity():
    return api.Multigrid(clouds.cavity_hierarchy(40, 3, seed=12), [20] * 3, [3] * 3, reference_transfer=True)


def _state(mg):
    out = {nm: mg.get_field(nm) for nm in ("u", "v", "u_new", "v_new", "p_old")}
    for l in range(mg.nl):
        out[f"p{l}"] = mg.get_field("p", l)
        out[f"src{l}"] = mg.get_field("source", l)
    return out


def _run(mg, kind, steps):
    for _ in range(steps):
        if kind == "fs_ref":
            mg.step(mgm.MODE_REFERENCE)
        elif kind == "fs_fp32":
            mg.step(mgm.MODE_FP32_IR)
        elif kind == "timple":
            mg.timple_step(mgm.MODE_REFERENCE)
        else:
            mg.heat_step()


def _start(mg, kind):
    mg.set_flow(Re=100.0, courant=0.5, omega=1.0, num_relax=2, num_vcycles=2)
    mg.set_solver(rel_tol=1e-8, max_iters=80)
    if kind == "heat":
        mg.heat_init(1)
    elif kind == "timple":
        mg.set_timple(2, 2, 1.0, 1.0)
        mg.apply_bc(mgm.BC_LID)
        mg.set_field("u_new", mg.get_field("u"))
    else:
        mg.apply_bc(mgm.BC_LID)


@pytest.mark.parametrize("kind", ["fs_ref", "fs_fp32", "timple", "heat"])
def test_restart_repeats_the_run(require_gpu, tmp_path, kind):
    ck = tmp_path / "state.ckpt"
    a = _cavity()
    try:
        _start(a, kind)
        _run(a, kind, 2)
        a.checkpoint_save(ck)
        _run(a, kind, 2)
        want = _state(a)
    finally:
        a.close()
    b = _cavity()
    try:
        _start(b, kind)
        b.checkpoint_load(ck)
        _run(b, kind, 2)
        got = _state(b)
    finally:
        b.close()
    for nm in want:
        assert np.array_equal(got[nm], want[nm]), nm
    assert any(np.abs(v).max() > 0 for v in want.values())


def test_checkpoint_rejects_other_levels(require_gpu, tmp_path):
    ck = tmp_path / "state.ckpt"
    a = _cavity()
    try:
        _start(a, "fs_ref")
        a.checkpoint_save(ck)
    finally:
        a.close()
    b = api.Multigrid(clouds.cavity_hierarchy(40, 3, seed=13), [20] * 3, [3] * 3, reference_transfer=True)
    try:
        with pytest.raises(Exception, match="does not match"):
            b.checkpoint_load(ck)
    finally:
        b.close()
    raw = bytearray(ck.read_bytes())
    raw[-20] ^= 0xFF
    ck.write_bytes(bytes(raw))
    c = _cavity()
    try:
        with pytest.raises(Exception, match="checksum"):
            c.checkpoint_load(ck)
    finally:
        c.close()


def test_solution_csv_format(require_gpu, tmp_path):
    mg = _cavity()
    try:
        _start(mg, "fs_ref")
        _run(mg, "fs_ref", 2)
        out = tmp_path / "Solution.csv"
        mg.write_solution(out, pressure="p")
        g = mg.geometry(0)
        cols = [g["x"], g["y"], g["z"], mg.get_field("u"), mg.get_field("v"), mg.get_field("w"), mg.get_field("p")]
        want = "".join(", ".join("%f" % c[i] for c in cols) + "\n" for i in range(mg.n(0)))
        assert out.read_text() == want
    finally:
        mg.close()
