"""Regenerates the golden fixtures in this folder from the REFERENCE's own code.

    make -C oracle REF=<reference tree>   # builds oracle/_ref/libref.so from the reference sources
    python tests/golden/make_golden.py

Each fixture runs the reference's set-up pipeline (find_cloud_index,
rcm_reordering_with_boundarynodes, correct_normal_directions,
calculate_avg_dx, create_prolongation_and_restriction_matrices,
create_derivative_matrices) on a seeded synthetic cloud, then two
fractional_step_explicit calls (in-place Gauss-Seidel sweeps, as the C build
runs them), and stores inputs and outputs in an .npz.  The tests compare the
CPU oracle restatement against these files bit for bit; they never need the
reference tree at run time.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from multigrid_meshless_b200 import clouds  # noqa: E402
from oracle import oracle as O  # noqa: E402

CASES = {
    # name: (cloud builder, ks, polys, bc kind, flow)
    "cavity2d_24": (lambda: clouds.cavity_hierarchy(24, 2, seed=11), [20, 20], [3, 3], 0,
                    dict(courant=0.5, Re=100.0, omega=1.2, num_vcycles=2, num_relax=3)),
    "annulus2d_h006": (lambda: clouds.annulus_hierarchy(0.06, 2, seed=5), [30, 30], [4, 4], 1,
                       dict(courant=0.5, Re=100.0, omega=1.0, num_vcycles=2, num_relax=3)),
    "cube3d_8": (lambda: [clouds.cube3d(8, seed=3)], [30], [2], 0,
                 dict(courant=0.3, Re=400.0, omega=1.0, num_vcycles=1, num_relax=2)),
}


def make(name):
    build, ks, polys, bc, flow = CASES[name]
    cl = build()
    levels = O.ref_pipeline(cl, ks, polys)
    R = O.ref_lib()
    R.ref_set_flow(flow["courant"], flow["Re"], flow["omega"], flow["num_vcycles"], flow["num_relax"])
    R.ref_fields_alloc()
    R.ref_bc(bc)
    dt = R.ref_dt()
    out = {"dt": dt, "ks": np.array(ks), "polys": np.array(polys), "bc": bc}
    for key, val in flow.items():
        out["flow_" + key] = val
    for l, (c, L) in enumerate(zip(cl, levels)):
        pre = f"l{l}_"
        for nm in ("x", "y", "z", "nx", "ny", "nz", "btag"):
            out[pre + "in_" + nm] = getattr(c, nm)
        out[pre + "in_nb"] = c.nb
        for nm in ("x", "y", "z", "nx", "ny", "nz", "btag", "cloud", "rpts", "ppts"):
            out[pre + nm] = getattr(L, nm)
        out[pre + "d_avg"] = L.d_avg
        for nm in ("Dx", "Dy", "Dz", "lap", "lapP", "restr", "prol"):
            v = getattr(L, nm)
            if v is not None:
                out[pre + nm] = v
    n0 = levels[0].n
    for s in range(2):
        err = R.ref_step()
        out[f"step{s}_err"] = err
        for nm in ("u", "v", "w", "p", "u_new", "v_new", "source"):
            a = np.zeros(n0)
            R.ref_field_get(0, O.FIELD[nm], a)
            out[f"step{s}_{nm}"] = a
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "levels", [L.n for L in levels], "dt", dt)


if __name__ == "__main__":
    for nm in (sys.argv[1:] or CASES):
        make(nm)
