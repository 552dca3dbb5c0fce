#!/usr/bin/env python
"""bench.py -- NS steps/s & Poisson ms at 1M nodes, Poisson solved to a 1e-8
relative residual: FP32-in-FP64 refinement vs plain FP64 on the GPU.

Workload (the 1M-node 2D lid-driven cavity): unit square, 1000 x 1000 jittered
Cartesian nodes (999,996 after the corner nodes are removed), 6 levels each
coarser by 4x, PHS degree 3, polynomial degree 4 (15 terms), 30-node stencils,
Courant 0.3, Re drawn from U[100, 1000] (the timed episode at the first
held-out draw), timed past the start-up transient (--eval-start steps from
rest).  A step is one fractional step (momentum, divergence, Poisson solve to
1e-8, velocity correction) through the C ABI.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's own C implementation of the step
(oracle/_ref/libref.so, compiled from the reference sources; serial C, one
core) on the full 1M-node workload, its set-up built untimed by the
restatement (bit-identical to the reference's set-up) on all host cores.
Under torchrun each rank runs an independent replica on its own GPU
("replicas only": the path has no exchange step); rank 0 prints the line.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "NS steps/s & Poisson ms @1M nodes, 1e-8 resid: learned+FP32 vs plain FP64 GPU"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--m", type=int, default=1000, help="nodes per side of the fine cavity level")
    ap.add_argument("--levels", type=int, default=6)
    ap.add_argument("--k", type=int, default=30)
    ap.add_argument("--poly", type=int, default=4)
    ap.add_argument("--Re", type=float, default=None,
                    help="Reynolds number of the timed episode (default: the first held-out draw of U[100, 1000])")
    ap.add_argument("--courant", type=float, default=0.3,
                    help="Courant number of the learned-warm-start protocol (explicit Euler is stable at 0.3 on "
                         "the 1M cavity; 0.5 grows within ~12 steps)")
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--cheb-degree", type=int, default=3)
    ap.add_argument("--cheb-ratio", type=float, default=20.0)
    ap.add_argument("--episode", type=int, default=10,
                    help="steps per episode from rest of the other workloads (annulus, cube, TIMPLE)")
    ap.add_argument("--sample-m", type=int, default=128, help="cavity size of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned warm-start measurement")
    ap.add_argument("--no-half", action="store_true", help="skip the FP16-operator measurement")
    ap.add_argument("--train-episodes", type=int, default=10, help="training episodes from rest (Re ~ U[100, 1000])")
    ap.add_argument("--train-steps", type=int, default=200, help="steps per training episode (2000 in all)")
    ap.add_argument("--eval-episodes", type=int, default=2, help="held-out episodes at unseen Re")
    ap.add_argument("--eval-steps", type=int, default=100, help="steps per held-out episode (200 in all)")
    ap.add_argument("--learn-iters", type=int, default=2000, help="Adam iterations of the GPU training")
    ap.add_argument("--eval-start", type=int, default=300,
                    help="untimed steps from rest before an episode's collected or timed steps (the cavity's "
                         "start-up transient; 0 times the steps right after rest)")
    ap.add_argument("--w-mse", type=float, default=1.0, help="weight of the increment MSE in the training loss")
    ap.add_argument("--w-res", type=float, default=0.0,
                    help="weight of the smoothed-residual term in the training loss (mgm_mpnn_set_loss)")
    ap.add_argument("--host-driven", action="store_true",
                    help="run every arm with the solve's loops driven from the host (V-cycle graphs without "
                         "conditional nodes, so that a profiler sees each kernel launch)")
    ap.add_argument("--workload", choices=["cavity", "annulus", "timple", "cube", "shell-batch"], default="cavity",
                    help="cavity: the headline (1M-node cavity); annulus / cube / shell-batch: the other configs, "
                         "each printing its own line")
    return ap.parse_args()


def workload(a):
    return {
        "workload": (f"2D lid-driven cavity, {a.m}x{a.m} jittered nodes, {a.levels} levels (/4), PHS3 + poly{a.poly}, "
                     f"k={a.k}, Courant {a.courant:g}, Re ~ U[100, 1000]; learned warm start trained on "
                     f"{a.train_episodes * a.train_steps} steps, timed on a held-out episode at Re={a.Re:g}; "
                     f"Poisson to {a.tol:g} rel. residual"),
        "nodes": a.m * a.m - 4,
        "levels": a.levels,
        "k": a.k,
        "poly_degree": a.poly,
        "Re": a.Re,
        "courant": a.courant,
        "rel_tol": a.tol,
        "l2": "inputs larger than L2 (operators + hierarchy ~2 GB per step, L2 126 MB)",
        "seed": 1,
        "step": ("host-driven solve loops (--host-driven)" if a.host_driven else
                 "one CUDA graph launch per step (solve loops as conditional nodes)"),
        "episodes": (f"each arm starts from the same saved state of an episode at Re={a.Re:g}: the lid BC applied "
                     f"at rest (p = 0), {a.eval_start} untimed steps (FP32 V-cycles, extrapolated guess), then per "
                     f"arm {a.warmup} untimed and the timed steps"),
    }


# ---------------------------------------------------------------------------
# CPU: the reference's own fractional step
# ---------------------------------------------------------------------------
class _QuietStdout:
    """The reference prints its parameters and a line per step: send fd 1 to
    /dev/null while it runs."""

    def __enter__(self):
        sys.stdout.flush()
        self.devnull = os.open(os.devnull, os.O_WRONLY)
        self.saved = os.dup(1)
        os.dup2(self.devnull, 1)
        return self

    def __exit__(self, *exc):
        os.dup2(self.saved, 1)
        os.close(self.devnull)
        os.close(self.saved)
        return False


def _ref_steps(R, O, levels, a, steps, warmup, opt):
    """warmup + timed steps of the reference's fractional_step_explicit on
    levels already handed to it, in episodes of a.episode steps from rest
    (initial_conditions + boundary_conditions of init_LDC.c re-applied,
    untimed), with the reference's own V-cycle settings: 10 V-cycles of 3 SOR
    sweeps, omega 1.0 (its V-cycle never reaches 1e-8)."""
    R.ref_set_flow(a.courant, a.Re, 1.0, 10, 3)
    R.ref_fields_alloc()
    R.ref_bc(0)
    R.ref_dt()
    done = 0
    secs = 0.0
    for phase, count in (("warmup", warmup), ("timed", steps)):
        for _ in range(count):
            if done % a.episode == 0:
                R.ref_bc(0)
            t0 = time.perf_counter()
            R.ref_step()
            if phase == "timed":
                secs += time.perf_counter() - t0
            done += 1
    return secs / max(steps, 1)


def reference_full(a, steps, warmup):
    """The reference's own fractional_step_explicit at the full workload (the
    1M-node cavity of our arm, same seed, k, polynomial degree and levels):
    the set-up is built untimed by the restatement (oracle/mgm_oracle.c,
    libm powers, OpenMP over rows), whose clouds, reorder, normals, spacing,
    operators and transfer weights are pinned bit for bit to the reference's
    own set-up, and handed to the reference's structures (oracle/ref_shim.c);
    then K steps of the reference's code (oracle/_ref/libref.so, gcc -O2,
    serial C: one core) are timed.  Without the reference build, the
    restatement's own step (in-place sweeps, as the C build runs them) is
    timed instead (kind "port")."""
    from multigrid_meshless_b200 import clouds, replicas
    from oracle import oracle as O
    cl = clouds.cavity_hierarchy(a.m, a.levels, seed=replicas.replica_seed(1, 0))
    ks, polys = [a.k] * a.levels, [a.poly] * a.levels
    t0 = time.perf_counter()
    levels = O.orc_pipeline(cl, ks, polys, reference_rows=True)
    setup_s = time.perf_counter() - t0
    with _QuietStdout():
        if O.ref_available():
            kind = "reference"
            R = O.ref_load_levels(levels)
            per = _ref_steps(R, O, levels, a, steps, warmup, "O2")
        else:
            kind = "port"
            S = O.OracleSolver(levels, a.Re, a.courant, 1.0, 3, 10, jacobi=False)
            for _ in range(warmup):
                S.step()
            t1 = time.perf_counter()
            for _ in range(steps):
                S.step()
            per = (time.perf_counter() - t1) / max(steps, 1)
    return {"kind": kind, "sec_per_step": per, "nodes": cl[0].n, "levels": a.levels, "setup_s": setup_s,
            "setup_threads": os.cpu_count()}


def reference_sample(a, steps, warmup, opt="O2"):
    """The reference's own fractional_step_explicit (its own set-up, then
    timed steps) on a cavity of a.sample-m nodes per side with the workload's
    stencil size, polynomial degree and the same construction, 3 levels; the
    -O0 build is the reference compiled as its README documents."""
    from multigrid_meshless_b200 import clouds
    from oracle import oracle as O
    nl = 3
    cl = clouds.cavity_hierarchy(a.sample_m, nl, seed=1)
    ks, polys = [a.k] * nl, [a.poly] * nl
    t0 = time.perf_counter()
    with _QuietStdout():
        if O.ref_available(opt=opt):
            kind = "reference"
            levels = O.ref_pipeline(cl, ks, polys, with_weights=True, opt=opt)
            R = O.ref_lib(opt=opt)
            setup_s = time.perf_counter() - t0
            per = _ref_steps(R, O, levels, a, steps, warmup, opt)
        else:
            kind = "port"
            levels = O.orc_pipeline(cl, ks, polys)
            setup_s = time.perf_counter() - t0
            S = O.OracleSolver(levels, a.Re, a.courant, 1.0, 3, 10, jacobi=False)
            for _ in range(warmup):
                S.step()
            t1 = time.perf_counter()
            for _ in range(steps):
                S.step()
            per = (time.perf_counter() - t1) / max(steps, 1)
    return {"kind": kind, "sec_per_step": per, "nodes": cl[0].n, "levels": nl, "setup_s": setup_s, "opt": opt}


def convergent_cpu_sample(a):
    """The library's convergent FP64 solve restated on the CPU
    (oracle/fgmres_oracle.c, OpenMP on every host core) on the sample cavity
    (a.sample_m^2 nodes, 3 levels, the workload's k and polynomial degree):
    ms per Poisson solve to a.tol from zero with a smooth source, V-cycles,
    threads.  The reference's own solver never reaches a tolerance."""
    import numpy as np

    from multigrid_meshless_b200 import clouds
    from oracle import oracle as O
    cl = clouds.cavity_hierarchy(a.sample_m, 3, seed=1)
    P = O.solver_transfer(O.orc_pipeline(cl, [a.k] * 3, [a.poly] * 3, reference_rows=False))
    S = O.ConvergentSolver(P)
    L = P[0]
    b = np.where(L.btag == 0, np.cos(np.pi * L.x) * np.cos(np.pi * L.y), 0.0)
    S.solve(b, tol=a.tol)  # warm-up
    reps = 5
    t0 = time.perf_counter()
    for _ in range(reps):
        p, it, rr, ok = S.solve(b, tol=a.tol, cheb_degree=a.cheb_degree, cheb_ratio=a.cheb_ratio)
    sec = (time.perf_counter() - t0) / reps
    return {"ms_per_solve": sec * 1e3, "vcycles": it, "rel_res": rr, "converged": bool(ok), "nodes": L.n,
            "threads": os.cpu_count()}


def cpu_baseline_entry(a, s, full_nodes):
    """A bounded sample scaled to the metric's unit: the sample's steps/s
    times (sample nodes / workload nodes), the step's work being linear in
    the node count at fixed k and V-cycle count."""
    val = (1.0 / s["sec_per_step"]) * (s["nodes"] / full_nodes)
    return {
        "value": val,
        "unit": "steps/s",
        "cores": 1,
        "kind": s["kind"],
        "sample": (f"fractional_step_explicit of the reference C code (gcc -{s['opt']}, one core) on a "
                   f"{a.sample_m}x{a.sample_m} cavity of the same construction ({s['nodes']} nodes, {s['levels']} "
                   f"levels, k={a.k}, poly {a.poly}) with its own V-cycle (10 V-cycles x 3 SOR sweeps, omega 1.0; "
                   f"it never reaches 1e-8); {s['sec_per_step'] * 1e3:.1f} ms per sample step, scaled by node count "
                   f"to {full_nodes} nodes; the reference's own set-up of the sample took {s['setup_s']:.1f} s"),
    }


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
            # nvidia-smi takes a moment to start: wait (at most 5 s) for its first
            # sample, so that a short timed region is still sampled
            t_end = time.time() + 5.0
            while time.time() < t_end and self.proc.poll() is None and os.path.getsize(self.path) == 0:
                time.sleep(0.02)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if self.proc is None:
            return out
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return out
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        out.update(sm_mhz=statistics.median(sm) if sm else None, sm_max_mhz=max(mx) if mx else None,
                   reasons=sorted(reasons), samples=len(rows))
        return out


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback 6.65 TB/s"


# DRAM bytes per launch of the level-0 FP32 smoother step (k_level_v4<0>) from
# one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum, one launch) of
# level 0 of the 1M-node cavity; the summary with its command is committed
# under profiles/.  Scaled by node count in the bench line's `traffic`.
NCU_L0_SMOOTHER_DRAM_BYTES = 200_900_000
NCU_L0_SMOOTHER_NODES = 999_996


def ncu_traffic():
    return {"dram_bytes_per_launch": float(NCU_L0_SMOOTHER_DRAM_BYTES), "nodes": float(NCU_L0_SMOOTHER_NODES)}


# ---------------------------------------------------------------------------
# step-level roofline: algorithmic bytes of every kernel of a fractional step
# ---------------------------------------------------------------------------
def step_bytes(sizes, dim, deg, fp32, vcycles, cycles, solves, steps, guesses=0):
    """Compulsory HBM bytes of `steps` fractional steps whose Poisson solves
    took `vcycles` Arnoldi steps (V-cycles) over `cycles` restart-cycle starts
    and `solves` solves: every array a kernel reads or writes counted once per
    launch, gathered vectors once per element.  sizes: [(n, nb, k)] per level.
    Per V-cycle and level l above the coarsest: a start kernel (r, dinv, btag
    in; e out), deg Chebyshev steps and deg boundary-row solves before the
    coarse correction, the residual, the restriction into l+1, the
    prolongation from l+1, one boundary-row solve and deg Chebyshev steps with
    their boundary-row solves after it; at the coarsest level the dense
    inverse.  The FGMRES in FP64: per Arnoldi step j the V-cycle's input and
    output copies, w = A z_j, the Gram-Schmidt passes over V_0..V_{j+1}
    (re-orthogonalisation passes not counted), the normalisation; per restart
    start the true residual and V_0's scaling, per cycle the update
    p += Z y; per step momentum, divergence, correction and the solve's
    right-hand-side copy.  guesses: 1 adds the extrapolated initial guess
    (history direction, its A-product, the minimal-residual dots, the update,
    the history copies), 2 also the network's inference (features, encoder,
    four message-passing layers with their index and weight streams and the
    64-wide BF16 activations, decoder) and its Chebyshev cleaning."""
    s = 4 if fp32 else 8            # V-cycle vector bytes
    slot = 6 if fp32 else 12        # weight + index per stencil slot (FP32 + int16 / FP64 + int32)
    n0, _, k0 = sizes[0]
    vc = 0.0
    L = len(sizes)
    for l in range(L - 1):
        n, nb, k = sizes[l]
        nc, _, kc = sizes[l + 1]
        cheb = n * (k * slot + 5 * s + 1 + (s * (deg - 1) / deg))   # e, r, dinv in; e', d out; d in; btag
        resid = n * (k * slot + 3 * s + 1)
        bnd = nb * (k * (s + 4) + 3 * s)
        start = n * (3 * s + 1)
        restrict = nc * (k * slot + 4 + s) + n * s                  # rows of l+1 gather l's residual
        prolong = n * (kc * slot + 4 + 2 * s) + nc * s
        vc += start + 2 * deg * cheb + (2 * deg + 1) * bnd + resid + restrict + prolong
    nc = sizes[-1][0]
    vc += nc * nc * s + 2 * nc * s
    per_vcycles = vcycles * vc
    # FGMRES (FP64 vectors, pinned FP64 operator with int32 indices)
    j_per_cycle = vcycles / max(cycles - solves, 1)  # Arnoldi steps per working cycle (each solve ends on a check)
    krylov = 0.0
    J = int(round(j_per_cycle))
    per_cycle_arnoldi = 0.0
    for j in range(max(J, 1)):
        per_cycle_arnoldi += (8 + s) * n0 + 2 * s * n0 + n0 * (12 * k0 + 8 + s) \
            + (j + 2) * 8 * n0 + (j + 3) * 8 * n0 + 16 * n0
    krylov += per_cycle_arnoldi * (vcycles / max(J, 1))
    krylov += cycles * (n0 * (12 * k0 + 24) + 16 * n0)            # true residual, V_0 scaling
    krylov += (cycles - solves) * (J * s * n0 + 16 * n0)          # p += Z y
    ops = 3 if dim == 2 else 4
    step = n0 * (ops * k0 * 8 + 4 * k0 + 8 * 8) + 2 * n0 * (2 * k0 * 8 + 4 * k0 + 5 * 8) + 16 * n0
    if guesses >= 1:
        resid = n0 * (12 * k0 + 24)
        apply = n0 * (12 * k0 + 16)
        step += 24 * n0 + 32 * n0 + resid + apply + 2 * 24 * n0 + 24 * n0
    if guesses >= 2:
        n, nb, k = sizes[0]
        cheb = n * (k * slot + 5 * s + 1 + (s * (deg - 1) / deg))
        bnd = nb * (k * (s + 4) + 3 * s)
        infer = 48 * n0 + 32 * n0 + (24 + 128) * n0 + 4 * (128 + 8 * k0 + 128) * n0 + 132 * n0 + 12 * n0
        clean = 16 * n0 + 24 * n0 + n0 * (12 * k0 + 24) + 12 * n0 + n0 * (3 * s + 1) + deg * (cheb + bnd) + 24 * n0
        step += infer + clean + n0 * (12 * k0 + 16) + 3 * 24 * n0
    return per_vcycles + krylov + steps * step


# ---------------------------------------------------------------------------
# learned warm start: trained on the GPU on plain-solver episodes, evaluated on
# held-out episodes with and without it
# ---------------------------------------------------------------------------
def c5_reynolds(a):
    """Seeded Reynolds numbers ~ U[100, 1000] of the training and held-out episodes."""
    from multigrid_meshless_b200.clouds import uniform
    return 100.0 + 900.0 * uniform(7, 0, a.train_episodes), 100.0 + 900.0 * uniform(7, 1, a.eval_episodes)


def develop(a, mg, mgm, Re, path=None):
    """An episode at Re brought past the cavity's start-up transient: the lid
    BC applied at rest (p = 0), then a.eval_start untimed steps with FP32
    V-cycles and the extrapolated guess (any mode gives the same flow to the
    tolerance).  With `path`, the state is saved there (mgm_checkpoint_save)."""
    mg.set_flow(Re=float(Re), courant=a.courant)
    mg.set_initial_guess(mgm.GUESS_EXTRAPOLATE)
    mg.apply_bc(mgm.BC_LID)
    if a.eval_start:
        mg.run_steps(mgm.MODE_FP32_IR, a.eval_start)
    if path:
        mg.checkpoint_save(path)


def c5_protocol(a, mg, mgm, seed, tmpdir):
    """The learned warm start as the C5 protocol asks: the network is trained
    on the GPU on a.train_episodes x a.train_steps fractional steps of the
    plain solver (Re ~ U[100, 1000], every solve to the tolerance), then four
    arms run the same a.eval_episodes x a.eval_steps held-out steps at unseen
    Re: plain FP64 (the previous step's pressure as the initial guess),
    FP32-in-FP64, FP32 with the extrapolated guess p_prev + c (p_prev -
    p_prev2), and learned + FP32 (the minimal-residual combination of that
    direction and the network's).  Every episode, training and held-out, is
    first brought a.eval_start steps past rest (develop); the held-out arms
    all start from the same saved state of their episode.  Every solve still
    V-cycles to the tolerance; pressures are compared with the FP64 arm's at
    the end of each held-out episode."""
    import ctypes as C

    import numpy as np

    from multigrid_meshless_b200 import _lib
    L = _lib.load()
    re_train, re_eval = c5_reynolds(a)
    t0 = time.perf_counter()
    _lib.check(L.mgm_mpnn_init(mg.h, seed, a.train_episodes * a.train_steps))
    _lib.check(L.mgm_mpnn_set_loss(mg.h, C.c_float(a.w_mse), C.c_float(a.w_res)))
    for Re in re_train:
        develop(a, mg, mgm, Re)
        _lib.check(L.mgm_mpnn_collect(mg.h, mgm.MODE_FP32_IR, a.train_steps))
    collect_s = time.perf_counter() - t0
    cnt = C.c_int()
    _lib.check(L.mgm_mpnn_dataset_size(mg.h, C.byref(cnt)))
    losses = np.zeros(a.learn_iters)
    t0 = time.perf_counter()
    _lib.check(L.mgm_mpnn_train(mg.h, 0, cnt.value, a.learn_iters, 1e-3, seed, losses.ctypes.data))
    mg.sync()
    train_s = time.perf_counter() - t0
    out = {"steps_train": int(cnt.value), "episodes_train": a.train_episodes, "Re_train": [float(r) for r in re_train],
           "steps_eval": a.eval_episodes * a.eval_steps, "episodes_eval": a.eval_episodes,
           "Re_eval": [float(r) for r in re_eval], "courant": a.courant, "adam_iters": a.learn_iters,
           "episode_start_step": a.eval_start, "loss_weights": {"mse": a.w_mse, "residual": a.w_res},
           "loss_first": float(losses[:50].mean()), "loss_last": float(losses[-50:].mean()),
           "collect_s": collect_s, "train_s": train_s}
    starts = []
    for i, Re in enumerate(re_eval):
        path = os.path.join(tmpdir, f"heldout{i}.ckpt")
        develop(a, mg, mgm, Re, path)
        starts.append((Re, path))
    arms, pressures = {}, {}
    G = mgm.GUESS_EXTRAPOLATE
    for name, mode, flags in (("fp64", mgm.MODE_FP64, 0), ("fp32", mgm.MODE_FP32_IR, 0),
                              ("fp32_extrapolated", mgm.MODE_FP32_IR, G),
                              ("learned_fp32", mgm.MODE_FP32_IR, G | mgm.GUESS_LEARNED)):
        tot = [0.0, 0.0, 0]
        ps, lsr = [], []
        for Re, path in starts:
            mg.set_flow(Re=float(Re), courant=a.courant)
            mg.checkpoint_load(path)
            mg.set_initial_guess(flags)
            ms_, pms_, vc_, _ = mg.run_steps(mode, a.eval_steps)
            tot[0] += ms_; tot[1] += pms_; tot[2] += vc_
            ps.append(mg.get_field("p"))
            lsr.append(float(np.log10(max(mg.solve_start_residual(), 1e-300))))
        steps = a.eval_episodes * a.eval_steps
        arms[name] = {"ms_per_step": tot[0] / steps, "poisson_ms": tot[1] / steps, "vcycles_per_step": tot[2] / steps,
                      "steps_per_s": steps / (tot[0] / 1e3),
                      "start_rel_residual": 10.0 ** (sum(lsr) / len(lsr))}
        pressures[name] = ps
    mg.set_initial_guess(0)
    rel = lambda x, y: max(float(np.linalg.norm(u - v) / np.linalg.norm(v)) for u, v in zip(x, y))
    out.update(arms)
    lf, f32, ex, f64 = arms["learned_fp32"], arms["fp32"], arms["fp32_extrapolated"], arms["fp64"]
    out["vcycles_saved_per_step_vs_fp32"] = f32["vcycles_per_step"] - lf["vcycles_per_step"]
    out["vcycles_saved_per_step_vs_extrapolation"] = ex["vcycles_per_step"] - lf["vcycles_per_step"]
    out["speedup_learned_fp32_vs_fp64"] = f64["ms_per_step"] / lf["ms_per_step"]
    out["speedup_learned_fp32_vs_fp32"] = f32["ms_per_step"] / lf["ms_per_step"]
    out["speedup_fp32_vs_fp64"] = f64["ms_per_step"] / f32["ms_per_step"]
    for name in ("fp32", "fp32_extrapolated", "learned_fp32"):
        out[f"pressure_rel_l2_{name}_vs_fp64"] = rel(pressures[name], pressures["fp64"])
    out["start_rel_residual_note"] = ("geometric mean over the held-out solves of |b - A p0| / |b| at each solve's "
                                      "start (p0 its initial guess); one V-cycle reduces it about 3x")
    out["note"] = (f"held-out episodes at unseen Re, each arm from the same saved state {a.eval_start} steps past "
                   "rest; pressures compared after each episode with the plain FP64 arm's (each solve to the "
                   "tolerance)")
    return out


# ---------------------------------------------------------------------------
def run_ours(a, rank, world, local_rank):
    import numpy as np

    import multigrid_meshless_b200 as mgm
    from multigrid_meshless_b200 import api, clouds

    from multigrid_meshless_b200 import replicas

    api.set_device(local_rank)
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist_
        torch.cuda.set_device(local_rank)
        dist_.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
        dist = dist_
    timing = replicas.Timing(dist, f"cuda:{local_rank}")
    barrier, max_over_ranks = timing.barrier, timing.max_over_ranks

    t0 = time.perf_counter()
    cl = clouds.cavity_hierarchy(a.m, a.levels, seed=replicas.replica_seed(1, rank))
    mg = api.Multigrid(cl, [a.k] * a.levels, [a.poly] * a.levels)
    setup_s = time.perf_counter() - t0
    setup_launches = api.kernel_launches()
    print(f"setup_launches={setup_launches}", file=sys.stderr, flush=True)
    n = mg.n()
    mg.set_solver(rel_tol=a.tol, max_iters=100, cheb_degree=a.cheb_degree, cheb_ratio=a.cheb_ratio)
    mg.use_step_graph(not a.host_driven)

    fast = mgm.MODE_FP32_IR
    LEARNED = mgm.GUESS_EXTRAPOLATE | mgm.GUESS_LEARNED

    # the learned warm start, trained on the GPU and evaluated on held-out
    # steps (every rank trains its own network on its own replica)
    tmpdir = tempfile.mkdtemp(prefix="mgm_bench_")
    learned = None
    head_flags = mgm.GUESS_EXTRAPOLATE
    if not a.no_learned:
        learned = c5_protocol(a, mg, mgm, replicas.replica_seed(1, rank), tmpdir)
        head_flags = LEARNED

    # the timed episode at a.Re, brought past the start-up transient once;
    # every arm below starts from this saved state
    start = os.path.join(tmpdir, "timed.ckpt")
    develop(a, mg, mgm, a.Re, start)

    counts = {}

    def arm(mode, flags, steps, warm):
        """the timed episode from its saved state: `warm` untimed steps, then
        `steps` timed steps (device time of the steps only)"""
        mg.set_flow(Re=a.Re, courant=a.courant)
        mg.checkpoint_load(start)
        mg.set_initial_guess(flags)
        if warm:
            mg.run_steps(mode, warm)
        barrier()
        mg.sync()
        out = mg.run_steps(mode, steps)
        counts[(mode, flags)] = list(mg.solve_counters())
        return out

    def smoother_pass(steps):
        """CUDA events around every level-0 smoother launch, recorded inside
        the V-cycle graphs of a host-driven pass of the same steps (event
        nodes cannot sit in the step graph's conditional bodies): total ms,
        launches, algorithmic bytes per launch"""
        mg.profile_smoother(True)
        arm(fast, head_flags, 1, 0)  # captures the V-cycle graphs with their event nodes
        mg.sync()
        s0 = mg.profile_read()
        arm(fast, head_flags, steps, 0)
        s1 = mg.profile_read()
        mg.profile_smoother(False)
        return s1[0] - s0[0], s1[1] - s0[1], s1[2]

    # the denominator: plain FP64 V-cycles in FP64 FGMRES, the previous
    # pressure as the initial guess
    plain_ms, plain_pms, plain_vc, _ = arm(mgm.MODE_FP64, 0, a.steps, a.warmup)
    plain_ms = max_over_ranks(plain_ms)

    # headline: learned warm start + FP32 V-cycles in FP64 FGMRES, each step
    # one graph launch (the solve's loops as conditional nodes), device-timed
    # on the library's stream
    clocks = ClockSampler(local_rank)
    clocks.start()
    l0 = api.kernel_launches()
    ms, pms, vc, err = arm(fast, head_flags, a.steps, a.warmup)
    launches = api.kernel_launches() - l0
    ck = clocks.stop()
    barrier()
    ms = max_over_ranks(ms)
    head_counts = counts[(fast, head_flags)]

    # FP32 without any guess beyond the previous pressure, on the same steps
    f32_ms, f32_pms, f32_vc, _ = arm(fast, 0, a.steps, a.warmup)
    f32_ms = max_over_ranks(f32_ms)

    # the headline steps with the solve's loops driven from the host (one read
    # of the loop flags per Arnoldi step, V-cycle graphs): what the one-graph step saves
    mg.use_step_graph(False)
    hd_ms, hd_pms, hd_vc, _ = arm(fast, head_flags, a.steps, a.warmup)
    mg.use_step_graph(not a.host_driven)
    hd_ms = max_over_ranks(hd_ms)

    # the headline steps with the V-cycle's kernels launched the ordinary way
    # (no programmatic dependent launch): what chaining them saves
    mg.use_launch_chaining(False)
    uc_ms, uc_pms, uc_vc, _ = arm(fast, head_flags, a.steps, a.warmup)
    mg.use_launch_chaining(True)
    uc_ms = max_over_ranks(uc_ms)

    # ... and with the small levels' V-cycle as one cooperative launch
    # (mgm_use_fused_coarse, opt-in) instead of a kernel per operation
    fused_on = mg.fused_coarse_available()
    mg.use_fused_coarse(True)
    uf_ms, uf_pms, uf_vc, _ = arm(fast, head_flags, a.steps, a.warmup)
    mg.use_fused_coarse(False)
    uf_ms = max_over_ranks(uf_ms)

    # the dominant kernel's launches, timed by events (roofline)
    sm_ms, sm_launch, sm_bytes = smoother_pass(a.steps)

    # the same steps with the FP16 operator (D^-1 A) in the FP32 V-cycle
    # (mgm_use_half_operator); reported beside the headline, not as it
    half = None
    if not a.no_half:
        mg.use_half_operator(True)
        half_ms, half_pms, half_vc, half_err = arm(fast, head_flags, a.steps, a.warmup)
        half_ms = max_over_ranks(half_ms)
        h_ms, h_launch, h_bytes = smoother_pass(min(a.steps, 10))
        mg.use_half_operator(False)
        h_avg_s = (h_ms / 1e3) / max(h_launch, 1)
        half = {"steps_per_s": a.steps * world / (half_ms / 1e3), "ms_per_step": half_ms / a.steps,
                "poisson_ms": half_pms / a.steps, "vcycles_per_step": half_vc / a.steps,
                "steady_err_last": half_err,
                "level0_smoother": {"kernel": "k_level_h4<0> (FP16 D^-1 A + int16 offsets, one 16-byte load "
                                              "per slot per 4 interleaved rows, rows in difference form)",
                                    "bytes_per_launch": h_bytes, "launches": h_launch,
                                    "avg_launch_us": h_avg_s * 1e6,
                                    "achieved_gbs": h_bytes / h_avg_s / 1e9 if h_launch else None}}

    # end to end through the public API with page-locked host buffers:
    # per step H2D of u, v and D2H of u, v, p (the reference's `update host(field[0])`)
    bufs = [api.PinnedArray(n) for _ in range(5)]
    mg.set_flow(Re=a.Re, courant=a.courant)
    mg.checkpoint_load(start)
    mg.set_initial_guess(head_flags)
    if a.warmup:
        mg.run_steps(fast, a.warmup)
    bufs[0].array[:] = mg.get_field("u")
    bufs[1].array[:] = mg.get_field("v")
    barrier()
    mg.sync()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        mg.step_host(fast, bufs[0].ptr, bufs[1].ptr, bufs[2].ptr, bufs[3].ptr, bufs[4].ptr)
        bufs[0].array, bufs[2].array = bufs[2].array, bufs[0].array
        bufs[0].ptr, bufs[2].ptr = bufs[2].ptr, bufs[0].ptr
        bufs[1].array, bufs[3].array = bufs[3].array, bufs[1].array
        bufs[1].ptr, bufs[3].ptr = bufs[3].ptr, bufs[1].ptr
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s)
    finite = bool(np.all(np.isfinite(bufs[0].array)))
    for b in bufs:
        b.free()
    mg.set_initial_guess(0)

    line = None
    if rank == 0:
        steps_total = a.steps * world
        value = steps_total / (ms / 1e3)
        peak, peak_src = measured_peak()
        avg_launch_s = (sm_ms / 1e3) / max(sm_launch, 1)
        achieved = sm_bytes / avg_launch_s / 1e9 if sm_launch else None
        sizes = [tuple(mg.sizes[l][:3]) for l in range(mg.nl)]
        sb = step_bytes(sizes, 2, a.cheb_degree, True, *head_counts, a.steps,
                        guesses=2 if head_flags & mgm.GUESS_LEARNED else 1)
        step_roof = {"bytes_per_step": sb / a.steps, "achieved": sb / (ms / 1e3) / 1e9, "unit": "GB/s",
                     "frac": sb / (ms / 1e3) / 1e9 / peak,
                     "vcycles": head_counts[0], "restart_cycle_starts": head_counts[1], "solves": head_counts[2],
                     "model": ("compulsory bytes of every kernel of the step (step_bytes in bench.py): V-cycle "
                               "levels, FP64 FGMRES, momentum/divergence/correction; re-orthogonalisation "
                               "passes not counted")}
        tr = ncu_traffic()
        traffic = None
        if tr and tr.get("nodes"):
            traffic = float(tr["dram_bytes_per_launch"]) * (n / float(tr["nodes"]))
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "steps/s",
            "n_gpus": world,
            "steps": a.steps,
            "warmup": a.warmup,
            "ms_per_step": ms / a.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 V-cycle inside f64 FGMRES (f64 operators, residuals, solution)",
            "data": "synthetic (seeded jittered cloud, no mesh files)",
            "config": workload(a),
            "poisson_ms": pms / a.steps,
            "vcycles_per_step": vc / a.steps,
            "steady_err_last": err,
            "plain_fp64": {"steps_per_s": a.steps * world / (plain_ms / 1e3), "ms_per_step": plain_ms / a.steps,
                           "poisson_ms": plain_pms / a.steps, "vcycles_per_step": plain_vc / a.steps,
                           "note": "FP64 V-cycle in FP64 FGMRES, previous pressure as the initial guess, same steps"},
            "speedup_vs_plain_fp64": plain_ms / ms,
            "fp32_no_guess": {"steps_per_s": a.steps * world / (f32_ms / 1e3), "ms_per_step": f32_ms / a.steps,
                              "poisson_ms": f32_pms / a.steps, "vcycles_per_step": f32_vc / a.steps},
            "host_driven_fp32": {"ms_per_step": hd_ms / a.steps, "poisson_ms": hd_pms / a.steps,
                                 "vcycles_per_step": hd_vc / a.steps,
                                 "note": ("the same steps with the solve's loops driven from the host (one read of "
                                          "the loop flags per Arnoldi step, each V-cycle a graph replay); the "
                                          "headline runs each step as one graph launch")},
            "unchained_fp32": {"ms_per_step": uc_ms / a.steps, "poisson_ms": uc_pms / a.steps,
                               "vcycles_per_step": uc_vc / a.steps,
                               "note": ("the headline steps with the V-cycle's kernels launched without "
                                        "programmatic dependent launch (mgm_use_launch_chaining(0))")},
            "fused_coarse_fp32": {"ms_per_step": uf_ms / a.steps, "poisson_ms": uf_pms / a.steps,
                                  "vcycles_per_step": uf_vc / a.steps, "fused_available": fused_on,
                                  "note": ("the headline steps with the levels below 65,536 rows as one cooperative "
                                           "launch per V-cycle (mgm_use_fused_coarse(1)) instead of one kernel per "
                                           "operation")},
            "learned_warm_start": learned,
            "half_operator": half,
            "headline_arm": ("learned warm start (minimal-residual combination of the network's increment and "
                             "the last pressure increment) + FP32 V-cycle inside FP64 FGMRES"
                             if head_flags & mgm.GUESS_LEARNED else
                             "FP32 V-cycle inside FP64 FGMRES with the extrapolated initial guess (no network: "
                             "--no-learned)"),
            "e2e": {"value": steps_total / e2e_s, "unit": "steps/s", "h2d_bytes_per_step": 2 * 8 * n,
                    "d2h_bytes_per_step": 3 * 8 * n, "finite": finite},
            "roofline": {"bound": "hbm", "kernel": ("level-0 FP32 Chebyshev smoother step (k_level_v4<0>: FP32 "
                                                    "weights + int16 offsets, slots sorted by neighbour, four rows "
                                                    "per thread with vector loads)"),
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                         "bytes_per_launch": sm_bytes, "launches": sm_launch,
                         "avg_launch_us": avg_launch_s * 1e6, "peak_source": peak_src,
                         "timing": ("CUDA events around every level-0 smoother launch, recorded inside the V-cycle "
                                    "graphs of a host-driven pass of the same steps after the timed region"),
                         "step": step_roof},
            "clocks": ck,
            "gpu_launches": launches,
            "setup_s": setup_s,
        }
        if world == 1 and not a.no_cpu_baseline:
            s = reference_sample(a, steps=3, warmup=1)
            cb = cpu_baseline_entry(a, s, n)
            # the same sample through the reference compiled as its README
            # documents (-O0), beside the -O2 figure
            s0 = reference_sample(a, steps=2, warmup=0, opt="O0")
            cs = convergent_cpu_sample(a)
            cb["variants"] = {"reference_gcc_O2_1core": cb["value"],
                              "reference_gcc_O0_1core": cpu_baseline_entry(a, s0, n)["value"],
                              "note": ("the reference's OpenACC builds (nvc -acc multicore / GPU) are unavailable on "
                                       "this box (no nvc); its C code is serial")}
            cs["ms_per_solve_scaled_to_workload"] = cs["ms_per_solve"] * n / cs["nodes"]
            cs["note"] = ("the library's convergent FP64 solve restated in C (oracle/fgmres_oracle.c, OpenMP, "
                          f"{cs['threads']} threads) on the {a.sample_m}^2 sample, solved to {a.tol:g} from zero; "
                          "scaled by node count to the workload; the GPU's Poisson ms per step is poisson_ms")
            cb["convergent_fp64_cpu"] = cs
            line["cpu_baseline"] = cb
    mg.close()
    shutil.rmtree(tmpdir, ignore_errors=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return line


# ---------------------------------------------------------------------------
# the other configurations (one GPU, each its own line)
# ---------------------------------------------------------------------------
def run_other(a):
    import numpy as np

    import multigrid_meshless_b200 as mgm
    from multigrid_meshless_b200 import api, clouds
    t0 = time.perf_counter()
    timple = a.workload == "timple"
    if a.workload in ("annulus", "timple"):
        nl, k, poly, Re, courant, deg, ratio = 6, 30, 4, 100.0, 0.5, 4, 10.0
        cl = clouds.annulus_hierarchy(clouds.annulus_h_for_nodes(1_000_000), nl, seed=1)
        bc = mgm.BC_TAYLOR_COUETTE
        desc = (f"2D Taylor-Couette annulus r in [0.5, 1], jittered polar nodes, {nl} levels (/4), PHS3 + poly{poly}, "
                f"k={k}, Re={Re:g}, Courant {courant:g}, inner wall u_theta = 1")
    else:
        nl, k, poly, Re, courant, deg, ratio = 4, 35, 2, 400.0, 0.3, 4, 10.0
        cl = clouds.cube_hierarchy(128, nl, seed=1)
        bc = mgm.BC_LID
        desc = (f"3D lid-driven cube, 128^3 jittered nodes (edges/corners removed), {nl} levels (/8), PHS3 + "
                f"poly{poly}, k={k}, Re={Re:g}, Courant {courant:g}")
    mg = api.Multigrid(cl, [k] * nl, [poly] * nl)
    setup_s = time.perf_counter() - t0
    n = mg.n()
    mg.set_flow(Re=Re, courant=courant)
    mg.set_solver(rel_tol=a.tol, max_iters=100, cheb_degree=deg, cheb_ratio=ratio)

    # the explicit scheme is diffusion-unstable at these spacings; the annulus
    # grows faster than the cavity, so its episodes are shorter.  TIMPLE (the
    # reference main's solver, iter_timple 1 and iter_momentum 5 as shipped)
    # grows from its third step from rest at 1M nodes: episodes of 2 steps
    if timple:
        mg.set_timple(1, 5, 1.0, 1.0)
        episode = 2
    else:
        episode = min(a.episode, 5) if a.workload == "annulus" else a.episode

    def arm(mode, steps):
        tot = [0.0, 0.0, 0, 0.0]
        done = 0
        while done < steps:
            m_ = min(episode, steps - done)
            mg.apply_bc(bc)
            if timple:
                ms_, vc_, err_ = mg.timple_run(mode, m_)
                pms_ = float("nan")
            else:
                ms_, pms_, vc_, err_ = mg.run_steps(mode, m_)
            tot[0] += ms_; tot[1] += pms_; tot[2] += vc_; tot[3] = err_
            done += m_
        return tot
    arm(mgm.MODE_FP32_IR, a.warmup)
    arm(mgm.MODE_FP64, min(a.warmup, 2))
    pl = arm(mgm.MODE_FP64, a.steps)
    clocks = ClockSampler(0)
    clocks.start()
    l0 = api.kernel_launches()
    ms, pms, vc, err = arm(mgm.MODE_FP32_IR, a.steps)
    launches = api.kernel_launches() - l0
    ck = clocks.stop()
    # the level-0 smoother's launches timed by CUDA events in the V-cycle
    # graphs of a host-driven pass of the same steps (roofline)
    mg.profile_smoother(True)
    arm(mgm.MODE_FP32_IR, 1)
    mg.sync()
    sm0 = mg.profile_read()
    arm(mgm.MODE_FP32_IR, a.steps)
    sm1 = mg.profile_read()
    mg.profile_smoother(False)
    sm_ms, sm_launch, sm_bytes = sm1[0] - sm0[0], sm1[1] - sm0[1], sm1[2]
    peak, peak_src = measured_peak()
    avg = (sm_ms / 1e3) / max(sm_launch, 1)
    ach = sm_bytes / avg / 1e9 if sm_launch else None
    compat = None
    if timple:
        # the same TIMPLE steps with compatible right-hand sides
        # (mgm_set_compatible_rhs): bounded, so one episode of all the steps
        mg.set_compatible_rhs(True)
        mg.apply_bc(bc)
        mg.timple_run(mgm.MODE_FP32_IR, min(a.warmup, 2))
        mg.apply_bc(bc)
        c_ms, c_vc, c_err = mg.timple_run(mgm.MODE_FP32_IR, a.steps)
        mg.set_compatible_rhs(False)
        compat = {"steps_per_s": a.steps / (c_ms / 1e3), "ms_per_step": c_ms / a.steps,
                  "vcycles_per_step": c_vc / a.steps, "steady_err_last": c_err,
                  "episodes": f"one episode of {a.steps} steps from rest",
                  "note": ("p' source projected along lap_Poison's left null vector before the pinned solve; "
                           "without it the pin's singular response grows, hence the two-step episodes above")}
    mg.close()
    if timple:
        desc += ", TIMPLE steps (iter_timple 1, iter_momentum 5), p' to the tolerance"
    metric = ("TIMPLE steps/s, p' to 1e-8 resid: FP32-in-FP64 vs plain FP64 GPU (annulus)" if timple else
              f"NS steps/s & Poisson ms, 1e-8 resid: FP32-in-FP64 vs plain FP64 GPU ({a.workload})")
    nan_none = (lambda x: None if x != x else x)
    return {
        "metric": metric,
        "value": a.steps / (ms / 1e3), "unit": "steps/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 V-cycle inside f64 FGMRES", "data": "synthetic (seeded jittered cloud, no mesh files)",
        "config": {"workload": desc, "nodes": n, "levels": nl, "k": k, "poly_degree": poly, "rel_tol": a.tol,
                   "cheb_degree": deg, "cheb_ratio": ratio,
                   "episodes": f"steps in episodes of {episode} from rest"},
        "poisson_ms": nan_none(pms / a.steps), "vcycles_per_step": vc / a.steps, "steady_err_last": err,
        "plain_fp64": {"steps_per_s": a.steps / (pl[0] / 1e3), "ms_per_step": pl[0] / a.steps,
                       "poisson_ms": nan_none(pl[1] / a.steps), "vcycles_per_step": pl[2] / a.steps},
        "roofline": {"bound": "hbm", "kernel": "level-0 FP32 Chebyshev smoother step", "achieved": ach,
                     "peak": peak, "unit": "GB/s", "frac": (ach / peak) if ach else None,
                     "bytes_per_launch": sm_bytes, "launches": sm_launch, "avg_launch_us": avg * 1e6,
                     "peak_source": peak_src},
        "clocks": ck, "gpu_launches": launches, "setup_s": setup_s,
        **({"compatible_rhs": compat} if compat is not None else {}),
    }


def weights_flops(rep):
    """FP64 throughput of the one-launch weight assembly: per system of order
    N the Gauss-Jordan elimination on [A | I] (N pivots, each updating N - 1
    rows of 2N entries with a multiply and a subtract: 4 N^2 (N - 1) flops;
    the operator rows' products are not counted) over the launch's time."""
    flops = sum(c["systems"] * 4.0 * c["order"] ** 2 * (c["order"] - 1) for c in rep["classes"])
    sec = rep["weights_ms"] / 1e3
    return {"gj_flops": flops, "achieved_fp64_tflops": flops / sec / 1e12 if sec > 0 else None,
            "flops_note": ("Gauss-Jordan flops only (4 N^2 (N - 1) per system); no measured FP64 peak is available "
                           "on this pool to divide by")}


def run_batch(a):
    import numpy as np

    import multigrid_meshless_b200 as mgm
    from multigrid_meshless_b200 import api, clouds
    nl, nrhs = 4, 64
    t0 = time.perf_counter()
    h = clouds.shell_h_for_nodes(int(3_000_000 * 0.875))
    cl = clouds.shell_hierarchy(h, nl, seed=1)
    ks = [clouds.shell_stencil_sizes(cl[0], 40, 60)] + [clouds.shell_stencil_sizes(c, 25, 35) for c in cl[1:]]
    polys = [3] + [2] * (nl - 1)
    b = api.Batch(cl, ks, polys, autotune=True)
    setup_s = time.perf_counter() - t0
    print(f"setup_launches={api.kernel_launches()}", file=sys.stderr, flush=True)
    rep = b.weights_report()
    lev = b.level(0)
    c0 = clouds.Cloud(lev["x"], lev["y"], lev["z"], lev["nx"], lev["ny"], lev["nz"], lev["btag"], 0, 3, 0.0,
                      "shell3d", {"r_in": 0.5, "r_out": 1.0})
    f0 = clouds.gaussian_fields(c0, nrhs, seed=5)
    inner = lev["btag"] == 0
    f0[:, ~inner] = 0.0
    f0[:, inner] -= f0[:, inner].mean(1, keepdims=True)
    f0[:, 0] = 0.0
    # right-hand sides and solutions in page-locked host memory (the copies of
    # the end-to-end number run from it)
    pin_rhs, pin_sol = api.PinnedArray(f0.size), api.PinnedArray(f0.size)
    f = pin_rhs.array.reshape(f0.shape)
    f[:] = f0
    sol_buf = pin_sol.array.reshape(f0.shape)
    b.set_solver(a.tol, 24, 4, 10.0)
    arms = {}
    for name, mode in (("fp32", mgm.MODE_FP32_IR), ("fp64", mgm.MODE_FP64)):
        b.solve(f, mode, out=sol_buf)  # warm-up (allocates the Krylov space)
        dev, wall, vcs, worst = 0.0, 0.0, 0, 0.0
        reps = max(1, min(a.steps, 3))
        for _ in range(reps):
            t1 = time.perf_counter()
            sol, vc, rr, ms = b.solve(f, mode, out=sol_buf)
            wall += time.perf_counter() - t1
            dev += ms
            vcs += vc
            worst = max(worst, float(rr.max()))
        arms[name] = {"ms_per_solve": dev / reps, "wall_ms_per_solve": wall * 1e3 / reps, "vcycles": vcs / reps,
                      "worst_rel_res": worst, "sol": sol.copy()}
    rel = max(float(np.linalg.norm(x - y) / np.linalg.norm(y)) for x, y in zip(arms["fp32"]["sol"], arms["fp64"]["sol"]))
    for v in arms.values():
        v.pop("sol")
    n_tot = sum(c.n for c in cl)
    b.close()
    pin_rhs.free()
    pin_sol.free()
    return {
        "metric": "64 Poisson right-hand sides to 1e-8 through one batched V-cycle (3D shell, per-node stencils)",
        "value": nrhs / (arms["fp32"]["ms_per_solve"] / 1e3), "unit": "RHS solved/s", "n_gpus": 1,
        "steps": 3, "warmup": 1, "ms_per_step": arms["fp32"]["ms_per_solve"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 V-cycle inside f64 FGMRES",
        "data": "synthetic (seeded shell cloud, seeded sums of 8 Gaussians)",
        "config": {"workload": f"3D sphere-in-sphere shell r in [0.5, 1], {n_tot} nodes over {nl} levels (/8), "
                               f"k 40/60 (poly 3) on the fine level and 25/35 (poly 2) below by boundary proximity",
                   "nodes_total": n_tot, "nodes_fine": cl[0].n, "levels": nl,
                   "nrhs": nrhs, "rel_tol": a.tol},
        "weights": dict(rep, **weights_flops(rep)),
        "fp32": arms["fp32"], "fp64": arms["fp64"],
        "solution_rel_l2_fp32_vs_fp64": rel,
        "e2e": {"value": nrhs / (arms["fp32"]["wall_ms_per_solve"] / 1e3), "unit": "RHS solved/s",
                "h2d_bytes_per_step": nrhs * cl[0].n * 8, "d2h_bytes_per_step": nrhs * cl[0].n * 8},
        "setup_s": setup_s,
    }


def run_reference(a, rank):
    """The reference arm: the reference's own fractional step at the full
    workload (reference_full), one JSON line on rank 0; other ranks exit."""
    if rank != 0:
        return None
    a.episode = a.warmup + max(a.steps, 1)  # one episode from rest
    s = reference_full(a, steps=max(a.steps, 1), warmup=a.warmup)
    val = 1.0 / s["sec_per_step"]
    cfg = workload(a)
    cfg["reference_solver"] = ("the reference's own multigrid_Poisson_solver: a fixed 10 V-cycles of 3 SOR sweeps "
                               "(omega 1.0) per step; it has no tolerance test and never reaches 1e-8")
    cfg["episodes"] = (f"one episode from rest at Re={a.Re:g}: {a.warmup} warm-up and {max(a.steps, 1)} timed steps "
                       "(the reference's work per step does not depend on the flow: a fixed V-cycle count)")
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": val,
        "unit": "steps/s",
        "n_gpus": a.gpus,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": 1e3 / val,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded jittered cloud, no mesh files)",
        "config": cfg,
        "cpu_baseline": {
            "value": val, "unit": "steps/s", "cores": 1, "kind": s["kind"],
            "sample": (f"fractional_step_explicit of the reference C code (gcc -O2, serial: one core) on the full "
                       f"workload ({s['nodes']} nodes, {s['levels']} levels), {a.steps} timed steps after "
                       f"{a.warmup} warm-up steps, in episodes of {a.episode} from rest; the set-up was built untimed "
                       f"by the restatement (bit-identical to the reference's own set-up) in {s['setup_s']:.1f} s "
                       f"on {s['setup_threads']} threads and handed to the reference's structures"),
        },
        "e2e": {"value": val, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "setup_s": s["setup_s"],
    }


def main():
    a = parse()
    if a.Re is None:
        a.Re = float(c5_reynolds(a)[1][0])
    from multigrid_meshless_b200.replicas import env_rank
    rank, world, local_rank = env_rank()
    if a.impl == "reference":
        line = run_reference(a, rank)
    elif a.workload == "shell-batch":
        line = run_batch(a) if rank == 0 else None
    elif a.workload in ("annulus", "timple", "cube"):
        line = run_other(a) if rank == 0 else None
    else:
        line = run_ours(a, rank, world, local_rank)
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
