#!/usr/bin/env python
"""bench.py -- NS steps/s & Poisson ms at 1M nodes, Poisson solved to a 1e-8
relative residual: FP32-in-FP64 refinement vs plain FP64 on the GPU.

Workload (the 1M-node 2D lid-driven cavity): unit square, 1000 x 1000 jittered
Cartesian nodes (999,996 after the corner nodes are removed), 6 levels each
coarser by 4x, PHS degree 3, polynomial degree 4 (15 terms), 30-node stencils,
Re = 100, Courant 0.5.  A step is one fractional step (momentum, divergence,
Poisson solve to 1e-8, velocity correction) through the C ABI.

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
    ap.add_argument("--Re", type=float, default=100.0)
    ap.add_argument("--courant", type=float, default=0.5)
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--cheb-degree", type=int, default=3)
    ap.add_argument("--cheb-ratio", type=float, default=20.0)
    ap.add_argument("--episode", type=int, default=10,
                    help="steps per episode from rest (the explicit scheme is unstable beyond ~12 steps at 1M nodes)")
    ap.add_argument("--sample-m", type=int, default=128, help="cavity size of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned warm-start measurement")
    ap.add_argument("--no-half", action="store_true", help="skip the FP16-operator measurement")
    ap.add_argument("--learn-episodes", type=int, default=12, help="training episodes (Re ~ U[100, 1000])")
    ap.add_argument("--learn-iters", type=int, default=400, help="Adam iterations of the GPU training")
    ap.add_argument("--workload", choices=["cavity", "annulus", "timple", "cube", "shell-batch"], default="cavity",
                    help="cavity: the headline (1M-node cavity); annulus / cube / shell-batch: the other configs, "
                         "each printing its own line")
    return ap.parse_args()


def workload(a):
    return {
        "workload": f"2D lid-driven cavity, {a.m}x{a.m} jittered nodes, {a.levels} levels (/4), PHS3 + poly{a.poly}, "
                    f"k={a.k}, Re={a.Re:g}, Courant {a.courant:g}, Poisson to {a.tol:g} rel. residual",
        "nodes": a.m * a.m - 4,
        "levels": a.levels,
        "k": a.k,
        "poly_degree": a.poly,
        "Re": a.Re,
        "courant": a.courant,
        "rel_tol": a.tol,
        "l2": "inputs larger than L2 (operators + hierarchy ~2 GB per step, L2 126 MB)",
        "seed": 1,
        "episodes": f"steps run in episodes of {a.episode} from rest (lid BC re-applied, p = 0; untimed resets)",
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
NCU_L0_SMOOTHER_DRAM_BYTES = 200_700_000
NCU_L0_SMOOTHER_NODES = 999_996


def ncu_traffic():
    return {"dram_bytes_per_launch": float(NCU_L0_SMOOTHER_DRAM_BYTES), "nodes": float(NCU_L0_SMOOTHER_NODES)}


# ---------------------------------------------------------------------------
# step-level roofline: algorithmic bytes of every kernel of a fractional step
# ---------------------------------------------------------------------------
def step_bytes(sizes, dim, deg, fp32, vcycles, cycles, solves, steps):
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
    right-hand-side copy."""
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
    return per_vcycles + krylov + steps * step


# ---------------------------------------------------------------------------
# learned warm start: trained on the GPU on plain-solver episodes, evaluated on
# held-out episodes with and without it
# ---------------------------------------------------------------------------
def learned_arm(a, mg, mgm, n):
    import ctypes as C

    import numpy as np

    from multigrid_meshless_b200 import _lib
    from multigrid_meshless_b200.clouds import uniform
    L = _lib.load()
    ep_len = a.episode
    n_train, n_eval = a.learn_episodes, 2
    res_train = 100.0 + 900.0 * uniform(7, 0, n_train)
    res_eval = 100.0 + 900.0 * uniform(7, 1, n_eval)
    t0 = time.perf_counter()
    _lib.check(L.mgm_mpnn_init(mg.h, 1, n_train * ep_len))
    for Re in res_train:
        mg.set_flow(Re=float(Re), courant=a.courant)
        mg.apply_bc(mgm.BC_LID)
        _lib.check(L.mgm_mpnn_collect(mg.h, mgm.MODE_FP32_IR, ep_len))
    collect_s = time.perf_counter() - t0
    cnt = C.c_int()
    _lib.check(L.mgm_mpnn_dataset_size(mg.h, C.byref(cnt)))
    n_fit = max(1, cnt.value - ep_len)
    losses = np.zeros(a.learn_iters)
    t0 = time.perf_counter()
    _lib.check(L.mgm_mpnn_train(mg.h, 0, n_fit, a.learn_iters, 1e-3, 1, losses.ctypes.data))
    train_s = time.perf_counter() - t0
    held = C.c_double()
    _lib.check(L.mgm_mpnn_eval(mg.h, n_fit, cnt.value - n_fit, C.byref(held)))
    out = {"episodes_train": int(n_train), "steps_train": int(cnt.value), "episodes_eval": n_eval,
           "steps_eval": n_eval * ep_len, "Re_train": "U[100, 1000] (seeded)",
           "Re_eval": [float(r) for r in res_eval], "adam_iters": a.learn_iters,
           "loss_first": float(losses[:20].mean()), "loss_last": float(losses[-20:].mean()),
           "loss_held_out_samples": float(held.value), "collect_s": collect_s, "train_s": train_s}
    arms = {}
    pressures = {}
    for name, mode, warm in (("fp64", mgm.MODE_FP64, 0), ("fp32", mgm.MODE_FP32_IR, 0),
                             ("learned_fp32", mgm.MODE_FP32_IR, 1)):
        _lib.check(L.mgm_set_warm_start(mg.h, warm))
        tot = [0.0, 0.0, 0]
        ps = []
        for Re in res_eval:
            mg.set_flow(Re=float(Re), courant=a.courant)
            mg.apply_bc(mgm.BC_LID)
            ms_, pms_, vc_, _ = mg.run_steps(mode, ep_len)
            tot[0] += ms_; tot[1] += pms_; tot[2] += vc_
            ps.append(mg.get_field("p"))
        steps = n_eval * ep_len
        arms[name] = {"ms_per_step": tot[0] / steps, "poisson_ms": tot[1] / steps, "vcycles_per_step": tot[2] / steps}
        pressures[name] = ps
    _lib.check(L.mgm_set_warm_start(mg.h, 0))
    mg.set_flow(Re=a.Re, courant=a.courant)
    rel = lambda x, y: max(float(np.linalg.norm(u - v) / np.linalg.norm(v)) for u, v in zip(x, y))
    out.update(arms)
    out["vcycles_saved_per_step"] = arms["fp32"]["vcycles_per_step"] - arms["learned_fp32"]["vcycles_per_step"]
    out["speedup_learned_fp32_vs_fp64"] = arms["fp64"]["ms_per_step"] / arms["learned_fp32"]["ms_per_step"]
    out["speedup_fp32_vs_fp64"] = arms["fp64"]["ms_per_step"] / arms["fp32"]["ms_per_step"]
    out["pressure_rel_l2_learned_fp32_vs_fp64"] = rel(pressures["learned_fp32"], pressures["fp64"])
    out["pressure_rel_l2_fp32_vs_fp64"] = rel(pressures["fp32"], pressures["fp64"])
    out["note"] = ("held-out episodes of a.episode steps from rest at unseen Re; the FP64 arm is the plain FP64 "
                   "V-cycle solve, pressures compared after each episode")
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
    mg.set_flow(Re=a.Re, courant=a.courant)
    mg.set_solver(rel_tol=a.tol, max_iters=100, cheb_degree=a.cheb_degree, cheb_ratio=a.cheb_ratio)
    mg.apply_bc(mgm.BC_LID)

    fast = mgm.MODE_FP32_IR

    counts = {}

    def arm(mode, steps):
        """steps fractional steps in episodes from rest; device time of the steps only"""
        tot = [0.0, 0.0, 0, 0.0]
        cnt = [0, 0, 0]
        done = 0
        while done < steps:
            m_ = min(a.episode, steps - done)
            mg.apply_bc(mgm.BC_LID)
            ms_, pms_, vc_, err_ = mg.run_steps(mode, m_)
            tot[0] += ms_; tot[1] += pms_; tot[2] += vc_; tot[3] = err_
            for i, v in enumerate(mg.solve_counters()):
                cnt[i] += v
            done += m_
        counts[mode] = cnt
        return tot

    def smoother_pass(steps):
        """CUDA events around every level-0 smoother launch, recorded inside
        the V-cycle graphs of a host-driven pass of the same steps (event
        nodes cannot sit in the step graph's conditional bodies): total ms,
        launches, algorithmic bytes per launch"""
        mg.profile_smoother(True)
        arm(fast, 1)  # captures the V-cycle graphs with their event nodes
        mg.sync()
        s0 = mg.profile_read()
        arm(fast, steps)
        s1 = mg.profile_read()
        mg.profile_smoother(False)
        return s1[0] - s0[0], s1[1] - s0[1], s1[2]

    # warm-up (captures the step graphs), then the plain FP64 arm
    arm(fast, a.warmup)
    arm(mgm.MODE_FP64, min(a.warmup, 2))
    barrier()
    mg.sync()
    plain_ms, plain_pms, plain_vc, _ = arm(mgm.MODE_FP64, a.steps)
    plain_ms = max_over_ranks(plain_ms)

    # headline: FP32-in-FP64 refinement, each step one graph launch (the
    # solve's loops as conditional nodes), device-timed on the library's stream
    barrier()
    mg.sync()
    clocks = ClockSampler(local_rank)
    clocks.start()
    l0 = api.kernel_launches()
    ms, pms, vc, err = arm(fast, a.steps)
    launches = api.kernel_launches() - l0
    ck = clocks.stop()
    barrier()
    ms = max_over_ranks(ms)
    head_counts = list(counts[fast])

    # the same steps with the solve's loops driven from the host (one read of
    # the loop flags per Arnoldi step, V-cycle graphs): what the one-graph step saves
    mg.use_step_graph(False)
    arm(fast, min(a.warmup, 2))
    mg.sync()
    hd_ms, hd_pms, hd_vc, _ = arm(fast, a.steps)
    mg.use_step_graph(True)
    hd_ms = max_over_ranks(hd_ms)

    # the dominant kernel's launches, timed by events (roofline)
    sm_ms, sm_launch, sm_bytes = smoother_pass(a.steps)

    # the same steps with the FP16 operator (D^-1 A) in the FP32 V-cycle
    # (mgm_use_half_operator); reported beside the headline, not as it
    half = None
    if not a.no_half:
        mg.use_half_operator(True)
        arm(fast, min(a.warmup, 2))
        barrier()
        mg.sync()
        half_ms, half_pms, half_vc, half_err = arm(fast, a.steps)
        barrier()
        half_ms = max_over_ranks(half_ms)
        h_ms, h_launch, h_bytes = smoother_pass(min(a.steps, a.episode))
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
    barrier()
    mg.sync()
    e2e_s = 0.0
    done = 0
    while done < a.steps:
        m_ = min(a.episode, a.steps - done)
        mg.apply_bc(mgm.BC_LID)
        bufs[0].array[:] = mg.get_field("u")
        bufs[1].array[:] = mg.get_field("v")
        t0 = time.perf_counter()
        for _ in range(m_):
            mg.step_host(fast, bufs[0].ptr, bufs[1].ptr, bufs[2].ptr, bufs[3].ptr, bufs[4].ptr)
            bufs[0].array, bufs[2].array = bufs[2].array, bufs[0].array
            bufs[0].ptr, bufs[2].ptr = bufs[2].ptr, bufs[0].ptr
            bufs[1].array, bufs[3].array = bufs[3].array, bufs[1].array
            bufs[1].ptr, bufs[3].ptr = bufs[3].ptr, bufs[1].ptr
        e2e_s += time.perf_counter() - t0
        done += m_
    e2e_s = max_over_ranks(e2e_s)
    finite = bool(np.all(np.isfinite(bufs[0].array)))
    for b in bufs:
        b.free()
    learned = None
    if rank == 0 and not a.no_learned:
        learned = learned_arm(a, mg, mgm, n)

    line = None
    if rank == 0:
        steps_total = a.steps * world
        value = steps_total / (ms / 1e3)
        peak, peak_src = measured_peak()
        avg_launch_s = (sm_ms / 1e3) / max(sm_launch, 1)
        achieved = sm_bytes / avg_launch_s / 1e9 if sm_launch else None
        sizes = [tuple(mg.sizes[l][:3]) for l in range(mg.nl)]
        sb = step_bytes(sizes, 2, a.cheb_degree, True, *head_counts, a.steps)
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
                           "poisson_ms": plain_pms / a.steps, "vcycles_per_step": plain_vc / a.steps},
            "host_driven_fp32": {"ms_per_step": hd_ms / a.steps, "poisson_ms": hd_pms / a.steps,
                                 "vcycles_per_step": hd_vc / a.steps,
                                 "note": ("the same steps with the solve's loops driven from the host (one read of "
                                          "the loop flags per Arnoldi step, each V-cycle a graph replay); the "
                                          "headline runs each step as one graph launch")},
            "learned_warm_start": learned,
            "half_operator": half,
            "headline_arm": ("FP32 V-cycle inside FP64 FGMRES without the learned warm start (the faster arm: "
                             "the measured learned arm is in learned_warm_start)"),
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
            cb["variants"] = {"reference_gcc_O2_1core": cb["value"],
                              "reference_gcc_O0_1core": cpu_baseline_entry(a, s0, n)["value"],
                              "note": ("the reference's OpenACC builds (nvc -acc multicore / GPU) are unavailable on "
                                       "this box (no nvc); its C code is serial")}
            line["cpu_baseline"] = cb
    mg.close()
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
    f = clouds.gaussian_fields(c0, nrhs, seed=5)
    inner = lev["btag"] == 0
    f[:, ~inner] = 0.0
    f[:, inner] -= f[:, inner].mean(1, keepdims=True)
    f[:, 0] = 0.0
    b.set_solver(a.tol, 24, 4, 10.0)
    arms = {}
    for name, mode in (("fp32", mgm.MODE_FP32_IR), ("fp64", mgm.MODE_FP64)):
        b.solve(f, mode)  # warm-up (allocates the Krylov space)
        dev, wall, vcs, worst = 0.0, 0.0, 0, 0.0
        reps = max(1, min(a.steps, 3))
        for _ in range(reps):
            t1 = time.perf_counter()
            sol, vc, rr, ms = b.solve(f, mode)
            wall += time.perf_counter() - t1
            dev += ms
            vcs += vc
            worst = max(worst, float(rr.max()))
        arms[name] = {"ms_per_solve": dev / reps, "wall_ms_per_solve": wall * 1e3 / reps, "vcycles": vcs / reps,
                      "worst_rel_res": worst, "sol": sol}
    rel = max(float(np.linalg.norm(x - y) / np.linalg.norm(y)) for x, y in zip(arms["fp32"]["sol"], arms["fp64"]["sol"]))
    for v in arms.values():
        v.pop("sol")
    n_tot = sum(c.n for c in cl)
    b.close()
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
        "weights": {k_: v for k_, v in rep.items()},
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
    s = reference_full(a, steps=max(a.steps, 1), warmup=a.warmup)
    val = 1.0 / s["sec_per_step"]
    cfg = workload(a)
    cfg["reference_solver"] = ("the reference's own multigrid_Poisson_solver: a fixed 10 V-cycles of 3 SOR sweeps "
                               "(omega 1.0) per step; it has no tolerance test and never reaches 1e-8")
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
