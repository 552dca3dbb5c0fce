"""ctypes front-end of the CPU checkers (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
legs import this module.  It loads
  * oracle/liboracle.so   -- the project's restatement of the reference hot path
                            (mgm_oracle.c), and
  * oracle/_ref/libref.so -- the reference's own C code compiled from its
                            sources (ref_shim.c), when it has been built.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_ORC = {}
_REF = {}

dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
ip = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


# orc_read_gmsh / ref_read_mesh: path, dim, cap, x, y, z, nx, ny, nz, btag, corner, &nb, &num_elem, &d_avg
_MESH_ARGS = [C.c_char_p, C.c_int, C.c_int] + [C.c_void_p] * 8 + [C.POINTER(C.c_int), C.POINTER(C.c_int),
                                                                   C.POINTER(C.c_double)]


def read_mesh(path, dim, reference=False):
    """read_PointStructure (mesh_functions.h:172-476) on a Gmsh file, by the
    restatement (orc_read_gmsh) or, with reference=True, by the reference's
    own reader (_ref/libref.so; the path must be shorter than 50 characters).
    Returns a dict of the level's arrays and counts."""
    fn = ref_lib().ref_read_mesh if reference else lib().orc_read_gmsh
    nb, ne, da = C.c_int(), C.c_int(), C.c_double()
    nulls = [None] * 8
    n = fn(str(path).encode(), dim, 0, *nulls, C.byref(nb), C.byref(ne), C.byref(da))
    if n < 0:
        raise RuntimeError(f"cannot read {path}")
    out = {nm: np.zeros(n) for nm in ("x", "y", "z", "nx", "ny", "nz")}
    out["btag"] = np.zeros(n, np.uint8)
    out["corner"] = np.zeros(n, np.uint8)
    arrs = [out[k].ctypes.data_as(C.c_void_p) for k in ("x", "y", "z", "nx", "ny", "nz", "btag", "corner")]
    n2 = fn(str(path).encode(), dim, n, *arrs, C.byref(nb), C.byref(ne), C.byref(da))
    assert n2 == n
    out.update(n=n, nb=nb.value, num_elem=ne.value, d_avg=da.value)
    return out


def lib(crpow: bool = False):
    """liboracle.so (libm pow, as the reference) or liboracle_crpow.so
    (correctly rounded powers, as the CUDA path)."""
    key = "crpow" if crpow else "libm"
    if key not in _ORC:
        path = os.path.join(HERE, "liboracle_crpow.so" if crpow else "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run `make -C oracle`")
        L = C.CDLL(path)
        L.orc_knn_cloud.argtypes = [C.c_int, C.c_int, dp, dp, dp, u8p, C.c_int, C.c_int, ip]
        L.orc_cs_new.argtypes = [C.c_int]
        L.orc_cs_new.restype = C.c_void_p
        L.orc_cs_free.argtypes = [C.c_void_p]
        L.orc_cs_level.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, ip, dp, u8p, C.c_int, C.c_void_p,
                                   C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.orc_cs_prepare.argtypes = [C.c_void_p]
        L.orc_cs_solve.argtypes = [C.c_void_p, dp, dp, C.c_double, C.c_int, C.c_int, C.c_double,
                                   C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.orc_cs_solve.restype = C.c_int
        L.orc_count_ties.argtypes = [C.c_int, C.c_int, dp, dp, dp, C.c_int, ip]
        L.orc_count_ties.restype = C.c_long
        L.orc_nearest.argtypes = [C.c_int, dp, dp, dp, C.c_int, dp, dp, dp, C.c_int, ip]
        L.orc_bfs_order.argtypes = [C.c_int, C.c_int, ip, ip]
        L.orc_bfs_order.restype = C.c_int
        L.orc_apply_order.argtypes = [C.c_int, C.c_int, ip, dp, dp, dp, dp, dp, dp, u8p, ip]
        L.orc_correct_normals.argtypes = [C.c_int, C.c_int, dp, dp, dp, u8p, ip, dp, dp, dp]
        L.orc_avg_dx.argtypes = [C.c_int, C.c_int, C.c_int, dp, dp, dp, u8p, ip]
        L.orc_avg_dx.restype = C.c_double
        L.orc_dt.argtypes = [C.c_double, C.c_double, C.c_double]
        L.orc_dt.restype = C.c_double
        L.orc_derivative_weights.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, dp, dp, dp, dp, dp, dp,
                                             u8p, ip, dp, dp, dp, dp, dp]
        L.orc_transfer_weights.argtypes = [C.c_int, dp, dp, dp, u8p, ip, C.c_int, C.c_int,
                                           C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, dp, dp, dp, ip, dp]
        L.orc_spmv.argtypes = [C.c_int, C.c_int, dp, ip, dp, dp]
        L.orc_ctx_new.restype = C.c_void_p
        L.orc_ctx_new.argtypes = [C.c_int, C.c_int]
        L.orc_ctx_free.argtypes = [C.c_void_p]
        L.orc_ctx_level.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, ip, u8p, dp, dp, dp, dp, dp, dp, dp, dp,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, dp, dp, dp]
        L.orc_ctx_fields.argtypes = [C.c_void_p] + [dp] * 13
        L.orc_ctx_params.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_float, C.c_int, C.c_int, C.c_int]
        L.orc_multigrid.argtypes = [C.c_void_p]
        L.orc_relaxation.argtypes = [C.c_void_p, C.c_int]
        L.orc_step.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.orc_step.restype = C.c_double
        for nm in ("orc_intermediate_velocity", "orc_mass_residual"):
            getattr(L, nm).argtypes = [C.c_void_p]
        L.orc_update_velocity.argtypes = [C.c_void_p]
        L.orc_update_velocity.restype = C.c_double
        L.orc_ctx_timple.argtypes = [C.c_void_p, dp, C.c_int, C.c_int, C.c_double, C.c_double]
        L.orc_timple_step.argtypes = [C.c_void_p]
        L.orc_timple_step.restype = C.c_double
        for nm in ("orc_timple_momentum", "orc_timple_mass", "orc_timple_multigrid", "orc_timple_update_velocity",
                   "orc_timple_boundary_pressure"):
            getattr(L, nm).argtypes = [C.c_void_p]
        L.orc_read_gmsh.argtypes = _MESH_ARGS
        L.orc_read_gmsh.restype = C.c_int
        L.orc_ctx_coords.argtypes = [C.c_void_p, C.c_int, dp, dp, dp]
        L.orc_gauss_jordan.argtypes = [C.c_int, dp, dp]
        for nm in ("orc_heat_init", "orc_heat_boundary_rhs", "orc_heat_step"):
            getattr(L, nm).argtypes = [C.c_void_p, C.c_int]
        L.orc_heat_step.restype = C.c_double
        _ORC[key] = L
    return _ORC[key]


def _ref_name(timple, heat, opt="O2"):
    if opt == "O0":
        return "libref_O0.so"
    return "libref_heat.so" if heat else ("libref_timple.so" if timple else "libref.so")


def ref_available(timple: bool = False, heat: bool = False, opt: str = "O2") -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", _ref_name(timple, heat, opt)))


def ref_lib(timple: bool = False, heat: bool = False, opt: str = "O2"):
    """_ref/libref.so (fractional-step build), _ref/libref_timple.so (the
    reference's TIMPLE solver) or _ref/libref_heat.so (the heat-conduction
    program's routines); each is its own library with its own globals.
    opt="O0": _ref/libref_O0.so, the fractional-step build compiled without
    optimisation, as the reference's README compiles it."""
    key = "heat" if heat else ("timple" if timple else "fs")
    if opt == "O0":
        key = "fs_O0"
    if key not in _REF:
        path = os.path.join(HERE, "_ref", _ref_name(timple, heat, opt))
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run `make -C oracle ref REF=<reference tree>` where the reference tree exists")
        L = C.CDLL(path)
        L.ref_begin.argtypes = [C.c_int, C.c_int, C.c_int]
        L.ref_set_flow.argtypes = [C.c_double, C.c_double, C.c_float, C.c_int, C.c_int]
        L.ref_set_level.argtypes = [C.c_int, C.c_int, C.c_int, dp, dp, dp, dp, dp, dp, u8p, C.c_int, C.c_int, C.c_double]
        for nm in ("ref_clouds", "ref_rcm", "ref_normals", "ref_derivatives", "ref_relaxation", "ref_residuals",
                   "ref_restrict", "ref_prolongate"):
            getattr(L, nm).argtypes = [C.c_int]
        L.ref_avg_dx.argtypes = [C.c_int]
        L.ref_avg_dx.restype = C.c_double
        L.ref_set_davg.argtypes = [C.c_int, C.c_double]
        L.ref_num_poly_terms.argtypes = [C.c_int]
        L.ref_get_geometry.argtypes = [C.c_int, dp, dp, dp, dp, dp, dp, u8p, ip]
        L.ref_get_ops.argtypes = [C.c_int, dp, dp, dp, dp, dp]
        L.ref_get_transfer.argtypes = [C.c_int, ip, ip, C.c_void_p, C.c_void_p]
        L.ref_load_ops.argtypes = [C.c_int, ip, dp, dp, C.c_void_p, dp, dp]
        L.ref_load_transfer.argtypes = [C.c_int, ip, ip, C.c_void_p, C.c_void_p]
        if not heat:
            L.ref_bc.argtypes = [C.c_int]
        L.ref_dt.restype = C.c_double
        L.ref_set_dt.argtypes = [C.c_double]
        L.ref_field_get.argtypes = [C.c_int, C.c_int, dp]
        L.ref_field_set.argtypes = [C.c_int, C.c_int, dp]
        L.ref_spmv.argtypes = [C.c_int, C.c_int, dp, dp]
        L.ref_gauss_jordan.argtypes = [C.c_int, dp, dp]
        L.ref_read_mesh.argtypes = _MESH_ARGS
        L.ref_read_mesh.restype = C.c_int
        if heat:
            L.ref_heat_init.argtypes = [C.c_int]
            L.ref_heat_step.argtypes = [C.c_int]
            L.ref_heat_step.restype = C.c_double
        elif timple:
            L.ref_timple_params.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double]
            L.ref_timple_step.restype = C.c_double
        else:
            L.ref_step.restype = C.c_double
        _REF[key] = L
    return _REF[key]


# field ids of ref_shim.c:field_ptr
FIELD = {"u": 0, "v": 1, "w": 2, "p": 3, "u_new": 4, "v_new": 5, "w_new": 6, "u_old": 7, "v_old": 8,
         "w_old": 9, "res": 10, "source": 11, "dpdn": 12, "dpdx": 13, "dpdy": 14, "dpdz": 15, "p_old": 16,
         "pprime": 17}


@dataclass
class Level:
    """One level after the reference's set-up pipeline (arrays row-major [n][k])."""
    n: int
    nb: int
    k: int
    dim: int
    poly: int
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    nx: np.ndarray
    ny: np.ndarray
    nz: np.ndarray
    btag: np.ndarray
    cloud: np.ndarray
    d_avg: float = 0.0
    Dx: np.ndarray | None = None
    Dy: np.ndarray | None = None
    Dz: np.ndarray | None = None
    lap: np.ndarray | None = None
    lapP: np.ndarray | None = None
    rpts: np.ndarray | None = None
    ppts: np.ndarray | None = None
    restr: np.ndarray | None = None   # [n][k of finer level]
    prol: np.ndarray | None = None    # [n][k of coarser level]


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def ref_pipeline(clouds, ks, polys, phs=3, with_weights=True, search_scale=0.3, timple=False, heat=False, opt="O2"):
    """Runs read_complete_mesh_data's steps (minus the file reader) and
    create_derivative_matrices through the reference's own code (in the
    TIMPLE or heat-conduction build when asked)."""
    R = ref_lib(timple, heat, opt)
    nl = len(clouds)
    dim = clouds[0].dim
    R.ref_begin(dim, phs, nl)
    for l, c in enumerate(clouds):
        R.ref_set_level(l, c.n, c.nb, _f64(c.x), _f64(c.y), _f64(c.z), _f64(c.nx), _f64(c.ny), _f64(c.nz),
                        np.ascontiguousarray(c.btag, np.uint8), polys[l], ks[l], search_scale * c.h)
        R.ref_clouds(l)
        R.ref_rcm(l)
        R.ref_normals(l)
        R.ref_avg_dx(l)
    out = []
    for l, c in enumerate(clouds):
        n, k = c.n, ks[l]
        a = {nm: np.zeros(n) for nm in ("x", "y", "z", "nx", "ny", "nz")}
        bt = np.zeros(n, np.uint8)
        cl = np.zeros(n * k, np.int32)
        R.ref_get_geometry(l, a["x"], a["y"], a["z"], a["nx"], a["ny"], a["nz"], bt, cl)
        d_avg = R.ref_avg_dx(l)
        out.append(Level(n, c.nb, k, dim, polys[l], a["x"], a["y"], a["z"], a["nx"], a["ny"], a["nz"], bt,
                         cl.reshape(n, k), d_avg))
    if with_weights:
        R.ref_rp()
        for l in range(nl):
            R.ref_derivatives(l)
        for l, L in enumerate(out):
            n, k = L.n, L.k
            ops = [np.zeros(n * k) for _ in range(5)]
            R.ref_get_ops(l, *ops)
            L.Dx, L.Dy, L.Dz, L.lap, L.lapP = [o.reshape(n, k) for o in ops]
            if dim != 3:
                L.Dz = None
            rp = np.zeros(n, np.int32); pp = np.zeros(n, np.int32)
            restr = np.zeros(n * out[l - 1].k) if l > 0 else None
            prol = np.zeros(n * out[l + 1].k) if l < nl - 1 else None
            R.ref_get_transfer(l, rp, pp,
                               restr.ctypes.data if restr is not None else None,
                               prol.ctypes.data if prol is not None else None)
            L.rpts, L.ppts = rp, pp
            L.restr = restr.reshape(n, out[l - 1].k) if restr is not None else None
            L.prol = prol.reshape(n, out[l + 1].k) if prol is not None else None
    return out


def ref_load_levels(levels, phs=3, timple=False):
    """Hands levels set up elsewhere (geometry after the reorder, clouds,
    operators, transfer points and weights -- e.g. orc_pipeline's, which are
    pinned bit for bit to the reference's own set-up) to the reference's
    structures, so that its own step routines run on them without repeating
    the set-up.  Returns the reference library handle."""
    R = ref_lib(timple)
    nl = len(levels)
    dim = levels[0].dim
    R.ref_begin(dim, phs, nl)
    for l, L in enumerate(levels):
        R.ref_set_level(l, L.n, L.nb, _f64(L.x), _f64(L.y), _f64(L.z), _f64(L.nx), _f64(L.ny), _f64(L.nz),
                        np.ascontiguousarray(L.btag, np.uint8), L.poly, L.k, L.d_avg)
    for l, L in enumerate(levels):
        dz = _f64(L.Dz.ravel()) if L.Dz is not None else None
        R.ref_load_ops(l, np.ascontiguousarray(L.cloud.ravel(), np.int32), _f64(L.Dx.ravel()), _f64(L.Dy.ravel()),
                       dz.ctypes.data if dz is not None else None, _f64(L.lap.ravel()), _f64(L.lapP.ravel()))
        restr = _f64(L.restr.ravel()) if l > 0 else None
        prol = _f64(L.prol.ravel()) if l < nl - 1 else None
        R.ref_load_transfer(l, np.ascontiguousarray(L.rpts, np.int32), np.ascontiguousarray(L.ppts, np.int32),
                            restr.ctypes.data if restr is not None else None,
                            prol.ctypes.data if prol is not None else None)
    return R


def orc_level_setup(c, k, crpow=False):
    """kNN -> breadth-first reorder -> normals -> d_avg on one cloud (restatement)."""
    O = lib(crpow)
    n = c.n
    x, y, z = _f64(c.x).copy(), _f64(c.y).copy(), _f64(c.z).copy()
    nx, ny, nz = _f64(c.nx).copy(), _f64(c.ny).copy(), _f64(c.nz).copy()
    bt = np.ascontiguousarray(c.btag, np.uint8).copy()
    cl = np.zeros(n * k, np.int32)
    O.orc_knn_cloud(n, c.nb, x, y, z, bt, k, c.dim, cl)
    q1 = np.zeros(n, np.int32)
    cnt = O.orc_bfs_order(n, k, cl, q1)
    if cnt != n:
        raise RuntimeError(f"stencil graph disconnected: reached {cnt} of {n} nodes")
    O.orc_apply_order(n, k, q1, x, y, z, nx, ny, nz, bt, cl)
    O.orc_correct_normals(n, k, x, y, z, bt, cl, nx, ny, nz)
    d_avg = O.orc_avg_dx(n, k, c.dim, x, y, z, bt, cl)
    return dict(x=x, y=y, z=z, nx=nx, ny=ny, nz=nz, btag=bt, cloud=cl.reshape(n, k), d_avg=d_avg, queue1=q1)


def orc_pipeline(clouds, ks, polys, phs=3, with_weights=True, reference_rows=True, crpow=False):
    """The restatement of ref_pipeline.  reference_rows=False builds the
    transfer weights for every non-boundary row (convergent-solver variant)."""
    O = lib(crpow)
    dim = clouds[0].dim
    nl = len(clouds)
    out = []
    for l, c in enumerate(clouds):
        s = orc_level_setup(c, ks[l], crpow)
        out.append(Level(c.n, c.nb, ks[l], dim, polys[l], s["x"], s["y"], s["z"], s["nx"], s["ny"], s["nz"],
                         s["btag"], s["cloud"], s["d_avg"]))
    # create_prolongation_and_restriction_matrices (mesh_functions.h:874-893)
    for l, L in enumerate(out):
        nxt = out[l + 1] if l < nl - 1 else L
        prv = out[l - 1] if l > 0 else L
        L.ppts = np.zeros(L.n, np.int32)
        O.orc_nearest(L.n, L.x, L.y, L.z, nxt.n, nxt.x, nxt.y, nxt.z, dim, L.ppts)
        L.rpts = np.zeros(L.n, np.int32)
        O.orc_nearest(L.n, L.x, L.y, L.z, prv.n, prv.x, prv.y, prv.z, dim, L.rpts)
    if not with_weights:
        return out
    for l, L in enumerate(out):
        if l < nl - 1:
            C_ = out[l + 1]
            W = np.zeros(L.n * C_.k)
            O.orc_transfer_weights(L.n, L.x, L.y, L.z, L.btag, L.ppts, L.nb, 0 if reference_rows else 1,
                                   C_.n, C_.k, dim, phs, C_.poly, C_.x, C_.y, C_.z,
                                   np.ascontiguousarray(C_.cloud.ravel()), W)
            L.prol = W.reshape(L.n, C_.k)
        if l > 0:
            F = out[l - 1]
            W = np.zeros(L.n * F.k)
            O.orc_transfer_weights(L.n, L.x, L.y, L.z, L.btag, L.rpts, L.nb, 0 if reference_rows else 1,
                                   F.n, F.k, dim, phs, F.poly, F.x, F.y, F.z,
                                   np.ascontiguousarray(F.cloud.ravel()), W)
            L.restr = W.reshape(L.n, F.k)
        n, k = L.n, L.k
        ops = [np.zeros(n * k) for _ in range(5)]
        O.orc_derivative_weights(n, k, dim, phs, L.poly, L.x, L.y, L.z, L.nx, L.ny, L.nz, L.btag,
                                 np.ascontiguousarray(L.cloud.ravel()), *ops)
        L.Dx, L.Dy, L.Dz, L.lap, L.lapP = [o.reshape(n, k) for o in ops]
        if dim != 3:
            L.Dz = None
    return out


class OracleSolver:
    """Reference-semantics fractional step on restated levels (mgm_oracle.c)."""

    def __init__(self, levels, Re, courant, omega, num_relax, num_vcycles, jacobi=True, dt=None):
        O = lib()
        self.O = O
        self.levels = levels
        L0 = levels[0]
        self.h = O.orc_ctx_new(len(levels), L0.dim)
        self.keep = []
        self.p, self.source, self.res = [], [], []
        for l, L in enumerate(levels):
            p = np.zeros(L.n); s = np.zeros(L.n); r = np.zeros(L.n)
            self.p.append(p); self.source.append(s); self.res.append(r)
            Dz = L.Dz if L.Dz is not None else np.zeros((L.n, L.k))
            arrs = [np.ascontiguousarray(L.cloud.ravel(), np.int32), L.btag, L.nx, L.ny, L.nz,
                    np.ascontiguousarray(L.Dx.ravel()), np.ascontiguousarray(L.Dy.ravel()),
                    np.ascontiguousarray(Dz.ravel()), np.ascontiguousarray(L.lap.ravel()),
                    np.ascontiguousarray(L.lapP.ravel())]
            rp = np.ascontiguousarray(L.rpts, np.int32)
            pp = np.ascontiguousarray(L.ppts, np.int32)
            restr = np.ascontiguousarray(L.restr.ravel()) if L.restr is not None else None
            prol = np.ascontiguousarray(L.prol.ravel()) if L.prol is not None else None
            self.keep += arrs + [rp, pp, restr, prol]
            O.orc_ctx_level(self.h, l, L.n, L.k, *arrs, rp.ctypes.data, pp.ctypes.data,
                            restr.ctypes.data if restr is not None else None,
                            prol.ctypes.data if prol is not None else None, p, s, r)
        n = L0.n
        self.f = {nm: np.zeros(n) for nm in ("u", "v", "w", "u_new", "v_new", "w_new", "u_old", "v_old", "w_old",
                                             "dpdn", "dpdx", "dpdy", "dpdz")}
        O.orc_ctx_fields(self.h, *[self.f[nm] for nm in ("u", "v", "w", "u_new", "v_new", "w_new", "u_old",
                                                         "v_old", "w_old", "dpdn", "dpdx", "dpdy", "dpdz")])
        if dt is None:
            dt = O.orc_dt(L0.d_avg, Re, courant)
        self.dt = dt
        O.orc_ctx_params(self.h, dt, Re, omega, num_relax, num_vcycles, 1 if jacobi else 0)

    def step(self):
        mr = C.c_double(0)
        e = self.O.orc_step(self.h, C.byref(mr))
        return e, mr.value

    def multigrid(self):
        self.O.orc_multigrid(self.h)

    def __del__(self):
        try:
            self.O.orc_ctx_free(self.h)
        except Exception:
            pass


class TimpleSolver(OracleSolver):
    """Reference-semantics TIMPLE step (time_implicit_solver, timple_solver.h:40-70)
    on restated levels: self.p[l] is pprime of level l, self.p_old the pressure."""

    def __init__(self, levels, Re, courant, omega, num_relax, num_vcycles, iter_timple, iter_momentum, facRe, facdt,
                 jacobi=True, dt=None):
        super().__init__(levels, Re, courant, omega, num_relax, num_vcycles, jacobi=jacobi, dt=dt)
        self.p_old = np.zeros(levels[0].n)
        self.O.orc_ctx_timple(self.h, self.p_old, iter_timple, iter_momentum, facRe, facdt)

    def step(self):
        return self.O.orc_timple_step(self.h)


class HeatSolver(OracleSolver):
    """The heat-conduction program (mg_heat_conduction.c:43-83 with
    heat_conduction.h:24-113, init/init_heat_conduction.c:14-67) on restated
    levels: self.p[l], self.source[l] as the program leaves them; level 0's
    lap_Poison is a private copy (set_boundary_rhs turns its x == 0 boundary
    rows into Dirichlet rows)."""

    def __init__(self, levels, omega, num_relax, num_vcycles, wave=1, jacobi=True):
        import dataclasses
        lv = list(levels)
        lv[0] = dataclasses.replace(levels[0], lapP=np.array(levels[0].lapP, dtype=np.float64, copy=True))
        super().__init__(lv, 100.0, 0.5, omega, num_relax, num_vcycles, jacobi=jacobi, dt=1.0)
        self.wave = wave
        for l, L in enumerate(lv):
            xyz = [np.ascontiguousarray(a, np.float64) for a in (L.x, L.y, L.z)]
            self.keep += xyz
            self.O.orc_ctx_coords(self.h, l, *xyz)
        self.lapP0 = self.keep[9]    # level 0's lap_Poison as the context holds it
        self.O.orc_heat_init(self.h, wave)

    def boundary_rhs(self):
        self.O.orc_heat_boundary_rhs(self.h, self.wave)

    def step(self):
        return self.O.orc_heat_step(self.h, self.wave)


def phs_system(n_pts, poly, seed=0, phs=3, dim=2):
    """A PHS + polynomial saddle-point matrix (create_A_matrix_from_cloud_indices,
    rbf.h:42-77) of a seeded point cloud, row-major, for the dense-inverse tests."""
    rng = np.random.default_rng(seed)
    p = rng.uniform(-1, 1, (n_pts, dim)) * 0.05
    p[0] = 0.0
    ex = [(i, j) for i in range(poly + 1) for j in range(poly + 1 - i)]
    N = n_pts + len(ex)
    A = np.zeros((N, N))
    r = np.sqrt(((p[:, None, :] - p[None, :, :]) ** 2).sum(-1))
    A[:n_pts, :n_pts] = r ** phs
    for t, (a, b) in enumerate(ex):
        v = (p[:, 0] - p[0, 0]) ** a * (p[:, 1] - p[0, 1]) ** b
        A[:n_pts, n_pts + t] = v
        A[n_pts + t, :n_pts] = v
    return A


def lid_bc(L, f):
    """init_LDC.c:16-44 on level 0: u = 1 where |y - 1| < 1e-9."""
    f["u"][:] = 0; f["v"][:] = 0; f["w"][:] = 0
    top = np.abs(L.y - 1.0) < 1e-9
    f["u"][top] = 1.0


def tc_bc(L, f):
    """init_TC.c:17-54 on level 0: inner wall r = 0.5 rotating, u = -y/r, v = x/r."""
    for nm in ("u", "v", "w", "u_new", "v_new", "w_new"):
        f[nm][:] = 0
    r = np.sqrt(L.x * L.x + L.y * L.y)
    inner = np.abs(r - 0.5) < 1e-9
    f["u"][inner] = -L.y[inner] / r[inner]
    f["v"][inner] = L.x[inner] / r[inner]
    f["u_new"][inner] = f["u"][inner]
    f["v_new"][inner] = f["v"][inner]


def pinned_operator(lapP, cloud):
    """lap_Poison as a scipy CSR matrix with row 0 replaced by p[0] = 0 -- the
    system the reference's multigrid aims at (it re-pins p to node 0 after every
    sweep, fractional_step_solver.h:180-183)."""
    import scipy.sparse as sp
    n, k = lapP.shape
    A = sp.csr_matrix((np.ascontiguousarray(lapP.ravel()).copy(), np.ascontiguousarray(cloud.ravel()).astype(np.int64),
                       np.arange(0, n * k + 1, k)), shape=(n, n))
    A = A.tolil()
    A[0, :] = 0
    A[0, 0] = 1.0
    return A.tocsr()


def pinned_poisson_direct(lapP, cloud, b):
    """FP64 direct solve of the pinned system (the converged answer every
    iterative mode is compared with).  b[0] is taken as 0."""
    import scipy.sparse.linalg as spla
    A = pinned_operator(lapP, cloud)
    bb = np.array(b, dtype=np.float64)
    bb[0] = 0.0
    return spla.spsolve(A.tocsc(), bb)


def solver_transfer(levels, crpow=False, phs=3):
    """The convergent solver's transfer weights on restated levels (set as
    L.s_restr / L.s_prol): restriction into level l from l-1 with
    create_restriction_matrix's interpolation on every non-boundary row,
    prolongation into l from l+1 with create_prolongation_matrix's on every
    row (mesh_functions.h:533-670)."""
    O = lib(crpow)
    nl = len(levels)
    for l, L in enumerate(levels):
        dim = L.dim
        L.s_restr = L.s_prol = None
        if l > 0:
            F = levels[l - 1]
            W = np.zeros(L.n * F.k)
            O.orc_transfer_weights(L.n, L.x, L.y, L.z, L.btag, L.rpts, 0, 1, F.n, F.k, dim, phs, F.poly, F.x, F.y,
                                   F.z, np.ascontiguousarray(F.cloud.ravel()), W)
            L.s_restr = W.reshape(L.n, F.k)
        if l < nl - 1:
            Cn = levels[l + 1]
            W = np.zeros(L.n * Cn.k)
            O.orc_transfer_weights(L.n, L.x, L.y, L.z, L.btag, L.ppts, 0, 0, Cn.n, Cn.k, dim, phs, Cn.poly, Cn.x,
                                   Cn.y, Cn.z, np.ascontiguousarray(Cn.cloud.ravel()), W)
            L.s_prol = W.reshape(L.n, Cn.k)
    return levels


class ConvergentSolver:
    """The library's convergent FP64 Poisson solve restated on the CPU
    (oracle/fgmres_oracle.c, OpenMP): FGMRES preconditioned by a V-cycle of
    Chebyshev smoothing, exact boundary rows, RBF restriction/prolongation and
    a dense coarsest inverse.  levels need cloud, lapP, btag, rpts, ppts and
    s_restr / s_prol (solver_transfer)."""

    def __init__(self, levels, crpow=False):
        self.O = lib(crpow)
        self.h = self.O.orc_cs_new(len(levels))
        self.keep = []
        nl = len(levels)
        for l, L in enumerate(levels):
            cl = np.ascontiguousarray(L.cloud, np.int32)
            lp = np.ascontiguousarray(L.lapP, np.float64)
            bt = np.ascontiguousarray(L.btag, np.uint8)
            rp = np.ascontiguousarray(L.rpts, np.int32)
            pp = np.ascontiguousarray(L.ppts, np.int32)
            rw = np.ascontiguousarray(L.s_restr, np.float64) if l > 0 else None
            pw = np.ascontiguousarray(L.s_prol, np.float64) if l < nl - 1 else None
            self.keep += [cl, lp, bt, rp, pp, rw, pw]
            kr = levels[l - 1].k if l > 0 else 0
            kp = levels[l + 1].k if l < nl - 1 else 0
            self.O.orc_cs_level(self.h, l, L.n, L.k, cl, lp, bt, kr, rp.ctypes.data,
                                rw.ctypes.data if rw is not None else None, kp, pp.ctypes.data,
                                pw.ctypes.data if pw is not None else None)
        self.O.orc_cs_prepare(self.h)

    def solve(self, b, p0=None, tol=1e-8, max_iters=100, cheb_degree=3, cheb_ratio=20.0):
        """(p, V-cycles, relative residual, converged) of the pinned system (b[0] taken as 0)."""
        p = np.zeros(len(b)) if p0 is None else np.array(p0, np.float64)
        it, rr = C.c_int(), C.c_double()
        st = self.O.orc_cs_solve(self.h, np.ascontiguousarray(b, np.float64), p, tol, max_iters, cheb_degree,
                                 cheb_ratio, C.byref(it), C.byref(rr))
        return p, it.value, rr.value, st == 0

    def __del__(self):
        try:
            self.O.orc_cs_free(self.h)
        except Exception:
            pass


def pinned_lu(lapP, cloud):
    """One sparse LU factorisation of the pinned system (SuperLU, minimum
    degree on A^T + A), for many right-hand sides: returns solve(b) with b[0]
    taken as 0.  The FP64 direct answer of every converged solve, at sizes
    (~250k nodes) where refactoring per right-hand side would be too slow."""
    import scipy.sparse.linalg as spla
    lu = spla.splu(pinned_operator(lapP, cloud).tocsc(), permc_spec="MMD_AT_PLUS_A")

    def solve(b):
        bb = np.array(b, dtype=np.float64)
        bb[0] = 0.0
        return lu.solve(bb)
    return solve


def compatible_pinned_direct(lapP, cloud, btag, b):
    """FP64 direct solve of lap_Poison p = b - alpha w, pinned p[0] = 0, where
    w is 1 on interior rows and alpha = z.b / z.w with z the left null vector
    of the singular lap_Poison (z = A_pinned^-T (e_0 - row 0 of lap_Poison)):
    the answer of the solve modes with compatible right-hand sides."""
    import scipy.sparse.linalg as spla
    n = lapP.shape[0]
    lu = spla.splu(pinned_operator(lapP, cloud).tocsc())
    row0 = np.zeros(n)
    np.add.at(row0, np.asarray(cloud[0], np.int64), lapP[0])
    e0 = np.zeros(n)
    e0[0] = 1.0
    z = lu.solve(e0 - row0, trans="T")
    w = (np.asarray(btag) == 0).astype(np.float64)
    bb = np.array(b, dtype=np.float64) - (z @ b) / (z @ w) * w
    bb[0] = 0.0
    return lu.solve(bb)


def rel_residual(lapP, cloud, b, p):
    A = pinned_operator(lapP, cloud)
    bb = np.array(b, dtype=np.float64)
    bb[0] = 0.0
    r = bb - A @ p
    return float(np.linalg.norm(r) / np.linalg.norm(bb))


def levels_from_device(mg):
    """Oracle Level objects holding the operators a device hierarchy built
    (so the restated step runs on bit-identical weights)."""
    out = []
    for l in range(mg.nl):
        g = mg.geometry(l)
        ops = mg.operators(l)
        tr = mg.transfer(l)
        n, nb, k, _ = mg.sizes[l]
        L = Level(n, nb, k, mg.dim, 0, g["x"], g["y"], g["z"], g["nx"], g["ny"], g["nz"], g["btag"], g["cloud"],
                  g["d_avg"], ops["Dx"], ops["Dy"], ops.get("Dz"), ops["lap"], ops["lapP"], tr["rpts"], tr["ppts"],
                  tr["restr"], tr["prol"])
        out.append(L)
    return out
