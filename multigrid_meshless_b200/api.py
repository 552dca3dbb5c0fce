"""Python mirror of the reference's call surface, on top of the C ABI.

Function names follow the reference (Multigrid_meshless header_files/*.h):

  find_cloud_index            kdtree_functions.h:113-151   -> knn_cloud()
  find_nearest_point          kdtree_functions.h:153-175   -> nearest_points()
  rcm_reordering_with_boundarynodes  mesh_functions.h:774-872 -> bfs_order(), apply_order()
  correct_normal_directions   mesh_functions.h:478-527     -> correct_normals()
  calculate_avg_dx            mesh_functions.h:895-910     -> avg_dx()
  create_derivative_matrices  rbf.h:401-421                -> derivative_weights()
  create_{restriction,prolongation}_matrix  mesh_functions.h:533-670 -> transfer_weights()
  multiply_sparse_matrix_vector_gpu  mat_lib.h:80-89       -> spmv()
  read_PointStructure         mesh_functions.h:172-476     -> read_gmsh()
  matrixInverse_Gauss_Jordan  mat_lib.h:423-491            -> gauss_jordan()
  create_laplacian_for_Poisson  rbf.h:382-399              -> laplacian_for_poisson()
  relaxation / calculate_residuals / restrict_residuals / prolongate_corrections
                              fractional_step_solver.h:168-246 -> Multigrid.ref_routine()
  fractional_step_explicit    fractional_step_solver.h:47-71 -> Multigrid.step()

Arrays at this boundary use the reference's layout: node vectors of length n
and stencil rows [n][k].  Every call runs on the GPU through libmgm.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, load, ptr


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _u8(a):
    return np.ascontiguousarray(a, dtype=np.uint8)


def knn_cloud(x, y, z, btag, nb, k, dim):
    L = load()
    n = len(x)
    out = np.zeros((n, k), np.int32)
    check(L.mgm_knn_cloud(n, nb, dim, _f(x), _f(y), _f(z), _u8(btag), k, out))
    return out


def nearest_points(x1, y1, z1, x2, y2, z2, dim):
    L = load()
    out = np.zeros(len(x1), np.int32)
    check(L.mgm_nearest_points(len(x1), _f(x1), _f(y1), _f(z1), len(x2), _f(x2), _f(y2), _f(z2), dim, out))
    return out


def bfs_order(cloud):
    L = load()
    cloud = _i(cloud)
    n, k = cloud.shape
    q = np.zeros(n, np.int32)
    check(L.mgm_bfs_order(n, k, cloud, q))
    return q


def apply_order(queue1, x, y, z, nx, ny, nz, btag, cloud):
    """Returns permuted copies (x, y, z, nx, ny, nz, btag, cloud)."""
    L = load()
    arrs = [_f(a).copy() for a in (x, y, z, nx, ny, nz)]
    bt = _u8(btag).copy()
    cl = _i(cloud).copy()
    n, k = cl.shape
    check(L.mgm_apply_order(n, k, _i(queue1), *arrs, bt, cl))
    return (*arrs, bt, cl)


def correct_normals(x, y, z, btag, cloud, nx, ny, nz):
    L = load()
    cl = _i(cloud)
    n, k = cl.shape
    nx, ny, nz = _f(nx).copy(), _f(ny).copy(), _f(nz).copy()
    check(L.mgm_correct_normals(n, k, _f(x), _f(y), _f(z), _u8(btag), cl, nx, ny, nz))
    return nx, ny, nz


def avg_dx(x, y, z, btag, cloud, dim):
    L = load()
    cl = _i(cloud)
    n, k = cl.shape
    d = C.c_double(0)
    check(L.mgm_avg_dx(n, k, dim, _f(x), _f(y), _f(z), _u8(btag), cl, C.byref(d)))
    return d.value


def derivative_weights(x, y, z, nx, ny, nz, btag, cloud, dim, phs, poly_degree):
    """Returns dict Dx, Dy, (Dz), lap, lapP, each [n][k]."""
    L = load()
    cl = _i(cloud)
    n, k = cl.shape
    out = {nm: np.zeros((n, k)) for nm in ("Dx", "Dy", "lap", "lapP")}
    Dz = np.zeros((n, k)) if dim == 3 else None
    check(L.mgm_derivative_weights(n, k, dim, phs, poly_degree, _f(x), _f(y), _f(z), _f(nx), _f(ny), _f(nz),
                                   _u8(btag), cl, out["Dx"], out["Dy"], ptr(Dz), out["lap"], out["lapP"]))
    if Dz is not None:
        out["Dz"] = Dz
    return out


def transfer_weights(tx, ty, tz, tbtag, src_pt, rows_from, only_interior, sx, sy, sz, scloud, dim, phs, poly_src):
    L = load()
    scl = _i(scloud)
    ns, ks = scl.shape
    nt = len(tx)
    W = np.zeros((nt, ks))
    check(L.mgm_transfer_weights(nt, _f(tx), _f(ty), _f(tz), _u8(tbtag), _i(src_pt), rows_from, only_interior,
                                 ns, ks, dim, phs, poly_src, _f(sx), _f(sy), _f(sz), scl, W))
    return W


def spmv(D, cloud, f):
    L = load()
    D = _f(D)
    n, k = D.shape
    out = np.zeros(n)
    check(L.mgm_spmv(n, k, D, _i(cloud), _f(f), out))
    return out


def gauss_jordan(A):
    """matrixInverse_Gauss_Jordan (mat_lib.h:423-491) of a square matrix on the GPU."""
    A = np.ascontiguousarray(A, dtype=np.float64)
    n = A.shape[0]
    inv = np.zeros((n, n))
    check(load().mgm_gauss_jordan(n, A, inv))
    return inv


def laplacian_for_poisson(Dx, Dy, Dz, lap, nx, ny, nz, btag):
    """create_laplacian_for_Poisson (rbf.h:382-399): lap on interior rows, the
    normal derivative on boundary rows ([n][k] arrays; Dz, nz None in 2D)."""
    Dx = _f(Dx)
    n, k = Dx.shape
    dim = 2 if Dz is None else 3
    Dz = None if Dz is None else _f(Dz)
    nz = None if nz is None else _f(nz)
    out = np.zeros((n, k))
    check(load().mgm_laplacian_for_poisson(n, k, dim, Dx, _f(Dy), ptr(Dz), _f(lap), _f(nx), _f(ny), ptr(nz),
                                           _u8(btag), out))
    return out


def read_gmsh(path, dim):
    """read_PointStructure (mesh_functions.h:172-476): one level's nodes from a
    Gmsh 2.2 ASCII file, as a clouds.Cloud (normals unnormalised, corner nodes
    removed; meta holds num_elem, d_avg and the corner tags)."""
    from .clouds import Cloud
    L = load()
    h = C.c_void_p()
    check(L.mgm_mesh_read(str(path).encode(), int(dim), C.byref(h)))
    try:
        n, nb, ne, da = C.c_int(), C.c_int(), C.c_int(), C.c_double()
        check(L.mgm_mesh_info(h, C.byref(n), C.byref(nb), C.byref(ne), C.byref(da)))
        a = {nm: np.zeros(n.value) for nm in ("x", "y", "z", "nx", "ny", "nz")}
        bt = np.zeros(n.value, np.uint8)
        ct = np.zeros(n.value, np.uint8)
        check(L.mgm_mesh_get(h, a["x"], a["y"], a["z"], a["nx"], a["ny"], a["nz"], bt, ct))
    finally:
        L.mgm_mesh_free(h)
    return Cloud(a["x"], a["y"], a["z"], a["nx"], a["ny"], a["nz"], bt, nb.value, int(dim), da.value, kind="gmsh",
                 meta={"num_elem": ne.value, "d_avg": da.value, "corner": ct, "path": str(path)})


def kernel_launches() -> int:
    return int(load().mgm_kernel_launches())


def set_device(device: int):
    check(load().mgm_set_device(device))


class Multigrid:
    """A device-resident multigrid hierarchy (the reference's PointStructure
    array after read_complete_mesh_data + create_derivative_matrices, and its
    FieldVariables after copyin_*_to_gpu)."""

    def __init__(self, clouds, ks, polys, phs=3, reference_transfer=False):
        self.L = load()
        self.nl = len(clouds)
        self.dim = clouds[0].dim
        h = self.L.mgm_create(self.dim, phs, self.nl)
        if not h:
            raise _lib.MgmError(-1, self.L.mgm_last_error().decode())
        self.h = h
        for l, c in enumerate(clouds):
            check(self.L.mgm_set_level(h, l, c.n, c.nb, _f(c.x), _f(c.y), _f(c.z), _f(c.nx), _f(c.ny), _f(c.nz),
                                       _u8(c.btag), polys[l], ks[l]))
        check(self.L.mgm_setup(h, _lib.SETUP_REFERENCE_TRANSFER if reference_transfer else 0))
        self.sizes = []
        for l in range(self.nl):
            n, nb, k, npl = C.c_int(), C.c_int(), C.c_int(), C.c_int()
            check(self.L.mgm_level_size(h, l, C.byref(n), C.byref(nb), C.byref(k), C.byref(npl)))
            self.sizes.append((n.value, nb.value, k.value, npl.value))
        self.reference_transfer = reference_transfer

    def close(self):
        if getattr(self, "h", None):
            self.L.mgm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def n(self, l=0):
        return self.sizes[l][0]

    def geometry(self, l):
        n, nb, k, _ = self.sizes[l]
        a = {nm: np.zeros(n) for nm in ("x", "y", "z", "nx", "ny", "nz")}
        a["btag"] = np.zeros(n, np.uint8)
        a["cloud"] = np.zeros((n, k), np.int32)
        check(self.L.mgm_get_geometry(self.h, l, *(ptr(a[nm]) for nm in ("x", "y", "z", "nx", "ny", "nz", "btag",
                                                                            "cloud"))))
        d = C.c_double()
        check(self.L.mgm_level_d_avg(self.h, l, C.byref(d)))
        a["d_avg"] = d.value
        return a

    def operators(self, l):
        n, nb, k, _ = self.sizes[l]
        out = {nm: np.zeros((n, k)) for nm in ("Dx", "Dy", "lap", "lapP")}
        Dz = np.zeros((n, k)) if self.dim == 3 else None
        check(self.L.mgm_get_operators(self.h, l, ptr(out["Dx"]), ptr(out["Dy"]), ptr(Dz), ptr(out["lap"]),
                                       ptr(out["lapP"])))
        if Dz is not None:
            out["Dz"] = Dz
        return out

    def transfer(self, l):
        n = self.sizes[l][0]
        rp = np.zeros(n, np.int32)
        pp = np.zeros(n, np.int32)
        restr = np.zeros((n, self.sizes[l - 1][2])) if (l > 0 and self.reference_transfer) else None
        prol = np.zeros((n, self.sizes[l + 1][2])) if (l < self.nl - 1 and self.reference_transfer) else None
        check(self.L.mgm_get_transfer(self.h, l, ptr(rp), ptr(pp), ptr(restr), ptr(prol)))
        return {"rpts": rp, "ppts": pp, "restr": restr, "prol": prol}

    def solver_transfer(self, l):
        """The convergent solver's restriction into level l (interior rows,
        [n][k of l-1]) and prolongation into level l (all rows, [n][k of l+1])."""
        n = self.sizes[l][0]
        restr = np.zeros((n, self.sizes[l - 1][2])) if l > 0 else None
        prol = np.zeros((n, self.sizes[l + 1][2])) if l < self.nl - 1 else None
        check(self.L.mgm_get_solver_transfer(self.h, l, ptr(restr), ptr(prol)))
        return {"restr": restr, "prol": prol}

    def compact(self, l, which):
        """The FP32 V-cycle's copy of level l's operator (which="op"), the
        restriction into it ("restr") or the prolongation into it ("prol"),
        decoded as the level kernels read it: (idx [n][k], w [n][k] float32,
        True where the gathers come from int16 offsets)."""
        code = {"op": 0, "restr": 1, "prol": 2}[which]
        n = self.sizes[l][0]
        k = self.sizes[l][2] if code == 0 else self.sizes[l - 1 if code == 1 else l + 1][2]
        idx = np.zeros((n, k), np.int32)
        w = np.zeros((n, k), np.float32)
        flag = C.c_int()
        check(self.L.mgm_get_compact(self.h, l, code, ptr(idx), ptr(w), C.byref(flag)))
        return idx, w, bool(flag.value)

    def set_flow(self, Re, courant, omega=1.0, num_relax=3, num_vcycles=10, dt=0.0):
        check(self.L.mgm_set_flow(self.h, Re, courant, omega, num_relax, num_vcycles, dt))
        d = C.c_double()
        check(self.L.mgm_get_dt(self.h, C.byref(d)))
        self.dt = d.value
        return self.dt

    def set_solver(self, rel_tol=1e-8, max_iters=60, cheb_degree=3, cheb_ratio=6.0):
        check(self.L.mgm_set_solver(self.h, rel_tol, max_iters, cheb_degree, cheb_ratio))

    def use_compact(self, enable=True):
        check(self.L.mgm_use_compact(self.h, 1 if enable else 0))

    def set_timple(self, iter_timple=1, iter_momentum=1, facRe=1.0, facdt=1.0):
        check(self.L.mgm_set_timple(self.h, iter_timple, iter_momentum, facRe, facdt))

    def write_solution(self, path, pressure="p_old"):
        """Solution.csv in the format of mg_NS_solver.c:83-88 (x y z u v w pressure)."""
        check(self.L.mgm_write_solution(self.h, str(path).encode(), _lib.FIELD[pressure]))

    def checkpoint_save(self, path):
        check(self.L.mgm_checkpoint_save(self.h, str(path).encode()))

    def checkpoint_load(self, path):
        check(self.L.mgm_checkpoint_load(self.h, str(path).encode()))

    REF_ROUTINES = {"relaxation": 0, "residuals": 1, "restrict": 2, "prolongate": 3}

    def ref_routine(self, level, routine):
        """One routine of the fractional step's reference-semantics multigrid:
        relaxation / residuals on `level`, restrict from `level` into level+1,
        prolongate from level+1 into `level` (fractional_step_solver.h:168-246)."""
        check(self.L.mgm_ref_routine(self.h, int(level), self.REF_ROUTINES[routine]))

    def timple_run(self, mode, nsteps):
        """nsteps TIMPLE steps timed on the device: (step_ms, p' V-cycles, steady_err)."""
        sm, vc, e = C.c_double(), C.c_longlong(), C.c_double()
        check(self.L.mgm_timple_run(self.h, mode, nsteps, C.byref(sm), C.byref(vc), C.byref(e)))
        return sm.value, vc.value, e.value

    def heat_init(self, wave_number=1):
        """The heat-conduction program's set-up (init_heat_conduction.c:14-67)."""
        check(self.L.mgm_heat_init(self.h, int(wave_number)))

    def heat_step(self):
        """One pass of mg_heat_conduction.c's time loop; returns the sum of the
        squared changes of level-0 p."""
        e = C.c_double()
        check(self.L.mgm_heat_step(self.h, C.byref(e)))
        return e.value

    def timple_step(self, mode=_lib.MODE_REFERENCE):
        """time_implicit_solver (timple_solver.h:40-70); returns the steady-state error."""
        e = C.c_double()
        check(self.L.mgm_timple_step(self.h, mode, C.byref(e)))
        return e.value

    def timple_part(self, part, mode=_lib.MODE_REFERENCE):
        check(self.L.mgm_timple_part(self.h, _lib.TIMPLE_PARTS[part], mode))

    def use_tiled(self, enable=True):
        check(self.L.mgm_use_tiled(self.h, 1 if enable else 0))

    def set_compatible_rhs(self, enable=True):
        """Project every Poisson source onto the consistent subspace of the
        singular lap_Poison before the pinned solve; no reference counterpart."""
        check(self.L.mgm_set_compatible_rhs(self.h, 1 if enable else 0))

    def use_half_operator(self, enable=True):
        """FP32_IR V-cycle on the FP16 operator D^-1 A (large levels); no reference counterpart."""
        check(self.L.mgm_use_half_operator(self.h, 1 if enable else 0))

    def use_graphs(self, enable=True):
        check(self.L.mgm_use_graphs(self.h, 1 if enable else 0))

    def use_launch_chaining(self, enable=True):
        """Programmatic dependent launch between the V-cycle's kernels (default on)."""
        check(self.L.mgm_use_launch_chaining(self.h, 1 if enable else 0))

    def use_fused_coarse(self, enable=True):
        """The small levels' V-cycle as one cooperative launch (opt-in; default off)."""
        check(self.L.mgm_use_fused_coarse(self.h, 1 if enable else 0))

    def fused_coarse_available(self):
        v = C.c_int()
        check(self.L.mgm_fused_coarse_available(self.h, C.byref(v)))
        return bool(v.value)

    def solve_counters(self):
        """(V-cycles, restart-cycle starts, solves) of the last run_steps / step."""
        v, c, n = C.c_longlong(), C.c_longlong(), C.c_longlong()
        check(self.L.mgm_solve_counters(self.h, C.byref(v), C.byref(c), C.byref(n)))
        return v.value, c.value, n.value

    def solve_start_residual(self):
        """Geometric mean of the relative residual each solve of the last run started from."""
        v = C.c_double()
        check(self.L.mgm_solve_start_residual(self.h, C.byref(v)))
        return v.value

    def set_initial_guess(self, flags):
        """MGM_GUESS_* flags of the steps' Poisson solves (0: previous pressure)."""
        check(self.L.mgm_set_initial_guess(self.h, int(flags)))

    def use_step_graph(self, enable=True):
        check(self.L.mgm_use_step_graph(self.h, 1 if enable else 0))

    def apply_bc(self, kind=_lib.BC_LID):
        check(self.L.mgm_apply_bc(self.h, kind))

    def set_field(self, name, values, l=0):
        check(self.L.mgm_set_field(self.h, l, _lib.FIELD[name], _f(values)))

    def get_field(self, name, l=0):
        out = np.zeros(self.sizes[l][0])
        check(self.L.mgm_get_field(self.h, l, _lib.FIELD[name], out))
        return out

    def step(self, mode=_lib.MODE_FP64):
        e = C.c_double()
        check(self.L.mgm_step(self.h, mode, C.byref(e)))
        return e.value

    def intermediate_velocity(self):
        check(self.L.mgm_intermediate_velocity(self.h))

    def mass_residual(self):
        check(self.L.mgm_mass_residual(self.h))

    def poisson(self, mode):
        check(self.L.mgm_poisson(self.h, mode))

    def update_velocity(self, with_mass=False):
        m = C.c_double()
        check(self.L.mgm_update_velocity(self.h, C.byref(m) if with_mass else None))
        return m.value

    def last_solve(self):
        it, rr = C.c_int(), C.c_double()
        check(self.L.mgm_last_solve(self.h, C.byref(it), C.byref(rr)))
        return it.value, rr.value

    def solve_poisson(self, b, p0=None, mode=_lib.MODE_FP64):
        n = self.sizes[0][0]
        p = np.zeros(n) if p0 is None else _f(p0).copy()
        it, rr = C.c_int(), C.c_double()
        check(self.L.mgm_solve_poisson(self.h, mode, _f(b), p, C.byref(it), C.byref(rr)))
        return p, it.value, rr.value

    def sync(self):
        check(self.L.mgm_sync(self.h))

    def run_steps(self, mode, nsteps):
        """nsteps fractional steps timed on the device: (step_ms, poisson_ms, vcycles, steady_err)."""
        sm, pm, vc, e = C.c_double(), C.c_double(), C.c_longlong(), C.c_double()
        check(self.L.mgm_run_steps(self.h, mode, nsteps, C.byref(sm), C.byref(pm), C.byref(vc), C.byref(e)))
        return sm.value, pm.value, vc.value, e.value

    def step_host(self, mode, u_in=None, v_in=None, u_out=None, v_out=None, p_out=None):
        """One step with host buffers (ctypes pointers / None)."""
        e = C.c_double()
        check(self.L.mgm_step_host(self.h, mode, u_in, v_in, None, u_out, v_out, None, p_out, C.byref(e)))
        return e.value

    def profile_smoother(self, enable=True):
        check(self.L.mgm_profile_smoother(self.h, 1 if enable else 0))

    def profile_read(self):
        ms, nl, by = C.c_double(), C.c_longlong(), C.c_longlong()
        check(self.L.mgm_profile_read(self.h, C.byref(ms), C.byref(nl), C.byref(by)))
        return ms.value, nl.value, by.value


class PinnedArray:
    """A page-locked host array (mgm_host_alloc) viewed as numpy."""

    def __init__(self, n, dtype=np.float64):
        self.L = load()
        nbytes = int(n) * np.dtype(dtype).itemsize
        self.ptr = self.L.mgm_host_alloc(nbytes)
        if not self.ptr:
            raise _lib.MgmError(_lib.MGM_ERR_NOMEM, self.L.mgm_last_error().decode())
        buf = (C.c_char * nbytes).from_address(self.ptr)
        self.array = np.frombuffer(buf, dtype=dtype, count=int(n))

    def free(self):
        if self.ptr:
            self.array = None
            self.L.mgm_host_free(self.ptr)
            self.ptr = None


class Batch:
    """A hierarchy with a stencil size per node, assembled in one persistent
    weight launch, solving many Poisson right-hand sides through one V-cycle
    (mgm_batch_* in include/mgm.h).  Node arrays come back in the reordered
    order; operators are CSR (row_ptr, col, values)."""

    def __init__(self, clouds, k_per_node, polys, phs=3, autotune=True):
        self.L = load()
        self.nl = len(clouds)
        self.dim = clouds[0].dim
        h = self.L.mgm_batch_create(self.dim, phs, self.nl)
        if not h:
            raise _lib.MgmError(-1, self.L.mgm_last_error().decode())
        self.h = h
        for l, c in enumerate(clouds):
            check(self.L.mgm_batch_set_level(h, l, c.n, c.nb, _f(c.x), _f(c.y), _f(c.z), _f(c.nx), _f(c.ny),
                                             _f(c.nz), _u8(c.btag), polys[l], _i(k_per_node[l])))
        check(self.L.mgm_batch_setup(h, _lib.BATCH_AUTOTUNE if autotune else 0))
        self.sizes = []
        for l in range(self.nl):
            n, nb = C.c_int(), C.c_int()
            nnz, rn, pn = C.c_longlong(), C.c_longlong(), C.c_longlong()
            check(self.L.mgm_batch_level_size(h, l, C.byref(n), C.byref(nb), C.byref(nnz), C.byref(rn), C.byref(pn)))
            self.sizes.append((n.value, nb.value, nnz.value, rn.value, pn.value))

    def close(self):
        if getattr(self, "h", None):
            self.L.mgm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def n(self, l=0):
        return self.sizes[l][0]

    def weights_report(self):
        wm, tm = C.c_double(), C.c_double()
        ns = C.c_longlong()
        nt, sm, cta = C.c_int(), C.c_int(), C.c_int()
        check(self.L.mgm_batch_weights_report(self.h, C.byref(wm), C.byref(tm), C.byref(ns), C.byref(nt),
                                              C.byref(sm), C.byref(cta)))
        cnt = C.c_int()
        check(self.L.mgm_batch_num_classes(self.h, C.byref(cnt)))
        classes = []
        for i in range(cnt.value):
            N, s, t, us = C.c_int(), C.c_longlong(), C.c_int(), C.c_double()
            check(self.L.mgm_batch_class(self.h, i, C.byref(N), C.byref(s), C.byref(t), C.byref(us)))
            classes.append({"order": N.value, "systems": s.value, "team_threads": t.value,
                            "us_per_system": us.value})
        return {"weights_ms": wm.value, "tuning_ms": tm.value, "systems": ns.value, "tiles": nt.value,
                "smem_bytes": sm.value, "ctas_per_sm": cta.value, "classes": classes}

    def level(self, l):
        n, nb, nnz, _, _ = self.sizes[l]
        a = {nm: np.zeros(n) for nm in ("x", "y", "z", "nx", "ny", "nz")}
        a["btag"] = np.zeros(n, np.uint8)
        a["k"] = np.zeros(n, np.int32)
        a["row_ptr"] = np.zeros(n + 1, np.int32)
        a["col"] = np.zeros(max(nnz, 1), np.int32)
        for nm in ("Dx", "Dy", "Dz", "lap", "lapP"):
            a[nm] = np.zeros(max(nnz, 1)) if (nm != "Dz" or self.dim == 3) else None
        check(self.L.mgm_batch_get_level(self.h, l, *(ptr(a[nm]) for nm in (
            "x", "y", "z", "nx", "ny", "nz", "btag", "k", "row_ptr", "col", "Dx", "Dy", "Dz", "lap", "lapP"))))
        return a

    def transfer(self, l):
        n, _, _, rn, pn = self.sizes[l]
        a = {"rpts": np.zeros(n, np.int32), "ppts": np.zeros(n, np.int32)}
        if l > 0:
            a.update(r_ptr=np.zeros(n + 1, np.int32), r_col=np.zeros(max(rn, 1), np.int32), r_w=np.zeros(max(rn, 1)))
        if l < self.nl - 1:
            a.update(p_ptr=np.zeros(n + 1, np.int32), p_col=np.zeros(max(pn, 1), np.int32), p_w=np.zeros(max(pn, 1)))
        check(self.L.mgm_batch_get_transfer(self.h, l, *(ptr(a.get(nm)) for nm in (
            "rpts", "ppts", "r_ptr", "r_col", "r_w", "p_ptr", "p_col", "p_w"))))
        return a

    def set_solver(self, rel_tol=1e-8, restart=24, cheb_degree=3, cheb_ratio=20.0):
        check(self.L.mgm_batch_set_solver(self.h, rel_tol, restart, cheb_degree, cheb_ratio))

    def solve(self, rhs, mode=_lib.MODE_FP32_IR, out=None):
        """rhs [nrhs][n0] -> (solutions [nrhs][n0], V-cycles, rel. residuals [nrhs], device ms).
        rhs and out (the solutions' array, allocated when None) may be views
        of PinnedArray buffers: the copies to and from the device then run
        from page-locked memory."""
        rhs = _f(np.atleast_2d(rhs))
        nrhs = rhs.shape[0]
        sol = np.zeros_like(rhs) if out is None else out
        if sol.shape != rhs.shape or sol.dtype != np.float64 or not sol.flags["C_CONTIGUOUS"]:
            raise ValueError("out must be a C-contiguous float64 array shaped like rhs")
        vc = C.c_int()
        rr = np.zeros(nrhs)
        ms = C.c_double()
        check(self.L.mgm_batch_solve(self.h, mode, nrhs, rhs, sol, C.byref(vc), rr, C.byref(ms)))
        return sol, vc.value, rr, ms.value
