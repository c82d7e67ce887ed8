"""Python binding of the C ABI in include/sipg_b200.h (ctypes + numpy).

Host-side mirror used by the tests and the benchmark. It loads the in-tree
libsipg_b200.so and fails loudly when it is missing: there is no CPU fallback
for any operation of the solve path.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsipg_b200.so")

SIPG_OK = 0
SIPG_NOT_CONVERGED = 1
SIPG_BREAKDOWN = 2
SIPG_INVALID_ARG = 3
SIPG_OUT_OF_MEMORY = 4
SIPG_CANCELLED = 5
SIPG_CUDA_ERROR = 6
SIPG_NO_DEVICE = 7

MM_NONE, MM_SCALAR, MM_NODAL = 0, 1, 2
BC_DIRICHLET, BC_NEUMANN, BC_SLIP = 0, 1, 2
FP64, FP32 = 64, 32
SOLVER_CG, SOLVER_INV_MASS, SOLVER_JACOBI, SOLVER_BLOCK_JACOBI, SOLVER_PMULTIGRID = 0, 1, 2, 3, 4

_lib = None


class SipgError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"sipg status {status}: {msg}")
        self.status = status


class SolveInfo(C.Structure):
    _fields_ = [("iters", C.c_int), ("rel_res", C.c_double), ("abs_res", C.c_double),
                ("true_rel_res", C.c_double), ("setup_ms", C.c_double), ("solve_ms", C.c_double),
                ("status", C.c_int)]


class SolverOpts(C.Structure):
    _fields_ = [("rel_tol", C.c_double), ("abs_tol", C.c_double), ("max_iter", C.c_int),
                ("nullspace", C.c_int), ("precision", C.c_int), ("inv_mass_factor", C.c_double),
                ("ref_volume_block", C.c_int), ("n_levels", C.c_int), ("orders", C.c_int * 4),
                ("cheb_order", C.c_int), ("eig_safety", C.c_double), ("eig_ratio", C.c_double),
                ("eig_iters", C.c_int), ("coarse_iters", C.c_int), ("check_every", C.c_int),
                ("coarse_kind", C.c_int), ("amg_coarse_max", C.c_int), ("amg_strength", C.c_double),
                ("graphs", C.c_int), ("assembled_max_order", C.c_int), ("smoother", C.c_int),
                ("cheb_orders", C.c_int * 4), ("pre_it", C.c_int * 4), ("post_it", C.c_int * 4),
                ("amg_cheb_order", C.c_int), ("amg_reuse_interpolation", C.c_int)]


def lib():
    """Load the native library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C ins-solver_b200`")
        _lib = C.CDLL(LIB_PATH)
        _lib.sipg_last_error.restype = C.c_char_p
    return _lib


def check(st):
    if st != SIPG_OK:
        raise SipgError(st, lib().sipg_last_error().decode())
    return st


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int)) if a is not None else None


class DeviceVector:
    """A device copy of a host array, allocated through the library's own helpers
    (no torch or CUDA toolkit needed by the caller)."""

    def __init__(self, host):
        self.host = np.ascontiguousarray(host)
        self.nbytes = self.host.nbytes
        self._p = C.c_void_p()
        check(lib().sipg_dev_alloc(C.c_size_t(self.nbytes), C.byref(self._p)))
        check(lib().sipg_memcpy_h2d(self._p, self.host.ctypes.data_as(C.c_void_p), C.c_size_t(self.nbytes)))

    @property
    def ptr(self):
        return self._p.value

    def get(self):
        out = np.empty_like(self.host)
        check(lib().sipg_device_synchronize())
        check(lib().sipg_memcpy_d2h(out.ctypes.data_as(C.c_void_p), self._p, C.c_size_t(self.nbytes)))
        return out

    def __del__(self):
        if getattr(self, "_p", None) is not None and self._p.value:
            lib().sipg_dev_free(self._p)
            self._p = None


def extrapolate_initial_guess(times, history, t_new):
    """Initial guess at t_new from previous solutions (host arrays), the polynomial
    through (times[i], history[i]) -- initial_guess_extrapolation of the reference."""
    hs = [np.ascontiguousarray(h, dtype=np.float64) for h in history]
    t = np.ascontiguousarray(times, dtype=np.float64)
    out = np.empty_like(hs[0])
    ptrs = (C.c_void_p * len(hs))(*[h.ctypes.data for h in hs])
    check(lib().sipg_extrapolate_initial_guess_host(len(hs), _dp(t), ptrs, C.c_double(t_new),
                                                    C.c_size_t(out.size), _dp(out)))
    return out


def extrapolate_initial_guess_device(times, history_ptrs, t_new, n, out_ptr, stream=None):
    """Device variant: history_ptrs and out_ptr are device pointers of n FP64 values."""
    t = np.ascontiguousarray(times, dtype=np.float64)
    ptrs = (C.c_void_p * len(history_ptrs))(*history_ptrs)
    check(lib().sipg_extrapolate_initial_guess(len(history_ptrs), _dp(t), ptrs, C.c_double(t_new),
                                               C.c_size_t(n), C.c_void_p(out_ptr), C.c_void_p(stream or 0)))


def device_count():
    n = C.c_int(0)
    check(lib().sipg_device_count(C.byref(n)))
    return n.value


def ref_sizes(dim, order):
    Np, Nfp, Nf, Nperm = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    check(lib().sipg_ref_sizes(dim, order, C.byref(Np), C.byref(Nfp), C.byref(Nf), C.byref(Nperm)))
    return Np.value, Nfp.value, Nf.value, Nperm.value


def ref_tables(dim, order):
    """Reference element tables (row-major numpy arrays)."""
    Np, Nfp, Nf, Nperm = ref_sizes(dim, order)
    t = {k: np.zeros(Np) for k in ("r", "s", "t")}
    for k in ("Dr", "Ds", "Dt", "M"):
        t[k] = np.zeros((Np, Np))
    t["MMF"] = np.zeros((Nf, Np, Np))
    t["EMAT"] = np.zeros((Np, Nf * Nfp))
    t["fmask"] = np.zeros((Nf, Nfp), dtype=np.int32)
    t["perm_pos"] = np.zeros((Nperm, Nfp), dtype=np.int32)
    check(lib().sipg_ref_tables(dim, order, _dp(t["r"]), _dp(t["s"]), _dp(t["t"]), _dp(t["Dr"]),
                                _dp(t["Ds"]), _dp(t["Dt"]), _dp(t["M"]), _dp(t["MMF"]),
                                _dp(t["EMAT"]), _ip(t["fmask"]), _ip(t["perm_pos"])))
    t.update(Np=Np, Nfp=Nfp, Nf=Nf, dim=dim, order=order)
    return t


def interp_matrix(dim, q, p):
    Npp = ref_sizes(dim, p)[0]
    Npq = ref_sizes(dim, q)[0]
    P = np.zeros((Npp, Npq))
    check(lib().sipg_interp_matrix(dim, q, p, _dp(P)))
    return P


def box_mesh(dim, n, jitter=0.0, seed=0):
    Nv, K = C.c_int(), C.c_int()
    check(lib().sipg_box_mesh_sizes(dim, n, C.byref(Nv), C.byref(K)))
    vx = np.zeros((Nv.value, dim))
    e2v = np.zeros((K.value, dim + 1), dtype=np.int32)
    check(lib().sipg_box_mesh(dim, n, C.c_double(jitter), C.c_uint64(seed), _dp(vx), _ip(e2v)))
    return vx, e2v


class Mesh:
    """Resident mesh (DGMesh3D / DGMesh2D stand-in)."""

    def __init__(self, dim, vx, e2v):
        self.dim = dim
        vx = np.ascontiguousarray(vx, dtype=np.float64)
        e2v = np.ascontiguousarray(e2v, dtype=np.int32)
        self.h = C.c_void_p()
        check(lib().sipg_mesh_create(dim, vx.shape[0], _dp(vx), e2v.shape[0], _ip(e2v), C.byref(self.h)))
        K, F, Kb = C.c_int(), C.c_int(), C.c_int()
        check(lib().sipg_mesh_sizes(self.h, C.byref(K), C.byref(F), C.byref(Kb)))
        self.K, self.F, self.Kb = K.value, F.value, Kb.value

    @classmethod
    def box(cls, dim, n, jitter=0.0, seed=0, geometry_bits=32):
        vx, e2v = box_mesh(dim, n, jitter, seed)
        m = cls(dim, vx, e2v)
        if geometry_bits != 32:
            m.set_geometry_precision(geometry_bits)
        return m

    def set_geometry_precision(self, bits):
        """Geometric factors of the FP32 kernels in BF16 (16) or FP32 (32), before the
        mesh's first device use (sipg_mesh_set_geometry_precision)."""
        check(lib().sipg_mesh_set_geometry_precision(self.h, bits))

    def export(self, order):
        """Per-order host data in the reference's form (dict of numpy arrays)."""
        Np, Nfp, Nf, _ = ref_sizes(self.dim, order)
        K, F, Kb, dim = self.K, self.F, self.Kb, self.dim
        d = dict(geof=np.zeros((K, 10 if dim == 3 else 5)))
        for k in ("nx", "ny", "nz", "sJ", "fscale"):
            d[k] = np.zeros((K, Nf))
        d["face2cells"] = np.zeros((F, 2), np.int32)
        d["faceNum"] = np.zeros((F, 2), np.int32)
        d["fmaskL"] = np.zeros((F, Nfp), np.int32)
        d["fmaskR"] = np.zeros((F, Nfp), np.int32)
        d["bface2cell"] = np.zeros(Kb, np.int32)
        d["bfaceNum"] = np.zeros(Kb, np.int32)
        d["bface_centroid"] = np.zeros((Kb, dim))
        for k in ("x", "y", "z"):
            d[k] = np.zeros((K, Np))
        check(lib().sipg_mesh_export(self.h, order, _dp(d["geof"]), _dp(d["nx"]), _dp(d["ny"]),
                                     _dp(d["nz"]), _dp(d["sJ"]), _dp(d["fscale"]),
                                     _ip(d["face2cells"]), _ip(d["faceNum"]), _ip(d["fmaskL"]),
                                     _ip(d["fmaskR"]), _ip(d["bface2cell"]), _ip(d["bfaceNum"]),
                                     _dp(d["bface_centroid"]), _dp(d["x"]), _dp(d["y"]), _dp(d["z"])))
        d.update(K=K, F=F, Kb=Kb, Np=Np, Nfp=Nfp, Nf=Nf, dim=dim, order=order)
        return d

    def device_bytes(self):
        b = C.c_size_t()
        check(lib().sipg_mesh_device_bytes(self.h, C.byref(b)))
        return b.value

    def __del__(self):
        if getattr(self, "h", None) and self.h:
            lib().sipg_mesh_destroy(self.h)
            self.h = None



def ins_advection(mesh, order, dt, a0, a1, b0, b1, vel, vel_old, N_old, vel_bc):
    """Non-linear advection step (sipg_ins_advection_host): returns (N, velT),
    each (3, K, Np); vel_bc: Kb velocity boundary types (0 no-slip, 1 slip,
    2 natural outflow)."""
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (vel, vel_old, N_old)]
    bc = np.ascontiguousarray(vel_bc, dtype=np.int32).reshape(-1)
    N = np.zeros_like(arrs[0])
    velT = np.zeros_like(arrs[0])
    check(lib().sipg_ins_advection_host(mesh.h, order, C.c_double(dt), C.c_double(a0), C.c_double(a1),
                                        C.c_double(b0), C.c_double(b1), _dp(arrs[0]), _dp(arrs[1]), _dp(arrs[2]),
                                        _ip(bc), _dp(N), _dp(velT)))
    return N, velT


def ins_pressure_neumann(mesh, order, reynolds, vel, N, mu, rho, vel_bc):
    """Curl-curl Neumann data of the multiphase pressure step
    (sipg_ins_pressure_neumann_host): returns dPdN (K, 4, Nfp), nonzero on the
    no-slip and slip wall faces; vel, N: (3, K, Np); mu, rho: (K, Np)."""
    v, n = (np.ascontiguousarray(a, dtype=np.float64) for a in (vel, N))
    m, r = (np.ascontiguousarray(a, dtype=np.float64) for a in (mu, rho))
    bc = np.ascontiguousarray(vel_bc, dtype=np.int32).reshape(-1)
    nfp = (order + 1) * (order + 2) // 2
    out = np.zeros((v.shape[1], 4, nfp))
    check(lib().sipg_ins_pressure_neumann_host(mesh.h, order, C.c_double(reynolds), _dp(v), _dp(n), _dp(m),
                                               _dp(r), _ip(bc), _dp(out)))
    return out


class Ins3DOpts(C.Structure):
    """sipg_ins3d_opts: the MPINSSolver3D configuration of the two-phase time step,
    with the pressure (p-multigrid) and viscous (Jacobi-PCG) solver options."""
    _fields_ = [("order", C.c_int), ("reynolds", C.c_double), ("rho0", C.c_double), ("rho1", C.c_double),
                ("mu0", C.c_double), ("mu1", C.c_double), ("gravity", C.c_double), ("ls_alpha", C.c_double),
                ("cfl", C.c_double), ("extrapolate_history", C.c_int), ("pr_over_int", C.c_int),
                ("reinit_freq", C.c_int), ("reinit_ic", C.c_int), ("ls_cap", C.c_double),
                ("pr_setup_every", C.c_int), ("viscous_kind", C.c_int),
                ("pressure", SolverOpts),
                ("viscous", SolverOpts)]


class Ins3DStepInfo(C.Structure):
    _fields_ = [("time", C.c_double), ("dt", C.c_double), ("pr_iters", C.c_int), ("vis_iters", C.c_int * 3),
                ("pr_rel_res", C.c_double), ("vis_rel_res", C.c_double * 3), ("max_vel", C.c_double),
                ("ms_advection", C.c_double), ("ms_pressure", C.c_double), ("ms_viscosity", C.c_double),
                ("ms_surface", C.c_double), ("ms_pressure_setup", C.c_double),
                ("ms_pressure_solve", C.c_double), ("proj_converged", C.c_ulonglong)]


def ins3d_default_opts(**kw):
    """Defaults of sipg_ins3d_default_opts with overrides: plain fields by name,
    precision (the pressure V-cycle's), and pr_<field> / vis_<field> for the
    pressure and viscous solver options (pr_rel_tol, vis_max_iter, pr_cheb_order ...)."""
    o = Ins3DOpts()
    check(lib().sipg_ins3d_default_opts(C.byref(o)))
    for k, v in kw.items():
        if k == "precision":
            o.pressure.precision = v
        elif k in ("pr_over_int", "pr_setup_every", "viscous_kind", "reinit_freq", "reinit_ic", "ls_cap"):
            setattr(o, k, v)
        elif k.startswith("pr_"):
            setattr(o.pressure, k[3:], v)
        elif k.startswith("vis_"):
            setattr(o.viscous, k[4:], v)
        else:
            setattr(o, k, v)
    return o


class Ins3D:
    """Two-phase 3D time step on the device (sipg_ins3d_*): MPINSSolver3D's init /
    step / field access with its level set, no-slip walls and natural outflow."""

    def __init__(self, mesh, vel_bc, opts=None, **kw):
        self.mesh = mesh
        self.o = opts if opts is not None else ins3d_default_opts(**kw)
        self.Np = ref_sizes(3, self.o.order)[0]
        bc = np.ascontiguousarray(vel_bc, dtype=np.int32).reshape(-1)
        self.h = C.c_void_p()
        check(lib().sipg_ins3d_create(mesh.h, C.byref(self.o), _ip(bc), C.byref(self.h)))

    def set_state(self, vel, s):
        v = np.ascontiguousarray(vel, dtype=np.float64)
        q = np.ascontiguousarray(s, dtype=np.float64)
        check(lib().sipg_ins3d_set_state_host(self.h, _dp(v), _dp(q)))

    def step(self, nsteps=1):
        info = Ins3DStepInfo()
        check(lib().sipg_ins3d_step(self.h, nsteps, C.byref(info)))
        return info

    def state(self):
        K, Np = self.mesh.K, self.Np
        vel, pr, s, rho, mu = np.zeros((3, K, Np)), *(np.zeros((K, Np)) for _ in range(4))
        check(lib().sipg_ins3d_get_state_host(self.h, _dp(vel), _dp(pr), _dp(s), _dp(rho), _dp(mu)))
        return dict(vel=vel, pr=pr, s=s, rho=rho, mu=mu)

    def close(self):
        if self.h:
            lib().sipg_ins3d_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ls_reinit(mesh, order, s, ls_cap=1.0):
    """Closest-point reinitialisation of a level set (sipg_ls_reinit_host): returns the
    new (K, Np) values."""
    out = np.array(s, dtype=np.float64, order="C", copy=True)
    check(lib().sipg_ls_reinit_host(mesh.h, order, C.c_double(ls_cap), _dp(out)))
    return out


def projection_factor(dim, dt):
    """The penalty factor INSSolverBase{3D,2D}::project_velocity passes to the
    element-local solve: dt in 3D (src/solvers/3d/ins_solver_base.cpp:1082),
    dt * 1e3 in 2D (src/solvers/2d/ins_solver_base.cpp:916)."""
    return dt if dim == 3 else dt * 1e3


def project_velocity(mesh, order, dt, dp, velT, factor=None):
    """Element-local velocity projection (div_div = 1) on host arrays.

    dp (pressure gradient) and velT: (dim, K, Np). Returns (velTT, stats) with
    stats = (cells, converged cells, iterations summed over cells)."""
    dp = np.ascontiguousarray(dp, dtype=np.float64)
    velT = np.ascontiguousarray(velT, dtype=np.float64)
    out = np.empty_like(velT)
    st = np.zeros(3)
    f = projection_factor(mesh.dim, dt) if factor is None else factor
    check(lib().sipg_project_velocity_host(mesh.h, order, C.c_double(dt), C.c_double(f), _dp(dp), _dp(velT),
                                           _dp(out), _dp(st)))
    return out, st


def project_velocity_device(mesh, order, dt, dp_ptr, velT_ptr, velTT_ptr, stats_ptr=None, factor=None,
                            stream=None):
    """Device variant: FP64 device pointers (dim x K x Np); stats_ptr, if given,
    points to 2 uint64 counters (converged elements, iterations)."""
    f = projection_factor(mesh.dim, dt) if factor is None else factor
    check(lib().sipg_project_velocity(mesh.h, order, C.c_double(dt), C.c_double(f), C.c_void_p(dp_ptr),
                                      C.c_void_p(velT_ptr), C.c_void_p(velTT_ptr), C.c_void_p(stats_ptr or 0),
                                      C.c_void_p(stream or 0)))


def pressure_projection(mesh, order, dt, pr, velT, rho=None, factor=None):
    """Pressure projection step on host arrays: grad p with the central flux
    (divided by rho when given), then the element-local velocity projection.
    pr, rho: (K, Np); velT: (dim, K, Np). Returns (velTT, stats)."""
    pr = np.ascontiguousarray(pr, dtype=np.float64)
    velT = np.ascontiguousarray(velT, dtype=np.float64)
    r = None if rho is None else np.ascontiguousarray(rho, dtype=np.float64)
    out = np.empty_like(velT)
    st = np.zeros(3)
    f = projection_factor(mesh.dim, dt) if factor is None else factor
    check(lib().sipg_pressure_projection_host(mesh.h, order, C.c_double(dt), C.c_double(f), _dp(pr), _dp(r),
                                              _dp(velT), _dp(out), _dp(st)))
    return out, st


def pressure_rhs(mesh, order, dt, velT, dPdN=None, dPdN_old=None, b0=1.0, b1=0.0):
    """Right-hand side of the pressure solve on host arrays: J M (-div_c(velT) / dt
    + LIFT (b0 dPdN + b1 dPdN_old)). velT: (dim, K, Np); dPdN, dPdN_old:
    (K, dim + 1, Nfp) or None. Returns (rhs (K, Np), updated dPdN_old or None)."""
    velT = np.ascontiguousarray(velT, dtype=np.float64)
    dn = None if dPdN is None else np.ascontiguousarray(dPdN, dtype=np.float64)
    do = None if dPdN_old is None else np.array(dPdN_old, dtype=np.float64, order="C", copy=True)
    rhs = np.empty(velT.shape[1:])
    check(lib().sipg_pressure_rhs_host(mesh.h, order, C.c_double(dt), C.c_double(b0), C.c_double(b1), _dp(velT),
                                       _dp(dn), _dp(do), _dp(rhs)))
    return rhs, do

class Operator:
    """SIPG operator on a resident mesh (Poisson / Helmholtz / viscous)."""

    def __init__(self, mesh, order, ncomp=1):
        self.mesh = mesh
        self.order = order
        self.ncomp = ncomp
        self.h = C.c_void_p()
        check(lib().sipg_op_create(mesh.h, order, ncomp, C.byref(self.h)))
        self.Np, self.Nfp = ref_sizes(mesh.dim, order)[:2]
        self.K = mesh.K

    def shape(self):
        return (self.ncomp, self.K, self.Np)

    def set_factor(self, factor):
        f = None if factor is None else np.ascontiguousarray(factor, dtype=np.float64)
        check(lib().sipg_op_set_factor(self.h, _dp(f)))

    def set_mm(self, mode, scalar=0.0, mm=None):
        m = None if mm is None else np.ascontiguousarray(mm, dtype=np.float64)
        check(lib().sipg_op_set_mm(self.h, mode, C.c_double(scalar), _dp(m)))

    def set_bc_types(self, types):
        t = np.ascontiguousarray(types, dtype=np.int32).reshape(-1)
        check(lib().sipg_op_set_bc_types(self.h, _ip(t)))

    def set_kernel(self, kind):
        """0: tensor cores where available (default), 1: CUDA cores."""
        check(lib().sipg_op_set_kernel(self.h, int(kind)))

    def set_pin(self, elem, node=0):
        check(lib().sipg_op_set_pin(self.h, elem, node))

    def apply_host(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        check(lib().sipg_op_apply_host(self.h, _dp(x), _dp(y)))
        return y

    def apply_device(self, precision, x_ptr, y_ptr, stream=None):
        check(lib().sipg_op_apply(self.h, precision, C.c_void_p(x_ptr), C.c_void_p(y_ptr),
                                  C.c_void_p(stream or 0)))

    def apply_bc_host(self, bc, rhs):
        bc = np.ascontiguousarray(bc, dtype=np.float64)
        out = np.ascontiguousarray(rhs, dtype=np.float64).copy()
        check(lib().sipg_op_apply_bc_host(self.h, _dp(bc), _dp(out)))
        return out

    def diag_host(self):
        d = np.zeros(self.shape())
        check(lib().sipg_op_diag_host(self.h, _dp(d)))
        return d

    def block_diag_host(self, invert=False, ref_volume_block=False):
        b = np.zeros(self.shape() + (self.Np,))
        check(lib().sipg_op_block_diag_host(self.h, int(invert), int(ref_volume_block), _dp(b)))
        return b

    def oi_sizes(self):
        """(nq, nqs): volume and per-face surface cubature points of the
        over-integrated factor."""
        nq, nqs = C.c_int(), C.c_int()
        check(lib().sipg_op_oi_sizes(self.h, C.byref(nq), C.byref(nqs)))
        return nq.value, nqs.value

    def oi_points(self):
        """Physical coordinates of the cubature points: (dim, K, nq) and (dim, K, Nf, nqs)."""
        nq, nqs = self.oi_sizes()
        d, K = self.mesh.dim, self.mesh.K
        xv = np.zeros((d, K, nq))
        xs = np.zeros((d, K, d + 1, nqs))
        check(lib().sipg_op_oi_points_host(self.h, _dp(xv), _dp(xs)))
        return xv, xs

    def set_factor_oi(self, fvol, fsurf):
        """Over-integrated factor: fvol (K, nq) and fsurf (K, Nf, nqs) at the
        points of oi_points()."""
        fvol = np.ascontiguousarray(fvol, dtype=np.float64)
        fsurf = np.ascontiguousarray(fsurf, dtype=np.float64)
        check(lib().sipg_op_set_factor_oi(self.h, _dp(fvol), _dp(fsurf)))

    def element_blocks_host(self):
        """Assembled element-row blocks (order 1 or 2, scalar): array
        [1 + Nf, Np (row), Np (column), K]; block s = 1 + f couples to the
        neighbour across face f in that neighbour's node order."""
        K = self.mesh.K
        nf = self.mesh.dim + 1
        b = np.zeros((nf + 1, self.Np, self.Np, K))
        check(lib().sipg_op_element_blocks_host(self.h, _dp(b)))
        return b

    def __del__(self):
        if getattr(self, "h", None) and self.h:
            lib().sipg_op_destroy(self.h)
            self.h = None


class Amg:
    """Algebraic coarse hierarchy (host build) below the p=1 level."""

    def __init__(self, h):
        self.h = h
        nl, cn = C.c_int(), C.c_int()
        check(lib().sipg_amg_sizes(self.h, C.byref(nl), C.byref(cn)))
        self.nlevels, self.coarse_n = nl.value, cn.value

    @classmethod
    def p0(cls, K, Nf, sJ, tau, nbr, bc_dirichlet, coarse_max=1000, strength=0.08, singular=False):
        """Element-wise constant coarse space (penalty graph Laplacian)."""
        sJ = np.ascontiguousarray(sJ, dtype=np.float64)
        tau = np.ascontiguousarray(tau, dtype=np.float64)
        nbr = np.ascontiguousarray(nbr, dtype=np.int32)
        bd = np.ascontiguousarray(bc_dirichlet, dtype=np.int32)
        h = C.c_void_p()
        check(lib().sipg_amg_build(K, Nf, _dp(sJ), _dp(tau), _ip(nbr), len(bd), _ip(bd), coarse_max,
                                   C.c_double(strength), int(singular), C.byref(h)))
        return cls(h)

    @classmethod
    def p1(cls, mesh, factor1, tau1, bc_dirichlet, mm_mode=0, mm_scalar=0.0, mm1=None, coarse_max=1000,
           strength=0.08, singular=False):
        """Continuous piecewise-linear coarse space (Galerkin of the p=1 operator)."""
        f = None if factor1 is None else np.ascontiguousarray(factor1, dtype=np.float64)
        t = np.ascontiguousarray(tau1, dtype=np.float64)
        bd = np.ascontiguousarray(bc_dirichlet, dtype=np.int32)
        m = None if mm1 is None else np.ascontiguousarray(mm1, dtype=np.float64)
        h = C.c_void_p()
        check(lib().sipg_amg_build_p1(mesh.h, _dp(f), _dp(t), _ip(bd), mm_mode, C.c_double(mm_scalar), _dp(m),
                                      coarse_max, C.c_double(strength), int(singular), C.byref(h)))
        return cls(h)

    def csr(self, level, which):
        """(rows, cols, ptr, idx, val) of A (0), P (1) or R (2) at a level."""
        r, c, z = C.c_int(), C.c_int(), C.c_int()
        check(lib().sipg_amg_level(self.h, level, which, C.byref(r), C.byref(c), C.byref(z), None, None, None))
        ptr = np.zeros(r.value + 1, np.int32)
        idx = np.zeros(z.value, np.int32)
        val = np.zeros(z.value)
        check(lib().sipg_amg_level(self.h, level, which, None, None, None, _ip(ptr), _ip(idx), _dp(val)))
        return r.value, c.value, ptr, idx, val

    def coarse_inverse(self):
        inv = np.zeros((self.coarse_n, self.coarse_n))
        check(lib().sipg_amg_coarse_inverse(self.h, _dp(inv)))
        return inv

    def __del__(self):
        if getattr(self, "h", None) and self.h:
            lib().sipg_amg_destroy(self.h)
            self.h = None


class ServerOpts(C.Structure):
    _fields_ = [("slots", C.c_int), ("hbm_budget_bytes", C.c_size_t)]


class RequestResult(C.Structure):
    _fields_ = [("status", C.c_int), ("info", SolveInfo), ("queue_ms", C.c_double), ("run_ms", C.c_double),
                ("total_ms", C.c_double), ("error", C.c_char * 160)]


class Server:
    """Serving loop: concurrent solves of independent requests (sipg_server_*)."""

    def __init__(self, slots=2, hbm_budget_bytes=0):
        self.h = C.c_void_p()
        o = ServerOpts(slots, hbm_budget_bytes)
        check(lib().sipg_server_create(C.byref(o), C.byref(self.h)))
        self._pending = {}

    def submit(self, op, kind, opts, b, x0=None):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b) if x0 is None else np.ascontiguousarray(x0, dtype=np.float64).copy()
        rid = C.c_longlong()
        check(lib().sipg_server_submit(self.h, op.h, kind, C.byref(opts) if opts is not None else None,
                                       _dp(b), _dp(x), C.byref(rid)))
        self._pending[rid.value] = (op, x)
        return rid.value

    def wait(self, rid):
        res = RequestResult()
        check(lib().sipg_server_wait(self.h, C.c_longlong(rid), C.byref(res)))
        op, x = self._pending.pop(rid)
        return x, res

    def poll(self, rid):
        res = RequestResult()
        done = C.c_int()
        check(lib().sipg_server_poll(self.h, C.c_longlong(rid), C.byref(done), C.byref(res)))
        if not done.value:
            return None
        op, x = self._pending.pop(rid)
        return x, res

    def cancel(self, rid):
        check(lib().sipg_server_cancel(self.h, C.c_longlong(rid)))

    def stats(self):
        a, q, r = C.c_int(), C.c_int(), C.c_int()
        b = C.c_size_t()
        check(lib().sipg_server_stats(self.h, C.byref(a), C.byref(b), C.byref(q), C.byref(r)))
        return {"resident": a.value, "resident_bytes": b.value, "queued": q.value, "running": r.value}

    def close(self):
        if getattr(self, "h", None) and self.h:
            lib().sipg_server_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def default_opts(kind):
    o = SolverOpts()
    check(lib().sipg_solver_default_opts(kind, C.byref(o)))
    return o


class Solver:
    """Linear solver (LinearSolver / ViscousSolver3D stand-in)."""

    def __init__(self, op, kind, opts=None):
        self.op = op
        self.kind = kind
        self.opts = opts if opts is not None else default_opts(kind)
        self.h = C.c_void_p()
        check(lib().sipg_solver_create(op.h, kind, C.byref(self.opts), C.byref(self.h)))

    def setup(self):
        check(lib().sipg_solver_setup(self.h))

    def solve_host(self, b, x0=None):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b) if x0 is None else np.ascontiguousarray(x0, dtype=np.float64).copy()
        info = SolveInfo()
        st = lib().sipg_solver_solve_host(self.h, _dp(b), _dp(x), C.byref(info))
        if st not in (SIPG_OK, SIPG_NOT_CONVERGED, SIPG_BREAKDOWN):
            check(st)
        return x, info

    def solve_device(self, b_ptr, x_ptr):
        info = SolveInfo()
        st = lib().sipg_solver_solve(self.h, C.c_void_p(b_ptr), C.c_void_p(x_ptr), C.byref(info))
        if st not in (SIPG_OK, SIPG_NOT_CONVERGED, SIPG_BREAKDOWN):
            check(st)
        return info

    def __del__(self):
        if getattr(self, "h", None) and self.h:
            lib().sipg_solver_destroy(self.h)
            self.h = None
