"""ctypes wrapper of the CPU checkers. TEST INFRASTRUCTURE ONLY.

Loads oracle/liboracle.so (the plain-C restatement) and, when it has been
built, oracle/_ref/libsipgref.so (the reference's own kernels driven by
ref_harness.cpp). Only tests, the smoke check and the CPU-baseline leg of the
benchmark use this module.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libsipgref.so")

VMF_FLUX_BUG = 1
REF_BLOCK_DIAG = 2
PRE_NONE, PRE_INV_MASS, PRE_FACTOR_INV_MASS, PRE_JACOBI, PRE_BLOCK_JACOBI, PRE_PMG = range(6)

DP = C.POINTER(C.c_double)
IP = C.POINTER(C.c_int)


class OracleMesh(C.Structure):
    _fields_ = [("dim", C.c_int), ("order", C.c_int), ("Np", C.c_int), ("Nfp", C.c_int),
                ("Nf", C.c_int), ("K", C.c_int), ("F", C.c_int), ("Kb", C.c_int),
                ("Dr", DP), ("Ds", DP), ("Dt", DP), ("M", DP), ("MMF", DP), ("EMAT", DP),
                ("fmask", IP), ("geof", DP), ("nx", DP), ("ny", DP), ("nz", DP), ("sJ", DP),
                ("fscale", DP), ("face2cells", IP), ("faceNum", IP), ("fmaskL", IP),
                ("fmaskR", IP), ("bface2cell", IP), ("bfaceNum", IP)]


class SolveInfo(C.Structure):
    _fields_ = [("iters", C.c_int), ("abs_res", C.c_double), ("rel_res", C.c_double),
                ("converged", C.c_int), ("setup_s", C.c_double), ("solve_s", C.c_double),
                ("iter_s", C.c_double)]


class OracleCsr(C.Structure):
    _fields_ = [("rows", C.c_int), ("cols", C.c_int), ("ptr", IP), ("idx", IP), ("val", DP)]


class SolverOpts(C.Structure):
    _fields_ = [("ncomp", C.c_int), ("bc_types", IP), ("factor", DP), ("mm_factor", DP),
                ("mm_scalar", C.c_double), ("flags", C.c_int), ("precond", C.c_int),
                ("inv_mass_factor", C.c_double), ("abs_tol", C.c_double), ("rel_tol", C.c_double),
                ("max_iter", C.c_int), ("pin_dof", C.c_int), ("nullspace", C.c_int),
                ("pmg_nlevels", C.c_int), ("pmg_orders", IP), ("pmg_meshes", C.c_void_p),
                ("pmg_factors", C.POINTER(DP)), ("pmg_prolong", C.POINTER(DP)),
                ("cheb_order", C.c_int), ("eig_safety", C.c_double), ("eig_ratio", C.c_double),
                ("eig_iters", C.c_int), ("coarse_iters", C.c_int), ("coarse_kind", C.c_int),
                ("amg_nlevels", C.c_int), ("amg_A", C.POINTER(OracleCsr)), ("amg_P", C.POINTER(OracleCsr)),
                ("amg_R", C.POINTER(OracleCsr)), ("amg_Pdg", C.POINTER(OracleCsr)),
                ("amg_Rdg", C.POINTER(OracleCsr)), ("amg_coarse_inv", DP), ("amg_coarse_n", C.c_int),
                ("smoother", C.c_int), ("amg_cheb_order", C.c_int), ("mult", C.c_void_p),
                ("outer_mult", C.c_void_p)]


_libs = {}


def _load(path):
    if path not in _libs:
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run `make -C oracle`")
        _libs[path] = C.CDLL(path)
    return _libs[path]


def oracle_lib():
    return _load(ORACLE_SO)


def ref_lib():
    return _load(REF_SO)


def have_ref():
    return os.path.exists(REF_SO)


def _d(a):
    return a.ctypes.data_as(DP) if a is not None else None


def _i(a):
    return a.ctypes.data_as(IP) if a is not None else None


class OMesh:
    """Holds the arrays an OracleMesh points to (keeps them alive)."""

    def __init__(self, tables, export):
        self.keep = []

        def d(a):
            a = np.ascontiguousarray(a, dtype=np.float64)
            self.keep.append(a)
            return _d(a)

        def i(a):
            a = np.ascontiguousarray(a, dtype=np.int32)
            self.keep.append(a)
            return _i(a)

        t, e = tables, export
        self.s = OracleMesh(t["dim"], t["order"], t["Np"], t["Nfp"], t["Nf"], e["K"], e["F"], e["Kb"],
                            d(t["Dr"]), d(t["Ds"]), d(t["Dt"]), d(t["M"]), d(t["MMF"]), d(t["EMAT"]),
                            i(t["fmask"]), d(e["geof"]), d(e["nx"]), d(e["ny"]), d(e["nz"]), d(e["sJ"]),
                            d(e["fscale"]), i(e["face2cells"]), i(e["faceNum"]), i(e["fmaskL"]),
                            i(e["fmaskR"]), i(e["bface2cell"]), i(e["bfaceNum"]))
        self.K, self.Np, self.Nfp, self.Kb, self.dim = e["K"], t["Np"], t["Nfp"], e["Kb"], t["dim"]


def _comp_ptrs(arr, ncomp, K, Np):
    arr = arr.reshape(ncomp, K, Np)
    ptrs = (DP * ncomp)(*[arr[c].ctypes.data_as(DP) for c in range(ncomp)])
    return ptrs


def mult(om, x, bc_types, factor=None, mm=None, mm_scalar=0.0, flags=0, use_ref=False):
    ncomp = x.shape[0]
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros_like(x)
    bct = np.ascontiguousarray(bc_types, dtype=np.int32).reshape(-1)
    f = None if factor is None else np.ascontiguousarray(factor, dtype=np.float64)
    m = None if mm is None else np.ascontiguousarray(mm, dtype=np.float64)
    xp = _comp_ptrs(x, ncomp, om.K, om.Np)
    yp = _comp_ptrs(y, ncomp, om.K, om.Np)
    if use_ref:
        st = ref_lib().ref_mult(C.byref(om.s), ncomp, _i(bct), _d(f), _d(m), C.c_double(mm_scalar),
                                flags, xp, yp)
        assert st == 0, "reference build lacks this dim/order"
    else:
        oracle_lib().oracle_mult(C.byref(om.s), ncomp, _i(bct), _d(f), _d(m), C.c_double(mm_scalar),
                                 flags, xp, yp)
    return y


def apply_bc(om, bc, rhs, bc_types, factor=None, use_ref=False):
    ncomp = rhs.shape[0]
    out = np.ascontiguousarray(rhs, dtype=np.float64).copy()
    bc = np.ascontiguousarray(bc, dtype=np.float64)
    bct = np.ascontiguousarray(bc_types, dtype=np.int32).reshape(-1)
    f = None if factor is None else np.ascontiguousarray(factor, dtype=np.float64)
    bp = (DP * ncomp)(*[bc[c].ctypes.data_as(DP) for c in range(ncomp)])
    rp = _comp_ptrs(out, ncomp, om.K, om.Np)
    if use_ref:
        assert ref_lib().ref_apply_bc(C.byref(om.s), ncomp, _i(bct), _d(f), bp, rp) == 0
    else:
        oracle_lib().oracle_apply_bc(C.byref(om.s), ncomp, _i(bct), _d(f), bp, rp)
    return out


def diag(om, ncomp, bc_types, factor=None, mm=None, mm_scalar=0.0, use_ref=False):
    out = np.zeros((ncomp, om.K, om.Np))
    bct = np.ascontiguousarray(bc_types, dtype=np.int32).reshape(-1)
    f = None if factor is None else np.ascontiguousarray(factor, dtype=np.float64)
    m = None if mm is None else np.ascontiguousarray(mm, dtype=np.float64)
    if use_ref:
        assert ref_lib().ref_diag(C.byref(om.s), ncomp, _i(bct), _d(f), _d(m), C.c_double(mm_scalar), _d(out)) == 0
    else:
        oracle_lib().oracle_diag(C.byref(om.s), ncomp, _i(bct), _d(f), _d(m), C.c_double(mm_scalar), _d(out))
    return out


def block_diag(om, ncomp, bc_types, factor=None, mm=None, mm_scalar=0.0, flags=0, inv=False,
               use_ref=False):
    out = np.zeros((ncomp, om.K, om.Np, om.Np))
    bct = np.ascontiguousarray(bc_types, dtype=np.int32).reshape(-1)
    f = None if factor is None else np.ascontiguousarray(factor, dtype=np.float64)
    m = None if mm is None else np.ascontiguousarray(mm, dtype=np.float64)
    if use_ref:
        assert ref_lib().ref_block_diag(C.byref(om.s), ncomp, _i(bct), _d(f), _d(m),
                                        C.c_double(mm_scalar), int(inv), _d(out)) == 0
    else:
        oracle_lib().oracle_block_diag(C.byref(om.s), ncomp, _i(bct), _d(f), _d(m),
                                       C.c_double(mm_scalar), flags, int(inv), _d(out))
    return out


def solve(om, b, bc_types, precond=PRE_NONE, factor=None, mm=None, mm_scalar=0.0, flags=0,
          abs_tol=1e-9, rel_tol=1e-8, max_iter=500, inv_mass_factor=1.0, pin_dof=-1, nullspace=0,
          x0=None, pmg=None, use_ref=False, ref_applies=False, outer_mult=None):
    """Solve with the oracle (or the reference-kernel harness). pmg: dict with
    orders, meshes (OMesh per level), factors, prolong, cheb_order, eig_safety,
    eig_ratio, eig_iters, coarse_iters, smoother (0 Jacobi, 1 element-block
    Jacobi), amg_cheb_order and amg (a hierarchy with the csr / coarse_inverse
    accessors). ref_applies: the oracle's solver with every operator apply
    done by the reference's own kernels (oracle/_ref ref_mult). outer_mult: an
    oracle_mult_fn (ctypes function) for the outer operator alone."""
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros_like(b) if x0 is None else np.ascontiguousarray(x0, dtype=np.float64).copy()
    bct = np.ascontiguousarray(bc_types, dtype=np.int32).reshape(-1)
    f = None if factor is None else np.ascontiguousarray(factor, dtype=np.float64)
    m = None if mm is None else np.ascontiguousarray(mm, dtype=np.float64)
    o = SolverOpts()
    o.ncomp = b.shape[0]
    o.bc_types = _i(bct)
    o.factor = _d(f)
    o.mm_factor = _d(m)
    o.mm_scalar = mm_scalar
    o.flags = flags
    o.precond = precond
    o.inv_mass_factor = inv_mass_factor
    o.abs_tol = abs_tol
    o.rel_tol = rel_tol
    o.max_iter = max_iter
    o.pin_dof = pin_dof
    o.nullspace = nullspace
    keep = []
    if pmg is not None:
        nl = len(pmg["orders"])
        orders = np.array(pmg["orders"], dtype=np.int32)
        meshes = (OracleMesh * nl)(*[mm_.s for mm_ in pmg["meshes"]])
        facs = [None if fa is None else np.ascontiguousarray(fa, dtype=np.float64) for fa in pmg["factors"]]
        fptr = (DP * nl)(*[_d(fa) if fa is not None else None for fa in facs])
        prol = [np.ascontiguousarray(P, dtype=np.float64) for P in pmg["prolong"]]
        pptr = (DP * max(1, nl - 1))(*[_d(P) for P in prol])
        keep += [orders, meshes, facs, fptr, prol, pptr]
        o.pmg_nlevels = nl
        o.pmg_orders = _i(orders)
        o.pmg_meshes = C.cast(meshes, C.c_void_p)
        o.pmg_factors = fptr
        o.pmg_prolong = pptr
        o.cheb_order = pmg.get("cheb_order", 4)
        o.eig_safety = pmg.get("eig_safety", 1.1)
        o.eig_ratio = pmg.get("eig_ratio", 30.0)
        o.eig_iters = pmg.get("eig_iters", 20)
        o.coarse_iters = pmg.get("coarse_iters", 20)
        o.smoother = pmg.get("smoother", 0)
        o.amg_cheb_order = pmg.get("amg_cheb_order", 0)
        amg = pmg.get("amg")
        if amg is not None:
            nl = amg.nlevels
            mats = {w: [amg.csr(l, w) for l in range(nl)] for w in (0, 1, 2)}
            arrs = []

            def mk(t):
                rows, cols, ptr, idx, val = t
                arrs.extend([ptr, idx, val])
                return OracleCsr(rows, cols, _i(ptr), _i(idx), _d(val))
            A = (OracleCsr * nl)(*[mk(t) for t in mats[0]])
            P = (OracleCsr * nl)(*[mk(t) for t in mats[1]])
            R = (OracleCsr * nl)(*[mk(t) for t in mats[2]])
            inv = np.ascontiguousarray(amg.coarse_inverse())
            Pdg = (OracleCsr * 1)(mk(amg.csr(-1, 1)))
            Rdg = (OracleCsr * 1)(mk(amg.csr(-1, 2)))
            keep += [arrs, A, P, R, inv, Pdg, Rdg]
            o.amg_Pdg, o.amg_Rdg = Pdg, Rdg
            o.coarse_kind = 1
            o.amg_nlevels = nl
            o.amg_A, o.amg_P, o.amg_R = A, P, R
            o.amg_coarse_inv = _d(inv)
            o.amg_coarse_n = amg.coarse_n
    if ref_applies:
        o.mult = C.cast(ref_lib().ref_mult, C.c_void_p).value
    if outer_mult is not None:
        o.outer_mult = C.cast(outer_mult, C.c_void_p).value
    info = SolveInfo()
    if use_ref:
        assert ref_lib().ref_solve(C.byref(om.s), C.byref(o), _d(b), _d(x), C.byref(info)) == 0
    else:
        oracle_lib().oracle_solve(C.byref(om.s), C.byref(o), _d(b), _d(x), C.byref(info))
    return x, info


def proj_h(om):
    """Per-element penalty length of the velocity projection (K values)."""
    h = np.zeros(om.K)
    oracle_lib().oracle_proj_h(C.byref(om.s), _d(h))
    return h


def project_velocity(om, dt, factor, dp, velT, use_ref=False):
    """Element-local velocity projection (pr_projection_method == 1).

    dp, velT: (dim, K, Np). Returns (velTT, stats) with stats = (cells,
    converged cells, iterations summed over cells)."""
    dp = np.ascontiguousarray(dp, dtype=np.float64)
    velT = np.ascontiguousarray(velT, dtype=np.float64)
    out = np.zeros_like(velT)
    st = np.zeros(3)
    args = (C.byref(om.s), C.c_double(dt), C.c_double(factor), _d(dp), _d(velT), _d(out), _d(st))
    if use_ref:
        assert ref_lib().ref_project_velocity(*args) == 0
    else:
        oracle_lib().oracle_project_velocity(*args)
    return out, st


def grad_central(om, p):
    """Central-flux DG gradient (dim, K, Np) of the nodal field p (K, Np)."""
    p = np.ascontiguousarray(p, dtype=np.float64)
    g = np.zeros((om.dim, om.K, om.Np))
    oracle_lib().oracle_grad_central(C.byref(om.s), _d(p), _d(g))
    return g


def pressure_rhs(om, dt, velT, dPdN=None, dPdN_old=None, b0=1.0, b1=0.0):
    """J M (-div_c(velT) / dt + LIFT (b0 dPdN + b1 dPdN_old)); returns (rhs, dPdN_old updated)."""
    velT = np.ascontiguousarray(velT, dtype=np.float64)
    dn = None if dPdN is None else np.ascontiguousarray(dPdN, dtype=np.float64)
    do = None if dPdN_old is None else np.array(dPdN_old, dtype=np.float64, order="C", copy=True)
    rhs = np.zeros((om.K, om.Np))
    oracle_lib().oracle_pressure_rhs(C.byref(om.s), C.c_double(dt), C.c_double(b0), C.c_double(b1), _d(velT),
                                     _d(dn), _d(do), _d(rhs))
    return rhs, do
