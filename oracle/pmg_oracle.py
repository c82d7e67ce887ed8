"""p-multigrid preconditioned FPCG solves of the oracle, set up from the oracle's
own modules only. TEST INFRASTRUCTURE ONLY (tests/, the smoke check, the CPU
legs of the benchmark).

Everything here comes from oracle/: the reference element and meshes
(dg_oracle), the algebraic coarse hierarchy (amg_oracle) and the C solver
(liboracle.so, oracle_solve); the operator applies are the C restatement or,
with ref_applies=True, the reference's own kernels compiled in oracle/_ref.
The configuration mirrors the reference's [p-multigrid] keys
(examples/3d/oscillating_droplet/config.ini:24-31: orders, cheb_orders,
eigen_val_saftey_factor) with the library's default choices for the rest:
orders 3 -> 2 -> 1, Chebyshev(4) on the element-block Jacobi preconditioned
operator, eigenvalue bound from 20 power iterations x 1.1, lower bound / 30,
one pre- and one post-smoothing sweep, a continuous-P1 smoothed-aggregation
coarse hierarchy to at most 2048 unknowns with Chebyshev(2) smoothing on its levels.
"""
import ctypes as C

import numpy as np

import amg_oracle as A
import dg_oracle as D
import oracle_py as O

DEFAULTS = dict(cheb_order=4, eig_safety=1.1, eig_ratio=30.0, eig_iters=20, coarse_iters=20, smoother=1,
                amg_cheb_order=2, amg_coarse_max=2048, amg_strength=0.08)


def levels(mesh, dim, orders, factor, bc_types, reuse=None, **over):
    """pmg dict for oracle_py.solve: per-order meshes, interpolated factors,
    prolongations, the AMG hierarchy and the smoother settings. reuse: the pmg
    dict of an earlier set-up on the same mesh whose aggregates and prolongators
    the new hierarchy keeps (reuse-interpolation)."""
    cfg = dict(DEFAULTS, **over)
    meshes, facs, prol = [], [], []
    for lv, p in enumerate(orders):
        t = D.ref_tables(dim, p)
        meshes.append(O.OMesh(t, mesh.export(p, t)))
        f = None if factor is None else np.ascontiguousarray(factor @ D.interp_matrix(dim, orders[0], p).T)
        facs.append(f)
        if lv + 1 < len(orders):
            prol.append(D.interp_matrix(dim, orders[lv + 1], p))
    out = dict(orders=list(orders), meshes=meshes, factors=facs, prolong=prol, **cfg)
    if orders[-1] == 1 and cfg.get("coarse_kind", 1) == 1:
        Nf = dim + 1
        tau1 = np.zeros((mesh.K, Nf))
        f1 = facs[-1]
        O.oracle_lib().oracle_tau(C.byref(meshes[-1].s), O._d(f1), O._d(tau1))
        bct = np.asarray(bc_types).reshape(-1)
        bd = (bct == D.BC_DIRICHLET).astype(np.int32)
        t1 = D.ref_tables(dim, 1)
        A0, Pdg = A.p1_continuous_operator(t1, mesh, f1, tau1, bd)
        if reuse is not None:
            out["amg"] = reuse["amg"].reuse(A0)
        else:
            out["amg"] = A.Hierarchy(A0, Pdg, cfg["amg_coarse_max"], cfg["amg_strength"], singular=not bd.any())
    return out


def solve_poisson(case, orders=(3, 2, 1), rel_tol=1e-8, max_iter=200, ref_applies=False, reuse=None,
                  outer_mult=None, **over):
    """FP64 p-multigrid FPCG of a dg_oracle workload (pinned DOF or nullspace
    projection as the case says). reuse: the pmg dict of an earlier solve on the
    same mesh whose algebraic prolongators are kept. outer_mult: the outer
    operator when it is not the nodal one of case["factor"] (the over-integrated
    operator, oi_oracle.outer_mult; the levels keep the nodal factor). Returns
    (x, info, pmg)."""
    mesh, e, t = case["mesh"], case["export"], case["tables"]
    om = O.OMesh(t, e)
    pmg = levels(mesh, e["dim"], orders, case["factor"], case["bc_types"], reuse=reuse, **over)
    pin = case.get("pin")
    pin_dof = -1 if pin is None else pin[0] * t["Np"] + pin[1]
    x, info = O.solve(om, case["rhs"], case["bc_types"], O.PRE_PMG, case["factor"], abs_tol=0.0,
                      rel_tol=rel_tol, max_iter=max_iter, pin_dof=pin_dof, nullspace=0 if pin else 1,
                      pmg=pmg, ref_applies=ref_applies, outer_mult=outer_mult)
    return x, info, pmg
