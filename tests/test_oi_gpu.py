"""The over-integrated factor operator (sipg_op_set_factor_oi) against its oracle
(oracle/oi_oracle.py): cubature points, applies (2D/3D, orders 1-4, interior,
Dirichlet and Neumann faces, a two-phase factor sampled at the points, a pinned
DOF), the nodal operator for a constant factor, symmetry, and the FP64 and mixed
p-multigrid solves against the oracle's FPCG on the same operator (the V-cycle on
the nodal projection of the factor in both)."""
import numpy as np
import pytest

import dg_oracle as D
import oi_oracle as OI
import oracle_py as O
import pmg_oracle as P
import sipg
import workloads as W
from helpers import rel_err

pytestmark = pytest.mark.gpu


def two_phase_at(xyz, n, ratio=1000.0, shift=0.0):
    z = xyz[2] if xyz.shape[0] == 3 else np.full_like(xyz[0], 0.5)
    return 1.0 / D.two_phase_rho(xyz[0], xyz[1], z, 1.0 / n, ratio=ratio,
                                 center=(0.5 + shift, 0.5, 0.5 - shift))


def bct_of(Kb, kind):
    if kind == 2:
        return (np.arange(Kb) % 2).astype(np.int32)[None]
    return np.full((1, Kb), kind, np.int32)


CASES = [(3, 3, 1, 1), (3, 3, 2, 0), (3, 3, 3, 2), (3, 4, 3, 1), (3, 2, 4, 2), (2, 6, 2, 0), (2, 6, 3, 2),
         (2, 5, 4, 1)]


def setup_case(dim, n, p, bnd, pin=False):
    gm = sipg.Mesh.box(dim, n, jitter=0.1, seed=3)
    om = D.Mesh.box(dim, n, 0.1, 3)
    op = sipg.Operator(gm, p, 1)
    bct = bct_of(gm.Kb, bnd)
    op.set_bc_types(bct)
    xv, xs = op.oi_points()
    fv, fs = two_phase_at(xv, n), two_phase_at(xs, n)
    if pin:
        op.set_pin(3, 1)
    op.set_factor_oi(fv, fs)
    return gm, om, op, bct, fv, fs


@pytest.mark.parametrize("dim,n,p,bnd", CASES)
def test_points_and_apply_match_the_oracle(dim, n, p, bnd):
    gm, om, op, bct, fv, fs = setup_case(dim, n, p, bnd)
    xv, xs = op.oi_points()
    ov, os_ = OI.points(om, p)
    assert np.abs(xv - ov).max() < 1e-12 and np.abs(xs - os_).max() < 1e-12
    x = np.random.default_rng(11).uniform(-1.0, 1.0, (gm.K, op.Np))
    want = OI.apply(om, p, x, fv, fs, bct)
    assert rel_err(op.apply_host(x[None])[0], want) < 1e-12


@pytest.mark.parametrize("dim,n,p,bnd", [(3, 3, 3, 2), (2, 6, 4, 0)])
def test_constant_factor_gives_the_nodal_operator(dim, n, p, bnd):
    gm = sipg.Mesh.box(dim, n, jitter=0.1, seed=3)
    oi, nodal = sipg.Operator(gm, p, 1), sipg.Operator(gm, p, 1)
    for o in (oi, nodal):
        o.set_bc_types(bct_of(gm.Kb, bnd))
    nq, nqs = oi.oi_sizes()
    oi.set_factor_oi(np.ones((gm.K, nq)), np.ones((gm.K, dim + 1, nqs)))
    x = np.random.default_rng(5).uniform(-1.0, 1.0, (1, gm.K, oi.Np))
    assert rel_err(oi.apply_host(x), nodal.apply_host(x)) < 1e-12
    # back to a nodal factor: the nodal apply again
    oi.set_factor(np.full((gm.K, oi.Np), 2.0))
    assert rel_err(oi.apply_host(x), 2.0 * nodal.apply_host(x)) < 1e-12


def test_operator_is_symmetric_and_pinning_replaces_the_row_and_column():
    gm, om, op, bct, fv, fs = setup_case(3, 3, 3, 1, pin=True)
    rng = np.random.default_rng(2)
    u, v = rng.uniform(-1.0, 1.0, (2, 1, gm.K, op.Np))
    Au, Av = op.apply_host(u), op.apply_host(v)
    assert abs(np.sum(v * Au) - np.sum(u * Av)) < 1e-12 * abs(np.sum(u * Au))
    # pinned DOF (3, 1): other rows see it as zero, its own row keeps the diagonal
    x = u[0].copy()
    want = OI.apply(om, 3, np.where(np.arange(op.Np)[None] == 1, np.where(np.arange(gm.K)[:, None] == 3, 0.0, x), x),
                    fv, fs, bct)
    unit = np.zeros_like(x)
    unit[3, 1] = 1.0
    want[3, 1] = OI.apply(om, 3, unit, fv, fs, bct)[3, 1] * x[3, 1]
    assert rel_err(op.apply_host(x[None])[0], want) < 1e-12


def oi_case(n, ratio=1000.0, shift=0.0):
    """The two-phase Poisson problem of the benchmark (GRF right-hand side, Neumann
    walls, constants projected out) with the factor at the cubature points."""
    gc = W.poisson3d_two_phase(n, order=3, n_modes=64, pin=False)
    oc = D.poisson3d_two_phase(n, order=3, n_modes=64, pin=False)
    op = sipg.Operator(gc["mesh"], 3, 1)
    op.set_bc_types(gc["bc_types"])
    xv, xs = op.oi_points()
    fv, fs = two_phase_at(xv, n, ratio, shift), two_phase_at(xs, n, ratio, shift)
    op.set_factor_oi(fv, fs)
    proj = np.einsum("iq,eq->ei", OI.projection(3, 3), fv)
    return gc, dict(oc, factor=proj), op, fv, fs


@pytest.mark.parametrize("precision", [sipg.FP64, sipg.FP32], ids=["fp64", "mixed"])
def test_pmultigrid_solve_on_the_over_integrated_operator_matches_the_oracle(precision):
    n = 4
    gc, oc, op, fv, fs = oi_case(n)
    cb = OI.outer_mult(oc["mesh"], 3, fv, fs, oc["bc_types"])
    xo, io, _ = P.solve_poisson(oc, outer_mult=cb)
    assert io.converged
    o = sipg.default_opts(sipg.SOLVER_PMULTIGRID)
    o.precision, o.rel_tol, o.abs_tol, o.max_iter, o.nullspace = precision, 1e-8, 0.0, 500, 1
    s = sipg.Solver(op, sipg.SOLVER_PMULTIGRID, o)
    x, info = s.solve_host(gc["rhs"])
    assert info.status == sipg.SIPG_OK
    assert abs(info.iters - io.iters) <= 1
    assert info.true_rel_res <= 1e-8
    err = float(np.linalg.norm(x - xo) / np.linalg.norm(xo))
    assert err <= (1e-9 if precision == sipg.FP64 else 1e-5)
    # the true residual is the over-integrated operator's
    r = gc["rhs"] - OI.apply(oc["mesh"], 3, x.reshape(-1, op.Np), fv, fs, oc["bc_types"]).reshape(gc["rhs"].shape)
    assert np.linalg.norm(r - r.mean()) <= 2e-8 * np.linalg.norm(gc["rhs"])


def test_new_over_integrated_factor_then_set_up_again():
    """A time step: the density moves, set_factor_oi, set-up again, solve; the
    result equals a fresh solver's on the new factor within the solve tolerance."""
    n = 4
    gc, oc, op, fv, fs = oi_case(n)
    o = sipg.default_opts(sipg.SOLVER_PMULTIGRID)
    o.precision, o.rel_tol, o.abs_tol, o.max_iter, o.nullspace = sipg.FP32, 1e-8, 0.0, 500, 1
    s = sipg.Solver(op, sipg.SOLVER_PMULTIGRID, o)
    s.solve_host(gc["rhs"])
    xv, xs = op.oi_points()
    fv2, fs2 = two_phase_at(xv, n, shift=0.08), two_phase_at(xs, n, shift=0.08)
    op.set_factor_oi(fv2, fs2)
    s.setup()
    x, info = s.solve_host(gc["rhs"])
    assert info.status == sipg.SIPG_OK and info.true_rel_res <= 1e-8
    _, _, op2, _, _ = oi_case(n, shift=0.08)
    x2, info2 = sipg.Solver(op2, sipg.SOLVER_PMULTIGRID, o).solve_host(gc["rhs"])
    assert rel_err(x, x2) < 1e-5
