"""The vector (u, v, w) viscous solve with slip walls against the reference's own
solver: ViscousSolver3D's flexible PCG with the factor inverse-mass and the
Jacobi preconditioners (src/solvers/3d/slip_matrix/viscous_solver.cpp:177-301,
:357-453), driven through the reference's cg3_* and vmf_3d_* kernels in
oracle/_ref (ref_solve) on the same operator (c M + K, slip on every third
boundary face, Dirichlet elsewhere) and right-hand side."""
import numpy as np
import pytest

import oracle_py as O
import sipg
from helpers import make_op, random_case, rel_err

pytestmark = pytest.mark.gpu

KINDS = {"factor_inv_mass": (sipg.SOLVER_INV_MASS, O.PRE_FACTOR_INV_MASS), "jacobi": (sipg.SOLVER_JACOBI, O.PRE_JACOBI)}


@pytest.mark.skipif(not O.have_ref(), reason="oracle/_ref not built")
@pytest.mark.parametrize("order", [2, 3])
@pytest.mark.parametrize("kind", list(KINDS))
def test_slip_viscous_fpcg_matches_the_reference_solver(order, kind):
    c = 50.0  # mass coefficient of the viscous operator (g0 Re / dt in the reference)
    mesh, t, e, om, x, f, m, bct = random_case(3, 3, order, 3, seed=40 + order, slip=True, factor=False)
    b = np.random.default_rng(7).uniform(-1.0, 1.0, x.shape)
    tol = 1e-9 * float(np.linalg.norm(b))
    gpu_kind, ref_kind = KINDS[kind]
    xr, ir = O.solve(om, b, bct, ref_kind, None, None, c, abs_tol=tol, rel_tol=0.0, max_iter=5000,
                     inv_mass_factor=1.0 / c, use_ref=True)
    assert ir.converged
    op = make_op(mesh, order, 3, None, None, mm_scalar=c, bct=bct)
    o = sipg.default_opts(gpu_kind)
    o.abs_tol, o.rel_tol, o.max_iter, o.inv_mass_factor = tol, 0.0, 5000, 1.0 / c
    xg, info = sipg.Solver(op, gpu_kind, o).solve_host(b)
    assert info.status == sipg.SIPG_OK
    assert abs(info.iters - ir.iters) <= 1
    assert rel_err(xg, xr) < 1e-8
