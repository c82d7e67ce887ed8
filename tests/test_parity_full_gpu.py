"""GPU results against the oracle at the benchmark configurations' full sizes,
and for the p-multigrid configuration the benchmark times.

* The configuration the benchmark solves (the library's defaults: element-block
  Jacobi Chebyshev(4) smoothing, FP16/assembled low-order levels in the FP32
  V-cycle, a continuous-P1 smoothed-aggregation coarse space with Chebyshev(2))
  is compared with the oracle's p-multigrid, whose coarse hierarchy, meshes and
  reference element come from oracle/ alone (amg_oracle, dg_oracle).
* Applies at full size against the reference's own kernels (oracle/_ref):
  the two-phase Poisson operator at 24^3 x 6 = 82,944 tets, p = 3, and the
  Helmholtz operator I/(nu dt) - Laplacian at 48^3 x 6 = 663,552 tets, p = 4.
* The two-phase Poisson solve at 24^3 x 6 in FP64 (solution within 1e-9 of the
  oracle's, iterations +-1) and in mixed precision (iterations +-1 of the
  oracle's FP64 solve, true relative residual <= 1e-8, error against the oracle
  stated), and the committed FP32 copy of the oracle solution that the
  benchmark reports its error against.
"""
import os

import numpy as np
import pytest

import dg_oracle as D
import oracle_py as O
import pmg_oracle as P
import sipg
import workloads as W
from helpers import TOL_FP64, DevArray, rel_err

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
C2_FIXTURE = os.path.join(HERE, "golden", "c2", "c2_oracle_solution.npz")

# Measured error of the TF32 tensor-core apply (FP32 data, 10-bit operand
# mantissa, FP32 accumulation) against the reference's FP64 kernels, relative
# max-norm: the bound below is about twice the figure measured on a B200.
TF32_C2_BOUND = 2e-3
TF32_C3_BOUND = 1e-3
# Mixed-precision solution against the FP64 oracle solution (relative L2).
MIXED_C2_BOUND = 1e-5


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def gpu_solver(case, precision, pin):
    op = sipg.Operator(case["mesh"], case["tables"]["order"], 1)
    op.set_bc_types(case["bc_types"])
    op.set_factor(case["factor"])
    if pin:
        op.set_pin(*case["pin"])
    o = sipg.default_opts(sipg.SOLVER_PMULTIGRID)
    o.precision, o.rel_tol, o.abs_tol, o.max_iter = precision, 1e-8, 0.0, 500
    o.nullspace = 0 if pin else 1
    return op, sipg.Solver(op, sipg.SOLVER_PMULTIGRID, o)


def fp32_apply(op, x):
    xd = DevArray(x.astype(np.float32))
    yd = DevArray(np.zeros_like(x, dtype=np.float32))
    op.apply_device(sipg.FP32, xd.p, yd.p)
    return yd.get().astype(np.float64)


# ------------------------------------------------ the timed configuration, small
@pytest.mark.parametrize("pin", [True, False], ids=["pinned", "nullspace"])
def test_default_pmultigrid_fp64_matches_oracle(pin):
    gc = W.poisson3d_two_phase(4, order=3, n_modes=64, pin=pin)
    oc = D.poisson3d_two_phase(4, order=3, n_modes=64, pin=pin)
    xo, io, _ = P.solve_poisson(oc)
    assert io.converged
    _, s = gpu_solver(gc, sipg.FP64, pin)
    x, info = s.solve_host(gc["rhs"])
    assert info.status == sipg.SIPG_OK
    assert abs(info.iters - io.iters) <= 1
    assert rel_l2(x, xo) <= 1e-9


@pytest.mark.parametrize("n", [4, 8])
def test_default_pmultigrid_mixed_against_oracle(n):
    gc = W.poisson3d_two_phase(n, order=3, n_modes=64, pin=False)
    oc = D.poisson3d_two_phase(n, order=3, n_modes=64, pin=False)
    xo, io, _ = P.solve_poisson(oc)
    _, s = gpu_solver(gc, sipg.FP32, False)
    x, info = s.solve_host(gc["rhs"])
    assert info.status == sipg.SIPG_OK
    assert abs(info.iters - io.iters) <= 1
    assert info.true_rel_res <= 1e-8
    err = rel_l2(x, xo)
    print(f"mixed p-MG at {n}^3 x 6: {info.iters} iterations (oracle FP64 {io.iters}), "
          f"relative L2 error against the FP64 oracle {err:.2e}")
    assert err <= MIXED_C2_BOUND


# ------------------------------------------- the next time step: set-up again
def moved_factor(case, n, shift):
    """1 / rho of the two-phase case with the heavy sphere moved by (shift, 0, -shift)."""
    e = case["export"]
    return 1.0 / D.two_phase_rho(e["x"], e["y"], e["z"], 1.0 / n, center=(0.5 + shift, 0.5, 0.5 - shift))


@pytest.mark.parametrize("precision", [sipg.FP64, sipg.FP32], ids=["fp64", "mixed"])
def test_second_time_step_reuses_interpolation_like_the_oracle(precision):
    """A solve, then the density moves and the solver is set up again (the
    reference's per-step reset before the pressure solve). The library keeps the
    first set-up's aggregates and prolongators and recomputes the level operators,
    smoother data and coarsest inverse on the device; the oracle's hierarchy does
    the same from its own first set-up (Hierarchy.reuse). A coarse limit of 40
    unknowns gives three algebraic levels at 6^3 x 6."""
    n, cmax, shift = 6, 40, 0.08
    gc = W.poisson3d_two_phase(n, order=3, n_modes=64, pin=False)
    oc = D.poisson3d_two_phase(n, order=3, n_modes=64, pin=False)
    _, io1, pmg1 = P.solve_poisson(oc, amg_coarse_max=cmax)
    assert pmg1["amg"].nlevels >= 3
    oc2 = dict(oc, factor=moved_factor(oc, n, shift))
    xo, io, _ = P.solve_poisson(oc2, reuse=pmg1, amg_coarse_max=cmax)
    assert io1.converged and io.converged
    op = sipg.Operator(gc["mesh"], 3, 1)
    op.set_bc_types(gc["bc_types"])
    op.set_factor(gc["factor"])
    o = sipg.default_opts(sipg.SOLVER_PMULTIGRID)
    o.precision, o.rel_tol, o.abs_tol, o.max_iter, o.nullspace = precision, 1e-8, 0.0, 500, 1
    o.amg_coarse_max = cmax
    s = sipg.Solver(op, sipg.SOLVER_PMULTIGRID, o)
    _, i1 = s.solve_host(gc["rhs"])
    assert i1.status == sipg.SIPG_OK and abs(i1.iters - io1.iters) <= 1
    op.set_factor(moved_factor(gc, n, shift))
    s.setup()
    x, info = s.solve_host(gc["rhs"])
    assert info.status == sipg.SIPG_OK
    assert abs(info.iters - io.iters) <= 1
    assert info.true_rel_res <= 1e-8
    assert rel_l2(x, xo) <= (1e-9 if precision == sipg.FP64 else MIXED_C2_BOUND)


def test_set_up_without_reuse_equals_a_fresh_solver():
    """amg_reuse_interpolation = 0 aggregates again at every set-up: a solver set
    up a second time on a new factor gives the iterates of a solver created on it."""
    n, shift = 6, 0.08
    gc = W.poisson3d_two_phase(n, order=3, n_modes=64, pin=False)
    f2 = moved_factor(gc, n, shift)
    res = []
    for fresh in (False, True):
        op = sipg.Operator(gc["mesh"], 3, 1)
        op.set_bc_types(gc["bc_types"])
        op.set_factor(f2 if fresh else gc["factor"])
        o = sipg.default_opts(sipg.SOLVER_PMULTIGRID)
        o.precision, o.rel_tol, o.abs_tol, o.max_iter, o.nullspace = sipg.FP64, 1e-8, 0.0, 500, 1
        o.amg_coarse_max, o.amg_reuse_interpolation = 40, 0
        s = sipg.Solver(op, sipg.SOLVER_PMULTIGRID, o)
        if not fresh:
            s.solve_host(gc["rhs"])
            op.set_factor(f2)
            s.setup()
        res.append(s.solve_host(gc["rhs"]))
    (xa, ia), (xb, ib) = res
    assert ia.iters == ib.iters and np.array_equal(xa, xb)


# ------------------------------------------------------- full-size applies
@pytest.fixture(scope="module")
def c2():
    c = W.poisson3d_two_phase(24, order=3, n_modes=256, pin=False)
    op = sipg.Operator(c["mesh"], 3, 1)
    op.set_bc_types(c["bc_types"])
    op.set_factor(c["factor"])
    return c, op, O.OMesh(c["tables"], c["export"])


def test_c2_fp64_apply_matches_reference_kernels(c2):
    c, op, om = c2
    x = np.random.default_rng(21).uniform(-1.0, 1.0, (1, c["mesh"].K, op.Np))
    want = O.mult(om, x, c["bc_types"], c["factor"], use_ref=True)
    assert rel_err(op.apply_host(x), want) < TOL_FP64


def test_c2_tf32_apply_error_against_reference_kernels(c2):
    c, op, om = c2
    x = np.random.default_rng(22).uniform(-1.0, 1.0, (1, c["mesh"].K, op.Np))
    want = O.mult(om, x, c["bc_types"], c["factor"], use_ref=True)
    err = rel_err(fp32_apply(op, x), want)
    print(f"TF32 apply at 24^3 x 6, p = 3: relative max-norm error {err:.2e} (L2 {rel_l2(fp32_apply(op, x), want):.2e})")
    assert err < TF32_C2_BOUND


@pytest.fixture(scope="module")
def c3():
    h = W.helmholtz3d(48, order=4)
    op = sipg.Operator(h["mesh"], 4, 1)
    op.set_bc_types(h["bc_types"])
    op.set_mm(sipg.MM_SCALAR, h["mm"])
    om = O.OMesh(sipg.ref_tables(3, 4), h["mesh"].export(4))
    want = O.mult(om, h["x"], h["bc_types"], None, None, h["mm"], use_ref=True)
    return h, op, want


def test_c3_helmholtz_fp64_apply_matches_reference_kernels(c3):
    h, op, want = c3
    assert rel_err(op.apply_host(h["x"]), want) < TOL_FP64


def test_c3_helmholtz_tf32_apply_error_against_reference_kernels(c3):
    h, op, want = c3
    got = fp32_apply(op, h["x"])
    err = rel_err(got, want)
    print(f"TF32 apply at 48^3 x 6, p = 4 Helmholtz: relative max-norm error {err:.2e} (L2 {rel_l2(got, want):.2e})")
    assert err < TF32_C3_BOUND


# ---------------------------------------------------------- full-size solves
@pytest.fixture(scope="module")
def c2_oracle():
    oc = D.poisson3d_two_phase(24, order=3, n_modes=256, pin=False)
    xo, io, _ = P.solve_poisson(oc)
    assert io.converged
    return xo, io


def test_c2_fp64_pmultigrid_matches_oracle(c2, c2_oracle):
    c, op, _ = c2
    xo, io = c2_oracle
    _, s = gpu_solver(c, sipg.FP64, False)
    x, info = s.solve_host(c["rhs"])
    assert info.status == sipg.SIPG_OK
    assert abs(info.iters - io.iters) <= 1
    assert rel_l2(x, xo) <= 1e-9


def test_c2_mixed_pmultigrid_against_oracle(c2, c2_oracle):
    c, op, _ = c2
    xo, io = c2_oracle
    _, s = gpu_solver(c, sipg.FP32, False)
    x, info = s.solve_host(c["rhs"])
    assert info.status == sipg.SIPG_OK
    assert abs(info.iters - io.iters) <= 1
    assert info.true_rel_res <= 1e-8
    err = rel_l2(x, xo)
    print(f"mixed p-MG at 24^3 x 6: {info.iters} iterations (oracle FP64 {io.iters}), true relative residual "
          f"{info.true_rel_res:.2e}, relative L2 error against the FP64 oracle {err:.2e}")
    assert err <= MIXED_C2_BOUND


def test_c2_committed_fixture_is_the_oracle_solution(c2_oracle):
    xo, io = c2_oracle
    g = np.load(C2_FIXTURE)
    assert int(g["iters"]) == io.iters
    assert rel_l2(g["x"].astype(np.float64), xo) < 1e-7
    assert abs(float(g["x_sum"]) - float(xo.sum())) <= 1e-9 * float(np.abs(xo).sum())
