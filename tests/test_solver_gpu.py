"""CUDA solvers against the oracle: CG / Jacobi / block-Jacobi / inverse-mass
PCG (reference golden counts), p-multigrid FP64 and mixed precision."""
import numpy as np
import pytest

import oracle_py as O
import sipg
import workloads as W
from helpers import GOLDEN, golden_setup, load_golden, make_op, rel_err

pytestmark = pytest.mark.gpu

KIND = {"cg": sipg.SOLVER_CG, "jacobi": sipg.SOLVER_JACOBI, "bjacobi": sipg.SOLVER_BLOCK_JACOBI,
        "invmass": sipg.SOLVER_INV_MASS}


@pytest.mark.parametrize("path", [p for p in GOLDEN if "slip" not in p], ids=lambda p: p.split("/")[-1][:-4])
@pytest.mark.parametrize("name", ["cg", "jacobi", "invmass", "bjacobi"])
def test_krylov_matches_reference_golden(path, name):
    g = load_golden(path)
    mesh, t, e, om = golden_setup(g)
    ref_iters = int(g[f"solve_{name}_iters"])
    if name == "bjacobi" and ref_iters > 500:
        pytest.skip("reference block-Jacobi stagnates with its 3D volume block")
    bd = np.zeros_like(g["bct"])
    op = make_op(mesh, g["order"], 1, g.get("factor"), g.get("mm"), mm_scalar=1.0, bct=bd)
    if g.get("mm") is None:
        op.set_mm(sipg.MM_SCALAR, 1.0)
    o = sipg.default_opts(KIND[name])
    o.abs_tol, o.rel_tol, o.max_iter, o.ref_volume_block = 1e-10, 0.0, 2000, 1
    s = sipg.Solver(op, KIND[name], o)
    x, info = s.solve_host(g["solve_b"])
    assert abs(info.iters - ref_iters) <= 1
    assert rel_err(x, g[f"solve_{name}_x"]) < 1e-8


def _pmg_oracle_levels(mesh, orders, factor, bct, amg=True):
    import ctypes as C
    meshes, facs, prol = [], [], []
    for l, p in enumerate(orders):
        t = sipg.ref_tables(3, p)
        meshes.append(O.OMesh(t, mesh.export(p)))
        I = sipg.interp_matrix(3, orders[0], p)
        facs.append(factor @ I.T)
        if l + 1 < len(orders):
            prol.append(sipg.interp_matrix(3, orders[l + 1], p))
    out = dict(orders=orders, meshes=meshes, factors=facs, prolong=prol, cheb_order=4,
               eig_safety=1.1, eig_ratio=30.0, eig_iters=20, coarse_iters=20)
    if amg:
        tau1 = np.zeros((mesh.K, 4))
        f1 = np.ascontiguousarray(facs[-1])
        O.oracle_lib().oracle_tau(C.byref(meshes[-1].s), O._d(f1), O._d(tau1))
        bd = (np.asarray(bct)[0] == sipg.BC_DIRICHLET).astype(np.int32)
        out["amg"] = sipg.Amg.p1(mesh, f1, tau1, bd, coarse_max=2048, strength=0.08, singular=not bd.any())
    return out


@pytest.fixture(scope="module")
def two_phase():
    return W.poisson3d_two_phase(4, order=3, n_modes=64)


def _pmg_solver(case, precision, coarse_kind=1, pin=True):
    op = make_op(case["mesh"], 3, 1, case["factor"], bct=case["bc_types"])
    if pin:
        op.set_pin(*case["pin"])
    o = sipg.default_opts(sipg.SOLVER_PMULTIGRID)
    o.rel_tol, o.abs_tol, o.max_iter, o.precision = 1e-8, 0.0, 200, precision
    o.coarse_kind = coarse_kind
    o.nullspace = 0 if pin else 1
    o.smoother = 0  # the oracle's p-multigrid smooths with point Jacobi
    o.amg_cheb_order = 0  # and uses the order levels' Chebyshev degree on the algebraic levels
    return op, sipg.Solver(op, sipg.SOLVER_PMULTIGRID, o)


@pytest.mark.parametrize("coarse_kind", [0, 1], ids=["coarse_cg", "coarse_amg"])
def test_pmultigrid_fp64_matches_oracle(two_phase, coarse_kind):
    c = two_phase
    om = O.OMesh(c["tables"], c["export"])
    pmg = _pmg_oracle_levels(c["mesh"], [3, 2, 1], c["factor"], c["bc_types"], amg=coarse_kind == 1)
    xo, io = O.solve(om, c["rhs"], c["bc_types"], O.PRE_PMG, c["factor"], abs_tol=0.0, rel_tol=1e-8,
                     max_iter=200, pin_dof=0, pmg=pmg)
    assert io.converged
    op, s = _pmg_solver(c, sipg.FP64, coarse_kind)
    x, info = s.solve_host(c["rhs"])
    assert info.status == sipg.SIPG_OK
    assert abs(info.iters - io.iters) <= 1
    assert rel_err(x, xo) < 1e-9
    assert info.true_rel_res < 1e-8


def test_pmultigrid_nullspace_fp64_matches_oracle(two_phase):
    c = W.poisson3d_two_phase(4, order=3, n_modes=64, pin=False)
    om = O.OMesh(c["tables"], c["export"])
    pmg = _pmg_oracle_levels(c["mesh"], [3, 2, 1], c["factor"], c["bc_types"])
    xo, io = O.solve(om, c["rhs"], c["bc_types"], O.PRE_PMG, c["factor"], abs_tol=0.0, rel_tol=1e-8,
                     max_iter=200, nullspace=1, pmg=pmg)
    op, s = _pmg_solver(c, sipg.FP64, 1, pin=False)
    x, info = s.solve_host(c["rhs"])
    assert info.status == sipg.SIPG_OK
    assert abs(info.iters - io.iters) <= 1
    assert rel_err(x, xo) < 1e-9


def test_pmultigrid_mixed_precision_reaches_fp64_tolerance(two_phase):
    c = W.poisson3d_two_phase(6, order=3, n_modes=64, pin=False)
    _, s64 = _pmg_solver(c, sipg.FP64, pin=False)
    x64, i64 = s64.solve_host(c["rhs"])
    _, s32 = _pmg_solver(c, sipg.FP32, pin=False)
    x32, i32 = s32.solve_host(c["rhs"])
    assert i32.status == sipg.SIPG_OK
    assert abs(i32.iters - i64.iters) <= 1
    assert i32.true_rel_res <= 1e-8
    assert rel_err(x32, x64) < 1e-6


def test_poisson2d_manufactured_solution_converges():
    errs = []
    for n in (8, 16, 32):
        c = W.poisson2d_manufactured(n, order=3)
        op = make_op(c["mesh"], 3, 1, bct=c["bc_types"])
        o = sipg.default_opts(sipg.SOLVER_BLOCK_JACOBI)
        o.rel_tol, o.abs_tol, o.max_iter = 1e-10, 0.0, 5000
        x, info = sipg.Solver(op, sipg.SOLVER_BLOCK_JACOBI, o).solve_host(c["rhs"])
        assert info.status == sipg.SIPG_OK
        errs.append(np.abs(x - c["exact"]).max())
    rates = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    assert rates.min() > 3.0, (errs, rates)


def test_nullspace_projection_solves_pure_neumann(two_phase):
    c = two_phase
    op = make_op(c["mesh"], 3, 1, c["factor"], bct=c["bc_types"])
    o = sipg.default_opts(sipg.SOLVER_JACOBI)
    o.rel_tol, o.abs_tol, o.max_iter, o.nullspace = 1e-8, 0.0, 3000, 1
    b = c["rhs"].copy()
    b -= b.mean()
    x, info = sipg.Solver(op, sipg.SOLVER_JACOBI, o).solve_host(b)
    assert info.status == sipg.SIPG_OK
    assert info.true_rel_res < 1e-7


def test_not_converged_and_invalid_arguments_report_status(two_phase):
    c = two_phase
    op = make_op(c["mesh"], 3, 1, c["factor"], bct=c["bc_types"])
    op.set_pin(*c["pin"])
    o = sipg.default_opts(sipg.SOLVER_JACOBI)
    o.max_iter = 2
    x, info = sipg.Solver(op, sipg.SOLVER_JACOBI, o).solve_host(c["rhs"])
    assert info.status == sipg.SIPG_NOT_CONVERGED and info.iters == 2
    with pytest.raises(sipg.SipgError) as ei:
        sipg.Operator(c["mesh"], 5, 1)
    assert ei.value.status == sipg.SIPG_INVALID_ARG
    b = c["rhs"].copy()
    b[0, 5, 3] = np.nan
    x, info = sipg.Solver(op, sipg.SOLVER_JACOBI, o).solve_host(b)
    assert info.status == sipg.SIPG_BREAKDOWN


@pytest.mark.parametrize("precision", [sipg.FP64, sipg.FP32], ids=["fp64", "mixed"])
def test_graph_replayed_iterations_match_eager_launches(precision):
    """Outer iterations replayed from captured CUDA graphs give the same iterates
    as kernels launched one by one, and a coefficient change after the capture
    is picked up (the graphs are captured again)."""
    c = W.poisson3d_two_phase(5, order=3, n_modes=64, pin=False)
    out = {}
    for graphs in (0, 1):
        op = make_op(c["mesh"], 3, 1, c["factor"], bct=c["bc_types"])
        o = sipg.default_opts(sipg.SOLVER_PMULTIGRID)
        o.rel_tol, o.abs_tol, o.max_iter, o.precision, o.nullspace = 1e-8, 0.0, 200, precision, 1
        o.graphs = graphs
        s = sipg.Solver(op, sipg.SOLVER_PMULTIGRID, o)
        x1, i1 = s.solve_host(c["rhs"])
        x2, i2 = s.solve_host(c["rhs"])            # replays the graphs captured by the first solve
        op.set_factor(2.0 * c["factor"])          # the operator changes: graphs must be rebuilt
        s.setup()
        x3, i3 = s.solve_host(c["rhs"])
        out[graphs] = (x1, i1, x2, i2, x3, i3)
        assert i1.status == i2.status == i3.status == sipg.SIPG_OK
        assert np.array_equal(x1, x2)
        assert rel_err(x3, 0.5 * x1) < 1e-6
    e, g = out[0], out[1]
    for k in (0, 2, 4):
        assert e[k + 1].iters == g[k + 1].iters
        assert np.array_equal(e[k], g[k])


@pytest.mark.parametrize("precision", [sipg.FP64, sipg.FP32], ids=["fp64", "mixed"])
def test_device_resident_loop_matches_host_loop(precision):
    """The outer loop run on the device (conditional while-node, stopping test on
    the device) runs the host-driven loop's kernels: the same iterations and the
    same iterates, reproducible run to run, and a coefficient change after the
    capture is picked up."""
    c = W.poisson3d_two_phase(5, order=3, n_modes=64, pin=False)
    out = {}
    for graphs in (1, 2):
        op = make_op(c["mesh"], 3, 1, c["factor"], bct=c["bc_types"])
        o = sipg.default_opts(sipg.SOLVER_PMULTIGRID)
        o.rel_tol, o.abs_tol, o.max_iter, o.precision, o.nullspace = 1e-10, 0.0, 200, precision, 1
        o.graphs = graphs
        s = sipg.Solver(op, sipg.SOLVER_PMULTIGRID, o)
        x1, i1 = s.solve_host(c["rhs"])
        x2, i2 = s.solve_host(c["rhs"])
        op.set_factor(2.0 * c["factor"])
        s.setup()
        x3, i3 = s.solve_host(c["rhs"])
        out[graphs] = (x1, i1, x3, i3)
        assert i1.status == i2.status == i3.status == sipg.SIPG_OK
        assert np.array_equal(x1, x2) and i1.iters == i2.iters
        assert rel_err(x3, 0.5 * x1) < 1e-8
        assert i1.true_rel_res < 1e-9
    h, d = out[1], out[2]
    assert h[1].iters == d[1].iters and h[3].iters == d[3].iters
    assert np.array_equal(d[0], h[0]) and np.array_equal(d[2], h[2])


def test_device_resident_loop_chunks_and_iteration_limit():
    """A solve longer than one device launch (64 iterations) continues across
    launches with the host loop's iteration count, and the iteration limit stops
    the device loop exactly."""
    c = W.poisson3d_two_phase(5, order=3, n_modes=64, pin=False)
    op = make_op(c["mesh"], 3, 1, c["factor"], bct=c["bc_types"])
    res = {}
    for graphs in (1, 2):
        o = sipg.default_opts(sipg.SOLVER_JACOBI)
        o.rel_tol, o.abs_tol, o.max_iter, o.nullspace = 1e-9, 0.0, 2000, 1
        o.graphs = graphs
        x, info = sipg.Solver(op, sipg.SOLVER_JACOBI, o).solve_host(c["rhs"])
        assert info.status == sipg.SIPG_OK and info.iters > 130
        res[graphs] = (x, info)
        o.max_iter = 77
        _, lim = sipg.Solver(op, sipg.SOLVER_JACOBI, o).solve_host(c["rhs"])
        assert lim.status == sipg.SIPG_NOT_CONVERGED and lim.iters == 77
    assert res[1][1].iters == res[2][1].iters
    assert np.array_equal(res[2][0], res[1][0])


@pytest.mark.parametrize("precision", [sipg.FP64, sipg.FP32], ids=["fp64", "mixed"])
def test_assembled_low_order_levels_match_matrix_free(precision):
    """The p=1 (and p=2) levels applied from stored element blocks, assembled by
    probing the matrix-free apply, give the matrix-free solver's iterates."""
    c = W.poisson3d_two_phase(5, order=3, n_modes=64, pin=False)
    res = {}
    for amo in (0, 1, 2):
        op = make_op(c["mesh"], 3, 1, c["factor"], bct=c["bc_types"])
        o = sipg.default_opts(sipg.SOLVER_PMULTIGRID)
        o.rel_tol, o.abs_tol, o.max_iter, o.precision, o.nullspace = 1e-8, 0.0, 200, precision, 1
        o.assembled_max_order = amo
        x, info = sipg.Solver(op, sipg.SOLVER_PMULTIGRID, o).solve_host(c["rhs"])
        assert info.status == sipg.SIPG_OK
        res[amo] = (x, info)
    for amo in (1, 2):
        assert abs(res[amo][1].iters - res[0][1].iters) <= (0 if precision == sipg.FP64 else 1)
        assert rel_err(res[amo][0], res[0][0]) < (1e-10 if precision == sipg.FP64 else 1e-6)


@pytest.mark.parametrize("precision", [sipg.FP64, sipg.FP32], ids=["fp64", "mixed"])
@pytest.mark.parametrize("n", [6, 16], ids=["full-blocks", "packed-blocks"])
def test_block_jacobi_smoothing_converges_faster_to_the_same_solution(precision, n):
    """Chebyshev on the element-block-Jacobi preconditioned operator (bf16 blocks
    in the FP32 V-cycle) needs fewer outer iterations than point Jacobi and
    reaches the same solution; 6^3 x 6 = 1,296 elements store full blocks,
    16^3 x 6 = 24,576 (at least 148 x 128 per level) packed symmetric triangles."""
    c = W.poisson3d_two_phase(n, order=3, n_modes=64, pin=False)
    out = {}
    for sm in (0, 1):
        op = make_op(c["mesh"], 3, 1, c["factor"], bct=c["bc_types"])
        o = sipg.default_opts(sipg.SOLVER_PMULTIGRID)
        o.rel_tol, o.abs_tol, o.max_iter, o.precision, o.nullspace = 1e-9, 0.0, 200, precision, 1
        o.smoother = sm
        out[sm] = sipg.Solver(op, sipg.SOLVER_PMULTIGRID, o).solve_host(c["rhs"])
    (x0, i0), (x1, i1) = out[0], out[1]
    assert i0.status == i1.status == sipg.SIPG_OK
    assert i1.iters < i0.iters
    assert i1.true_rel_res < 1e-9
    assert rel_err(x1, x0) < 1e-6


def test_per_level_chebyshev_degrees_and_sweeps():
    """The [p-multigrid] per-level keys: cheb_orders, pre_it, post_it."""
    c = W.poisson3d_two_phase(5, order=3, n_modes=64, pin=False)
    base = None
    for ch, pre, post in (((4, 4, 4), (1, 1, 1), (1, 1, 1)), ((3, 2, 4), (2, 1, 1), (1, 0, 1)),
                          ((4, 2, 2), (1, 1, 2), (0, 1, 2))):
        op = make_op(c["mesh"], 3, 1, c["factor"], bct=c["bc_types"])
        o = sipg.default_opts(sipg.SOLVER_PMULTIGRID)
        o.rel_tol, o.abs_tol, o.max_iter, o.nullspace = 1e-9, 0.0, 300, 1
        for i in range(3):
            o.cheb_orders[i], o.pre_it[i], o.post_it[i] = ch[i], pre[i], post[i]
        x, info = sipg.Solver(op, sipg.SOLVER_PMULTIGRID, o).solve_host(c["rhs"])
        assert info.status == sipg.SIPG_OK and info.true_rel_res < 1e-9
        if base is None:
            base = x
        else:
            assert rel_err(x, base) < 1e-6


def test_2d_block_jacobi_cg_config_matches_oracle():
    """The reference's CPU-runnable configuration: unit square, 64 x 64 quads split
    into 8,192 triangles, p = 3, zero Dirichlet walls, RHS M(8 pi^2 sin(2 pi x)
    sin(2 pi y)), block-Jacobi CG in FP64 to a 1e-10 relative residual; the solution
    agrees with the oracle's to 1e-9 (relative L2) and the iteration counts to 1."""
    c = W.poisson2d_manufactured(64, order=3)
    om = O.OMesh(c["tables"], c["export"])
    xo, io = O.solve(om, c["rhs"], c["bc_types"], O.PRE_BLOCK_JACOBI, abs_tol=0.0, rel_tol=1e-10, max_iter=5000)
    assert io.converged
    op = make_op(c["mesh"], 3, 1, bct=c["bc_types"])
    o = sipg.default_opts(sipg.SOLVER_BLOCK_JACOBI)
    o.rel_tol, o.abs_tol, o.max_iter = 1e-10, 0.0, 5000
    x, info = sipg.Solver(op, sipg.SOLVER_BLOCK_JACOBI, o).solve_host(c["rhs"])
    assert info.status == sipg.SIPG_OK
    assert abs(info.iters - io.iters) <= 1
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-9
