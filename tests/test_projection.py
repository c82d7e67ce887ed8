"""Element-local velocity projection (INSSolverBase3D::project_velocity with
div_div = 1, src/solvers/3d/ins_solver_base.cpp:1052-1124; 2D
src/solvers/2d/ins_solver_base.cpp:894-955).

CPU: the oracle's restatement against the golden vectors made by the
reference's own kernels (ins_proj_setup_0/1, ins_3d_proj_rhs, ins_3d_proj_pen,
ins_3d_proj_cg_precon and the 2D twins) and against those kernels on fresh
cases. GPU: sipg_project_velocity(_host) against the oracle, the device
counters, argument errors, and a full-size case (32^3 x 6 tets, p = 3).

Tolerances. 3D: the solve is preconditioned by the inverse mass matrix and
converges in a few iterations per element, so results agree to round-off
(TOL_PROJ_3D) with identical iteration counts. 2D: the reference's CG is
unpreconditioned and stops on the absolute |r|_2^2 < 1e-16 of a system scaled by
the element Jacobian (J ~ h^2), so the solution is fixed only to about
|A^-1| * 1e-8 ~ 1e-5 of its size: round-off in a different summation order moves
the last iterates by that much and the iteration count of an element by one
(the test allows one iteration per element on the total).
"""
import glob
import os

import numpy as np
import pytest

import oracle_py as O
import sipg
from helpers import rel_err

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN_PROJ = sorted(glob.glob(os.path.join(HERE, "golden", "projection", "*.npz")))

TOL_PROJ_3D = 1e-12
TOL_PROJ_2D = 2e-4


def case(dim, n, order, seed, dt, jitter=0.1):
    mesh = sipg.Mesh.box(dim, n, jitter=jitter, seed=seed)
    t, e = sipg.ref_tables(dim, order), mesh.export(order)
    rng = np.random.default_rng(seed)
    velT = rng.uniform(-1, 1, (dim, e["K"], t["Np"]))
    dp = rng.uniform(-1, 1, (dim, e["K"], t["Np"]))
    return mesh, O.OMesh(t, e), velT, dp


def check_close(dim, got, gst, want, wst):
    assert gst[0] == wst[0] and gst[1] == wst[1], (gst, wst)
    if dim == 3:
        assert rel_err(got, want) < TOL_PROJ_3D
        assert gst[2] == wst[2], (gst, wst)
    else:
        assert rel_err(got, want) < TOL_PROJ_2D
        assert abs(gst[2] - wst[2]) <= wst[0], (gst, wst)  # at most one iteration per element


@pytest.mark.parametrize("path", GOLDEN_PROJ, ids=[os.path.basename(p)[:-4] for p in GOLDEN_PROJ])
def test_oracle_matches_reference_golden(path):
    g = dict(np.load(path))
    dim, n, order, seed = int(g["dim"]), int(g["n"]), int(g["order"]), int(g["seed"])
    mesh = sipg.Mesh.box(dim, n, jitter=float(g["jitter"]), seed=seed)
    t, e = sipg.ref_tables(dim, order), mesh.export(order)
    assert np.array_equal(e["geof"], g["geof"]), "mesh builder drifted from the golden fixture"
    got, st = O.project_velocity(O.OMesh(t, e), float(g["dt"]), float(g["factor"]), g["dp"], g["velT"])
    check_close(dim, got, st, g["velTT"], g["stats"])


@pytest.mark.parametrize("dim,n,order,dt", [(3, 3, 2, 1e-2), (3, 2, 4, 5e-2), (2, 5, 1, 1e-3), (2, 4, 4, 1e-3)])
def test_oracle_matches_reference_kernels(dim, n, order, dt):
    if not O.have_ref():
        pytest.skip("oracle/_ref not built (the reference tree is not available)")
    _, om, velT, dp = case(dim, n, order, 7 + order, dt)
    f = sipg.projection_factor(dim, dt)
    a, sa = O.project_velocity(om, dt, f, dp, velT)
    b, sb = O.project_velocity(om, dt, f, dp, velT, use_ref=True)
    check_close(dim, a, sa, b, sb)


def test_oracle_penalty_length_is_inverse_max_interior_fscale():
    mesh, om, _, _ = case(3, 3, 2, 1, 1e-2)
    e = mesh.export(2)
    h = O.proj_h(om)
    inner = np.zeros_like(e["fscale"])
    for (eL, eR), (fL, fR) in zip(e["face2cells"], e["faceNum"]):
        inner[eL, fL] = e["fscale"][eL, fL]
        inner[eR, fR] = e["fscale"][eR, fR]
    assert np.array_equal(h, 1.0 / inner.max(axis=1))


def test_projection_factor_follows_the_reference():
    assert sipg.projection_factor(3, 2e-3) == 2e-3
    assert sipg.projection_factor(2, 2e-3) == pytest.approx(2.0)


@pytest.mark.gpu
@pytest.mark.parametrize("path", GOLDEN_PROJ, ids=[os.path.basename(p)[:-4] for p in GOLDEN_PROJ])
def test_gpu_matches_reference_golden(path):
    g = dict(np.load(path))
    dim, order = int(g["dim"]), int(g["order"])
    mesh = sipg.Mesh.box(dim, int(g["n"]), jitter=float(g["jitter"]), seed=int(g["seed"]))
    got, st = sipg.project_velocity(mesh, order, float(g["dt"]), g["dp"], g["velT"], factor=float(g["factor"]))
    check_close(dim, got, st, g["velTT"], g["stats"])


@pytest.mark.gpu
@pytest.mark.parametrize("dim,n,order,dt", [(3, 3, 1, 1e-2), (3, 3, 2, 1e-2), (3, 3, 3, 1e-3), (3, 3, 3, 0.2),
                                            (3, 2, 4, 1e-2), (2, 6, 1, 1e-3), (2, 6, 2, 1e-3), (2, 6, 3, 1e-4),
                                            (2, 4, 4, 1e-3)])
def test_gpu_matches_oracle(dim, n, order, dt):
    mesh, om, velT, dp = case(dim, n, order, 100 + 10 * dim + order, dt)
    want, wst = O.project_velocity(om, dt, sipg.projection_factor(dim, dt), dp, velT)
    got, gst = sipg.project_velocity(mesh, order, dt, dp, velT)
    check_close(dim, got, gst, want, wst)


@pytest.mark.gpu
def test_gpu_device_entry_point_counters_and_repeatability():
    dim, order, dt = 3, 3, 0.05
    mesh, om, velT, dp = case(dim, 3, order, 3, dt)
    host, hst = sipg.project_velocity(mesh, order, dt, dp, velT)
    d_dp, d_v = sipg.DeviceVector(dp), sipg.DeviceVector(velT)
    d_out = sipg.DeviceVector(np.zeros_like(velT))
    d_st = sipg.DeviceVector(np.full(2, 12345, np.uint64))
    for _ in range(2):  # the counters are zeroed by every call
        sipg.project_velocity_device(mesh, order, dt, d_dp.ptr, d_v.ptr, d_out.ptr, d_st.ptr)
        assert np.array_equal(d_out.get(), host)
        st = d_st.get()
        assert st[0] == hst[1] and st[1] == hst[2]


@pytest.mark.gpu
def test_gpu_rejects_aliasing_and_bad_arguments():
    mesh, _, velT, dp = case(3, 2, 2, 1, 1e-2)
    d_dp, d_v = sipg.DeviceVector(dp), sipg.DeviceVector(velT)
    with pytest.raises(sipg.SipgError):
        sipg.project_velocity_device(mesh, 2, 1e-2, d_dp.ptr, d_v.ptr, d_v.ptr)
    with pytest.raises(sipg.SipgError):
        sipg.project_velocity_device(mesh, 5, 1e-2, d_dp.ptr, d_v.ptr, d_dp.ptr)
    with pytest.raises(sipg.SipgError):
        sipg.project_velocity(mesh, 2, float("nan"), dp, velT)


@pytest.mark.gpu
def test_gpu_full_size_32cube_p3():
    """32^3 x 6 = 196,608 tets at p = 3 (the rising-bubble mesh): every element
    converges, the result equals the oracle's, and a field with zero pressure
    gradient that is constant per element is returned unchanged (its divergence
    vanishes to round-off, so the initial residual is below the tolerance and no
    iteration runs)."""
    dim, order, dt = 3, 3, 1e-3
    mesh, om, velT, dp = case(dim, 32, order, 20261203, dt)
    got, st = sipg.project_velocity(mesh, order, dt, dp, velT)
    assert st[0] == st[1] == mesh.K
    want, wst = O.project_velocity(om, dt, dt, dp, velT)
    check_close(dim, got, st, want, wst)
    const = np.repeat(velT[:, :, :1], velT.shape[2], axis=2)
    out, st0 = sipg.project_velocity(mesh, order, dt, np.zeros_like(dp), const)
    assert st0[2] == 0
    assert rel_err(out, const) < 1e-13


# ---- pressure projection step: central-flux gradient (/ rho) fused with the projection

def poly_case(dim, n, order, seed=3):
    """A continuous polynomial of degree `order` at the nodes, with its gradient."""
    mesh = sipg.Mesh.box(dim, n, jitter=0.1, seed=seed)
    t, e = sipg.ref_tables(dim, order), mesh.export(order)
    x, y = e["x"], e["y"]
    z = e["z"] if dim == 3 else np.zeros_like(x)
    s = x + 2 * y - z
    p = s ** order + 0.5 * x
    g = [order * s ** (order - 1) + 0.5, 2 * order * s ** (order - 1), -order * s ** (order - 1)]
    return mesh, O.OMesh(t, e), p, np.stack(g[:dim])


@pytest.mark.parametrize("dim,order", [(3, 2), (3, 3), (3, 4), (2, 2), (2, 4)])
def test_oracle_central_gradient_is_exact_for_continuous_polynomials(dim, order):
    _, om, p, g = poly_case(dim, 3 if dim == 3 else 5, order)
    assert np.abs(O.grad_central(om, p) - g).max() < 1e-9 * max(1.0, np.abs(g).max())


def test_oracle_central_gradient_is_linear_and_kills_constants():
    """On a discontinuous field: linear in p, and a constant adds nothing."""
    mesh, om, _, _ = poly_case(3, 3, 3)
    rng = np.random.default_rng(4)
    p = rng.uniform(-1, 1, (om.K, om.Np))
    g = O.grad_central(om, p)
    a = O.grad_central(om, 2.0 * p + 1.0)
    assert np.abs(a - 2.0 * g).max() < 1e-11 * np.abs(g).max()  # linear, constants have zero gradient


def pressure_chain_oracle(om, dim, dt, pr, rho, velT):
    g = O.grad_central(om, pr)
    if rho is not None:
        g = g / rho[None]
    return O.project_velocity(om, dt, sipg.projection_factor(dim, dt), g, velT)


@pytest.mark.gpu
@pytest.mark.parametrize("dim,n,order,dt,two_phase", [(3, 3, 3, 1e-2, True), (3, 3, 2, 1e-2, False),
                                                       (3, 2, 4, 1e-2, True), (3, 3, 1, 1e-2, False),
                                                       (2, 6, 3, 1e-3, True), (2, 6, 2, 1e-3, False)])
def test_gpu_pressure_projection_matches_oracle(dim, n, order, dt, two_phase):
    mesh, om, velT, _ = case(dim, n, order, 200 + 10 * dim + order, dt)
    rng = np.random.default_rng(order)
    pr = rng.uniform(-1, 1, (om.K, om.Np))
    rho = rng.uniform(1.0, 1000.0, (om.K, om.Np)) if two_phase else None
    want, wst = pressure_chain_oracle(om, dim, dt, pr, rho, velT)
    got, gst = sipg.pressure_projection(mesh, order, dt, pr, velT, rho=rho)
    check_close(dim, got, gst, want, wst)


@pytest.mark.gpu
@pytest.mark.parametrize("dim,order", [(3, 3), (3, 4), (2, 3)])
def test_gpu_central_gradient_alone(dim, order):
    """factor = 0, dt = -1 and velT = 0 leave velTT = grad p / rho (the initial
    residual is exactly zero): the gradient against the oracle, and exact for a
    continuous polynomial."""
    mesh, om, p, g = poly_case(dim, 3 if dim == 3 else 5, order)
    zero = np.zeros((dim, om.K, om.Np))
    got, st = sipg.pressure_projection(mesh, order, -1.0, p, zero, factor=0.0)
    assert st[2] == 0
    assert np.abs(got - g).max() < 1e-9 * np.abs(g).max()
    rng = np.random.default_rng(9)
    q = rng.uniform(-1, 1, p.shape)
    rho = rng.uniform(1.0, 10.0, p.shape)
    got, _ = sipg.pressure_projection(mesh, order, -1.0, q, zero, rho=rho, factor=0.0)
    assert rel_err(got, O.grad_central(om, q) / rho[None]) < 1e-12


@pytest.mark.gpu
def test_gpu_fused_step_equals_gradient_then_projection():
    dim, order, dt = 3, 3, 0.05
    mesh, om, velT, _ = case(dim, 3, order, 77, dt)
    rng = np.random.default_rng(1)
    pr = rng.uniform(-1, 1, (om.K, om.Np))
    rho = rng.uniform(1.0, 1000.0, (om.K, om.Np))
    grad, _ = sipg.pressure_projection(mesh, order, -1.0, pr, np.zeros_like(velT), rho=rho, factor=0.0)
    two_step, st2 = sipg.project_velocity(mesh, order, dt, grad, velT)
    fused, st1 = sipg.pressure_projection(mesh, order, dt, pr, velT, rho=rho)
    assert np.array_equal(fused, two_step) and np.array_equal(st1, st2)


# ---- pressure right-hand side: central-flux divergence, dPdN update and lift, mass

def vec_poly_case(dim, n, order, seed=5):
    """A continuous polynomial velocity field of degree `order` and its divergence."""
    mesh = sipg.Mesh.box(dim, n, jitter=0.1, seed=seed)
    t, e = sipg.ref_tables(dim, order), mesh.export(order)
    x, y = e["x"], e["y"]
    z = e["z"] if dim == 3 else np.zeros_like(x)
    s = x - y + 2 * z
    u = [s ** order, x * 0.5 + y ** order, (x + z) ** order]
    div = order * s ** (order - 1) + order * y ** (order - 1)
    if dim == 3:
        div = div + order * (x + z) ** (order - 1)
    return mesh, t, e, O.OMesh(t, e), np.stack(u[:dim]), div


@pytest.mark.parametrize("dim,order", [(3, 2), (3, 3), (2, 3), (2, 4)])
def test_oracle_pressure_rhs_divergence_is_exact_for_continuous_polynomials(dim, order):
    mesh, t, e, om, u, div = vec_poly_case(dim, 3 if dim == 3 else 5, order)
    dt = 0.01
    rhs, _ = O.pressure_rhs(om, dt, u)
    J = e["geof"][:, -1]
    want = J[:, None] * ((-div / dt) @ t["M"].T)
    assert np.abs(rhs - want).max() < 1e-9 * np.abs(want).max()


def test_oracle_pressure_rhs_neumann_term_is_the_face_mass():
    """LIFT then mass is EMAT: with velT = 0, rhs = J EMAT (b0 dPdN + b1 dPdN_old)."""
    mesh, t, e, om, u, _ = vec_poly_case(3, 2, 3)
    rng = np.random.default_rng(2)
    shp = (om.K, 4, t["Nfp"])
    dn, do = rng.uniform(-1, 1, shp), rng.uniform(-1, 1, shp)
    rhs, do2 = O.pressure_rhs(om, 0.01, np.zeros_like(u), dn, do, b0=2.0, b1=-1.0)
    new = 2.0 * dn - do
    assert np.array_equal(do2, new)
    want = e["geof"][:, -1][:, None] * (new.reshape(om.K, -1) @ t["EMAT"].T)
    assert np.abs(rhs - want).max() < 1e-11 * np.abs(want).max()


@pytest.mark.gpu
@pytest.mark.parametrize("dim,n,order", [(3, 3, 3), (3, 3, 1), (3, 2, 4), (3, 3, 2), (2, 6, 3), (2, 5, 2)])
def test_gpu_pressure_rhs_matches_oracle(dim, n, order):
    mesh, om, velT, _ = case(dim, n, order, 300 + 10 * dim + order, 1e-2)
    rng = np.random.default_rng(order + 10 * dim)
    shp = (om.K, dim + 1, sipg.ref_sizes(dim, order)[1])
    dn, do = rng.uniform(-1, 1, shp), rng.uniform(-1, 1, shp)
    want, wdo = O.pressure_rhs(om, 1e-2, velT, dn, do, b0=2.0, b1=-1.0)
    got, gdo = sipg.pressure_rhs(mesh, order, 1e-2, velT, dn, do, b0=2.0, b1=-1.0)
    assert rel_err(got, want) < 1e-12
    assert rel_err(gdo, wdo) < 1e-15
    got0, none = sipg.pressure_rhs(mesh, order, 1e-2, velT)  # no Neumann data
    want0, _ = O.pressure_rhs(om, 1e-2, velT)
    assert none is None and rel_err(got0, want0) < 1e-12


@pytest.mark.gpu
def test_gpu_pressure_rhs_exact_divergence():
    dim, order = 3, 3
    mesh, t, e, om, u, div = vec_poly_case(dim, 3, order)
    got, _ = sipg.pressure_rhs(mesh, order, 0.01, u)
    want = e["geof"][:, -1][:, None] * ((-div / 0.01) @ t["M"].T)
    assert np.abs(got - want).max() < 1e-9 * np.abs(want).max()


@pytest.mark.gpu
@pytest.mark.parametrize("dim,n,order", [(3, 4, 3), (3, 3, 4), (2, 8, 3), (3, 3, 2)])
def test_viscous_rhs_matches_the_reference_kernel_and_mass(dim, n, order):
    """sipg_viscous_rhs_host: mp_ins_3d_vis_0 then mesh->mass on each component
    (src/solvers/3d/mp_ins_solver.cpp:669-694) as one kernel, against the
    reference's own mp_ins_3d_vis_0 (oracle/_ref) followed by J M per element."""
    import ctypes as C
    mesh = sipg.Mesh.box(dim, n, jitter=0.1, seed=3 + order)
    t, e = sipg.ref_tables(dim, order), mesh.export(order)
    K, Np = mesh.K, t["Np"]
    rng = np.random.default_rng(order + 10 * dim)
    rho = rng.uniform(1.0, 1000.0, (K, Np))
    vel = rng.uniform(-1.0, 1.0, (dim, K, Np))
    fact0, fact1 = 1e3 / 1e-3, 1.5 * 1e3 / 1e-3
    rhs = np.zeros_like(vel)
    mm = np.zeros_like(rho)
    sipg.check(sipg.lib().sipg_viscous_rhs_host(mesh.h, order, C.c_double(fact0), C.c_double(fact1),
                                                O._d(rho), O._d(np.ascontiguousarray(vel)), O._d(rhs), O._d(mm)))
    J = e["geof"][:, -1]
    want = J[None, :, None] * ((fact0 * rho[None] * vel) @ t["M"].T)
    assert np.abs(rhs - want).max() <= 1e-13 * np.abs(want).max()
    assert np.abs(mm - fact1 * rho).max() <= 1e-15 * np.abs(fact1 * rho).max()
    if dim == 3 and O.have_ref():
        # the reference's kernel on the first elements, then the mass
        om = O.OMesh(t, e)
        for el in range(4):
            args = [np.array([fact0]), np.array([fact1]), rho[el].copy(), np.zeros(Np), np.zeros(1)]
            args += [vel[c, el].copy() for c in range(3)] + [np.zeros(Np) for _ in range(4)]
            ptrs = (C.c_void_p * len(args))(*[a.ctypes.data_as(C.c_void_p) for a in args])
            assert O.ref_lib().ref_kernel(C.byref(om.s), b"mp_ins_3d_vis_0", ptrs) == 0
            for c in range(3):
                ref = J[el] * (t["M"] @ args[8 + c])
                assert np.abs(rhs[c, el] - ref).max() <= 1e-13 * np.abs(ref).max()
            assert np.abs(mm[el] - args[11]).max() <= 1e-15 * np.abs(args[11]).max()
