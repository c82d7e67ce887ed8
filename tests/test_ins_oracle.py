"""The time-step oracle (oracle/ins_oracle.py) against the reference's own
kernels: the non-linear advection step of INSSolverBase3D::advec_current_non_linear
/ advec_standard (src/solvers/3d/ins_solver_base.cpp:224-329, 451-480) run through
ins_3d_advec_0 (cells), ins_3d_advec_1 (interior faces), ins_3d_advec_2 (boundary
faces: no-slip, slip, natural outflow) and ins_3d_advec_3 (cells) compiled in
oracle/_ref, with the toolkit glue (mesh->div, the LIFT op2_gemv) restated."""
import ctypes as C

import numpy as np
import pytest

import dg_oracle as D
import ins_oracle as I
import oracle_py as O

pytestmark = pytest.mark.skipif(not O.have_ref(), reason="oracle/_ref not built")


def call(om, name, args):
    keep = []
    ptrs = []
    for a in args:
        if isinstance(a, list):  # a face argument: pointers to the two cells' data
            arr = (C.c_void_p * len(a))(*[x.ctypes.data_as(C.c_void_p) for x in a])
            keep.append(arr)
            ptrs.append(C.cast(arr, C.c_void_p))
        else:
            ptrs.append(a.ctypes.data_as(C.c_void_p))
    pa = (C.c_void_p * len(ptrs))(*ptrs)
    assert O.ref_lib().ref_kernel(C.byref(om.s), name.encode(), pa) == 0, name


def reference_advection(mesh, t, om, dt, a0, a1, b0, b1, u, u_old, N_old, vel_bc):
    K, Np, Nf, Nfp = mesh.K, t["Np"], t["Nf"], t["Nfp"]
    fm, pp = t["fmask"], t["perm_pos"]
    F = np.zeros((3, 3, K, Np))
    for e in range(K):
        outs = [np.zeros(Np) for _ in range(9)]
        call(om, "ins_3d_advec_0", [u[0, e].copy(), u[1, e].copy(), u[2, e].copy()] + outs)
        for c in range(3):
            for d in range(3):
                F[c, d, e] = outs[3 * c + d]
    N = np.stack([I.divergence(mesh, I._tables(t["order"]), F[c]) for c in range(3)])
    flux = np.zeros((3, K, Nf * Nfp))
    rows = [[np.ascontiguousarray(u[c, e]) for e in range(K)] for c in range(3)]
    fl = [[np.zeros(Nf * Nfp) for _ in range(K)] for _ in range(3)]
    nrm = np.stack([mesh.nx, mesh.ny, mesh.nz], 2)
    for (L, R), (fL, fR), sLR, sRL in zip(mesh.face2cells, mesh.faceNum, mesh.sLR, mesh.sRL):
        fmL_corr = np.ascontiguousarray(fm[fL][pp[sRL]], dtype=np.int32)  # L nodes in R's face order
        fmR_corr = np.ascontiguousarray(fm[fR][pp[sLR]], dtype=np.int32)  # R nodes in L's face order
        args = [np.array([fL, fR], np.int32), fmL_corr, fmR_corr,
                np.array([nrm[L, fL, 0], nrm[R, fR, 0]]), np.array([nrm[L, fL, 1], nrm[R, fR, 1]]),
                np.array([nrm[L, fL, 2], nrm[R, fR, 2]]), np.array([mesh.fscale[L, fL], mesh.fscale[R, fR]]),
                [rows[0][L], rows[0][R]], [rows[1][L], rows[1][R]], [rows[2][L], rows[2][R]],
                [fl[0][L], fl[0][R]], [fl[1][L], fl[1][R]], [fl[2][L], fl[2][R]]]
        call(om, "ins_3d_advec_1", args)
    bct = np.asarray(vel_bc).reshape(-1)
    e_x = mesh.export(t["order"], t)
    for b, (e, f) in enumerate(zip(mesh.bface2cell, mesh.bfaceNum)):
        args = [np.array([0.0]), np.array([bct[b]], np.int32), np.array([f], np.int32),
                np.array([nrm[e, f, 0]]), np.array([nrm[e, f, 1]]), np.array([nrm[e, f, 2]]),
                np.array([mesh.fscale[e, f]]), e_x["x"][e].copy(), e_x["y"][e].copy(), e_x["z"][e].copy(),
                rows[0][e], rows[1][e], rows[2][e], fl[0][e], fl[1][e], fl[2][e]]
        call(om, "ins_3d_advec_2", args)
    for c in range(3):
        for e in range(K):
            flux[c, e] = fl[c][e]
    LIFT = I._tables(t["order"])["LIFT"]
    N = N + flux @ LIFT.T
    velT = np.zeros_like(u)
    for e in range(K):
        outs = [np.zeros(Np) for _ in range(3)]
        args = [np.array([a0]), np.array([a1]), np.array([b0]), np.array([b1]), np.array([dt])]
        args += [u[c, e].copy() for c in range(3)] + [u_old[c, e].copy() for c in range(3)]
        args += [N[c, e].copy() for c in range(3)] + [N_old[c, e].copy() for c in range(3)] + outs
        call(om, "ins_3d_advec_3", args)
        for c in range(3):
            velT[c, e] = outs[c]
    return N, velT


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("scale", [0.5, 3.0], ids=["slow", "fast"])
def test_advection_matches_the_reference_kernels(p, scale):
    mesh = D.Mesh.box(3, 3, 0.1, 5)
    t = D.ref_tables(3, p)
    om = O.OMesh(t, mesh.export(p, t))
    rng = np.random.default_rng(p)
    u, u_old, N_old = rng.uniform(-scale, scale, (3, 3, mesh.K, t["Np"]))
    vel_bc = (np.arange(mesh.Kb) % 3).astype(np.int32)  # no-slip, slip, outflow
    dt, a0, a1, b0, b1 = 1e-3, 2.0, -0.5, 2.0, -1.0
    N, velT = I.advection(mesh, p, dt, a0, a1, b0, b1, u, u_old, N_old, vel_bc)
    Nr, velTr = reference_advection(mesh, t, om, dt, a0, a1, b0, b1, u, u_old, N_old, vel_bc)
    assert np.abs(N - Nr).max() <= 1e-12 * np.abs(Nr).max()
    assert np.abs(velT - velTr).max() <= 1e-12 * np.abs(velTr).max()


def test_advection_of_a_uniform_flow_vanishes_inside():
    """u constant: u (x) u is constant, its divergence zero, interior jumps zero."""
    mesh = D.Mesh.box(3, 3, 0.1, 5)
    t = D.ref_tables(3, 2)
    u = np.zeros((3, mesh.K, t["Np"]))
    u[0], u[1], u[2] = 0.3, -0.2, 0.1
    N = I.nonlinear(mesh, 2, u, np.full(mesh.Kb, I.BC_OUTFLOW, np.int32))
    assert np.abs(N).max() < 1e-12


@pytest.mark.parametrize("p", [1, 2, 3])
def test_pressure_neumann_data_matches_the_reference_kernels(p):
    """curl, mp_ins_3d_pr_mu, curl, then mp_ins_3d_pr_0 on every boundary face
    (the curls are the restated toolkit glue, as in the oracle)."""
    mesh = D.Mesh.box(3, 3, 0.1, 5)
    t = D.ref_tables(3, p)
    e_x = mesh.export(p, t)
    om = O.OMesh(t, e_x)
    rng = np.random.default_rng(20 + p)
    u, N = rng.uniform(-1, 1, (2, 3, mesh.K, t["Np"]))
    mu = rng.uniform(1.0, 100.0, (mesh.K, t["Np"]))
    rho = rng.uniform(1.0, 1000.0, (mesh.K, t["Np"]))
    vel_bc = (np.arange(mesh.Kb) % 3).astype(np.int32)
    re = 123.0
    want = I.pressure_neumann(mesh, p, u, N, mu, rho, vel_bc, re)
    tt = I._tables(p)
    cu = I.curl(mesh, tt, u)
    for e in range(mesh.K):
        rows = [np.ascontiguousarray(cu[c, e]) for c in range(3)]
        call(om, "mp_ins_3d_pr_mu", [mu[e].copy()] + rows)
        for c in range(3):
            cu[c, e] = rows[c]
    c2 = I.curl(mesh, tt, cu)
    O.ref_lib().ref_set_reynolds(C.c_double(re))
    got = np.zeros((mesh.K, t["Nf"] * t["Nfp"]))
    nrm = np.stack([mesh.nx, mesh.ny, mesh.nz], 2)
    for b, (e, f) in enumerate(zip(mesh.bface2cell, mesh.bfaceNum)):
        args = [np.array([0.0]), np.array([vel_bc[b]], np.int32), np.array([f], np.int32),
                np.array([nrm[e, f, 0]]), np.array([nrm[e, f, 1]]), np.array([nrm[e, f, 2]]),
                np.array([mesh.fscale[e, f]]), e_x["x"][e].copy(), e_x["y"][e].copy(), e_x["z"][e].copy(),
                N[0, e].copy(), N[1, e].copy(), N[2, e].copy(), c2[0, e].copy(), c2[1, e].copy(), c2[2, e].copy(),
                rho[e].copy(), got[e]]
        call(om, "mp_ins_3d_pr_0", args)
    assert np.abs(got.reshape(want.shape) - want).max() <= 1e-12 * np.abs(want).max()


def reference_ls_rhs(mesh, t, om, e_x, q, u, vel_bc):
    """AdvectionSolver3D::rhs through advec_3d_0, advec_3d_flux and ls_advec_3d_bc
    (div_weak and the LIFT are the restated glue)."""
    K, Np, Nf, Nfp = mesh.K, t["Np"], t["Nf"], t["Nfp"]
    fm, pp = t["fmask"], t["perm_pos"]
    F = np.zeros((3, K, Np))
    for e in range(K):
        outs = [np.zeros(Np) for _ in range(3)]
        call(om, "advec_3d_0", [q[e].copy(), u[0, e].copy(), u[1, e].copy(), u[2, e].copy()] + outs)
        for d in range(3):
            F[d, e] = outs[d]
    out = I.weak_divergence(mesh, I._tables(t["order"]), F)
    qs = [np.ascontiguousarray(q[e]) for e in range(K)]
    us = [[np.ascontiguousarray(u[c, e]) for e in range(K)] for c in range(3)]
    fl = [np.zeros(Nf * Nfp) for _ in range(K)]
    nrm = np.stack([mesh.nx, mesh.ny, mesh.nz], 2)
    for (L, R), (fL, fR), sLR, sRL in zip(mesh.face2cells, mesh.faceNum, mesh.sLR, mesh.sRL):
        args = [np.array([fL, fR], np.int32), np.ascontiguousarray(fm[fL][pp[sRL]], dtype=np.int32),
                np.ascontiguousarray(fm[fR][pp[sLR]], dtype=np.int32),
                np.array([nrm[L, fL, 0], nrm[R, fR, 0]]), np.array([nrm[L, fL, 1], nrm[R, fR, 1]]),
                np.array([nrm[L, fL, 2], nrm[R, fR, 2]]), np.array([mesh.fscale[L, fL], mesh.fscale[R, fR]]),
                [qs[L], qs[R]], [us[0][L], us[0][R]], [us[1][L], us[1][R]], [us[2][L], us[2][R]], [fl[L], fl[R]]]
        call(om, "advec_3d_flux", args)
    bct = np.asarray(vel_bc).reshape(-1)
    for b, (e, f) in enumerate(zip(mesh.bface2cell, mesh.bfaceNum)):
        args = [np.array([f], np.int32), np.array([bct[b]], np.int32), e_x["x"][e].copy(), e_x["y"][e].copy(),
                e_x["z"][e].copy(), np.array([nrm[e, f, 0]]), np.array([nrm[e, f, 1]]), np.array([nrm[e, f, 2]]),
                np.array([mesh.fscale[e, f]]), qs[e], us[0][e], us[1][e], us[2][e], fl[e]]
        call(om, "ls_advec_3d_bc", args)
    return out - np.stack(fl) @ I._tables(t["order"])["LIFT"].T


@pytest.mark.parametrize("p", [1, 2, 3])
def test_level_set_step_matches_the_reference_kernels(p):
    mesh = D.Mesh.box(3, 3, 0.1, 5)
    t = D.ref_tables(3, p)
    e_x = mesh.export(p, t)
    om = O.OMesh(t, e_x)
    rng = np.random.default_rng(40 + p)
    s = rng.uniform(-1, 1, (mesh.K, t["Np"]))
    u = rng.uniform(-2, 2, (3, mesh.K, t["Np"]))
    vel_bc = (np.arange(mesh.Kb) % 3).astype(np.int32)
    dt = 2e-3
    # the three stages through runge_kutta_0 / runge_kutta_1
    val = s.copy()
    rk = [np.zeros_like(s) for _ in range(3)]
    rkQ = np.zeros_like(s)

    def rk0_call(stage):
        for e in range(mesh.K):
            row = rkQ[e].copy()
            call(om, "runge_kutta_0", [np.array([stage], np.int32), np.array([dt]), val[e].copy(), rk[0][e].copy(),
                                       rk[1][e].copy(), row])
            rkQ[e] = row

    rk0_call(-1)
    for j in range(3):
        rk[j] = reference_ls_rhs(mesh, t, om, e_x, rkQ, u, vel_bc)
        if j != 2:
            rk0_call(j)
    for e in range(mesh.K):
        row = val[e].copy()
        call(om, "runge_kutta_1", [np.array([dt]), row, rk[0][e].copy(), rk[1][e].copy(), rk[2][e].copy()])
        val[e] = row
    want = I.ls_advect(mesh, p, dt, s, u, vel_bc)
    assert np.abs(val - want).max() <= 1e-12 * np.abs(want).max()
    # ls_step
    O.ref_lib().ref_set_fluid(C.c_double(1.0), C.c_double(1e-3), C.c_double(1.0), C.c_double(1e-2))
    rho, mu = np.zeros_like(s), np.zeros_like(s)
    for e in range(mesh.K):
        r_, m_ = np.zeros(t["Np"]), np.zeros(t["Np"])
        call(om, "ls_step", [np.array([0.3]), val[e].copy(), r_, m_])
        rho[e], mu[e] = r_, m_
    rw, mw = I.ls_props(val, 0.3, 1.0, 1e-3, 1.0, 1e-2)
    assert np.abs(rho - rw).max() <= 1e-14 and np.abs(mu - mw).max() <= 1e-14


def test_level_set_step_preserves_a_constant_in_a_uniform_flow():
    """q = const, u = const: the weak divergence and the interior fluxes cancel;
    the rhs is the boundary outflow of a constant only on boundary elements."""
    mesh = D.Mesh.box(3, 3, 0.1, 5)
    t = D.ref_tables(3, 2)
    q = np.full((mesh.K, t["Np"]), 0.7)
    u = np.zeros((3, mesh.K, t["Np"]))
    u[0], u[1], u[2] = 0.3, -0.2, 0.1
    r = I.ls_rhs(mesh, 2, q, u, np.full(mesh.Kb, I.BC_OUTFLOW, np.int32))
    inner = np.all(mesh.nbr >= 0, axis=1)
    assert np.abs(r[inner]).max() < 1e-12


def _bubble(mesh, p, center=(0.5, 0.3, 0.5), radius=0.25):
    t = D.ref_tables(3, p)
    e = mesh.export(p, t)
    s = np.sqrt((e["x"] - center[0]) ** 2 + (e["y"] - center[1]) ** 2 + (e["z"] - center[2]) ** 2) - radius
    return s, np.zeros((3, mesh.K, t["Np"]))


def test_two_phase_step_oracle_lifts_a_light_bubble():
    """Three steps of the composed oracle from rest: gravity with a bubble 1000 times
    lighter than its surroundings makes the fluid in it rise and the rest sink."""
    mesh = D.Mesh.box(3, 3, 0.1, 5)
    s, vel = _bubble(mesh, 2)
    st = I.TwoPhaseStep(mesh, 2, np.zeros(mesh.Kb, np.int32), 100.0, 1.0, 1e-3, 1.0, 1e-2, gravity=9.81,
                        ls_alpha=2.0)
    st.set_state(vel, s)
    ups = []
    for _ in range(3):
        st.step()
        assert st.pr_info.iters < 5000
        ups.append(st.vel[1][s < 0].mean())
    assert 0 < ups[0] < ups[1] < ups[2]
    assert st.vel[1][s > 0.1].mean() < 0
    assert st.time == pytest.approx(3 * st.dt)


def _plane_distance(e, nrm=(0.3, 1.0, -0.2), y0=0.45):
    n = np.asarray(nrm) / np.linalg.norm(nrm)
    return n[0] * (e["x"] - 0.5) + n[1] * (e["y"] - y0) + n[2] * (e["z"] - 0.5)


@pytest.mark.parametrize("p", [2, 3])
def test_reinit_recovers_the_distance_to_a_plane(p):
    """A linear level set is its own polynomial in every element: the closest points are
    exact, so three times the distance comes back as the distance."""
    mesh = D.Mesh.box(3, 3, 0.1, 5)
    e = mesh.export(p, D.ref_tables(3, p))
    dist = _plane_distance(e)
    got = I.ls_reinit(mesh, p, 3.0 * dist)
    assert np.abs(got - np.clip(dist, -1.0, 1.0)).max() < 1e-12


def test_reinit_converges_to_the_distance_to_a_sphere():
    errs = []
    for n in (3, 5):
        mesh = D.Mesh.box(3, n, 0.1, 5)
        e = mesh.export(2, D.ref_tables(3, 2))
        d = np.sqrt((e["x"] - 0.5) ** 2 + (e["y"] - 0.45) ** 2 + (e["z"] - 0.5) ** 2) - 0.3
        got = I.ls_reinit(mesh, 2, 2.0 * d)
        assert np.all(np.sign(got) == np.sign(d))
        errs.append(np.abs(got - d)[np.abs(d) < 0.1].max())
    assert errs[0] < 0.02 and errs[1] < errs[0] / 2
