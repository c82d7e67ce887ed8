"""The steps of the 3D incompressible time step around the pressure and viscous
solves, restated in numpy. TEST INFRASTRUCTURE ONLY (tests/, the CPU legs of
the benchmark).

ls_advect / ls_props: the level-set step of LevelSetSolver3D::step and getRhoMu
(src/solvers/3d/ls_solver.cpp:192-200, 243-257): AdvectionSolver3D::step's three
Runge-Kutta stages (src/solvers/3d/advection_solver.cpp:24-72, runge_kutta_0/1) of
rhs = div_weak(u q) - LIFT(flux) (advection_solver.cpp:84-120: advec_3d_0,
mesh->div_weak of OP2-DG-Toolkit, unvendored, restated as M^-1 D_r^T M, the upwind
advec_3d_flux and ls_advec_3d_bc), then ls_step's smoothed Heaviside.

pressure_neumann: the curl-curl Neumann data of the multiphase pressure step,
MPINSSolver3D::apply_pressure_neumann_bc (src/solvers/3d/mp_ins_solver.cpp:450-493).

TwoPhaseStep: MPINSSolver3D::step (src/solvers/3d/mp_ins_solver.cpp:245-285) composed
of the pieces above, the oracle's pressure right-hand side, gradient, velocity
projection and conjugate-gradient solves (oracle/oracle_py.py) run to a tight
tolerance, and the level-set step.

advection: INSSolverBase3D::advec_current_non_linear and advec_standard
(src/solvers/3d/ins_solver_base.cpp:224-329, 451-480): the flux tensor
u (x) u at the nodes (ins_3d_advec_0), its strong-form divergence (mesh->div of
OP2-DG-Toolkit, unvendored, restated: sum_d sum_r dr_r/dx_d D_r f_d), the
Lax-Friedrichs face fluxes (ins_3d_advec_1 on interior faces, ins_3d_advec_2 on
boundary faces: no-slip, slip and natural outflow), lifted by LIFT = M^-1 EMAT
(op2_gemv), and the extrapolated intermediate velocity (ins_3d_advec_3):
  velT = a0 u + a1 u_old - dt (b0 N + b1 N_old).
The boundary kernel's wave speed is stored in an int (ins_3d_advec_2.h:44,
`int maxVel = 0.0`), so it is the floor of the largest |n . u| over the face;
the restatement keeps that.
"""
import numpy as np

import dg_oracle as D
import oracle_py as O

BC_NO_SLIP, BC_SLIP, BC_OUTFLOW = 0, 1, 2


def _tables(p):
    t = D.ref_tables(3, p)
    t["LIFT"] = np.linalg.solve(t["M"], t["EMAT"])
    return t


def divergence(mesh, t, f):
    """sum_d d f_d / dx_d for f: (3, K, Np) nodal (strong form, element-local)."""
    Dm = [t["Dr"], t["Ds"], t["Dt"]]
    out = np.zeros(f.shape[1:])
    for d in range(3):
        for r in range(3):
            out += mesh.G[:, r, d][:, None] * (f[d] @ Dm[r].T)
    return out


def face_flux(mesh, t, u, vel_bc):
    """(3, K, Nf, Nfp): the Lax-Friedrichs flux of ins_3d_advec_1/2 per element
    face node (element-centric: each interior face from both sides)."""
    K, Nf, Nfp = mesh.K, t["Nf"], t["Nfp"]
    fm, pp = t["fmask"], t["perm_pos"]
    out = np.zeros((3, K, Nf, Nfp))
    nrm = np.stack([mesh.nx, mesh.ny, mesh.nz], 2)  # K x Nf x 3
    bct = np.asarray(vel_bc).reshape(-1)
    for e in range(K):
        for f in range(Nf):
            n = nrm[e, f]
            fs = mesh.fscale[e, f]
            uM = u[:, e, fm[f]]  # 3 x Nfp
            nb = mesh.nbr[e, f]
            if nb >= 0:
                g, sg = mesh.nbr_face[e, f], mesh.nbr_perm[e, f]
                uP = u[:, nb, fm[g][pp[sg]]]
                nP = nrm[nb, g]
                lvel = n @ uM
                rvel = nP @ uP
                lam = np.maximum(np.abs(lvel), np.abs(rvel))
                out[:, e, f] = 0.5 * fs * (-(uM * lvel - uP * (n @ uP)) - lam * (uP - uM))
            else:
                b = -nb - 1
                kind = bct[b]
                if kind == BC_NO_SLIP:
                    uR = np.zeros_like(uM)
                elif kind == BC_SLIP:
                    nn = n / np.linalg.norm(n)
                    uR = uM - np.outer(nn, nn @ uM)
                else:
                    uR = uM.copy()
                lvel, rvel = n @ uM, n @ uR
                lam = float(int(max(0.0, np.maximum(np.abs(lvel), np.abs(rvel)).max())))
                out[:, e, f] = 0.5 * fs * (-(uM * lvel - uR * rvel) - lam * (uR - uM))
    return out


def nonlinear(mesh, p, u, vel_bc):
    """N = div(u (x) u) + LIFT(flux), (3, K, Np)."""
    t = _tables(p)
    F = np.einsum("cki,dki->cdki", u, u)  # F[c][d] = u_c u_d
    N = np.stack([divergence(mesh, t, F[c]) for c in range(3)])
    fl = face_flux(mesh, t, u, vel_bc).reshape(3, mesh.K, -1)
    return N + fl @ t["LIFT"].T


def gradient(mesh, t, f):
    """(3, K, Np): d f / dx_d, strong form, element-local."""
    Dm = [t["Dr"], t["Ds"], t["Dt"]]
    return np.stack([sum(mesh.G[:, r, d][:, None] * (f @ Dm[r].T) for r in range(3)) for d in range(3)])


def curl(mesh, t, u):
    """mesh->curl (OP2-DG-Toolkit, unvendored, restated): the strong-form,
    element-local curl of a nodal vector field (3, K, Np)."""
    g = [gradient(mesh, t, u[c]) for c in range(3)]  # g[c][d] = d u_c / dx_d
    return np.stack([g[2][1] - g[1][2], g[0][2] - g[2][0], g[1][0] - g[0][1]])


def pressure_neumann(mesh, p, u, N, mu, rho, vel_bc, reynolds, grav=0.0):
    """dPdN (K, Nf, Nfp) of MPINSSolver3D::apply_pressure_neumann_bc
    (src/solvers/3d/mp_ins_solver.cpp:450-493): curl(mu curl u) (mesh->curl,
    mp_ins_3d_pr_mu, mesh->curl), then on no-slip and slip walls (mp_ins_3d_pr_0)
    fscale n . (-N - curl2 / (Re rho)) at the face nodes; zero elsewhere (natural
    outflow and interior faces)."""
    t = _tables(p)
    c2 = curl(mesh, t, curl(mesh, t, u) * mu[None])
    K, Nf, Nfp = mesh.K, t["Nf"], t["Nfp"]
    out = np.zeros((K, Nf, Nfp))
    bct = np.asarray(vel_bc).reshape(-1)
    nrm = np.stack([mesh.nx, mesh.ny, mesh.nz], 2)
    for e in range(K):
        for f in range(Nf):
            nb = mesh.nbr[e, f]
            if nb >= 0 or bct[-nb - 1] not in (BC_NO_SLIP, BC_SLIP):
                continue
            m = t["fmask"][f]
            res = -(N[:, e, m] + _gravity(grav)[:, None]) - c2[:, e, m] / (reynolds * rho[e, m])
            out[e, f] = mesh.fscale[e, f] * (nrm[e, f] @ res)
    return out


def _gravity(grav):
    """The body force -grav along y as the term added to N (the 2D solver's
    ins_advec_intermediate_vel_grav_2d.h adds 1 / Fr^2 to N_y)."""
    return np.array([0.0, grav, 0.0])


def advection(mesh, p, dt, a0, a1, b0, b1, u, u_old, N_old, vel_bc, grav=0.0):
    """(N, velT) of one advection step; grav: body force -grav along y, added to
    N_y in the extrapolation only."""
    N = nonlinear(mesh, p, u, vel_bc)
    G = _gravity(grav)[:, None, None]
    velT = (a0 * u + a1 * u_old) - dt * (b0 * (N + G) + b1 * (N_old + G))
    return N, velT


def weak_divergence(mesh, t, F):
    """mesh->div_weak (OP2-DG-Toolkit, unvendored, restated): the weak-form
    divergence M^-1 int grad(phi) . F of F (3, K, Np), i.e. sum_d sum_r dr/dx_d
    Dw_r F_d with the weak derivatives Dw_r = M^-1 D_r^T M."""
    Minv = np.linalg.inv(t["M"])
    out = np.zeros(F.shape[1:])
    for r, Dm in enumerate([t["Dr"], t["Ds"], t["Dt"]]):
        Dw = Minv @ Dm.T @ t["M"]
        for d in range(3):
            out += mesh.G[:, r, d][:, None] * (F[d] @ Dw.T)
    return out


def ls_face_flux(mesh, t, q, u, vel_bc):
    """(K, Nf, Nfp): advec_3d_flux on interior faces (upwind on the element's own
    normal velocity) and ls_advec_3d_bc on no-slip, slip and outflow faces."""
    K, Nf = mesh.K, t["Nf"]
    fm, pp = t["fmask"], t["perm_pos"]
    nrm = np.stack([mesh.nx, mesh.ny, mesh.nz], 2)
    out = np.zeros((K, Nf, t["Nfp"]))
    bct = np.asarray(vel_bc).reshape(-1)
    for e in range(K):
        for f in range(Nf):
            m = fm[f]
            un = nrm[e, f] @ u[:, e, m]
            qM = q[e, m]
            nb = mesh.nbr[e, f]
            if nb >= 0:
                qP = q[nb, fm[mesh.nbr_face[e, f]][pp[mesh.nbr_perm[e, f]]]]
                out[e, f] = mesh.fscale[e, f] * (un * 0.5 * (qM + qP) + 0.5 * np.abs(un) * (qM - qP))
            else:
                assert bct[-nb - 1] in (BC_NO_SLIP, BC_SLIP, BC_OUTFLOW)
                out[e, f] = mesh.fscale[e, f] * un * qM
    return out


def ls_rhs(mesh, p, q, u, vel_bc):
    """div_weak(u q) - LIFT(flux), (K, Np)."""
    t = _tables(p)
    out = weak_divergence(mesh, t, u * q[None])
    return out - ls_face_flux(mesh, t, q, u, vel_bc).reshape(mesh.K, -1) @ t["LIFT"].T


def ls_advect(mesh, p, dt, s, u, vel_bc):
    """One AdvectionSolver3D::step: the stages of runge_kutta_0 / runge_kutta_1, the
    second stage point being s + 0.5 dt (rk0 / 4 + rk1 / 4) as the reference has it."""
    rk0 = ls_rhs(mesh, p, s, u, vel_bc)
    rk1 = ls_rhs(mesh, p, s + dt * rk0, u, vel_bc)
    rk2 = ls_rhs(mesh, p, s + 0.5 * dt * (rk0 / 4.0 + rk1 / 4.0), u, vel_bc)
    return s + dt * (rk0 / 6.0 + rk1 / 6.0 + 2.0 * rk2 / 3.0)


def ls_props(s, alpha, rho0, rho1, mu0, mu1):
    """ls_step: rho, mu from the smoothed Heaviside tanh(pi s / alpha)."""
    step = np.tanh(np.pi * s / alpha)
    return 0.5 * rho0 * (1 + step) + 0.5 * rho1 * (1 - step), 0.5 * mu0 * (1 + step) + 0.5 * mu1 * (1 - step)


def lagrange_extrapolate(times, fields, t):
    """The initial guess through the pressure history (initial_guess_extrapolation)."""
    out = np.zeros_like(fields[0])
    for i, (ti, fi) in enumerate(zip(times, fields)):
        w = 1.0
        for j, tj in enumerate(times):
            if j != i:
                w *= (t - tj) / (ti - tj)
        out += w * fi
    return out


class TwoPhaseStep:
    """MPINSSolver3D::step on host arrays: advection (+ body force), pressure
    (Neumann data, right-hand side, solve with factor 1/rho, gradient / rho and the
    velocity projection), viscosity (right-hand side, three Helmholtz solves with
    factor mu and mass factor g0 Re rho / dt, zero Dirichlet data on no-slip
    walls), the level-set step, then the time-step update. Solves run to rel_tol."""

    def __init__(self, mesh, p, vel_bc, reynolds, rho0, rho1, mu0, mu1, gravity=0.0, ls_alpha=24.0, cfl=1.0,
                 history=3, rel_tol=1e-11, reinit_freq=24, reinit_ic=1, ls_cap=1.0, over_int=False):
        self.mesh, self.p = mesh, p
        self.t = D.ref_tables(3, p)
        self.om = O.OMesh(self.t, mesh.export(p, self.t))
        self.vel_bc = np.asarray(vel_bc, np.int32).reshape(-1)
        assert np.all((self.vel_bc >= BC_NO_SLIP) & (self.vel_bc <= BC_OUTFLOW))
        self.pr_bct = np.where(self.vel_bc == BC_OUTFLOW, 0, 1).astype(np.int32)  # Dirichlet / Neumann
        # velocity: Dirichlet 0 on no-slip walls, slip, Neumann on outflow; with a slip wall
        # the three components are one vector solve (uses_slip_bcs, ViscousSolver3D)
        self.slip = bool(np.any(self.vel_bc == BC_SLIP))
        vt = np.select([self.vel_bc == BC_NO_SLIP, self.vel_bc == BC_SLIP], [0, 2], 1).astype(np.int32)
        self.vis_bct = np.repeat(vt[None], 3, axis=0) if self.slip else vt
        self.nullspace = int(np.all(self.pr_bct == 1))
        self.re, self.rho0, self.rho1, self.mu0, self.mu1 = reynolds, rho0, rho1, mu0, mu1
        self.grav, self.cfl, self.history, self.rel_tol = gravity, cfl, history, rel_tol
        self.reinit_freq, self.reinit_ic, self.ls_cap = reinit_freq, reinit_ic, ls_cap
        self.over_int = over_int
        fs = mesh.fscale[mesh.nbr >= 0]
        self.h = 1.0 / fs.max()
        self.alpha = ls_alpha / fs.min()

    def _props(self):
        self.rho, self.mu = ls_props(self.s, self.alpha, self.rho0, self.rho1, self.mu0, self.mu1)

    def _next_dt(self):
        self.max_vel = max(1.0, float(np.sqrt(np.max(np.sum(self.vel ** 2, axis=0)))))
        self.dt = self.cfl * self.h / ((self.p + 1) ** 2 * self.max_vel)

    def set_state(self, vel, s):
        self.vel = np.array(vel, dtype=np.float64)
        self.vel_old = self.vel.copy()
        self.s = np.array(s, dtype=np.float64)
        K, Np, Nfp = self.mesh.K, self.t["Np"], self.t["Nfp"]
        self.N_old = np.zeros((3, K, Np))
        self.dPdN_old = np.zeros((K, 4, Nfp))
        self.pr = np.zeros((K, Np))
        self.hist = []
        self.time = 0.0
        self.a0, self.a1, self.b0, self.b1, self.g0 = 1.0, 0.0, 1.0, 0.0, 1.0
        self.reinit_counter = 0
        if self.reinit_ic:
            self.s = ls_reinit(self.mesh, self.p, self.s, self.ls_cap)
        self._props()
        self._next_dt()

    def _solve(self, b, bct, x0, **kw):
        x, info = O.solve(self.om, b[None], bct, precond=O.PRE_JACOBI, rel_tol=self.rel_tol, abs_tol=1e-300,
                          max_iter=20000, x0=x0[None], **kw)
        return x[0], info

    def _solve_oi(self, rhs, x0):
        """update_pressure_matrices_oi (mp_ins_solver.cpp:524-544): 1/rho of the level
        set at the volume and surface cubature points (the element's interpolant of s
        there), the over-integrated operator as the solve's operator (its nodal
        projection for the Jacobi preconditioner only)."""
        import oi_oracle as OI
        m, t = self.mesh, self.t
        e_x = m.export(self.p, t)
        xyz = np.stack([e_x["x"], e_x["y"], e_x["z"]], -1)
        xv, xs = OI.points(m, self.p)  # 3 x K x nq, 3 x K x Nf x nqs
        K, nq = xv.shape[1], xv.shape[2]
        Nf, nqs = xs.shape[2], xs.shape[3]
        sv, ss = np.zeros((K, nq)), np.zeros((K, Nf, nqs))
        for e in range(K):
            pol = _ElementPoly(t, m.G[e], xyz[e, 0], self.s[e])
            sv[e] = pol.value(xv[:, e].T)
            ss[e] = pol.value(xs[:, e].reshape(3, -1).T).reshape(Nf, nqs)
        rho_v, _ = ls_props(sv, self.alpha, self.rho0, self.rho1, self.mu0, self.mu1)
        rho_s, _ = ls_props(ss, self.alpha, self.rho0, self.rho1, self.mu0, self.mu1)
        fv, fs = 1.0 / rho_v, 1.0 / rho_s
        cb = OI.outer_mult(m, self.p, fv, fs, self.pr_bct)
        nodal = fv @ OI.projection(3, self.p).T
        return self._solve(rhs, self.pr_bct, x0, factor=nodal, nullspace=self.nullspace, outer_mult=cb)

    def step(self):
        m, p, dt = self.mesh, self.p, self.dt
        N, velT = advection(m, p, dt, self.a0, self.a1, self.b0, self.b1, self.vel, self.vel_old, self.N_old,
                            self.vel_bc, self.grav)
        dPdN = pressure_neumann(m, p, self.vel, N, self.mu, self.rho, self.vel_bc, self.re, self.grav)
        rhs, _ = O.pressure_rhs(self.om, dt, velT, dPdN, self.dPdN_old, self.b0, self.b1)
        if self.history and self.hist:
            x0 = lagrange_extrapolate([h[0] for h in self.hist], [h[1] for h in self.hist], self.time + dt)
        else:
            x0 = self.pr
        if self.over_int:
            self.pr, self.pr_info = self._solve_oi(rhs, x0)
        else:
            self.pr, self.pr_info = self._solve(rhs, self.pr_bct, x0, factor=1.0 / self.rho, nullspace=self.nullspace)
        if self.history:
            self.hist = (self.hist + [(self.time + dt, self.pr.copy())])[-self.history:]
        dp = O.grad_central(self.om, self.pr) / self.rho[None]
        velTT, _ = O.project_velocity(self.om, dt, dt, dp, velT)
        M, J = self.t["M"], m.J
        mmf = self.g0 * self.re / dt * self.rho
        vel_new = np.zeros_like(self.vel)
        b = np.stack([J[:, None] * ((self.re / dt * self.rho * velTT[c]) @ M.T) for c in range(3)])
        if self.slip:
            x, _ = O.solve(self.om, b, self.vis_bct, precond=O.PRE_JACOBI, rel_tol=self.rel_tol, abs_tol=1e-300,
                           max_iter=20000, x0=self.vel_old, factor=self.mu, mm=mmf)
            vel_new[:] = x
        else:
            for c in range(3):
                vel_new[c], _ = self._solve(b[c], self.vis_bct, self.vel_old[c], factor=self.mu, mm=mmf)
        self.s = ls_advect(m, p, dt, self.s, vel_new, self.vel_bc)
        self.reinit_counter += 1
        if self.reinit_freq > 0 and self.reinit_counter >= self.reinit_freq:
            self.s = ls_reinit(m, p, self.s, self.ls_cap)
            self.reinit_counter = 0
        self._props()
        self.vel_old, self.vel, self.N_old, self.dPdN_old = self.vel, vel_new, N, dPdN
        self.time += dt
        self.a0, self.a1, self.b0, self.b1, self.g0 = 2.0, -0.5, 2.0, -1.0, 1.5
        self._next_dt()


# ---- level-set reinitialisation (LevelSetSolver3D::reinitLS, src/solvers/3d/ls_solver.cpp:
# 719-860; sampleInterface and simplified_newton, src/solvers/3d/ls_solver_cpu.cpp:291-487;
# newton_kernel and newton_method, ls_solver.cpp:259-480), in the deterministic form the
# library runs: each element's own polynomial instead of the stencil fit, samples started at
# the reference nodes scaled by 0.75 and dropped when the sampling Newton fails (no random
# restarts), brute-force closest samples instead of the KD-tree, no kink detection.

def _mono_exps(p):
    return [(a, b, n - a - b) for n in range(p + 1) for a in range(n, -1, -1) for b in range(n - a, -1, -1)]


class _ElementPoly:
    """The nodal interpolant of one element as a polynomial in its reference coordinates,
    evaluated at physical points: value, gradient and Hessian (xx, yy, zz, xy, xz, yz)."""

    def __init__(self, t, G, x0, sval):
        self.ex = _mono_exps(t["order"])
        r0 = np.array([t["r"][0], t["s"][0], t["t"][0]])
        self.r0, self.G, self.x0 = r0, G, x0
        V = np.array([[t["r"][i] ** a * t["s"][i] ** b * t["t"][i] ** c for (a, b, c) in self.ex]
                      for i in range(t["Np"])])
        self.c = np.linalg.solve(V, sval)

    def ref(self, x):
        return self.r0 + self.G @ (np.asarray(x) - self.x0)

    def value(self, x):
        """Values at the physical points x (n x 3)."""
        r = self.r0[None] + (np.asarray(x) - self.x0[None]) @ self.G.T
        return sum(ck * r[:, 0] ** a * r[:, 1] ** b * r[:, 2] ** c for ck, (a, b, c) in zip(self.c, self.ex))

    def to_phys(self, r):
        return self.x0 + np.linalg.solve(self.G, np.asarray(r) - self.r0)

    def eval(self, x):
        r = self.ref(x)
        v, g, H = 0.0, np.zeros(3), np.zeros((3, 3))
        for ck, e in zip(self.c, self.ex):
            p = [r[d] ** e[d] for d in range(3)]
            dp = [e[d] * r[d] ** (e[d] - 1) if e[d] > 0 else 0.0 for d in range(3)]
            ddp = [e[d] * (e[d] - 1) * r[d] ** (e[d] - 2) if e[d] > 1 else 0.0 for d in range(3)]
            v += ck * p[0] * p[1] * p[2]
            g += ck * np.array([dp[0] * p[1] * p[2], p[0] * dp[1] * p[2], p[0] * p[1] * dp[2]])
            for i in range(3):
                for j in range(3):
                    f = [p[0], p[1], p[2]]
                    if i == j:
                        f[i] = ddp[i]
                    else:
                        f[i], f[j] = dp[i], dp[j]
                    H[i, j] += ck * f[0] * f[1] * f[2]
        gx = self.G.T @ g
        Hx = self.G.T @ H @ self.G
        return v, gx, np.array([Hx[0, 0], Hx[1, 1], Hx[2, 2], Hx[0, 1], Hx[0, 2], Hx[1, 2]])

    def inside(self, x, eps=1e-10):
        r = self.ref(x)
        return r[0] >= -1 - eps and r[1] >= -1 - eps and r[2] >= -1 - eps and r.sum() <= -1 + eps


def _solve4(A, b):
    """newtoncp_gepp (ls_solver.cpp:259-295): Gaussian elimination with partial pivoting."""
    A, b = A.copy(), b.copy()
    for i in range(4):
        j = i + int(np.argmax(np.abs(A[i:, i])))
        if abs(A[j, i]) <= abs(A[i, i]):
            j = i
        if j != i:
            A[[i, j]] = A[[j, i]]
            b[[i, j]] = b[[j, i]]
        if abs(A[i, i]) < 1.0e4 * np.finfo(float).eps:
            return None
        f = 1.0 / A[i, i]
        A[i + 1:, i] *= f
        for r in range(i + 1, 4):
            A[r, i + 1:] -= A[r, i] * A[i, i + 1:]
            b[r] -= A[r, i] * b[i]
    for i in range(3, -1, -1):
        b[i] = (b[i] - A[i, i + 1:] @ b[i + 1:]) / A[i, i]
    return b


def ls_reinit(mesh, p, s, ls_cap=1.0):
    """The reinitialised level set (K, Np) of s (K, Np)."""
    t = D.ref_tables(3, p)
    e_x = mesh.export(p, t)
    xyz = np.stack([e_x["x"], e_x["y"], e_x["z"]], -1)  # K x Np x 3
    K, Np = s.shape
    h = 1.0 / mesh.fscale[mesh.nbr >= 0].min()
    tol = max(1e-18, 1e-4 * h * h)
    polys, samples, scell = {}, [], []
    cells = [e for e in range(K) if np.any((s[e] >= 0.0) != (s[e, 0] >= 0.0))]
    for e in cells:
        pol = _ElementPoly(t, mesh.G[e], xyz[e, 0], s[e])
        polys[e] = pol
        for j in range(Np):
            x = pol.to_phys(0.75 * np.array([t["r"][j], t["s"][j], t["t"][j]]))
            conv = False
            for _ in range(100):
                v, g, _h = pol.eval(x)
                sq = g @ g
                if sq > 1e-14:
                    g = g * (v / sq)
                x = x - g
                if g @ g < tol:
                    conv = True
                    break
            samples.append(x if conv and pol.inside(x) else np.full(3, np.nan))
            scell.append(e)
    out = np.where(s < 0.0, -ls_cap, ls_cap).astype(float)
    if not samples:
        return out
    S = np.array(samples)
    Sf = np.where(np.isnan(S), np.inf, S)
    pts = xyz.reshape(-1, 3)
    near = np.empty(len(pts), dtype=int)
    for i0 in range(0, len(pts), 4096):
        d2 = ((pts[i0:i0 + 4096, None, :] - Sf[None]) ** 2).sum(-1)
        near[i0:i0 + 4096] = np.argmin(d2, axis=1)
    valid = ~np.isnan(S[:, 0])
    w = ls_cap + 2.0 * h
    flat = s.reshape(-1)
    res = out.reshape(-1)
    for node in range(len(pts)):
        first = node // Np * Np
        b0, bi = near[first], near[node]
        if not (valid[b0] and valid[bi]):
            continue
        d0 = ((S[b0] - pts[first]) ** 2).sum()
        if d0 >= w * w:
            continue
        d1 = ((S[bi] - pts[node]) ** 2).sum()
        pol = polys[scell[bi]]
        nx = pts[node]
        pt = S[bi].copy()
        init = pt.copy()
        lam, conv = 0.0, False
        for step in range(50):
            old = pt.copy()
            v, g, hx = pol.eval(pt)
            g2 = g @ g
            if g2 < 1e-14:
                break
            if step == 0:
                lam = ((nx - pt) @ g) / g2
            f = np.array([*(pt - nx + lam * g), v])
            H = np.array([[1 + lam * hx[0], lam * hx[3], lam * hx[4], g[0]],
                          [lam * hx[3], 1 + lam * hx[1], lam * hx[5], g[1]],
                          [lam * hx[4], lam * hx[5], 1 + lam * hx[2], g[2]],
                          [g[0], g[1], g[2], 0.0]])
            sol = _solve4(H, f)
            if sol is None:
                lam = ((nx - pt) @ g) / g2
                d1v = (v / g2) * g
                d2v = pt - nx + lam * g
                m2 = d2v @ d2v
                if m2 > 0.01 * h * h:
                    d2v = d2v * (0.1 * h / np.sqrt(m2))
                pt = pt - (d1v + d2v)
            else:
                m2 = sol[:3] @ sol[:3]
                if m2 > 0.25 * h * h:
                    sol = sol * (0.5 * h / np.sqrt(m2))
                pt = pt - sol[:3]
                lam -= sol[3]
            if ((init - pt) ** 2).sum() > 2.25 * h * h:
                pt = old
                break
            if ((old - pt) ** 2).sum() < 1e-24:
                conv = True
                break
        dist2 = ((pt - nx) ** 2).sum() if conv else d1
        res[node] = (-1.0 if flat[node] < 0.0 else 1.0) * np.sqrt(dist2)
    return np.clip(res.reshape(K, Np), -ls_cap, ls_cap)
