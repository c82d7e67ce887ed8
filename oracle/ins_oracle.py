"""The steps of the 3D incompressible time step around the pressure and viscous
solves, restated in numpy. TEST INFRASTRUCTURE ONLY (tests/, the CPU legs of
the benchmark).

pressure_neumann: the curl-curl Neumann data of the multiphase pressure step,
MPINSSolver3D::apply_pressure_neumann_bc (src/solvers/3d/mp_ins_solver.cpp:450-493).

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


def pressure_neumann(mesh, p, u, N, mu, rho, vel_bc, reynolds):
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
            res = -N[:, e, m] - c2[:, e, m] / (reynolds * rho[e, m])
            out[e, f] = mesh.fscale[e, f] * (nrm[e, f] @ res)
    return out


def advection(mesh, p, dt, a0, a1, b0, b1, u, u_old, N_old, vel_bc):
    """(N, velT) of one advection step."""
    N = nonlinear(mesh, p, u, vel_bc)
    velT = (a0 * u + a1 * u_old) - dt * (b0 * N + b1 * N_old)
    return N, velT
