"""Over-integrated factor SIPG operator (the factor at cubature points), restated
from its bilinear form in physical coordinates. TEST INFRASTRUCTURE ONLY
(tests/, the CPU legs of the benchmark).

The library's stand-in for FactorPoissonMatrixFreeDiagOI3D (OP2-DG-Toolkit,
unvendored; selected at src/solvers/3d/mp_ins_solver.cpp:81-88, fed in
update_pressure_matrices_oi :524-544 with 1/rho at the volume and surface
cubature points after mp_ins_3d_pr_fact_oi_0/1, and its CUB3D_PROJ projection
as the nodal factor). Parity against the toolkit is unpinned (neither its
operator nor its cubature rules are in the reference tree); the restatement is
pinned by properties: with a constant factor it equals the nodal operator (whose
oracle is pinned against the reference's own kernels), it is symmetric, and its
rules are exact to the stated degrees.

Form, per element e and test function phi_i (n the outward normal of e, sJ the
face's surface Jacobian, weights in the reference / face-parameter domains):
  volume      sum_q w_q J f_q grad(phi_i) . grad(u)
  interior    sJ [ -1/2 sum_s w_s f-_s (n . grad u-)(x_s) phi_i(x_s)     own points
                   -1/2 sum_t w_t f+_t (n . grad u+)(x_t) phi_i(x_t)     neighbour's points
                   -1/2 sum_s w_s f-_s (n . grad phi_i)(x_s) [u](x_s)    own points
                   +tau/2 sum_s w_s [u](x_s) phi_i(x_s) ]                 [u] = u- - u+
  Dirichlet   sJ [ -sum_s w_s f_s (n . grad u) phi_i - sum_s w_s f_s (n . grad phi_i) u
                   + tau sum_s w_s u phi_i ]
  tau = 2(p+1)(p+2) max(fscale- max_s f-_s, fscale+ max_t f+_t) (boundary: own side)
Rules: collapsed Gauss-Legendre, p + 2 points per direction in the volume
(exact to degree 2p + 1), p + 1 on the faces (exact to 2p), face points given by
their barycentric coordinates in the face's vertex order.
"""
import ctypes as C
import itertools

import numpy as np

import dg_oracle as D


def _collapsed(dim, n):
    x, w = np.polynomial.legendre.leggauss(n)
    if dim == 1:
        return x[:, None], w
    pts, wts = [], []
    if dim == 2:
        for i, j in itertools.product(range(n), repeat=2):
            a, b = x[i], x[j]
            pts.append(((1 + a) * (1 - b) / 2 - 1, b))
            wts.append(w[i] * w[j] * (1 - b) / 2)
    else:
        for i, j, k in itertools.product(range(n), repeat=3):
            a, b, c = x[i], x[j], x[k]
            pts.append(((1 + a) * (1 - b) * (1 - c) / 4 - 1, (1 + b) * (1 - c) / 2 - 1, c))
            wts.append(w[i] * w[j] * w[k] * (1 - b) * (1 - c) ** 2 / 8)
    return np.array(pts), np.array(wts)


def rules(dim, p):
    """(rq: nq x dim reference points, wq, lam: nqs x dim face barycentrics, ws)."""
    rq, wq = _collapsed(dim, p + 2)
    a, ws = _collapsed(dim - 1, p + 1)
    if dim == 3:
        l1, l2 = (1 + a[:, 0]) / 2, (1 + a[:, 1]) / 2
        lam = np.stack([1 - l1 - l2, l1, l2], 1)
    else:
        lam = np.stack([(1 - a[:, 0]) / 2, (1 + a[:, 0]) / 2], 1)
    return rq, wq, lam, ws


def basis(dim, p, r):
    """Nodal basis of order p at reference points r (n x dim): (phi n x Np,
    dphi dim x n x Np reference derivatives)."""
    t = D.nodes(dim, p)
    ex = D._exponents(dim, p)
    Vi = np.linalg.inv(D._mono(ex, *[(1 + c) / 2 for c in t]))
    z = np.zeros(len(r))
    xyz = [(1 + r[:, d]) / 2 for d in range(dim)] + [z] * (3 - dim)
    phi = D._mono(ex, *xyz) @ Vi
    dphi = np.stack([0.5 * D._mono_grad(ex, *xyz, d) @ Vi for d in range(dim)])
    return phi, dphi


def _ref_coords(mesh, e, x):
    """Reference coordinates in elements e (K') of physical points x (K' x n x dim)."""
    P0 = mesh.vx[mesh.e2v[e, 0]]
    return np.einsum("ecd,end->enc", mesh.G[e], x - P0[:, None, :]) - 1.0


def points(mesh, p):
    """Physical coordinates of the volume points (dim x K x nq) and the surface
    points (dim x K x Nf x nqs), the layout of sipg_op_oi_points_host."""
    dim, K = mesh.dim, mesh.K
    rq, _, lam, _ = rules(dim, p)
    P = mesh.vx[mesh.e2v]
    F = 0.5 * (P[:, 1:, :] - P[:, :1, :])  # K x dim(c) x dim(d): dx_d / dr_c
    xv = P[:, :1, :] + np.einsum("qc,ecd->eqd", rq + 1.0, F)
    xs = np.stack([np.einsum("sa,ead->esd", lam, P[:, list(fv), :]) for fv in D.FACE_VERTS[dim]], 1)
    return np.moveaxis(xv, 2, 0), np.moveaxis(xs, 3, 0)


def projection(dim, p):
    """Np x nq: the L2 projection of volume-point values onto the nodes."""
    t = D.ref_tables(dim, p)
    rq, wq, _, _ = rules(dim, p)
    phi, _ = basis(dim, p, rq)
    return np.linalg.solve(t["M"], (wq[:, None] * phi).T)


def apply(mesh, p, u, fvol, fsurf, bc_types, mm=None):
    """y = A u for the over-integrated operator (scalar, u: K x Np); mm: K x Np
    nodal mass coefficient (J M diag(mm)) or None."""
    dim, K = mesh.dim, mesh.K
    t = D.ref_tables(dim, p)
    Nf = dim + 1
    rq, wq, lam, ws = rules(dim, p)
    bct = np.asarray(bc_types).reshape(-1)
    _, dphq = basis(dim, p, rq)
    gx = np.einsum("ecd,cqi->edqi", mesh.G, dphq)  # physical gradients at the volume points
    gu = np.einsum("edqi,ei->edq", gx, u)
    y = np.einsum("edqi,edq->ei", gx, (wq[None, None, :] * mesh.J[:, None, None] * fvol[:, None, :]) * gu)
    cpen = 2.0 * (p + 1) * (p + 2)
    xs_all = points(mesh, p)[1]  # dim x K x Nf x nqs
    nrm = np.stack([mesh.nx, mesh.ny, mesh.nz][:dim], 2)  # K x Nf x dim
    for f in range(Nf):
        nb = mesh.nbr[:, f]
        inner = nb >= 0
        bnd = ~inner
        dirich = np.zeros(K, bool)
        dirich[bnd] = bct[-nb[bnd] - 1] == D.BC_DIRICHLET
        act = inner | dirich
        if not act.any():
            continue
        e = np.where(act)[0]
        xs = np.moveaxis(xs_all[:, e, f, :], 0, 2)  # E x nqs x dim
        n = nrm[e, f]
        sJ = mesh.sJ[e, f]
        fs = sJ / mesh.J[e]
        fm = fsurf[e, f]
        own = _ref_coords(mesh, e, xs)
        ph, dph = basis(dim, p, own.reshape(-1, dim))
        ph = ph.reshape(len(e), -1, t["Np"])
        gph = np.einsum("ecd,cesi->esdi", mesh.G[e], dph.reshape(dim, len(e), -1, t["Np"]))
        dn = np.einsum("ed,esdi->esi", n, gph)  # n . grad phi_i at own points
        um = np.einsum("esi,ei->es", ph, u[e])
        dnum = np.einsum("esi,ei->es", dn, u[e])
        tau = cpen * fs * fm.max(axis=1)
        isin = inner[e]
        ue = np.zeros_like(um)
        if isin.any():
            ei, k = e[isin], nb[e[isin]]
            g = mesh.nbr_face[ei, f]
            # the neighbour at this element's points
            rn = _ref_coords(mesh, k, xs[isin])
            phn, _ = basis(dim, p, rn.reshape(-1, dim))
            ue[isin] = np.einsum("esi,ei->es", phn.reshape(len(ei), -1, t["Np"]), u[k])
            # the neighbour's own points of the shared face
            xt = np.moveaxis(xs_all[:, k, g, :], 0, 2)
            rk = _ref_coords(mesh, k, xt)
            _, dpk = basis(dim, p, rk.reshape(-1, dim))
            gk = np.einsum("ecd,cesi->esdi", mesh.G[k], dpk.reshape(dim, len(ei), -1, t["Np"]))
            dnup = np.einsum("ed,esdi,ei->es", n[isin], gk, u[k])  # n- . grad u+ at the neighbour's points
            re = _ref_coords(mesh, ei, xt)
            phe, _ = basis(dim, p, re.reshape(-1, dim))
            phe = phe.reshape(len(ei), -1, t["Np"])
            fp = fsurf[k, g]
            tau[isin] = np.maximum(tau[isin], cpen * (mesh.sJ[ei, f] / mesh.J[k]) * fp.max(axis=1))
            # -1/2 sum_t w_t f+_t (n . grad u+) phi_i at the neighbour's points
            yB = -0.5 * np.einsum("s,es,es,esi->ei", ws, fp, dnup, phe)
            y[ei] += sJ[isin, None] * yB
        h = np.where(isin, 0.5, 1.0)
        jump = np.where(isin[:, None], um - ue, 2.0 * um)
        yA = -h[:, None] * np.einsum("s,es,es,esi->ei", ws, fm, dnum, ph)
        yC = -0.5 * np.einsum("s,es,esi,es->ei", ws, fm, dn, jump)
        yD = 0.5 * tau[:, None] * np.einsum("s,es,esi->ei", ws, jump, ph)
        y[e] += sJ[:, None] * (yA + yC + yD)
    if mm is not None:
        y += mesh.J[:, None] * ((mm * u) @ t["M"].T)
    return y


def outer_mult(mesh, p, fvol, fsurf, bc_types):
    """An oracle_mult_fn (oracle_solver_opts.outer_mult) applying this operator
    to the outer solve's vectors; keep the returned object alive during the solve."""
    K, Np = mesh.K, D.sizes(mesh.dim, p)[0]
    FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_int,
                     C.POINTER(C.POINTER(C.c_double)), C.POINTER(C.POINTER(C.c_double)))

    def cb(_m, ncomp, _bct, _f, _mm, _mms, _flags, xs, ys):
        x = np.ctypeslib.as_array(xs[0], shape=(K * Np,)).reshape(K, Np)
        y = np.ctypeslib.as_array(ys[0], shape=(K * Np,)).reshape(K, Np)
        y[:] = apply(mesh, p, x, fvol, fsurf, bc_types)
        return 0
    return FN(cb)
