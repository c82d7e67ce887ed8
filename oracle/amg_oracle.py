"""Algebraic coarse hierarchy of the p-multigrid restated with numpy / scipy.sparse.

TEST INFRASTRUCTURE ONLY (tests/, the smoke check, the CPU legs of the
benchmark). The reference solves its p = 1 coarse problem with PETSc's
algebraic multigrid (`coarse_solver = petsc`, `[petsc-amg]`,
examples/3d/oscillating_droplet/config.ini:24-31,52-64; PETScPMultigrid is in
the unvendored OP2-DG-Toolkit). The design restated here, and implemented
separately in the library:
  * coarse space: continuous piecewise linears on the mesh vertices, injected
    into the p = 1 DG nodes (P_dg, R_dg = P_dg^T);
  * its operator: the exact Galerkin product of the p = 1 SIPG operator, which
    for continuous functions keeps the volume term J sum_d Dx_d^T M F Dx_d and
    the Dirichlet face terms sJ (tau MF - MF F Dn - Dn^T MF F) (+ J M c for a
    mass term), assembled per element (fvmf_3d_mult_flux.h:13-22 and
    factor_viscous_matrix.cpp:233-286 give the apply these are the Galerkin
    entries of);
  * smoothed aggregation below it: greedy aggregation over strong connections
    |a_ij| >= theta sqrt(a_ii a_jj), tentative piecewise-constant prolongator
    smoothed by (I - 4/(3 rho) D^-1 A), rho the Gershgorin bound of D^-1 A,
    Galerkin coarse operators R A P, until at most coarse_max unknowns; a level
    that keeps more than 60 % of its rows is aggregated again with theta / 4
    (up to three times); the coarsest level is inverted densely (a 1e-8 relative
    diagonal shift and the projection onto the complement of the constants for a
    singular, pure Neumann problem).
"""
import numpy as np
import scipy.sparse as sp

MIN_COARSENING = 0.6
MAX_DENSE_COARSE = 8192


def p1_continuous_operator(tables1, mesh, factor1, tau1, bc_dirichlet, mm_mode=0, mm_scalar=0.0, mm1=None):
    """Galerkin operator of the p = 1 SIPG operator on continuous P1 (Nv x Nv CSR)
    and the vertex-to-DG-node injection P_dg ((K Np) x Nv).

    tables1: order-1 reference tables; mesh: dg_oracle.Mesh; factor1, mm1: K x Np1
    (None: 1 / absent); tau1: K x Nf; bc_dirichlet: per boundary face 0/1."""
    dim, K, Np = mesh.dim, mesh.K, tables1["Np"]
    assert Np == dim + 1
    Dm = np.stack([tables1["Dr"], tables1["Ds"], tables1["Dt"]][:dim])  # dim x Np x Np
    M = tables1["M"]
    G = mesh.G  # K x dim(r) x dim(x)
    J = mesh.J
    f = np.ones((K, Np)) if factor1 is None else np.asarray(factor1)
    Dx = np.einsum("erd,rij->edij", G, Dm)  # d/dx_d at the nodes
    T = J[:, None, None, None] * np.einsum("ik,ek,edkj->edij", M, f, Dx)
    B = np.einsum("edki,edkj->eij", Dx, T)
    bd = np.asarray(bc_dirichlet).astype(bool)
    for b in np.where(bd)[0]:
        e, fc = mesh.bface2cell[b], mesh.bfaceNum[b]
        n = np.array([mesh.nx[e, fc], mesh.ny[e, fc], mesh.nz[e, fc]])[:dim]
        Dn = np.einsum("r,rij->ij", G[e] @ n, Dm)
        mf = tables1["MMF"][fc]
        fe = f[e]
        term = mf @ (fe[:, None] * Dn) + (Dn.T @ mf) * fe[None, :]
        B[e] += mesh.sJ[e, fc] * (tau1[e, fc] * mf - term)
    if mm_mode == 1:
        B += mm_scalar * J[:, None, None] * M[None]
    elif mm_mode == 2:
        B += J[:, None, None] * M[None] * np.asarray(mm1)[:, None, :]
    v = mesh.e2v
    rows = np.repeat(v, Np, axis=1).ravel()
    cols = np.tile(v, (1, Np)).ravel()
    Nv = mesh.vx.shape[0]
    A = sp.csr_matrix((B.ravel(), (rows, cols)), shape=(Nv, Nv))
    A.sum_duplicates()
    A.sort_indices()
    Pdg = sp.csr_matrix((np.ones(K * Np), (np.arange(K * Np), v.ravel())), shape=(K * Np, Nv))
    return A, Pdg


def _aggregate(A, theta):
    n = A.shape[0]
    ptr, idx, val = A.indptr, A.indices, A.data
    diag = A.diagonal()
    agg = -np.ones(n, dtype=np.int64)

    def strong(i, k):
        j = idx[k]
        return j != i and abs(val[k]) >= theta * np.sqrt(abs(diag[i] * diag[j]))
    na = 0
    for i in range(n):  # seeds whose strong neighbourhood is still free
        if agg[i] >= 0:
            continue
        ks = range(ptr[i], ptr[i + 1])
        if any(strong(i, k) and agg[idx[k]] >= 0 for k in ks):
            continue
        agg[i] = na
        for k in ks:
            if strong(i, k):
                agg[idx[k]] = na
        na += 1
    for i in range(n):  # leftovers join their strongest aggregated neighbour
        if agg[i] >= 0:
            continue
        best, bw = -1, 0.0
        for k in range(ptr[i], ptr[i + 1]):
            j = idx[k]
            if j == i or agg[j] < 0:
                continue
            if abs(val[k]) > bw:
                bw, best = abs(val[k]), agg[j]
        if best >= 0:
            agg[i] = best
        else:
            agg[i] = na
            na += 1
    return agg, na


class Hierarchy:
    """Same accessors as the library's host hierarchy: nlevels, coarse_n,
    csr(level, 0 A / 1 P / 2 R) and csr(-1, 1 P_dg / 2 R_dg), coarse_inverse()."""

    def __init__(self, A0, Pdg, coarse_max=1000, strength=0.08, singular=False):
        self.A, self.P, self.R = [A0.tocsr()], [], []
        self.Pdg, self.Rdg = Pdg.tocsr(), Pdg.T.tocsr()
        while self.A[-1].shape[0] > coarse_max and len(self.A) < 16:
            A = self.A[-1]
            theta = strength
            agg, na = _aggregate(A, theta)
            for _ in range(3):
                if na <= MIN_COARSENING * A.shape[0]:
                    break
                theta *= 0.25
                agg, na = _aggregate(A, theta)
            if na > MIN_COARSENING * A.shape[0] or na < 1:
                break
            n = A.shape[0]
            Tm = sp.csr_matrix((np.ones(n), (np.arange(n), agg)), shape=(n, na))
            d = A.diagonal()
            dinv = np.where(d != 0.0, 1.0 / np.where(d != 0.0, d, 1.0), 0.0)
            rho = (abs(A).sum(axis=1).A1 * np.abs(dinv)).max()
            S = sp.identity(n, format="csr") - (4.0 / (3.0 * rho)) * sp.diags(dinv) @ A
            P = (S @ Tm).tocsr()
            P.sort_indices()
            R = P.T.tocsr()
            R.sort_indices()
            Ac = (R @ (A @ P)).tocsr()
            Ac.sort_indices()
            self.P.append(P)
            self.R.append(R)
            self.A.append(Ac)
        self.singular = singular
        self._coarse()

    def reuse(self, A0):
        """The hierarchy of a new level-0 operator with the same sparsity, keeping
        this one's aggregates and prolongators (PETSc GAMG with reuse-interpolation,
        the reference's `[petsc-amg] reuse-interpolation = 1`,
        examples/3d/oscillating_droplet/config.ini:59): only the Galerkin
        products and the coarsest inverse are recomputed."""
        h = object.__new__(Hierarchy)
        h.P, h.R, h.Pdg, h.Rdg, h.singular = self.P, self.R, self.Pdg, self.Rdg, self.singular
        h.A = [A0.tocsr()]
        for P, R in zip(self.P, self.R):
            Ac = (R @ (h.A[-1] @ P)).tocsr()
            Ac.sort_indices()
            h.A.append(Ac)
        h._coarse()
        return h

    def _coarse(self):
        singular = self.singular
        C = self.A[-1].toarray()
        n = C.shape[0]
        if n > MAX_DENSE_COARSE:
            raise RuntimeError("algebraic coarsening stalled")
        if singular:
            C = C + 1e-8 * np.abs(np.diag(C)).max() * np.eye(n)
        inv = np.linalg.inv(C)
        if singular:
            inv = inv - inv.sum(axis=1, keepdims=True) / n - inv.sum(axis=0, keepdims=True) / n + inv.sum() / n**2
        self.inv = inv
        self.nlevels = len(self.A)
        self.coarse_n = n

    def csr(self, level, which):
        if level < 0:
            m = self.Pdg if which == 1 else self.Rdg
        else:
            m = (self.A, self.P, self.R)[which][level] if (which == 0 or level < len(self.P)) else None
            if m is None:
                return 0, 0, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0)
        m = m.tocsr()
        m.sort_indices()
        return (m.shape[0], m.shape[1], m.indptr.astype(np.int32), m.indices.astype(np.int32),
                m.data.astype(np.float64))

    def coarse_inverse(self):
        return self.inv
