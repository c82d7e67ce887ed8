"""Reference element, box meshes and workloads restated in numpy.

TEST INFRASTRUCTURE ONLY: used by tests/, the smoke check and the CPU legs of
the benchmark (the reference arm builds its inputs here, so that process never
loads the CUDA library). It restates what the reference takes from the
unvendored OP2-DG-Toolkit (DGConstants: Dr/Ds/Dt, Mass, MM_F0..3, FMASK,
EMAT; DGMesh2D/3D: geof, nx/ny/nz/sJ/fscale, face2cells, faceNum, fmaskL/R,
bface2cells, bfaceNum), as the kernels consume it: geof order
src/kernels/fvmf_3d_grad.h:4-12, per-face data
src/solvers/3d/slip_matrix/factor_viscous_matrix.cpp:213-218, FMASK indexing
src/kernels/fvmf_3d_calc_tau_faces.h:6.

The construction is independent of the library's C++ one:
  * nodes: the published warp-and-blend construction (Hesthaven & Warburton,
    Nodal Discontinuous Galerkin Methods, 2008: Nodes2D sec. 6.1, Nodes3D with
    WarpShiftFace3D sec. 10.2), vectorised over the nodes;
  * operators from the monomial basis x^a y^b z^c of the unit simplex
    (x = (1+r)/2, ...), differentiated exactly, with the mass and face-mass
    matrices from the closed-form Dirichlet integrals
    int x^a y^b z^c = a! b! c! / (a+b+c+dim)!  (no quadrature);
  * meshes: splitmix64 jitter, Kuhn split and face matching by sorting the
    face vertex keys.
The data conventions (node order, face numbering, face-node order, the
orientation codes and the per-face records) are the library's, so both sides
can be compared entry by entry.
"""
import functools
import math

import numpy as np

TWO_PI = 6.283185307179586

# face -> local vertices: 3D face 0: t=-1, 1: s=-1, 2: r+s+t=-1, 3: r=-1;
# 2D face 0: s=-1, 1: r+s=0, 2: r=-1
FACE_VERTS = {3: ((0, 1, 2), (0, 1, 3), (1, 2, 3), (0, 2, 3)), 2: ((0, 1), (1, 2), (0, 2))}
# orientation codes: position a on this face -> position PERMS[s][a] on the neighbour's face
PERMS = {3: ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)), 2: ((0, 1), (1, 0))}
BC_DIRICHLET, BC_NEUMANN, BC_SLIP = 0, 1, 2


def sizes(dim, p):
    Np = (p + 1) * (p + 2) // 2 if dim == 2 else (p + 1) * (p + 2) * (p + 3) // 6
    Nfp = p + 1 if dim == 2 else (p + 1) * (p + 2) // 2
    return Np, Nfp, dim + 1


# ---------------------------------------------------------------- nodes
def _lgl(N):
    """Legendre-Gauss-Lobatto points (ascending)."""
    inner = np.sort(np.polynomial.legendre.Legendre.basis(N).deriv().roots().real)
    return np.concatenate([[-1.0], inner, [1.0]])


def _warpfactor(N, rout):
    """Warpfactor (sec. 6.1): equidistant interpolant of LGL - equidistant, / (1 - r^2)."""
    req = np.linspace(-1.0, 1.0, N + 1)
    disp = _lgl(N) - req
    warp = np.zeros_like(rout)
    for k in range(N + 1):
        lk = np.ones_like(rout)
        for m in range(N + 1):
            if m != k:
                lk = lk * (rout - req[m]) / (req[k] - req[m])
        warp += lk * disp[k]
    inside = np.abs(rout) < 1.0 - 1e-10
    return np.where(inside, warp / np.where(inside, 1.0 - rout * rout, 1.0), 0.0)


def _nodes2d(N):
    alpopt = (0.0, 0.0, 1.4152, 0.1001, 0.2751, 0.9800, 1.0999, 1.2832, 1.3648, 1.4773, 1.4959, 1.5743,
              1.5770, 1.6223, 1.6258)
    alpha = alpopt[N - 1] if N < 16 else 5.0 / 3.0
    L1 = np.array([n / N for n in range(N + 1) for m in range(N + 1 - n)])
    L3 = np.array([m / N for n in range(N + 1) for m in range(N + 1 - n)])
    L2 = 1.0 - L1 - L3
    x = -L2 + L3
    y = (-L2 - L3 + 2.0 * L1) / math.sqrt(3.0)
    w1 = 4 * L2 * L3 * _warpfactor(N, L3 - L2) * (1 + (alpha * L1) ** 2)
    w2 = 4 * L1 * L3 * _warpfactor(N, L1 - L3) * (1 + (alpha * L2) ** 2)
    w3 = 4 * L1 * L2 * _warpfactor(N, L2 - L1) * (1 + (alpha * L3) ** 2)
    x = x + w1 + math.cos(2 * math.pi / 3) * w2 + math.cos(4 * math.pi / 3) * w3
    y = y + math.sin(2 * math.pi / 3) * w2 + math.sin(4 * math.pi / 3) * w3
    l1 = (math.sqrt(3.0) * y + 1.0) / 3.0
    l2 = (-3.0 * x - math.sqrt(3.0) * y + 2.0) / 6.0
    l3 = (3.0 * x - math.sqrt(3.0) * y + 2.0) / 6.0
    return -l2 + l3 - l1, -l2 - l3 + l1, np.zeros_like(l1)


def _evalwarp(p, xnodes, xout):
    """evalwarp (sec. 10.2) with equidistant nodes listed from +1 down to -1."""
    xeq = np.array([-1.0 + 2.0 * (p - i) / p for i in range(p + 1)])
    warp = np.zeros_like(xout)
    for i in range(p + 1):
        d = np.full_like(xout, xnodes[i] - xeq[i])
        for j in range(1, p):
            if i != j:
                d = d * (xout - xeq[j]) / (xeq[i] - xeq[j])
        if i != 0:
            d = -d / (xeq[i] - xeq[0])
        if i != p:
            d = d / (xeq[i] - xeq[p])
        warp += d
    return warp


def _evalshift(p, pval, L1, L2, L3):
    gx = -_lgl(p)
    w1 = L2 * L3 * 4 * _evalwarp(p, gx, L3 - L2) * (1 + (pval * L1) ** 2)
    w2 = L1 * L3 * 4 * _evalwarp(p, gx, L1 - L3) * (1 + (pval * L2) ** 2)
    w3 = L1 * L2 * 4 * _evalwarp(p, gx, L2 - L1) * (1 + (pval * L3) ** 2)
    dx = w1 + math.cos(2 * math.pi / 3) * w2 + math.cos(4 * math.pi / 3) * w3
    dy = math.sin(2 * math.pi / 3) * w2 + math.sin(4 * math.pi / 3) * w3
    return dx, dy


def _nodes3d(p):
    alphastore = (0.0, 0.0, 0.0, 0.1002, 1.1332, 1.5608, 1.3413, 1.2577, 1.1603, 1.10153, 0.6080, 0.4523,
                  0.8856, 0.8717, 0.9655)
    alpha = alphastore[p - 1] if p <= 15 else 1.0
    tol = 1e-10
    idx = [(n, m, q) for n in range(p + 1) for m in range(p + 1 - n) for q in range(p + 1 - n - m)]
    re = np.array([-1.0 + 2.0 * q / p for n, m, q in idx])
    se = np.array([-1.0 + 2.0 * m / p for n, m, q in idx])
    te = np.array([-1.0 + 2.0 * n / p for n, m, q in idx])
    L1, L2, L3, L4 = (1 + te) / 2, (1 + se) / 2, -(1 + re + se + te) / 2, (1 + re) / 2
    s3, s6 = math.sqrt(3.0), math.sqrt(6.0)
    v1 = np.array([-1, -1 / s3, -1 / s6])
    v2 = np.array([1, -1 / s3, -1 / s6])
    v3 = np.array([0, 2 / s3, -1 / s6])
    v4 = np.array([0, 0, 3 / s6])
    t1 = np.array([v2 - v1, v2 - v1, v3 - v2, v3 - v1])
    t2 = np.array([v3 - 0.5 * (v1 + v2), v4 - 0.5 * (v1 + v2), v4 - 0.5 * (v2 + v3), v4 - 0.5 * (v1 + v3)])
    t1 /= np.linalg.norm(t1, axis=1)[:, None]
    t2 /= np.linalg.norm(t2, axis=1)[:, None]
    X = np.outer(L3, v1) + np.outer(L4, v2) + np.outer(L2, v3) + np.outer(L1, v4)
    shift = np.zeros_like(X)
    order = ((L1, L2, L3, L4), (L2, L1, L3, L4), (L3, L1, L4, L2), (L4, L1, L3, L2))
    for face, (La, Lb, Lc, Ld) in enumerate(order):
        w1, w2 = _evalshift(p, alpha, Lb, Lc, Ld)
        blend = Lb * Lc * Ld
        denom = (Lb + 0.5 * La) * (Lc + 0.5 * La) * (Ld + 0.5 * La)
        ok = denom > tol
        blend = np.where(ok, (1 + (alpha * La) ** 2) * blend / np.where(ok, denom, 1.0), blend)
        shift += np.outer(blend * w1, t1[face]) + np.outer(blend * w2, t2[face])
        on_face = (La < tol) & ((Lb > tol).astype(int) + (Lc > tol) + (Ld > tol) < 3)
        shift[on_face] = np.outer(w1[on_face], t1[face]) + np.outer(w2[on_face], t2[face])
    X = X + shift
    A = 0.5 * np.stack([v2 - v1, v3 - v1, v4 - v1], axis=1)
    rst = np.linalg.solve(A, (X - 0.5 * (v2 + v3 + v4 - v1)).T).T
    return rst[:, 0], rst[:, 1], rst[:, 2]


def _bary(dim, r, s, t):
    """Barycentric coordinates of the reference vertices, shape (nverts, n)."""
    if dim == 2:
        return np.stack([-(r + s) / 2, (1 + r) / 2, (1 + s) / 2])
    return np.stack([-(1 + r + s + t) / 2, (1 + r) / 2, (1 + s) / 2, (1 + t) / 2])


def nodes(dim, p):
    r, s, t = _nodes2d(p) if dim == 2 else _nodes3d(p)
    r, s, t = r.copy(), s.copy(), t.copy()
    # coordinates within 1e-12 of a face are put exactly on it
    lam = _bary(dim, r, s, t)
    for i in range(len(r)):
        for v in range(1, dim + 1):
            if abs(lam[v, i]) < 1e-12:
                if v == 1:
                    r[i] = -1.0
                elif v == 2:
                    s[i] = -1.0
                else:
                    t[i] = -1.0
        if abs(_bary(dim, r[i:i + 1], s[i:i + 1], t[i:i + 1])[0, 0]) < 1e-12:
            if dim == 2:
                s[i] = -r[i]
            else:
                t[i] = -1.0 - r[i] - s[i]
    return r, s, t


# ------------------------------------------------------ monomial operators
def _exponents(dim, p):
    if dim == 1:
        return [(a, 0, 0) for a in range(p + 1)]
    if dim == 2:
        return [(a, b, 0) for a in range(p + 1) for b in range(p + 1 - a)]
    return [(a, b, c) for a in range(p + 1) for b in range(p + 1 - a) for c in range(p + 1 - a - b)]


def _mono(ex, x, y, z):
    return np.stack([x ** a * y ** b * z ** c for a, b, c in ex], axis=1)


def _mono_grad(ex, x, y, z, d):
    cols = []
    for e in ex:
        k = e[d]
        if k == 0:
            cols.append(np.zeros_like(x))
            continue
        e2 = list(e)
        e2[d] -= 1
        cols.append(k * x ** e2[0] * y ** e2[1] * z ** e2[2])
    return np.stack(cols, axis=1)


def _dirichlet_gram(ex, dim):
    """G[m][n] = integral over the unit simplex of monomial m times monomial n."""
    G = np.zeros((len(ex), len(ex)))
    for i, a in enumerate(ex):
        for j, b in enumerate(ex):
            s = [a[k] + b[k] for k in range(3)]
            G[i, j] = (math.factorial(s[0]) * math.factorial(s[1]) * math.factorial(s[2])
                       / math.factorial(sum(s) + dim))
    return G


def ref_tables(dim, p):
    """Reference-element tables in the library's conventions (row-major)."""
    Np, Nfp, Nf = sizes(dim, p)
    r, s, t = nodes(dim, p)
    x, y, z = (1 + r) / 2, (1 + s) / 2, (1 + t) / 2
    ex = _exponents(dim, p)
    V = _mono(ex, x, y, z)
    Vi = np.linalg.inv(V)
    D = [0.5 * _mono_grad(ex, x, y, z, d) @ Vi for d in range(dim)]
    # the unit simplex is the reference one scaled by 1/2 per axis: volume factor 2^dim
    M = (2.0 ** dim) * Vi.T @ _dirichlet_gram(ex, dim) @ Vi
    lam = _bary(dim, r, s, t)
    fmask = np.zeros((Nf, Nfp), np.int32)
    fb = []
    for f, fv in enumerate(FACE_VERTS[dim]):
        opp = [v for v in range(dim + 1) if v not in fv][0]
        on = [i for i in range(Np) if abs(lam[opp, i]) <= 1e-10]
        assert len(on) == Nfp
        keys = [tuple(lam[a, i] for a in fv) for i in on]

        def cmp(j, k):  # lexicographic on the face barycentrics, equal within 1e-9
            for a, b in zip(keys[j], keys[k]):
                if abs(a - b) > 1e-9:
                    return -1 if a < b else 1
            return 0
        order = sorted(range(Nfp), key=functools.cmp_to_key(cmp))
        fmask[f] = [on[j] for j in order]
        fb.append(np.array([keys[j] for j in order]))
    for f in range(1, Nf):
        assert np.abs(fb[f] - fb[0]).max() < 1e-9
    perms = PERMS[dim]
    perm_pos = np.zeros((len(perms), Nfp), np.int32)
    for sg, sigma in enumerate(perms):
        for j in range(Nfp):
            target = np.zeros(dim)
            target[list(sigma)] = fb[0][j]
            hit = np.where(np.abs(fb[0] - target).max(axis=1) < 1e-9)[0]
            perm_pos[sg, j] = hit[0]
    # face mass in the face parameter domain (reference triangle of area 2, or
    # interval of length 2): unit-face monomials in the face barycentrics of
    # face vertices 1 and 2, scaled by the area ratio 2^(dim-1)
    exf = _exponents(dim - 1, p)
    Gf = _dirichlet_gram(exf, dim - 1)
    MMF = np.zeros((Nf, Np, Np))
    EMAT = np.zeros((Np, Nf * Nfp))
    for f in range(Nf):
        u = fb[f][:, 1]
        v = fb[f][:, 2] if dim == 3 else np.zeros(Nfp)
        Vf = _mono(exf, u, v, np.zeros(Nfp))
        Vfi = np.linalg.inv(Vf)
        MF = (2.0 ** (dim - 1)) * Vfi.T @ Gf @ Vfi
        MMF[f][np.ix_(fmask[f], fmask[f])] = MF
        EMAT[fmask[f], f * Nfp:(f + 1) * Nfp] = MF
    return dict(r=r, s=s, t=t, Dr=D[0], Ds=D[1], Dt=D[2] if dim == 3 else np.zeros((Np, Np)), M=M, MMF=MMF,
                EMAT=EMAT, fmask=fmask, perm_pos=perm_pos, Np=Np, Nfp=Nfp, Nf=Nf, dim=dim, order=p)


def interp_matrix(dim, q, p):
    """Order-q nodal values -> order-p nodes (Np(p) x Np(q)): the order-q Lagrange
    basis evaluated at the order-p nodes."""
    rq = nodes(dim, q)
    rp = nodes(dim, p)
    ex = _exponents(dim, q)
    Vq = _mono(ex, *[(1 + c) / 2 for c in rq])
    Vp = _mono(ex, *[(1 + c) / 2 for c in rp])
    return Vp @ np.linalg.inv(Vq)


# -------------------------------------------------------------------- mesh
def _splitmix_uniform(seed, count):
    """`count` splitmix64 draws mapped to [0, 1) by their top 53 bits."""
    mask = (1 << 64) - 1
    s = seed & mask
    out = np.empty(count)
    for i in range(count):
        s = (s + 0x9E3779B97F4A7C15) & mask
        z = s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
        z ^= z >> 31
        out[i] = (z >> 11) * (1.0 / 9007199254740992.0)
    return out


def box_mesh(dim, n, jitter=0.0, seed=0):
    """Unit square (n x n quads, 2 triangles each along the (0,0)-(1,1) diagonal)
    or unit cube (n^3 hexes, 6 Kuhn tetrahedra each); interior vertices jittered
    by U(-jitter h, jitter h) per coordinate (every vertex draws, boundary ones
    discard theirs)."""
    h = 1.0 / n
    m = n + 1
    nv = m ** dim
    u = _splitmix_uniform(seed, nv * dim).reshape(nv, dim)
    d = (2 * u - 1) * jitter * h
    grid = np.indices((m,) * dim).reshape(dim, -1)[::-1].T  # vertex id = i + m j (+ m^2 k), i fastest
    vx = grid * h
    interior = np.all((grid > 0) & (grid < n), axis=1)
    vx[interior] += d[interior]

    def vid(*c):
        return sum(ci * m ** a for a, ci in enumerate(c))
    e2v = []
    if dim == 2:
        for j in range(n):
            for i in range(n):
                a, b, c, dd = vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)
                e2v += [(a, b, c), (a, c, dd)]
    else:
        axes = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))
        for k in range(n):
            for j in range(n):
                for i in range(n):
                    for ax in axes:
                        c = [0, 0, 0]
                        v0 = vid(i, j, k)
                        c[ax[0]] = 1
                        v1 = vid(i + c[0], j + c[1], k + c[2])
                        c[ax[1]] = 1
                        v2 = vid(i + c[0], j + c[1], k + c[2])
                        e2v.append((v0, v1, v2, vid(i + 1, j + 1, k + 1)))
    return vx, np.array(e2v, dtype=np.int32)


class Mesh:
    """Simplicial mesh: orientation, affine geometric factors, face matching."""

    def __init__(self, dim, vx, e2v):
        self.dim = dim
        self.vx = np.asarray(vx, dtype=np.float64)
        e2v = np.array(e2v, dtype=np.int32)
        K = e2v.shape[0]
        P = self.vx[e2v]  # K x nv x dim
        F = 0.5 * (P[:, 1:, :] - P[:, :1, :]).transpose(0, 2, 1)  # F[e][d][c] = dx_d / dr_c
        det = np.linalg.det(F)
        flip = det < 0
        e2v[flip, 1], e2v[flip, 2] = e2v[flip, 2].copy(), e2v[flip, 1].copy()
        self.e2v = e2v
        self.K = K
        P = self.vx[e2v]
        F = 0.5 * (P[:, 1:, :] - P[:, :1, :]).transpose(0, 2, 1)
        J = np.linalg.det(F)
        G = np.linalg.inv(F)  # G[e][c][d] = dr_c / dx_d
        self.J, self.G = J, G
        if dim == 3:
            self.geof = np.concatenate([G.reshape(K, 9), J[:, None]], axis=1)
            nrm = np.stack([-G[:, 2], -G[:, 1], G[:, 0] + G[:, 1] + G[:, 2], -G[:, 0]], axis=1)
        else:
            self.geof = np.stack([G[:, 0, 0], G[:, 0, 1], G[:, 1, 0], G[:, 1, 1], J], axis=1)
            nrm = np.stack([-G[:, 1], G[:, 0] + G[:, 1], -G[:, 0]], axis=1)
        ln = np.linalg.norm(nrm, axis=2)
        self.nx = nrm[:, :, 0] / ln
        self.ny = nrm[:, :, 1] / ln
        self.nz = nrm[:, :, 2] / ln if dim == 3 else np.zeros_like(ln)
        self.sJ = ln * J[:, None]
        self.fscale = self.sJ / J[:, None]
        self._match_faces()

    def _match_faces(self):
        dim, K = self.dim, self.K
        Nf = dim + 1
        fv = np.array(FACE_VERTS[dim])
        gv = self.e2v[:, fv]  # K x Nf x dim global face vertices
        key = np.sort(gv, axis=2).reshape(K * Nf, dim)
        order = np.lexsort(key.T[::-1])
        ks = key[order]
        same = np.all(ks[1:] == ks[:-1], axis=1)
        first = order[:-1][same]
        second = order[1:][same]
        lo, hi = np.minimum(first, second), np.maximum(first, second)
        byclose = np.argsort(hi, kind="stable")
        lo, hi = lo[byclose], hi[byclose]
        self.face2cells = np.stack([lo // Nf, hi // Nf], axis=1).astype(np.int32)
        self.faceNum = np.stack([lo % Nf, hi % Nf], axis=1).astype(np.int32)
        perms = np.array(PERMS[dim])

        def sigma(a_idx, b_idx):
            ga = gv.reshape(K * Nf, dim)[a_idx]
            gb = gv.reshape(K * Nf, dim)[b_idx]
            pos = np.argmax(ga[:, :, None] == gb[:, None, :], axis=2)  # own position a -> neighbour position
            return np.argmax(np.all(pos[:, None, :] == perms[None, :, :], axis=2), axis=1)
        self.sLR = sigma(lo, hi)
        self.sRL = sigma(hi, lo)
        self.nbr = np.zeros(K * Nf, np.int32)
        self.nbr_face = np.zeros(K * Nf, np.int32)
        self.nbr_perm = np.zeros(K * Nf, np.int32)
        self.nbr[lo], self.nbr[hi] = hi // Nf, lo // Nf
        self.nbr_face[lo], self.nbr_face[hi] = hi % Nf, lo % Nf
        self.nbr_perm[lo], self.nbr_perm[hi] = self.sLR, self.sRL
        matched = np.zeros(K * Nf, bool)
        matched[lo] = matched[hi] = True
        bidx = np.where(~matched)[0]
        self.nbr[bidx] = -(np.arange(len(bidx)) + 1)
        self.bface2cell = (bidx // Nf).astype(np.int32)
        self.bfaceNum = (bidx % Nf).astype(np.int32)
        self.bface_centroid = self.vx[gv.reshape(K * Nf, dim)[bidx]].mean(axis=1)
        self.nbr = self.nbr.reshape(K, Nf)
        self.nbr_face = self.nbr_face.reshape(K, Nf)
        self.nbr_perm = self.nbr_perm.reshape(K, Nf)
        self.F, self.Kb = len(lo), len(bidx)

    @classmethod
    def box(cls, dim, n, jitter=0.0, seed=0):
        return cls(dim, *box_mesh(dim, n, jitter, seed))

    def export(self, order, tables=None):
        """Per-order data in the reference's form (the library's export layout)."""
        t = tables or ref_tables(self.dim, order)
        dim, Nfp = self.dim, t["Nfp"]
        fm, pp = t["fmask"], t["perm_pos"]
        fL, fR = self.faceNum[:, 0], self.faceNum[:, 1]
        fmaskL = fm[fL]
        fmaskR = fm[fR[:, None], pp[self.sLR]]
        lam = _bary(dim, t["r"], t["s"], t["t"])  # nv x Np
        P = self.vx[self.e2v]  # K x nv x dim
        X = np.einsum("vi,evd->edi", lam, P)
        d = dict(geof=self.geof, nx=self.nx, ny=self.ny, nz=self.nz, sJ=self.sJ, fscale=self.fscale,
                 face2cells=self.face2cells, faceNum=self.faceNum, fmaskL=fmaskL.astype(np.int32),
                 fmaskR=fmaskR.astype(np.int32), bface2cell=self.bface2cell, bfaceNum=self.bfaceNum,
                 bface_centroid=self.bface_centroid, x=X[:, 0], y=X[:, 1],
                 z=X[:, 2] if dim == 3 else np.zeros_like(X[:, 0]),
                 K=self.K, F=self.F, Kb=self.Kb, Np=t["Np"], Nfp=Nfp, Nf=t["Nf"], dim=dim, order=order)
        return d


# --------------------------------------------------------------- workloads
def mass_apply(export, tables, f):
    """b = J M f per element (mesh->mass), f: (K, Np)."""
    return export["geof"][:, -1][:, None] * (f @ tables["M"].T)


def grf(points, corr_len=0.1, n_modes=256, seed=7):
    """Gaussian random field at points (N, dim): sqrt(2/n) sum_k cos(k.x + phase_k),
    wavevectors N(0, 1/corr_len^2) per axis, phases U(0, 2 pi), numpy PCG64(seed)."""
    rng = np.random.default_rng(seed)
    k = rng.normal(0.0, 1.0 / corr_len, (n_modes, points.shape[1]))
    ph = rng.uniform(0.0, 2 * np.pi, n_modes)
    out = np.zeros(points.shape[0])
    chunk = 1 << 15
    for s in range(0, points.shape[0], chunk):
        out[s:s + chunk] = np.cos(points[s:s + chunk] @ k.T + ph).sum(axis=1)
    return out * np.sqrt(2.0 / n_modes)


def two_phase_rho(x, y, z, h, ratio=1000.0, radius=0.25, center=(0.5, 0.5, 0.5), width=1.5):
    r = np.sqrt((x - center[0]) ** 2 + (y - center[1]) ** 2 + (z - center[2]) ** 2)
    return 1.0 + (ratio - 1.0) * 0.5 * (1.0 + np.tanh((radius - r) / (width * h)))


def poisson3d_two_phase(n, order=3, jitter=0.1, seed=20261203, rhs_seed=7, n_modes=256, pin=True):
    """3D variable-density Poisson on n^3 x 6 jittered tets: factor 1/rho (rho 1000
    in a sphere r = 0.25 at the centre, 1 outside, tanh over 1.5 h), right-hand side
    J M (GRF - its mass-weighted mean), Neumann walls, optionally DOF (0, 0) pinned."""
    mesh = Mesh.box(3, n, jitter, seed)
    t = ref_tables(3, order)
    e = mesh.export(order, t)
    rho = two_phase_rho(e["x"], e["y"], e["z"], 1.0 / n)
    pts = np.stack([e["x"].ravel(), e["y"].ravel(), e["z"].ravel()], 1)
    f = grf(pts, 0.1, n_modes, rhs_seed).reshape(e["K"], t["Np"])
    b = mass_apply(e, t, f)
    f = f - b.sum() / mass_apply(e, t, np.ones_like(f)).sum()
    b = mass_apply(e, t, f)
    if pin:
        b[0, 0] = 0.0
    bct = np.full((1, e["Kb"]), BC_NEUMANN, np.int32)
    return dict(mesh=mesh, export=e, tables=t, factor=1.0 / rho, rhs=b[None], bc_types=bct,
                pin=(0, 0) if pin else None, rho=rho)


def helmholtz3d(n, order=4, nu=1e-3, dt=1e-3, seed=11, jitter=0.1):
    """3D Helmholtz (I/(nu dt) - Laplacian), Dirichlet walls, input U(-1, 1)."""
    mesh = Mesh.box(3, n, jitter, 20261203)
    Np = sizes(3, order)[0]
    x = np.random.default_rng(seed).uniform(-1.0, 1.0, (1, mesh.K, Np))
    bct = np.full((1, mesh.Kb), BC_DIRICHLET, np.int32)
    return dict(mesh=mesh, x=x, bc_types=bct, mm=1.0 / (nu * dt), order=order)
