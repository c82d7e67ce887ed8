"""The over-integrated operator's oracle (oracle/oi_oracle.py) pinned by properties:
rules exact to their stated degrees, the nodal operator (oracle_mult, pinned against
the reference's kernels) when the factor is constant, symmetric for a varying factor,
and the L2 projection exact on polynomials of the element's order."""
import math

import numpy as np
import pytest

import dg_oracle as D
import oi_oracle as OI
import oracle_py as O


def _exact_monomial(dim, a):
    """Integral of prod_d ((1 + r_d) / 2)^a_d over the reference simplex."""
    s = sum(a)
    return (2.0 ** dim) * math.prod(math.factorial(k) for k in a) / math.factorial(s + dim)


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_rules_are_exact_to_their_degrees(dim, p):
    rq, wq, lam, ws = OI.rules(dim, p)
    for a in D._exponents(dim, 2 * p + 1):
        approx = np.sum(wq * np.prod([((1 + rq[:, d]) / 2) ** a[d] for d in range(dim)], axis=0))
        assert abs(approx - _exact_monomial(dim, a)) < 1e-13
    # face rule in the face barycentrics (measure 2 = the mass matrices' face measure)
    for a in D._exponents(dim, 2 * p):
        b = list(a[:dim - 1])
        approx = np.sum(ws * np.prod([lam[:, 1 + d] ** b[d] for d in range(dim - 1)], axis=0))
        assert abs(approx - _exact_monomial(dim - 1, b)) < 1e-13


CASES = [(3, 3, 1, 0), (3, 3, 2, 1), (3, 3, 3, 2), (2, 6, 2, 0), (2, 6, 3, 2), (2, 5, 4, 1)]


def _bct(mesh, kind):
    if kind == 2:
        return (np.arange(mesh.Kb) % 2).astype(np.int32)[None]
    return np.full((1, mesh.Kb), kind, np.int32)


@pytest.mark.parametrize("dim,n,p,bnd", CASES)
def test_constant_factor_equals_the_nodal_operator(dim, n, p, bnd):
    mesh = D.Mesh.box(dim, n, 0.1, 3)
    t = D.ref_tables(dim, p)
    e = mesh.export(p, t)
    bct = _bct(mesh, bnd)
    rng = np.random.default_rng(p)
    u = rng.uniform(-1, 1, (mesh.K, t["Np"]))
    nq, nqs = len(OI.rules(dim, p)[1]), len(OI.rules(dim, p)[3])
    y = OI.apply(mesh, p, u, np.ones((mesh.K, nq)), np.ones((mesh.K, dim + 1, nqs)), bct)
    want = O.mult(O.OMesh(t, e), u[None], bct)[0]
    assert np.abs(y - want).max() < 1e-12 * np.abs(want).max()


def _two_phase_at(xyz, n):
    z = xyz[2] if xyz.shape[0] == 3 else np.full_like(xyz[0], 0.5)
    return 1.0 / D.two_phase_rho(xyz[0], xyz[1], z, 1.0 / n, ratio=100.0)


@pytest.mark.parametrize("dim,n,p,bnd", CASES)
def test_varying_factor_operator_is_symmetric(dim, n, p, bnd):
    mesh = D.Mesh.box(dim, n, 0.1, 3)
    bct = _bct(mesh, bnd)
    xv, xs = OI.points(mesh, p)
    fv, fs = _two_phase_at(xv, n), _two_phase_at(xs, n)
    Np = D.sizes(dim, p)[0]
    rng = np.random.default_rng(7)
    u, v = rng.uniform(-1, 1, (2, mesh.K, Np))
    Au = OI.apply(mesh, p, u, fv, fs, bct)
    Av = OI.apply(mesh, p, v, fv, fs, bct)
    assert abs(np.sum(v * Au) - np.sum(u * Av)) < 1e-12 * abs(np.sum(u * Au))


@pytest.mark.parametrize("dim,p", [(2, 3), (3, 2), (3, 3)])
def test_projection_reproduces_polynomials(dim, p):
    rq = OI.rules(dim, p)[0]
    phi, _ = OI.basis(dim, p, rq)
    P = OI.projection(dim, p)
    assert np.abs(P @ phi - np.eye(phi.shape[1])).max() < 1e-11
