"""Algebraic coarse hierarchy below p=1 (host build, no GPU): the continuous
P1 Galerkin operator against the DG operator of the oracle, Galerkin identities
of the aggregation levels."""
import ctypes as C

import numpy as np
import pytest

import oracle_py as O
import sipg
from helpers import random_case


def dense_dg_operator(om, bct, f):
    n = om.K * om.Np
    A = np.zeros((n, n))
    for j in range(n):
        x = np.zeros((1, om.K, om.Np))
        x.reshape(-1)[j] = 1.0
        A[:, j] = O.mult(om, x, bct, f).reshape(-1)
    return A


def csr_dense(t):
    rows, cols, ptr, idx, val = t
    M = np.zeros((rows, cols))
    for i in range(rows):
        M[i, idx[ptr[i]:ptr[i + 1]]] += val[ptr[i]:ptr[i + 1]]
    return M


@pytest.mark.parametrize("dirichlet", [True, False])
def test_p1_coarse_operator_is_galerkin_of_dg_operator(dirichlet):
    mesh, t, e, om, x, f, m, bct = random_case(3, 2, 1, 1, seed=12)
    bct[:] = 0 if dirichlet else 1
    tau = np.zeros((mesh.K, 4))
    O.oracle_lib().oracle_tau(C.byref(om.s), O._d(np.ascontiguousarray(f)), O._d(tau))
    amg = sipg.Amg.p1(mesh, f, tau, (bct[0] == 0).astype(np.int32), coarse_max=10, strength=0.08,
                      singular=not dirichlet)
    A1 = dense_dg_operator(om, bct, f)
    P = csr_dense(amg.csr(-1, 1))
    A0 = csr_dense(amg.csr(0, 0))
    G = P.T @ A1 @ P
    assert np.abs(G - A0).max() < 1e-12 * np.abs(A0).max()
    if not dirichlet:
        # without Dirichlet faces only the volume term survives: symmetric, constants in the kernel
        assert np.allclose(A0, A0.T, atol=1e-12 * np.abs(A0).max())
        assert np.abs(A0 @ np.ones(A0.shape[0])).max() < 1e-12 * np.abs(A0).max()


def test_aggregation_levels_are_galerkin_products():
    mesh, t, e, om, x, f, m, bct = random_case(3, 4, 1, 1, seed=2)
    bct[:] = 0
    tau = np.zeros((mesh.K, 4))
    O.oracle_lib().oracle_tau(C.byref(om.s), O._d(np.ascontiguousarray(f)), O._d(tau))
    amg = sipg.Amg.p1(mesh, f, tau, np.ones(mesh.Kb, np.int32), coarse_max=20, strength=0.08)
    assert amg.nlevels >= 2
    for l in range(amg.nlevels - 1):
        A, P, R = (csr_dense(amg.csr(l, w)) for w in (0, 1, 2))
        Ac = csr_dense(amg.csr(l + 1, 0))
        assert np.allclose(R, P.T)
        assert np.abs(R @ A @ P - Ac).max() < 1e-12 * np.abs(Ac).max()
        assert P.shape[1] < P.shape[0]
    inv = amg.coarse_inverse()
    Ac = csr_dense(amg.csr(amg.nlevels - 1, 0))
    assert np.abs(inv @ Ac - np.eye(Ac.shape[0])).max() < 1e-8


def test_weak_threshold_still_coarsens():
    """A strength threshold that leaves most connections weak (0.25 on a P1
    Laplacian) is lowered level by level, so every level keeps at most 60 % of
    the rows above it and the set-up stays fast."""
    import time
    mesh, t, e, om, x, f, m, bct = random_case(3, 10, 1, 1, seed=5)
    tau = np.zeros((mesh.K, 4))
    O.oracle_lib().oracle_tau(C.byref(om.s), O._d(np.ascontiguousarray(f)), O._d(tau))
    t0 = time.perf_counter()
    amg = sipg.Amg.p1(mesh, f, tau, np.zeros(mesh.Kb, np.int32), coarse_max=50, strength=0.25, singular=True)
    assert time.perf_counter() - t0 < 20.0
    rows = [amg.csr(l, 0)[0] for l in range(amg.nlevels)]
    assert len(rows) >= 2 and rows[-1] == amg.coarse_n
    for a, b in zip(rows, rows[1:]):
        assert b <= 0.6 * a
