"""The numpy / scipy restatement of the algebraic coarse hierarchy
(oracle/amg_oracle.py) against the library's host build (CPU only): the same
aggregates, level operators, transfers and coarsest inverse on jittered meshes
with a two-phase factor, for Neumann (singular) and Dirichlet problems, and on
the configuration the benchmark solves."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

import amg_oracle as A
import dg_oracle as D
import oracle_py as O
import sipg


def csr(t):
    rows, cols, ptr, idx, val = t
    return sp.csr_matrix((val, idx, ptr), shape=(rows, cols))


def build_both(n, dirichlet, coarse_max, seed=20261203):
    case = D.poisson3d_two_phase(n, order=3, n_modes=16, seed=seed)
    mesh = case["mesh"]
    t1 = D.ref_tables(3, 1)
    e1 = mesh.export(1, t1)
    f1 = np.ascontiguousarray(case["factor"] @ D.interp_matrix(3, 3, 1).T)
    om1 = O.OMesh(t1, e1)
    tau1 = np.zeros((mesh.K, 4))
    O.oracle_lib().oracle_tau(C.byref(om1.s), O._d(f1), O._d(tau1))
    bd = np.full(mesh.Kb, 1 if dirichlet else 0, np.int32)
    A0, Pdg = A.p1_continuous_operator(t1, mesh, f1, tau1, bd)
    mine = A.Hierarchy(A0, Pdg, coarse_max=coarse_max, strength=0.08, singular=not dirichlet)
    lm = sipg.Mesh(3, mesh.vx, mesh.e2v)
    theirs = sipg.Amg.p1(lm, f1, tau1, bd, coarse_max=coarse_max, strength=0.08, singular=not dirichlet)
    return mine, theirs


# (24, False, 2048) is the benchmark's two-phase configuration (24^3 x 6 tets,
# Neumann walls, default coarse size): 15,625 -> 1,919 unknowns; (24, False, 1000)
# one level more (-> 870).
@pytest.mark.parametrize("n,dirichlet,coarse_max", [(4, False, 30), (5, True, 40), (6, False, 100),
                                                    (24, False, 2048), (24, False, 1000)])
def test_hierarchy_matches_the_library(n, dirichlet, coarse_max):
    mine, theirs = build_both(n, dirichlet, coarse_max)
    assert mine.nlevels == theirs.nlevels and mine.coarse_n == theirs.coarse_n
    for lvl in range(mine.nlevels):
        for w in (0, 1, 2) if lvl + 1 < mine.nlevels else (0,):
            a, b = csr(mine.csr(lvl, w)), csr(theirs.csr(lvl, w))
            assert a.shape == b.shape
            # scipy drops products that cancel to exactly zero; compare values
            assert abs(a - b).max() <= 1e-12 * abs(b).max(), (lvl, w)
    for w in (1, 2):
        assert abs(csr(mine.csr(-1, w)) - csr(theirs.csr(-1, w))).max() == 0.0
    ci, cj = mine.coarse_inverse(), theirs.coarse_inverse()
    assert np.abs(ci - cj).max() <= 1e-8 * np.abs(cj).max()
