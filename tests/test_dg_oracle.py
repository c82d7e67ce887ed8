"""The numpy restatement of the reference element, meshes and workloads
(oracle/dg_oracle.py) against the library's own construction (CPU only).

The two are built differently (monomial basis with closed-form simplex
integrals against a Legendre basis with collapsed quadrature; sorted-key face
matching against a hash scan), so agreement to round-off pins each against the
other where the unvendored OP2-DG-Toolkit cannot.
"""
import numpy as np
import pytest

import dg_oracle as D
import sipg
import workloads as W


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / scale if a.size else 0.0


@pytest.mark.parametrize("dim,order", [(d, p) for d in (2, 3) for p in (1, 2, 3, 4)])
def test_reference_tables_match_the_library(dim, order):
    a, b = sipg.ref_tables(dim, order), D.ref_tables(dim, order)
    # the monomial Vandermonde at p = 4 has a condition number near 1e3: 1e-12
    for k in ("r", "s", "t", "Dr", "Ds", "Dt", "M", "MMF", "EMAT"):
        assert rel(b[k], a[k]) < 1e-12, k
    for k in ("fmask", "perm_pos"):
        assert np.array_equal(a[k], b[k]), k
    for q in range(1, order):
        assert rel(D.interp_matrix(dim, q, order), sipg.interp_matrix(dim, q, order)) < 1e-12


@pytest.mark.parametrize("dim,n,jitter,seed", [(2, 6, 0.1, 3), (2, 4, 0.0, 0), (3, 3, 0.1, 77), (3, 4, 0.2, 5)])
def test_box_meshes_and_exports_match_the_library(dim, n, jitter, seed):
    vx, e2v = sipg.box_mesh(dim, n, jitter, seed)
    vx2, e2v2 = D.box_mesh(dim, n, jitter, seed)
    assert np.array_equal(vx, vx2) and np.array_equal(e2v, e2v2)
    m1, m2 = sipg.Mesh(dim, vx, e2v), D.Mesh(dim, vx2, e2v2)
    assert (m1.K, m1.F, m1.Kb) == (m2.K, m2.F, m2.Kb)
    for order in (1, 3):
        a, b = m1.export(order), m2.export(order)
        for k, v in a.items():
            if isinstance(v, np.ndarray):
                if v.dtype.kind == "i":
                    assert np.array_equal(v, b[k]), k
                else:
                    assert np.abs(v - b[k]).max() <= 1e-13 * max(1.0, np.abs(v).max()), k
            else:
                assert v == b[k], k


def test_two_phase_workload_matches_the_library():
    a = W.poisson3d_two_phase(4, order=3, n_modes=64)
    b = D.poisson3d_two_phase(4, order=3, n_modes=64)
    assert rel(b["factor"], a["factor"]) < 1e-14
    assert rel(b["rhs"], a["rhs"]) < 1e-12
    assert np.array_equal(a["bc_types"], b["bc_types"]) and a["pin"] == b["pin"]


def test_helmholtz_workload_matches_the_library():
    a, b = W.helmholtz3d(3), D.helmholtz3d(3)
    assert np.array_equal(a["x"], b["x"]) and np.array_equal(a["bc_types"], b["bc_types"])
    assert a["mm"] == b["mm"]
