"""Reference element tables: exactness identities (no GPU)."""
import numpy as np
import pytest

import sipg


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("order", [1, 2, 3, 4])
def test_derivatives_exact_on_polynomials(dim, order):
    t = sipg.ref_tables(dim, order)
    r, s, tt = t["r"], t["s"], t["t"]
    # d/dr of r^order, d/ds of s^order * r^0, d/dt of t^order
    p = order
    assert np.allclose(t["Dr"] @ r**p, p * r ** (p - 1), atol=1e-11)
    assert np.allclose(t["Ds"] @ s**p, p * s ** (p - 1), atol=1e-11)
    if dim == 3:
        assert np.allclose(t["Dt"] @ tt**p, p * tt ** (p - 1), atol=1e-11)
    assert np.allclose(t["Dr"] @ np.ones_like(r), 0, atol=1e-12)


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("order", [1, 2, 3, 4])
def test_mass_and_face_mass(dim, order):
    t = sipg.ref_tables(dim, order)
    one = np.ones(t["Np"])
    vol = 2.0 if dim == 2 else 4.0 / 3.0
    assert abs(one @ t["M"] @ one - vol) < 1e-12
    assert np.allclose(t["M"], t["M"].T, atol=1e-15)
    assert np.linalg.eigvalsh(t["M"]).min() > 0
    # each face parameter domain has measure 2 (edge length / reference triangle area)
    for f in range(t["Nf"]):
        assert abs(one @ t["MMF"][f] @ one - 2.0) < 1e-12
    # EMAT rows are zero off the face nodes
    for f in range(t["Nf"]):
        cols = slice(f * t["Nfp"], (f + 1) * t["Nfp"])
        off = np.setdiff1d(np.arange(t["Np"]), t["fmask"][f])
        assert np.abs(t["EMAT"][off, cols]).max() < 5e-13


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("order", [1, 2, 3, 4])
def test_face_nodes_and_orientation_tables(dim, order):
    t = sipg.ref_tables(dim, order)
    Nfp, Nf = t["Nfp"], t["Nf"]
    assert t["fmask"].shape == (Nf, Nfp)
    for f in range(Nf):
        assert len(set(t["fmask"][f].tolist())) == Nfp
    # identity orientation maps every face node to itself; every table is a permutation
    assert np.array_equal(t["perm_pos"][0], np.arange(Nfp))
    for row in t["perm_pos"]:
        assert sorted(row.tolist()) == list(range(Nfp))


@pytest.mark.parametrize("dim", [2, 3])
def test_interp_matrix_reproduces_polynomials(dim):
    for q, p in ((1, 2), (2, 3), (1, 3), (3, 4)):
        P = sipg.interp_matrix(dim, q, p)
        tq, tp = sipg.ref_tables(dim, q), sipg.ref_tables(dim, p)
        fq = tq["r"] ** q + tq["s"]
        fp = tp["r"] ** q + tp["s"]
        assert np.allclose(P @ fq, fp, atol=1e-12)
        assert np.allclose(P.sum(axis=1), 1.0, atol=1e-12)
