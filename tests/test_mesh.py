"""Mesh builder: connectivity, orientation and geometry (no GPU)."""
import numpy as np
import pytest

import sipg


@pytest.mark.parametrize("dim,n", [(2, 6), (3, 3)])
@pytest.mark.parametrize("order", [1, 3, 4])
def test_face_matching_and_geometry(dim, n, order):
    mesh = sipg.Mesh.box(dim, n, jitter=0.1, seed=5)
    e = mesh.export(order)
    K, F, Kb, Nf = e["K"], e["F"], e["Kb"], e["Nf"]
    assert K == (2 * n * n if dim == 2 else 6 * n**3)
    assert 2 * F + Kb == Nf * K
    assert Kb == (4 * n if dim == 2 else 12 * n * n)
    X = np.stack([e["x"], e["y"], e["z"]], -1)
    for fc in range(F):
        eL, eR = e["face2cells"][fc]
        fL, fR = e["faceNum"][fc]
        assert np.abs(X[eL, e["fmaskL"][fc]] - X[eR, e["fmaskR"][fc]]).max() < 1e-13
        nL = np.array([e["nx"][eL, fL], e["ny"][eL, fL], e["nz"][eL, fL]])
        nR = np.array([e["nx"][eR, fR], e["ny"][eR, fR], e["nz"][eR, fR]])
        assert np.abs(nL + nR).max() < 1e-12
        assert abs(e["sJ"][eL, fL] - e["sJ"][eR, fR]) < 1e-12 * e["sJ"][eL, fL]
    J = e["geof"][:, -1]
    assert (J > 0).all()
    vol = J.sum() * (2.0 if dim == 2 else 4.0 / 3.0)
    assert abs(vol - 1.0) < 1e-12
    # boundary faces lie on the unit box
    c = e["bface_centroid"]
    on = np.isclose(c, 0.0, atol=1e-14) | np.isclose(c, 1.0, atol=1e-14)
    assert on.any(axis=1).all()


def test_fscale_is_sJ_over_J():
    mesh = sipg.Mesh.box(3, 2, jitter=0.1, seed=1)
    e = mesh.export(2)
    assert np.allclose(e["fscale"], e["sJ"] / e["geof"][:, 9:10], rtol=1e-14)


def test_jitter_is_seeded_and_bounded():
    vx1, _ = sipg.box_mesh(3, 4, 0.1, 20261203)
    vx2, _ = sipg.box_mesh(3, 4, 0.1, 20261203)
    vx0, _ = sipg.box_mesh(3, 4, 0.0, 20261203)
    assert np.array_equal(vx1, vx2)
    assert np.abs(vx1 - vx0).max() <= 0.1 / 4 + 1e-15
