"""The time-step kernels around the solves against the time-step oracle
(oracle/ins_oracle.py, itself pinned against the reference's kernels in
tests/test_ins_oracle.py): the fused non-linear advection step, the curl-curl
pressure Neumann data and the level-set reinitialisation."""
import numpy as np
import pytest

import dg_oracle as D
import ins_oracle as I
import sipg
from helpers import rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("scale", [0.5, 3.0], ids=["slow", "fast"])
def test_advection_matches_the_oracle(p, scale):
    n = 3
    gm = sipg.Mesh.box(3, n, jitter=0.1, seed=5)
    om = D.Mesh.box(3, n, 0.1, 5)
    Np = sipg.ref_sizes(3, p)[0]
    rng = np.random.default_rng(10 + p)
    u, u_old, N_old = rng.uniform(-scale, scale, (3, 3, gm.K, Np))
    vel_bc = (np.arange(gm.Kb) % 3).astype(np.int32)
    args = (1e-3, 2.0, -0.5, 2.0, -1.0)
    N, velT = sipg.ins_advection(gm, p, *args, u, u_old, N_old, vel_bc)
    Nw, velTw = I.advection(om, p, *args, u, u_old, N_old, vel_bc)
    # p = 4: the oracle's monomial-basis reference tables agree with the library's to
    # about 1e-13, which the derivatives of the quadratic flux amplify (1.1e-11 measured)
    tol = 1e-12 if p < 4 else 1e-10
    assert rel_err(N, Nw) < tol
    assert rel_err(velT, velTw) < tol


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_pressure_neumann_data_match_the_oracle(p):
    n = 3
    gm = sipg.Mesh.box(3, n, jitter=0.1, seed=5)
    om = D.Mesh.box(3, n, 0.1, 5)
    Np = sipg.ref_sizes(3, p)[0]
    rng = np.random.default_rng(30 + p)
    u, N = rng.uniform(-1, 1, (2, 3, gm.K, Np))
    mu = rng.uniform(1.0, 100.0, (gm.K, Np))
    rho = rng.uniform(1.0, 1000.0, (gm.K, Np))
    vel_bc = (np.arange(gm.Kb) % 3).astype(np.int32)
    got = sipg.ins_pressure_neumann(gm, p, 123.0, u, N, mu, rho, vel_bc)
    want = I.pressure_neumann(om, p, u, N, mu, rho, vel_bc, 123.0)
    # two derivative passes amplify the last-bit differences of the reference tables
    assert rel_err(got, want) < (1e-12 if p < 4 else 1e-10)
    # outflow faces and interior faces carry no data
    assert np.all(got[want == 0.0] == 0.0)


def test_pressure_neumann_data_vanish_without_walls():
    gm = sipg.Mesh.box(3, 2, jitter=0.1, seed=1)
    Np = sipg.ref_sizes(3, 2)[0]
    rng = np.random.default_rng(3)
    u, N = rng.uniform(-1, 1, (2, 3, gm.K, Np))
    ones = np.ones((gm.K, Np))
    got = sipg.ins_pressure_neumann(gm, 2, 10.0, u, N, ones, ones, np.full(gm.Kb, 2, np.int32))
    assert not got.any()


def _reinit_case(n, p):
    gm = sipg.Mesh.box(3, n, jitter=0.1, seed=5)
    om = D.Mesh.box(3, n, 0.1, 5)
    e = om.export(p, D.ref_tables(3, p))
    d = np.sqrt((e["x"] - 0.5) ** 2 + (e["y"] - 0.3) ** 2 + (e["z"] - 0.5) ** 2) - 0.25
    return gm, om, e, 2.0 * d + 0.05 * np.sin(5.0 * e["x"]) * np.cos(3.0 * e["z"])


@pytest.mark.parametrize("p", [2, 3])
def test_reinit_matches_the_oracle(p):
    gm, om, _, s = _reinit_case(3, p)
    got = sipg.ls_reinit(gm, p, s)
    want = I.ls_reinit(om, p, s)
    assert rel_err(got, want) < 1e-9


def test_reinit_recovers_the_distance_to_a_plane():
    gm, om, e, _ = _reinit_case(4, 3)
    nrm = np.array([0.3, 1.0, -0.2]) / np.linalg.norm([0.3, 1.0, -0.2])
    dist = nrm[0] * (e["x"] - 0.5) + nrm[1] * (e["y"] - 0.45) + nrm[2] * (e["z"] - 0.5)
    got = sipg.ls_reinit(gm, 3, 3.0 * dist)
    assert np.abs(got - dist).max() < 1e-12
