"""Assembled element-row blocks of the low-order levels (sipg_op_element_blocks_host):
the block-sparse product of the blocks equals the matrix-free FP64 apply and the
oracle's apply for every face and boundary type the levels meet (interior faces
with a varying nodal factor, Dirichlet and Neumann walls, a nodal mass term, a
pinned DOF), 2D and 3D, orders 1 and 2."""
import numpy as np
import pytest

import oracle_py as O
import sipg
from helpers import make_op, rel_err

pytestmark = pytest.mark.gpu


def neighbours(e):
    """K x Nf neighbour table (-1 on boundary faces) from the mesh export."""
    nbr = -np.ones((e["K"], e["Nf"]), np.int64)
    for (c0, c1), (f0, f1) in zip(np.asarray(e["face2cells"]).reshape(-1, 2), np.asarray(e["faceNum"]).reshape(-1, 2)):
        nbr[c0, f0] = c1
        nbr[c1, f1] = c0
    return nbr


def block_product(b, nbr, x):
    """y[e, r] = sum_s sum_c b[s, r, c, e] x[k_s(e), c], k_0 = e, k_(1+f) = nbr[e, f]."""
    y = np.einsum("rce,ec->er", b[0], x)
    for f in range(nbr.shape[1]):
        k = nbr[:, f]
        xs = np.where((k >= 0)[:, None], x[np.maximum(k, 0)], 0.0)
        y += np.einsum("rce,ec->er", b[1 + f], xs)
    return y


CASES = [
    # dim, n, order, boundary (0 Dirichlet, 1 Neumann, 2 mixed), factor, nodal mass, pin
    (3, 4, 1, 1, True, False, False),
    (3, 4, 2, 1, True, False, False),
    (3, 4, 2, 0, True, True, False),
    (3, 4, 1, 2, False, False, True),
    (3, 4, 2, 1, True, False, True),
    (2, 8, 1, 2, True, False, False),
    (2, 8, 2, 0, True, True, False),
]


@pytest.mark.parametrize("dim,n,order,bnd,fac,mass,pin", CASES)
def test_element_blocks_reproduce_the_apply(dim, n, order, bnd, fac, mass, pin):
    mesh = sipg.Mesh.box(dim, n, jitter=0.1, seed=5)
    e = mesh.export(order)
    t = sipg.ref_tables(dim, order)
    K, Np = e["K"], t["Np"]
    rng = np.random.default_rng(31 + 7 * order + dim)
    f = rng.uniform(0.001, 1.0, (K, Np)) if fac else None
    mm = rng.uniform(1.0, 50.0, (K, Np)) if mass else None
    if bnd == 2:
        bct = (np.arange(e["Kb"]) % 2).astype(np.int32)[None]
    else:
        bct = np.full((1, e["Kb"]), bnd, np.int32)
    op = make_op(mesh, order, 1, f, mm, bct=bct)
    if pin:
        op.set_pin(3, 1)
    b = op.element_blocks_host()
    assert b.shape == (dim + 2, Np, Np, K)
    x = rng.uniform(-1.0, 1.0, (K, Np))
    y = block_product(b, neighbours(e), x)
    assert rel_err(y[None], op.apply_host(x[None])) < 1e-12
    if not pin:
        om = O.OMesh(t, e)
        want = O.mult(om, x[None], bct, f, mm, 0.0)
        assert rel_err(y[None], want) < 1e-12
