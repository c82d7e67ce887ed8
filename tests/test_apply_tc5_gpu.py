"""The tcgen05 FP32 apply (TF32 MMAs with TMEM accumulators, kernel 3 at p = 3
in 3D) against the FP64 oracle and against the mma.sync tensor-core kernels
(kernel 0), on meshes from a partial first tile to several tiles per CTA, with
a nodal factor, nodal and scalar mass terms, mixed Dirichlet / Neumann walls
and a pinned DOF."""
import ctypes as C

import numpy as np
import pytest

import oracle_py as O
import sipg
from helpers import DevArray, make_op, random_case, rel_err

pytestmark = pytest.mark.gpu

# TF32 operands rounded to nearest (2^-11) with FP32 accumulation against the
# FP64 oracle: the relative max-norm error measured on a B200 is about 3e-4.
TOL_TC5 = 1e-3


def fp32_apply(op, x, kernel):
    op.set_kernel(kernel)
    xd = DevArray(x.astype(np.float32))
    yd = DevArray(np.full(x.shape, 7.0, dtype=np.float32))
    op.apply_device(sipg.FP32, xd.p, yd.p)
    out = yd.get().astype(np.float64)
    op.set_kernel(0)
    return out


def timeouts():
    n = C.c_ulonglong()
    sipg.check(sipg.lib().sipg_kernel_wait_timeouts(C.byref(n)))
    return n.value


# 162 tets: two tiles, the second partial; 1,296 and 6,000: ten and 47 tiles;
# 24^3 x 6 = 82,944: 648 tiles, several per CTA
@pytest.mark.parametrize("n", [3, 6, 10, 24])
@pytest.mark.parametrize("variant", ["factor", "helmholtz_nodal", "helmholtz_scalar", "poisson"])
def test_tcgen05_apply_matches_oracle_and_mma_sync(n, variant):
    if n == 24 and variant != "factor":
        pytest.skip("one variant at the largest size")
    mesh, t, e, om, x, f, m, bct = random_case(3, n, 3, 1, seed=17 * n + len(variant),
                                               factor=variant in ("factor", "helmholtz_nodal"),
                                               mm=variant == "helmholtz_nodal")
    scalar = 2.5e3 if variant == "helmholtz_scalar" else 0.0
    op = make_op(mesh, 3, 1, f, m, mm_scalar=scalar, bct=bct)
    want = O.mult(om, x, bct, f, m, scalar)
    got = fp32_apply(op, x, 3)
    prev = fp32_apply(op, x, 0)
    err = rel_err(got, want)
    print(f"{variant} n={n}: tcgen05 {err:.2e}, mma.sync {rel_err(prev, want):.2e}")
    assert err < TOL_TC5
    assert rel_err(got, prev) < 2 * TOL_TC5
    assert timeouts() == 0


def test_tcgen05_apply_pinned_dof():
    mesh, t, e, om, x, f, m, bct = random_case(3, 5, 3, 1, seed=9)
    op = make_op(mesh, 3, 1, f, bct=bct)
    pe, pn = 131, 7
    op.set_pin(pe, pn)
    xs = x.copy()
    xs[0, pe, pn] = 0.0
    want = O.mult(om, xs, bct, f)
    d = O.diag(om, 1, bct, f)
    want[0, pe, pn] = d[0, pe, pn] * x[0, pe, pn]
    assert rel_err(fp32_apply(op, x, 3), want) < TOL_TC5
    assert timeouts() == 0


def test_tcgen05_static_scratch_entry_point_matches_apply():
    mesh, t, e, om, x, f, m, bct = random_case(3, 8, 3, 1, seed=12)
    op = make_op(mesh, 3, 1, f, bct=bct)
    want = fp32_apply(op, x, 3)
    op.set_kernel(3)
    xd = DevArray(x.astype(np.float32))
    yd = DevArray(np.zeros(x.shape, np.float32))
    st = sipg.lib().sipg_op_apply_static_scratch(op.h, sipg.FP32, C.c_void_p(xd.p), C.c_void_p(yd.p), C.c_void_p(0))
    op.set_kernel(0)
    assert st == sipg.SIPG_OK
    assert np.array_equal(yd.get().astype(np.float64), want)
