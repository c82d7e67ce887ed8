"""sipg_op_apply_static_scratch (the allocation-free apply) against sipg_op_apply.

Both run the same kernels; the static-scratch entry point takes the face-trace
scratch of the two-pass tensor-core apply from a fixed device array instead of
cudaMalloc. Outputs are compared on two calls in a row, device memory is
checked to stay constant across calls on an operator that was never applied,
and an operator whose traces exceed the fixed size is rejected with an error.
"""
import ctypes as C

import numpy as np
import pytest

import sipg
from helpers import TOL_FP32, TOL_FP64, DevArray, make_op, random_case, rel_err

pytestmark = pytest.mark.gpu

SENTINEL = 7.0


def static_apply(op, precision, x, y):
    return sipg.lib().sipg_op_apply_static_scratch(op.h, precision, C.c_void_p(x.p), C.c_void_p(y.p),
                                                   C.c_void_p(0))


def dtype_of(precision):
    return np.float64 if precision == sipg.FP64 else np.float32


def reference_apply(op, precision, x):
    xd = DevArray(x.astype(dtype_of(precision)))
    yd = DevArray(np.zeros_like(x, dtype=dtype_of(precision)))
    op.apply_device(precision, xd.p, yd.p)
    return yd.get().astype(np.float64)


@pytest.mark.parametrize("precision", [sipg.FP64, sipg.FP32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("dim,n,order", [(3, 4, 3), (3, 3, 2), (2, 8, 3), (3, 3, 4)])
def test_static_scratch_apply_matches_apply_twice(dim, n, order, precision):
    mesh, t, e, om, x, f, m, bct = random_case(dim, n, order, 1, seed=101 + 7 * order + dim)
    op = make_op(mesh, order, 1, f, None, bct=bct)
    want = reference_apply(op, precision, x)
    xd = DevArray(x.astype(dtype_of(precision)))
    tol = TOL_FP64 if precision == sipg.FP64 else TOL_FP32
    for _ in range(2):
        yd = DevArray(np.full_like(x, SENTINEL, dtype=dtype_of(precision)))
        st = static_apply(op, precision, xd, yd)
        assert st == sipg.SIPG_OK, sipg.lib().sipg_last_error().decode()
        got = yd.get().astype(np.float64)
        assert rel_err(got, want) < tol


def test_static_scratch_apply_allocates_no_device_memory():
    import torch
    # 10^3 x 6 = 6,000 tets at p = 3: sipg_op_apply would allocate 3.84 MB (FP64) and
    # 1.92 MB (FP32) of traces, above the 2 MiB granularity of device allocations,
    # so a trace allocation shows up in the device's free memory.
    dim, n, order = 3, 10, 3
    trace_bytes = 6000 * 4 * 20 * (8 + 4)
    # warm-up on one operator: the one-time set-up and the first launch of each kernel
    mesh, t, e, om, x, f, m, bct = random_case(dim, n, order, 1, seed=5)
    warm = make_op(mesh, order, 1, f, None, bct=bct)
    for prec in (sipg.FP64, sipg.FP32):
        xd = DevArray(x.astype(dtype_of(prec)))
        yd = DevArray(np.zeros_like(x, dtype=dtype_of(prec)))
        assert static_apply(warm, prec, xd, yd) == sipg.SIPG_OK
    bufs = {p: (DevArray(x.astype(dtype_of(p))), DevArray(np.zeros_like(x, dtype=dtype_of(p))))
            for p in (sipg.FP64, sipg.FP32)}
    # The free-memory figure is device-wide, so an unrelated allocation in between
    # (another process, an allocator growing its cache) can lower it: measure on a
    # fresh, never-applied operator up to three times and accept any attempt in
    # which free memory dropped by less than half the traces sipg_op_apply would take.
    drops = []
    for attempt in range(3):
        fresh = make_op(mesh, order, 1, f, None, bct=bct)
        sipg.check(sipg.lib().sipg_device_synchronize())
        free0 = torch.cuda.mem_get_info()[0]
        outs = {}
        for prec, (xd, yd) in bufs.items():
            for _ in range(2):
                assert static_apply(fresh, prec, xd, yd) == sipg.SIPG_OK
            outs[prec] = yd.get().astype(np.float64)
        sipg.check(sipg.lib().sipg_device_synchronize())
        drops.append(free0 - torch.cuda.mem_get_info()[0])
        for prec, tol in ((sipg.FP64, TOL_FP64), (sipg.FP32, TOL_FP32)):
            assert rel_err(outs[prec], reference_apply(fresh, prec, x)) < tol
        if drops[-1] < trace_bytes // 2:
            break
    assert min(drops) < trace_bytes // 2, f"free device memory dropped by {drops} bytes"


def test_static_scratch_rejects_operators_beyond_its_size():
    # 26^3 x 6 = 105,456 tets at p=3: FP64 traces need 67.5 MB > 64 MiB, FP32 traces 33.7 MB fit
    mesh = sipg.Mesh.box(3, 26, jitter=0.1, seed=3)
    op = sipg.Operator(mesh, 3, 1)
    K, Np = op.K, op.Np
    rng = np.random.default_rng(9)
    x = rng.uniform(-1, 1, (1, K, Np))
    xd = DevArray(x)
    yd = DevArray(np.full_like(x, SENTINEL))
    st = static_apply(op, sipg.FP64, xd, yd)
    assert st == sipg.SIPG_INVALID_ARG
    msg = sipg.lib().sipg_last_error().decode()
    assert "static scratch holds" in msg and str(K) in msg
    assert np.all(yd.get() == SENTINEL)  # nothing was launched
    x32 = DevArray(x.astype(np.float32))
    y32 = DevArray(np.zeros_like(x, dtype=np.float32))
    for _ in range(2):
        assert static_apply(op, sipg.FP32, x32, y32) == sipg.SIPG_OK, sipg.lib().sipg_last_error().decode()
        assert rel_err(y32.get().astype(np.float64), reference_apply(op, sipg.FP32, x)) < TOL_FP32
