"""Serving loop (sipg_server_*): requests of different meshes, orders and
operators solved concurrently give the same results as alone; queued requests
can be cancelled; the HBM budget rejects what can never fit."""
import ctypes as C
import time

import numpy as np
import pytest

import sipg
import workloads as W
from helpers import make_op


def test_server_without_device_reports_status():
    if sipg.device_count() > 0:
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    o = sipg.ServerOpts(2, 0)
    st = sipg.lib().sipg_server_create(C.byref(o), C.byref(h))
    assert st in (sipg.SIPG_NO_DEVICE, sipg.SIPG_CUDA_ERROR)
    bad = sipg.ServerOpts(0, 0)
    assert sipg.lib().sipg_server_create(C.byref(bad), C.byref(h)) == sipg.SIPG_INVALID_ARG


def _cases():
    out = []
    c = W.poisson3d_two_phase(4, order=3, n_modes=64, pin=False)
    op = make_op(c["mesh"], 3, 1, c["factor"], bct=c["bc_types"])
    o = sipg.default_opts(sipg.SOLVER_PMULTIGRID)
    o.rel_tol, o.abs_tol, o.max_iter, o.precision, o.nullspace = 1e-8, 0.0, 200, sipg.FP32, 1
    out.append((op, sipg.SOLVER_PMULTIGRID, o, c["rhs"].reshape(-1)))
    c2 = W.poisson2d_manufactured(8, order=2)
    op2 = make_op(c2["mesh"], 2, 1, bct=c2["bc_types"])
    o2 = sipg.default_opts(sipg.SOLVER_PMULTIGRID)
    o2.rel_tol, o2.abs_tol, o2.max_iter, o2.n_levels = 1e-10, 0.0, 200, 2
    o2.orders[0], o2.orders[1] = 2, 1
    out.append((op2, sipg.SOLVER_PMULTIGRID, o2, c2["rhs"].reshape(-1)))
    h = W.helmholtz3d(3, order=2)
    op3 = sipg.Operator(h["mesh"], 2, 1)
    op3.set_bc_types(h["bc_types"])
    op3.set_mm(sipg.MM_SCALAR, 1e3)
    o3 = sipg.default_opts(sipg.SOLVER_JACOBI)
    o3.rel_tol, o3.abs_tol, o3.max_iter = 1e-10, 0.0, 2000
    rng = np.random.default_rng(3)
    out.append((op3, sipg.SOLVER_JACOBI, o3, rng.uniform(-1, 1, h["mesh"].K * op3.Np)))
    return out


@pytest.mark.gpu
def test_results_are_the_same_alone_and_in_the_mix():
    cases = _cases()
    alone = []
    for op, kind, o, b in cases:
        x, info = sipg.Solver(op, kind, o).solve_host(b)
        assert info.status == sipg.SIPG_OK
        alone.append(x)
    srv = sipg.Server(slots=3)
    ids = []
    for rep in range(3):
        for i, (op, kind, o, b) in enumerate(cases):
            ids.append((i, srv.submit(op, kind, o, b)))
    for i, rid in ids:
        x, res = srv.wait(rid)
        assert res.status == sipg.SIPG_OK, (res.status, res.error)
        assert res.total_ms >= res.run_ms >= 0.0
        assert np.array_equal(x, alone[i]), (i, np.abs(x - alone[i]).max())
    st = srv.stats()
    assert st["resident"] == len(cases) and st["queued"] == 0 and st["running"] == 0
    srv.close()


@pytest.mark.gpu
def test_cancel_and_budget_rejection():
    cases = _cases()
    op, kind, o, b = cases[2]
    srv = sipg.Server(slots=1)
    long_opts = sipg.default_opts(sipg.SOLVER_CG)
    long_opts.rel_tol, long_opts.abs_tol, long_opts.max_iter = 1e-300, 0.0, 200000
    first = srv.submit(op, sipg.SOLVER_CG, long_opts, b)      # occupies the only slot
    queued = srv.submit(op, kind, o, b)
    srv.cancel(queued)                                       # dropped while queued
    x, res = srv.wait(queued)
    assert res.status == sipg.SIPG_CANCELLED
    time.sleep(0.2)
    srv.cancel(first)                                        # stops after its current iteration
    x, res = srv.wait(first)
    assert res.status == sipg.SIPG_CANCELLED
    assert res.info.iters < 200000
    srv.close()
    tiny = sipg.Server(slots=1, hbm_budget_bytes=1024)
    with pytest.raises(sipg.SipgError) as e:
        tiny.submit(op, kind, o, b)
    assert e.value.status == sipg.SIPG_OUT_OF_MEMORY
    tiny.close()
