"""Shared helpers for the tests: golden fixtures, seeded cases, tolerances."""
import glob
import os

import numpy as np

import oracle_py as O
import sipg

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))

# Tolerances (relative, max-norm over the output vector)
TOL_FP64 = 1e-13   # FP64 apply / diag / lift vs oracle
TOL_FP32 = 2e-5    # FP32 apply vs FP64 oracle (FP32 arithmetic, FP32 geometry)
TOL_TF32 = 1e-2    # FP32 data on TF32 tensor cores (10-bit operand mantissa) vs FP64 oracle


def rel_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def load_golden(path):
    g = dict(np.load(path))
    for k in ("dim", "n", "order", "ncomp", "seed"):
        g[k] = int(g[k])
    g["jitter"] = float(g["jitter"])
    return g


def golden_setup(g):
    mesh = sipg.Mesh.box(g["dim"], g["n"], jitter=g["jitter"], seed=g["seed"])
    t = sipg.ref_tables(g["dim"], g["order"])
    e = mesh.export(g["order"])
    assert np.array_equal(e["geof"], g["geof"]), "mesh builder drifted from the golden fixture"
    return mesh, t, e, O.OMesh(t, e)


def random_case(dim, n, order, ncomp, seed, jitter=0.1, slip=False, factor=True, mm=False):
    mesh = sipg.Mesh.box(dim, n, jitter=jitter, seed=seed)
    t = sipg.ref_tables(dim, order)
    e = mesh.export(order)
    rng = np.random.default_rng(seed)
    K, Np, Kb = e["K"], t["Np"], e["Kb"]
    x = rng.uniform(-1, 1, (ncomp, K, Np))
    f = rng.uniform(0.2, 3.0, (K, Np)) if factor else None
    m = rng.uniform(0.5, 2.0, (K, Np)) if mm else None
    bct = rng.integers(0, 2, (ncomp, Kb)).astype(np.int32)
    if slip:
        bct[:, ::3] = 2
    return mesh, t, e, O.OMesh(t, e), x, f, m, bct


class DevArray:
    """Device buffer through the library's own allocation helpers."""

    def __init__(self, host):
        import ctypes as C
        self.host = np.ascontiguousarray(host)
        self.nbytes = self.host.nbytes
        self.ptr = C.c_void_p()
        sipg.check(sipg.lib().sipg_dev_alloc(C.c_size_t(self.nbytes), C.byref(self.ptr)))
        sipg.check(sipg.lib().sipg_memcpy_h2d(self.ptr, self.host.ctypes.data_as(C.c_void_p), C.c_size_t(self.nbytes)))

    @property
    def p(self):
        return self.ptr.value

    def get(self):
        import ctypes as C
        out = np.empty_like(self.host)
        sipg.check(sipg.lib().sipg_device_synchronize())
        sipg.check(sipg.lib().sipg_memcpy_d2h(out.ctypes.data_as(C.c_void_p), self.ptr, C.c_size_t(self.nbytes)))
        return out

    def __del__(self):
        if getattr(self, "ptr", None) is not None and self.ptr.value:
            sipg.lib().sipg_dev_free(self.ptr)
            self.ptr = None


def make_op(mesh, order, ncomp, f=None, m=None, mm_scalar=0.0, bct=None):
    op = sipg.Operator(mesh, order, ncomp)
    if bct is not None:
        op.set_bc_types(bct)
    if f is not None:
        op.set_factor(f)
    if m is not None:
        op.set_mm(sipg.MM_NODAL, 0.0, m)
    elif mm_scalar:
        op.set_mm(sipg.MM_SCALAR, mm_scalar)
    return op
