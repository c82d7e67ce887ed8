#!/usr/bin/env python3
"""Generate golden vectors from the reference's own kernels.

Runs the reference-kernel build (oracle/_ref/libsipgref.so: src/kernels/*.h of
TobyFlynn/INS-Solver specialised by oracle/gen_ref_kernels.py and driven in the
order of FactorViscousMatrix3D / ViscousSolver3D) on small seeded meshes and
stores inputs and outputs as .npz fixtures next to this script. Build the
libraries first: `make -C oracle && make -C ins-solver_b200`.

usage: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "ins-solver_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle_py as O  # noqa: E402
import sipg  # noqa: E402

# (dim, n, order, ncomp, slip, factor, mm, label)
CASES = [
    (2, 4, 1, 1, False, False, False, "d2p1_poisson"),
    (2, 4, 3, 1, False, True, False, "d2p3_factor"),
    (2, 4, 4, 2, True, True, True, "d2p4_vec_slip_mm"),
    (3, 2, 1, 1, False, True, False, "d3p1_factor"),
    (3, 2, 2, 3, True, True, True, "d3p2_vec_slip_mm"),
    (3, 2, 3, 1, False, True, False, "d3p3_factor"),
    (3, 2, 3, 1, False, False, True, "d3p3_helmholtz_nodal"),
    (3, 2, 4, 1, False, False, False, "d3p4_poisson"),
    (3, 2, 4, 3, True, True, False, "d3p4_vec_slip"),
]


def case_inputs(dim, n, order, ncomp, slip, factor, mm, seed):
    mesh = sipg.Mesh.box(dim, n, jitter=0.1, seed=seed)
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
    bc = rng.uniform(-1, 1, (ncomp, Kb, t["Nfp"]))
    return mesh, t, e, x, f, m, bct, bc


def main():
    for i, (dim, n, order, ncomp, slip, factor, mm, label) in enumerate(CASES):
        seed = 1000 + i
        mesh, t, e, x, f, m, bct, bc = case_inputs(dim, n, order, ncomp, slip, factor, mm, seed)
        om = O.OMesh(t, e)
        y = O.mult(om, x, bct, f, m, 0.0, use_ref=True)
        y_vmf = O.mult(om, x, bct, None, None, 2.5, flags=O.VMF_FLUX_BUG, use_ref=True) if dim == 3 else None
        dg = O.diag(om, ncomp, bct, f, m, use_ref=True)
        blk = O.block_diag(om, ncomp, bct, f, m, 0.0, use_ref=True)
        rhs = O.apply_bc(om, bc, np.zeros_like(x), bct, f, use_ref=True)
        out = dict(dim=dim, n=n, order=order, ncomp=ncomp, seed=seed, jitter=0.1, x=x, bct=bct, bc=bc,
                   geof=e["geof"], y=y, diag=dg, blocks0=blk[0], rhs=rhs)
        if f is not None:
            out["factor"] = f
        if m is not None:
            out["mm"] = m
        if y_vmf is not None:
            out["y_vmf_bug"] = y_vmf
        # solves through the reference's CG / flexible PCG (Dirichlet everywhere, SPD)
        if not slip:
            bd = np.zeros_like(bct)
            b = O.mult(om, x, bd, f, m, 1.0, use_ref=True)
            for pre, name in ((O.PRE_NONE, "cg"), (O.PRE_JACOBI, "jacobi"), (O.PRE_BLOCK_JACOBI, "bjacobi"),
                              (O.PRE_INV_MASS, "invmass")):
                xs, info = O.solve(om, b, bd, pre, f, m, 1.0, abs_tol=1e-10, rel_tol=0.0, max_iter=2000,
                                   use_ref=True)
                out[f"solve_{name}_x"] = xs
                out[f"solve_{name}_iters"] = info.iters
                out[f"solve_{name}_res"] = info.abs_res
            out["solve_b"] = b
        np.savez_compressed(os.path.join(HERE, label + ".npz"), **out)
        print(label, "K", e["K"], "Np", t["Np"])


if __name__ == "__main__":
    main()
