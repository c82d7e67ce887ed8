#!/usr/bin/env python3
"""Generate golden vectors of the element-local velocity projection from the
reference's own kernels.

Runs oracle/_ref/libsipgref.so (ins_proj_setup_0/1, ins_3d_proj_rhs,
ins_3d_proj_pen, ins_3d_proj_cg_precon and their 2D twins from
TobyFlynn/INS-Solver src/kernels, specialised by oracle/gen_ref_kernels.py and
driven in the order of INSSolverBase3D::project_velocity) on small seeded
meshes and stores inputs and outputs as .npz fixtures next to this script.
Build the libraries first: `make -C oracle && make -C ins-solver_b200`.

usage: python tests/golden/projection/make_golden_projection.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.join(ROOT, "ins-solver_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle_py as O  # noqa: E402
import sipg  # noqa: E402

# (dim, n, order, dt, label)
CASES = [
    (3, 2, 1, 1e-2, "proj_d3p1"),
    (3, 2, 3, 1e-2, "proj_d3p3"),
    (3, 2, 4, 1e-1, "proj_d3p4_large_dt"),
    (2, 4, 2, 1e-3, "proj_d2p2"),
    (2, 4, 3, 1e-3, "proj_d2p3"),
]
JITTER = 0.1


def main():
    for k, (dim, n, order, dt, label) in enumerate(CASES):
        seed = 40 + k
        mesh = sipg.Mesh.box(dim, n, jitter=JITTER, seed=seed)
        t, e = sipg.ref_tables(dim, order), mesh.export(order)
        om = O.OMesh(t, e)
        rng = np.random.default_rng(seed)
        velT = rng.uniform(-1, 1, (dim, e["K"], t["Np"]))
        dp = rng.uniform(-1, 1, (dim, e["K"], t["Np"]))
        factor = sipg.projection_factor(dim, dt)
        velTT, stats = O.project_velocity(om, dt, factor, dp, velT, use_ref=True)
        np.savez_compressed(os.path.join(HERE, label + ".npz"), dim=dim, n=n, order=order, seed=seed,
                            jitter=JITTER, dt=dt, factor=factor, geof=e["geof"], velT=velT, dp=dp,
                            velTT=velTT, stats=stats)
        print(label, e["K"], stats)


if __name__ == "__main__":
    main()
