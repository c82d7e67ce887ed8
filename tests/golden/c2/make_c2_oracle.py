"""Writes tests/golden/c2/c2_oracle_solution.npz: the FP64 oracle solution of
the benchmark's two-phase Poisson problem (24^3 x 6 = 82,944 jittered tets,
p = 3, density ratio 1000, Gaussian-random-field right-hand side, Neumann walls
with the constant nullspace projected out), p-multigrid FPCG to a relative
residual of 1e-8 with the library's default V-cycle (element-block Jacobi
Chebyshev(4), continuous-P1 smoothed-aggregation coarse levels).

Everything comes from oracle/ (numpy mesh and reference element, the numpy
coarse hierarchy, the C solver): no CUDA library is loaded. The solution is
stored in FP32 (6.6 MB; the mixed solve's error against it is ~1e-6, far
above FP32's 6e-8), with the oracle's iteration count, final relative residual,
the right-hand side's norm and a float64 checksum of the full solution.

Usage: python tests/golden/c2/make_c2_oracle.py [out.npz]
"""
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402

import dg_oracle as D  # noqa: E402
import pmg_oracle as P  # noqa: E402

N, ORDER = 24, 3


def main():
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "c2_oracle_solution.npz")
    t0 = time.time()
    case = D.poisson3d_two_phase(N, order=ORDER, n_modes=256, pin=False)
    x, info, _ = P.solve_poisson(case, rel_tol=1e-8, max_iter=500)
    assert info.converged
    np.savez_compressed(out, x=x.astype(np.float32), iters=info.iters, rel_res=info.rel_res,
                        rhs_norm=np.linalg.norm(case["rhs"]), x_norm=np.linalg.norm(x),
                        x_sum=x.sum(dtype=np.float64), n=N, order=ORDER)
    print(f"{out}: {info.iters} iterations, relative residual {info.rel_res:.3e}, "
          f"oracle set-up {info.setup_s:.1f} s, iterations {info.solve_s:.1f} s, total {time.time() - t0:.1f} s")


if __name__ == "__main__":
    main()
