/* CPU oracle for the SIPG pressure/viscous solve path (FP64, plain C).
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker for the CUDA path: only the
 * tests, the smoke check and the CPU-baseline leg of the benchmark may load
 * it. The product library never links or calls it.
 *
 * It restates, step by step, the reference's algorithm:
 *   - FactorViscousMatrix3D::mult (src/solvers/3d/slip_matrix/factor_viscous_matrix.cpp:96-310)
 *     and its 2D twin (src/solvers/2d/slip_matrix/factor_viscous_matrix.cpp:87-200),
 *     with the scalar Poisson / Helmholtz operators as the one-component case;
 *   - the penalty (src/kernels/fvmf_3d_calc_tau_faces.h, fvmf_3d_calc_tau_bfaces.h);
 *   - boundary lifting apply_bc (src/kernels/fvmf_3d_apply_bc.h);
 *   - diagonal and block diagonal (factor_viscous_matrix.cpp:312-451);
 *   - CG / flexible PCG (src/solvers/3d/slip_matrix/viscous_solver.cpp:89-453);
 *   - the p-multigrid preconditioned CG (restated from the configuration keys
 *     of the unvendored PETScPMultigrid, see pmg section below).
 *
 * Data conventions (shared with the CUDA path): constant matrices are
 * row-major A[i*ncols+j]; per-element vectors are [K][Np]; per-element-face
 * data is [K][Nf]; geof is [K][10] (rx ry rz sx sy sz tx ty tz J) in 3D and
 * [K][5] (rx ry sx sy J) in 2D.
 */
#ifndef SIPG_ORACLE_H
#define SIPG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int dim, order, Np, Nfp, Nf, K, F, Kb;
  const double *Dr, *Ds, *Dt; /* Np x Np */
  const double *M;            /* Np x Np */
  const double *MMF;          /* Nf x Np x Np face mass embedded in the volume */
  const double *EMAT;         /* Np x (Nf*Nfp) */
  const int *fmask;           /* Nf x Nfp */
  const double *geof;         /* K x ngeof */
  const double *nx, *ny, *nz, *sJ, *fscale; /* K x Nf */
  const int *face2cells, *faceNum;          /* F x 2 */
  const int *fmaskL, *fmaskR;               /* F x Nfp */
  const int *bface2cell, *bfaceNum;         /* Kb */
} oracle_mesh;

/* flags */
#define ORACLE_VMF_FLUX_BUG 1   /* drop n_z*avg_z as src/kernels/vmf_3d_mult_flux.h:9-11 does */
#define ORACLE_REF_BLOCK_DIAG 2 /* volume block as the reference computes it (fvmf_3d_op1.h:17-18, fvmf_2d_op1.h:20-37) */

/* Penalty per element face (K x Nf). factor may be NULL (constant 1). */
void oracle_tau(const oracle_mesh *m, const double *factor, double *tau);

/* y_c = A x_c for ncomp components (1, or dim for the vector slip operator).
 * bc_types: ncomp x Kb (0 Dirichlet, 1 Neumann, 2 slip). factor: K x Np or NULL.
 * mm_factor: K x Np or NULL; mm_scalar used when mm_factor is NULL (0 = none). */
void oracle_mult(const oracle_mesh *m, int ncomp, const int *bc_types, const double *factor,
                 const double *mm_factor, double mm_scalar, int flags, const double *const *x,
                 double *const *y);

/* rhs_c += boundary lifting of bc data (ncomp x Kb x Nfp). */
void oracle_apply_bc(const oracle_mesh *m, int ncomp, const int *bc_types, const double *factor,
                     const double *const *bc, double *const *rhs);

/* Diagonal of A per component (ncomp x K x Np). */
void oracle_diag(const oracle_mesh *m, int ncomp, const int *bc_types, const double *factor,
                 const double *mm_factor, double mm_scalar, double *diag);

/* Diagonal blocks (ncomp x K x Np x Np, row-major) and, if inv != 0, their inverses. */
void oracle_block_diag(const oracle_mesh *m, int ncomp, const int *bc_types,
                       const double *factor, const double *mm_factor, double mm_scalar,
                       int flags, int inv, double *blocks);

/* CSR matrix (algebraic levels of the coarse solve). */
typedef struct {
  int rows, cols;
  const int *ptr, *idx;
  const double *val;
} oracle_csr;

/* Solvers. Preconditioner kinds follow ViscousSolver3D::Preconditioners. */
enum {
  ORACLE_PRE_NONE = 0,
  ORACLE_PRE_INV_MASS = 1,
  ORACLE_PRE_FACTOR_INV_MASS = 2,
  ORACLE_PRE_JACOBI = 3,
  ORACLE_PRE_BLOCK_JACOBI = 4,
  ORACLE_PRE_PMG = 5
};

typedef struct {
  int iters;
  double abs_res;      /* final ||r||_2 */
  double rel_res;      /* final ||r||_2 / ||b||_2 */
  int converged;
  double setup_s;      /* wall seconds of the preconditioner set-up */
  double solve_s;      /* wall seconds of the iterations (initial residual included) */
  double iter_s;       /* wall seconds per iteration after the first preconditioner application */
} oracle_solve_info;

/* Operator apply with oracle_mult's arguments; returns 0 on success. Lets a
 * solve run on another implementation of the same apply (the reference's own
 * kernels in oracle/_ref, ref_mult). */
typedef int (*oracle_mult_fn)(const oracle_mesh *m, int ncomp, const int *bc_types, const double *factor,
                              const double *mm_factor, double mm_scalar, int flags, const double *const *x,
                              double *const *y);

typedef struct {
  int ncomp;
  const int *bc_types;
  const double *factor;
  const double *mm_factor;
  double mm_scalar;
  int flags;
  int precond;
  double inv_mass_factor;    /* FACTOR_INV_MASS */
  double abs_tol, rel_tol;   /* stop when ||r|| < max(abs_tol, rel_tol*||b||) */
  int max_iter;
  int pin_dof;               /* >= 0: pinned DOF (row and column replaced by the diagonal) */
  int nullspace;             /* project out constants (pure Neumann) */
  /* p-multigrid settings (PRE_PMG) */
  int pmg_nlevels;
  const int *pmg_orders;     /* e.g. {3,2,1} */
  const oracle_mesh *pmg_meshes; /* one mesh view per level (same elements, that order) */
  const double *const *pmg_factors;   /* factor per level (NULL for constant) */
  const double *const *pmg_prolong;   /* level l+1 -> l prolongation (Np_l x Np_{l+1}) */
  int cheb_order;
  double eig_safety;         /* eigenvalue safety factor (eigen_val_saftey_factor) */
  double eig_ratio;          /* lambda_min = lambda_max / eig_ratio */
  int eig_iters;             /* power iterations for lambda_max */
  int coarse_iters;          /* Jacobi-PCG iterations on the coarsest level (coarse_kind 0) */
  /* coarse_kind 1: below the last order, restrict to element-wise constants and
   * run a V-cycle over an algebraic hierarchy of CSR operators */
  int coarse_kind;
  int amg_nlevels;
  const oracle_csr *amg_A, *amg_P, *amg_R; /* per level (P, R: level l <-> l+1) */
  const oracle_csr *amg_Pdg, *amg_Rdg;     /* last-order DG unknowns <-> algebraic level 0 */
  const double *amg_coarse_inv;            /* dense inverse of the coarsest operator */
  int amg_coarse_n;
  /* smoother of the order levels: 0 Jacobi (inverse diagonal), 1 element-block
   * Jacobi (inverse diagonal blocks of the operator, pinned DOF included) */
  int smoother;
  int amg_cheb_order;        /* Chebyshev degree on the algebraic levels (0: cheb_order) */
  oracle_mult_fn mult;       /* every operator apply of the solve (NULL: oracle_mult) */
  oracle_mult_fn outer_mult; /* the outer Krylov operator only, when it differs from the
                                preconditioner's (the over-integrated operator); NULL: mult */
} oracle_solver_opts;

/* Solve A x = b (x holds the initial guess on entry). ncomp components are
 * stored one after the other (ncomp x K x Np). */
void oracle_solve(const oracle_mesh *m, const oracle_solver_opts *o, const double *b, double *x,
                  oracle_solve_info *info);

/* Estimate of lambda_max of D^-1 A on one level (power iteration from a
 * seeded start vector), exposed for tests. */
double oracle_pmg_lambda_max(const oracle_mesh *m, const int *bc_types, const double *factor,
                             int pin_dof, int iters);

/* Velocity projection (pr_projection_method == 1): per-element penalty length
 * h (K values) and the element-local projection solve; see sipg_oracle.c. */
void oracle_proj_h(const oracle_mesh *m, double *h);
void oracle_project_velocity(const oracle_mesh *m, double dt, double factor, const double *dp,
                             const double *velT, double *velTT, double *stats);
/* Central-flux DG gradient of p (K x Np) into grad (dim x K x Np). */
void oracle_grad_central(const oracle_mesh *m, const double *p, double *grad);
/* Pressure right-hand side J M (-div_c(velT)/dt + LIFT (b0 dPdN + b1 dPdN_old)). */
void oracle_pressure_rhs(const oracle_mesh *m, double dt, double b0, double b1, const double *velT,
                         const double *dPdN, double *dPdN_old, double *rhs);

#ifdef __cplusplus
}
#endif
#endif
