/* sipg_b200.h -- C ABI of the B200-native SIPG pressure/viscous solve path.
 *
 * Drop-in boundary for INS-Solver's pressure/viscous linear-solve hot path.
 * Plain pointers and sizes only; every entry point returns an int status
 * (SIPG_OK = 0) and never aborts the process; sipg_last_error() describes the
 * last failure on the calling thread. The reference reports solver failure as
 * `bool solve(...)` and aborts on setup errors (dg_abort); the C++ shim classes
 * in include/ins_solver_b200/ map these statuses back to the reference's forms.
 *
 * Each declaration names the reference interface it replaces (paths inside
 * the TobyFlynn/INS-Solver tree). Vectors are FP64, element-major [K][Np]
 * (the layout of an op_dat with dim Np), components stacked one after another.
 */
#ifndef SIPG_B200_H
#define SIPG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference: bool converged + dg_abort) */
#define SIPG_OK 0
#define SIPG_NOT_CONVERGED 1  /* solve(): residual above tolerance after max_iter */
#define SIPG_BREAKDOWN 2      /* solve(): NaN/Inf or p.Ap <= 0 */
#define SIPG_INVALID_ARG 3
#define SIPG_OUT_OF_MEMORY 4  /* also: request rejected by the HBM admission budget */
#define SIPG_CANCELLED 5      /* served request cancelled or timed out */
#define SIPG_CUDA_ERROR 6
#define SIPG_NO_DEVICE 7

typedef struct sipg_mesh sipg_mesh;
typedef struct sipg_op sipg_op;
typedef struct sipg_solver sipg_solver;
typedef struct sipg_server sipg_server;
typedef struct sipg_amg sipg_amg;

const char *sipg_last_error(void);
int sipg_version(void);

/* ---- device memory helpers (plain CUDA runtime calls, for callers without a
 * CUDA toolkit of their own; the reference owns data through OP2 op_dats) */
int sipg_device_count(int *n);
int sipg_dev_alloc(size_t bytes, void **ptr);
int sipg_dev_free(void *ptr);
int sipg_memcpy_h2d(void *dst, const void *src, size_t bytes);
int sipg_memcpy_d2h(void *dst, const void *src, size_t bytes);
int sipg_device_synchronize(void);

/* ---- reference element tables (replace DGConstants / dg_*_kernel / FMASK of
 * the unvendored OP2-DG-Toolkit, used e.g. at src/kernels/fvmf_3d_op1_diag.h:2-5).
 * Matrices are row-major. Any output pointer may be NULL. */
int sipg_ref_sizes(int dim, int order, int *Np, int *Nfp, int *Nfaces, int *Nperm);
int sipg_ref_tables(int dim, int order, double *r, double *s, double *t, double *Dr, double *Ds,
                    double *Dt, double *M, double *MMF, double *EMAT, int *fmask, int *perm_pos);
/* Prolongation from order q to order p (Np(p) x Np(q)), the p-multigrid transfer. */
int sipg_interp_matrix(int dim, int q, int p, double *P);

/* ---- synthetic meshes: unit square n x n x 2 triangles, unit cube n^3 x 6
 * tetrahedra (Kuhn split); interior vertices jittered by +-jitter*h from seed. */
int sipg_box_mesh_sizes(int dim, int n, int *Nv, int *K);
int sipg_box_mesh(int dim, int n, double jitter, uint64_t seed, double *vx, int *e2v);

/* ---- mesh: replaces DGMesh3D/DGMesh2D construction and init
 * (src/ins3d.cpp:154, :203; geof/face data consumed by
 * src/solvers/3d/slip_matrix/factor_viscous_matrix.cpp:47-92). Builds the
 * connectivity and geometry on the host and keeps it resident on the GPU. */
int sipg_mesh_create(int dim, int Nv, const double *vx, int K, const int *e2v, sipg_mesh **out);
int sipg_mesh_sizes(const sipg_mesh *m, int *K, int *F, int *Kb);
/* Host copies of the per-order mesh data in the reference's form (any NULL
 * pointer is skipped): geof K x (10|5); nx, ny, nz, sJ, fscale K x Nf;
 * face2cells, faceNum F x 2; fmaskL, fmaskR F x Nfp; bface2cell, bfaceNum Kb;
 * bface_centroid Kb x dim; x, y, z K x Np node coordinates. */
int sipg_mesh_export(const sipg_mesh *m, int order, double *geof, double *nx, double *ny,
                     double *nz, double *sJ, double *fscale, int *face2cells, int *faceNum,
                     int *fmaskL, int *fmaskR, int *bface2cell, int *bfaceNum,
                     double *bface_centroid, double *x, double *y, double *z);
int sipg_mesh_device_bytes(const sipg_mesh *m, size_t *bytes);
/* Precision of the geometric factors the FP32 kernels read (no reference counterpart:
 * the reference's geometric factors are DG_FP): 32 (default) or 16, the FP32 factors and
 * the tensor-core geometry blocks derived from them rounded to BF16 (ties to even,
 * stored in FP32 words); the FP64 kernels keep FP64 factors. Call before the mesh's
 * first device use (SIPG_INVALID_ARG after). */
int sipg_mesh_set_geometry_precision(sipg_mesh *m, int bits);
void sipg_mesh_destroy(sipg_mesh *m);

/* ---- operator: replaces PoissonMatrixFreeDiag3D / FactorPoissonMatrixFreeDiag3D /
 * MMPoissonMatrixFree3D / FactorMMPoissonMatrixFreeDiag3D (unvendored; created at
 * src/solvers/3d/mp_ins_solver.cpp:87, src/solvers/3d/ins_solver.cpp:91,139) and the
 * vendored FactorViscousMatrix3D / ViscousMatrix3D (ncomp = dim, slip coupling). */
#define SIPG_MM_NONE 0
#define SIPG_MM_SCALAR 1
#define SIPG_MM_NODAL 2
#define SIPG_BC_DIRICHLET 0
#define SIPG_BC_NEUMANN 1
#define SIPG_BC_SLIP 2
#define SIPG_FP64 64
#define SIPG_FP32 32

int sipg_op_create(sipg_mesh *m, int order, int ncomp, sipg_op **out);
/* set_factor(op_dat) (factor_viscous_matrix.cpp:70-72); NULL = constant 1. Host FP64 K x Np. */
int sipg_op_set_factor(sipg_op *op, const double *factor);
/* set_mm_factor(op_dat) (:74-76) or MMPoissonMatrixFree3D::set_factor(DG_FP). */
int sipg_op_set_mm(sipg_op *op, int mode, double scalar, const double *mm);
/* set_bc_types (:41-45): ncomp x Kb ints, 0 Dirichlet, 1 Neumann, 2 slip. */
int sipg_op_set_bc_types(sipg_op *op, const int *types);
/* Pin one DOF (element, node): its row and column become diag * identity. -1 clears. */
int sipg_op_set_pin(sipg_op *op, int elem, int node);
/* mult(in, out) (factor_viscous_matrix.cpp:96-310). x, y: device pointers,
 * ncomp x K x Np of double (SIPG_FP64) or float (SIPG_FP32). stream: cudaStream_t or NULL. */
int sipg_op_apply(sipg_op *op, int precision, const void *x, void *y, void *stream);
/* Same with host FP64 buffers (copies in and out inside the call). */
int sipg_op_apply_host(sipg_op *op, const double *x, double *y);
/* Allocation-free apply. No counterpart in the reference (its mult has no
 * scratch of its own; OP2 leases temporaries from a dat pool). Same arguments,
 * kernels and results as sipg_op_apply, but the face-trace scratch of the
 * two-pass tensor-core apply comes from a fixed array of
 * SIPG_STATIC_SCRATCH_BYTES compiled into the library, not from cudaMalloc,
 * for callers that cannot allocate device memory at apply time. The first call
 * on each device (current device) does a one-time set-up, a symbol-address
 * lookup; make it before any stream capture. Operators whose scratch would
 * exceed the limit get SIPG_INVALID_ARG; the scratch holds
 * K * (dim+1) * roundup(2 * roundup(Nfp, 2), 4) values of the precision's size
 * (at p = 3 in 3D: 209,715 elements FP32, 104,857 FP64). With lazy module
 * loading (the CUDA default) the array takes device memory from the first use
 * of the library's kernels in a context; with CUDA_MODULE_LOADING=EAGER every
 * context that loads the library reserves it at start-up. There is one scratch per
 * device: calls that overlap in time on one device race on it, so order them
 * on one stream or synchronise between them. Nothing in it needs to start at
 * zero. */
#define SIPG_STATIC_SCRATCH_BYTES (64u << 20)
int sipg_op_apply_static_scratch(sipg_op *op, int precision, const void *x, void *y, void *stream);
/* Kernel selection of apply(): 0 tensor cores where the operator allows it
 * (scalar operators: mma.sync TF32 MMAs for SIPG_FP32, FP64 MMAs for SIPG_FP64),
 * 1 the CUDA-core kernel, 2 the same tensor-core kernels as 0, 3 SIPG_FP32 on
 * tcgen05 TF32 MMAs with TMEM accumulators where the order has those kernels
 * (3D p = 3; otherwise as 0). No reference counterpart (the reference has one
 * OP2 path). */
int sipg_op_set_kernel(sipg_op *op, int kind);
/* apply_bc (factor_viscous_matrix.cpp:47-68): rhs += lifted bc data; host buffers,
 * bc: ncomp x Kb x Nfp, rhs: ncomp x K x Np (updated in place). */
int sipg_op_apply_bc_host(sipg_op *op, const double *bc, double *rhs);
/* calc_diag (:312-366) -> host diag ncomp x K x Np. */
int sipg_op_diag_host(sipg_op *op, double *diag);
/* calc_inv_block_diag (:368-451) -> host blocks ncomp x K x Np x Np (row-major);
 * invert != 0 returns the inverses. ref_volume_block != 0 reproduces the
 * reference's volume block formula (fvmf_3d_op1.h:17-18). */
int sipg_op_block_diag_host(sipg_op *op, int invert, int ref_volume_block, double *blocks);
/* ---- over-integrated factor: FactorPoissonMatrixFreeDiagOI3D (OP2-DG-Toolkit,
 * unvendored), selected by [pressure-solve] over_int (src/solvers/3d/
 * mp_ins_solver.cpp:81-88) and set in update_pressure_matrices_oi (:524-544).
 * The factor (1/rho) is given at nq volume cubature points per element
 * (mat_free_set_factor_oi) and at nqs surface cubature points per element face
 * (mat_free_set_factor_surf_oi); the operator integrates every SIPG term with
 * these points (the symmetric form: each face term that carries one side's
 * factor uses that side's points) and uses the L2 projection of the volume
 * values as its nodal factor (set_factor(CUB3D_PROJ f), the coarse levels'
 * factor). The rules are the library's own (collapsed Gauss-Legendre, exact to
 * degree 2p + 1 in the volume and 2p on the faces; the toolkit's are not in the
 * reference tree): sipg_op_oi_points_host gives their physical coordinates,
 * where the caller evaluates rho (getRhoVolOI / getRhoSurfOI). Scalar operators;
 * sipg_op_set_factor returns to the nodal factor. */
int sipg_op_oi_sizes(const sipg_op *op, int *nq, int *nqs);
/* xyz_vol: dim x K x nq, xyz_surf: dim x K x (dim + 1) x nqs (either may be NULL). */
int sipg_op_oi_points_host(sipg_op *op, double *xyz_vol, double *xyz_surf);
/* fvol: K x nq, fsurf: K x (dim + 1) x nqs, host pointers (synchronous) ... */
int sipg_op_set_factor_oi(sipg_op *op, const double *fvol, const double *fsurf);
/* ... or device pointers, ordered on `stream`. */
int sipg_op_set_factor_oi_device(sipg_op *op, const double *fvol, const double *fsurf, void *stream);

/* The assembled form of a scalar operator of order 1 or 2: per element row e its
 * Np x Np blocks against itself (s = 0) and against the neighbour across each
 * face f (s = 1 + f; zero on boundary faces), columns in the neighbour's node
 * order, layout blocks[((s * Np + r) * Np + c) * K + e], (dim + 2) Np^2 K values.
 * These are the element-block matrices the p-multigrid applies on its low-order
 * levels; they stand in for the assembled coarse matrices of OP2-DG-Toolkit
 * (PoissonCoarseMatrix, unvendored) behind the reference's PETSc coarse solve. */
int sipg_op_element_blocks_host(sipg_op *op, double *blocks);
int sipg_op_sizes(const sipg_op *op, int *K, int *Np, int *Nfp, int *ncomp);
void sipg_op_destroy(sipg_op *op);

/* ---- solver: replaces LinearSolver and its subclasses (src/solvers/3d/
 * ins_solver_base.cpp:149-184, :1522-1536; solve at mp_ins_solver.cpp:632) and
 * ViscousSolver3D (src/solvers/3d/slip_matrix/viscous_solver.cpp:63-453). */
#define SIPG_SOLVER_CG 0             /* ViscousSolver3D, Preconditioners::NONE */
#define SIPG_SOLVER_INV_MASS 1       /* PETScInvMassSolver / INV_MASS, FACTOR_INV_MASS */
#define SIPG_SOLVER_JACOBI 2         /* PETScJacobiSolver / JACOBI */
#define SIPG_SOLVER_BLOCK_JACOBI 3   /* PETScBlockJacobiSolver / BLOCK_JACOBI */
#define SIPG_SOLVER_PMULTIGRID 4     /* PETScPMultigrid */

typedef struct {
  int iters;
  double rel_res;     /* ||b - A x|| / ||b|| (recursive residual) */
  double abs_res;
  double true_rel_res;/* recomputed with an explicit FP64 apply at the end */
  double setup_ms;
  double solve_ms;
  int status;
} sipg_solve_info;

typedef struct {
  double rel_tol, abs_tol;   /* set_tol_and_iter (ins_solver_base.cpp:153-183) */
  int max_iter;
  int nullspace;             /* set_nullspace: project out constants */
  int precision;             /* preconditioner precision: SIPG_FP64 or SIPG_FP32 (mixed) */
  double inv_mass_factor;    /* PETScInvMassSolver::setFactor */
  int ref_volume_block;      /* block Jacobi: reference's volume block formula */
  /* [p-multigrid] keys (examples/3d/oscillating_droplet/config.ini:24-31) */
  int n_levels;
  int orders[4];             /* e.g. 3,2,1 */
  int cheb_order;            /* Chebyshev degree per smoothing sweep */
  double eig_safety;         /* eigen_val_saftey_factor */
  double eig_ratio;          /* lambda_min = lambda_max * safety / eig_ratio */
  int eig_iters;
  int coarse_iters;          /* Jacobi-PCG iterations on the coarsest order (coarse_kind 0) */
  int check_every;           /* host convergence check period (iterations) */
  int coarse_kind;           /* 0: Jacobi-PCG on the lowest order; 1: algebraic multigrid on the
                                continuous piecewise-linear space (coarse_solver = petsc/amg) */
  int amg_coarse_max;        /* unknowns of the densely inverted coarsest level (default 2048; inverted on the device) */
  double amg_strength;       /* aggregation strength threshold */
  int graphs;                /* 2: the outer iterations after the first run inside one CUDA graph
                                whose conditional while-node repeats an iteration until the
                                stopping test on the device ends it (host reads once per 64
                                iterations; falls back to 1 where unsupported); 1: each outer
                                iteration after the first is replayed from a captured CUDA graph;
                                0: kernels are launched one by one. The three run the same
                                kernels: identical iterates. */
  int assembled_max_order;   /* p-multigrid levels below the finest with this order or lower apply
                                their operator as stored element blocks (assembled once from the
                                matrix-free apply, scalar operators, orders <= 2; in the FP32
                                V-cycle p = 1 blocks are FP32 and p = 2 blocks FP16 scaled per
                                element); 0: all matrix-free; -1 (default): 2 in the FP32 V-cycle,
                                1 in the FP64 V-cycle */
  int smoother;              /* p-multigrid smoothing: 0 Chebyshev on the point-Jacobi (diagonal)
                                preconditioned operator, 1 on the element-block-Jacobi one */
  /* per p-multigrid level (the [p-multigrid] keys cheb_orders, pre_it, post_it of
   * examples/3d/oscillating_droplet/config.ini:24-31): Chebyshev degree (0: cheb_order)
   * and Chebyshev sweeps before and after the coarse-level correction */
  int cheb_orders[4];
  int pre_it[4];
  int post_it[4];
  int amg_cheb_order;        /* Chebyshev degree on the algebraic coarse levels (0: cheb_order);
                                default 2 (the coarse correction needs no more at C2: same
                                iteration count as degree 4) */
  int amg_reuse_interpolation; /* [petsc-amg] reuse-interpolation (examples/3d/oscillating_droplet/
                                config.ini:59, default 1): later set-ups keep the aggregates and
                                prolongators of the first and recompute only the level operators
                                (Galerkin products), their smoother data and the coarsest inverse,
                                all on the device; 0: aggregate again at every set-up. A change of
                                the boundary types or of the problem's singularity aggregates again. */
} sipg_solver_opts;

int sipg_solver_default_opts(int kind, sipg_solver_opts *o);
int sipg_solver_create(sipg_op *op, int kind, const sipg_solver_opts *o, sipg_solver **out);
/* Re-run the setup that depends on the operator's coefficients (diagonals,
 * blocks, eigenvalue bounds, coarse operators); call after set_factor. */
int sipg_solver_setup(sipg_solver *s);
/* solve(rhs, ans): device FP64 pointers (ncomp x K x Np); x holds the initial guess. */
int sipg_solver_solve(sipg_solver *s, const double *b, double *x, sipg_solve_info *info);
/* Same with host buffers, copies inside the call (end-to-end path). */
int sipg_solver_solve_host(sipg_solver *s, const double *b, double *x, sipg_solve_info *info);
void sipg_solver_destroy(sipg_solver *s);

/* ---- algebraic coarse hierarchy below p=0: the B200 stand-in for the PETSc
 * algebraic multigrid the reference uses as its p-multigrid coarse solver
 * (coarse_solver = petsc, [petsc-amg], examples/3d/oscillating_droplet/config.ini:24-31,52-64).
 * Host-side build from the p=0 Galerkin operator (graph Laplacian with face
 * weights sJ*tau); the solver builds and uploads it itself, these entry points
 * expose it for inspection. sJ, tau, nbr: K x Nf; bc_dirichlet: Kb flags. */
int sipg_amg_build(int K, int Nf, const double *sJ, const double *tau, const int *nbr, int Kb,
                   const int *bc_dirichlet, int coarse_max, double strength, int singular,
                   sipg_amg **out);
/* Continuous piecewise-linear coarse space (the default of the p-multigrid):
 * Galerkin operator of the p=1 SIPG operator restricted to continuous functions
 * (volume and Dirichlet-boundary terms), host-side from the mesh; factor1 and
 * tau1 are the p=1 level's nodal factor (K x (dim+1), NULL = 1) and penalty
 * (K x (dim+1)); mm1: nodal mass factor or NULL. */
int sipg_amg_build_p1(sipg_mesh *m, const double *factor1, const double *tau1, const int *bc_dirichlet,
                      int mm_mode, double mm_scalar, const double *mm1, int coarse_max, double strength,
                      int singular, sipg_amg **out);
int sipg_amg_sizes(const sipg_amg *a, int *nlevels, int *coarse_n);
/* which: 0 operator A, 1 prolongation P (to level+1's unknowns), 2 restriction R = P^T;
 * level -1 is the transfer between the p=1 DG unknowns and level 0 (P, R only).
 * Call with NULL arrays to get rows/cols/nnz, then with arrays of those sizes. */
int sipg_amg_level(const sipg_amg *a, int level, int which, int *rows, int *cols, int *nnz, int *ptr,
                   int *idx, double *val);
int sipg_amg_coarse_inverse(const sipg_amg *a, double *inv);
void sipg_amg_destroy(sipg_amg *a);

/* ---- serving loop: no reference counterpart (the reference solves one system at
 * a time inside its time step). Requests (an operator on a resident mesh, solver
 * kind and options, a right-hand side) arrive at any time; up to `slots` solves
 * run concurrently, each on its own CUDA stream, so their kernels overlap on the
 * device. A queued request is admitted as soon as a slot is free, its operator is
 * not busy with another request, and its solver state fits the HBM budget
 * (solver states stay resident between requests for the same operator and
 * options, least recently used first out when the budget needs room). */
typedef struct {
  int slots;                  /* concurrent solves (worker threads), >= 1 */
  size_t hbm_budget_bytes;    /* device bytes for resident solver state; 0: 90% of the free memory */
} sipg_server_opts;

typedef struct {
  int status;                 /* SIPG_OK, SIPG_NOT_CONVERGED, SIPG_BREAKDOWN, SIPG_CANCELLED, ... */
  sipg_solve_info info;
  double queue_ms;            /* submit -> start */
  double run_ms;              /* start -> done (includes a solver set-up on first use) */
  double total_ms;            /* submit -> done */
  char error[160];            /* why the request failed (status other than OK, NOT_CONVERGED,
                                 BREAKDOWN, CANCELLED); empty otherwise */
} sipg_request_result;

int sipg_server_create(const sipg_server_opts *o, sipg_server **out);
/* b: host right-hand side, copied at submit; x: host initial guess, read at start,
 * overwritten with the solution; it must stay valid until the request is done. */
int sipg_server_submit(sipg_server *s, sipg_op *op, int kind, const sipg_solver_opts *o, const double *b,
                       double *x, long long *id);
/* done = 1 and res filled once the request has finished. */
int sipg_server_poll(sipg_server *s, long long id, int *done, sipg_request_result *res);
int sipg_server_wait(sipg_server *s, long long id, sipg_request_result *res);
/* A queued request is dropped; a running one stops after its current iteration. */
int sipg_server_cancel(sipg_server *s, long long id);
/* Resident solver states and bytes accounted against the budget. */
int sipg_server_stats(sipg_server *s, int *resident_solvers, size_t *resident_bytes, int *queued, int *running);
void sipg_server_destroy(sipg_server *s);

/* ---- initial guess: replaces initial_guess_extrapolation(mesh, pr_history, pr,
 * time + dt) (src/solvers/3d/ins_solver.cpp:342-343, mp_ins_solver.cpp:629-630;
 * history kept by add_to_pr_history, ins_solver_base.cpp:1374-1388). out = the
 * polynomial through the n_hist (1..8) points (times[i], hist[i]) evaluated at
 * t_new (Lagrange form; one point copies it). n values per vector; device
 * pointers (stream: cudaStream_t or NULL) or, in the _host variant, host pointers. */
int sipg_extrapolate_initial_guess(int n_hist, const double *times, const double *const *hist, double t_new,
                                   size_t n, double *out, void *stream);
int sipg_extrapolate_initial_guess_host(int n_hist, const double *times, const double *const *hist,
                                        double t_new, size_t n, double *out);

/* ---- velocity projection: replaces INSSolverBase3D::project_velocity with
 * div_div = 1 (pr_projection_method 1, src/solvers/3d/ins_solver_base.cpp:1052-1124;
 * 2D src/solvers/2d/ins_solver_base.cpp:894-955): the OP2 loops
 * ins_3d_proj_rhs, mesh->mass, ins_3d_proj_pen and ins_3d_proj_cg_precon
 * (2D: ins_2d_proj_rhs, ins_2d_proj_pen, ins_proj_cg_2d) as one kernel, with the
 * penalty length h of ins_proj_setup_0/1 (ins_solver_base.cpp:201-214) cached
 * on the mesh. Per element: velTT = velT - dt * dp, then the element-local CG
 * solve of (J M + pen G^T D^T J M D G) velTT = J M velTT_0 from velTT_0,
 * pen = factor * h / (order + 1); 3D preconditioned by (1/J) M^-1 and stopped
 * at |r|_2 < 1e-8, 2D unpreconditioned and stopped at |r|_2^2 < 1e-16, both
 * after at most 100 iterations. The reference passes factor = dt in 3D and
 * dt * 1e3 in 2D. dp (grad p), velT and velTT hold dim components one after the
 * other (dim x K x Np); velTT must not alias dp or velT. Device pointers; stats,
 * if not NULL, is a device array of 2 counters (converged elements, iterations
 * summed over elements) that the call zeroes and the kernel fills, the
 * reference's num_converge / num_iter (num_cells is K). The _host variant takes
 * host arrays, is synchronous, and returns stats = {cells, converged,
 * iterations} as doubles. */
int sipg_project_velocity(sipg_mesh *m, int order, double dt, double factor, const double *dp,
                          const double *velT, double *velTT, unsigned long long *stats, void *stream);
int sipg_project_velocity_host(sipg_mesh *m, int order, double dt, double factor, const double *dp,
                               const double *velT, double *velTT, double *stats);

/* ---- pressure projection step: replaces, in MPINSSolver3D::pressure
 * (src/solvers/3d/mp_ins_solver.cpp:650-661; INSSolver3D::pressure
 * ins_solver.cpp:358-363), the sequence mesh->grad_with_central_flux(pr, dpdx,
 * dpdy, dpdz) (OP2-DG-Toolkit, unvendored), update_pressure_gradient (grad p /
 * rho, mp_ins_3d_pr_2.h, mp_ins_solver.cpp:546-552) and project_velocity, as
 * one kernel: grad p = G^T (Dr, Ds, Dt) pr + LIFT (fscale n (pr+ - pr-) / 2) over
 * interior faces (central flux; boundary faces add nothing), divided by rho
 * when rho is not NULL (the two-phase solver; NULL for INSSolver3D), then the
 * element-local projection of sipg_project_velocity. pr and rho: K x Np; velT,
 * velTT: dim x K x Np; stats as there. Device pointers, or host pointers in the
 * synchronous _host variant. */
int sipg_pressure_projection(sipg_mesh *m, int order, double dt, double factor, const double *pr,
                             const double *rho, const double *velT, double *velTT, unsigned long long *stats,
                             void *stream);
int sipg_pressure_projection_host(sipg_mesh *m, int order, double dt, double factor, const double *pr,
                                  const double *rho, const double *velT, double *velTT, double *stats);

/* ---- pressure right-hand side: replaces, in INSSolver3D::pressure
 * (src/solvers/3d/ins_solver.cpp:313-322; 2D src/solvers/2d/ins_solver.cpp:269,
 * 309-319; MPINSSolver3D mp_ins_solver.cpp:581-612 with its own dPdN update),
 * mesh->div_with_central_flux(velT) (OP2-DG-Toolkit, unvendored), ins_3d_pr_1 /
 * ins_pressure_rhs_2d (divVelT *= -1/dt; dPdN_old = b0 dPdN + b1 dPdN_old), the
 * LIFT of dPdN_old and mesh->mass, as one kernel:
 *   rhs = J M ( -div_c(velT) / dt + LIFT (b0 dPdN + b1 dPdN_old) ),
 * div_c = sum_d d(u_d)/dx_d + LIFT (fscale n . (u+ - u-) / 2) over interior faces
 * (central flux; boundary faces add nothing). dPdN_old is updated in place. The
 * Neumann data dPdN (the curl-curl boundary term of ins_3d_pr_0.h / mp_ins_3d_pr_0.h:
 * sipg_ins_pressure_neumann in 3D, else the caller's) and dPdN_old are K x (dim + 1) x Nfp in the
 * face-node order of the reference's FMASK, or NULL (zero; dPdN_old NULL is not
 * written). velT: dim x K x Np; rhs: K x Np. The Dirichlet data of
 * ins_3d_pr_dirichlet enter through sipg_op_apply_bc_host as before. Device
 * pointers, or host pointers in the synchronous _host variant. */
int sipg_pressure_rhs(sipg_mesh *m, int order, double dt, double b0, double b1, const double *velT,
                      const double *dPdN, double *dPdN_old, double *rhs, void *stream);
int sipg_pressure_rhs_host(sipg_mesh *m, int order, double dt, double b0, double b1, const double *velT,
                           const double *dPdN, double *dPdN_old, double *rhs);

/* Viscous right-hand side of the two-phase time step, MPINSSolver3D::viscosity
 * (src/solvers/3d/mp_ins_solver.cpp:669-694): mp_ins_3d_vis_0 then mesh->mass on
 * each component, as one kernel. rhs_c = J M (fact0 rho velTT_c), mm_factor =
 * fact1 rho (the mass factor of the viscous Helmholtz operator); fact0 =
 * Re / dt, fact1 = g0 Re / dt. rho, mm_factor: K x Np; velTT, rhs: dim x K x Np
 * (device pointers, or host pointers in the synchronous _host variant). The
 * boundary data of ins_3d_vis_{x,y,z} come from the problem's callbacks and enter
 * through sipg_op_apply_bc_host. */
int sipg_viscous_rhs(sipg_mesh *m, int order, double fact0, double fact1, const double *rho, const double *velTT,
                     double *rhs, double *mm_factor, void *stream);
int sipg_viscous_rhs_host(sipg_mesh *m, int order, double fact0, double fact1, const double *rho,
                          const double *velTT, double *rhs, double *mm_factor);

/* Non-linear advection step of the 3D time step, INSSolverBase3D::advec_current_non_linear
 * and advec_standard (src/solvers/3d/ins_solver_base.cpp:224-329, 451-480): N = div(u (x) u)
 * with Lax-Friedrichs face fluxes (ins_3d_advec_0/1/2 and LIFT) and the extrapolated
 * velocity velT = a0 u + a1 u_old - dt (b0 N + b1 N_old) (ins_3d_advec_3), in one kernel.
 * vel, vel_old, N_old, N, velT: 3 x K x Np; vel_bc: Kb velocity boundary types of the
 * reference's problem_specific_3d.h (0 no-slip, 1 slip, 2 natural outflow). Device
 * pointers on `stream`, or host pointers in the synchronous _host variant. */
int sipg_ins_advection(sipg_mesh *m, int order, double dt, double a0, double a1, double b0, double b1,
                       const double *vel, const double *vel_old, const double *N_old, const int *vel_bc,
                       double *N, double *velT, void *stream);
int sipg_ins_advection_host(sipg_mesh *m, int order, double dt, double a0, double a1, double b0, double b1,
                            const double *vel, const double *vel_old, const double *N_old, const int *vel_bc,
                            double *N, double *velT);

/* Curl-curl Neumann data of the multiphase pressure step, MPINSSolver3D::
 * apply_pressure_neumann_bc (src/solvers/3d/mp_ins_solver.cpp:450-493): on no-slip and
 * slip walls dPdN = fscale n . (-N - curl(mu curl u) / (Re rho)) at the face nodes
 * (mesh->curl, mp_ins_3d_pr_mu, mp_ins_3d_pr_0), zero on the other faces; the input
 * of sipg_pressure_rhs. With mu = rho = 1 it is the single-phase INSSolver3D's
 * ins_3d_pr_0 (src/kernels/ins_3d_pr_0.h). vel, N: 3 x K x Np; mu, rho: K x Np;
 * dPdN: K x 4 x Nfp. */
int sipg_ins_pressure_neumann(sipg_mesh *m, int order, double reynolds, const double *vel, const double *N,
                              const double *mu, const double *rho, const int *vel_bc, double *dPdN, void *stream);
int sipg_ins_pressure_neumann_host(sipg_mesh *m, int order, double reynolds, const double *vel, const double *N,
                                   const double *mu, const double *rho, const int *vel_bc, double *dPdN);

/* ---- two-phase time step: replaces MPINSSolver3D (src/solvers/3d/mp_ins_solver.cpp:
 * 182-285: init, step = advection, pressure, viscosity, surface) with its level set
 * (LevelSetSolver3D, src/solvers/3d/ls_solver.cpp:106-257) for problems with no-slip
 * and slip walls and natural outflow, no surface tension, sub-cycling, filtering or
 * shock capturing. Every field stays on the device; a step runs
 *   advection     sipg_ins_advection's kernel, plus the body force;
 *   pressure      Neumann data (sipg_ins_pressure_neumann), right-hand side
 *                 (sipg_pressure_rhs), factor 1/rho, p-multigrid set-up and solve from
 *                 the extrapolated initial guess, sipg_pressure_projection;
 *   viscosity     sipg_viscous_rhs, factor mu and mass factor g0 Re rho / dt, set-up and
 *                 three Jacobi-PCG solves (FactorMMPoissonMatrixFreeDiag3D +
 *                 PETScJacobiSolver) with zero Dirichlet data on no-slip walls, or with
 *                 slip walls one solve of the vector operator (ViscousSolver3D);
 *   surface       the level-set advection (three Runge-Kutta stages), every reinit_freq
 *                 steps its reinitialisation (sipg_ls_reinit_host), then rho and mu;
 * then dt = cfl h / ((p+1)^2 max(1, max |u|)) (INSSolverBase3D::max_vel) and the second-
 * order coefficients (a0, a1, b0, b1, g0) = (2, -0.5, 2, -1, 1.5) after the first step. */
typedef struct {
  int order;                 /* DG order */
  double reynolds;           /* r_ynolds */
  double rho0, rho1;         /* density where s > 0 and where s < 0 (fluid-constants) */
  double mu0, mu1;           /* viscosity likewise */
  double gravity;            /* body force -gravity along y; 0: none, as the reference's 3D
                                solver (the 2D solver's gravity adds it to N_y,
                                ins_advec_intermediate_vel_grav_2d.h; here also to the
                                pressure Neumann data) */
  double ls_alpha;           /* interface half-width alpha in units of the largest element
                                size (level-set-options alpha, default 24) */
  double cfl;                /* multiplies the reference's time step (1) */
  int extrapolate_history;   /* pressure initial guess from this many past solutions (3);
                                0: the previous pressure */
  int pr_over_int;           /* [pressure-solve] over_int: 1/rho at the cubature points of the
                                over-integrated operator (update_pressure_matrices_oi,
                                mp_ins_solver.cpp:524-544), the V-cycle on its nodal
                                projection; 0: the nodal factor 1/rho. The pressure gradient
                                of the projection step is the nodal one either way. */
  int reinit_freq;           /* level-set-options reinit_freq: reinitialise every this many steps
                                (24); 0: never */
  int reinit_ic;             /* level-set-options reinit_ic: reinitialise the initial level set (1) */
  double ls_cap;             /* LS_CAP of problem_specific_3d.h (1): the reinitialised level set's bound */
  int pr_setup_every;        /* the pressure p-multigrid set up again every this many steps (1,
                                the reference's update_pressure_matrices every step); between
                                set-ups the outer operator (and in nodal mode the finest
                                level) takes the new factor while the smoother blocks,
                                eigenvalue bounds and coarse levels lag: a fixed
                                preconditioner per solve, the same tolerance */
  int viscous_kind;          /* [viscous-solve] preconditioner: SIPG_SOLVER_JACOBI (default,
                                PETScJacobiSolver), SIPG_SOLVER_BLOCK_JACOBI
                                (PETScBlockJacobiSolver, mp_ins_solver.cpp:113-121), or
                                SIPG_SOLVER_PMULTIGRID with viscous.n_levels 0: the FP64
                                flexible PCG preconditioned by viscous.coarse_iters
                                Jacobi-PCG iterations on the same operator in
                                viscous.precision (SIPG_FP32: TF32 applies); no reference
                                counterpart, same tolerance as the Jacobi solve */
  /* The pressure p-multigrid (SIPG_SOLVER_PMULTIGRID: precision of the V-cycle,
   * tolerances, [p-multigrid] keys; n_levels 0 = orders p, p-1, ..., 1; nullspace is
   * set from the boundary types) and the viscous Jacobi-PCG options. Defaults: the
   * tolerances of setup_pressure_viscous_solvers (ins_solver_base.cpp:149-184) and
   * eigen_val_saftey_factor 2.5 of the reference's 3D two-phase examples
   * (examples/3d/oscillating_droplet/config.ini:30). */
  sipg_solver_opts pressure;
  sipg_solver_opts viscous;
} sipg_ins3d_opts;

typedef struct {
  double time, dt;           /* after the step: the time reached and the next dt */
  int pr_iters, vis_iters[3];
  double pr_rel_res, vis_rel_res[3];
  double max_vel;            /* max(1, max |u|) after the step */
  double ms_advection, ms_pressure, ms_viscosity, ms_surface; /* device time per part */
  double ms_pressure_setup;  /* of ms_pressure: new factor (and over-integrated blocks) and the
                                p-multigrid set-up */
  double ms_pressure_solve;  /* of ms_pressure: the solve */
  unsigned long long proj_converged; /* elements whose velocity projection converged */
} sipg_ins3d_step_info;

typedef struct sipg_ins3d sipg_ins3d;
int sipg_ins3d_default_opts(sipg_ins3d_opts *o);
/* Closest-point reinitialisation of a level set alone, LevelSetSolver3D::reinitLS
 * (src/solvers/3d/ls_solver.cpp:719-860) as the time step runs it: the zero set sampled
 * in the elements where s changes sign, each node's closest sample, a Newton
 * closest-point iteration on that element's polynomial, s = +-distance clamped to
 * +-ls_cap (ls_post_reinit). s: K x Np host array, in place. */
int sipg_ls_reinit_host(sipg_mesh *m, int order, double ls_cap, double *s);
/* vel_bc: Kb velocity boundary types (0 no-slip, 1 slip, 2 natural outflow). With a slip
 * wall the three velocity components are solved together on the vector operator
 * (uses_slip_bcs: FactorViscousMatrix3D + ViscousSolver3D, mp_ins_solver.cpp:95-110, 699-790;
 * vis_iters then repeats the one solve's count). */
int sipg_ins3d_create(sipg_mesh *m, const sipg_ins3d_opts *o, const int *vel_bc, sipg_ins3d **out);
/* Initial velocity (3 x K x Np) and level set (K x Np), host arrays: the reference's
 * ps3d_set_ic / ps3d_set_surface callbacks evaluated by the caller. Sets time 0, the
 * first-order coefficients, rho and mu, and the first dt. */
int sipg_ins3d_set_state_host(sipg_ins3d *ins, const double *vel, const double *s);
/* nsteps steps; info (may be NULL) describes the last one. */
int sipg_ins3d_step(sipg_ins3d *ins, int nsteps, sipg_ins3d_step_info *info);
/* Copies of the current fields (NULL: skipped): vel 3 x K x Np, pr, s, rho, mu K x Np. */
int sipg_ins3d_get_state_host(sipg_ins3d *ins, double *vel, double *pr, double *s, double *rho, double *mu);
void sipg_ins3d_destroy(sipg_ins3d *ins);

/* Number of kernels this library has launched so far in the process
 * (diagnostics for benchmarks; no reference counterpart). */
int sipg_launch_count(unsigned long long *n);

/* Bounded waits inside the library's kernels on the current device that ran
 * out (an MMA completion never arrived); the kernel that saw one stopped its
 * work. 0 in a healthy run (diagnostics; no reference counterpart). */
int sipg_kernel_wait_timeouts(unsigned long long *n);

#ifdef __cplusplus
}
#endif
#endif
