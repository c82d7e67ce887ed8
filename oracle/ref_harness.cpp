// Reference-kernel harness: the reference's own OP2 user kernels, specialised
// per (dimension, order) by gen_ref_kernels.py, driven call-for-call in the
// reference's order. TEST INFRASTRUCTURE ONLY: built into oracle/_ref/ from the
// sources under the reference tree, used to pin the oracle and as the CPU
// baseline of the benchmark. Exposes the oracle's signatures with a ref_ prefix.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <vector>

#include "sipg_oracle.h"

#define DG_MAT_IND(row, col, num_rows, num_cols) ((row) + (col) * (num_rows))
using std::fmax;
using std::isnan;


// One namespace per (dim, order); geof index macros follow the shared layout.
#define RX_IND 0
#define RY_IND 1

#define DIM 2
#define SX_IND 2
#define SY_IND 3
#define J_IND 4

namespace d2p1 { constexpr int ORDER = 1, NP = 3, NPF = 2, NF = 3;
#include "ref_harness_pre.inc"
#include "_ref/gen/d2p1/all.h"
#include "_ref/gen/d2p1/dispatch.inc"
#include "ref_harness_body.inc"
}
namespace d2p2 { constexpr int ORDER = 2, NP = 6, NPF = 3, NF = 3;
#include "ref_harness_pre.inc"
#include "_ref/gen/d2p2/all.h"
#include "_ref/gen/d2p2/dispatch.inc"
#include "ref_harness_body.inc"
}
namespace d2p3 { constexpr int ORDER = 3, NP = 10, NPF = 4, NF = 3;
#include "ref_harness_pre.inc"
#include "_ref/gen/d2p3/all.h"
#include "_ref/gen/d2p3/dispatch.inc"
#include "ref_harness_body.inc"
}
namespace d2p4 { constexpr int ORDER = 4, NP = 15, NPF = 5, NF = 3;
#include "ref_harness_pre.inc"
#include "_ref/gen/d2p4/all.h"
#include "_ref/gen/d2p4/dispatch.inc"
#include "ref_harness_body.inc"
}
#undef DIM
#undef SX_IND
#undef SY_IND
#undef J_IND

#define DIM 3
#define RZ_IND 2
#define SX_IND 3
#define SY_IND 4
#define SZ_IND 5
#define TX_IND 6
#define TY_IND 7
#define TZ_IND 8
#define J_IND 9
namespace d3p1 { constexpr int ORDER = 1, NP = 4, NPF = 3, NF = 4;
#include "ref_harness_pre.inc"
#include "_ref/gen/d3p1/all.h"
#include "_ref/gen/d3p1/dispatch.inc"
#include "ref_harness_body.inc"
}
namespace d3p2 { constexpr int ORDER = 2, NP = 10, NPF = 6, NF = 4;
#include "ref_harness_pre.inc"
#include "_ref/gen/d3p2/all.h"
#include "_ref/gen/d3p2/dispatch.inc"
#include "ref_harness_body.inc"
}
namespace d3p3 { constexpr int ORDER = 3, NP = 20, NPF = 10, NF = 4;
#include "ref_harness_pre.inc"
#include "_ref/gen/d3p3/all.h"
#include "_ref/gen/d3p3/dispatch.inc"
#include "ref_harness_body.inc"
}
namespace d3p4 { constexpr int ORDER = 4, NP = 35, NPF = 15, NF = 4;
#include "ref_harness_pre.inc"
#include "_ref/gen/d3p4/all.h"
#include "_ref/gen/d3p4/dispatch.inc"
#include "ref_harness_body.inc"
}

#define DISPATCH(CALL)                                              \
  switch (m->dim * 10 + m->order) {                                 \
    case 21: d2p1::CALL; return 0;                                  \
    case 22: d2p2::CALL; return 0;                                  \
    case 23: d2p3::CALL; return 0;                                  \
    case 24: d2p4::CALL; return 0;                                  \
    case 31: d3p1::CALL; return 0;                                  \
    case 32: d3p2::CALL; return 0;                                  \
    case 33: d3p3::CALL; return 0;                                  \
    case 34: d3p4::CALL; return 0;                                  \
    default: return -1;                                             \
  }

extern "C" {
// The Reynolds number of the multiphase pressure boundary kernel, every build.
void ref_set_reynolds(double re) {
  d2p1::r_ynolds = d2p2::r_ynolds = d2p3::r_ynolds = d2p4::r_ynolds = re;
  d3p1::r_ynolds = d3p2::r_ynolds = d3p3::r_ynolds = d3p4::r_ynolds = re;
}
// The fluid constants of ls_step, every 3D build.
void ref_set_fluid(double r0, double r1, double m0, double m1) {
  d3p1::rho0 = d3p2::rho0 = d3p3::rho0 = d3p4::rho0 = r0;
  d3p1::rho1 = d3p2::rho1 = d3p3::rho1 = d3p4::rho1 = r1;
  d3p1::mu0 = d3p2::mu0 = d3p3::mu0 = d3p4::mu0 = m0;
  d3p1::mu1 = d3p2::mu1 = d3p3::mu1 = d3p4::mu1 = m1;
}
int ref_mult(const oracle_mesh *m, int ncomp, const int *bc_types, const double *factor,
             const double *mm_factor, double mm_scalar, int flags, const double *const *x,
             double *const *y) {
  DISPATCH(mult_api(m, ncomp, bc_types, factor, mm_factor, mm_scalar, flags, x, y))
}
int ref_apply_bc(const oracle_mesh *m, int ncomp, const int *bc_types, const double *factor,
                 const double *const *bc, double *const *rhs) {
  DISPATCH(apply_bc_api(m, ncomp, bc_types, factor, bc, rhs))
}
int ref_diag(const oracle_mesh *m, int ncomp, const int *bc_types, const double *factor,
             const double *mm_factor, double mm_scalar, double *diag) {
  DISPATCH(diag_api(m, ncomp, bc_types, factor, mm_factor, mm_scalar, diag))
}
int ref_block_diag(const oracle_mesh *m, int ncomp, const int *bc_types, const double *factor,
                   const double *mm_factor, double mm_scalar, int inv, double *blocks) {
  DISPATCH(block_diag_api(m, ncomp, bc_types, factor, mm_factor, mm_scalar, inv, blocks))
}
int ref_solve(const oracle_mesh *m, const oracle_solver_opts *o, const double *b, double *x,
              oracle_solve_info *info) {
  DISPATCH(solve_api(m, o, b, x, info))
}
int ref_project_velocity(const oracle_mesh *m, double dt, double factor, const double *dp,
                         const double *velT, double *velTT, double *stats) {
  DISPATCH(project_velocity_api(m, dt, factor, dp, velT, velTT, stats))
}
// One reference kernel by name on caller buffers (args: its arguments in order),
// with the reference-element tables of m; -1 for an unknown name or element.
int ref_kernel(const oracle_mesh *m, const char *name, void **args) {
  switch (m->dim * 10 + m->order) {
    case 21: d2p1::load_constants(m); return d2p1::call_kernel(name, args);
    case 22: d2p2::load_constants(m); return d2p2::call_kernel(name, args);
    case 23: d2p3::load_constants(m); return d2p3::call_kernel(name, args);
    case 24: d2p4::load_constants(m); return d2p4::call_kernel(name, args);
    case 31: d3p1::load_constants(m); return d3p1::call_kernel(name, args);
    case 32: d3p2::load_constants(m); return d3p2::call_kernel(name, args);
    case 33: d3p3::load_constants(m); return d3p3::call_kernel(name, args);
    case 34: d3p4::load_constants(m); return d3p4::call_kernel(name, args);
    default: return -1;
  }
}
}
