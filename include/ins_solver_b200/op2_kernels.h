// Per-element forms of the reference's OP2 user kernels on the solve path.
//
// Each function has the name and the argument list of a kernel under the
// reference's src/kernels/ (for example fvmf_3d_mult_flux.h:1-5,
// cg3_update_res.h:1-3) and computes the same values for one cell (or one face,
// for the face loops), so that a caller that drives those kernels through
// op_par_loop can call these instead, and so that each kernel can be checked on
// its own against the reference. The fused tensor-core kernels of libsipg_b200
// are the performance path; these are the per-kernel drop-ins.
//
// Compile-time sizes replace the reference build's macros: the polynomial order
// is the template argument ORDER (DG_ORDER), the dimension is part of the name
// (fvmf_3d_* / vmf_3d_* / cg3_* in 3D, fvmf_2d_* / vmf_2d_* / cg_* in 2D; the
// kernels the two builds share take DIM as well), and DG_FP is double.
// The reference-element tables that the reference's kernels read by name
// (dg_Dr_kernel, dg_Ds_kernel, dg_Dt_kernel, dg_Mass_kernel, dg_MM_F0..3_kernel,
// dg_InvMass_kernel, FMASK) come from ref_tables<DIM, ORDER>(), which the program defines for every
// (DIM, ORDER) it uses, as the reference's build generates those constants.
//
// SIPG_OP2_REF_QUIRKS (default 1) keeps the reference's statements where they
// differ from the SIPG formula they implement (vmf_3d_mult_flux.h:10-11 drops
// the n_z term of n . {grad u}; fvmf_3d_op1.h:17-18 multiplies without the
// transpose; fvmf_2d_op1.h:20-37 applies the factor between the transposed
// derivative and the mass matrix); 0 gives the corrected forms.
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define SIPG_OP2_HD __host__ __device__ inline
#else
#define SIPG_OP2_HD inline
#endif

#ifndef SIPG_OP2_REF_QUIRKS
#define SIPG_OP2_REF_QUIRKS 1
#endif

namespace ins_solver_b200 {
namespace op2 {

// Sizes of one (DIM, ORDER) and the positions in geof (3D: rx ry rz sx sy sz tx
// ty tz J; 2D: rx ry sx sy J).
template <int DIM, int ORDER>
struct Dg {
  static constexpr int NP = DIM == 3 ? (ORDER + 1) * (ORDER + 2) * (ORDER + 3) / 6 : (ORDER + 1) * (ORDER + 2) / 2;
  static constexpr int NPF = DIM == 3 ? (ORDER + 1) * (ORDER + 2) / 2 : ORDER + 1;
  static constexpr int NUM_FACES = DIM + 1;
  static constexpr int RX = 0, RY = 1, RZ = 2;
  static constexpr int SX = DIM == 3 ? 3 : 2, SY = DIM == 3 ? 4 : 3, SZ = 5;
  static constexpr int TX = 6, TY = 7, TZ = 8;
  static constexpr int J = DIM == 3 ? 9 : 4;
  // penalty constant of fvmf_*_calc_tau_*: 2 (p + 1) (p + 2)
  static constexpr double TAU_ORDER = 2.0 * (ORDER + 1) * (ORDER + 2);
};

// Reference-element tables of one (DIM, ORDER): NP x NP matrices column-major
// (entry (i, j) at i + j * NP, as the dg_*_kernel constants), MM_F[f] the face
// mass of face f embedded in the volume, fmask the volume node of each face node
// (NUM_FACES x NPF, as FMASK).
struct RefTables {
  const double *Dr, *Ds, *Dt, *Mass;
  const double *MM_F[4];
  const int *fmask;
  const double *InvMass;  // inverse of Mass (dg_InvMass_kernel), read by the projection solve
};

template <int DIM, int ORDER>
SIPG_OP2_HD const RefTables &ref_tables();

namespace detail {

SIPG_OP2_HD double dmax(double a, double b) { return a > b ? a : b; }

// y = A x for a column-major NP x NP matrix (op2_in_kernel_gemv, no transpose)
template <int NP>
SIPG_OP2_HD void matvec(const double *A, const double *x, double *y) {
  for (int i = 0; i < NP; ++i) {
    double s = 0.0;
    for (int j = 0; j < NP; ++j) s += A[i + j * NP] * x[j];
    y[i] = s;
  }
}

// Physical derivative matrix of direction d (0 x, 1 y, 2 z), column-major:
// Dd = r_d Dr + s_d Ds (+ t_d Dt)
template <int DIM, int ORDER>
SIPG_OP2_HD double dphys(const RefTables &t, const double *geof, int d, int ind) {
  using G = Dg<DIM, ORDER>;
  const int r = d == 0 ? G::RX : d == 1 ? G::RY : G::RZ;
  const int s = d == 0 ? G::SX : d == 1 ? G::SY : G::SZ;
  double v = geof[r] * t.Dr[ind] + geof[s] * t.Ds[ind];
  if (DIM == 3) v += geof[d == 0 ? G::TX : d == 1 ? G::TY : G::TZ] * t.Dt[ind];
  return v;
}

}  // namespace detail

// ---------------------------------------------------------------- CG (cg3_*.h: 3 components, cg_*.h: 2)

template <int ORDER>
SIPG_OP2_HD void cg3_alpha(double *tmp_alpha_0, double *tmp_alpha_1, const double *r0, const double *r1,
                           const double *r2, const double *p0, const double *p1, const double *p2, const double *Ax0,
                           const double *Ax1, const double *Ax2) {
  double rr = 0.0, pap = 0.0;
  for (int i = 0; i < Dg<3, ORDER>::NP; ++i) {
    rr += r0[i] * r0[i] + r1[i] * r1[i] + r2[i] * r2[i];
    pap += p0[i] * Ax0[i] + p1[i] * Ax1[i] + p2[i] * Ax2[i];
  }
  *tmp_alpha_0 += rr;
  *tmp_alpha_1 += pap;
}

template <int ORDER>
SIPG_OP2_HD void cg3_alpha_pre(double *tmp_alpha_0, double *tmp_alpha_1, const double *r0, const double *r1,
                               const double *r2, const double *z0, const double *z1, const double *z2,
                               const double *p0, const double *p1, const double *p2, const double *Ax0,
                               const double *Ax1, const double *Ax2) {
  double rz = 0.0, pap = 0.0;
  for (int i = 0; i < Dg<3, ORDER>::NP; ++i) {
    rz += r0[i] * z0[i] + r1[i] * z1[i] + r2[i] * z2[i];
    pap += p0[i] * Ax0[i] + p1[i] * Ax1[i] + p2[i] * Ax2[i];
  }
  *tmp_alpha_0 += rz;
  *tmp_alpha_1 += pap;
}

template <int ORDER>
SIPG_OP2_HD void cg3_block_jacobi(const double *u_pre_mat, const double *v_pre_mat, const double *w_pre_mat,
                                  const double *u_in, const double *v_in, const double *w_in, double *u_out,
                                  double *v_out, double *w_out) {
  constexpr int NP = Dg<3, ORDER>::NP;
  detail::matvec<NP>(u_pre_mat, u_in, u_out);
  detail::matvec<NP>(v_pre_mat, v_in, v_out);
  detail::matvec<NP>(w_pre_mat, w_in, w_out);
}

template <int ORDER>
SIPG_OP2_HD void cg3_compute_beta(double *beta, const double *r0, const double *r1, const double *r2) {
  double s = 0.0;
  for (int i = 0; i < Dg<3, ORDER>::NP; ++i) s += r0[i] * r0[i] + r1[i] * r1[i] + r2[i] * r2[i];
  *beta += s;
}

template <int ORDER>
SIPG_OP2_HD void cg3_compute_beta_pre(double *beta, const double *r0, const double *r1, const double *r2,
                                      const double *z0, const double *z1, const double *z2) {
  double s = 0.0;
  for (int i = 0; i < Dg<3, ORDER>::NP; ++i) s += r0[i] * z0[i] + r1[i] * z1[i] + r2[i] * z2[i];
  *beta += s;
}

template <int ORDER>
SIPG_OP2_HD void cg3_compute_beta_pre_flex(double *beta, const double *r0, const double *r1, const double *r2,
                                           const double *z0, const double *z1, const double *z2, const double *z0_1,
                                           const double *z1_1, const double *z2_1) {
  double s = 0.0;
  for (int i = 0; i < Dg<3, ORDER>::NP; ++i)
    s += r0[i] * (z0[i] - z0_1[i]) + r1[i] * (z1[i] - z1_1[i]) + r2[i] * (z2[i] - z2_1[i]);
  *beta += s;
}

template <int ORDER>
SIPG_OP2_HD void cg3_jacobi(const double *u_diag, const double *v_diag, const double *w_diag, const double *u_in,
                            const double *v_in, const double *w_in, double *u, double *v, double *w) {
  for (int i = 0; i < Dg<3, ORDER>::NP; ++i) {
    u[i] = u_in[i] / u_diag[i];
    v[i] = v_in[i] / v_diag[i];
    w[i] = w_in[i] / w_diag[i];
  }
}

template <int ORDER>
SIPG_OP2_HD void cg3_recp_factor_inv_mass(const double *factor, double *u, double *v, double *w) {
  for (int i = 0; i < Dg<3, ORDER>::NP; ++i) {
    u[i] /= factor[i];
    v[i] /= factor[i];
    w[i] /= factor[i];
  }
}

template <int ORDER>
SIPG_OP2_HD void cg3_residual(double *residual, const double *rhs0, const double *rhs1, const double *rhs2,
                              double *r0, double *r1, double *r2) {
  double s = 0.0;
  for (int i = 0; i < Dg<3, ORDER>::NP; ++i) {
    r0[i] = rhs0[i] - r0[i];
    r1[i] = rhs1[i] - r1[i];
    r2[i] = rhs2[i] - r2[i];
    s += r0[i] * r0[i] + r1[i] * r1[i] + r2[i] * r2[i];
  }
  *residual += s;
}

template <int ORDER>
SIPG_OP2_HD void cg3_update_ans(const double *alpha, const double *p0, const double *p1, const double *p2, double *u,
                                double *v, double *w) {
  for (int i = 0; i < Dg<3, ORDER>::NP; ++i) {
    u[i] += *alpha * p0[i];
    v[i] += *alpha * p1[i];
    w[i] += *alpha * p2[i];
  }
}

template <int ORDER>
SIPG_OP2_HD void cg3_update_p(const double *beta, const double *r0, const double *r1, const double *r2, double *p0,
                              double *p1, double *p2) {
  for (int i = 0; i < Dg<3, ORDER>::NP; ++i) {
    p0[i] = r0[i] + *beta * p0[i];
    p1[i] = r1[i] + *beta * p1[i];
    p2[i] = r2[i] + *beta * p2[i];
  }
}

template <int ORDER>
SIPG_OP2_HD void cg3_update_res(const double *alpha, double *residual, const double *Ap0, const double *Ap1,
                                const double *Ap2, double *r0, double *r1, double *r2) {
  double s = 0.0;
  for (int i = 0; i < Dg<3, ORDER>::NP; ++i) {
    r0[i] -= *alpha * Ap0[i];
    r1[i] -= *alpha * Ap1[i];
    r2[i] -= *alpha * Ap2[i];
    s += r0[i] * r0[i] + r1[i] * r1[i] + r2[i] * r2[i];
  }
  *residual += s;
}

template <int ORDER>
SIPG_OP2_HD void cg_alpha(double *tmp_alpha_0, double *tmp_alpha_1, const double *r0, const double *r1,
                          const double *p0, const double *p1, const double *Ax0, const double *Ax1) {
  double rr = 0.0, pap = 0.0;
  for (int i = 0; i < Dg<2, ORDER>::NP; ++i) {
    rr += r0[i] * r0[i] + r1[i] * r1[i];
    pap += p0[i] * Ax0[i] + p1[i] * Ax1[i];
  }
  *tmp_alpha_0 += rr;
  *tmp_alpha_1 += pap;
}

template <int ORDER>
SIPG_OP2_HD void cg_alpha_pre(double *tmp_alpha_0, double *tmp_alpha_1, const double *r0, const double *r1,
                              const double *z0, const double *z1, const double *p0, const double *p1,
                              const double *Ax0, const double *Ax1) {
  double rz = 0.0, pap = 0.0;
  for (int i = 0; i < Dg<2, ORDER>::NP; ++i) {
    rz += r0[i] * z0[i] + r1[i] * z1[i];
    pap += p0[i] * Ax0[i] + p1[i] * Ax1[i];
  }
  *tmp_alpha_0 += rz;
  *tmp_alpha_1 += pap;
}

template <int ORDER>
SIPG_OP2_HD void cg_block_jacobi(const double *u_pre_mat, const double *v_pre_mat, const double *u_in,
                                 const double *v_in, double *u_out, double *v_out) {
  constexpr int NP = Dg<2, ORDER>::NP;
  detail::matvec<NP>(u_pre_mat, u_in, u_out);
  detail::matvec<NP>(v_pre_mat, v_in, v_out);
}

template <int ORDER>
SIPG_OP2_HD void cg_compute_beta(double *beta, const double *r0, const double *r1) {
  double s = 0.0;
  for (int i = 0; i < Dg<2, ORDER>::NP; ++i) s += r0[i] * r0[i] + r1[i] * r1[i];
  *beta += s;
}

template <int ORDER>
SIPG_OP2_HD void cg_compute_beta_pre(double *beta, const double *r0, const double *r1, const double *z0,
                                     const double *z1) {
  double s = 0.0;
  for (int i = 0; i < Dg<2, ORDER>::NP; ++i) s += r0[i] * z0[i] + r1[i] * z1[i];
  *beta += s;
}

template <int ORDER>
SIPG_OP2_HD void cg_compute_beta_pre_flex(double *beta, const double *r0, const double *r1, const double *z0,
                                          const double *z1, const double *z0_1, const double *z1_1) {
  double s = 0.0;
  for (int i = 0; i < Dg<2, ORDER>::NP; ++i) s += r0[i] * (z0[i] - z0_1[i]) + r1[i] * (z1[i] - z1_1[i]);
  *beta += s;
}

template <int ORDER>
SIPG_OP2_HD void cg_jacobi(const double *u_diag, const double *v_diag, const double *u_in, const double *v_in,
                           double *u, double *v) {
  for (int i = 0; i < Dg<2, ORDER>::NP; ++i) {
    u[i] = u_in[i] / u_diag[i];
    v[i] = v_in[i] / v_diag[i];
  }
}

template <int ORDER>
SIPG_OP2_HD void cg_recp_factor_inv_mass(const double *factor, double *u, double *v) {
  for (int i = 0; i < Dg<2, ORDER>::NP; ++i) {
    u[i] /= factor[i];
    v[i] /= factor[i];
  }
}

template <int ORDER>
SIPG_OP2_HD void cg_residual(double *residual, const double *rhs0, const double *rhs1, double *r0, double *r1) {
  double s = 0.0;
  for (int i = 0; i < Dg<2, ORDER>::NP; ++i) {
    r0[i] = rhs0[i] - r0[i];
    r1[i] = rhs1[i] - r1[i];
    s += r0[i] * r0[i] + r1[i] * r1[i];
  }
  *residual += s;
}

template <int ORDER>
SIPG_OP2_HD void cg_update_ans(const double *alpha, const double *p0, const double *p1, double *u, double *v) {
  for (int i = 0; i < Dg<2, ORDER>::NP; ++i) {
    u[i] += *alpha * p0[i];
    v[i] += *alpha * p1[i];
  }
}

template <int ORDER>
SIPG_OP2_HD void cg_update_p(const double *beta, const double *r0, const double *r1, double *p0, double *p1) {
  for (int i = 0; i < Dg<2, ORDER>::NP; ++i) {
    p0[i] = r0[i] + *beta * p0[i];
    p1[i] = r1[i] + *beta * p1[i];
  }
}

template <int ORDER>
SIPG_OP2_HD void cg_update_res(const double *alpha, double *residual, const double *Ap0, const double *Ap1,
                               double *r0, double *r1) {
  double s = 0.0;
  for (int i = 0; i < Dg<2, ORDER>::NP; ++i) {
    r0[i] -= *alpha * Ap0[i];
    r1[i] -= *alpha * Ap1[i];
    s += r0[i] * r0[i] + r1[i] * r1[i];
  }
  *residual += s;
}

// ---------------------------------------------------------------- small cell kernels (both builds)

template <int DIM, int ORDER>
SIPG_OP2_HD void constant_mult(const double *constant, double *val) {
  for (int i = 0; i < Dg<DIM, ORDER>::NP; ++i) val[i] *= *constant;
}

template <int DIM, int ORDER>
SIPG_OP2_HD void copy_dg_np(const double *in, double *out) {
  for (int i = 0; i < Dg<DIM, ORDER>::NP; ++i) out[i] = in[i];
}

template <int DIM, int ORDER>
SIPG_OP2_HD void copy_dg_np_mat(const double *in, double *out) {
  constexpr int NP = Dg<DIM, ORDER>::NP;
  for (int i = 0; i < NP * NP; ++i) out[i] = in[i];
}

template <int DIM, int ORDER>
SIPG_OP2_HD void reciprocal(const double *in, double *out) {
  for (int i = 0; i < Dg<DIM, ORDER>::NP; ++i) out[i] = 1.0 / in[i];
}

template <int DIM, int ORDER>
SIPG_OP2_HD void zero_npf_3(double *x, double *y, double *z) {
  using G = Dg<DIM, ORDER>;
  for (int i = 0; i < G::NUM_FACES * G::NPF; ++i) x[i] = y[i] = z[i] = 0.0;
}

// factor = 1 / rho (the pressure Poisson coefficient)
template <int DIM, int ORDER>
SIPG_OP2_HD void poisson_pr_fact(const double *rho, double *factor) {
  for (int i = 0; i < Dg<DIM, ORDER>::NP; ++i) factor[i] = 1.0 / rho[i];
}

// viscous Helmholtz coefficients: factor = mu, mmFactor = mmConst rho
template <int DIM, int ORDER>
SIPG_OP2_HD void poisson_vis_fact(const double *mmConst, const double *mu, const double *rho, double *factor,
                                  double *mmFactor) {
  for (int i = 0; i < Dg<DIM, ORDER>::NP; ++i) {
    factor[i] = mu[i];
    mmFactor[i] = *mmConst * rho[i];
  }
}

// ---------------------------------------------------------------- penalty (fvmf_*_calc_tau_*, vmf_calc_tau_*)

namespace detail {
// interior face: tau of both sides = 2 (p + 1) (p + 2) max over the face nodes of
// max(fscale_L f_L, fscale_R f_R)
template <int DIM, int ORDER>
SIPG_OP2_HD void tau_faces(const int *faceNum, const int *fmaskR_corrected, const double *fscale,
                           const double **factor, double **tau) {
  using G = Dg<DIM, ORDER>;
  const int *fm = ref_tables<DIM, ORDER>().fmask + faceNum[0] * G::NPF;
  double m = 0.0;
  for (int j = 0; j < G::NPF; ++j)
    m = dmax(m, G::TAU_ORDER * dmax(fscale[0] * factor[0][fm[j]], fscale[1] * factor[1][fmaskR_corrected[j]]));
  tau[0][faceNum[0]] = m;
  tau[1][faceNum[1]] = m;
}
// boundary face: 2 (p + 1) (p + 2) fscale max over the face nodes of f
template <int DIM, int ORDER>
SIPG_OP2_HD void tau_bfaces(const int *faceNum, const double *fscale, const double *factor, double *tau) {
  using G = Dg<DIM, ORDER>;
  const int *fm = ref_tables<DIM, ORDER>().fmask + faceNum[0] * G::NPF;
  double m = factor[fm[0]];
  for (int j = 1; j < G::NPF; ++j) m = dmax(m, factor[fm[j]]);
  tau[faceNum[0]] = m * (G::TAU_ORDER * fscale[0]);
}
}  // namespace detail

template <int ORDER>
SIPG_OP2_HD void fvmf_3d_calc_tau_faces(const int *faceNum, const int *fmaskR_corrected, const double *fscale,
                                        const double **factor, double **tau) {
  detail::tau_faces<3, ORDER>(faceNum, fmaskR_corrected, fscale, factor, tau);
}
// 2D: the neighbour's face nodes are its own face's nodes, in reverse order when *reverse
template <int ORDER>
SIPG_OP2_HD void fvmf_2d_calc_tau_faces(const int *faceNum, const bool *reverse, const double *fscale,
                                        const double **factor, double **tau) {
  using G = Dg<2, ORDER>;
  const int *fR = ref_tables<2, ORDER>().fmask + faceNum[1] * G::NPF;
  int fmaskR[G::NPF];
  for (int j = 0; j < G::NPF; ++j) fmaskR[j] = fR[*reverse ? G::NPF - 1 - j : j];
  detail::tau_faces<2, ORDER>(faceNum, fmaskR, fscale, factor, tau);
}
template <int ORDER>
SIPG_OP2_HD void fvmf_3d_calc_tau_bfaces(const int *faceNum, const double *fscale, const double *factor,
                                         double *tau) {
  detail::tau_bfaces<3, ORDER>(faceNum, fscale, factor, tau);
}
template <int ORDER>
SIPG_OP2_HD void fvmf_2d_calc_tau_bfaces(const int *faceNum, const double *fscale, const double *factor,
                                         double *tau) {
  detail::tau_bfaces<2, ORDER>(faceNum, fscale, factor, tau);
}

// constant coefficient
template <int DIM, int ORDER>
SIPG_OP2_HD void vmf_calc_tau_faces(const int *faceNum, const double *fscale, double **tau) {
  const double t = Dg<DIM, ORDER>::TAU_ORDER * detail::dmax(fscale[0], fscale[1]);
  tau[0][faceNum[0]] = t;
  tau[1][faceNum[1]] = t;
}
template <int DIM, int ORDER>
SIPG_OP2_HD void vmf_calc_tau_bfaces(const int *faceNum, const double *fscale, double *tau) {
  tau[faceNum[0]] = Dg<DIM, ORDER>::TAU_ORDER * fscale[0];
}

// ---------------------------------------------------------------- apply: volume terms

// reference derivatives (in place) -> f G^T grad: ux = f (rx ur + sx us + tx ut), ...
template <int ORDER>
SIPG_OP2_HD void fvmf_3d_grad(const double *geof, const double *fact, double *ux, double *uy, double *uz, double *vx,
                              double *vy, double *vz, double *wx, double *wy, double *wz) {
  using G = Dg<3, ORDER>;
  double *comp[3][3] = {{ux, uy, uz}, {vx, vy, vz}, {wx, wy, wz}};
  for (int m = 0; m < G::NP; ++m)
    for (int c = 0; c < 3; ++c) {
      const double ur = comp[c][0][m], us = comp[c][1][m], ut = comp[c][2][m];
      comp[c][0][m] = fact[m] * (geof[G::RX] * ur + geof[G::SX] * us + geof[G::TX] * ut);
      comp[c][1][m] = fact[m] * (geof[G::RY] * ur + geof[G::SY] * us + geof[G::TY] * ut);
      comp[c][2][m] = fact[m] * (geof[G::RZ] * ur + geof[G::SZ] * us + geof[G::TZ] * ut);
    }
}

template <int ORDER>
SIPG_OP2_HD void fvmf_2d_grad(const double *geof, const double *factor, double *ux, double *uy, double *vx,
                              double *vy) {
  using G = Dg<2, ORDER>;
  double *comp[2][2] = {{ux, uy}, {vx, vy}};
  for (int m = 0; m < G::NP; ++m)
    for (int c = 0; c < 2; ++c) {
      const double ur = comp[c][0][m], us = comp[c][1][m];
      comp[c][0][m] = factor[m] * (geof[G::RX] * ur + geof[G::SX] * us);
      comp[c][1][m] = factor[m] * (geof[G::RY] * ur + geof[G::SY] * us);
    }
}

// physical -> reference-direction components for the transposed derivative: (q_r, q_s, q_t) = G q
template <int ORDER>
SIPG_OP2_HD void vmf_3d_mult_cells_geof(const double *geof, double *u_x, double *u_y, double *u_z, double *v_x,
                                        double *v_y, double *v_z, double *w_x, double *w_y, double *w_z) {
  using G = Dg<3, ORDER>;
  double *comp[3][3] = {{u_x, u_y, u_z}, {v_x, v_y, v_z}, {w_x, w_y, w_z}};
  for (int n = 0; n < G::NP; ++n)
    for (int c = 0; c < 3; ++c) {
      const double qx = comp[c][0][n], qy = comp[c][1][n], qz = comp[c][2][n];
      comp[c][0][n] = geof[G::RX] * qx + geof[G::RY] * qy + geof[G::RZ] * qz;
      comp[c][1][n] = geof[G::SX] * qx + geof[G::SY] * qy + geof[G::SZ] * qz;
      comp[c][2][n] = geof[G::TX] * qx + geof[G::TY] * qy + geof[G::TZ] * qz;
    }
}

template <int ORDER>
SIPG_OP2_HD void vmf_2d_mult_cells_geof(const double *geof, double *u_x, double *u_y, double *v_x, double *v_y) {
  using G = Dg<2, ORDER>;
  double *comp[2][2] = {{u_x, u_y}, {v_x, v_y}};
  for (int c = 0; c < 2; ++c)
    for (int n = 0; n < G::NP; ++n) {
      const double qx = comp[c][0][n], qy = comp[c][1][n];
      comp[c][0][n] = geof[G::RX] * qx + geof[G::RY] * qy;
      comp[c][1][n] = geof[G::SX] * qx + geof[G::SY] * qy;
    }
}

namespace detail {
// out_c += J M (mm in_c): nodal mm (per-node factor inside the product) or scalar
template <int DIM, int ORDER, int NC>
SIPG_OP2_HD void mass_terms(const double *geof, const double *mm, bool nodal, const double *const *in,
                            double *const *out) {
  using G = Dg<DIM, ORDER>;
  const double *M = ref_tables<DIM, ORDER>().Mass;
  for (int m = 0; m < G::NP; ++m)
    for (int c = 0; c < NC; ++c) {
      double s = 0.0;
      for (int n = 0; n < G::NP; ++n) s += (nodal ? mm[n] * M[m + n * G::NP] : M[m + n * G::NP]) * in[c][n];
      out[c][m] += nodal ? s * geof[G::J] : *mm * s * geof[G::J];
    }
}
}  // namespace detail

template <int ORDER>
SIPG_OP2_HD void fvmf_3d_mult_mm_geof(const double *geof, const double *mm_factor, const double *u_in,
                                      const double *v_in, const double *w_in, double *u_out, double *v_out,
                                      double *w_out) {
  const double *in[3] = {u_in, v_in, w_in};
  double *out[3] = {u_out, v_out, w_out};
  detail::mass_terms<3, ORDER, 3>(geof, mm_factor, true, in, out);
}
template <int ORDER>
SIPG_OP2_HD void fvmf_2d_mult_mm_geof(const double *geof, const double *mm_factor, const double *u, const double *v,
                                      double *u_out, double *v_out) {
  const double *in[2] = {u, v};
  double *out[2] = {u_out, v_out};
  detail::mass_terms<2, ORDER, 2>(geof, mm_factor, true, in, out);
}
template <int ORDER>
SIPG_OP2_HD void vmf_3d_mult_mm_geof(const double *geof, const double *mm_factor, const double *u, const double *v,
                                     const double *w, double *u_out, double *v_out, double *w_out) {
  const double *in[3] = {u, v, w};
  double *out[3] = {u_out, v_out, w_out};
  detail::mass_terms<3, ORDER, 3>(geof, mm_factor, false, in, out);
}
template <int ORDER>
SIPG_OP2_HD void vmf_2d_mult_mm_geof(const double *geof, const double *mm_factor, const double *u, const double *v,
                                     double *u_out, double *v_out) {
  const double *in[2] = {u, v};
  double *out[2] = {u_out, v_out};
  detail::mass_terms<2, ORDER, 2>(geof, mm_factor, false, in, out);
}

// ---------------------------------------------------------------- apply: boundary traces (vmf_*_mult_avg_jump)

namespace detail {
// Boundary face faceNum[0] of a cell: Dirichlet components add 2 u and grad u at
// the face nodes to the jump / average buffers, Neumann ones nothing; when every
// component is slip (type 2) the normal projection n n^T of u and of each
// derivative component is added instead.
template <int DIM, int ORDER>
SIPG_OP2_HD void avg_jump(const int *const *bc, const int *faceNum, const double *const *n,
                          const double *const *u, const double *const (*du)[3], double *const *jump,
                          double *const (*avg)[3]) {
  using G = Dg<DIM, ORDER>;
  const int *fm = ref_tables<DIM, ORDER>().fmask + faceNum[0] * G::NPF;
  bool slip = true;
  for (int c = 0; c < DIM; ++c) slip = slip && *bc[c] == 2;
  for (int j = 0; j < G::NPF; ++j) {
    const int m = fm[j], k = faceNum[0] * G::NPF + j;
    if (slip) {
      for (int c = 0; c < DIM; ++c) {
        double pu = 0.0, pd[3] = {0.0, 0.0, 0.0};
        for (int e = 0; e < DIM; ++e) {
          const double nn = *n[c] * *n[e];
          pu += nn * u[e][m];
          for (int d = 0; d < DIM; ++d) pd[d] += nn * du[e][d][m];
        }
        jump[c][k] += 2.0 * pu;
        for (int d = 0; d < DIM; ++d) avg[c][d][k] += pd[d];
      }
    } else {
      for (int c = 0; c < DIM; ++c)
        if (*bc[c] == 0) {
          jump[c][k] += 2.0 * u[c][m];
          for (int d = 0; d < DIM; ++d) avg[c][d][k] += du[c][d][m];
        }
    }
  }
}
}  // namespace detail

template <int ORDER>
SIPG_OP2_HD void vmf_3d_mult_avg_jump(const int *u_bc_type, const int *v_bc_type, const int *w_bc_type,
                                      const int *faceNum, const double *nx, const double *ny, const double *nz,
                                      const double *u, const double *u_x, const double *u_y, const double *u_z,
                                      const double *v, const double *v_x, const double *v_y, const double *v_z,
                                      const double *w, const double *w_x, const double *w_y, const double *w_z,
                                      double *u_jump, double *u_x_avg, double *u_y_avg, double *u_z_avg,
                                      double *v_jump, double *v_x_avg, double *v_y_avg, double *v_z_avg,
                                      double *w_jump, double *w_x_avg, double *w_y_avg, double *w_z_avg) {
  const int *bc[3] = {u_bc_type, v_bc_type, w_bc_type};
  const double *n[3] = {nx, ny, nz};
  const double *uu[3] = {u, v, w};
  const double *du[3][3] = {{u_x, u_y, u_z}, {v_x, v_y, v_z}, {w_x, w_y, w_z}};
  double *jump[3] = {u_jump, v_jump, w_jump};
  double *avg[3][3] = {{u_x_avg, u_y_avg, u_z_avg}, {v_x_avg, v_y_avg, v_z_avg}, {w_x_avg, w_y_avg, w_z_avg}};
  detail::avg_jump<3, ORDER>(bc, faceNum, n, uu, du, jump, avg);
}

template <int ORDER>
SIPG_OP2_HD void vmf_2d_mult_avg_jump(const int *u_bc_type, const int *v_bc_type, const int *faceNum,
                                      const double *nx, const double *ny, const double *u, const double *u_x,
                                      const double *u_y, const double *v, const double *v_x, const double *v_y,
                                      double *u_jump, double *u_x_avg, double *u_y_avg, double *v_jump,
                                      double *v_x_avg, double *v_y_avg) {
  const int *bc[2] = {u_bc_type, v_bc_type};
  const double *n[2] = {nx, ny};
  const double *uu[2] = {u, v};
  const double *du[2][3] = {{u_x, u_y, nullptr}, {v_x, v_y, nullptr}};
  double *jump[2] = {u_jump, v_jump};
  double *avg[2][3] = {{u_x_avg, u_y_avg, nullptr}, {v_x_avg, v_y_avg, nullptr}};
  detail::avg_jump<2, ORDER>(bc, faceNum, n, uu, du, jump, avg);
}

// ---------------------------------------------------------------- apply: face fluxes (*_mult_flux)

namespace detail {
// Per face node of each face i: with h = [u]/2 and s = n . {grad u},
//   jump <- sJ (tau h - s),  avg_d <- -n_d sJ f h
// (f the nodal factor at the face node, 1 for the constant-coefficient form;
// drop_nz: the n_z term of s left out, as vmf_3d_mult_flux.h:10-11).
template <int DIM, int ORDER, int NC>
SIPG_OP2_HD void flux(const double *const *n, const double *sJ, const double *tau, const double *factor,
                      bool drop_nz, double *const *jump, double *const (*avg)[3]) {
  using G = Dg<DIM, ORDER>;
  const int *fmask = ref_tables<DIM, ORDER>().fmask;
  for (int c = 0; c < NC; ++c)
    for (int i = 0; i < G::NUM_FACES; ++i)
      for (int j = 0; j < G::NPF; ++j) {
        const int k = i * G::NPF + j;
        const double h = 0.5 * jump[c][k];
        double s = 0.0;
        for (int d = 0; d < DIM; ++d)
          if (!(drop_nz && d == 2)) s += n[d][i] * avg[c][d][k];
        const double f = factor ? factor[fmask[k]] : 1.0;
        jump[c][k] = sJ[i] * (tau[i] * h - s);
        for (int d = 0; d < DIM; ++d) avg[c][d][k] = n[d][i] * sJ[i] * f * -h;
      }
}
}  // namespace detail

template <int ORDER>
SIPG_OP2_HD void fvmf_3d_mult_flux(const double *nx, const double *ny, const double *nz, const double *sJ,
                                   const double *tau, const double *factor, double *u_jump, double *u_avg_x,
                                   double *u_avg_y, double *u_avg_z, double *v_jump, double *v_avg_x,
                                   double *v_avg_y, double *v_avg_z, double *w_jump, double *w_avg_x,
                                   double *w_avg_y, double *w_avg_z) {
  const double *n[3] = {nx, ny, nz};
  double *jump[3] = {u_jump, v_jump, w_jump};
  double *avg[3][3] = {{u_avg_x, u_avg_y, u_avg_z}, {v_avg_x, v_avg_y, v_avg_z}, {w_avg_x, w_avg_y, w_avg_z}};
  detail::flux<3, ORDER, 3>(n, sJ, tau, factor, false, jump, avg);
}

template <int ORDER>
SIPG_OP2_HD void fvmf_2d_mult_flux(const double *nx, const double *ny, const double *sJ, const double *tau,
                                   const double *factor, double *u_jump, double *u_x_avg, double *u_y_avg,
                                   double *v_jump, double *v_x_avg, double *v_y_avg) {
  const double *n[2] = {nx, ny};
  double *jump[2] = {u_jump, v_jump};
  double *avg[2][3] = {{u_x_avg, u_y_avg, nullptr}, {v_x_avg, v_y_avg, nullptr}};
  detail::flux<2, ORDER, 2>(n, sJ, tau, factor, false, jump, avg);
}

template <int ORDER>
SIPG_OP2_HD void vmf_3d_mult_flux(const double *nx, const double *ny, const double *nz, const double *sJ,
                                  const double *tau, double *u_jump, double *u_x_avg, double *u_y_avg,
                                  double *u_z_avg, double *v_jump, double *v_x_avg, double *v_y_avg, double *v_z_avg,
                                  double *w_jump, double *w_x_avg, double *w_y_avg, double *w_z_avg) {
  const double *n[3] = {nx, ny, nz};
  double *jump[3] = {u_jump, v_jump, w_jump};
  double *avg[3][3] = {{u_x_avg, u_y_avg, u_z_avg}, {v_x_avg, v_y_avg, v_z_avg}, {w_x_avg, w_y_avg, w_z_avg}};
  detail::flux<3, ORDER, 3>(n, sJ, tau, nullptr, SIPG_OP2_REF_QUIRKS != 0, jump, avg);
}

template <int ORDER>
SIPG_OP2_HD void vmf_2d_mult_flux(const double *nx, const double *ny, const double *sJ, const double *tau,
                                  double *u_jump, double *u_x_avg, double *u_y_avg, double *v_jump, double *v_x_avg,
                                  double *v_y_avg) {
  const double *n[2] = {nx, ny};
  double *jump[2] = {u_jump, v_jump};
  double *avg[2][3] = {{u_x_avg, u_y_avg, nullptr}, {v_x_avg, v_y_avg, nullptr}};
  detail::flux<2, ORDER, 2>(n, sJ, tau, nullptr, false, jump, avg);
}

// ---------------------------------------------------------------- diagonal / block-diagonal mass terms

template <int DIM, int ORDER>
SIPG_OP2_HD void mm_diag(const double *factor, const double *geof, double *diag) {
  using G = Dg<DIM, ORDER>;
  const double *M = ref_tables<DIM, ORDER>().Mass;
  for (int i = 0; i < G::NP; ++i) diag[i] += factor[i] * geof[G::J] * M[i + i * G::NP];
}
template <int DIM, int ORDER>
SIPG_OP2_HD void mm_block_diag(const double *factor, const double *geof, double *op1) {
  using G = Dg<DIM, ORDER>;
  const double *M = ref_tables<DIM, ORDER>().Mass;
  for (int j = 0; j < G::NP; ++j)
    for (int i = 0; i < G::NP; ++i) op1[i + j * G::NP] += factor[i] * geof[G::J] * M[i + j * G::NP];
}

template <int ORDER>
SIPG_OP2_HD void fvmf_3d_mm_diag(const double *factor, const double *geof, double *diag) {
  mm_diag<3, ORDER>(factor, geof, diag);
}
template <int ORDER>
SIPG_OP2_HD void fvmf_2d_mm_diag(const double *factor, const double *geof, double *diag) {
  mm_diag<2, ORDER>(factor, geof, diag);
}
template <int ORDER>
SIPG_OP2_HD void fvmf_3d_mm_block_diag(const double *factor, const double *geof, double *op1) {
  mm_block_diag<3, ORDER>(factor, geof, op1);
}
template <int ORDER>
SIPG_OP2_HD void fvmf_2d_mm_block_diag(const double *factor, const double *geof, double *op1) {
  mm_block_diag<2, ORDER>(factor, geof, op1);
}


// ---------------------------------------------------------------- diagonal and block diagonal (calc_diag, calc_inv_block_diag)

namespace detail {

// n . grad in reference coordinates with its rows scaled by f (none when f is null):
// D[i + j NP] = f_i sum_r (n . g_r) D_r[i + j NP], g_r the rows of geof
template <int DIM, int ORDER>
SIPG_OP2_HD void normal_deriv(const double *n, const double *geof, const double *f, double *D) {
  using G = Dg<DIM, ORDER>;
  constexpr int NP = G::NP;
  const RefTables &t = ref_tables<DIM, ORDER>();
  double c[3];
  c[0] = n[0] * geof[G::RX] + n[1] * geof[G::RY];
  c[1] = n[0] * geof[G::SX] + n[1] * geof[G::SY];
  c[2] = 0.0;
  if (DIM == 3) {
    c[0] += n[2] * geof[G::RZ];
    c[1] += n[2] * geof[G::SZ];
    c[2] = n[0] * geof[G::TX] + n[1] * geof[G::TY] + n[2] * geof[G::TZ];
  }
  for (int j = 0; j < NP; ++j)
    for (int i = 0; i < NP; ++i) {
      const int ind = i + j * NP;
      double v = c[0] * t.Dr[ind] + c[1] * t.Ds[ind];
      if (DIM == 3) v += c[2] * t.Dt[ind];
      D[ind] = f ? v * f[i] : v;
    }
}

// (MF D + D^T MF)_ij, the consistency and symmetry terms of a face
template <int NP>
SIPG_OP2_HD double face_sym(const double *MF, const double *D, int i, int j) {
  double s = 0.0;
  for (int k = 0; k < NP; ++k) s += MF[i + k * NP] * D[k + j * NP] + D[k + i * NP] * MF[k + j * NP];
  return s;
}

// interior-face penalty from the two sides' nodal factors at the matched face nodes
template <int DIM, int ORDER>
SIPG_OP2_HD double pair_gtau(const int *fmaskL, const int *fmaskR, const double *fscale, const double *const *factor) {
  using G = Dg<DIM, ORDER>;
  double g = 0.0;
  for (int j = 0; j < G::NPF; ++j)
    g = dmax(g, G::TAU_ORDER * dmax(fscale[0] * factor[0][fmaskL[j]], fscale[1] * factor[1][fmaskR[j]]));
  return g;
}

// boundary-face penalty: max over the face nodes of 2 (p + 1) (p + 2) fscale f
template <int DIM, int ORDER>
SIPG_OP2_HD double bface_gtau(const int *fmaskB, double fscale, const double *factor) {
  using G = Dg<DIM, ORDER>;
  double g = 0.0;
  for (int j = 0; j < G::NPF; ++j) g = dmax(g, G::TAU_ORDER * fscale * factor[fmaskB[j]]);
  return g;
}

// Volume block J sum_d D_d^T M F D_d (F the nodal factor), or the reference's
// forms: 3D sum_d D_d (J M F D_d); 2D J sum_d D_d^T F (M D_d).
template <int DIM, int ORDER>
SIPG_OP2_HD void volume_block(const double *geof, const double *factor, double *op1) {
  using G = Dg<DIM, ORDER>;
  constexpr int NP = G::NP;
  const RefTables &t = ref_tables<DIM, ORDER>();
  const double J = geof[G::J];
  double D[NP * NP], T[NP * NP];
  const bool ref2d = SIPG_OP2_REF_QUIRKS && DIM == 2, ref3d = SIPG_OP2_REF_QUIRKS && DIM == 3;
  if (ref2d) {
    // D: x derivative, T = M D; Dy: y derivative, Ty = M Dy
    double Dy[NP * NP], Ty[NP * NP];
    for (int j = 0; j < NP; ++j)
      for (int i = 0; i < NP; ++i) {
        D[i + j * NP] = dphys<DIM, ORDER>(t, geof, 0, i + j * NP);
        Dy[i + j * NP] = dphys<DIM, ORDER>(t, geof, 1, i + j * NP);
      }
    for (int j = 0; j < NP; ++j)
      for (int i = 0; i < NP; ++i) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < NP; ++k) {
          a += t.Mass[i + k * NP] * D[k + j * NP];
          b += t.Mass[i + k * NP] * Dy[k + j * NP];
        }
        T[i + j * NP] = a;
        Ty[i + j * NP] = b;
      }
    for (int j = 0; j < NP; ++j)
      for (int i = 0; i < NP; ++i) {
        double s = 0.0;
        for (int k = 0; k < NP; ++k)
          s += factor[k] * (D[k + i * NP] * T[k + j * NP] + Dy[k + i * NP] * Ty[k + j * NP]);
        op1[i + j * NP] = s * J;
      }
    return;
  }
  for (int d = 0; d < DIM; ++d) {
    for (int j = 0; j < NP; ++j)
      for (int i = 0; i < NP; ++i) D[i + j * NP] = dphys<DIM, ORDER>(t, geof, d, i + j * NP);
    for (int j = 0; j < NP; ++j)
      for (int i = 0; i < NP; ++i) {
        double s = 0.0;
        for (int k = 0; k < NP; ++k) s += t.Mass[i + k * NP] * (D[k + j * NP] * factor[k]);
        T[i + j * NP] = J * s;
      }
    for (int j = 0; j < NP; ++j)
      for (int i = 0; i < NP; ++i) {
        double s = 0.0;
        for (int k = 0; k < NP; ++k) s += (ref3d ? D[i + k * NP] : D[k + i * NP]) * T[k + j * NP];
        op1[i + j * NP] = (d == 0 ? 0.0 : op1[i + j * NP]) + s;
      }
  }
}

// Its diagonal, J sum_d (D_d^T M F D_d)_ii.
template <int DIM, int ORDER>
SIPG_OP2_HD void volume_diag(const double *geof, const double *factor, double *diag) {
  using G = Dg<DIM, ORDER>;
  constexpr int NP = G::NP;
  const RefTables &t = ref_tables<DIM, ORDER>();
  double D[NP * NP], T[NP * NP];
  for (int i = 0; i < NP; ++i) diag[i] = 0.0;
  for (int d = 0; d < DIM; ++d) {
    for (int j = 0; j < NP; ++j)
      for (int i = 0; i < NP; ++i) D[i + j * NP] = dphys<DIM, ORDER>(t, geof, d, i + j * NP) * factor[i];
    for (int j = 0; j < NP; ++j)
      for (int i = 0; i < NP; ++i) {
        double s = 0.0;
        for (int k = 0; k < NP; ++k) s += t.Mass[i + k * NP] * D[k + j * NP];
        T[i + j * NP] = s;
      }
    for (int i = 0; i < NP; ++i)
      for (int k = 0; k < NP; ++k) diag[i] += dphys<DIM, ORDER>(t, geof, d, k + i * NP) * T[k + i * NP];
  }
  for (int i = 0; i < NP; ++i) diag[i] *= geof[G::J];
}

// Interior face (fvmf_*_op2_diag / _block_diag): for each side s,
//   block_s += sJ_s / 2 (gtau MF_s - (MF_s D_s + D_s^T MF_s)), D_s = n_s . grad with rows f_s
template <int DIM, int ORDER>
SIPG_OP2_HD void face_pair(const int *faceNum, const int *fmaskR, const double *const *n, const double *fscale,
                           const double *sJ, const double *const *geof, const double *const *factor, double *outL,
                           double *outR, bool block) {
  using G = Dg<DIM, ORDER>;
  constexpr int NP = G::NP;
  const RefTables &t = ref_tables<DIM, ORDER>();
  const double gtau = pair_gtau<DIM, ORDER>(t.fmask + faceNum[0] * G::NPF, fmaskR, fscale, factor);
  double D[NP * NP];
  for (int s = 0; s < 2; ++s) {
    double ns[3] = {n[0][s], n[1][s], DIM == 3 ? n[2][s] : 0.0};
    normal_deriv<DIM, ORDER>(ns, geof[s], factor[s], D);
    const double *MF = t.MM_F[faceNum[s]];
    double *out = s == 0 ? outL : outR;
    if (block) {
      for (int j = 0; j < NP; ++j)
        for (int i = 0; i < NP; ++i) {
          double a = 0.0;
          for (int k = 0; k < NP; ++k) a += MF[i + k * NP] * D[k + j * NP];
          out[i + j * NP] = out[i + j * NP] + (-0.5 * sJ[s]) * a;
        }
      for (int j = 0; j < NP; ++j)
        for (int i = 0; i < NP; ++i) {
          double a = 0.0;
          for (int k = 0; k < NP; ++k) a += D[k + i * NP] * MF[k + j * NP];
          out[i + j * NP] = out[i + j * NP] + (-0.5 * sJ[s]) * a;
        }
      const double c = 0.5 * sJ[s] * gtau;
      for (int j = 0; j < NP; ++j)
        for (int i = 0; i < NP; ++i) out[i + j * NP] += c * MF[i + j * NP];
    } else {
      for (int i = 0; i < NP; ++i)
        out[i] += 0.5 * sJ[s] * (gtau * MF[i + i * NP] - face_sym<NP>(MF, D, i, i));
    }
  }
}

// Boundary face (fvmf_*_bop_diag / _block_diag): Dirichlet components add
// sJ (gtau MF - (MF D + D^T MF)), Neumann ones nothing; when every component is
// slip, each adds sJ n_c^2 (gtau MF - (MF D + D^T MF)).
template <int DIM, int ORDER>
SIPG_OP2_HD void face_bnd(const int *faceNum, const int *const *bc, const double *const *n, const double *fscale,
                          const double *sJ, const double *geof, const double *factor, double *const *out,
                          bool block) {
  using G = Dg<DIM, ORDER>;
  constexpr int NP = G::NP;
  const RefTables &t = ref_tables<DIM, ORDER>();
  bool slip = true, any = false;
  for (int c = 0; c < DIM; ++c) {
    slip = slip && *bc[c] == 2;
    any = any || *bc[c] == 0;
  }
  if (!slip && !any) return;
  double D[NP * NP];
  const double ns[3] = {*n[0], *n[1], DIM == 3 ? *n[2] : 0.0};
  normal_deriv<DIM, ORDER>(ns, geof, factor, D);
  const double gtau = bface_gtau<DIM, ORDER>(t.fmask + faceNum[0] * G::NPF, *fscale, factor);
  const double *MF = t.MM_F[faceNum[0]];
  for (int c = 0; c < DIM; ++c) {
    if (!slip && *bc[c] != 0) continue;
    const double w = slip ? *sJ * ns[c] * ns[c] : *sJ;
    if (block) {
      for (int j = 0; j < NP; ++j)
        for (int i = 0; i < NP; ++i)
          out[c][i + j * NP] += w * (gtau * MF[i + j * NP] - face_sym<NP>(MF, D, i, j));
    } else {
      for (int i = 0; i < NP; ++i) out[c][i] += w * (gtau * MF[i + i * NP] - face_sym<NP>(MF, D, i, i));
    }
  }
}

// Boundary lifting of one boundary face (fvmf_*_apply_bc with the nodal factor,
// vmf_*_apply_bc without): Dirichlet data g adds gtau sJ MF g - D^T (sJ MF g),
// Neumann data adds sJ MF g, slip nothing.
template <int DIM, int ORDER>
SIPG_OP2_HD void lift_bc(const int *faceNum, const int *const *bc, const double *const *n, const double *fscale,
                         const double *sJ, const double *geof, const double *fact, const double *const *g,
                         double *const *rhs) {
  using G = Dg<DIM, ORDER>;
  constexpr int NP = G::NP;
  const RefTables &t = ref_tables<DIM, ORDER>();
  const int *fm = t.fmask + faceNum[0] * G::NPF;
  const double *MF = t.MM_F[faceNum[0]];
  for (int c = 0; c < DIM; ++c) {
    if (*bc[c] == 1) {
      for (int i = 0; i < NP; ++i)
        for (int j = 0; j < G::NPF; ++j) rhs[c][i] += *sJ * MF[i + fm[j] * NP] * g[c][j];
      continue;
    }
    if (*bc[c] != 0) continue;
    double D[NP * NP], tmp[NP];
    for (int j = 0; j < NP; ++j)
      for (int i = 0; i < NP; ++i) {
        const int ind = i + j * NP;
        double v = 0.0;
        for (int d = 0; d < DIM; ++d) v += *n[d] * dphys<DIM, ORDER>(t, geof, d, ind);
        D[ind] = fact ? v * fact[i] : v;
      }
    double gtau = G::TAU_ORDER * *fscale;
    if (fact) {
      double m = fact[fm[0]];
      for (int j = 1; j < G::NPF; ++j) m = dmax(m, fact[fm[j]]);
      gtau = m * gtau;
    }
    for (int i = 0; i < NP; ++i) {
      tmp[i] = 0.0;
      for (int j = 0; j < G::NPF; ++j) {
        rhs[c][i] += gtau * *sJ * MF[i + fm[j] * NP] * g[c][j];
        tmp[i] += *sJ * MF[i + fm[j] * NP] * g[c][j];
      }
    }
    for (int i = 0; i < NP; ++i)
      for (int j = 0; j < NP; ++j) rhs[c][i] += -D[j + i * NP] * tmp[j];
  }
}

}  // namespace detail

template <int ORDER>
SIPG_OP2_HD void fvmf_3d_op1(const double *geof, const double *factor, double *op1) {
  detail::volume_block<3, ORDER>(geof, factor, op1);
}
template <int ORDER>
SIPG_OP2_HD void fvmf_2d_op1(const double *geof, const double *factor, double *op1) {
  detail::volume_block<2, ORDER>(geof, factor, op1);
}
template <int ORDER>
SIPG_OP2_HD void fvmf_3d_op1_diag(const double *geof, const double *factor, double *diag) {
  detail::volume_diag<3, ORDER>(geof, factor, diag);
}
template <int ORDER>
SIPG_OP2_HD void fvmf_2d_op1_diag(const double *geof, const double *factor, double *diag) {
  detail::volume_diag<2, ORDER>(geof, factor, diag);
}

template <int ORDER>
SIPG_OP2_HD void fvmf_3d_op2_diag(const int *faceNum, const int *fmaskL_corrected, const int *fmaskR_corrected,
                                  const double *nx, const double *ny, const double *nz, const double *fscale,
                                  const double *sJ, const double **geof, const double **factor, double *diagL,
                                  double *diagR) {
  (void)fmaskL_corrected;  // the reference takes the left side's nodes from FMASK
  const double *n[3] = {nx, ny, nz};
  detail::face_pair<3, ORDER>(faceNum, fmaskR_corrected, n, fscale, sJ, geof, factor, diagL, diagR, false);
}
template <int ORDER>
SIPG_OP2_HD void fvmf_3d_op2_block_diag(const int *faceNum, const int *fmaskL_corrected, const int *fmaskR_corrected,
                                        const double *nx, const double *ny, const double *nz, const double *fscale,
                                        const double *sJ, const double **geof, const double **factor, double *op1L,
                                        double *op1R) {
  (void)fmaskL_corrected;
  const double *n[3] = {nx, ny, nz};
  detail::face_pair<3, ORDER>(faceNum, fmaskR_corrected, n, fscale, sJ, geof, factor, op1L, op1R, true);
}

namespace detail {
// 2D: the right side's nodes are its face's nodes, reversed when *reverse
template <int ORDER>
SIPG_OP2_HD void fmask_2d_right(const int *faceNum, const bool *reverse, int *fmaskR) {
  using G = Dg<2, ORDER>;
  const int *fR = ref_tables<2, ORDER>().fmask + faceNum[1] * G::NPF;
  for (int j = 0; j < G::NPF; ++j) fmaskR[j] = fR[*reverse ? G::NPF - 1 - j : j];
}
}  // namespace detail

template <int ORDER>
SIPG_OP2_HD void fvmf_2d_op2_diag(const int *faceNum, const bool *reverse, const double *nx, const double *ny,
                                  const double *fscale, const double *sJ, const double **geof, const double **factor,
                                  double *diagL, double *diagR) {
  int fmaskR[Dg<2, ORDER>::NPF];
  detail::fmask_2d_right<ORDER>(faceNum, reverse, fmaskR);
  const double *n[3] = {nx, ny, nullptr};
  detail::face_pair<2, ORDER>(faceNum, fmaskR, n, fscale, sJ, geof, factor, diagL, diagR, false);
}
template <int ORDER>
SIPG_OP2_HD void fvmf_2d_op2_block_diag(const int *faceNum, const bool *reverse, const double *nx, const double *ny,
                                        const double *fscale, const double *sJ, const double **geof,
                                        const double **factor, double *op1L, double *op1R) {
  int fmaskR[Dg<2, ORDER>::NPF];
  detail::fmask_2d_right<ORDER>(faceNum, reverse, fmaskR);
  const double *n[3] = {nx, ny, nullptr};
  detail::face_pair<2, ORDER>(faceNum, fmaskR, n, fscale, sJ, geof, factor, op1L, op1R, true);
}

template <int ORDER>
SIPG_OP2_HD void fvmf_3d_bop_diag(const int *faceNum, const int *u_bc_type, const int *v_bc_type,
                                  const int *w_bc_type, const double *nx, const double *ny, const double *nz,
                                  const double *fscale, const double *sJ, const double *geof, const double *factor,
                                  double *u_diag, double *v_diag, double *w_diag) {
  const int *bc[3] = {u_bc_type, v_bc_type, w_bc_type};
  const double *n[3] = {nx, ny, nz};
  double *out[3] = {u_diag, v_diag, w_diag};
  detail::face_bnd<3, ORDER>(faceNum, bc, n, fscale, sJ, geof, factor, out, false);
}
template <int ORDER>
SIPG_OP2_HD void fvmf_3d_bop_block_diag(const int *faceNum, const int *u_bc_type, const int *v_bc_type,
                                        const int *w_bc_type, const double *nx, const double *ny, const double *nz,
                                        const double *fscale, const double *sJ, const double *geof,
                                        const double *factor, double *u_op1, double *v_op1, double *w_op1) {
  const int *bc[3] = {u_bc_type, v_bc_type, w_bc_type};
  const double *n[3] = {nx, ny, nz};
  double *out[3] = {u_op1, v_op1, w_op1};
  detail::face_bnd<3, ORDER>(faceNum, bc, n, fscale, sJ, geof, factor, out, true);
}
template <int ORDER>
SIPG_OP2_HD void fvmf_2d_bop_diag(const int *faceNum, const int *u_bc_type, const int *v_bc_type, const double *nx,
                                  const double *ny, const double *fscale, const double *sJ, const double *geof,
                                  const double *factor, double *u_diag, double *v_diag) {
  const int *bc[2] = {u_bc_type, v_bc_type};
  const double *n[2] = {nx, ny};
  double *out[2] = {u_diag, v_diag};
  detail::face_bnd<2, ORDER>(faceNum, bc, n, fscale, sJ, geof, factor, out, false);
}
template <int ORDER>
SIPG_OP2_HD void fvmf_2d_bop_block_diag(const int *faceNum, const int *u_bc_type, const int *v_bc_type,
                                        const double *nx, const double *ny, const double *fscale, const double *sJ,
                                        const double *geof, const double *factor, double *u_op1, double *v_op1) {
  const int *bc[2] = {u_bc_type, v_bc_type};
  const double *n[2] = {nx, ny};
  double *out[2] = {u_op1, v_op1};
  detail::face_bnd<2, ORDER>(faceNum, bc, n, fscale, sJ, geof, factor, out, true);
}

// ---------------------------------------------------------------- boundary lifting of the right-hand side (apply_bc)

template <int ORDER>
SIPG_OP2_HD void fvmf_3d_apply_bc(const int *faceNum, const int *u_bc_type, const int *v_bc_type,
                                  const int *w_bc_type, const double *nx, const double *ny, const double *nz,
                                  const double *fscale, const double *sJ, const double *geof, const double *fact,
                                  const double *u_bc, const double *v_bc, const double *w_bc, double *u_rhs,
                                  double *v_rhs, double *w_rhs) {
  const int *bc[3] = {u_bc_type, v_bc_type, w_bc_type};
  const double *n[3] = {nx, ny, nz};
  const double *g[3] = {u_bc, v_bc, w_bc};
  double *rhs[3] = {u_rhs, v_rhs, w_rhs};
  detail::lift_bc<3, ORDER>(faceNum, bc, n, fscale, sJ, geof, fact, g, rhs);
}
template <int ORDER>
SIPG_OP2_HD void vmf_3d_apply_bc(const int *faceNum, const int *u_bc_type, const int *v_bc_type, const int *w_bc_type,
                                 const double *nx, const double *ny, const double *nz, const double *fscale,
                                 const double *sJ, const double *geof, const double *u_bc, const double *v_bc,
                                 const double *w_bc, double *u_rhs, double *v_rhs, double *w_rhs) {
  const int *bc[3] = {u_bc_type, v_bc_type, w_bc_type};
  const double *n[3] = {nx, ny, nz};
  const double *g[3] = {u_bc, v_bc, w_bc};
  double *rhs[3] = {u_rhs, v_rhs, w_rhs};
  detail::lift_bc<3, ORDER>(faceNum, bc, n, fscale, sJ, geof, nullptr, g, rhs);
}
template <int ORDER>
SIPG_OP2_HD void fvmf_2d_apply_bc(const int *faceNum, const int *u_bc_type, const int *v_bc_type, const double *nx,
                                  const double *ny, const double *fscale, const double *sJ, const double *geof,
                                  const double *factor, const double *u_bc, const double *v_bc, double *u_rhs,
                                  double *v_rhs) {
  const int *bc[2] = {u_bc_type, v_bc_type};
  const double *n[2] = {nx, ny};
  const double *g[2] = {u_bc, v_bc};
  double *rhs[2] = {u_rhs, v_rhs};
  detail::lift_bc<2, ORDER>(faceNum, bc, n, fscale, sJ, geof, factor, g, rhs);
}
template <int ORDER>
SIPG_OP2_HD void vmf_2d_apply_bc(const int *faceNum, const int *u_bc_type, const int *v_bc_type, const double *nx,
                                 const double *ny, const double *fscale, const double *sJ, const double *geof,
                                 const double *u_bc, const double *v_bc, double *u_rhs, double *v_rhs) {
  const int *bc[2] = {u_bc_type, v_bc_type};
  const double *n[2] = {nx, ny};
  const double *g[2] = {u_bc, v_bc};
  double *rhs[2] = {u_rhs, v_rhs};
  detail::lift_bc<2, ORDER>(faceNum, bc, n, fscale, sJ, geof, nullptr, g, rhs);
}

// ---- velocity projection, div_div = 1: INSSolverBase3D::project_velocity
// (src/solvers/3d/ins_solver_base.cpp:1052-1124, set-up :201-214) and
// INSSolverBase2D::project_velocity (src/solvers/2d/ins_solver_base.cpp:894-955).
// The fused performance path is sipg_project_velocity.

// face loop of the set-up: each side of an interior face writes its fscale into
// its cell's per-face slots (ins_proj_setup_0.h)
template <int DIM, int ORDER>
SIPG_OP2_HD void ins_proj_setup_0(const int *faceNum, const double *fscale, double **f0) {
  for (int side = 0; side < 2; ++side) f0[side][faceNum[side]] += fscale[side];
}

// h = 1 / the largest per-face fscale of the cell (ins_proj_setup_1.h)
template <int DIM, int ORDER>
SIPG_OP2_HD void ins_proj_setup_1(const double *fscale, double *h) {
  double m = 0.0;
  for (int f = 0; f < Dg<DIM, ORDER>::NUM_FACES; ++f) m = std::fmax(m, fscale[f]);
  *h = 1.0 / m;
}

// velTT = velT - dt grad p, copied to the projection right-hand side (ins_3d_proj_rhs.h)
template <int ORDER>
SIPG_OP2_HD void ins_3d_proj_rhs(const double *dt, const double *dpdx, const double *dpdy, const double *dpdz,
                                 const double *uT, const double *vT, const double *wT, double *uTT, double *vTT,
                                 double *wTT, double *proj0, double *proj1, double *proj2) {
  for (int i = 0; i < Dg<3, ORDER>::NP; ++i) {
    proj0[i] = uTT[i] = uT[i] - *dt * dpdx[i];
    proj1[i] = vTT[i] = vT[i] - *dt * dpdy[i];
    proj2[i] = wTT[i] = wT[i] - *dt * dpdz[i];
  }
}

template <int ORDER>
SIPG_OP2_HD void ins_2d_proj_rhs(const double *dt, const double *dpdx, const double *dpdy, const double *uT,
                                 const double *vT, double *uTT, double *vTT, double *proj0, double *proj1) {
  for (int i = 0; i < Dg<2, ORDER>::NP; ++i) {
    proj0[i] = uTT[i] = uT[i] - *dt * dpdx[i];
    proj1[i] = vTT[i] = vT[i] - *dt * dpdy[i];
  }
}

// penalty of the element solve: pen = factor h / (p + 1), pen_f = factor. The
// reference also forms the mass-weighted velocity magnitude from (a0 u0 + a1 u1,
// ...), which does not enter either output (ins_3d_proj_pen.h:24-25).
template <int ORDER>
SIPG_OP2_HD void ins_3d_proj_pen(const double *factor, const double *a0, const double *a1, const double *geof,
                                 const double *u0, const double *v0, const double *w0, const double *u1,
                                 const double *v1, const double *w1, const double *h, double *pen, double *pen_f) {
  (void)a0, (void)a1, (void)geof, (void)u0, (void)v0, (void)w0, (void)u1, (void)v1, (void)w1;
  *pen = *factor * (*h / ((double)ORDER + 1.0));
  *pen_f = *factor;
}

template <int ORDER>
SIPG_OP2_HD void ins_2d_proj_pen(const double *factor, const double *a0, const double *a1, const double *geof,
                                 const double *u0, const double *v0, const double *u1, const double *v1,
                                 const double *h, double *pen, double *pen_f) {
  (void)a0, (void)a1, (void)geof, (void)u0, (void)v0, (void)u1, (void)v1;
  *pen = *factor * (*h / ((double)ORDER + 1.0));
  *pen_f = *factor;
}

namespace detail {

// out_c = pen * (G^T D^T (J M (D G v)))_c + J (M v_c), with every product summed
// over j in order and the sums combined as op2_in_kernel_gemv combines them.
template <int DIM, int ORDER>
SIPG_OP2_HD void proj_operator(const double *geof, double pen, double *const *v, double *const *out) {
  using G = Dg<DIM, ORDER>;
  constexpr int NP = G::NP;
  const RefTables &t = ref_tables<DIM, ORDER>();
  const double *Dk[3] = {t.Dr, t.Ds, t.Dt};
  const int gi[3][3] = {{G::RX, G::RY, G::RZ}, {G::SX, G::SY, G::SZ}, {G::TX, G::TY, G::TZ}};
  const double J = geof[G::J];
  double gv[3][NP], div[NP], mdiv[NP];
  for (int i = 0; i < NP; ++i)
    for (int k = 0; k < DIM; ++k) {
      double s = geof[gi[k][0]] * v[0][i] + geof[gi[k][1]] * v[1][i];
      if (DIM == 3) s += geof[gi[k][2]] * v[2][i];
      gv[k][i] = s;
    }
  for (int k = 0; k < DIM; ++k)
    for (int i = 0; i < NP; ++i) {
      double s = 0.0;
      for (int j = 0; j < NP; ++j) s += Dk[k][i + j * NP] * gv[k][j];
      div[i] = k == 0 ? s : div[i] + s;
    }
  for (int i = 0; i < NP; ++i) {
    double s = 0.0;
    for (int j = 0; j < NP; ++j) s += t.Mass[i + j * NP] * div[j];
    mdiv[i] = J * s;
  }
  for (int k = 0; k < DIM; ++k)
    for (int i = 0; i < NP; ++i) {
      double s = 0.0;
      for (int j = 0; j < NP; ++j) s += Dk[k][j + i * NP] * mdiv[j];
      gv[k][i] = s;
    }
  for (int i = 0; i < NP; ++i)
    for (int c = 0; c < DIM; ++c) {
      double s = geof[gi[0][c]] * gv[0][i] + geof[gi[1][c]] * gv[1][i];
      if (DIM == 3) s += geof[gi[2][c]] * gv[2][i];
      out[c][i] = s;
    }
  for (int c = 0; c < DIM; ++c)
    for (int i = 0; i < NP; ++i) {
      double s = 0.0;
      for (int j = 0; j < NP; ++j) s += t.Mass[i + j * NP] * v[c][j];
      out[c][i] = pen * out[c][i] + J * s;
    }
}

// sum over the nodes of a[0] b[0] + a[1] b[1] (+ a[2] b[2])
template <int DIM, int NP>
SIPG_OP2_HD double proj_dot(double *const *a, double *const *b) {
  double s = 0.0;
  for (int i = 0; i < NP; ++i) {
    double t = a[0][i] * b[0][i] + a[1][i] * b[1][i];
    if (DIM == 3) t += a[2][i] * b[2][i];
    s += t;
  }
  return s;
}

// Element-local CG of the projection: 3D preconditioned by (1/J) M^-1 and
// stopped at |r|_2 < 1e-8 (ins_3d_proj_cg_precon.h), 2D unpreconditioned and
// stopped at |r|_2^2 < 1e-16 (ins_proj_cg_2d.h); at most 100 iterations. The
// iteration that meets the tolerance is not counted, as in the reference.
template <int DIM, int ORDER>
SIPG_OP2_HD void proj_cg(const double *geof, const double *pen, const double *const *rhs, double *const *x,
                         int *cell_g, int *conv_g, double *iter_g) {
  using G = Dg<DIM, ORDER>;
  constexpr int NP = G::NP;
  constexpr bool pre = DIM == 3;
  const double tol = pre ? 1e-8 : 1e-16;
  const double inv_J = 1.0 / geof[G::J];
  const double *Mi = ref_tables<DIM, ORDER>().InvMass;
  double rb[3][NP], zb[3][NP], pb[3][NP], ab[3][NP];
  double *r[3] = {rb[0], rb[1], rb[2]}, *z[3] = {zb[0], zb[1], zb[2]};
  double *p[3] = {pb[0], pb[1], pb[2]}, *ap[3] = {ab[0], ab[1], ab[2]};
  auto precondition = [&]() {
    for (int c = 0; c < DIM; ++c)
      for (int i = 0; i < NP; ++i) {
        if (pre) {
          double s = 0.0;
          for (int j = 0; j < NP; ++j) s += Mi[i + j * NP] * r[c][j];
          z[c][i] = inv_J * s;
        } else {
          z[c][i] = r[c][i];
        }
      }
  };
  proj_operator<DIM, ORDER>(geof, *pen, x, ap);
  for (int c = 0; c < DIM; ++c)
    for (int i = 0; i < NP; ++i) r[c][i] = rhs[c][i] - ap[c][i];
  double res = proj_dot<DIM, NP>(r, r);
  if (pre) res = std::sqrt(res);
  precondition();
  for (int c = 0; c < DIM; ++c)
    for (int i = 0; i < NP; ++i) p[c][i] = z[c][i];
  double it = 0.0;
  while (res > tol && it < 100.0) {
    proj_operator<DIM, ORDER>(geof, *pen, p, ap);
    const double alpha = proj_dot<DIM, NP>(r, z) / proj_dot<DIM, NP>(p, ap);
    // r_old . z_old (3D) or r_old . r_old (2D) for beta, taken before r moves
    const double rz_old = pre ? proj_dot<DIM, NP>(r, z) : proj_dot<DIM, NP>(r, r);
    for (int c = 0; c < DIM; ++c)
      for (int i = 0; i < NP; ++i) x[c][i] = x[c][i] + alpha * p[c][i];
    for (int c = 0; c < DIM; ++c)
      for (int i = 0; i < NP; ++i) r[c][i] = r[c][i] - alpha * ap[c][i];
    res = proj_dot<DIM, NP>(r, r);
    if (pre) res = std::sqrt(res);
    if (res < tol) break;
    precondition();
    const double beta = (pre ? proj_dot<DIM, NP>(r, z) : proj_dot<DIM, NP>(r, r)) / rz_old;
    for (int c = 0; c < DIM; ++c)
      for (int i = 0; i < NP; ++i) p[c][i] = z[c][i] + beta * p[c][i];
    it += 1.0;
  }
  *cell_g += 1;
  *iter_g += it;
  if (it < 100.0 && !std::isnan(res)) *conv_g += 1;
}

}  // namespace detail

template <int ORDER>
SIPG_OP2_HD void ins_3d_proj_cg_precon(const double *geof, const double *pen, const double *rhs0,
                                       const double *rhs1, const double *rhs2, double *u, double *v, double *w,
                                       int *cell_g, int *conv_g, double *iter_g) {
  const double *rhs[3] = {rhs0, rhs1, rhs2};
  double *x[3] = {u, v, w};
  detail::proj_cg<3, ORDER>(geof, pen, rhs, x, cell_g, conv_g, iter_g);
}

template <int ORDER>
SIPG_OP2_HD void ins_proj_cg_2d(const double *geof, const double *pen, const double *rhs0, const double *rhs1,
                                double *u, double *v, int *cell_g, int *conv_g, double *iter_g) {
  const double *rhs[3] = {rhs0, rhs1, rhs1};
  double *x[3] = {u, v, v};
  detail::proj_cg<2, ORDER>(geof, pen, rhs, x, cell_g, conv_g, iter_g);
}

// ---- pressure step around the solve (src/solvers/3d/ins_solver.cpp:313-322,
// mp_ins_solver.cpp:581-612, :546-552, :676-692; 2D src/solvers/2d/ins_solver.cpp:309-319).
// The fused performance path is sipg_pressure_rhs / sipg_pressure_projection.

// divVelT <- -divVelT / dt; dPdN_old <- b0 dPdN + b1 dPdN_old (ins_3d_pr_1.h)
template <int ORDER>
SIPG_OP2_HD void ins_3d_pr_1(const double *b0, const double *b1, const double *dt, const double *dPdN,
                             double *dPdN_old, double *divVelT) {
  using G = Dg<3, ORDER>;
  const double inv_dt = 1.0 / *dt;
  for (int i = 0; i < G::NP; ++i) divVelT[i] = -divVelT[i] * inv_dt;
  for (int i = 0; i < G::NUM_FACES * G::NPF; ++i) dPdN_old[i] = (*b0) * dPdN[i] + (*b1) * dPdN_old[i];
}

// the 2D twin (ins_pressure_rhs_2d.h)
template <int ORDER>
SIPG_OP2_HD void ins_pressure_rhs_2d(const double *b0, const double *b1, const double *dt, const double *dPdN,
                                     double *dPdNOld, double *divVelT) {
  using G = Dg<2, ORDER>;
  const double inv_dt = 1.0 / *dt;
  for (int i = 0; i < G::NP; ++i) divVelT[i] = -divVelT[i] * inv_dt;
  for (int i = 0; i < G::NUM_FACES * G::NPF; ++i) dPdNOld[i] = (*b0) * dPdN[i] + (*b1) * dPdNOld[i];
}

// dPdNOld <- b0 dPdN + b1 dPdNOld (mp_ins_pr_bc_dpdn_factors.h)
template <int DIM, int ORDER>
SIPG_OP2_HD void mp_ins_pr_bc_dpdn_factors(const double *b0, const double *b1, const double *dPdN,
                                           double *dPdNOld) {
  using G = Dg<DIM, ORDER>;
  for (int i = 0; i < G::NUM_FACES * G::NPF; ++i) dPdNOld[i] = (*b0) * dPdN[i] + (*b1) * dPdNOld[i];
}

// div <- div * factor (mp_ins_pr_div_factor.h; the caller passes -1 / dt)
template <int DIM, int ORDER>
SIPG_OP2_HD void mp_ins_pr_div_factor(const double *_div_factor, double *div) {
  const double f = *_div_factor;
  for (int i = 0; i < Dg<DIM, ORDER>::NP; ++i) div[i] *= f;
}

// grad p <- grad p / rho (mp_ins_3d_pr_2.h, update_pressure_gradient)
template <int ORDER>
SIPG_OP2_HD void mp_ins_3d_pr_2(const double *rho, double *dpdx, double *dpdy, double *dpdz) {
  for (int i = 0; i < Dg<3, ORDER>::NP; ++i) {
    dpdx[i] /= rho[i];
    dpdy[i] /= rho[i];
    dpdz[i] /= rho[i];
  }
}

// viscous right-hand side rho u Re/dt and the mass factor g0 Re/dt rho of the
// two-phase Helmholtz solve (mp_ins_3d_vis_0.h; mu and art_vis are not changed:
// the reference leaves its artificial-viscosity update commented out)
template <int ORDER>
SIPG_OP2_HD void mp_ins_3d_vis_0(const double *fact0, const double *fact1, const double *rho, double *mu,
                                 const double *art_vis, const double *u, const double *v, const double *w,
                                 double *rhs0, double *rhs1, double *rhs2, double *mm_factor) {
  (void)mu, (void)art_vis;
  for (int i = 0; i < Dg<3, ORDER>::NP; ++i) {
    rhs0[i] = u[i] * *fact0 * rho[i];
    rhs1[i] = v[i] * *fact0 * rho[i];
    rhs2[i] = w[i] * *fact0 * rho[i];
    mm_factor[i] = *fact1 * rho[i];
  }
}

}  // namespace op2
}  // namespace ins_solver_b200
