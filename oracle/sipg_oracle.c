/* CPU oracle for the SIPG solve path. TEST INFRASTRUCTURE ONLY (see header).
 *
 * Every routine cites the reference file:line it restates. The DG-Toolkit glue
 * that the reference calls but does not vendor (mesh->jump, mesh->avg,
 * mesh->mass, mesh->inv_mass, op2_gemv) is restated from its call-site meaning:
 *   jump(u)  : per element face node, u_own - u_neighbour (interior faces only)
 *   avg(q)   : per element face node, (q_own + q_neighbour) / 2 (interior faces only)
 *   mass(q)  : q <- J * M * q
 *   op2_gemv : per element y = alpha * A x + beta * y (A^T when transposed)
 */
#define _POSIX_C_SOURCE 199309L
#include "sipg_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define IDX(e, i, n) ((size_t)(e) * (n) + (i))

static double wall_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static int ngeof(const oracle_mesh *m) { return m->dim == 3 ? 10 : 5; }

/* geof accessors: 3D rx ry rz sx sy sz tx ty tz J, 2D rx ry sx sy J */
static void geo_unpack(const oracle_mesh *m, int e, double G[3][3], double *J) {
  const double *g = m->geof + (size_t)e * ngeof(m);
  memset(G, 0, sizeof(double) * 9);
  if (m->dim == 3) {
    for (int c = 0; c < 3; ++c)
      for (int d = 0; d < 3; ++d) G[c][d] = g[c * 3 + d];
    *J = g[9];
  } else {
    G[0][0] = g[0]; G[0][1] = g[1]; G[1][0] = g[2]; G[1][1] = g[3];
    *J = g[4];
  }
}

/* Position of volume node `node` among face f's nodes. */
static int face_pos(const oracle_mesh *m, int f, int node) {
  for (int k = 0; k < m->Nfp; ++k)
    if (m->fmask[f * m->Nfp + k] == node) return k;
  return -1;
}

/* ---------------------------------------------------------------- penalty */
/* fvmf_3d_calc_tau_faces.h:1-14, fvmf_3d_calc_tau_bfaces.h:1-12 (2D: fvmf_2d_calc_tau_*);
 * with factor == NULL this is vmf_calc_tau_faces.h:1-7 / vmf_calc_tau_bfaces.h:1-5. */
void oracle_tau(const oracle_mesh *m, const double *factor, double *tau) {
  const int Nfp = m->Nfp, Np = m->Np, Nf = m->Nf, p = m->order;
  const double c = 2.0 * (p + 1) * (p + 2);
  for (int fc = 0; fc < m->F; ++fc) {
    int eL = m->face2cells[2 * fc], eR = m->face2cells[2 * fc + 1];
    int fL = m->faceNum[2 * fc], fR = m->faceNum[2 * fc + 1];
    double fsL = m->fscale[IDX(eL, fL, Nf)], fsR = m->fscale[IDX(eR, fR, Nf)];
    double gtau = 0.0;
    for (int j = 0; j < Nfp; ++j) {
      double fl = factor ? factor[IDX(eL, m->fmaskL[fc * Nfp + j], Np)] : 1.0;
      double fr = factor ? factor[IDX(eR, m->fmaskR[fc * Nfp + j], Np)] : 1.0;
      gtau = fmax(gtau, c * fmax(fsL * fl, fsR * fr));
    }
    tau[IDX(eL, fL, Nf)] = gtau;
    tau[IDX(eR, fR, Nf)] = gtau;
  }
  for (int b = 0; b < m->Kb; ++b) {
    int e = m->bface2cell[b], f = m->bfaceNum[b];
    double g = factor ? factor[IDX(e, m->fmask[f * Nfp], Np)] : 1.0;
    for (int j = 1; j < Nfp; ++j)
      if (factor) g = fmax(g, factor[IDX(e, m->fmask[f * Nfp + j], Np)]);
    tau[IDX(e, f, Nf)] = g * c * m->fscale[IDX(e, f, Nf)];
  }
}

/* ------------------------------------------------------------------- mult */
/* Restates FactorViscousMatrix3D::mult, factor_viscous_matrix.cpp:96-310
 * (2D: src/solvers/2d/slip_matrix/factor_viscous_matrix.cpp:87-200). */
void oracle_mult(const oracle_mesh *m, int ncomp, const int *bc_types, const double *factor,
                 const double *mm_factor, double mm_scalar, int flags, const double *const *x,
                 double *const *y) {
  const int Np = m->Np, Nfp = m->Nfp, Nf = m->Nf, K = m->K, dim = m->dim;
  const int NF = Nf * Nfp;
  double *tau = (double *)malloc(sizeof(double) * K * Nf);
  oracle_tau(m, factor, tau); /* mat_free_pre_compute_tau, :78-94 */
  const double *Dm[3] = {m->Dr, m->Ds, m->Dt};
  /* q[c][d]: K x Np gradient work arrays (u_x.. w_z), jump[c], avg[c][d]: K x NF */
  double *q[3][3], *jump[3], *avg[3][3];
  for (int c = 0; c < ncomp; ++c) {
    jump[c] = (double *)calloc((size_t)K * NF, sizeof(double));
    for (int d = 0; d < dim; ++d) {
      q[c][d] = (double *)calloc((size_t)K * Np, sizeof(double));
      avg[c][d] = (double *)calloc((size_t)K * NF, sizeof(double)); /* zero_npf_3, :145-163 */
    }
  }
  for (int c = 0; c < ncomp; ++c) {
    /* op2_gemv_halo_exchange(DR/DS/DT), :109-117 */
#pragma omp parallel for schedule(static)
    for (int e = 0; e < K; ++e)
      for (int d = 0; d < dim; ++d)
        for (int i = 0; i < Np; ++i) {
          double s = 0.0;
          for (int j = 0; j < Np; ++j) s += Dm[d][i * Np + j] * x[c][IDX(e, j, Np)];
          q[c][d][IDX(e, i, Np)] = s;
        }
    /* fvmf_3d_grad, :119-130 (fvmf_3d_grad.h:13-33) */
#pragma omp parallel for schedule(static)
    for (int e = 0; e < K; ++e) {
      double G[3][3], J;
      geo_unpack(m, e, G, &J);
      for (int i = 0; i < Np; ++i) {
        double ur[3] = {0, 0, 0};
        for (int d = 0; d < dim; ++d) ur[d] = q[c][d][IDX(e, i, Np)];
        double f = factor ? factor[IDX(e, i, Np)] : 1.0;
        for (int d = 0; d < dim; ++d) {
          double s = 0.0;
          for (int r = 0; r < dim; ++r) s += G[r][d] * ur[r];
          q[c][d][IDX(e, i, Np)] = f * s;
        }
      }
    }
  }
  /* mesh->jump / mesh->avg over interior faces, :165-176 (every element face
   * belongs to one face: the loop writes disjoint slots) */
#pragma omp parallel for schedule(static)
  for (int fc = 0; fc < m->F; ++fc) {
    int eL = m->face2cells[2 * fc], eR = m->face2cells[2 * fc + 1];
    int fL = m->faceNum[2 * fc], fR = m->faceNum[2 * fc + 1];
    for (int j = 0; j < Nfp; ++j) {
      int nL = m->fmaskL[fc * Nfp + j], nR = m->fmaskR[fc * Nfp + j];
      int kL = face_pos(m, fL, nL), kR = face_pos(m, fR, nR);
      for (int c = 0; c < ncomp; ++c) {
        double uL = x[c][IDX(eL, nL, Np)], uR = x[c][IDX(eR, nR, Np)];
        jump[c][IDX(eL, fL * Nfp + kL, NF)] += uL - uR;
        jump[c][IDX(eR, fR * Nfp + kR, NF)] += uR - uL;
        for (int d = 0; d < dim; ++d) {
          double a = 0.5 * (q[c][d][IDX(eL, nL, Np)] + q[c][d][IDX(eR, nR, Np)]);
          avg[c][d][IDX(eL, fL * Nfp + kL, NF)] += a;
          avg[c][d][IDX(eR, fR * Nfp + kR, NF)] += a;
        }
      }
    }
  }
  /* vmf_3d_mult_avg_jump over boundary faces, :178-211 (vmf_3d_mult_avg_jump.h:9-80) */
  for (int b = 0; b < m->Kb; ++b) {
    int e = m->bface2cell[b], f = m->bfaceNum[b];
    double n[3] = {m->nx[IDX(e, f, Nf)], m->ny[IDX(e, f, Nf)], dim == 3 ? m->nz[IDX(e, f, Nf)] : 0.0};
    int all_slip = ncomp == dim;
    for (int c = 0; c < ncomp; ++c) all_slip &= bc_types[c * m->Kb + b] == 2;
    for (int j = 0; j < Nfp; ++j) {
      int node = m->fmask[f * Nfp + j];
      size_t fi = IDX(e, f * Nfp + j, NF);
      if (all_slip) {
        /* projection n n^T applied to (u, v, w) and to each gradient direction */
        for (int c = 0; c < ncomp; ++c) {
          double pu = 0.0;
          for (int k = 0; k < ncomp; ++k) pu += n[c] * n[k] * x[k][IDX(e, node, Np)];
          jump[c][fi] += 2.0 * pu;
          for (int d = 0; d < dim; ++d) {
            double pq = 0.0;
            for (int k = 0; k < ncomp; ++k) pq += n[c] * n[k] * q[k][d][IDX(e, node, Np)];
            avg[c][d][fi] += pq;
          }
        }
        continue;
      }
      for (int c = 0; c < ncomp; ++c) {
        if (bc_types[c * m->Kb + b] != 0) continue; /* Neumann (and lone slip): nothing */
        jump[c][fi] += 2.0 * x[c][IDX(e, node, Np)];
        for (int d = 0; d < dim; ++d) avg[c][d][fi] += q[c][d][IDX(e, node, Np)];
      }
    }
  }
  /* fvmf_3d_mult_flux, :213-231 (fvmf_3d_mult_flux.h:6-24; vmf_3d_mult_flux.h with the flag) */
#pragma omp parallel for schedule(static)
  for (int e = 0; e < K; ++e)
    for (int f = 0; f < Nf; ++f) {
      double n[3] = {m->nx[IDX(e, f, Nf)], m->ny[IDX(e, f, Nf)], dim == 3 ? m->nz[IDX(e, f, Nf)] : 0.0};
      double sJ = m->sJ[IDX(e, f, Nf)], t = tau[IDX(e, f, Nf)];
      for (int j = 0; j < Nfp; ++j) {
        size_t fi = IDX(e, f * Nfp + j, NF);
        double fac = factor ? factor[IDX(e, m->fmask[f * Nfp + j], Np)] : 1.0;
        for (int c = 0; c < ncomp; ++c) {
          double hj = 0.5 * jump[c][fi];
          double sum = 0.0;
          int dmax = (flags & ORACLE_VMF_FLUX_BUG) && dim == 3 ? 2 : dim;
          for (int d = 0; d < dmax; ++d) sum += n[d] * avg[c][d][fi];
          jump[c][fi] = sJ * (t * hj - sum);
          for (int d = 0; d < dim; ++d) avg[c][d][fi] = n[d] * sJ * fac * -hj;
        }
      }
    }
  /* mesh->mass, EMAT lifts, geometric transform, D^T and mm term, :233-286 */
  for (int c = 0; c < ncomp; ++c) {
#pragma omp parallel for schedule(static)
    for (int e = 0; e < K; ++e) {
      double tmp[64];
      double G[3][3], J;
      geo_unpack(m, e, G, &J);
      double w[3][64];
      for (int d = 0; d < dim; ++d) {
        for (int i = 0; i < Np; ++i) {
          double s = 0.0;
          for (int j = 0; j < Np; ++j) s += m->M[i * Np + j] * q[c][d][IDX(e, j, Np)];
          tmp[i] = J * s;
        }
        for (int i = 0; i < Np; ++i) {
          double s = 0.0;
          for (int k = 0; k < NF; ++k) s += m->EMAT[i * NF + k] * avg[c][d][IDX(e, k, NF)];
          w[d][i] = tmp[i] + s;
        }
      }
      double *out = y[c] + (size_t)e * Np;
      for (int i = 0; i < Np; ++i) {
        double s = 0.0;
        for (int k = 0; k < NF; ++k) s += m->EMAT[i * NF + k] * jump[c][IDX(e, k, NF)];
        out[i] = s;
      }
      /* vmf_3d_mult_cells_geof.h:4-22: w_r = sum_d G[r][d] w_d */
      double wr[3][64];
      for (int i = 0; i < Np; ++i)
        for (int r = 0; r < dim; ++r) {
          double s = 0.0;
          for (int d = 0; d < dim; ++d) s += G[r][d] * w[d][i];
          wr[r][i] = s;
        }
      for (int r = 0; r < dim; ++r)
        for (int i = 0; i < Np; ++i) {
          double s = 0.0;
          for (int j = 0; j < Np; ++j) s += Dm[r][j * Np + i] * wr[r][j];
          out[i] += s;
        }
      /* fvmf_3d_mult_mm_geof.h:5-19 */
      if (mm_factor || mm_scalar != 0.0) {
        const double *u = x[c] + (size_t)e * Np;
        for (int i = 0; i < Np; ++i) {
          double s = 0.0;
          for (int j = 0; j < Np; ++j) {
            double mmv = mm_factor ? mm_factor[IDX(e, j, Np)] : mm_scalar;
            s += mmv * m->M[i * Np + j] * u[j];
          }
          out[i] += s * J;
        }
      }
    }
  }
  for (int c = 0; c < ncomp; ++c) {
    free(jump[c]);
    for (int d = 0; d < dim; ++d) { free(q[c][d]); free(avg[c][d]); }
  }
  free(tau);
}

/* Face derivative matrix D_n = factor-row-scaled (n . grad) for element e:
 * D[i][j] = f_i * sum_r (n . grad r) Dr[i][j]  (fvmf_3d_op2_diag.h:42-52). */
static void normal_deriv_matrix(const oracle_mesh *m, int e, const double n[3],
                                const double *factor, double *D) {
  const int Np = m->Np, dim = m->dim;
  double G[3][3], J;
  geo_unpack(m, e, G, &J);
  const double *Dm[3] = {m->Dr, m->Ds, m->Dt};
  double rf[3] = {0, 0, 0};
  for (int r = 0; r < dim; ++r)
    for (int d = 0; d < dim; ++d) rf[r] += n[d] * G[r][d];
  for (int i = 0; i < Np; ++i) {
    double f = factor ? factor[IDX(e, i, Np)] : 1.0;
    for (int j = 0; j < Np; ++j) {
      double s = 0.0;
      for (int r = 0; r < dim; ++r) s += rf[r] * Dm[r][i * Np + j];
      D[i * Np + j] = s * f;
    }
  }
}

/* ----------------------------------------------------------------- apply_bc */
/* fvmf_3d_apply_bc.h:29-85 (2D: fvmf_2d_apply_bc.h). */
void oracle_apply_bc(const oracle_mesh *m, int ncomp, const int *bc_types, const double *factor,
                     const double *const *bc, double *const *rhs) {
  const int Np = m->Np, Nfp = m->Nfp, Nf = m->Nf, p = m->order;
  double *D = (double *)malloc(sizeof(double) * Np * Np);
  double *tmp = (double *)malloc(sizeof(double) * Np);
  for (int b = 0; b < m->Kb; ++b) {
    int e = m->bface2cell[b], f = m->bfaceNum[b];
    double n[3] = {m->nx[IDX(e, f, Nf)], m->ny[IDX(e, f, Nf)], m->dim == 3 ? m->nz[IDX(e, f, Nf)] : 0.0};
    double sJ = m->sJ[IDX(e, f, Nf)], fs = m->fscale[IDX(e, f, Nf)];
    const double *mmF = m->MMF + (size_t)f * Np * Np;
    for (int c = 0; c < ncomp; ++c) {
      int t = bc_types[c * m->Kb + b];
      const double *g = bc[c] + (size_t)b * Nfp;
      double *out = rhs[c] + (size_t)e * Np;
      if (t == 0) {
        normal_deriv_matrix(m, e, n, factor, D);
        double gtau = factor ? factor[IDX(e, m->fmask[f * Nfp], Np)] : 1.0;
        for (int j = 1; j < Nfp; ++j)
          if (factor) gtau = fmax(gtau, factor[IDX(e, m->fmask[f * Nfp + j], Np)]);
        gtau *= 2.0 * (p + 1) * (p + 2) * fs;
        for (int i = 0; i < Np; ++i) {
          tmp[i] = 0.0;
          for (int j = 0; j < Nfp; ++j) {
            double mm = mmF[i * Np + m->fmask[f * Nfp + j]];
            out[i] += gtau * sJ * mm * g[j];
            tmp[i] += sJ * mm * g[j];
          }
        }
        for (int i = 0; i < Np; ++i)
          for (int j = 0; j < Np; ++j) out[i] += -D[j * Np + i] * tmp[j];
      } else if (t == 1) {
        for (int i = 0; i < Np; ++i)
          for (int j = 0; j < Nfp; ++j) out[i] += sJ * mmF[i * Np + m->fmask[f * Nfp + j]] * g[j];
      }
    }
  }
  free(D);
  free(tmp);
}

/* ------------------------------------------------------------- diagonals */
/* Volume block J * Dx^T M F Dx summed over directions (exact), or the
 * reference's forms with ORACLE_REF_BLOCK_DIAG: 3D fvmf_3d_op1.h:17-18
 * (D * (J M F D)), 2D fvmf_2d_op1.h:20-37 (J Dx^T F M Dx). */
static void volume_block(const oracle_mesh *m, int e, const double *factor, int flags,
                         double *blk) {
  const int Np = m->Np, dim = m->dim;
  double G[3][3], J;
  geo_unpack(m, e, G, &J);
  const double *Dm[3] = {m->Dr, m->Ds, m->Dt};
  double *Dx = (double *)malloc(sizeof(double) * Np * Np);
  double *T = (double *)malloc(sizeof(double) * Np * Np);
  memset(blk, 0, sizeof(double) * Np * Np);
  for (int d = 0; d < dim; ++d) {
    for (int i = 0; i < Np; ++i)
      for (int j = 0; j < Np; ++j) {
        double s = 0.0;
        for (int r = 0; r < dim; ++r) s += G[r][d] * Dm[r][i * Np + j];
        Dx[i * Np + j] = s;
      }
    int ref2d = (flags & ORACLE_REF_BLOCK_DIAG) && dim == 2;
    /* T = J M F Dx (or J F M Dx for the 2D reference form) */
    for (int i = 0; i < Np; ++i)
      for (int j = 0; j < Np; ++j) {
        double s = 0.0;
        for (int k = 0; k < Np; ++k) {
          double fk = factor ? factor[IDX(e, k, Np)] : 1.0;
          double fi = factor ? factor[IDX(e, i, Np)] : 1.0;
          s += m->M[i * Np + k] * (ref2d ? fi : fk) * Dx[k * Np + j];
        }
        T[i * Np + j] = J * s;
      }
    int ref3d = (flags & ORACLE_REF_BLOCK_DIAG) && dim == 3;
    for (int i = 0; i < Np; ++i)
      for (int j = 0; j < Np; ++j) {
        double s = 0.0;
        for (int k = 0; k < Np; ++k) s += (ref3d ? Dx[i * Np + k] : Dx[k * Np + i]) * T[k * Np + j];
        blk[i * Np + j] += s;
      }
  }
  free(Dx);
  free(T);
}

/* Face block: scale * (gtau * MF - (MF D + D^T MF)) (fvmf_3d_op2_block_diag.h,
 * fvmf_3d_bop_block_diag.h). */
static void face_block(const oracle_mesh *m, int f, const double *D, double gtau,
                       double scale, double *blk) {
  const int Np = m->Np;
  const double *mmF = m->MMF + (size_t)f * Np * Np;
  for (int i = 0; i < Np; ++i)
    for (int j = 0; j < Np; ++j) {
      double s = 0.0;
      for (int k = 0; k < Np; ++k) s += mmF[i * Np + k] * D[k * Np + j] + D[k * Np + i] * mmF[k * Np + j];
      blk[i * Np + j] += scale * (gtau * mmF[i * Np + j] - s);
    }
}

static double interior_gtau(const oracle_mesh *m, int fc, const double *factor) {
  const int Np = m->Np, Nfp = m->Nfp, Nf = m->Nf, p = m->order;
  int eL = m->face2cells[2 * fc], eR = m->face2cells[2 * fc + 1];
  int fL = m->faceNum[2 * fc], fR = m->faceNum[2 * fc + 1];
  double gtau = 0.0;
  for (int j = 0; j < Nfp; ++j) {
    double fl = factor ? factor[IDX(eL, m->fmask[fL * Nfp + j], Np)] : 1.0;
    double fr = factor ? factor[IDX(eR, m->fmaskR[fc * Nfp + j], Np)] : 1.0;
    gtau = fmax(gtau, 2.0 * (p + 1) * (p + 2) *
                          fmax(m->fscale[IDX(eL, fL, Nf)] * fl, m->fscale[IDX(eR, fR, Nf)] * fr));
  }
  return gtau;
}

static double boundary_gtau(const oracle_mesh *m, int b, const double *factor) {
  const int Np = m->Np, Nfp = m->Nfp, Nf = m->Nf, p = m->order;
  int e = m->bface2cell[b], f = m->bfaceNum[b];
  double gtau = 0.0;
  for (int j = 0; j < Nfp; ++j) {
    double fv = factor ? factor[IDX(e, m->fmask[f * Nfp + j], Np)] : 1.0;
    gtau = fmax(gtau, 2.0 * (p + 1) * (p + 2) * m->fscale[IDX(e, f, Nf)] * fv);
  }
  return gtau;
}

/* calc_inv_block_diag, factor_viscous_matrix.cpp:368-451 (and the inverse). */
static void invert_inplace(double *A, int n);

void oracle_block_diag(const oracle_mesh *m, int ncomp, const int *bc_types,
                       const double *factor, const double *mm_factor, double mm_scalar,
                       int flags, int inv, double *blocks) {
  const int Np = m->Np, Nf = m->Nf, K = m->K, NN = Np * Np;
  double *D = (double *)malloc(sizeof(double) * NN);
  double *blk = (double *)malloc(sizeof(double) * NN);
#pragma omp parallel for schedule(static)
  for (int e = 0; e < K; ++e) {
    double *blk = blocks + (size_t)e * NN; /* built in the first component's slot */
    volume_block(m, e, factor, flags, blk); /* fvmf_3d_op1 */
    /* mass term: the operator scales columns (fvmf_3d_mult_mm_geof.h:12); the
     * reference's block scales rows (fvmf_3d_mm_block_diag.h:7) */
    if (mm_factor || mm_scalar != 0.0) {
      double G[3][3], J;
      geo_unpack(m, e, G, &J);
      for (int i = 0; i < Np; ++i)
        for (int j = 0; j < Np; ++j)
          blk[i * Np + j] += (mm_factor ? mm_factor[IDX(e, (flags & ORACLE_REF_BLOCK_DIAG) ? i : j, Np)]
                                        : mm_scalar) * J * m->M[i * Np + j];
    }
    for (int c = 1; c < ncomp; ++c) memcpy(blocks + ((size_t)c * K + e) * NN, blk, sizeof(double) * NN);
  }
  /* fvmf_3d_op2_block_diag over interior faces */
  for (int fc = 0; fc < m->F; ++fc) {
    double gtau = interior_gtau(m, fc, factor);
    for (int side = 0; side < 2; ++side) {
      int e = m->face2cells[2 * fc + side], f = m->faceNum[2 * fc + side];
      double n[3] = {m->nx[IDX(e, f, Nf)], m->ny[IDX(e, f, Nf)], m->dim == 3 ? m->nz[IDX(e, f, Nf)] : 0.0};
      normal_deriv_matrix(m, e, n, factor, D);
      memset(blk, 0, sizeof(double) * NN);
      face_block(m, f, D, gtau, 0.5 * m->sJ[IDX(e, f, Nf)], blk);
      for (int c = 0; c < ncomp; ++c) {
        double *B = blocks + ((size_t)c * K + e) * NN;
        for (int i = 0; i < NN; ++i) B[i] += blk[i];
      }
    }
  }
  /* fvmf_3d_bop_block_diag over boundary faces */
  for (int b = 0; b < m->Kb; ++b) {
    int e = m->bface2cell[b], f = m->bfaceNum[b];
    double n[3] = {m->nx[IDX(e, f, Nf)], m->ny[IDX(e, f, Nf)], m->dim == 3 ? m->nz[IDX(e, f, Nf)] : 0.0};
    int all_slip = ncomp == m->dim;
    for (int c = 0; c < ncomp; ++c) all_slip &= bc_types[c * m->Kb + b] == 2;
    double gtau = boundary_gtau(m, b, factor);
    normal_deriv_matrix(m, e, n, factor, D);
    for (int c = 0; c < ncomp; ++c) {
      double scale;
      if (all_slip) scale = m->sJ[IDX(e, f, Nf)] * n[c] * n[c];
      else if (bc_types[c * m->Kb + b] == 0) scale = m->sJ[IDX(e, f, Nf)];
      else continue;
      memset(blk, 0, sizeof(double) * NN);
      face_block(m, f, D, gtau, scale, blk);
      double *B = blocks + ((size_t)c * K + e) * NN;
      for (int i = 0; i < NN; ++i) B[i] += blk[i];
    }
  }
  if (inv)
    for (size_t i = 0; i < (size_t)ncomp * K; ++i) invert_inplace(blocks + i * NN, Np);
  free(D);
  free(blk);
}

/* calc_diag, factor_viscous_matrix.cpp:312-366: the diagonal of the blocks
 * above (fvmf_3d_op1_diag, fvmf_3d_op2_diag, fvmf_3d_mm_diag, fvmf_3d_bop_diag). */
void oracle_diag(const oracle_mesh *m, int ncomp, const int *bc_types, const double *factor,
                 const double *mm_factor, double mm_scalar, double *diag) {
  const int Np = m->Np, K = m->K;
  double *blocks = (double *)malloc(sizeof(double) * (size_t)ncomp * K * Np * Np);
  oracle_block_diag(m, ncomp, bc_types, factor, mm_factor, mm_scalar, 0, 0, blocks);
  for (size_t b = 0; b < (size_t)ncomp * K; ++b)
    for (int i = 0; i < Np; ++i) diag[b * Np + i] = blocks[(b * Np + i) * Np + i];
  free(blocks);
}

static void invert_inplace(double *A, int n) {
  double *a = (double *)malloc(sizeof(double) * n * n);
  double *v = (double *)malloc(sizeof(double) * n * n);
  memcpy(a, A, sizeof(double) * n * n);
  memset(v, 0, sizeof(double) * n * n);
  for (int i = 0; i < n; ++i) v[i * n + i] = 1.0;
  for (int c = 0; c < n; ++c) {
    int piv = c;
    for (int i = c + 1; i < n; ++i)
      if (fabs(a[i * n + c]) > fabs(a[piv * n + c])) piv = i;
    if (piv != c)
      for (int j = 0; j < n; ++j) {
        double t = a[c * n + j]; a[c * n + j] = a[piv * n + j]; a[piv * n + j] = t;
        t = v[c * n + j]; v[c * n + j] = v[piv * n + j]; v[piv * n + j] = t;
      }
    double d = a[c * n + c];
    for (int j = 0; j < n; ++j) { a[c * n + j] /= d; v[c * n + j] /= d; }
    for (int i = 0; i < n; ++i) {
      if (i == c) continue;
      double f = a[i * n + c];
      for (int j = 0; j < n; ++j) { a[i * n + j] -= f * a[c * n + j]; v[i * n + j] -= f * v[c * n + j]; }
    }
  }
  memcpy(A, v, sizeof(double) * n * n);
  free(a);
  free(v);
}

/* ---------------------------------------------------------------- solvers */
typedef struct {
  const oracle_mesh *m;
  int ncomp;
  const int *bc_types;
  const double *factor, *mm_factor;
  double mm_scalar;
  int flags;
  int pin_dof;
  double pin_scale;
  oracle_mult_fn mult;  /* NULL: oracle_mult */
} op_ctx;

static size_t vec_len(const op_ctx *o) { return (size_t)o->ncomp * o->m->K * o->m->Np; }

/* Operator with an optional pinned DOF: y = A x~ (x~ = x with x[pin] = 0),
 * then y[pin] = A_pin,pin * x[pin]. */
static void op_apply(const op_ctx *o, const double *x, double *y) {
  size_t n = vec_len(o), per = (size_t)o->m->K * o->m->Np;
  const double *xs[3] = {NULL, NULL, NULL};
  double *ys[3] = {NULL, NULL, NULL};
  double *xc = NULL, xpin = 0.0;
  if (o->pin_dof >= 0) {
    xc = (double *)malloc(sizeof(double) * n);
    memcpy(xc, x, sizeof(double) * n);
    xpin = x[o->pin_dof];
    xc[o->pin_dof] = 0.0;
    x = xc;
  }
  for (int c = 0; c < o->ncomp; ++c) { xs[c] = x + c * per; ys[c] = y + c * per; }
  if (o->mult) {
    if (o->mult(o->m, o->ncomp, o->bc_types, o->factor, o->mm_factor, o->mm_scalar, o->flags, xs, ys) != 0)
      memset(y, 0xff, sizeof(double) * n); /* NaN: an apply the hook cannot do poisons the solve */
  } else {
    oracle_mult(o->m, o->ncomp, o->bc_types, o->factor, o->mm_factor, o->mm_scalar, o->flags, xs, ys);
  }
  if (xc) {
    y[o->pin_dof] = o->pin_scale * xpin;
    free(xc);
  }
}

static double dot(const double *a, const double *b, size_t n) {
  double s = 0.0;
  for (size_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

/* ---- p-multigrid (restated design; PETScPMultigrid is unvendored, its keys
 * orders / cheb_orders / eigen_val_saftey_factor are read from
 * examples/3d/oscillating_droplet/config.ini:24-31).
 * V-cycle: Chebyshev(k) pre-smoothing with Jacobi scaling on
 * [lmax*safety/ratio, lmax*safety], residual restriction by P^T, recursive
 * coarse correction prolongated by P, Chebyshev(k) post-smoothing; the
 * coarsest level runs a fixed number of Jacobi-PCG iterations from zero. */
typedef struct {
  op_ctx op;
  double *dinv;
  double *binv;    /* smoother 1: inverse diagonal blocks, row-major per element (else NULL) */
  double lmax;
  const double *P; /* prolongation from the next level */
  int np_next;
} pmg_level;

/* out = S in for the level's smoother S: D^-1 (Jacobi) or the inverse diagonal
 * blocks (element-block Jacobi). */
static void smoother_apply(const op_ctx *o, const double *dinv, const double *binv, const double *in,
                           double *out) {
  size_t n = (size_t)o->ncomp * o->m->K * o->m->Np;
  if (!binv) {
    for (size_t i = 0; i < n; ++i) out[i] = dinv[i] * in[i];
    return;
  }
  const int Np = o->m->Np;
  const size_t nb = n / Np;
#pragma omp parallel for schedule(static)
  for (size_t b = 0; b < nb; ++b)
    for (int i = 0; i < Np; ++i) {
      double s = 0.0;
      for (int j = 0; j < Np; ++j) s += binv[(b * Np + i) * Np + j] * in[b * Np + j];
      out[b * Np + i] = s;
    }
}

static uint64_t smix(uint64_t *s) {
  uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

/* Power iteration on S A (S the smoother: D^-1, or the inverse diagonal blocks
 * when binv != NULL) from start vector v0_i = U(-1,1) (splitmix64 seed 0x5eed);
 * lambda = ||S A v|| / ||v|| after `iters` normalised steps. */
static double power_lmax(const op_ctx *o, const double *dinv, const double *binv, int iters) {
  size_t n = vec_len(o);
  double *v = (double *)malloc(sizeof(double) * n), *w = (double *)malloc(sizeof(double) * n);
  double *t = (double *)malloc(sizeof(double) * n);
  uint64_t s = 0x5eedull;
  for (size_t i = 0; i < n; ++i) v[i] = 2.0 * ((smix(&s) >> 11) * (1.0 / 9007199254740992.0)) - 1.0;
  double lam = 0.0;
  for (int it = 0; it < iters; ++it) {
    double nv = sqrt(dot(v, v, n));
    for (size_t i = 0; i < n; ++i) v[i] /= nv;
    op_apply(o, v, t);
    smoother_apply(o, dinv, binv, t, w);
    lam = sqrt(dot(w, w, n));
    double *tt = v; v = w; w = tt;
  }
  free(v);
  free(w);
  free(t);
  return lam;
}

static void compute_dinv(const op_ctx *o, double *dinv) {
  size_t n = vec_len(o);
  oracle_diag(o->m, o->ncomp, o->bc_types, o->factor, o->mm_factor, o->mm_scalar, dinv);
  for (size_t i = 0; i < n; ++i) dinv[i] = 1.0 / dinv[i];
}

double oracle_pmg_lambda_max(const oracle_mesh *m, const int *bc_types, const double *factor,
                             int pin_dof, int iters) {
  op_ctx o = {m, 1, bc_types, factor, NULL, 0.0, 0, pin_dof, 0.0, NULL};
  size_t n = vec_len(&o);
  double *dinv = (double *)malloc(sizeof(double) * n);
  compute_dinv(&o, dinv);
  if (pin_dof >= 0) o.pin_scale = 1.0 / dinv[pin_dof];
  double l = power_lmax(&o, dinv, NULL, iters);
  free(dinv);
  return l;
}

/* Chebyshev smoothing of A z = r starting from (z, res = r - A z).
 * On exit z is updated and, if want_res, res = r - A z. */
static void chebyshev(const pmg_level *L, int k, double safety, double ratio, double *z,
                      double *res, int want_res) {
  size_t n = vec_len(&L->op);
  double hi = L->lmax * safety, lo = hi / ratio;
  double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
  double *d = (double *)malloc(sizeof(double) * n), *Ad = (double *)malloc(sizeof(double) * n);
  double *sr = (double *)malloc(sizeof(double) * n);
  double rho_old = 1.0 / sigma;
  smoother_apply(&L->op, L->dinv, L->binv, res, sr);
  for (size_t i = 0; i < n; ++i) d[i] = sr[i] / theta;
  for (int it = 0; it < k; ++it) {
    if (it > 0) {
      double rho = 1.0 / (2.0 * sigma - rho_old);
      smoother_apply(&L->op, L->dinv, L->binv, res, sr);
      for (size_t i = 0; i < n; ++i) d[i] = rho * rho_old * d[i] + (2.0 * rho / delta) * sr[i];
      rho_old = rho;
    }
    for (size_t i = 0; i < n; ++i) z[i] += d[i];
    if (it < k - 1 || want_res) {
      op_apply(&L->op, d, Ad);
      for (size_t i = 0; i < n; ++i) res[i] -= Ad[i];
    }
  }
  free(d);
  free(Ad);
  free(sr);
}

/* Fixed-count Jacobi-preconditioned CG from zero (coarsest level). */
static void coarse_cg(const pmg_level *L, int iters, const double *r, double *z) {
  size_t n = vec_len(&L->op);
  double *res = (double *)malloc(sizeof(double) * n), *p = (double *)malloc(sizeof(double) * n);
  double *s = (double *)malloc(sizeof(double) * n), *Ap = (double *)malloc(sizeof(double) * n);
  memset(z, 0, sizeof(double) * n);
  memcpy(res, r, sizeof(double) * n);
  for (size_t i = 0; i < n; ++i) s[i] = L->dinv[i] * res[i];
  memcpy(p, s, sizeof(double) * n);
  double rz = dot(res, s, n);
  for (int it = 0; it < iters && rz > 0.0; ++it) {
    op_apply(&L->op, p, Ap);
    double pAp = dot(p, Ap, n);
    if (!(pAp > 0.0)) break;
    double alpha = rz / pAp;
    for (size_t i = 0; i < n; ++i) { z[i] += alpha * p[i]; res[i] -= alpha * Ap[i]; }
    for (size_t i = 0; i < n; ++i) s[i] = L->dinv[i] * res[i];
    double rz_new = dot(res, s, n);
    double beta = rz_new / rz;
    rz = rz_new;
    for (size_t i = 0; i < n; ++i) p[i] = s[i] + beta * p[i];
  }
  free(res); free(p); free(s); free(Ap);
}

/* ---- algebraic levels below p=0 (element-wise constants) */
static void csr_mv(const oracle_csr *A, const double *x, double *y) {
  for (int i = 0; i < A->rows; ++i) {
    double s = 0.0;
    for (int k = A->ptr[i]; k < A->ptr[i + 1]; ++k) s += A->val[k] * x[A->idx[k]];
    y[i] = s;
  }
}

typedef struct {
  double *dinv;
  double lmax;
} amg_level;

static double csr_power_lmax(const oracle_csr *A, const double *dinv, int iters) {
  size_t n = (size_t)A->rows;
  double *v = (double *)malloc(sizeof(double) * n), *w = (double *)malloc(sizeof(double) * n);
  uint64_t s = 0x5eedull;
  for (size_t i = 0; i < n; ++i) v[i] = 2.0 * ((smix(&s) >> 11) * (1.0 / 9007199254740992.0)) - 1.0;
  double lam = 0.0;
  for (int it = 0; it < iters; ++it) {
    double nv = sqrt(dot(v, v, n));
    for (size_t i = 0; i < n; ++i) v[i] /= nv;
    csr_mv(A, v, w);
    for (size_t i = 0; i < n; ++i) w[i] *= dinv[i];
    lam = sqrt(dot(w, w, n));
    double *t = v; v = w; w = t;
  }
  free(v);
  free(w);
  return lam;
}

/* Chebyshev smoothing on a CSR level; same recurrence as chebyshev() above. */
static void csr_chebyshev(const oracle_csr *A, const amg_level *L, int k, double safety, double ratio,
                          double *z, double *res, int want_res) {
  size_t n = (size_t)A->rows;
  double hi = L->lmax * safety, lo = hi / ratio;
  double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
  double *d = (double *)malloc(sizeof(double) * n), *Ad = (double *)malloc(sizeof(double) * n);
  double rho_old = 1.0 / sigma;
  for (size_t i = 0; i < n; ++i) d[i] = L->dinv[i] * res[i] / theta;
  for (int it = 0; it < k; ++it) {
    if (it > 0) {
      double rho = 1.0 / (2.0 * sigma - rho_old);
      for (size_t i = 0; i < n; ++i) d[i] = rho * rho_old * d[i] + (2.0 * rho / delta) * L->dinv[i] * res[i];
      rho_old = rho;
    }
    for (size_t i = 0; i < n; ++i) z[i] += d[i];
    if (it < k - 1 || want_res) {
      csr_mv(A, d, Ad);
      for (size_t i = 0; i < n; ++i) res[i] -= Ad[i];
    }
  }
  free(d);
  free(Ad);
}

static void amg_vcycle(const oracle_solver_opts *o, const amg_level *al, int l, const double *r,
                       double *z) {
  const oracle_csr *A = &o->amg_A[l];
  size_t n = (size_t)A->rows;
  if (l == o->amg_nlevels - 1) {
    for (size_t i = 0; i < n; ++i) {
      double s = 0.0;
      for (size_t j = 0; j < n; ++j) s += o->amg_coarse_inv[i * n + j] * r[j];
      z[i] = s;
    }
    return;
  }
  size_t nc = (size_t)o->amg_A[l + 1].rows;
  double *res = (double *)malloc(sizeof(double) * n), *tmp = (double *)malloc(sizeof(double) * n);
  double *rc = (double *)malloc(sizeof(double) * nc), *zc = (double *)malloc(sizeof(double) * nc);
  memset(z, 0, sizeof(double) * n);
  memcpy(res, r, sizeof(double) * n);
  const int deg = o->amg_cheb_order > 0 ? o->amg_cheb_order : o->cheb_order;
  csr_chebyshev(A, &al[l], deg, o->eig_safety, o->eig_ratio, z, res, 1);
  csr_mv(&o->amg_R[l], res, rc);
  amg_vcycle(o, al, l + 1, rc, zc);
  csr_mv(&o->amg_P[l], zc, tmp);
  for (size_t i = 0; i < n; ++i) z[i] += tmp[i];
  csr_mv(A, z, tmp);
  for (size_t i = 0; i < n; ++i) res[i] = r[i] - tmp[i];
  csr_chebyshev(A, &al[l], deg, o->eig_safety, o->eig_ratio, z, res, 0);
  free(res); free(tmp); free(rc); free(zc);
}

static void vcycle(const pmg_level *lv, int nl, int l, const oracle_solver_opts *o,
                   const double *r, double *z, const amg_level *al);

/* Last order level with an algebraic coarse solve: Chebyshev, restriction to
 * the algebraic level 0 (R_dg), AMG V-cycle, prolongation (P_dg), Chebyshev. */
static void last_level_amg(const pmg_level *L, const oracle_solver_opts *o, const double *r,
                           double *z, const amg_level *al) {
  size_t n = vec_len(&L->op);
  size_t n0 = (size_t)o->amg_A[0].rows;
  double *res = (double *)malloc(sizeof(double) * n), *tmp = (double *)malloc(sizeof(double) * n);
  double *r0 = (double *)malloc(sizeof(double) * n0), *z0 = (double *)malloc(sizeof(double) * n0);
  memset(z, 0, sizeof(double) * n);
  memcpy(res, r, sizeof(double) * n);
  chebyshev(L, o->cheb_order, o->eig_safety, o->eig_ratio, z, res, 1);
  csr_mv(o->amg_Rdg, res, r0);
  amg_vcycle(o, al, 0, r0, z0);
  csr_mv(o->amg_Pdg, z0, tmp);
  for (size_t i = 0; i < n; ++i) z[i] += tmp[i];
  op_apply(&L->op, z, tmp);
  for (size_t i = 0; i < n; ++i) res[i] = r[i] - tmp[i];
  chebyshev(L, o->cheb_order, o->eig_safety, o->eig_ratio, z, res, 0);
  free(res); free(tmp); free(r0); free(z0);
}

static void vcycle(const pmg_level *lv, int nl, int l, const oracle_solver_opts *o,
                   const double *r, double *z, const amg_level *al) {
  const pmg_level *L = &lv[l];
  size_t n = vec_len(&L->op);
  if (l == nl - 1) {
    if (o->coarse_kind == 1) last_level_amg(L, o, r, z, al);
    else coarse_cg(L, o->coarse_iters, r, z);
    return;
  }
  const pmg_level *C = &lv[l + 1];
  size_t nc = vec_len(&C->op);
  double *res = (double *)malloc(sizeof(double) * n), *tmp = (double *)malloc(sizeof(double) * n);
  double *rc = (double *)calloc(nc, sizeof(double)), *zc = (double *)calloc(nc, sizeof(double));
  memset(z, 0, sizeof(double) * n);
  memcpy(res, r, sizeof(double) * n);
  chebyshev(L, o->cheb_order, o->eig_safety, o->eig_ratio, z, res, 1);
  /* restriction rc = P^T res, element by element */
  const int Np = L->op.m->Np, Npc = C->op.m->Np, K = L->op.m->K;
  for (int c = 0; c < L->op.ncomp; ++c)
    for (int e = 0; e < K; ++e)
      for (int j = 0; j < Npc; ++j) {
        double s = 0.0;
        for (int i = 0; i < Np; ++i) s += L->P[i * Npc + j] * res[((size_t)c * K + e) * Np + i];
        rc[((size_t)c * K + e) * Npc + j] = s;
      }
  vcycle(lv, nl, l + 1, o, rc, zc, al);
  for (int c = 0; c < L->op.ncomp; ++c)
    for (int e = 0; e < K; ++e)
      for (int i = 0; i < Np; ++i) {
        double s = 0.0;
        for (int j = 0; j < Npc; ++j) s += L->P[i * Npc + j] * zc[((size_t)c * K + e) * Npc + j];
        z[((size_t)c * K + e) * Np + i] += s;
      }
  op_apply(&L->op, z, tmp);
  for (size_t i = 0; i < n; ++i) res[i] = r[i] - tmp[i];
  chebyshev(L, o->cheb_order, o->eig_safety, o->eig_ratio, z, res, 0);
  free(res); free(tmp); free(rc); free(zc);
}

static void project_mean(double *v, size_t n) {
  double s = 0.0;
  for (size_t i = 0; i < n; ++i) s += v[i];
  s /= (double)n;
  for (size_t i = 0; i < n; ++i) v[i] -= s;
}

/* CG (viscous_solver.cpp:89-174) when precond == NONE, otherwise the flexible
 * PCG of viscous_solver.cpp:177-301 (beta = r.(z - z_old) / (r.z)_old).
 * Stop: ||r||_2 <= max(abs_tol, rel_tol * ||b||_2); the reference tests abs_tol only
 * (viscous_solver.cpp:116-117), which is rel_tol = 0. */
void oracle_solve(const oracle_mesh *m, const oracle_solver_opts *o, const double *b, double *x,
                  oracle_solve_info *info) {
  op_ctx op = {m, o->ncomp, o->bc_types, o->factor, o->mm_factor, o->mm_scalar, o->flags, o->pin_dof, 0.0,
               o->outer_mult ? o->outer_mult : o->mult};
  size_t n = vec_len(&op);
  const int Np = m->Np, K = m->K;
  const double t_setup = wall_s();
  double *dinv = NULL, *blocks = NULL;
  pmg_level *lv = NULL;
  amg_level *al = NULL;
  int nl = 0;
  if (o->pin_dof >= 0 || o->precond == ORACLE_PRE_JACOBI) {
    dinv = (double *)malloc(sizeof(double) * n);
    compute_dinv(&op, dinv);
    if (o->pin_dof >= 0) op.pin_scale = 1.0 / dinv[o->pin_dof];
  }
  if (o->precond == ORACLE_PRE_BLOCK_JACOBI) {
    blocks = (double *)malloc(sizeof(double) * (size_t)o->ncomp * K * Np * Np);
    oracle_block_diag(m, o->ncomp, o->bc_types, o->factor, o->mm_factor, o->mm_scalar, o->flags, 1, blocks);
  }
  if (o->precond == ORACLE_PRE_PMG) {
    nl = o->pmg_nlevels;
    lv = (pmg_level *)calloc(nl, sizeof(pmg_level));
    for (int l = 0; l < nl; ++l) {
      op_ctx ol = {&o->pmg_meshes[l], o->ncomp, o->bc_types, o->pmg_factors[l], NULL, 0.0, 0, o->pin_dof, 0.0,
                   o->mult};
      if (o->pin_dof >= 0) ol.pin_dof = (o->pin_dof / Np) * o->pmg_meshes[l].Np + (o->pin_dof % Np);
      lv[l].op = ol;
      size_t nlv = vec_len(&ol);
      lv[l].dinv = (double *)malloc(sizeof(double) * nlv);
      compute_dinv(&lv[l].op, lv[l].dinv);
      if (ol.pin_dof >= 0) lv[l].op.pin_scale = 1.0 / lv[l].dinv[ol.pin_dof];
      lv[l].binv = NULL;
      if (o->smoother == 1) {
        /* inverse diagonal blocks of the pinned operator: the pinned row and
         * column of its element's block become pin_scale * identity */
        const oracle_mesh *lm = &o->pmg_meshes[l];
        const int Npl = lm->Np;
        lv[l].binv = (double *)malloc(sizeof(double) * nlv * Npl);
        oracle_block_diag(lm, o->ncomp, o->bc_types, o->pmg_factors[l], NULL, 0.0, 0, 0, lv[l].binv);
        if (ol.pin_dof >= 0) {
          double *B = lv[l].binv + (size_t)(ol.pin_dof / Npl) * Npl * Npl;
          const int pn = ol.pin_dof % Npl;
          for (int i = 0; i < Npl; ++i)
            if (i != pn) { B[pn * Npl + i] = 0.0; B[i * Npl + pn] = 0.0; }
          B[pn * Npl + pn] = lv[l].op.pin_scale;
        }
#pragma omp parallel for schedule(static)
        for (size_t b = 0; b < nlv / Npl; ++b) invert_inplace(lv[l].binv + b * Npl * Npl, Npl);
      }
      lv[l].lmax = power_lmax(&lv[l].op, lv[l].dinv, lv[l].binv, o->eig_iters);
      lv[l].P = l < nl - 1 ? o->pmg_prolong[l] : NULL;
    }
    if (o->coarse_kind == 1) {
      al = (amg_level *)calloc(o->amg_nlevels, sizeof(amg_level));
      for (int l = 0; l + 1 < o->amg_nlevels; ++l) {
        const oracle_csr *A = &o->amg_A[l];
        al[l].dinv = (double *)malloc(sizeof(double) * A->rows);
        for (int i = 0; i < A->rows; ++i) {
          double d = 0.0;
          for (int k = A->ptr[i]; k < A->ptr[i + 1]; ++k)
            if (A->idx[k] == i) d = A->val[k];
          al[l].dinv[i] = 1.0 / d;
        }
        al[l].lmax = csr_power_lmax(A, al[l].dinv, o->eig_iters);
      }
    }
  }
  const double t_solve = wall_s();
  double *r = (double *)malloc(sizeof(double) * n), *z = (double *)malloc(sizeof(double) * n);
  double *zo = (double *)malloc(sizeof(double) * n), *p = (double *)malloc(sizeof(double) * n);
  double *Ap = (double *)malloc(sizeof(double) * n);
  double bnorm = sqrt(dot(b, b, n));
  double tol = fmax(o->abs_tol, o->rel_tol * bnorm);
  /* calc_res_explicit, :329-343 */
  op_apply(&op, x, Ap);
  for (size_t i = 0; i < n; ++i) r[i] = b[i] - Ap[i];
  if (o->nullspace) project_mean(r, n);
  double res = sqrt(dot(r, r, n));
#define PRECOND(in, out)                                                                   \
  do {                                                                                     \
    switch (o->precond) {                                                                  \
      case ORACLE_PRE_NONE: memcpy(out, in, sizeof(double) * n); break;                    \
      case ORACLE_PRE_INV_MASS:                                                            \
      case ORACLE_PRE_FACTOR_INV_MASS: {                                                   \
        double sc = o->precond == ORACLE_PRE_FACTOR_INV_MASS ? o->inv_mass_factor : 1.0;   \
        for (int c_ = 0; c_ < o->ncomp; ++c_)                                              \
          for (int e_ = 0; e_ < K; ++e_) {                                                 \
            double G_[3][3], J_;                                                           \
            geo_unpack(m, e_, G_, &J_);                                                    \
            const double *vi = in + ((size_t)c_ * K + e_) * Np;                            \
            double *vo = out + ((size_t)c_ * K + e_) * Np;                                 \
            for (int i_ = 0; i_ < Np; ++i_) {                                              \
              double s_ = 0.0;                                                             \
              for (int j_ = 0; j_ < Np; ++j_) s_ += minv[i_ * Np + j_] * vi[j_];           \
              vo[i_] = sc * s_ / J_;                                                       \
            }                                                                              \
          }                                                                                \
      } break;                                                                             \
      case ORACLE_PRE_JACOBI:                                                              \
        for (size_t i_ = 0; i_ < n; ++i_) out[i_] = in[i_] * dinv[i_];                     \
        break;                                                                             \
      case ORACLE_PRE_BLOCK_JACOBI:                                                        \
        for (size_t b_ = 0; b_ < (size_t)o->ncomp * K; ++b_)                               \
          for (int i_ = 0; i_ < Np; ++i_) {                                                \
            double s_ = 0.0;                                                               \
            for (int j_ = 0; j_ < Np; ++j_) s_ += blocks[(b_ * Np + i_) * Np + j_] * in[b_ * Np + j_]; \
            out[b_ * Np + i_] = s_;                                                        \
          }                                                                                \
        break;                                                                             \
      case ORACLE_PRE_PMG: vcycle(lv, nl, 0, o, in, out, al); break;                       \
    }                                                                                      \
    if (o->nullspace) project_mean(out, n);                                                \
  } while (0)
  double *minv = NULL;
  if (o->precond == ORACLE_PRE_INV_MASS || o->precond == ORACLE_PRE_FACTOR_INV_MASS) {
    minv = (double *)malloc(sizeof(double) * Np * Np);
    memcpy(minv, m->M, sizeof(double) * Np * Np);
    invert_inplace(minv, Np);
  }
  int iter = 0;
  double t_iter = wall_s();
  if (o->precond == ORACLE_PRE_NONE) {
    memcpy(p, r, sizeof(double) * n);
    while (res > tol && iter < o->max_iter) {
      op_apply(&op, p, Ap);
      double a0 = dot(r, r, n), a1 = dot(p, Ap, n);   /* cg3_alpha.h */
      double alpha = a0 / a1;
      for (size_t i = 0; i < n; ++i) x[i] += alpha * p[i]; /* cg3_update_ans.h */
      double b1 = dot(r, r, n);                          /* cg3_compute_beta.h */
      op_apply(&op, x, Ap);                              /* calc_res_explicit */
      for (size_t i = 0; i < n; ++i) r[i] = b[i] - Ap[i];
      if (o->nullspace) project_mean(r, n);
      res = sqrt(dot(r, r, n));
      double b0 = dot(r, r, n);
      double beta = b0 / b1;
      for (size_t i = 0; i < n; ++i) p[i] = r[i] + beta * p[i]; /* cg3_update_p.h */
      ++iter;
    }
  } else {
    PRECOND(r, z);
    memcpy(p, z, sizeof(double) * n);
    t_iter = wall_s();
    while (res > tol && iter < o->max_iter) {
      op_apply(&op, p, Ap);
      double a0 = dot(r, z, n), a1 = dot(p, Ap, n);  /* cg3_alpha_pre.h */
      double alpha = a0 / a1;
      for (size_t i = 0; i < n; ++i) x[i] += alpha * p[i];
      double b1 = dot(r, z, n);                        /* cg3_compute_beta_pre.h */
      for (size_t i = 0; i < n; ++i) r[i] -= alpha * Ap[i]; /* cg3_update_res.h */
      if (o->nullspace) project_mean(r, n);
      res = sqrt(dot(r, r, n));
      memcpy(zo, z, sizeof(double) * n);
      PRECOND(r, z);
      double b0 = 0.0;                                 /* cg3_compute_beta_pre_flex.h */
      for (size_t i = 0; i < n; ++i) b0 += r[i] * (z[i] - zo[i]);
      double beta = b0 / b1;
      for (size_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
      ++iter;
    }
  }
#undef PRECOND
  info->iters = iter;
  info->abs_res = res;
  info->rel_res = bnorm > 0 ? res / bnorm : res;
  info->converged = res <= tol;
  info->setup_s = t_solve - t_setup;
  info->solve_s = wall_s() - t_solve;
  info->iter_s = iter > 0 ? (wall_s() - t_iter) / iter : 0.0;
  free(r); free(z); free(zo); free(p); free(Ap);
  free(dinv); free(blocks); free(minv);
  if (lv) {
    for (int l = 0; l < nl; ++l) {
      free(lv[l].dinv);
      free(lv[l].binv);
    }
    free(lv);
  }
  if (al) {
    for (int l = 0; l + 1 < o->amg_nlevels; ++l) free(al[l].dinv);
    free(al);
  }
}

/* ------------------------------------------------- velocity projection */
/* Element length scale of the projection penalty: 1 / max over the element's
 * interior faces of fscale (ins_proj_setup_0.h:1-6 accumulates fscale into a
 * zeroed per-face array over interior faces only; ins_proj_setup_1.h:1-7 takes
 * the reciprocal of the maximum). Set-up at src/solvers/3d/ins_solver_base.cpp:201-214
 * (2D: src/solvers/2d/ins_solver_base.cpp:204-217). */
void oracle_proj_h(const oracle_mesh *m, double *h) {
  const int Nf = m->Nf;
  double *fs = (double *)calloc((size_t)m->K * Nf, sizeof(double));
  for (int fc = 0; fc < m->F; ++fc) {
    int eL = m->face2cells[2 * fc], eR = m->face2cells[2 * fc + 1];
    int fL = m->faceNum[2 * fc], fR = m->faceNum[2 * fc + 1];
    fs[IDX(eL, fL, Nf)] += m->fscale[IDX(eL, fL, Nf)];
    fs[IDX(eR, fR, Nf)] += m->fscale[IDX(eR, fR, Nf)];
  }
  for (int e = 0; e < m->K; ++e) {
    double mx = 0.0;
    for (int f = 0; f < Nf; ++f) mx = fmax(mx, fs[IDX(e, f, Nf)]);
    h[e] = 1.0 / mx;
  }
  free(fs);
}

/* One element of the divergence-penalised projection operator
 *   A v = J M v + pen * G^T D^T (J M (D G v)),
 * applied component-wise exactly as ins_3d_proj_cg_precon.h:31-51 writes it:
 * divergence d = Dr (G v)_r + Ds (G v)_s [+ Dt (G v)_t], m = J M d,
 * w_k = Dk^T m, out_c = sum_k G_kc w_k, then out_c <- pen * out_c + J M v_c. */
static void proj_op(int dim, int Np, const double *Dk[3], const double *M, const double G[3][3],
                    double J, double pen, double *const v[3], double *out[3], double *w) {
  double *dv = w, *mv = w + Np, *gv = w + 2 * Np; /* gv: 3 x Np */
  for (int i = 0; i < Np; ++i)
    for (int k = 0; k < dim; ++k) {
      double s = 0.0;
      for (int c = 0; c < dim; ++c) s += G[k][c] * v[c][i];
      gv[k * Np + i] = s;
    }
  for (int i = 0; i < Np; ++i) {
    double d = 0.0;
    for (int k = 0; k < dim; ++k) {
      double s = 0.0;
      for (int j = 0; j < Np; ++j) s += Dk[k][i * Np + j] * gv[k * Np + j];
      d += s;
    }
    dv[i] = d;
  }
  for (int i = 0; i < Np; ++i) {
    double s = 0.0;
    for (int j = 0; j < Np; ++j) s += M[i * Np + j] * dv[j];
    mv[i] = J * s;
  }
  for (int k = 0; k < dim; ++k)
    for (int i = 0; i < Np; ++i) {
      double s = 0.0;
      for (int j = 0; j < Np; ++j) s += Dk[k][j * Np + i] * mv[j];
      gv[k * Np + i] = s;
    }
  for (int c = 0; c < dim; ++c)
    for (int i = 0; i < Np; ++i) {
      double s = 0.0, mm = 0.0;
      for (int k = 0; k < dim; ++k) s += G[k][c] * gv[k * Np + i];
      for (int j = 0; j < Np; ++j) mm += M[i * Np + j] * v[c][j];
      out[c][i] = pen * s + J * mm;
    }
}

/* INSSolverBase3D::project_velocity with pr_projection_method == 1
 * (src/solvers/3d/ins_solver_base.cpp:1052-1124): per element,
 *   velTT = velT - dt * grad p                     (ins_3d_proj_rhs.h:1-13)
 *   b     = J M velTT                              (mesh->mass)
 *   pen   = factor * h / (p + 1)                   (ins_3d_proj_pen.h:24-25)
 *   solve A velTT = b from velTT by CG with the inverse mass matrix (1/J) M^-1
 *   as preconditioner, |r|_2 < 1e-8, at most 100 iterations
 *                                                  (ins_3d_proj_cg_precon.h:1-160).
 * 2D (src/solvers/2d/ins_solver_base.cpp:894-955, ins_proj_cg_2d.h): plain CG,
 * stopping on |r|_2^2 < 1e-16. The caller's factor is dt in 3D and dt * 1e3 in
 * 2D (ins_solver_base.cpp:1082 and 2D :916). stats = {cells, converged cells,
 * iterations summed over cells}; an element counts as converged when it stopped
 * before 100 iterations with a residual that is not NaN. dp, velT, velTT hold
 * dim components one after the other (dim x K x Np). */
void oracle_project_velocity(const oracle_mesh *m, double dt, double factor, const double *dp,
                             const double *velT, double *velTT, double *stats) {
  const int dim = m->dim, Np = m->Np, K = m->K, p = m->order;
  const size_t n = (size_t)K * Np;
  const int precond = dim == 3;
  const double tol = dim == 3 ? 1e-8 : 1e-16;
  const int max_iter = 100;
  const double *Dk[3] = {m->Dr, m->Ds, m->Dt};
  double *minv = (double *)malloc(sizeof(double) * Np * Np);
  memcpy(minv, m->M, sizeof(double) * Np * Np);
  invert_inplace(minv, Np);
  double *h = (double *)malloc(sizeof(double) * K);
  oracle_proj_h(m, h);
  double *buf = (double *)malloc(sizeof(double) * Np * 27);
  double cells = 0.0, conv = 0.0, iters = 0.0;
  for (int e = 0; e < K; ++e) {
    double G[3][3], J;
    geo_unpack(m, e, G, &J);
    const double pen = factor * (h[e] / ((double)p + 1.0));
    double *x[3], *r[3], *z[3], *pp[3], *ap[3], *b[3];
    for (int c = 0; c < 3; ++c) {
      x[c] = buf + (size_t)(c * 6 + 0) * Np; r[c] = buf + (size_t)(c * 6 + 1) * Np;
      z[c] = buf + (size_t)(c * 6 + 2) * Np; pp[c] = buf + (size_t)(c * 6 + 3) * Np;
      ap[c] = buf + (size_t)(c * 6 + 4) * Np; b[c] = buf + (size_t)(c * 6 + 5) * Np;
    }
    double *w = buf + (size_t)18 * Np;
    for (int c = 0; c < dim; ++c)
      for (int i = 0; i < Np; ++i)
        x[c][i] = velT[c * n + IDX(e, i, Np)] - dt * dp[c * n + IDX(e, i, Np)];
    for (int c = 0; c < dim; ++c)
      for (int i = 0; i < Np; ++i) {
        double s = 0.0;
        for (int j = 0; j < Np; ++j) s += m->M[i * Np + j] * x[c][j];
        b[c][i] = J * s;
      }
    proj_op(dim, Np, Dk, m->M, G, J, pen, x, ap, w);
    double res = 0.0;
    for (int c = 0; c < dim; ++c)
      for (int i = 0; i < Np; ++i) {
        r[c][i] = b[c][i] - ap[c][i];
        res += r[c][i] * r[c][i];
      }
    if (precond) res = sqrt(res);
    for (int c = 0; c < dim; ++c)
      for (int i = 0; i < Np; ++i) {
        double s = 0.0;
        if (precond) {
          for (int j = 0; j < Np; ++j) s += minv[i * Np + j] * r[c][j];
          s *= 1.0 / J;
        } else {
          s = r[c][i];
        }
        z[c][i] = s;
        pp[c][i] = s;
      }
    int it = 0;
    while (res > tol && it < max_iter) {
      proj_op(dim, Np, Dk, m->M, G, J, pen, pp, ap, w);
      double rz = 0.0, pap = 0.0;
      for (int c = 0; c < dim; ++c)
        for (int i = 0; i < Np; ++i) { rz += r[c][i] * z[c][i]; pap += pp[c][i] * ap[c][i]; }
      const double alpha = rz / pap;
      res = 0.0;
      for (int c = 0; c < dim; ++c)
        for (int i = 0; i < Np; ++i) {
          x[c][i] += alpha * pp[c][i];
          r[c][i] -= alpha * ap[c][i];
          res += r[c][i] * r[c][i];
        }
      if (precond) res = sqrt(res);
      if (res < tol) break;
      double rz_new = 0.0;
      for (int c = 0; c < dim; ++c)
        for (int i = 0; i < Np; ++i) {
          double s = 0.0;
          if (precond) {
            for (int j = 0; j < Np; ++j) s += minv[i * Np + j] * r[c][j];
            s *= 1.0 / J;
          } else {
            s = r[c][i];
          }
          z[c][i] = s;
          rz_new += r[c][i] * s;
        }
      const double beta = rz_new / rz;
      for (int c = 0; c < dim; ++c)
        for (int i = 0; i < Np; ++i) pp[c][i] = z[c][i] + beta * pp[c][i];
      ++it;
    }
    for (int c = 0; c < dim; ++c)
      for (int i = 0; i < Np; ++i) velTT[c * n + IDX(e, i, Np)] = x[c][i];
    cells += 1.0;
    iters += it;
    if (it < max_iter && !isnan(res)) conv += 1.0;
  }
  stats[0] = cells; stats[1] = conv; stats[2] = iters;
  free(buf); free(h); free(minv);
}

/* DGMesh3D::grad_with_central_flux (unvendored OP2-DG-Toolkit; called at
 * src/solvers/3d/mp_ins_solver.cpp:653 and ins_solver.cpp:361 before
 * project_velocity), restated in strong form with the central flux:
 *   grad_d p = sum_k G[k][d] (D_k p) + LIFT (fscale n_d ({p} - p^-))
 * over interior faces ({p} - p^- = (p^+ - p^-) / 2); a boundary face takes
 * p^+ = p^- and adds nothing. LIFT = M^-1 EMAT. grad holds dim components
 * (dim x K x Np). Parity of this glue with the toolkit is unpinned (the toolkit
 * is not vendored); it is pinned by its properties (exact for continuous
 * polynomials of degree <= p). */
void oracle_grad_central(const oracle_mesh *m, const double *p, double *grad) {
  const int dim = m->dim, Np = m->Np, Nfp = m->Nfp, Nf = m->Nf, K = m->K, NFN = Nf * Nfp;
  const size_t n = (size_t)K * Np;
  const double *Dk[3] = {m->Dr, m->Ds, m->Dt};
  const double *nrm[3] = {m->nx, m->ny, m->nz};
  double *minv = (double *)malloc(sizeof(double) * Np * Np);
  memcpy(minv, m->M, sizeof(double) * Np * Np);
  invert_inplace(minv, Np);
  double *lift = (double *)calloc((size_t)Np * NFN, sizeof(double));
  for (int i = 0; i < Np; ++i)
    for (int c = 0; c < NFN; ++c) {
      double s = 0.0;
      for (int j = 0; j < Np; ++j) s += minv[i * Np + j] * m->EMAT[(size_t)j * NFN + c];
      lift[(size_t)i * NFN + c] = s;
    }
  /* per element face node: (p^+ - p^-) / 2, zero on boundary faces */
  double *jmp = (double *)calloc((size_t)K * NFN, sizeof(double));
  for (int fc = 0; fc < m->F; ++fc) {
    const int eL = m->face2cells[2 * fc], eR = m->face2cells[2 * fc + 1];
    const int fL = m->faceNum[2 * fc], fR = m->faceNum[2 * fc + 1];
    for (int j = 0; j < Nfp; ++j) {
      const int nl = m->fmaskL[fc * Nfp + j], nr = m->fmaskR[fc * Nfp + j];
      const double pl = p[IDX(eL, nl, Np)], pr = p[IDX(eR, nr, Np)];
      jmp[IDX(eL, fL * Nfp + face_pos(m, fL, nl), NFN)] = 0.5 * (pr - pl);
      jmp[IDX(eR, fR * Nfp + face_pos(m, fR, nr), NFN)] = 0.5 * (pl - pr);
    }
  }
  for (int e = 0; e < K; ++e) {
    double G[3][3], J;
    geo_unpack(m, e, G, &J);
    for (int i = 0; i < Np; ++i) {
      double dr[3] = {0, 0, 0};
      for (int k = 0; k < dim; ++k)
        for (int j = 0; j < Np; ++j) dr[k] += Dk[k][i * Np + j] * p[IDX(e, j, Np)];
      for (int d = 0; d < dim; ++d) {
        double s = 0.0;
        for (int k = 0; k < dim; ++k) s += G[k][d] * dr[k];
        for (int f = 0; f < Nf; ++f) {
          const double w = m->fscale[IDX(e, f, Nf)] * nrm[d][IDX(e, f, Nf)];
          double l = 0.0;
          for (int k = 0; k < Nfp; ++k) l += lift[(size_t)i * NFN + f * Nfp + k] * jmp[IDX(e, f * Nfp + k, NFN)];
          s += w * l;
        }
        grad[d * n + IDX(e, i, Np)] = s;
      }
    }
  }
  free(jmp); free(lift); free(minv);
}

/* DGMesh3D::div_with_central_flux (unvendored OP2-DG-Toolkit), restated like
 * the gradient above: div u = sum_d sum_k G[k][d] (D_k u_d) + LIFT (fscale n .
 * (u+ - u-) / 2) over interior faces. u: dim x K x Np; div: K x Np. */
static void div_central(const oracle_mesh *m, const double *u, double *div) {
  const int dim = m->dim, Np = m->Np, K = m->K;
  const size_t n = (size_t)K * Np;
  double *g = (double *)malloc(sizeof(double) * dim * n);
  for (int d = 0; d < dim; ++d) {
    oracle_grad_central(m, u + d * n, g);
    for (size_t i = 0; i < n; ++i) div[i] = (d == 0 ? 0.0 : div[i]) + g[d * n + i];
  }
  free(g);
}

/* Right-hand side of the pressure solve: INSSolver3D::pressure
 * (src/solvers/3d/ins_solver.cpp:313-322): ins_3d_pr_1.h (divVelT *= -1/dt,
 * dPdN_old = b0 dPdN + b1 dPdN_old), then divVelT += LIFT dPdN_old
 * (op2_gemv), then mesh->mass; 2D src/solvers/2d/ins_solver.cpp:309-319
 * (ins_pressure_rhs_2d.h). dPdN, dPdN_old: K x Nf x Nfp or NULL. */
void oracle_pressure_rhs(const oracle_mesh *m, double dt, double b0, double b1, const double *velT,
                         const double *dPdN, double *dPdN_old, double *rhs) {
  const int Np = m->Np, Nf = m->Nf, Nfp = m->Nfp, K = m->K, NFN = Nf * Nfp;
  double *minv = (double *)malloc(sizeof(double) * Np * Np);
  memcpy(minv, m->M, sizeof(double) * Np * Np);
  invert_inplace(minv, Np);
  double *div = (double *)malloc(sizeof(double) * (size_t)K * Np);
  double *dn = (double *)calloc(NFN, sizeof(double));
  div_central(m, velT, div);
  const double factor = 1.0 / dt;
  for (int e = 0; e < K; ++e) {
    double G[3][3], J, pre[64];
    geo_unpack(m, e, G, &J);
    for (int c = 0; c < NFN; ++c) {
      const size_t fi = (size_t)e * NFN + c;
      dn[c] = (dPdN ? b0 * dPdN[fi] : 0.0) + (dPdN_old ? b1 * dPdN_old[fi] : 0.0);
      if (dPdN_old) dPdN_old[fi] = dn[c];
    }
    for (int i = 0; i < Np; ++i) {
      double l = 0.0;
      for (int c = 0; c < NFN; ++c) {
        double lift = 0.0;
        for (int j = 0; j < Np; ++j) lift += minv[i * Np + j] * m->EMAT[(size_t)j * NFN + c];
        l += lift * dn[c];
      }
      pre[i] = -div[IDX(e, i, Np)] * factor + l;
    }
    for (int i = 0; i < Np; ++i) {
      double s = 0.0;
      for (int j = 0; j < Np; ++j) s += m->M[i * Np + j] * pre[j];
      rhs[IDX(e, i, Np)] = J * s;
    }
  }
  free(dn); free(div); free(minv);
}
