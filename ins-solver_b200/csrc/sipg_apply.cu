// Fused SIPG apply kernel and penalty kernel. See sipg_apply.cuh for the
// phase structure and the reference routines each phase replaces.
#include "sipg_apply.cuh"
#include "vecops.cuh"

#include <algorithm>

namespace sipg {

namespace {

// Outward face normal direction (unnormalised) of face f from the inverse
// Jacobian G[r][d] = d r_r / d x_d: 3D faces t=-1, s=-1, r+s+t=-1, r=-1;
// 2D faces s=-1, r+s=0, r=-1.
template <int DIM, typename T>
__device__ __forceinline__ void face_normal(const T* g, int f, T n[3], T* sJ) {
  if (DIM == 3) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      T v;
      if (f == 0) v = -g[6 + d];
      else if (f == 1) v = -g[3 + d];
      else if (f == 2) v = (g[d] + g[3 + d]) + g[6 + d];
      else v = -g[d];
      n[d] = v;
    }
    T len = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    n[0] /= len; n[1] /= len; n[2] /= len;
    *sJ = len * g[9];
  } else {
#pragma unroll
    for (int d = 0; d < 2; ++d) {
      T v;
      if (f == 0) v = -g[2 + d];
      else if (f == 1) v = g[d] + g[2 + d];
      else v = -g[d];
      n[d] = v;
    }
    n[2] = T(0);
    T len = sqrt(n[0] * n[0] + n[1] * n[1]);
    n[0] /= len; n[1] /= len;
    *sJ = len * g[4];
  }
}

template <int DIM, typename T>
__device__ __forceinline__ T geo_G(const T* g, int r, int d) { return g[r * DIM + d]; }
template <int DIM, typename T>
__device__ __forceinline__ T geo_J(const T* g) { return g[DIM == 3 ? 9 : 4]; }

// Per-element shared-memory layout (units of T), one batch of `eb` elements.
template <int DIM, int P>
struct ElemLayout {
  using C = Cfg<DIM, P>;
  int nc;
  int u, unb, q, fu, ft, w, fac, facnb, geo, tau, size;
  __device__ __host__ ElemLayout(int ncomp) : nc(ncomp) {
    int o = 0;
    u = o; o += nc * C::NP;
    unb = o; o += nc * C::NF * C::NP;      // neighbour x; reused as W after P2
    q = o; o += nc * DIM * C::NP;
    fu = o; o += nc * C::NFNFP;            // neighbour n.q+ in P1, then Fu
    ft = o; o += nc * DIM * C::NFNFP;
    fac = o; o += C::NP;
    facnb = o; o += C::NFNFP;
    geo = o; o += C::NG * (1 + C::NF);
    tau = o; o += C::NF;
    w = unb;
    size = o;
  }
};

template <typename T, int DIM, int P>
__global__ void __launch_bounds__(256) sipg_apply_kernel(ApplyArgs<T> a) {
  using C = Cfg<DIM, P>;
  constexpr int NP = C::NP, NFP = C::NFP, NF = C::NF, NFNFP = C::NFNFP, LD = C::LD,
                LDE = C::LDE, NG = C::NG;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* cst = reinterpret_cast<T*>(smem_raw);
  const ElemLayout<DIM, P> L(a.ncomp);
  const int eb = a.eb, nc = a.ncomp;
  T* eb_base = cst + C::CONST_T;
  int* ib = reinterpret_cast<int*>(eb_base + (size_t)eb * L.size);  // nbr[eb][NF], code[eb][NF]
  int8_t* itab = reinterpret_cast<int8_t*>(ib + 2 * eb * NF);
  const T* Dm = cst + C::OFF_D;
  const T* Mm = cst + C::OFF_M;
  const T* Em = cst + C::OFF_E;
  const int8_t* fmask = itab;
  const int8_t* perm = itab + NF * NFP;

  for (int i = threadIdx.x; i < C::CONST_T; i += blockDim.x) cst[i] = a.consts[i];
  for (int i = threadIdx.x; i < C::ITAB; i += blockDim.x) itab[i] = a.itab[i];

  const int nbatch = (a.K + eb - 1) / eb;
  for (int batch = blockIdx.x; batch < nbatch; batch += gridDim.x) {
    const int e0 = batch * eb;
    const int ne = min(eb, a.K - e0);
    __syncthreads();
    // ---------------- P0: stage
    for (int i = threadIdx.x; i < ne * NF; i += blockDim.x) {
      int le = i / NF, f = i % NF;
      int e = e0 + le;
      ib[le * NF + f] = a.nbr[(size_t)e * NF + f];
      ib[eb * NF + le * NF + f] = (a.fcode[e] >> (8 * f)) & 0xff;
      eb_base[le * L.size + L.tau + f] = a.tau[(size_t)e * NF + f];
    }
    for (int i = threadIdx.x; i < ne * NG; i += blockDim.x) {
      int le = i / NG, k = i % NG;
      eb_base[le * L.size + L.geo + k] = a.geof[(size_t)(e0 + le) * NG + k];
    }
    for (int i = threadIdx.x; i < nc * ne * NP; i += blockDim.x) {
      int c = i / (ne * NP), r = i % (ne * NP);
      int le = r / NP, m = r % NP;
      int e = e0 + le;
      T v = a.x[((size_t)c * a.K + e) * NP + m];
      if (e == a.pin_elem && m == a.pin_node) v = T(0);
      eb_base[le * L.size + L.u + c * NP + m] = v;
    }
    for (int i = threadIdx.x; i < ne * NP; i += blockDim.x) {
      int le = i / NP, m = i % NP;
      eb_base[le * L.size + L.fac + m] = a.factor ? a.factor[(size_t)(e0 + le) * NP + m] : T(1);
    }
    __syncthreads();
    // neighbour data: x (all nodes), geometry, factor at the matched face nodes
    for (int i = threadIdx.x; i < ne * NF * NP * nc; i += blockDim.x) {
      int c = i / (ne * NF * NP), r = i % (ne * NF * NP);
      int lf = r / NP, m = r % NP;
      int le = lf / NF, f = lf % NF;
      int nb = ib[le * NF + f];
      T v = T(0);
      if (nb >= 0) {
        v = a.x[((size_t)c * a.K + nb) * NP + m];
        if (nb == a.pin_elem && m == a.pin_node) v = T(0);
      }
      eb_base[le * L.size + L.unb + (c * NF + f) * NP + m] = v;
    }
    for (int i = threadIdx.x; i < ne * NF * NG; i += blockDim.x) {
      int lf = i / NG, k = i % NG;
      int le = lf / NF, f = lf % NF;
      int nb = ib[le * NF + f];
      eb_base[le * L.size + L.geo + NG * (1 + f) + k] = nb >= 0 ? a.geof[(size_t)nb * NG + k] : T(0);
    }
    for (int i = threadIdx.x; i < ne * NFNFP; i += blockDim.x) {
      int le = i / NFNFP, k = i % NFNFP;
      int f = k / NFP, j = k % NFP;
      int nb = ib[le * NF + f];
      T v = T(1);
      if (nb >= 0 && a.factor) {
        int code = ib[eb * NF + le * NF + f];
        int nm = fmask[(code & 3) * NFP + perm[(code >> 2) * NFP + j]];
        v = a.factor[(size_t)nb * NP + nm];
      }
      eb_base[le * L.size + L.facnb + k] = v;
    }
    __syncthreads();
    // ---------------- P1: own gradient and neighbour normal flux
    for (int i = threadIdx.x; i < ne * nc * NP; i += blockDim.x) {
      int le = i / (nc * NP), r = i % (nc * NP);
      int c = r / NP, m = r % NP;
      T* E = eb_base + le * L.size;
      const T* u = E + L.u + c * NP;
      T gr[3] = {T(0), T(0), T(0)};
#pragma unroll 5
      for (int n = 0; n < NP; ++n) {
        T un = u[n];
#pragma unroll
        for (int d = 0; d < DIM; ++d) gr[d] += Dm[d * NP * LD + m * LD + n] * un;
      }
      const T* g = E + L.geo;
      T f = E[L.fac + m];
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        T s = T(0);
#pragma unroll
        for (int rr = 0; rr < DIM; ++rr) s += geo_G<DIM>(g, rr, d) * gr[rr];
        E[L.q + (c * DIM + d) * NP + m] = f * s;
      }
    }
    for (int i = threadIdx.x; i < ne * nc * NFNFP; i += blockDim.x) {
      int le = i / (nc * NFNFP), r = i % (nc * NFNFP);
      int c = r / NFNFP, k = r % NFNFP;
      int f = k / NFP, j = k % NFP;
      T* E = eb_base + le * L.size;
      int nb = ib[le * NF + f];
      T val = T(0);
      if (nb >= 0) {
        int code = ib[eb * NF + le * NF + f];
        int nm = fmask[(code & 3) * NFP + perm[(code >> 2) * NFP + j]];
        const T* un = E + L.unb + (c * NF + f) * NP;
        T gr[3] = {T(0), T(0), T(0)};
#pragma unroll 5
        for (int n = 0; n < NP; ++n) {
          T v = un[n];
#pragma unroll
          for (int d = 0; d < DIM; ++d) gr[d] += Dm[d * NP * LD + nm * LD + n] * v;
        }
        const T* gn = E + L.geo + NG * (1 + f);
        T n[3], sJ;
        face_normal<DIM>(E + L.geo, f, n, &sJ);
        T fn = E[L.facnb + k];
        T s = T(0);
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
          T qd = T(0);
#pragma unroll
          for (int rr = 0; rr < DIM; ++rr) qd += geo_G<DIM>(gn, rr, d) * gr[rr];
          s += n[d] * (fn * qd);
        }
        val = s;
      }
      E[L.fu + c * NFNFP + k] = val;  // n^- . q^+ (interior) ; overwritten by Fu in P2
    }
    __syncthreads();
    // ---------------- P2: face fluxes
    for (int i = threadIdx.x; i < ne * NFNFP; i += blockDim.x) {
      int le = i / NFNFP, k = i % NFNFP;
      int f = k / NFP, j = k % NFP;
      T* E = eb_base + le * L.size;
      const T* g = E + L.geo;
      T n[3], sJ;
      face_normal<DIM>(g, f, n, &sJ);
      const int m = fmask[f * NFP + j];
      const int nb = ib[le * NF + f];
      const T tau = E[L.tau + f];
      const T fm = E[L.fac + m];
      T jump[3], navg[3];
      if (nb >= 0) {
        int code = ib[eb * NF + le * NF + f];
        int nm = fmask[(code & 3) * NFP + perm[(code >> 2) * NFP + j]];
        for (int c = 0; c < nc; ++c) {
          T um = E[L.u + c * NP + m], up = E[L.unb + (c * NF + f) * NP + nm];
          jump[c] = um - up;
          T nq = T(0);
#pragma unroll
          for (int d = 0; d < DIM; ++d) nq += n[d] * E[L.q + (c * DIM + d) * NP + m];
          navg[c] = T(0.5) * (nq + E[L.fu + c * NFNFP + k]);
        }
      } else {
        const int b = -nb - 1;
        bool all_slip = nc == DIM;
        for (int c = 0; c < nc; ++c) all_slip = all_slip && a.bct[(size_t)c * a.Kb + b] == BC_SLIP;
        if (all_slip) {
          // vmf_3d_mult_avg_jump.h:9-41: normal projections of x and q
          T un = T(0), nqn = T(0);
          for (int c = 0; c < nc; ++c) {
            un += n[c] * E[L.u + c * NP + m];
            T nq = T(0);
#pragma unroll
            for (int d = 0; d < DIM; ++d) nq += n[d] * E[L.q + (c * DIM + d) * NP + m];
            nqn += n[c] * nq;
          }
          for (int c = 0; c < nc; ++c) {
            jump[c] = T(2) * n[c] * un;
            navg[c] = n[c] * nqn;
          }
        } else {
          for (int c = 0; c < nc; ++c) {
            int t = a.bct[(size_t)c * a.Kb + b];
            if (t == BC_DIRICHLET) {
              jump[c] = T(2) * E[L.u + c * NP + m];
              T nq = T(0);
#pragma unroll
              for (int d = 0; d < DIM; ++d) nq += n[d] * E[L.q + (c * DIM + d) * NP + m];
              navg[c] = nq;
            } else {
              jump[c] = T(0);
              navg[c] = T(0);
            }
          }
        }
      }
      // fvmf_3d_mult_flux.h:13-22; lifted q fluxes pre-transformed by G
      for (int c = 0; c < nc; ++c) {
        T hj = T(0.5) * jump[c];
        E[L.fu + c * NFNFP + k] = sJ * (tau * hj - navg[c]);
        T fq[3];
#pragma unroll
        for (int d = 0; d < DIM; ++d) fq[d] = n[d] * sJ * fm * -hj;
#pragma unroll
        for (int rr = 0; rr < DIM; ++rr) {
          T s = T(0);
#pragma unroll
          for (int d = 0; d < DIM; ++d) s += geo_G<DIM>(g, rr, d) * fq[d];
          E[L.ft + (c * DIM + rr) * NFNFP + k] = s;
        }
      }
    }
    __syncthreads();
    // ---------------- P3: q~_r = J sum_d G[r][d] q_d (in place, per node)
    for (int i = threadIdx.x; i < ne * nc * NP; i += blockDim.x) {
      int le = i / (nc * NP), r = i % (nc * NP);
      int c = r / NP, m = r % NP;
      T* E = eb_base + le * L.size;
      const T* g = E + L.geo;
      T J = geo_J<DIM>(g);
      T qd[3];
#pragma unroll
      for (int d = 0; d < DIM; ++d) qd[d] = E[L.q + (c * DIM + d) * NP + m];
#pragma unroll
      for (int rr = 0; rr < DIM; ++rr) {
        T s = T(0);
#pragma unroll
        for (int d = 0; d < DIM; ++d) s += geo_G<DIM>(g, rr, d) * qd[d];
        E[L.q + (c * DIM + rr) * NP + m] = J * s;
      }
    }
    __syncthreads();
    // ---------------- P4: W_r = M q~_r + EMAT Ft_r
    for (int i = threadIdx.x; i < ne * nc * NP; i += blockDim.x) {
      int le = i / (nc * NP), r = i % (nc * NP);
      int c = r / NP, m = r % NP;
      T* E = eb_base + le * L.size;
      T acc[3] = {T(0), T(0), T(0)};
#pragma unroll 5
      for (int n = 0; n < NP; ++n) {
        T mv = Mm[m * LD + n];
#pragma unroll
        for (int rr = 0; rr < DIM; ++rr) acc[rr] += mv * E[L.q + (c * DIM + rr) * NP + n];
      }
#pragma unroll 4
      for (int kk = 0; kk < NFNFP; ++kk) {
        T ev = Em[m * LDE + kk];
#pragma unroll
        for (int rr = 0; rr < DIM; ++rr) acc[rr] += ev * E[L.ft + (c * DIM + rr) * NFNFP + kk];
      }
#pragma unroll
      for (int rr = 0; rr < DIM; ++rr) E[L.w + (c * DIM + rr) * NP + m] = acc[rr];
    }
    __syncthreads();
    // ---------------- P5: y = EMAT Fu + sum_r D_r^T W_r + J M (mm x)
    for (int i = threadIdx.x; i < nc * ne * NP; i += blockDim.x) {
      int c = i / (ne * NP), r = i % (ne * NP);
      int le = r / NP, m = r % NP;
      T* E = eb_base + le * L.size;
      T acc = T(0);
#pragma unroll 4
      for (int kk = 0; kk < NFNFP; ++kk) acc += Em[m * LDE + kk] * E[L.fu + c * NFNFP + kk];
#pragma unroll 5
      for (int n = 0; n < NP; ++n) {
#pragma unroll
        for (int rr = 0; rr < DIM; ++rr) acc += Dm[rr * NP * LD + n * LD + m] * E[L.w + (c * DIM + rr) * NP + n];
      }
      const int e = e0 + le;
      if (a.mm_mode != MM_NONE) {
        T s = T(0);
        for (int n = 0; n < NP; ++n) {
          T mmv = a.mm_mode == MM_SCALAR ? a.mm_scalar : a.mm[(size_t)e * NP + n];
          s += mmv * Mm[m * LD + n] * E[L.u + c * NP + n];
        }
        acc += s * geo_J<DIM>(E + L.geo);
      }
      if (e == a.pin_elem && m == a.pin_node) acc = a.pin_scale * a.x[((size_t)c * a.K + e) * NP + m];
      const size_t yi = ((size_t)c * a.K + e) * NP + m;
      acc *= a.alpha;
      if (a.beta != T(0)) acc += a.beta * a.c[yi];
      a.y[yi] = acc;
    }
  }
}

// Penalty per element face: interior 2(p+1)(p+2) max_j max(fs- f-, fs+ f+),
// boundary 2(p+1)(p+2) fs max_j f (fvmf_3d_calc_tau_faces.h:3-13,
// fvmf_3d_calc_tau_bfaces.h:3-11). fscale = sJ / J.
template <typename T, int DIM, int P>
__global__ void sipg_tau_kernel(const int8_t* itab, const T* geof, const int* nbr,
                                const uint32_t* fcode, const T* factor, int K, T* tau) {
  using C = Cfg<DIM, P>;
  constexpr int NP = C::NP, NFP = C::NFP, NF = C::NF, NG = C::NG;
  const int8_t* fmask = itab;
  const int8_t* perm = itab + NF * NFP;
  const T c = T(2 * (P + 1) * (P + 2));
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < K * NF; i += gridDim.x * blockDim.x) {
    int e = i / NF, f = i % NF;
    const T* g = geof + (size_t)e * NG;
    T n[3], sJ;
    face_normal<DIM>(g, f, n, &sJ);
    T fs = sJ / geo_J<DIM>(g);
    int nb = nbr[i];
    T gt = T(0);
    if (nb >= 0) {
      int code = (fcode[e] >> (8 * f)) & 0xff;
      int fr = code & 3, sg = code >> 2;
      T fsr = fs * geo_J<DIM>(g) / geo_J<DIM>(geof + (size_t)nb * NG);  // sJ is shared by both sides
      for (int j = 0; j < NFP; ++j) {
        T fl = factor ? factor[(size_t)e * NP + fmask[f * NFP + j]] : T(1);
        T frv = factor ? factor[(size_t)nb * NP + fmask[fr * NFP + perm[sg * NFP + j]]] : T(1);
        gt = max(gt, c * max(fs * fl, fsr * frv));
      }
    } else {
      T fmx = factor ? factor[(size_t)e * NP + fmask[f * NFP]] : T(1);
      for (int j = 1; j < NFP; ++j)
        if (factor) fmx = max(fmx, factor[(size_t)e * NP + fmask[f * NFP + j]]);
      gt = fmx * c * fs;
    }
    tau[i] = gt;
  }
}

// Slip faces of the vector operator (every component of a boundary face of type 2,
// vmf_3d_mult_avg_jump.h:9-41): the face terms that couple the components,
//   un = n . u,  nqn = sum_c n_c (n . f grad u_c)  at each face node,
//   Fu_c = sJ (tau n_c un - n_c nqn),  Fq_(c,d) = -n_d sJ f n_c un,
// lifted as y_c += EMAT Fu_c + sum_r D_r^T EMAT (G Fq_c)_r. Added (times alpha) to
// per-component scalar applies, which give a slip face no face terms. One CTA per
// element that owns a boundary face.
template <typename T, int DIM, int P>
__global__ void __launch_bounds__(128) sipg_slip_kernel(ApplyArgs<T> a, const int* __restrict__ belems,
                                                        int n_belem) {
  using C = Cfg<DIM, P>;
  constexpr int NP = C::NP, NFP = C::NFP, NF = C::NF, NFNFP = C::NFNFP, LD = C::LD, LDE = C::LDE, NG = C::NG;
  __shared__ T u[DIM][NP], fac[NP], g[NG], W[DIM][DIM][NP];
  __shared__ T fu[DIM][NFNFP], ft[DIM][DIM][NFNFP];
  __shared__ int slipf[NF];
  const T* Dm = a.consts + C::OFF_D;
  const T* Em = a.consts + C::OFF_E;
  const int8_t* fmask = a.itab;
  const size_t K = (size_t)a.K;
  for (int it = blockIdx.x; it < n_belem; it += gridDim.x) {
    const int e = belems[it];
    __syncthreads();
    if (threadIdx.x < NF) {
      const int nb = a.nbr[(size_t)e * NF + threadIdx.x];
      int sl = 0;
      if (nb < 0) {
        sl = 1;
        for (int c = 0; c < DIM; ++c) sl &= a.bct[(size_t)c * a.Kb + (-nb - 1)] == BC_SLIP;
      }
      slipf[threadIdx.x] = sl;
    }
    for (int i = threadIdx.x; i < DIM * NP; i += blockDim.x) u[i / NP][i % NP] = a.x[((size_t)(i / NP) * K + e) * NP + i % NP];
    for (int i = threadIdx.x; i < NP; i += blockDim.x) fac[i] = a.factor ? a.factor[(size_t)e * NP + i] : T(1);
    for (int i = threadIdx.x; i < NG; i += blockDim.x) g[i] = a.geof[(size_t)e * NG + i];
    __syncthreads();
    bool any = false;
    for (int f = 0; f < NF; ++f) any |= slipf[f] != 0;
    if (!any) continue;
    for (int k = threadIdx.x; k < NFNFP; k += blockDim.x) {
      const int f = k / NFP, j = k - (k / NFP) * NFP;
      if (!slipf[f]) {
        for (int c = 0; c < DIM; ++c) {
          fu[c][k] = T(0);
          for (int r = 0; r < DIM; ++r) ft[c][r][k] = T(0);
        }
        continue;
      }
      const int m = fmask[f * NFP + j];
      T n[3], sJ;
      face_normal<DIM>(g, f, n, &sJ);
      const T tau = a.tau[(size_t)e * NF + f];
      T un = T(0), nqn = T(0);
      for (int c = 0; c < DIM; ++c) {
        T gr[3] = {T(0), T(0), T(0)};
        for (int q = 0; q < NP; ++q)
          for (int r = 0; r < DIM; ++r) gr[r] += Dm[r * NP * LD + m * LD + q] * u[c][q];
        T nq = T(0);
        for (int d = 0; d < DIM; ++d) {
          T qd = T(0);
          for (int r = 0; r < DIM; ++r) qd += geo_G<DIM>(g, r, d) * gr[r];
          nq += n[d] * qd;
        }
        un += n[c] * u[c][m];
        nqn += n[c] * (fac[m] * nq);
      }
      for (int c = 0; c < DIM; ++c) {
        fu[c][k] = sJ * (tau * n[c] * un - n[c] * nqn);
        for (int r = 0; r < DIM; ++r) {
          T s2 = T(0);
          for (int d = 0; d < DIM; ++d) s2 += geo_G<DIM>(g, r, d) * (-n[d] * sJ * fac[m] * n[c] * un);
          ft[c][r][k] = s2;
        }
      }
    }
    __syncthreads();
    // W_(c,r) = EMAT ft_(c,r)
    for (int t = threadIdx.x; t < DIM * DIM * NP; t += blockDim.x) {
      const int c = t / (DIM * NP), r = (t / NP) % DIM, q = t % NP;
      T s2 = T(0);
      for (int k = 0; k < NFNFP; ++k) s2 += Em[q * LDE + k] * ft[c][r][k];
      W[c][r][q] = s2;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < DIM * NP; t += blockDim.x) {
      const int c = t / NP, i = t % NP;
      T acc = T(0);
      for (int k = 0; k < NFNFP; ++k) acc += Em[i * LDE + k] * fu[c][k];
      for (int r = 0; r < DIM; ++r)
        for (int q = 0; q < NP; ++q) acc += Dm[r * NP * LD + q * LD + i] * W[c][r][q];
      a.y[((size_t)c * K + e) * NP + i] += a.alpha * acc;
    }
  }
}

template <typename T, int DIM, int P>
cudaError_t launch_slip_t(const ApplyArgs<T>& a, const int* belems, int n_belem, cudaStream_t s) {
  if (n_belem <= 0) return cudaSuccess;
  const int grid = std::max(1, std::min(n_belem, 148 * 16));
  sipg_slip_kernel<T, DIM, P><<<grid, 128, 0, s>>>(a, belems, n_belem);
  note_launch();
  return cudaGetLastError();
}

template <typename T, int DIM, int P>
cudaError_t launch_apply_t(const ApplyArgs<T>& a, int num_sms, cudaStream_t s) {
  using C = Cfg<DIM, P>;
  const ElemLayout<DIM, P> L(a.ncomp);
  size_t bytes = (size_t)(C::CONST_T + a.eb * L.size) * sizeof(T) + 2 * a.eb * C::NF * sizeof(int) + C::ITAB;
  auto k = sipg_apply_kernel<T, DIM, P>;
  cudaError_t err = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (err != cudaSuccess) return err;
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 256, bytes);
  per_sm = std::max(per_sm, 1);
  int nbatch = (a.K + a.eb - 1) / a.eb;
  int grid = std::min(nbatch, num_sms * per_sm);
  if (grid <= 0) return cudaSuccess;
  k<<<grid, 256, bytes, s>>>(a);
  note_launch();
  return cudaGetLastError();
}

template <typename T, int DIM, int P>
cudaError_t launch_tau_t(const int8_t* itab, const T* geof, const int* nbr, const uint32_t* fcode,
                         const T* factor, int K, T* tau, cudaStream_t s) {
  int n = K * (DIM + 1);
  int grid = std::max(1, std::min((n + 255) / 256, 148 * 8));
  sipg_tau_kernel<T, DIM, P><<<grid, 256, 0, s>>>(itab, geof, nbr, fcode, factor, K, tau);
  note_launch();
  return cudaGetLastError();
}

template <int DIM, int P>
size_t smem_bytes_t(int ncomp, int eb, bool fp64) {
  using C = Cfg<DIM, P>;
  const ElemLayout<DIM, P> L(ncomp);
  size_t ts = fp64 ? 8 : 4;
  return (size_t)(C::CONST_T + eb * L.size) * ts + 2 * eb * C::NF * sizeof(int) + C::ITAB;
}

}  // namespace

#define SIPG_DISPATCH(DIM_, ORDER_, ...)                                  \
  switch ((DIM_) * 10 + (ORDER_)) {                                       \
    case 21: { constexpr int D = 2, P = 1; __VA_ARGS__; }                        \
    case 22: { constexpr int D = 2, P = 2; __VA_ARGS__; }                        \
    case 23: { constexpr int D = 2, P = 3; __VA_ARGS__; }                        \
    case 24: { constexpr int D = 2, P = 4; __VA_ARGS__; }                        \
    case 31: { constexpr int D = 3, P = 1; __VA_ARGS__; }                        \
    case 32: { constexpr int D = 3, P = 2; __VA_ARGS__; }                        \
    case 33: { constexpr int D = 3, P = 3; __VA_ARGS__; }                        \
    case 34: { constexpr int D = 3, P = 4; __VA_ARGS__; }                        \
    default: break;                                                       \
  }

template <typename T>
cudaError_t launch_apply(int dim, int order, const ApplyArgs<T>& a, int num_sms, cudaStream_t s) {
  SIPG_DISPATCH(dim, order, return (launch_apply_t<T, D, P>(a, num_sms, s)));
  return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t launch_slip(int dim, int order, const ApplyArgs<T>& a, const int* belems, int n_belem, cudaStream_t s) {
  SIPG_DISPATCH(dim, order, return (launch_slip_t<T, D, P>(a, belems, n_belem, s)));
  return cudaErrorInvalidValue;
}

size_t apply_smem_bytes(int dim, int order, int ncomp, int eb, bool fp64) {
  SIPG_DISPATCH(dim, order, return smem_bytes_t<D, P>(ncomp, eb, fp64));
  return 0;
}

int apply_pick_eb(int dim, int order, int ncomp, bool fp64) {
  // Largest batch that keeps two CTAs per SM within 227 KB, else one CTA.
  const size_t limit2 = 113 * 1024, limit1 = 227 * 1024;
  int best = 0;
  for (int eb = 1; eb <= 64; ++eb)
    if (apply_smem_bytes(dim, order, ncomp, eb, fp64) <= limit2) best = eb;
  if (best >= 4) return std::min(best, 32);
  for (int eb = 1; eb <= 64; ++eb)
    if (apply_smem_bytes(dim, order, ncomp, eb, fp64) <= limit1) best = eb;
  return std::max(1, std::min(best, 32));
}

template <typename T>
cudaError_t launch_tau(int dim, int order, const int8_t* itab, const T* geof, const int* nbr,
                       const uint32_t* fcode, const T* factor, int K, T* tau, cudaStream_t s) {
  SIPG_DISPATCH(dim, order, return (launch_tau_t<T, D, P>(itab, geof, nbr, fcode, factor, K, tau, s)));
  return cudaErrorInvalidValue;
}

template cudaError_t launch_apply<double>(int, int, const ApplyArgs<double>&, int, cudaStream_t);
template cudaError_t launch_apply<float>(int, int, const ApplyArgs<float>&, int, cudaStream_t);
template cudaError_t launch_slip<double>(int, int, const ApplyArgs<double>&, const int*, int, cudaStream_t);
template cudaError_t launch_slip<float>(int, int, const ApplyArgs<float>&, const int*, int, cudaStream_t);
template cudaError_t launch_tau<double>(int, int, const int8_t*, const double*, const int*,
                                        const uint32_t*, const double*, int, double*, cudaStream_t);
template cudaError_t launch_tau<float>(int, int, const int8_t*, const float*, const int*,
                                       const uint32_t*, const float*, int, float*, cudaStream_t);

}  // namespace sipg
