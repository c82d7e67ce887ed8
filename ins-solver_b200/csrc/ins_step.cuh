// Device entry points of the 3D incompressible time step around the solves
// (ins_step.cu), used by the time-step driver (ins3d.cu).
#pragma once
#include <cuda_runtime.h>

#include "runtime.hpp"

namespace sipg {

// Non-linear advection and the extrapolated velocity; grav: body force -grav along y
// (0 for the reference's 3D solver).
void advection_device(sipg_mesh* m, int order, double dt, double a0, double a1, double b0, double b1, double grav,
                      const double* u, const double* u_old, const double* N_old, const int* vel_bc, double* N,
                      double* velT, cudaStream_t s);

// Curl-curl Neumann data of the pressure step (K x 4 x Nfp; zeroed first).
void pressure_neumann_device(sipg_mesh* m, int order, double reynolds, double grav, const double* u,
                             const double* N, const double* mu, const double* rho, const int* vel_bc, double* dPdN,
                             cudaStream_t s);

// Level-set fields: s is advanced in place through the stage buffers qa, qb and the
// stage derivatives rk0, rk1 (all K x Np); rho, mu, rrho = 1 / rho follow s.
struct LsFields {
  const double* u;  // velocity, 3 x K x Np
  double *s, *qa, *qb, *rk0, *rk1;
  double *rho, *mu, *rrho;
  unsigned long long* vmax;  // bits of max |u|^2 (device scalar), or null
  double alpha, rho0, rho1, mu0, mu1;
};

// One level-set advection step (three stages) followed by rho, mu and 1 / rho.
void ls_step_device(sipg_mesh* m, int order, double dt, const LsFields& f, cudaStream_t s);
// rho, mu, 1 / rho from s and max |u|^2 alone.
void ls_props_device(sipg_mesh* m, int order, const LsFields& f, cudaStream_t s);

// Work buffers of the level-set reinitialisation, kept across calls.
struct ReinitWork {
  DevBuf cells, count, samples, nearest, s_old, kept, flat;
};

// Closest-point reinitialisation of s (K x Np, in place): xyz the node coordinates
// (3 x K x Np), h the level set's length (1 / the smallest interior-face fscale),
// values clamped to +-ls_cap.
void ls_reinit_device(sipg_mesh* m, int order, const double* xyz, double* s, double h, double ls_cap,
                      ReinitWork& w, cudaStream_t st);

}  // namespace sipg
