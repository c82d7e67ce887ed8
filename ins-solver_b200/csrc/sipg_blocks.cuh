// Element block kernels: diagonal, diagonal blocks, block inverses, boundary lifting.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "sipg_apply.cuh"

namespace sipg {

enum BlockMode : int { BLOCK_DIAG_ONLY = 0, BLOCK_FULL = 1, BLOCK_INVERSE = 2 };

struct BlockArgs {
  const double* consts;   // Cfg constant blob (FP64)
  const int8_t* itab;     // fmask first
  const double* mf;       // Nf x Nfp x Nfp face mass (face-node ordering)
  const double* geof;
  const int* nbr;
  const double* tau;
  const double* factor;   // may be null
  int mm_mode;
  double mm_scalar;
  const double* mm;
  const uint8_t* bct;
  int Kb, K, ncomp;
  int ref_volume;         // reproduce the reference's block formulas
  int pin_elem, pin_node;
  double pin_scale;
  int mode;               // BlockMode
  double* out;            // ncomp x K x (Np | Np*Np)
};

struct ApplyBcArgs {
  const double* consts;
  const int8_t* itab;
  const double* mf;
  const double* geof;
  const int* nbr;
  const double* tau;
  const double* factor;
  const uint8_t* bct;
  int Kb, K, ncomp;
  const int* belems;      // elements owning boundary faces
  int n_belem;
  const double* bc;       // ncomp x Kb x Nfp
  double* rhs;            // ncomp x K x Np (+=)
};

cudaError_t launch_blocks(int dim, int order, const BlockArgs& a, cudaStream_t s);
cudaError_t launch_apply_bc(int dim, int order, const ApplyBcArgs& a, cudaStream_t s);

}  // namespace sipg
