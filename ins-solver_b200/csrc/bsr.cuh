// Element-block (block-sparse) form of a low-order SIPG operator.
//
// At p = 1 the matrix-free apply spends most of its time on per-element
// overheads (face geometry, traces, two launches) while the operator itself is
// small: an element row couples to itself and to its face neighbours only, in
// Np x Np blocks (4 x 4 for tetrahedra at p = 1). The p-multigrid applies such
// a level's operator eight times per V-cycle, so the levels at or below a
// chosen order store these blocks once and apply them as a block-sparse
// product (one thread per element row, coalesced block reads).
//
// The blocks are computed in FP64 by one kernel straight from the terms of the
// matrix-free apply (volume, face fluxes with the neighbour's factor and
// geometry, mass, pinned row), a thread per element row.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "runtime.hpp"

namespace sipg {

struct BsrOp {
  int K = 0, Np = 0, NF = 0, dim = 0;
  // values[((s * Np + r) * Np + c) * K + e]: block s of element row e, s = 0 the
  // element itself, s = 1 + f the neighbour across face f (zero at boundary faces)
  DevBuf v64, v32;
  // FP32 V-cycle, even Np: FP16 values scaled per element (10-bit mantissa like
  // the TF32 matrix-free apply, half the bytes of FP32) in the layout
  // v16[((s * Np + c) * K + e) * Np + r] = values / scale16[e], so that the Np
  // threads of an element row block read consecutive values
  DevBuf v16, scale16;
  // Block-Jacobi preconditioned blocks C = Bd^-1 A (Bd the diagonal block of the
  // element row), same layout and scaling as v16: one kernel per Chebyshev step
  // (k_bsr16_cheb) then updates the preconditioned residual directly
  DevBuf c16, cscale16;
  DevBuf c64;  // assembly workspace, kept for the next set-up
  const int* nbr = nullptr;  // mesh K x NF (device)
};

// Orders whose element blocks have an assembled apply (Np x Np registers per thread).
inline bool bsr_supported(int dim, int order, int ncomp) { return ncomp == 1 && order >= 1 && order <= 2 && dim >= 2; }

// Element-row blocks of a scalar operator of order 1 or 2 (FP64, the values
// layout above) on the device.
void element_blocks_device(const sipg_op* op, double* v, cudaStream_t s);

// Assemble in FP64; want32: also the FP32 V-cycle's copy
// (scaled FP16 for even Np, the FP64 values then released; FP32 otherwise).
// binv_rows (FP32 V-cycle, even Np): the inverse diagonal blocks, row-major per
// element, for the preconditioned copy C (binv_sym: with their symmetric part, as
// the packed smoother blocks hold them).
void bsr_assemble(sipg_op* op, BsrOp& B, bool want32, cudaStream_t s, const double* binv_rows = nullptr,
                  bool binv_sym = false);

// y = alpha * B x + beta * c, c = y when null (beta == 0: c is not read).
template <typename T>
void bsr_apply(const BsrOp& B, const T* x, T* y, T alpha, T beta, cudaStream_t s, const T* c = nullptr);

// One Chebyshev step on the block-Jacobi preconditioned operator of an assembled
// FP32 level (B.c16 present), with the preconditioned residual sres = Bd^-1 r kept
// current: sres -= C din, dout = c1 din + c2 sres, z += dout. din and dout are
// distinct buffers (neighbours read din). s0_scale != 0: sres is first set to
// s0_scale * din (the step after a first step din = c2 Bd^-1 r, s0_scale = 1 / c2).
void bsr_cheb_step(const BsrOp& B, const float* din, float* dout, float* sres, float* z, float c1, float c2,
                   float s0_scale, cudaStream_t s);


}  // namespace sipg
