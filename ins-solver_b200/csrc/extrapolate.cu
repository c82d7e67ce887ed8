// Initial guess by extrapolation in time of previous solutions.
//
// The reference keeps the pressure of the last EXTRAPOLATE_HISTORY_SIZE steps
// with their times (add_to_pr_history, src/solvers/3d/ins_solver_base.cpp:1374-1388)
// and, before each pressure solve, sets the initial guess from them
// (initial_guess_extrapolation(mesh, pr_history, pr, time + dt),
// src/solvers/3d/ins_solver.cpp:342-343, mp_ins_solver.cpp:629-630; the function
// itself lives in the unvendored OP2-DG-Toolkit). Here: the polynomial through
// the n history points (t_i, x_i), evaluated at t_new, i.e. x = sum_i w_i x_i with
// the Lagrange weights w_i = prod_{j != i} (t_new - t_j) / (t_i - t_j); one point
// copies it.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "../../include/sipg_b200.h"
#include "capi_util.hpp"
#include "pdl.cuh"
#include "vecops.cuh"

namespace sipg {
namespace {

constexpr int kMaxHist = 8;

struct Hist {
  const double* x[kMaxHist];
  double w[kMaxHist];
  int n;
};

__global__ void k_extrapolate(Hist h, size_t n, double* out) {
  pdl_enter();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < h.n; ++k) s += h.w[k] * h.x[k][i];
    out[i] = s;
  }
}

std::vector<double> lagrange_weights(int m, const double* t, double t_new) {
  std::vector<double> w(m, 1.0);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j)
      if (j != i) {
        if (t[i] == t[j]) throw Error(SIPG_INVALID_ARG, "history times must be distinct");
        w[i] *= (t_new - t[j]) / (t[i] - t[j]);
      }
  return w;
}

void check_args(int m, const double* t, const double* const* hist, const double* out) {
  if (m < 1 || m > kMaxHist || !t || !hist || !out) throw Error(SIPG_INVALID_ARG, "extrapolation arguments");
  for (int i = 0; i < m; ++i)
    if (!hist[i] || !std::isfinite(t[i])) throw Error(SIPG_INVALID_ARG, "extrapolation history entry");
}

}  // namespace
}  // namespace sipg

using namespace sipg;

extern "C" int sipg_extrapolate_initial_guess(int n_hist, const double* times, const double* const* hist,
                                              double t_new, size_t n, double* out, void* stream) {
  return guarded([&] {
    check_args(n_hist, times, hist, out);
    std::vector<double> w = lagrange_weights(n_hist, times, t_new);
    Hist h{};
    h.n = n_hist;
    for (int i = 0; i < n_hist; ++i) {
      h.x[i] = hist[i];
      h.w[i] = w[i];
    }
    const int g = (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 148 * 16));
    SIPG_CUDA(pdl_launch(k_extrapolate, dim3(g), dim3(256), 0, (cudaStream_t)stream, h, n, out));
    note_launch();
  });
}

extern "C" int sipg_extrapolate_initial_guess_host(int n_hist, const double* times, const double* const* hist,
                                                   double t_new, size_t n, double* out) {
  return guarded([&] {
    check_args(n_hist, times, hist, out);
    std::vector<double> w = lagrange_weights(n_hist, times, t_new);
    for (size_t i = 0; i < n; ++i) {
      double s = 0.0;
      for (int k = 0; k < n_hist; ++k) s += w[k] * hist[k][i];
      out[i] = s;
    }
  });
}
