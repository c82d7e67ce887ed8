// C ABI of the algebraic coarse hierarchy (host-side build), see amg.hpp.
#include <cstring>
#include <memory>

#include "../../include/sipg_b200.h"
#include "amg.hpp"
#include "capi_util.hpp"
#include "refelem.hpp"
#include "runtime.hpp"

struct sipg_amg {
  sipg::AmgHierarchy h;
};

using namespace sipg;

extern "C" {

int sipg_amg_build(int K, int Nf, const double* sJ, const double* tau, const int* nbr, int Kb,
                   const int* bc_dirichlet, int coarse_max, double strength, int singular,
                   sipg_amg** out) {
  return guarded([&] {
    if (K <= 0 || (Nf != 3 && Nf != 4) || !sJ || !tau || !nbr || !out || (Kb > 0 && !bc_dirichlet))
      throw Error(SIPG_INVALID_ARG, "amg_build arguments");
    std::vector<uint8_t> bd(Kb);
    for (int b = 0; b < Kb; ++b) bd[b] = bc_dirichlet[b] ? 1 : 0;
    Csr A0 = p0_operator(K, Nf, sJ, tau, nbr, bd);
    Csr Pdg;  // p=1 DG nodes x elements: every node of element e takes the element value
    const int Np = Nf;  // order 1: Np = dim + 1 = Nf
    Pdg.rows = K * Np;
    Pdg.cols = K;
    Pdg.ptr.resize(Pdg.rows + 1);
    for (int k = 0; k <= Pdg.rows; ++k) Pdg.ptr[k] = k;
    Pdg.idx.resize(Pdg.rows);
    for (int k = 0; k < Pdg.rows; ++k) Pdg.idx[k] = k / Np;
    Pdg.val.assign(Pdg.rows, 1.0);
    auto a = std::make_unique<sipg_amg>();
    a->h = build_amg(A0, Pdg, coarse_max, strength, singular != 0);
    *out = a.release();
  });
}

int sipg_amg_build_p1(sipg_mesh* m, const double* factor1, const double* tau1, const int* bc_dirichlet,
                      int mm_mode, double mm_scalar, const double* mm1, int coarse_max, double strength,
                      int singular, sipg_amg** out) {
  return guarded([&] {
    if (!m || !tau1 || !out || (m->Kb > 0 && !bc_dirichlet)) throw Error(SIPG_INVALID_ARG, "amg_build_p1 arguments");
    const Mesh& h = m->host_order(1);
    RefElement r1 = build_ref_element(m->dim, 1);
    std::vector<uint8_t> bd(m->Kb);
    for (int b = 0; b < m->Kb; ++b) bd[b] = bc_dirichlet[b] ? 1 : 0;
    Csr A0, Pdg;
    p1c_operator(r1, m->K, m->Nv, h.geof.data(), h.e2v.data(), factor1, tau1, h.sJ.data(), h.nx.data(),
                 h.ny.data(), h.nz.data(), h.nbr.data(), bd, mm_mode, mm_scalar, mm1, &A0, &Pdg);
    auto a = std::make_unique<sipg_amg>();
    a->h = build_amg(A0, Pdg, coarse_max, strength, singular != 0);
    *out = a.release();
  });
}

int sipg_amg_sizes(const sipg_amg* a, int* nlevels, int* coarse_n) {
  return guarded([&] {
    if (!a) throw Error(SIPG_INVALID_ARG, "null amg");
    if (nlevels) *nlevels = (int)a->h.levels.size();
    if (coarse_n) *coarse_n = a->h.coarse_n;
  });
}

int sipg_amg_level(const sipg_amg* a, int level, int which, int* rows, int* cols, int* nnz, int* ptr,
                   int* idx, double* val) {
  return guarded([&] {
    if (!a || level < -1 || level >= (int)a->h.levels.size() || which < 0 || which > 2)
      throw Error(SIPG_INVALID_ARG, "amg_level arguments");
    if (level == -1 && which == 0) throw Error(SIPG_INVALID_ARG, "level -1 has only P and R");
    const Csr& M = level == -1 ? (which == 1 ? a->h.Pdg : a->h.Rdg)
                               : (which == 0 ? a->h.levels[level].A
                                             : which == 1 ? a->h.levels[level].P : a->h.levels[level].R);
    if (rows) *rows = M.rows;
    if (cols) *cols = M.cols;
    if (nnz) *nnz = (int)M.nnz();
    if (ptr && !M.ptr.empty()) std::memcpy(ptr, M.ptr.data(), M.ptr.size() * sizeof(int));
    if (idx && M.nnz()) std::memcpy(idx, M.idx.data(), M.nnz() * sizeof(int));
    if (val && M.nnz()) std::memcpy(val, M.val.data(), M.nnz() * sizeof(double));
  });
}

int sipg_amg_coarse_inverse(const sipg_amg* a, double* inv) {
  return guarded([&] {
    if (!a || !inv) throw Error(SIPG_INVALID_ARG, "amg_coarse_inverse arguments");
    std::memcpy(inv, a->h.coarse_inv.data(), a->h.coarse_inv.size() * sizeof(double));
  });
}

void sipg_amg_destroy(sipg_amg* a) { delete a; }

}  // extern "C"
