// Two-phase 3D time step on the device: the counterpart of MPINSSolver3D
// (src/solvers/3d/mp_ins_solver.cpp:182-285, 394-448, 581-667, 669-790, 981-992)
// with its level set (LevelSetSolver3D, src/solvers/3d/ls_solver.cpp:106-257),
// for no-slip walls and natural outflow, without surface tension, sub-cycling,
// filtering, shock capturing or level-set reinitialisation. Every field stays in
// HBM; one stream orders the pointwise and element kernels, the solvers run on their
// own streams after a synchronisation (their set-up reads the operator state).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "../../include/sipg_b200.h"
#include "capi_util.hpp"
#include "ins_step.cuh"
#include "runtime.hpp"

using namespace sipg;

namespace {

void ok(int status, const char* what) {
  if (status != SIPG_OK) throw Error(status, std::string(what) + ": " + sipg_last_error());
}

// A linear solve that stops short is an error of the step, as the reference's
// dg_abort("Pressure solve failed to converge") is.
void solved(int status, const char* what, const sipg_solve_info& i) {
  if (status == SIPG_OK) return;
  char buf[160];
  std::snprintf(buf, sizeof(buf), "%s: status %d after %d iterations, relative residual %.3e", what, status, i.iters,
                i.rel_res);
  throw Error(status, buf);
}

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
  Timer() {
    SIPG_CUDA(cudaEventCreate(&a));
    SIPG_CUDA(cudaEventCreate(&b));
  }
  ~Timer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
};

}  // namespace

struct sipg_ins3d {
  sipg_mesh* m = nullptr;
  sipg_ins3d_opts o{};
  int Np = 0, Nfp = 0;
  size_t n = 0;  // K x Np
  cudaStream_t st = nullptr;
  DevBuf vel[2], N[2], velT, velTT, pr, dPdN[2];
  DevBuf s, qa, qb, rk0, rk1, rho, mu, rrho;
  DevBuf rhs, mmf, vbc, vmax, stats, xyz;
  ReinitWork rw;
  double h_ls = 0.0;
  int reinit_counter = 0;
  std::vector<DevBuf> hist;      // pressure history (ring), newest last in hist_order
  std::vector<double> hist_t;
  std::vector<int> hist_order;
  sipg_op *pop = nullptr, *vop = nullptr;
  sipg_solver *psol = nullptr, *vsol = nullptr;
  int cur = 0, vcomp = 1;
  long long pr_setups = 0;  // pressure steps since set_state (the set-up runs every pr_setup_every)
  double time = 0.0, dt = 0.0, a0 = 1.0, a1 = 0.0, b0 = 1.0, b1 = 0.0, g0 = 1.0;
  double h = 0.0, alpha = 0.0, max_vel = 1.0;
  bool have_state = false;
  Timer t_adv, t_pr, t_vis, t_surf;

  ~sipg_ins3d() {
    if (psol) sipg_solver_destroy(psol);
    if (vsol) sipg_solver_destroy(vsol);
    if (pop) sipg_op_destroy(pop);
    if (vop) sipg_op_destroy(vop);
    if (st) cudaStreamDestroy(st);
  }

  LsFields ls_fields(const double* u) {
    LsFields f{};
    f.u = u;
    f.s = s.as<double>();
    f.qa = qa.as<double>();
    f.qb = qb.as<double>();
    f.rk0 = rk0.as<double>();
    f.rk1 = rk1.as<double>();
    f.rho = rho.as<double>();
    f.mu = mu.as<double>();
    f.rrho = rrho.as<double>();
    f.vmax = vmax.as<unsigned long long>();
    f.alpha = alpha;
    f.rho0 = o.rho0;
    f.rho1 = o.rho1;
    f.mu0 = o.mu0;
    f.mu1 = o.mu1;
    return f;
  }

  // max(1, sqrt(max |u|^2)) from the device scalar the level-set kernels reduce into
  double read_max_vel() {
    unsigned long long bits = 0;
    SIPG_CUDA(cudaMemcpyAsync(&bits, vmax.p, sizeof(bits), cudaMemcpyDeviceToHost, st));
    SIPG_CUDA(cudaStreamSynchronize(st));
    double v2;
    std::memcpy(&v2, &bits, sizeof(v2));
    return std::max(1.0, std::sqrt(v2));
  }

  double next_dt() const { return o.cfl * h / ((o.order + 1) * (o.order + 1) * max_vel); }

  void pressure_guess() {
    const int nh = (int)hist_order.size();
    double* p = pr.as<double>();
    if (o.extrapolate_history <= 0 || nh == 0) return;  // previous pressure
    std::vector<double> times;
    std::vector<const double*> ptr;
    for (int i : hist_order) {
      times.push_back(hist_t[i]);
      ptr.push_back(hist[i].as<double>());
    }
    ok(sipg_extrapolate_initial_guess(nh, times.data(), ptr.data(), time + dt, n, p, st), "initial guess");
  }

  void add_history() {
    if (o.extrapolate_history <= 0) return;
    int slot;
    if ((int)hist_order.size() < o.extrapolate_history) {
      slot = (int)hist_order.size();
      hist.emplace_back(n * sizeof(double));
      hist_t.push_back(0.0);
    } else {
      slot = hist_order.front();
      hist_order.erase(hist_order.begin());
    }
    SIPG_CUDA(cudaMemcpyAsync(hist[slot].p, pr.p, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    hist_t[slot] = time + dt;
    hist_order.push_back(slot);
  }

  // LevelSetSolver3D::step's reinitialisation and ls_post_reinit, then rho, mu and max |u|
  // again from the new level set
  void reinit(const double* u) {
    ls_reinit_device(m, o.order, xyz.as<double>(), s.as<double>(), h_ls, o.ls_cap, rw, st);
    ls_props_device(m, o.order, ls_fields(u), st);
  }

  void step(sipg_ins3d_step_info* info) {
    const int nw = 1 - cur;
    double* u = vel[cur].as<double>();
    double* u_new = vel[nw].as<double>();
    const int* bc = vbc.as<int>();
    // advection (advec_standard)
    SIPG_CUDA(cudaEventRecord(t_adv.a, st));
    advection_device(m, o.order, dt, a0, a1, b0, b1, o.gravity, u, u_new, N[nw].as<double>(), bc, N[cur].as<double>(),
                     velT.as<double>(), st);
    SIPG_CUDA(cudaEventRecord(t_adv.b, st));
    // pressure
    SIPG_CUDA(cudaEventRecord(t_pr.a, st));
    pressure_neumann_device(m, o.order, o.reynolds, o.gravity, u, N[cur].as<double>(), mu.as<double>(),
                            rho.as<double>(), bc, dPdN[cur].as<double>(), st);
    ok(sipg_pressure_rhs(m, o.order, dt, b0, b1, velT.as<double>(), dPdN[cur].as<double>(), dPdN[nw].as<double>(),
                         rhs.as<double>(), st),
       "pressure right-hand side");
    SIPG_CUDA(cudaStreamSynchronize(st));
    const auto c0 = std::chrono::steady_clock::now();
    if (o.pr_over_int)
      set_factor_oi_level_set(pop, s.as<double>(), alpha, o.rho0, o.rho1, st);
    else
      set_factor_device(pop, rrho.as<double>(), st);
    pressure_guess();
    SIPG_CUDA(cudaStreamSynchronize(st));
    if (pr_setups++ % o.pr_setup_every == 0) ok(sipg_solver_setup(psol), "pressure set-up");
    const auto c1 = std::chrono::steady_clock::now();
    sipg_solve_info pi{};
    solved(sipg_solver_solve(psol, rhs.as<double>(), pr.as<double>(), &pi), "pressure solve", pi);
    add_history();
    ok(sipg_pressure_projection(m, o.order, dt, dt, pr.as<double>(), rho.as<double>(), velT.as<double>(),
                                velTT.as<double>(), stats.as<unsigned long long>(), st),
       "pressure projection");
    SIPG_CUDA(cudaEventRecord(t_pr.b, st));
    // viscosity
    SIPG_CUDA(cudaEventRecord(t_vis.a, st));
    ok(sipg_viscous_rhs(m, o.order, o.reynolds / dt, g0 * o.reynolds / dt, rho.as<double>(), velTT.as<double>(),
                        rhs.as<double>(), mmf.as<double>(), st),
       "viscous right-hand side");
    set_factor_device(vop, mu.as<double>(), st);
    set_mm_device(vop, SIPG_MM_NODAL, 0.0, mmf.as<double>(), st);
    SIPG_CUDA(cudaStreamSynchronize(st));
    ok(sipg_solver_setup(vsol), "viscous set-up");
    sipg_solve_info vi[3]{};
    if (vcomp == 3) {
      solved(sipg_solver_solve(vsol, rhs.as<double>(), u_new, &vi[0]), "viscous solve", vi[0]);
      vi[1] = vi[2] = vi[0];
    } else {
      for (int c = 0; c < 3; ++c)
        solved(sipg_solver_solve(vsol, rhs.as<double>() + c * n, u_new + c * n, &vi[c]), "viscous solve", vi[c]);
    }
    SIPG_CUDA(cudaEventRecord(t_vis.b, st));
    // surface (level set, then rho and mu)
    SIPG_CUDA(cudaEventRecord(t_surf.a, st));
    ls_step_device(m, o.order, dt, ls_fields(u_new), st);
    if (o.reinit_freq > 0 && ++reinit_counter >= o.reinit_freq) {
      reinit(u_new);
      reinit_counter = 0;
    }
    SIPG_CUDA(cudaEventRecord(t_surf.b, st));
    max_vel = read_max_vel();
    // update_time and the second-order coefficients (MPINSSolver3D::step)
    cur = nw;
    time += dt;
    a0 = 2.0;
    a1 = -0.5;
    b0 = 2.0;
    b1 = -1.0;
    g0 = 1.5;
    dt = next_dt();
    if (info) {
      unsigned long long cs[2] = {0, 0};
      SIPG_CUDA(cudaMemcpy(cs, stats.p, sizeof(cs), cudaMemcpyDeviceToHost));
      info->time = time;
      info->dt = dt;
      info->pr_iters = pi.iters;
      info->pr_rel_res = pi.rel_res;
      for (int c = 0; c < 3; ++c) {
        info->vis_iters[c] = vi[c].iters;
        info->vis_rel_res[c] = vi[c].rel_res;
      }
      info->max_vel = max_vel;
      float ms;
      SIPG_CUDA(cudaEventElapsedTime(&ms, t_adv.a, t_adv.b));
      info->ms_advection = ms;
      SIPG_CUDA(cudaEventElapsedTime(&ms, t_pr.a, t_pr.b));
      info->ms_pressure = ms;
      SIPG_CUDA(cudaEventElapsedTime(&ms, t_vis.a, t_vis.b));
      info->ms_viscosity = ms;
      SIPG_CUDA(cudaEventElapsedTime(&ms, t_surf.a, t_surf.b));
      info->ms_surface = ms;
      info->proj_converged = cs[0];
      info->ms_pressure_setup = std::chrono::duration<double, std::milli>(c1 - c0).count();
      info->ms_pressure_solve = pi.solve_ms;
    }
  }
};

extern "C" {

int sipg_ins3d_default_opts(sipg_ins3d_opts* o) {
  return guarded([&] {
    if (!o) throw Error(SIPG_INVALID_ARG, "null opts");
    std::memset(o, 0, sizeof(*o));
    o->order = 3;
    o->reynolds = 1.0;
    o->rho0 = o->rho1 = o->mu0 = o->mu1 = 1.0;
    o->ls_alpha = 24.0;  // level-set-options alpha (ls_solver.cpp:137)
    o->cfl = 1.0;
    o->extrapolate_history = 3;
    o->viscous_kind = SIPG_SOLVER_JACOBI;
    o->pr_setup_every = 1;
    o->reinit_freq = 24;  // level-set-options reinit_freq (ls_solver.cpp:146-148)
    o->reinit_ic = 1;     // reinit_ic (:158-159)
    o->ls_cap = 1.0;      // LS_CAP, include/problem_specific_3d.h
    // setup_pressure_viscous_solvers (ins_solver_base.cpp:149-184)
    ok(sipg_solver_default_opts(SIPG_SOLVER_PMULTIGRID, &o->pressure), "pressure options");
    o->pressure.rel_tol = 1e-8;
    o->pressure.abs_tol = 1e-9;
    o->pressure.max_iter = 500;
    o->pressure.n_levels = 0;
    o->pressure.eig_safety = 2.5;
    ok(sipg_solver_default_opts(SIPG_SOLVER_JACOBI, &o->viscous), "viscous options");
    o->viscous.rel_tol = 1e-8;
    o->viscous.abs_tol = 1e-9;
    o->viscous.max_iter = 5000;
  });
}

int sipg_ins3d_create(sipg_mesh* m, const sipg_ins3d_opts* o, const int* vel_bc, sipg_ins3d** out) {
  return guarded([&] {
    if (!m || !o || !out || (m->Kb && !vel_bc)) throw Error(SIPG_INVALID_ARG, "ins3d_create arguments");
    if (m->dim != 3) throw Error(SIPG_INVALID_ARG, "the two-phase time step is 3D");
    if (o->order < 1 || o->order > 4) throw Error(SIPG_INVALID_ARG, "order must be 1..4");
    if (!(o->reynolds > 0.0) || !(o->rho0 > 0.0) || !(o->rho1 > 0.0) || !(o->mu0 > 0.0) || !(o->mu1 > 0.0) ||
        !(o->ls_alpha > 0.0) || !(o->cfl > 0.0))
      throw Error(SIPG_INVALID_ARG, "ins3d constants must be positive");
    if (o->extrapolate_history < 0 || o->extrapolate_history > 8)
      throw Error(SIPG_INVALID_ARG, "extrapolate_history must be 0..8");
    if (!(o->ls_cap > 0.0) || o->reinit_freq < 0) throw Error(SIPG_INVALID_ARG, "ls_cap > 0 and reinit_freq >= 0");
    if (o->pr_setup_every < 1) throw Error(SIPG_INVALID_ARG, "pr_setup_every must be >= 1");
    if (o->viscous_kind != SIPG_SOLVER_JACOBI && o->viscous_kind != SIPG_SOLVER_BLOCK_JACOBI &&
        o->viscous_kind != SIPG_SOLVER_PMULTIGRID)
      throw Error(SIPG_INVALID_ARG,
                  "viscous_kind must be SIPG_SOLVER_JACOBI, SIPG_SOLVER_BLOCK_JACOBI or SIPG_SOLVER_PMULTIGRID");
    bool dirichlet_pr = false, slip = false;
    for (int b = 0; b < m->Kb; ++b) {
      if (vel_bc[b] < 0 || vel_bc[b] > 2)
        throw Error(SIPG_INVALID_ARG, "ins3d supports no-slip (0), slip (1) and natural outflow (2) boundaries");
      slip = slip || vel_bc[b] == 1;
    }
    // with slip walls the viscous solve is the coupled vector one (uses_slip_bcs:
    // FactorViscousMatrix3D + ViscousSolver3D), otherwise one component at a time
    const int vcomp = slip ? 3 : 1;
    std::vector<int> prt(m->Kb), vst((size_t)vcomp * m->Kb);
    for (int b = 0; b < m->Kb; ++b) {
      int vt;
      if (vel_bc[b] == 2) {  // natural outflow: pressure Dirichlet 0, velocity Neumann (ins_3d_pr_dirichlet)
        prt[b] = SIPG_BC_DIRICHLET;
        vt = SIPG_BC_NEUMANN;
        dirichlet_pr = true;
      } else {  // walls: pressure Neumann; velocity Dirichlet 0 (no-slip) or slip (ins_3d_vis_x)
        prt[b] = SIPG_BC_NEUMANN;
        vt = vel_bc[b] == 0 ? SIPG_BC_DIRICHLET : SIPG_BC_SLIP;
      }
      for (int c = 0; c < vcomp; ++c) vst[(size_t)c * m->Kb + b] = vt;
    }
    auto ins = std::make_unique<sipg_ins3d>();
    ins->m = m;
    ins->o = *o;
    m->ensure_device();
    const Mesh& hm = m->host_order(o->order);
    ins->Np = hm.Np;
    ins->Nfp = hm.Nfp;
    ins->n = (size_t)m->K * hm.Np;
    // h of INSSolverBase3D::init (1 / the largest interior-face fscale) and of
    // LevelSetSolver3D::init (1 / the smallest): calc_h_3d, calc_h_3d_max
    double fmax_ = 0.0, fmin_ = 1e300;
    for (int e = 0; e < m->K; ++e)
      for (int f = 0; f < 4; ++f)
        if (hm.nbr[(size_t)e * 4 + f] >= 0) {
          fmax_ = std::max(fmax_, hm.fscale[(size_t)e * 4 + f]);
          fmin_ = std::min(fmin_, hm.fscale[(size_t)e * 4 + f]);
        }
    if (fmax_ <= 0.0) throw Error(SIPG_INVALID_ARG, "mesh without interior faces");
    ins->h = 1.0 / fmax_;
    ins->h_ls = 1.0 / fmin_;
    ins->alpha = o->ls_alpha / fmin_;
    SIPG_CUDA(cudaStreamCreateWithFlags(&ins->st, cudaStreamNonBlocking));
    const size_t nb = ins->n * sizeof(double), nf = (size_t)m->K * 4 * hm.Nfp * sizeof(double);
    for (int i = 0; i < 2; ++i) {
      ins->vel[i] = DevBuf(3 * nb);
      ins->N[i] = DevBuf(3 * nb);
      ins->dPdN[i] = DevBuf(nf);
    }
    ins->velT = DevBuf(3 * nb);
    ins->velTT = DevBuf(3 * nb);
    ins->rhs = DevBuf(3 * nb);
    for (DevBuf* b : {&ins->pr, &ins->s, &ins->qa, &ins->qb, &ins->rk0, &ins->rk1, &ins->rho, &ins->mu, &ins->rrho,
                      &ins->mmf})
      *b = DevBuf(nb);
    ins->vbc = DevBuf(std::max<size_t>(1, m->Kb) * sizeof(int));
    if (m->Kb) ins->vbc.upload(vel_bc, m->Kb * sizeof(int));
    ins->vmax = DevBuf(sizeof(unsigned long long));
    {
      std::vector<double> xyz(3 * ins->n);
      std::copy(hm.x.begin(), hm.x.end(), xyz.begin());
      std::copy(hm.y.begin(), hm.y.end(), xyz.begin() + ins->n);
      std::copy(hm.z.begin(), hm.z.end(), xyz.begin() + 2 * ins->n);
      ins->xyz = DevBuf(3 * nb);
      ins->xyz.upload(xyz.data(), 3 * nb);
    }
    ins->stats = DevBuf(2 * sizeof(unsigned long long));
    // pressure: FactorPoissonMatrixFreeDiag3D + PETScPMultigrid, nullspace without Dirichlet faces
    ok(sipg_op_create(m, o->order, 1, &ins->pop), "pressure operator");
    ok(sipg_op_set_bc_types(ins->pop, prt.data()), "pressure boundary types");
    sipg_solver_opts po = o->pressure;
    po.nullspace = dirichlet_pr ? 0 : 1;
    if (po.n_levels == 0) {  // p-multigrid orders p, p-1, ..., 1 (the [p-multigrid] orders key)
      po.n_levels = o->order;
      for (int l = 0; l < 4; ++l) po.orders[l] = l < o->order ? o->order - l : 0;
    }
    ok(sipg_solver_create(ins->pop, SIPG_SOLVER_PMULTIGRID, &po, &ins->psol), "pressure solver");
    // viscosity: FactorMMPoissonMatrixFreeDiag3D + PETScJacobiSolver, one component at a
    // time, or with slip walls FactorViscousMatrix3D + ViscousSolver3D on (u, v, w)
    ins->vcomp = vcomp;
    ok(sipg_op_create(m, o->order, vcomp, &ins->vop), "viscous operator");
    ok(sipg_op_set_bc_types(ins->vop, vst.data()), "viscous boundary types");
    sipg_solver_opts vo = o->viscous;
    if (o->viscous_kind == SIPG_SOLVER_PMULTIGRID && vo.n_levels == 0) {
      // one level, no smoothing: the preconditioner is coarse_iters Jacobi-PCG iterations
      // on the viscous operator itself, in the viscous precision (FP32: TF32 applies),
      // inside the FP64 flexible PCG
      vo.n_levels = 1;
      vo.orders[0] = o->order;
      vo.smoother = 0;
      vo.coarse_kind = 0;
      vo.pre_it[0] = vo.post_it[0] = 0;
    }
    ok(sipg_solver_create(ins->vop, o->viscous_kind, &vo, &ins->vsol), "viscous solver");
    *out = ins.release();
  });
}

int sipg_ins3d_set_state_host(sipg_ins3d* ins, const double* vel, const double* s) {
  return guarded([&] {
    if (!ins || !vel || !s) throw Error(SIPG_INVALID_ARG, "ins3d_set_state arguments");
    const size_t nb = ins->n * sizeof(double);
    ins->vel[0].upload(vel, 3 * nb, ins->st);
    ins->vel[1].upload(vel, 3 * nb, ins->st);
    ins->s.upload(s, nb, ins->st);
    for (DevBuf* b : {&ins->N[0], &ins->N[1], &ins->velT, &ins->velTT})
      SIPG_CUDA(cudaMemsetAsync(b->p, 0, 3 * nb, ins->st));
    SIPG_CUDA(cudaMemsetAsync(ins->pr.p, 0, nb, ins->st));
    for (DevBuf* b : {&ins->dPdN[0], &ins->dPdN[1]}) SIPG_CUDA(cudaMemsetAsync(b->p, 0, b->bytes, ins->st));
    ins->hist_order.clear();
    ins->cur = 0;
    ins->time = 0.0;
    ins->a0 = 1.0;
    ins->a1 = 0.0;
    ins->b0 = 1.0;
    ins->b1 = 0.0;
    ins->g0 = 1.0;
    ins->reinit_counter = 0;
    ins->pr_setups = 0;
    if (ins->o.reinit_ic)
      ins->reinit(ins->vel[0].as<double>());
    else
      ls_props_device(ins->m, ins->o.order, ins->ls_fields(ins->vel[0].as<double>()), ins->st);
    ins->max_vel = ins->read_max_vel();
    ins->dt = ins->next_dt();
    ins->have_state = true;
  });
}

int sipg_ins3d_step(sipg_ins3d* ins, int nsteps, sipg_ins3d_step_info* info) {
  return guarded([&] {
    if (!ins || nsteps < 0) throw Error(SIPG_INVALID_ARG, "ins3d_step arguments");
    if (!ins->have_state) throw Error(SIPG_INVALID_ARG, "ins3d_step before set_state");
    for (int i = 0; i < nsteps; ++i) ins->step(i + 1 == nsteps ? info : nullptr);
  });
}

int sipg_ins3d_get_state_host(sipg_ins3d* ins, double* vel, double* pr, double* s, double* rho, double* mu) {
  return guarded([&] {
    if (!ins) throw Error(SIPG_INVALID_ARG, "null ins3d");
    const size_t nb = ins->n * sizeof(double);
    SIPG_CUDA(cudaStreamSynchronize(ins->st));
    if (vel) SIPG_CUDA(cudaMemcpy(vel, ins->vel[ins->cur].p, 3 * nb, cudaMemcpyDeviceToHost));
    if (pr) SIPG_CUDA(cudaMemcpy(pr, ins->pr.p, nb, cudaMemcpyDeviceToHost));
    if (s) SIPG_CUDA(cudaMemcpy(s, ins->s.p, nb, cudaMemcpyDeviceToHost));
    if (rho) SIPG_CUDA(cudaMemcpy(rho, ins->rho.p, nb, cudaMemcpyDeviceToHost));
    if (mu) SIPG_CUDA(cudaMemcpy(mu, ins->mu.p, nb, cudaMemcpyDeviceToHost));
  });
}

void sipg_ins3d_destroy(sipg_ins3d* ins) { delete ins; }

int sipg_ls_reinit_host(sipg_mesh* m, int order, double ls_cap, double* s) {
  return guarded([&] {
    if (!m || !s || !(ls_cap > 0.0)) throw Error(SIPG_INVALID_ARG, "ls_reinit arguments");
    if (m->dim != 3) throw Error(SIPG_INVALID_ARG, "the level-set reinitialisation is 3D");
    if (order < 1 || order > 4) throw Error(SIPG_INVALID_ARG, "order must be 1..4");
    m->ensure_device();
    const Mesh& hm = m->host_order(order);
    const size_t n = (size_t)m->K * hm.Np;
    double fmin_ = 1e300;
    for (int e = 0; e < m->K; ++e)
      for (int f = 0; f < 4; ++f)
        if (hm.nbr[(size_t)e * 4 + f] >= 0) fmin_ = std::min(fmin_, hm.fscale[(size_t)e * 4 + f]);
    if (fmin_ >= 1e300) throw Error(SIPG_INVALID_ARG, "mesh without interior faces");
    std::vector<double> xyz(3 * n);
    std::copy(hm.x.begin(), hm.x.end(), xyz.begin());
    std::copy(hm.y.begin(), hm.y.end(), xyz.begin() + n);
    std::copy(hm.z.begin(), hm.z.end(), xyz.begin() + 2 * n);
    DevBuf dx(3 * n * sizeof(double)), ds(n * sizeof(double));
    dx.upload(xyz.data(), 3 * n * sizeof(double));
    ds.upload(s, n * sizeof(double));
    ReinitWork w;
    ls_reinit_device(m, order, dx.as<double>(), ds.as<double>(), 1.0 / fmin_, ls_cap, w, 0);
    SIPG_CUDA(cudaMemcpy(s, ds.p, n * sizeof(double), cudaMemcpyDeviceToHost));
  });
}

}  // extern "C"
