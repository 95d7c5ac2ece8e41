// engine_tdvp.cpp -- TDVP time evolution on the device with a real prefactor: tdvp_twosite
// (algs/time.jl:288-363) and the single-site tdvp (:211-286), each step's propagator applied by
// krylovTimeEvol (:182-203: Lanczos with r vectors, exp(prefactor' T) e_1 as the combination).
//
// tdvp_twosite, rightward step at (iL, iR) with tau = prefactor / (L-1) / 2:
//   AA <- exp(tau H2) AA (the two-site Heff), truncated split psi[iL] = U, psi[iR] = D V,
//   Lenv[iR] <- Lupdate, psi[iR] <- exp(tau H1) psi[iR] (the single-site Heff at iR),
//   then the centre moves to iR and is normalised; leftward steps mirror this. One call is one
//   half sweep (L-1 steps), turning at the edge.
// tdvp, rightward step at i with tau = prefactor / L / 2: psi[i] <- exp(tau H1) psi[i],
//   truncated split psi[i] = U, C = D V, Lenv[i+1] <- Lupdate, C <- exp(tau H0) C (the zero-site
//   Heff, OC_update), psi[i+1] <- C psi[i+1], normalised. The reference runs L steps from the
//   edge, and its L-th step would read psi[L+1] (its turn test compares the centre with L+1);
//   here a call is L-1 steps, one half sweep, turning at the edge like the two-site form.
// Both forms evolve the bond and the site with the same sign of tau, as the reference does.
// Real tensors only: a complex prefactor (real-time evolution) needs complex tensors, which the
// engine does not hold.
#include <algorithm>
#include <chrono>
#include <cmath>

#include "engine_step.hpp"

namespace dmrg {
namespace {

// psi[i] <- exp(tau H1) psi[i] (krylovTimeEvol with singlesite_update); environments that read
// psi[i] are marked stale.
void evolve_site(dmrg_state* st, const dmrg_params& P, int i, double tau, Timing& tm,
                 StepOut& so) {
  dmrg_ctx* c = st->ctx;
  if (!st->Lvalid[i] || !st->Rvalid[i]) fail(DMRG_ERR_STATE, "environments are not built");
  HeffPlan hp;
  plan_heff1(st, i, hp);
  upload_heff(c, hp, 0, P.precision);
  const int64_t n = st->lay[i].size;
  const int kdim = std::max(2, std::min(P.krylov, 16));
  ensure(c, c->K, std::max<int64_t>(int64_t(kdim) * n, 1));
  ensure(c, c->H, std::max<int64_t>(n, 1));
  cuda_check(cudaMemcpyAsync(c->K.p, st->A[i].p, size_t(n) * sizeof(double),
                             cudaMemcpyDeviceToDevice, c->stream), "TDVP start vector");
  krylov_solve(st, P, hp, n, false, false, tm, so, tau, true);
  cuda_check(cudaMemcpyAsync(st->A[i].p, c->H.p, size_t(n) * sizeof(double),
                             cudaMemcpyDeviceToDevice, c->stream), "TDVP site");
  for (int k = i + 1; k < st->L; ++k) st->Lvalid[k] = 0;
  for (int k = 0; k < i; ++k) st->Rvalid[k] = 0;
}

void normalise(dmrg_state* st, int i) {
  dmrg_ctx* c = st->ctx;
  launch_mdot(c->stream, st->A[i].p, 0, 1, st->A[i].p, st->lay[i].size, c->d_partial,
              c->d_scal + lz::NRM);
  launch_scale_rsqrt(c->stream, st->A[i].p, st->lay[i].size, c->d_scal + lz::NRM);
  cuda_check(cudaGetLastError(), "centre normalisation");
}

}  // namespace

void do_tdvp(dmrg_state* st, const dmrg_params& P, double prefactor, bool twosite,
             dmrg_sweep_stats& out) {
  dmrg_ctx* c = st->ctx;
  const int L = st->L;
  if (L < 2) fail(DMRG_ERR_SHAPE, "TDVP needs at least two sites");
  if (!st->env_built) fail(DMRG_ERR_STATE, "call dmrg_env_build before dmrg_tdvp");
  if (!std::isfinite(prefactor)) fail(DMRG_ERR_ARG, "prefactor must be finite");
  std::memset(&out, 0, sizeof(out));
  c->tune = P.tune != 0;
  const long long g0 = c->graph_launches;
  const auto h0 = std::chrono::steady_clock::now();
  Timing tm(c, P.profile != 0);
  const int t0 = tm.record();
  const double tau = twosite ? prefactor / (L - 1) / 2.0 : prefactor / L / 2.0;
  // direction (algs/time.jl:297-304): from the left edge rightward, from the right edge
  // leftward, elsewhere rightward (origj = true)
  int j = st->oc == L - 1 ? -1 : 1;
  for (int n = 0; n < L - 1; ++n) {
    const int i = st->oc;
    StepOut so;
    double ef = 0.0;
    if (twosite) {
      const int iL = j > 0 ? i : i - 1, iR = j > 0 ? i + 1 : i;
      StepMode md;
      md.tdvp = true;
      md.tau = tau;
      twostep(st, P, j, iL, iR, false, tm, so, md);
      const int tenv = tm.begin();
      if (j > 0) lupdate(st, iL, &ef, P.precision); else rupdate(st, iR, &ef, P.precision);
      tm.end(tenv, 1);
      evolve_site(st, P, j > 0 ? iR : iL, tau, tm, so);
    } else {
      SiteMode md;
      md.tdvp = true;
      md.tau = tau;
      single_site_step(st, P, md, j, i, false, tm, so);
    }
    st->oc += j;
    normalise(st, st->oc);
    out.max_truncerr = std::max(out.max_truncerr, so.truncerr);
    out.biggest_m = std::max(out.biggest_m, so.m);
    out.n_matvec += so.nmv;
    out.wait_seconds += so.wait;
    out.heff_flops += so.heff_flops;
    out.env_flops += ef + so.env_flops;
    out.eig_max_n = std::max(out.eig_max_n, so.eig_max_n);
    if ((st->oc == L - 1 && j > 0) || (st->oc == 0 && j < 0)) j = -j;
  }
  st->dir = j;
  const int t1 = tm.record();
  cuda_check(cudaEventSynchronize(tm.event(t1)), "TDVP sync");
  if (split_form(P.precision)) check_mma_status(c);
  tuner_collect(c);
  // En of the last krylovTimeEvol call: the lowest eigenvalue of its Krylov tridiagonal, whose
  // download completed before the final event
  out.energy = c->h_scal[lz::EN];
  out.graph_launches = int(c->graph_launches - g0);
  float ms = 0;
  cudaEventElapsedTime(&ms, tm.event(t0), tm.event(t1));
  out.seconds = ms * 1e-3;
  tm.flush();
  out.heff_seconds = tm.acc[0];
  out.env_seconds = tm.acc[1];
  out.eig_seconds = tm.acc[2];
  out.vec_seconds = tm.acc[3];
  out.gemm_flops = tm.gemm.flops;
  out.gemm_seconds = tm.gemm.seconds;
  out.gemm_launches = tm.gemm.launches;
  out.host_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - h0).count();
  st->have_last = false;
}

}  // namespace dmrg
