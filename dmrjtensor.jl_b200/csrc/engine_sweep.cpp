// engine_sweep.cpp -- twostep (algs/DMRG.jl:362-405) and the optmps sweep
// (algs/optimizeMPS.jl:790-835) on the device.
//
// Per bond: normalise the centre tensor, AA = psi_L psi_R (one grouped GEMM), Krylov solve
// (reference 2-vector step or Lanczos-k with full re-orthogonalisation), reduced density matrix
// per centre-charge group (gather + one grouped GEMM), batched Jacobi eigensolve, global
// truncation on the host from the downloaded eigenvalues, split back into the two site tensors
// (copies + one grouped GEMM), then the environment update of the site left behind.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <map>

#include "engine_step.hpp"

namespace dmrg {

Sel select_kept(const std::vector<std::vector<double>>& vals, int maxm, int minm, double cutoff,
                double mag, double degen_rtol) {
  struct E { double v; int g, i; };
  std::vector<E> flat;
  for (int g = 0; g < int(vals.size()); ++g)
    for (int i = 0; i < int(vals[g].size()); ++i) flat.push_back({vals[g][i], g, i});
  std::stable_sort(flat.begin(), flat.end(), [](const E& a, const E& b) {
    if (a.v != b.v) return a.v > b.v;
    if (a.g != b.g) return a.g < b.g;
    return a.i < b.i;
  });
  Sel s;
  s.keep.assign(vals.size(), 0);
  const int N = int(flat.size());
  if (N == 0) return s;
  for (const E& e : flat) s.total += e.v;
  const double tot = mag == 0.0 ? s.total : mag;
  std::vector<double> tail(N + 1, 0.0);
  for (int k = N - 1; k >= 0; --k) tail[k] = tail[k + 1] + flat[k].v;
  int kc = N;
  for (int k = 1; k <= N; ++k)
    if (tail[k] <= cutoff * tot) { kc = k; break; }
  int k = std::max(minm, kc);
  if (maxm > 0) k = std::min(k, maxm);
  k = std::max(1, std::min(k, N));
  if (degen_rtol > 0 && k < N) {
    const double thr = degen_rtol * std::fabs(flat[k - 1].v);
    if (flat[k - 1].v - flat[k].v <= thr) {
      int jj = k - 1;
      while (jj >= 1 && flat[jj - 1].v - flat[jj].v <= thr) --jj;
      if (jj >= std::max(minm, 1)) k = jj;
    }
  }
  for (int n = 0; n < k; ++n) s.keep[flat[n].g] += 1;
  s.truncerr = tail[k];
  return s;
}

int Timing::record() {
  if (used == int(c->tev.size())) {
    cudaEvent_t e;
    cuda_check(cudaEventCreate(&e), "event create");
    c->tev.push_back(e);
  }
  cuda_check(cudaEventRecord(c->tev[used], c->stream), "event record");
  return used++;
}

void Timing::flush() {
  gemm.flush();
  for (const Span& sp : spans) {
    float ms = 0;
    cudaEventElapsedTime(&ms, c->tev[sp.a], c->tev[sp.b]);
    acc[sp.cat] += ms * 1e-3;
  }
  spans.clear();
  used = 0;
}

// Krylov solve: see engine_step.hpp. P.graph: everything of the solve after its first Heff
// application (which makes every scratch allocation the step needs) is captured into a CUDA graph
// and launched as one graph; the context keeps the executable graph and updates it in place from
// the next step's capture when the kernel sequence has the same shape (it does for a fixed Krylov
// dimension), so a step costs one graph update and one graph launch instead of one launch per
// kernel.
KrylovRun krylov_solve(dmrg_state* st, const dmrg_params& P, const HeffPlan& hp, int64_t n,
                       bool simple2, bool final_step, Timing& tm, StepOut& so, double tau,
                       bool expo) {
  dmrg_ctx* c = st->ctx;
  cudaStream_t s = c->stream;
  join_env(c);
  KrylovRun kr;
  kr.split = split_form(P.precision) != 0;
  const int kdim = std::max(2, std::min(P.krylov, 16));
  double* K = c->K.p;
  double* H = c->H.p;
  const bool use_graph = P.graph && !P.profile && !(c->batch && c->batch_on);
  bool capturing = false;
  auto heff = [&](const double* x, double* y) {
    const int th = tm.begin();
    apply_heff(st, hp.le, hp, x, y, P.precision, P.profile ? &tm.gemm : nullptr);
    cuda_check(cudaGetLastError(), "Heff");
    tm.end(th, 0);
    so.nmv += 1;
    so.heff_flops += hp.flops;
    if (use_graph && !capturing) {
      cuda_check(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "graph capture");
      capturing = true;
      c->capturing = true;
    }
  };

  // a breakdown (beta <= betatest) zeroes the remaining Krylov vectors instead of ending the
  // loop, and the Ritz step uses only the active ones
  double* scal = c->d_scal;
  int tv = -1;
  if (simple2) {
    // simplelanczos (algs/DMRG.jl:57-90): H is applied to AA before its normalisation
    heff(K, H);
    tv = tm.begin();
    launch_dot2(s, K, H, n, c->d_partial, scal + lz::KK);
    launch_lanczos2_orth(s, K, H, n, scal, c->d_partial);   // K /= |K|, H -= a1 K, |H|^2
    double* K1 = K + n;
    launch_next_vector(s, H, K1, n, scal, 0, P.betatest);
    cuda_check(cudaGetLastError(), "Krylov vector");
    tm.end(tv, 3);
    heff(K1, H);
    tv = tm.begin();
    launch_mdot(s, K1, 0, 1, H, n, c->d_partial, scal + lz::ALPHA + 1);
    launch_ritz(s, scal, 2, 0.0, false);
    launch_lincomb(s, K, n, 2, scal + lz::COEF, H, n);
    tm.end(tv, 3);
  } else {
    tv = tm.begin();
    launch_mdot(s, K, 0, 1, K, n, c->d_partial, scal + lz::KK);
    launch_scale_rsqrt(s, K, n, scal + lz::KK);
    tm.end(tv, 3);
    for (int jj = 0; jj < kdim; ++jj) {
      double* Kj = K + int64_t(jj) * n;
      heff(Kj, H);
      tv = tm.begin();
      launch_mdot(s, Kj, 0, 1, H, n, c->d_partial, scal + lz::ALPHA + jj);
      if (jj == kdim - 1) { tm.end(tv, 3); break; }
      launch_axpby(s, n, 0.0, scal + lz::ALPHA + jj, -1.0, Kj, 1.0, nullptr, 0, H, 0);
      if (jj > 0)
        launch_axpby(s, n, 0.0, scal + lz::BETA + jj - 1, -1.0, Kj - n, 1.0, nullptr, 0, H, 0);
      for (int pass = 0; pass < 2; ++pass) {   // full re-orthogonalisation (CGS2)
        launch_mdot(s, K, n, jj + 1, H, n, c->d_partial, scal + lz::CGS);
        launch_msub(s, K, n, jj + 1, scal + lz::CGS, H, n);
      }
      launch_mdot(s, H, 0, 1, H, n, c->d_partial, scal + lz::B2 + jj);
      launch_next_vector(s, H, K + int64_t(jj + 1) * n, n, scal, jj, P.betatest);
      tm.end(tv, 3);
    }
    tv = tm.begin();
    launch_ritz(s, scal, kdim, tau, expo);
    launch_lincomb(s, K, n, kdim, scal + lz::COEF, H, n);
    tm.end(tv, 3);
  }
  cuda_check(cudaGetLastError(), "Krylov step");
  if (capturing) {
    cudaGraph_t graph = nullptr;
    c->capturing = false;
    cuda_check(cudaStreamEndCapture(s, &graph), "graph capture end");
    bool updated = false;
    if (c->gexec) {
      cudaGraphExecUpdateResultInfo info{};
      updated = cudaGraphExecUpdate(c->gexec, graph, &info) == cudaSuccess;
      if (!updated) {
        cudaGetLastError();
        cudaGraphExecDestroy(c->gexec);
        c->gexec = nullptr;
      }
    }
    if (!updated) {
      const cudaError_t e = cudaGraphInstantiate(&c->gexec, graph, 0ull);
      if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        cuda_check(e, "graph instantiate");
      }
    }
    cudaGraphDestroy(graph);
    cuda_check(cudaGraphLaunch(c->gexec, s), "graph launch");
    c->graph_launches += 1;
  }
  // split form, last bond step of the sweep: the reported energy is the FP64 Rayleigh quotient
  // <psi|H|psi>/<psi|psi> of the Ritz vector (one FP64 matvec; the Krylov vectors are free now)
  kr.fp64_energy = kr.split && P.fp64_final && final_step && !expo;
  if (kr.fp64_energy) {
    const int th = tm.begin();
    apply_heff(st, hp.le, hp, H, K, DMRG_PREC_FP64, nullptr);
    tm.end(th, 0);
    so.nmv += 1;
    so.heff_flops += hp.flops;
    launch_dot2(s, H, K, n, c->d_partial, scal + lz::KK);
    to_host(c, c->h_scal + lz::KK, c->dv_scal ? c->dv_scal + lz::KK : nullptr, scal + lz::KK,
            2 * sizeof(double), "Rayleigh quotient D2H");
  }
  to_host(c, c->h_scal + lz::EN, c->dv_scal ? c->dv_scal + lz::EN : nullptr, scal + lz::EN,
          sizeof(double), "energy D2H");
  if (kr.split)   // timeout flag of the split GEMMs, read back with the energy (bytes of slot 20)
    to_host(c, c->h_scal + 20, c->dv_scal ? c->dv_scal + 20 : nullptr, c->d_status + STATUS_MMA,
            sizeof(int), "MMA status D2H");
  return kr;
}

void join_env(dmrg_ctx* c) {
  if (!c->env_pending) return;
  c->env_pending = false;
  cuda_check(cudaStreamWaitEvent(c->stream, c->env_join, 0), "environment join");
}

double krylov_energy(dmrg_ctx* c, const KrylovRun& kr) {
  double e = c->h_scal[lz::EN];
  if (kr.fp64_energy && c->h_scal[lz::KK] > 0) e = c->h_scal[lz::KH] / c->h_scal[lz::KK];
  if (kr.split) {
    int flag = 0;
    std::memcpy(&flag, c->h_scal + 20, sizeof(int));
    if (flag != 0) {
      cudaMemsetAsync(c->d_status + STATUS_MMA, 0, sizeof(int), c->stream);
      fail(DMRG_ERR_TIMEOUT, "split-precision GEMM: a tensor-core MMA completion wait gave up");
    }
  }
  return e;
}

void plan_rho(dmrg_ctx* c, std::vector<Group>& G, bool rows, RhoSolve& rs, int* eig_max_n) {
  // side = dimension of the density matrix that is diagonalised (rows of M, or its columns)
  rs.rows = rows;
  rs.mtot = rs.rtot = rs.wtot = 0;
  for (Group& g : G) {
    const int side = rows ? g.n : g.np;
    g.moff = rs.mtot; rs.mtot += int64_t(g.n) * g.np;
    g.roff = rs.rtot; rs.rtot += int64_t(side) * side;
    g.woff = rs.wtot; rs.wtot += side;
  }
  rs.W0 = rs.rtot;
  rs.WS0 = rs.rtot + rs.wtot;
  rs.U0 = rs.rtot + 4 * rs.wtot;
  rs.J0 = 2 * rs.rtot + 4 * rs.wtot;
  rs.etasks.clear();
  rs.ttasks.clear();
  rs.tgroup.clear();
  rs.uoff.assign(G.size(), 0);
  for (int gi = 0; gi < int(G.size()); ++gi) {
    const Group& g = G[gi];
    const int side = rows ? g.n : g.np;
    if (side == 0) continue;
    if (eig_max_n) *eig_max_n = std::max(*eig_max_n, side);
    if (side <= SYEVT_MID_NMAX) {
      TridTask t{};
      t.a_off = g.roff;
      t.w_off = rs.W0 + g.woff;
      t.ws_off = rs.WS0 + 3 * g.woff;
      t.u_off = rs.U0 + g.roff;
      t.n = side;
      rs.ttasks.push_back(t);
      rs.tgroup.push_back(gi);
      rs.uoff[gi] = t.u_off;
    } else {
      EigTask et{};
      et.a_off = g.roff;
      et.v_off = g.roff;
      et.w_off = rs.W0 + g.woff;
      et.n = side;
      rs.etasks.push_back(et);
      rs.uoff[gi] = g.roff;      // block Jacobi returns the eigenvectors in place
    }
  }
  const int64_t ews = eig_workspace(rs.etasks);
  ensure(c, c->M, std::max<int64_t>(rs.mtot, 1));
  ensure(c, c->R, std::max<int64_t>(rs.J0 + ews, 1));
  GemmList& grho = rs.grho;
  grho.clear();
  grho.tA = !rows;
  grho.tB = rows;
  for (const Group& g : G) {
    const int side = rows ? g.n : g.np;
    if (side == 0) continue;
    grho.add(g.roff, side, side, side, 1.0, 0.0);
    const int K2 = rows ? g.np : g.n;
    if (K2 > 0) grho.seg(g.moff, g.n, g.moff, g.n, K2);
  }
  tune_gemm(c, grho);
}

void launch_rho(dmrg_ctx* c, RhoSolve& rs, char* db) {
  run_gemm(c, rs.grho, db, c->M.p, c->M.n, c->M.p, c->M.n, c->R.p, c->R.n);
  run_trid_eigvals(c, c->R.p, c->R.n, rs.ttasks, 8);
  cuda_check(cudaGetLastError(), "density matrix and eigenvalue launch");
  run_eigs(c, c->R.p, c->R.n, rs.etasks, rs.J0, nullptr);
  // pinned destination: the transfer stays asynchronous and the host waits only in the step's
  // sync
  if (size_t(std::max<int64_t>(rs.wtot, 1)) > c->h_lam_cap) {
    if (c->h_lam) cudaFreeHost(c->h_lam);
    c->h_lam = nullptr;
    c->dv_lam = nullptr;
    c->h_lam_cap = 0;
    const size_t cap = std::max<size_t>(size_t(rs.wtot), 4096);
    cuda_check(cudaMallocHost(reinterpret_cast<void**>(&c->h_lam), cap * sizeof(double)),
               "pinned eigenvalue buffer");
    c->h_lam_cap = cap;
    c->dv_lam = device_view(c->h_lam);
  }
  to_host(c, c->h_lam, c->dv_lam, c->R.p + rs.W0, sizeof(double) * rs.wtot, "eigenvalues D2H");
}

std::vector<std::vector<double>> rho_values(dmrg_ctx* c, const std::vector<Group>& G,
                                            const RhoSolve& rs) {
  std::vector<std::vector<double>> vals(G.size());
  for (int g = 0; g < int(G.size()); ++g) {
    const int side = rs.rows ? G[g].n : G[g].np;
    vals[g].assign(c->h_lam + G[g].woff, c->h_lam + G[g].woff + side);
  }
  return vals;
}

void launch_rho_vectors(dmrg_ctx* c, const std::vector<Group>& G, const RhoSolve& rs) {
  std::vector<TridTask> vt;
  for (size_t a = 0; a < rs.ttasks.size(); ++a) {
    TridTask t = rs.ttasks[a];
    t.keep = G[rs.tgroup[a]].keep;
    if (t.keep > 0) vt.push_back(t);
  }
  cuda_check(cudaGetLastError(), "eigenvalue download");
  run_trid_vectors(c, c->R.p, c->R.n, vt, 6);
}

void twostep(dmrg_state* st, const dmrg_params& P, int j, int iL, int iR, bool final_step,
             Timing& tm, StepOut& so, const StepMode& mode) {
  dmrg_ctx* c = st->ctx;
  cudaStream_t s = c->stream;
  const MPOSite& ml = st->mpo->site[iL];
  const MPOSite& mr = st->mpo->site[iR];
  const Bond Bl = st->bond[iL];
  const Bond Bc = st->bond[iL + 1];
  const Bond Br = st->bond[iL + 2];
  const int d1 = ml.d, d2 = mr.d;
  if (!st->Lvalid[iL] || !st->Rvalid[iR]) fail(DMRG_ERR_STATE, "environments are not built");

  // psi[iL] (j>0) or psi[iR] (j<0) /= norm  (algs/DMRG.jl:365-369); the squared norm stays on
  // the device
  int tv = tm.begin();
  const int ic = j > 0 ? iL : iR;
  launch_mdot(s, st->A[ic].p, 0, 1, st->A[ic].p, st->lay[ic].size, c->d_partial,
              c->d_scal + lz::NRM);
  launch_scale_rsqrt(s, st->A[ic].p, st->lay[ic].size, c->d_scal + lz::NRM);
  cuda_check(cudaGetLastError(), "centre normalisation");

  HeffPlan hp;
  plan_heff(st, iL, hp);
  const TwoLayout& tl = hp.tl;
  const SiteLayout& la = st->lay[iL];
  const SiteLayout& lb = st->lay[iR];
  GemmList gaa;   // AA = contract(psiL, 3, psiR, 1)
  for (int ka = 0; ka < tl.nl; ++ka)
    for (int s1 = 0; s1 < d1; ++s1)
      for (int s2 = 0; s2 < d2; ++s2) {
        const int id = tl.idx(ka, s1, s2);
        const int kd = tl.kd[id];
        if (kd < 0) continue;
        gaa.add(tl.off[id], Bl.dim[ka], Bl.dim[ka], Br.dim[kd], 1.0, 0.0);
        const int kc = la.kb[ka * d1 + s1];
        if (kc >= 0 && lb.kb[kc * d2 + s2] == kd)
          gaa.seg(la.off[ka * d1 + s1], Bl.dim[ka], lb.off[kc * d2 + s2], Bc.dim[kc], Bc.dim[kc]);
      }
  const bool split = split_form(P.precision) != 0;
  if (split) prepare_split(hp);
  tune_gemm(c, hp.g1);
  tune_gemm(c, hp.g3);
  tune_gemm(c, gaa);
  Upload u;
  put_heff(u, hp);
  u.put(gaa);
  hp.dbase = u.send(c, 0);
  const int64_t n = tl.size;
  const int kdim = std::max(2, std::min(P.krylov, 16));
  ensure(c, c->K, std::max<int64_t>(int64_t(kdim) * n, 1));
  ensure(c, c->H, std::max<int64_t>(n, 1));
  run_gemm(c, gaa, hp.dbase, st->A[iL].p, st->A[iL].n, st->A[iR].p, st->A[iR].n, c->K.p, n);
  cuda_check(cudaGetLastError(), "two-site tensor");
  tm.end(tv, 3);

  const KrylovRun kr = mode.tdvp
      ? krylov_solve(st, P, hp, n, false, false, tm, so, mode.tau, true)
      : krylov_solve(st, P, hp, n, P.krylov <= 2, final_step, tm, so);
  const double* psi = c->H.p;

  // ---------------- reduced density matrix per centre-charge group (algs/DMRG.jl:425-429)
  const int te = tm.begin();
  std::map<QN, Group> gm;
  for (int ka = 0; ka < Bl.nsec(); ++ka)
    for (int s1 = 0; s1 < d1; ++s1) {
      Group& g = gm[Bl.q[ka] + ml.p[s1]];
      g.q = Bl.q[ka] + ml.p[s1];
      g.rows.push_back({ka, s1, g.n});
      g.n += Bl.dim[ka];
    }
  for (int kd = 0; kd < Br.nsec(); ++kd)
    for (int s2 = 0; s2 < d2; ++s2) {
      auto it = gm.find(Br.q[kd] - mr.p[s2]);
      if (it == gm.end()) continue;
      it->second.cols.push_back({kd, s2, it->second.np});
      it->second.np += Br.dim[kd];
    }
  std::vector<Group> G;
  for (auto& kv : gm) G.push_back(kv.second);
  std::vector<int> gofrow(size_t(Bl.nsec()) * d1, -1), rowoff(size_t(Bl.nsec()) * d1, 0);
  std::vector<int> coloff(size_t(Br.nsec()) * d2, -1);
  for (int g = 0; g < int(G.size()); ++g) {
    for (const Piece& p : G[g].rows) { gofrow[p.sec * d1 + p.s] = g; rowoff[p.sec * d1 + p.s] = p.off; }
    for (const Piece& p : G[g].cols) coloff[p.sec * d2 + p.s] = p.off;
  }
  RhoSolve rs;
  plan_rho(c, G, j > 0, rs, &so.eig_max_n);
  CopyList gather;
  for (int ka = 0; ka < tl.nl; ++ka)
    for (int s1 = 0; s1 < d1; ++s1)
      for (int s2 = 0; s2 < d2; ++s2) {
        const int id = tl.idx(ka, s1, s2);
        const int kd = tl.kd[id];
        if (kd < 0) continue;
        const Group& g = G[gofrow[ka * d1 + s1]];
        const int co = coloff[kd * d2 + s2];
        gather.add(tl.off[id], Bl.dim[ka], g.moff + rowoff[ka * d1 + s1] + int64_t(co) * g.n, g.n,
                   Bl.dim[ka], Br.dim[kd], 0, 1.0);
      }
  Upload u2;
  u2.put(gather);
  u2.put(rs.grho);
  char* db2 = u2.send(c, 1);
  run_copy(c, gather, db2, psi, n, c->M.p, c->M.n);
  launch_rho(c, rs, db2);
  const auto w0 = std::chrono::steady_clock::now();
  cuda_check(cudaStreamSynchronize(s), "eigen sync");
  so.wait = std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
  tuner_collect(c);
  so.energy = krylov_energy(c, kr);

  const std::vector<std::vector<double>> vals = rho_values(c, G, rs);
  // the two-site DMRG step truncates with mag = 1 (fsvd!, algs/DMRG.jl:387); the TDVP step with
  // the svd default mag = 0, weights relative to the total (its vector is not normalised)
  const Sel sel = select_kept(vals, P.maxm, P.minm, P.cutoff, mode.tdvp ? 0.0 : 1.0, P.degen_rtol);
  Bond C;
  std::vector<double> kept;
  for (int g = 0; g < int(G.size()); ++g) {
    G[g].keep = sel.keep[g];
    if (G[g].keep == 0) continue;
    G[g].kc = C.nsec();
    C.q.push_back(G[g].q);
    C.dim.push_back(G[g].keep);
    for (int a = 0; a < G[g].keep; ++a) kept.push_back(vals[g][a]);
  }
  std::sort(kept.begin(), kept.end(), std::greater<double>());
  so.D.resize(kept.size());
  for (size_t a = 0; a < kept.size(); ++a) so.D[a] = std::sqrt(std::max(kept[a], 0.0));
  so.truncerr = mode.tdvp ? (sel.total > 0 ? sel.truncerr / sel.total : 0.0) : sel.truncerr;
  so.m = int(kept.size());
  launch_rho_vectors(c, G, rs);
  const std::vector<int64_t>& uoff = rs.uoff;

  // ---------------- split back into the two site tensors (algs/DMRG.jl:389-395, 483-490)
  cuda_check(cudaGetLastError(), "eigenvectors");
  SiteLayout nl = make_site_layout(Bl, ml.p, C);
  SiteLayout nrl = make_site_layout(C, mr.p, Br);
  DBuf nA, nB;
  dalloc(c, nA, std::max<int64_t>(nl.size, 1));
  dalloc(c, nB, std::max<int64_t>(nrl.size, 1));
  CopyList cp;
  GemmList gs;
  if (j > 0) {
    gs.tA = true;
    for (int ka = 0; ka < Bl.nsec(); ++ka)
      for (int s1 = 0; s1 < d1; ++s1) {
        const int gi = gofrow[ka * d1 + s1];
        const Group& g = G[gi];
        if (g.keep == 0) continue;
        cp.add(uoff[gi] + rowoff[ka * d1 + s1], g.n, nl.off[ka * d1 + s1], Bl.dim[ka], Bl.dim[ka],
               g.keep, 0, 1.0);
      }
    for (int gi = 0; gi < int(G.size()); ++gi) {
      const Group& g = G[gi];
      if (g.keep == 0) continue;
      for (const Piece& p : g.cols) {   // p.sec = kd, p.s = s2
        if (nrl.kb[g.kc * d2 + p.s] != p.sec) continue;
        gs.add(nrl.off[g.kc * d2 + p.s], g.keep, g.keep, Br.dim[p.sec], 1.0, 0.0);
        gs.seg(uoff[gi], g.n, g.moff + int64_t(p.off) * g.n, g.n, g.n);
      }
    }
  } else {
    for (int gi = 0; gi < int(G.size()); ++gi) {
      const Group& g = G[gi];
      if (g.keep == 0) continue;
      for (const Piece& p : g.cols) {
        if (nrl.kb[g.kc * d2 + p.s] != p.sec) continue;
        cp.add(uoff[gi] + p.off, g.np, nrl.off[g.kc * d2 + p.s], g.keep, g.keep, Br.dim[p.sec], 1,
               1.0);
      }
      for (const Piece& p : g.rows) {   // p.sec = ka, p.s = s1
        gs.add(nl.off[p.sec * d1 + p.s], Bl.dim[p.sec], Bl.dim[p.sec], g.keep, 1.0, 0.0);
        if (g.np > 0) gs.seg(g.moff + p.off, g.n, uoff[gi], g.np, g.np);
      }
    }
  }
  tune_gemm(c, gs);
  Upload u3;
  u3.put(cp);
  u3.put(gs);
  char* db3 = u3.send(c, 3);
  cuda_check(cudaGetLastError(), "split upload");
  // the copy writes the site tensor that the environment update reads (nA for j > 0, nB for
  // j < 0): a sweep that overlaps its environment updates forks them off here
  if (j > 0) {
    run_copy(c, cp, db3, c->R.p, c->R.n, nA.p, nA.n);
    cuda_check(cudaGetLastError(), "split copy");
    if (c->env_overlap) cuda_check(cudaEventRecord(c->env_fork, s), "environment fork");
    run_gemm(c, gs, db3, c->R.p, c->R.n, c->M.p, c->M.n, nB.p, nB.n);
  } else {
    run_copy(c, cp, db3, c->R.p, c->R.n, nB.p, nB.n);
    cuda_check(cudaGetLastError(), "split copy");
    if (c->env_overlap) cuda_check(cudaEventRecord(c->env_fork, s), "environment fork");
    run_gemm(c, gs, db3, c->M.p, c->M.n, c->R.p, c->R.n, nA.p, nA.n);
  }
  cuda_check(cudaGetLastError(), "split");
  dfree(c, st->A[iL]);
  dfree(c, st->A[iR]);
  st->A[iL] = nA;
  st->A[iR] = nB;
  st->lay[iL] = nl;
  st->lay[iR] = nrl;
  st->bond[iL + 1] = C;
  if (j > 0) st->Rvalid[iL] = 0; else st->Lvalid[iL + 1] = 0;
  tm.end(te, 2);
}

void do_sweep(dmrg_state* st, const dmrg_params& P, dmrg_sweep_stats& out) {
  dmrg_ctx* c = st->ctx;
  const int L = st->L;
  if (L < 2) fail(DMRG_ERR_SHAPE, "a two-site sweep needs at least two sites");
  if (!st->env_built) fail(DMRG_ERR_STATE, "call dmrg_env_build before dmrg_sweep");
  std::memset(&out, 0, sizeof(out));
  c->tune = P.tune != 0;
  const long long g0 = c->graph_launches;
  const int svn = P.svnbond > 0 ? P.svnbond : (L + 1) / 2;
  const int svn_site = std::min(std::max(2, svn + 1), L) - 1;   // 0-based i of SvNcheck!
  const auto h0 = std::chrono::steady_clock::now();
  Timing tm(c, P.profile != 0);
  // Environment updates on their own stream (dmrg_ctx::env_stream), except in profiled sweeps
  // (their phase timings are taken on one stream) and in served solves (their Heff launches go
  // to the shared batcher).
  const bool overlap = !P.profile && !c->batch;
  if (overlap && !c->env_stream) {
    cuda_check(cudaStreamCreateWithFlags(&c->env_stream, cudaStreamNonBlocking), "env stream");
    cuda_check(cudaEventCreateWithFlags(&c->env_fork, cudaEventDisableTiming), "env event");
    cuda_check(cudaEventCreateWithFlags(&c->env_join, cudaEventDisableTiming), "env event");
  }
  // on every exit, errors included: the context's own stream back in place, nothing pending
  struct EnvGuard {
    dmrg_ctx* c;
    cudaStream_t main;
    ~EnvGuard() {
      c->stream = main;
      if (c->env_pending) cudaStreamWaitEvent(main, c->env_join, 0);
      c->env_pending = false;
      c->env_overlap = false;
    }
  } guard{c, c->stream};
  c->env_overlap = overlap;
  const int t0 = tm.record();
  int j = st->dir;
  const int j0 = j;
  const int nsteps = P.halfsweep ? L - 1 : 2 * (L - 1);   // halfsweep (algs/DMRG.jl:253)
  for (int ns = 0; ns < nsteps; ++ns) {
    const int i = st->oc;
    const int iL = j > 0 ? i : i - 1, iR = j > 0 ? i + 1 : i;
    StepOut so;
    twostep(st, P, j, iL, iR, ns == nsteps - 1, tm, so, StepMode{});
    const int tenv = tm.begin();
    double ef = 0.0;
    // split form: the environment updates run on the tensor cores too, except those of the
    // second half-sweep when the sweep's energy is the FP64 Rayleigh quotient (fp64_final): that
    // half-sweep builds, from the final site tensors, every environment the last bond step reads,
    // so the quotient is exact FP64 arithmetic on the final Ritz vector
    const int eprec = (split_form(P.precision) && !(P.fp64_final && (P.halfsweep || j != j0)))
                          ? P.precision : DMRG_PREC_FP64;
    if (overlap) {
      cuda_check(cudaStreamWaitEvent(c->env_stream, c->env_fork, 0), "environment fork");
      c->stream = c->env_stream;
    }
    if (j > 0) lupdate(st, i, &ef, eprec); else rupdate(st, i, &ef, eprec);
    cuda_check(cudaGetLastError(), "environment update");
    if (overlap) {
      c->stream = guard.main;
      cuda_check(cudaEventRecord(c->env_join, c->env_stream), "environment join");
      c->env_pending = true;
    }
    tm.end(tenv, 1);
    out.energy = so.energy;
    out.max_truncerr = std::max(out.max_truncerr, so.truncerr);
    out.biggest_m = std::max(out.biggest_m, so.m);
    out.n_matvec += so.nmv;
    out.wait_seconds += so.wait;
    out.heff_flops += so.heff_flops;
    out.env_flops += ef;
    out.eig_max_n = std::max(out.eig_max_n, so.eig_max_n);
    if (i == svn_site && j < 0) {
      double S = 0.0;
      for (double x : so.D) {
        const double p2 = x * x;
        if (p2 > 0) S -= p2 * std::log(p2);
      }
      out.entropy = S;
      for (int a = 0; a < 8; ++a) out.d_top[a] = a < int(so.D.size()) ? so.D[a] : 0.0;
    }
    st->oc += j;
    if ((st->oc == L - 1 && j > 0) || (st->oc == 0 && j < 0)) j = -j;
  }
  st->dir = j;
  join_env(c);
  const int t1 = tm.record();
  cuda_check(cudaEventSynchronize(tm.event(t1)), "sweep sync");
  if (split_form(P.precision)) check_mma_status(c);   // the last environment update
  tuner_collect(c);
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
}

}  // namespace dmrg
