// engine_3s.cpp -- single-site DMRG with subspace expansion ("3S") on the device: step3S
// (algs/DMRG.jl:324-360) with Lexpand / Rexpand (:273-287) and alpha_update (:289-302), the
// moves moveR! / moveL! with `condition` (lib/MPS/move.jl:124-199) in the density-matrix form,
// inside the optmps sweep (algs/optimizeMPS.jl:790-835).
//
// One bond step at site i, rightward (j > 0; the leftward step is its mirror image):
//   1. Lanczos on the single-site Heff (L[i] W[i] R[i], launches of the two-site plan with a
//      trivial second site) from psi[i]; the Ritz vector psi lands in c->H.
//   2. While alpha > noise_incr the centre is enlarged by the expansion term
//      P[a,t,(w',c)] = alpha sum L[a,w,b] psi[b,s,c] W[w,s,t,w']: the grouped GEMM X = L psi
//      (the Heff's first launch) and one MPO mixing launch that writes alpha W . X straight into
//      the expansion columns of the group matrices. Rows (a,t) are grouped by their charge; the
//      expansion column (w',c) has charge q(c) - r(w'), which may be a charge the bond lacks:
//      this is how the expansion brings new symmetry sectors into the bond.
//   3. Per group rho = M M^T, its eigensolve (shared with the two-site step), global truncation
//      with weights relative to the total (mag = 0): psi[i] = U (the kept eigenvectors), and
//      psi[i+1] <- (U^T M restricted to the original columns) psi[i+1] (two grouped GEMMs).
//   4. alpha_update on the host with the step's truncation error and energy.
// Leftward: P[(a,w),t,d] = alpha sum psi[a,s,c] W[w,s,t,w'] R[c,w',d] -- one mixing launch
// (alpha W . psi into a scratch Y laid out against R's rows) and one grouped GEMM Y R written
// into the expansion rows; rho = M^T M per column-charge group; psi[i] = V^T and
// psi[i-1] <- psi[i-1] (M restricted to the original rows) V.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <map>

#include "engine_step.hpp"

namespace dmrg {
namespace {

// alpha_update (algs/DMRG.jl:289-302), IEEE arithmetic as in the reference (a zero energy ratio
// gives an infinite or NaN site condition, never an exception).
double alpha_update(double alpha, double truncerr, double cutoff, double last_energy,
                    double energy, double noise_goal, double dalpha) {
  const bool trunc_check = truncerr <= std::max(cutoff, 1e-12);
  const bool err_est = std::fabs(energy - last_energy) <= std::max(std::fabs(energy * cutoff), 1e-12);
  const bool sitecond = std::fabs((truncerr * energy) / (last_energy / energy - 1.0)) > noise_goal;
  if (energy <= last_energy && (sitecond || err_est || trunc_check))
    alpha *= 1.0 - dalpha;
  else
    alpha *= 1.0 + dalpha;
  return std::max(std::min(alpha, 1.0), 1e-42);
}

// Global selection over the groups (mag = 0) and the new bond; fills so.D / m / truncerr.
Bond select_groups(std::vector<Group>& G, const std::vector<std::vector<double>>& vals,
                   const dmrg_params& P, StepOut& so) {
  const Sel sel = select_kept(vals, P.maxm, P.minm, P.cutoff, 0.0, P.degen_rtol);
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
  so.truncerr = sel.total > 0 ? sel.truncerr / sel.total : 0.0;
  so.m = int(kept.size());
  return C;
}

}  // namespace

void single_site_step(dmrg_state* st, const dmrg_params& P, const SiteMode& md, int j, int i,
                      bool final_step, Timing& tm, StepOut& so) {
  const double alpha = md.alpha, noise_incr = md.noise_incr;
  dmrg_ctx* c = st->ctx;
  cudaStream_t s = c->stream;
  const int L = st->L;
  const MPOSite& ms = st->mpo->site[i];
  const Bond Bl = st->bond[i];
  const Bond Br = st->bond[i + 1];
  const SiteLayout lay = st->lay[i];
  const int d = ms.d, wl = ms.wl, wr = ms.wr;
  if (!st->Lvalid[i] || !st->Rvalid[i]) fail(DMRG_ERR_STATE, "environments are not built");
  if ((j > 0 && i + 1 >= L) || (j < 0 && i < 1)) fail(DMRG_ERR_ARG, "3S step off the chain");

  // ---------------- 1. Lanczos on the single-site Heff
  int tv = tm.begin();
  HeffPlan hp;
  plan_heff1(st, i, hp);
  upload_heff(c, hp, 0, P.precision);
  const int64_t n = lay.size;
  const int kdim = std::max(2, std::min(P.krylov, 16));
  ensure(c, c->K, std::max<int64_t>(int64_t(kdim) * n, 1));
  ensure(c, c->H, std::max<int64_t>(n, 1));
  cuda_check(cudaMemcpyAsync(c->K.p, st->A[i].p, size_t(n) * sizeof(double),
                             cudaMemcpyDeviceToDevice, s), "3S start vector");
  tm.end(tv, 3);
  const KrylovRun kr = md.tdvp ? krylov_solve(st, P, hp, n, false, false, tm, so, md.tau, true)
                               : krylov_solve(st, P, hp, n, false, final_step, tm, so);
  const double* psi = c->H.p;
  const bool expand = !md.tdvp && alpha > noise_incr;   // alpha_condition (algs/DMRG.jl:335)

  const int te = tm.begin();
  std::map<QN, Group> gm;
  std::vector<Group> G;
  CopyList gather;
  MixList mexp;
  GemmList gexp;
  int64_t ytot = 0;   // doubles of the leftward expansion's scratch Y
  RhoSolve rs;
  if (j > 0) {
    // ---------------- 2. groups by row charge q(a) + p(t); original columns first
    for (int ka = 0; ka < Bl.nsec(); ++ka)
      for (int t = 0; t < d; ++t) {
        Group& g = gm[Bl.q[ka] + ms.p[t]];
        g.q = Bl.q[ka] + ms.p[t];
        g.rows.push_back({ka, t, g.n});
        g.n += Bl.dim[ka];
      }
    for (int kc = 0; kc < Br.nsec(); ++kc) {
      auto it = gm.find(Br.q[kc]);
      if (it == gm.end()) continue;
      it->second.cols.push_back({kc, -1, it->second.np});
      it->second.np += Br.dim[kc];
    }
    if (expand)
      for (int kbp = 0; kbp < Br.nsec(); ++kbp)
        for (int w2 = 0; w2 < wr; ++w2) {
          auto it = gm.find(Br.q[kbp] - ms.rr[w2]);
          if (it == gm.end()) continue;
          it->second.cols.push_back({kbp, w2, it->second.np});
          it->second.np += Br.dim[kbp];
        }
    for (auto& kv : gm) G.push_back(kv.second);
    plan_rho(c, G, true, rs, &so.eig_max_n);
    for (const Group& g : G) {
      const bool orig = !g.cols.empty() && g.cols[0].s < 0;
      for (const Piece& r : g.rows) {
        const int ka = r.sec, t = r.s;
        const int kc = lay.kb[ka * d + t];
        if (kc < 0) continue;
        if (!orig || g.cols[0].sec != kc) fail(DMRG_ERR_ARG, "internal plan check failed: 3S rows");
        gather.add(lay.off[ka * d + t], Bl.dim[ka], g.moff + r.off, g.n, Bl.dim[ka], Br.dim[kc], 0,
                   1.0);
      }
    }
    if (expand) {
      // X_kb = L_kb psi_kb (the Heff's first launch, hp.g1) has rows (a, w), columns (s, c)
      const EnvLayout& LL = st->Llay[i];
      std::vector<int64_t> xoff(Bl.nsec(), 0);
      int64_t x = 0;
      for (int kb = 0; kb < Bl.nsec(); ++kb) {
        xoff[kb] = x;
        x += int64_t(LL.rows[kb]) * lay.gcols[kb];
      }
      if (x != hp.x_size) fail(DMRG_ERR_ARG, "internal plan check failed: 3S expansion layout");
      std::vector<std::vector<const MPOSite::El*>> byTW(size_t(d) * wr);
      for (const auto& e : ms.nz) byTW[size_t(e.t) * wr + e.w2].push_back(&e);
      std::vector<MixTerm> terms;
      for (const Group& g : G)
        for (const Piece& p : g.cols) {
          if (p.s < 0) continue;
          const int kbp = p.sec, w2 = p.s;
          for (const Piece& r : g.rows) {
            const int ka = r.sec, t = r.s;
            terms.clear();
            for (const MPOSite::El* e : byTW[size_t(t) * wr + w2]) {
              const int kb = Bl.find(Bl.q[ka] + ms.rl[e->w]);
              if (kb < 0 || LL.other[kb * wl + e->w] != ka) continue;
              if (lay.kb[kb * d + e->s] != kbp) continue;
              const int64_t colA = (lay.off[kb * d + e->s] - lay.goff[kb]) / Bl.dim[kb];
              MixTerm tm{};
              tm.in_off = xoff[kb] + LL.rowoff[kb * wl + e->w] + colA * LL.rows[kb];
              tm.ld = LL.rows[kb];
              tm.coef = alpha * e->v;
              terms.push_back(tm);
            }
            if (terms.empty()) continue;
            mexp.add(g.moff + r.off + int64_t(p.off) * g.n, g.n, Bl.dim[ka], Br.dim[kbp]);
            for (const MixTerm& tm : terms) mexp.term(tm.in_off, tm.ld, tm.coef);
          }
        }
    }
  } else {
    // ---------------- 2'. groups by column charge q(d) - p(t) (t-major, so that the columns of a
    // group are those of the original row sector in site order); original rows first
    for (int t = 0; t < d; ++t)
      for (int kd = 0; kd < Br.nsec(); ++kd) {
        Group& g = gm[Br.q[kd] - ms.p[t]];
        g.q = Br.q[kd] - ms.p[t];
        g.cols.push_back({kd, t, g.np});
        g.np += Br.dim[kd];
      }
    for (int ka = 0; ka < Bl.nsec(); ++ka) {
      auto it = gm.find(Bl.q[ka]);
      if (it == gm.end()) continue;
      it->second.rows.push_back({ka, -1, it->second.n});
      it->second.n += Bl.dim[ka];
    }
    if (expand)
      for (int ka = 0; ka < Bl.nsec(); ++ka)
        for (int w = 0; w < wl; ++w) {
          auto it = gm.find(Bl.q[ka] - ms.rl[w]);
          if (it == gm.end()) continue;
          it->second.rows.push_back({ka, w, it->second.n});
          it->second.n += Bl.dim[ka];
        }
    for (auto& kv : gm) G.push_back(kv.second);
    plan_rho(c, G, false, rs, &so.eig_max_n);
    for (const Group& g : G) {
      if (g.rows.empty() || g.rows[0].s >= 0) continue;
      const int ka = g.rows[0].sec;
      if (lay.gcols[ka] != g.np) fail(DMRG_ERR_ARG, "internal plan check failed: 3S columns");
      if (g.np > 0) gather.add(lay.goff[ka], Bl.dim[ka], g.moff, g.n, Bl.dim[ka], g.np, 0, 1.0);
    }
    if (expand) {
      // Y_(ka,w,t)[a, (c,w')] = alpha sum_s W[w,s,t,w'] psi_(ka,s)[a,c], its columns laid out as
      // the rows of R_kd (kd the bra sector of q(ka) - r(w) + p(t)); then P = Y R_kd
      const EnvLayout& RL = st->Rlay[i];
      std::vector<std::vector<const MPOSite::El*>> byWTW(size_t(wl) * d * wr);
      for (const auto& e : ms.nz) byWTW[(size_t(e.w) * d + e.t) * wr + e.w2].push_back(&e);
      std::map<std::pair<int, int>, std::pair<int, int>> colpiece;   // (group, t) -> (kd, off)
      for (int gi = 0; gi < int(G.size()); ++gi)
        for (const Piece& p : G[gi].cols) colpiece[{gi, p.s}] = {p.sec, p.off};
      int64_t y = 0;
      for (int gi = 0; gi < int(G.size()); ++gi) {
        const Group& g = G[gi];
        for (const Piece& r : g.rows) {
          if (r.s < 0) continue;
          const int ka = r.sec, w = r.s;
          for (int t = 0; t < d; ++t) {
            auto it = colpiece.find({gi, t});
            if (it == colpiece.end()) continue;
            const int kd = it->second.first, coff = it->second.second;
            if (RL.rows[kd] == 0) continue;
            const int64_t yoff = y;
            y += int64_t(Bl.dim[ka]) * RL.rows[kd];
            for (int w2 = 0; w2 < wr; ++w2) {
              const int kc = RL.other[kd * wr + w2];
              if (kc < 0) continue;
              bool any = false;
              for (const MPOSite::El* e : byWTW[(size_t(w) * d + t) * wr + w2])
                if (lay.kb[ka * d + e->s] == kc) { any = true; break; }
              if (!any) continue;
              mexp.add(yoff + int64_t(RL.rowoff[kd * wr + w2]) * Bl.dim[ka], Bl.dim[ka], Bl.dim[ka],
                       Br.dim[kc]);
              for (const MPOSite::El* e : byWTW[(size_t(w) * d + t) * wr + w2])
                if (lay.kb[ka * d + e->s] == kc)
                  mexp.term(lay.off[ka * d + e->s], Bl.dim[ka], alpha * e->v);
            }
            gexp.add(g.moff + r.off + int64_t(coff) * g.n, g.n, Bl.dim[ka], Br.dim[kd], 1.0, 0.0);
            gexp.seg(yoff, Bl.dim[ka], RL.goff[kd], RL.rows[kd], RL.rows[kd]);
          }
        }
      }
      ytot = y;
      ensure(c, c->Y, std::max<int64_t>(y, 1));
      tune_gemm(c, gexp);
    }
  }

  Upload u2;
  u2.put(gather);
  u2.put(mexp);
  u2.put(gexp);
  u2.put(rs.grho);
  char* db2 = u2.send(c, 1);
  cuda_check(cudaMemsetAsync(c->M.p, 0, size_t(std::max<int64_t>(rs.mtot, 1)) * sizeof(double), s),
             "3S group matrices");
  run_copy(c, gather, db2, psi, n, c->M.p, c->M.n);
  if (expand && j > 0) {
    ensure(c, c->X, std::max<int64_t>(hp.x_size, 1));
    run_gemm(c, hp.g1, hp.dbase, st->Lenv[i].p, st->Lenv[i].n, psi, n, c->X.p, c->X.n);
    run_mix(c, mexp, db2, c->X.p, c->X.n, c->M.p, c->M.n);
  } else if (expand) {
    cuda_check(cudaMemsetAsync(c->Y.p, 0, size_t(ytot) * sizeof(double), s), "3S expansion");
    run_mix(c, mexp, db2, psi, n, c->Y.p, c->Y.n);
    run_gemm(c, gexp, db2, c->Y.p, c->Y.n, st->Renv[i].p, st->Renv[i].n, c->M.p, c->M.n);
  }
  cuda_check(cudaGetLastError(), "3S expansion");
  launch_rho(c, rs, db2);
  const auto w0 = std::chrono::steady_clock::now();
  cuda_check(cudaStreamSynchronize(s), "eigen sync");
  so.wait = std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
  tuner_collect(c);
  so.energy = krylov_energy(c, kr);

  // ---------------- 3. truncation and the new site tensors
  const std::vector<std::vector<double>> vals = rho_values(c, G, rs);
  const Bond C = select_groups(G, vals, P, so);
  launch_rho_vectors(c, G, rs);
  const std::vector<int64_t>& uoff = rs.uoff;
  CopyList cp;
  GemmList gv, gn;   // U^T M_orig (or M_orig V), then its product with the neighbour site
  DBuf nC, nN;       // new centre-side tensor psi[i], new neighbour psi[i+j]
  const int in = i + j;
  const MPOSite& mn = st->mpo->site[in];
  const SiteLayout& lo = st->lay[in];
  SiteLayout nlc, nln;
  int64_t vtot = 0;
  if (j > 0) {
    nlc = make_site_layout(Bl, ms.p, C);
    nln = make_site_layout(C, mn.p, st->bond[i + 2]);
    for (int gi = 0; gi < int(G.size()); ++gi) {
      const Group& g = G[gi];
      if (g.keep == 0) continue;
      for (const Piece& r : g.rows) {
        const int ka = r.sec, t = r.s;
        if (nlc.kb[ka * d + t] != g.kc) fail(DMRG_ERR_ARG, "internal plan check failed: 3S left");
        cp.add(uoff[gi] + r.off, g.n, nlc.off[ka * d + t], Bl.dim[ka], Bl.dim[ka], g.keep, 0, 1.0);
      }
      if (g.cols.empty() || g.cols[0].s >= 0) continue;   // a new sector: zero in psi[i+1]
      const int kc = g.cols[0].sec;
      if (nln.gcols[g.kc] != lo.gcols[kc]) fail(DMRG_ERR_ARG, "internal plan check failed: 3S right");
      gv.tA = true;
      gv.add(vtot, g.keep, g.keep, Br.dim[kc], 1.0, 0.0);
      gv.seg(uoff[gi], g.n, g.moff, g.n, g.n);
      if (lo.gcols[kc] > 0) {
        gn.add(nln.goff[g.kc], g.keep, g.keep, lo.gcols[kc], 1.0, 0.0);
        gn.seg(vtot, g.keep, lo.goff[kc], Br.dim[kc], Br.dim[kc]);
      }
      vtot += int64_t(g.keep) * Br.dim[kc];
    }
  } else {
    const Bond& B0 = st->bond[i - 1];
    const int d0 = mn.d;
    nlc = make_site_layout(C, ms.p, Br);
    nln = make_site_layout(B0, mn.p, C);
    std::vector<int> gof(Bl.nsec(), -1);
    std::vector<int64_t> voff(Bl.nsec(), -1);
    for (int gi = 0; gi < int(G.size()); ++gi) {
      const Group& g = G[gi];
      if (g.keep == 0) continue;
      for (const Piece& p : g.cols) {
        const int kd = p.sec, t = p.s;
        if (nlc.kb[g.kc * d + t] != kd) fail(DMRG_ERR_ARG, "internal plan check failed: 3S right");
        cp.add(uoff[gi] + p.off, g.np, nlc.off[g.kc * d + t], g.keep, g.keep, Br.dim[kd], 1, 1.0);
      }
      if (g.rows.empty() || g.rows[0].s >= 0) continue;   // a new sector: zero in psi[i-1]
      const int ka = g.rows[0].sec;
      gof[ka] = gi;
      voff[ka] = vtot;
      gv.add(vtot, Bl.dim[ka], Bl.dim[ka], g.keep, 1.0, 0.0);
      if (g.np > 0) gv.seg(g.moff, g.n, uoff[gi], g.np, g.np);
      vtot += int64_t(Bl.dim[ka]) * g.keep;
    }
    for (int kx = 0; kx < B0.nsec(); ++kx)
      for (int s0 = 0; s0 < d0; ++s0) {
        const int ka = lo.kb[kx * d0 + s0];
        if (ka < 0 || gof[ka] < 0) continue;
        const Group& g = G[gof[ka]];
        if (nln.kb[kx * d0 + s0] != g.kc) fail(DMRG_ERR_ARG, "internal plan check failed: 3S left");
        gn.add(nln.off[kx * d0 + s0], B0.dim[kx], B0.dim[kx], g.keep, 1.0, 0.0);
        gn.seg(lo.off[kx * d0 + s0], B0.dim[kx], voff[ka], Bl.dim[ka], Bl.dim[ka]);
      }
  }
  tune_gemm(c, gv);
  tune_gemm(c, gn);
  Upload u3;
  u3.put(cp);
  u3.put(gv);
  u3.put(gn);
  char* db3 = u3.send(c, 3);
  // the bond matrix (U^T M or M V, restricted to the original states): T1 in the 3S step; in the
  // TDVP step the start vector of its Krylov exponential, c->K (the environment update that comes
  // first uses T1 as scratch)
  DBuf& bmb = md.tdvp ? c->K : c->T1;
  ensure(c, bmb, std::max<int64_t>(md.tdvp ? int64_t(kdim) * vtot : vtot, 1));
  dalloc(c, nC, std::max<int64_t>(nlc.size, 1));
  dalloc(c, nN, std::max<int64_t>(nln.size, 1));
  cuda_check(cudaMemsetAsync(nN.p, 0, size_t(nN.n) * sizeof(double), s), "3S neighbour");
  run_copy(c, cp, db3, c->R.p, c->R.n, nC.p, nC.n);
  if (j > 0)
    run_gemm(c, gv, db3, c->R.p, c->R.n, c->M.p, c->M.n, bmb.p, bmb.n);
  else
    run_gemm(c, gv, db3, c->M.p, c->M.n, c->R.p, c->R.n, bmb.p, bmb.n);
  const Bond Bold = j > 0 ? Br : Bl;
  dfree(c, st->A[i]);
  st->A[i] = nC;
  st->lay[i] = nlc;
  st->bond[j > 0 ? i + 1 : i] = C;
  const double* bm = bmb.p;
  int64_t bmn = bmb.n;
  if (md.tdvp) {
    // tdvp (algs/time.jl:244-274): the environment across the new bond, then the bond matrix
    // evolved by exp(tau H0) with the zero-site Heff (OC_update, :205-209) between Lenv and Renv
    double ef = 0.0;
    if (j > 0) lupdate(st, i, &ef, P.precision); else rupdate(st, i, &ef, P.precision);
    so.env_flops += ef;
    HeffPlan hz;
    const int le = j > 0 ? i + 1 : i, re = j > 0 ? i : i - 1;
    plan_heff_bond(st, le, re, j > 0 ? C : Bold, j > 0 ? Bold : C, hz);
    if (hz.tl.size != vtot) fail(DMRG_ERR_ARG, "internal plan check failed: TDVP bond matrix");
    upload_heff(c, hz, 0, P.precision);
    ensure(c, c->H, std::max<int64_t>(vtot, 1));
    krylov_solve(st, P, hz, vtot, false, false, tm, so, md.tau, true);
    bm = c->H.p;
    bmn = c->H.n;
  }
  if (j > 0)
    run_gemm(c, gn, db3, bm, bmn, st->A[in].p, st->A[in].n, nN.p, nN.n);
  else
    run_gemm(c, gn, db3, st->A[in].p, st->A[in].n, bm, bmn, nN.p, nN.n);
  cuda_check(cudaGetLastError(), "single-site move");
  dfree(c, st->A[in]);
  st->A[in] = nN;
  st->lay[in] = nln;
  // environments that read a changed tensor and are not rebuilt by this step's update
  if (j > 0) {
    st->Rvalid[i] = 0;
    if (i + 2 < L) st->Lvalid[i + 2] = 0;
  } else {
    st->Lvalid[i] = 0;
    if (i >= 2) st->Rvalid[i - 2] = 0;
  }
  tm.end(te, 2);
}

void do_sweep3s(dmrg_state* st, const dmrg_params& P, const dmrg_noise& nz, double* noise,
                double last_energy, dmrg_sweep_stats& out) {
  dmrg_ctx* c = st->ctx;
  const int L = st->L;
  if (L < 2) fail(DMRG_ERR_SHAPE, "a 3S sweep needs at least two sites");
  if (!st->env_built) fail(DMRG_ERR_STATE, "call dmrg_env_build before dmrg_sweep3s");
  if (!(nz.noise_incr >= 0.0) || !(nz.noise_incr < 1.0) || !(*noise >= 0.0))
    fail(DMRG_ERR_ARG, "noise: alpha >= 0 and 0 <= noise_incr < 1");
  std::memset(&out, 0, sizeof(out));
  c->tune = P.tune != 0;
  const long long g0 = c->graph_launches;
  const int svn = P.svnbond > 0 ? P.svnbond : (L + 1) / 2;
  const int svn_site = std::min(std::max(2, svn + 1), L) - 1;   // 0-based i of SvNcheck!
  const auto h0 = std::chrono::steady_clock::now();
  Timing tm(c, P.profile != 0);
  const int t0 = tm.record();
  int j = st->dir;
  const int j0 = j;
  double alpha = *noise;
  const int nsteps = P.halfsweep ? L - 1 : 2 * (L - 1);   // halfsweep (algs/DMRG.jl:253)
  for (int ns = 0; ns < nsteps; ++ns) {
    const int i = st->oc;
    StepOut so;
    SiteMode md;
    md.alpha = alpha;
    md.noise_incr = nz.noise_incr;
    single_site_step(st, P, md, j, i, ns == nsteps - 1, tm, so);
    alpha = alpha_update(alpha, so.truncerr, P.cutoff, last_energy, so.energy, nz.noise_goal,
                         nz.noise_incr);
    const int tenv = tm.begin();
    double ef = 0.0;
    const int eprec = (split_form(P.precision) && !(P.fp64_final && (P.halfsweep || j != j0)))
                          ? P.precision : DMRG_PREC_FP64;
    if (j > 0) lupdate(st, i, &ef, eprec); else rupdate(st, i, &ef, eprec);
    cuda_check(cudaGetLastError(), "environment update");
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
  *noise = alpha;
  const int t1 = tm.record();
  cuda_check(cudaEventSynchronize(tm.event(t1)), "sweep sync");
  if (split_form(P.precision)) check_mma_status(c);
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
