// engine_contract.cpp -- the effective Hamiltonian and the environment updates as block plans.
//
// Heff psi (make2site / inline form, algs/DMRG.jl:48-54,69-73) in three launches:
//   1. X_kb = L_kb * psi_kb          one GEMM per ket sector kb (rows (a,w), cols (s1,s2,d))
//   2. Y = ops . X                   sparse two-site MPO ops[w,s1,t1,s2,t2,w''] mixing of blocks
//   3. psi'_(ka,t1,t2) = Y * R_ka'   one GEMM per output block, K = the stacked (d, w'') rows
// Lupdate / Rupdate (lib/MPO_MPS/Lupdate.jl:17-26, Rupdate.jl:17-26) in the same three shapes.
#include <algorithm>
#include <atomic>
#include <map>

#include "engine.hpp"

namespace dmrg {

namespace {
// Heff plan over the sites' combined physical index (p1, p2), between bonds Bl and Br, with the
// MPO bond labels rl of the left MPO site, the combined operator op, and the environments' layouts
void plan_heff_core(const Bond& Bl, const Bond& Br, const std::vector<QN>& p1,
                    const std::vector<QN>& p2, const std::vector<QN>& rl, const TwoSiteOp& op,
                    const EnvLayout& LL, const EnvLayout& RL, HeffPlan& hp);
}  // namespace

void plan_heff(const dmrg_state* st, int iL, HeffPlan& hp) {
  const int iR = iL + 1;
  hp.le = iL;
  hp.re = iR;
  plan_heff_core(st->bond[iL], st->bond[iL + 2], st->mpo->site[iL].p, st->mpo->site[iR].p,
                 st->mpo->site[iL].rl, st->mpo->two[iL], st->Llay[iL], st->Rlay[iR], hp);
}

void plan_heff1(const dmrg_state* st, int i, HeffPlan& hp) {
  static const std::vector<QN> trivial(1, QN());
  hp.le = i;
  hp.re = i;
  plan_heff_core(st->bond[i], st->bond[i + 1], st->mpo->site[i].p, trivial, st->mpo->site[i].rl,
                 st->mpo->one[i], st->Llay[i], st->Rlay[i], hp);
  if (hp.tl.size != st->lay[i].size)
    fail(DMRG_ERR_ARG, "internal plan check failed: single-site Heff layout");
}

void plan_heff_bond(const dmrg_state* st, int le, int re, const Bond& Bl, const Bond& Br,
                    HeffPlan& hp) {
  static const std::vector<QN> trivial(1, QN());
  if (le != re + 1 || re < 0 || le >= st->L) fail(DMRG_ERR_ARG, "zero-site Heff: bad bond");
  const MPOSite& ms = st->mpo->site[le];
  TwoSiteOp op;   // identity on the MPO bond
  op.d1 = op.d2 = 1;
  op.wl = op.wr = ms.wl;
  op.out.assign(size_t(ms.wl), {});
  for (int w = 0; w < ms.wl; ++w) op.out[w].push_back({w, 0, 0, 1.0});
  hp.le = le;
  hp.re = re;
  plan_heff_core(Bl, Br, trivial, trivial, ms.rl, op, st->Llay[le], st->Rlay[re], hp);
}

namespace {
void plan_heff_core(const Bond& Bl, const Bond& Br, const std::vector<QN>& p1,
                    const std::vector<QN>& p2, const std::vector<QN>& rl, const TwoSiteOp& op,
                    const EnvLayout& LL, const EnvLayout& RL, HeffPlan& hp) {
  hp.tl = make_two_layout(Bl, p1, p2, Br);
  const TwoLayout& tl = hp.tl;
  const int d1 = tl.d1, d2 = tl.d2, wl = op.wl, wr = op.wr;

  hp.g1.clear();
  hp.g3.clear();
  hp.mix.clear();
  hp.g1.tA = hp.g1.tB = false;
  hp.g3.tA = hp.g3.tB = false;

  std::vector<int64_t> xoff(Bl.nsec(), 0);
  int64_t x = 0;
  for (int kb = 0; kb < Bl.nsec(); ++kb) {
    xoff[kb] = x;
    x += int64_t(LL.rows[kb]) * tl.gcols[kb];
  }
  hp.x_size = x;
  for (int kb = 0; kb < Bl.nsec(); ++kb) {
    if (LL.rows[kb] == 0 || tl.gcols[kb] == 0) continue;
    hp.g1.add(xoff[kb], LL.rows[kb], LL.rows[kb], tl.gcols[kb], 1.0, 0.0);
    hp.g1.seg(LL.goff[kb], LL.rows[kb], tl.goff[kb], Bl.dim[kb], Bl.dim[kb]);
  }

  std::vector<int64_t> yoff(tl.kd.size(), -1);
  int64_t y = 0;
  for (int ka = 0; ka < tl.nl; ++ka)
    for (int t1 = 0; t1 < d1; ++t1)
      for (int t2 = 0; t2 < d2; ++t2) {
        const int id = tl.idx(ka, t1, t2);
        const int kap = tl.kd[id];
        if (kap < 0) continue;
        yoff[id] = y;
        y += int64_t(Bl.dim[ka]) * RL.rows[kap];
      }
  hp.y_size = y;

  for (int ka = 0; ka < tl.nl; ++ka) {
    const int dka = Bl.dim[ka];
    for (int t1 = 0; t1 < d1; ++t1)
      for (int t2 = 0; t2 < d2; ++t2) {
        const int id = tl.idx(ka, t1, t2);
        const int kap = tl.kd[id];
        if (kap < 0) continue;
        for (int w2 = 0; w2 < wr; ++w2) {
          const int kd = RL.other[kap * wr + w2];
          if (kd < 0) continue;
          hp.mix.add(yoff[id] + int64_t(RL.rowoff[kap * wr + w2]) * dka, dka, dka, Br.dim[kd]);
          for (const auto& tm : op.out[(size_t(t1) * d2 + t2) * wr + w2]) {
            const int kb = Bl.find(Bl.q[ka] + rl[tm.w]);
            if (kb < 0 || LL.other[kb * wl + tm.w] != ka) continue;
            const int id2 = tl.idx(kb, tm.s1, tm.s2);
            if (tl.kd[id2] != kd) continue;
            const int64_t colX = (tl.off[id2] - tl.goff[kb]) / Bl.dim[kb];
            hp.mix.term(xoff[kb] + LL.rowoff[kb * wl + tm.w] + colX * LL.rows[kb], LL.rows[kb],
                        tm.c);
          }
        }
      }
  }

  for (int ka = 0; ka < tl.nl; ++ka)
    for (int t1 = 0; t1 < d1; ++t1)
      for (int t2 = 0; t2 < d2; ++t2) {
        const int id = tl.idx(ka, t1, t2);
        const int kap = tl.kd[id];
        if (kap < 0) continue;
        hp.g3.add(tl.off[id], Bl.dim[ka], Bl.dim[ka], Br.dim[kap], 1.0, 0.0);
        if (RL.rows[kap] > 0)
          hp.g3.seg(yoff[id], Bl.dim[ka], RL.goff[kap], RL.rows[kap], RL.rows[kap]);
      }
  hp.flops = hp.g1.flops + hp.g3.flops + hp.mix.flops;
  static std::atomic<uint64_t> next_gen{1};
  hp.gen = next_gen.fetch_add(1);
  hp.split = hp.fused = false;
}
}  // namespace

void check_mma_status(dmrg_ctx* c) {
  int flag = 0;
  cuda_check(cudaMemcpy(&flag, c->d_status + STATUS_MMA, sizeof(int), cudaMemcpyDeviceToHost),
             "MMA status");
  if (flag != 0) {
    cudaMemset(c->d_status + STATUS_MMA, 0, sizeof(int));
    fail(DMRG_ERR_TIMEOUT, "split-precision GEMM: a tensor-core MMA completion wait gave up");
  }
}

// The mixing fused into the image pack of g3t's A panels (windows of the mixed blocks Y): each
// panel gets the mixing tasks that write its columns, in column order. False when g3t is not
// image-fed or some panel is not tiled exactly by them; the plan then keeps the mixing launch.
static bool plan_fusion(HeffPlan& hp) {
  const GemmList& g = hp.g3t;
  hp.fuse_range.assign(g.pa.size(), make_int2(0, 0));
  hp.fuse_cover.clear();
  if (g.bn == TF32_TILE_N_DIRECT || g.pa.empty()) return false;
  std::vector<std::pair<int64_t, int>> outs;   // (out_off, mixing task), written tasks only
  for (int i = 0; i < int(hp.mix.tasks.size()); ++i)
    if (hp.mix.tasks[i].rows > 0 && hp.mix.tasks[i].cols > 0)
      outs.emplace_back(hp.mix.tasks[i].out_off, i);
  std::sort(outs.begin(), outs.end());
  for (size_t pi = 0; pi < g.pa.size(); ++pi) {
    const ImgPanel& p = g.pa[pi];
    if (p.kcontig) return false;
    const int64_t end = p.off + int64_t(p.ld) * p.K;
    auto it = std::lower_bound(outs.begin(), outs.end(), std::make_pair(p.off, -1));
    hp.fuse_range[pi].x = int(hp.fuse_cover.size());
    int next = 0;
    for (; it != outs.end() && it->first < end; ++it) {
      const MixTask& t = hp.mix.tasks[it->second];
      if (t.ld != p.ld || t.rows != p.rows || (t.out_off - p.off) % p.ld != 0) return false;
      if ((t.out_off - p.off) / p.ld != next) return false;
      hp.fuse_cover.push_back(MixCover{next, t.cols, t.term0, t.nterm});
      next += t.cols;
    }
    if (next != p.K) return false;
    hp.fuse_range[pi].y = int(hp.fuse_cover.size()) - hp.fuse_range[pi].x;
  }
  return true;
}

void prepare_split(HeffPlan& hp) {
  hp.g1t = retile(hp.g1, TF32_TILE_M, split_tile_n(hp.g1));
  hp.g3t = retile(hp.g3, TF32_TILE_M, split_tile_n(hp.g3));
  hp.split = true;
  hp.fused = plan_fusion(hp);
}

void upload_heff(dmrg_ctx* c, HeffPlan& hp, int slot, int precision) {
  if (split_form(precision) && !hp.split) prepare_split(hp);
  tune_gemm(c, hp.g1);
  tune_gemm(c, hp.g3);
  Upload u;
  put_heff(u, hp);
  hp.dbase = u.send(c, slot);
}

void put_heff(Upload& u, HeffPlan& hp) {
  u.put(hp.g1);
  u.put(hp.mix);
  u.put(hp.g3);
  if (hp.split) {
    u.put(hp.g1t);
    u.put(hp.g3t);
    if (hp.fused) {
      hp.fr_off = u.put(hp.fuse_range);
      hp.fc_off = u.put(hp.fuse_cover);
    }
  }
}

void GemmProfile::begin(cudaStream_t s, double fl) {
  if (used == int(pool.size())) {
    cudaEvent_t a, b;
    cuda_check(cudaEventCreate(&a), "event");
    cuda_check(cudaEventCreate(&b), "event");
    pool.push_back(a);
    pool.push_back(b);
  }
  cudaEventRecord(pool[used], s);
  pending.push_back({used, fl});
  used += 2;
}
void GemmProfile::end(cudaStream_t s) { cudaEventRecord(pool[pending.back().first + 1], s); }
void GemmProfile::flush() {
  for (auto& pr : pending) {
    float ms = 0;
    cudaEventElapsedTime(&ms, pool[pr.first], pool[pr.first + 1]);
    seconds += ms * 1e-3;
    flops += pr.second;
    launches += 1;
  }
  pending.clear();
  used = 0;
}
GemmProfile::~GemmProfile() { for (auto e : pool) cudaEventDestroy(e); }

void apply_heff(dmrg_state* st, int iL, const HeffPlan& hp, const double* x, double* y,
                int precision, GemmProfile* prof) {
  dmrg_ctx* c = st->ctx;
  if (c->batch && c->batch_on) {   // a served solve: the server's shared launch
    batched_heff(c, st, iL, hp, x, y, precision);
    return;
  }
  ensure(c, c->X, std::max<int64_t>(hp.x_size, 1));
  ensure(c, c->Y, std::max<int64_t>(hp.y_size, 1));
  const int64_t n = hp.tl.size;
  // split forms: the two GEMM steps on a tensor-core split kernel; the MPO mixing stays FP64
  const int split = split_form(precision);
  if (split && !hp.split) fail(DMRG_ERR_STATE, "split-precision Heff lists were not uploaded");
  if (precision != DMRG_PREC_FP64 && !split)
    fail(DMRG_ERR_ARG, "precision: FP64, 3xTF32 and BF16x9 are the built forms");
  // split forms: the environments' images are packed once per plan (the first application)
  // and kept while this plan's applications follow one another; with the fused form the mixing
  // happens inside the pack of the second GEMM's operand
  const uint64_t want = hp.gen * 4 + uint64_t(split);
  if (prof) prof->begin(c->stream, hp.g1.flops);
  if (split) {
    SplitOpts o1;
    o1.a = ImgCache{&c->SL, &c->sl_key, want};
    run_gemm_split(c, hp.g1t, hp.dbase, st->Lenv[hp.le].p, st->Lenv[hp.le].n, x, n, c->X.p,
                   c->X.n, split, &o1);
  } else {
    run_gemm(c, hp.g1, hp.dbase, st->Lenv[hp.le].p, st->Lenv[hp.le].n, x, n, c->X.p, c->X.n);
  }
  if (prof) prof->end(c->stream);
  const bool fused = split && hp.fused;
  if (!fused) run_mix(c, hp.mix, hp.dbase, c->X.p, c->X.n, c->Y.p, c->Y.n);
  if (prof) prof->begin(c->stream, hp.g3.flops);
  if (split) {
    SplitOpts o3;
    o3.b = ImgCache{&c->SR, &c->sr_key, want};
    o3.fuse = fused ? &hp : nullptr;
    run_gemm_split(c, hp.g3t, hp.dbase, fused ? c->X.p : c->Y.p, fused ? c->X.n : c->Y.n,
                   st->Renv[hp.re].p, st->Renv[hp.re].n, y, n, split, &o3);
  } else
    run_gemm(c, hp.g3, hp.dbase, c->Y.p, c->Y.n, st->Renv[hp.re].p, st->Renv[hp.re].n, y, n);
  if (prof) prof->end(c->stream);
}

// ------------------------------------------------------------------ environments

void env_boundaries(dmrg_state* st) {
  dmrg_ctx* c = st->ctx;
  const int L = st->L;
  const Bond& b0 = st->bond[0];
  const Bond& bL = st->bond[L];
  const MPOSite& s0 = st->mpo->site[0];
  const MPOSite& sL = st->mpo->site[L - 1];
  if (b0.nsec() != 1 || b0.dim[0] != 1 || bL.nsec() != 1 || bL.dim[0] != 1)
    fail(DMRG_ERR_SHAPE, "edge bonds of the MPS must be one-dimensional");
  if (s0.wl != 1 || sL.wr != 1)
    fail(DMRG_ERR_SHAPE, "edge bonds of the MPO must be one-dimensional");
  st->Llay[0] = make_left_env_layout(b0, s0.rl);
  st->Rlay[L - 1] = make_right_env_layout(bL, sL.rr);
  if (st->Llay[0].other[0] != 0 || st->Rlay[L - 1].other[0] != 0)
    fail(DMRG_ERR_QN, "MPO edge labels do not connect the MPS edge sectors");
  const double one = 1.0;
  dalloc(c, st->Lenv[0], 1);
  dalloc(c, st->Renv[L - 1], 1);
  cuda_check(cudaMemcpyAsync(st->Lenv[0].p, &one, sizeof(double), cudaMemcpyHostToDevice, c->stream),
             "boundary");
  cuda_check(cudaMemcpyAsync(st->Renv[L - 1].p, &one, sizeof(double), cudaMemcpyHostToDevice,
                             c->stream), "boundary");
  cuda_check(cudaStreamSynchronize(c->stream), "boundary sync");
  st->Lvalid.assign(L, 0);
  st->Rvalid.assign(L, 0);
  st->Lvalid[0] = 1;
  st->Rvalid[L - 1] = 1;
}

void plan_left_step(const Bond& Bl, const Bond& Br, const MPOSite& ms, const SiteLayout& lay,
                    const EnvLayout& LL, StepPlan& sp) {
  sp.out = make_left_env_layout(Br, ms.rr);
  const EnvLayout& LN = sp.out;
  const int d = ms.d, wl = ms.wl, wr = ms.wr;

  GemmList& g1 = sp.g1;
  GemmList& g3 = sp.g3;
  MixList& mx = sp.mx;
  g1.clear();
  g3.clear();
  mx.clear();
  g3.tA = true;
  std::vector<int64_t> t1off(Bl.nsec(), 0);
  int64_t& t1 = sp.t1;
  t1 = 0;
  for (int kb = 0; kb < Bl.nsec(); ++kb) {
    t1off[kb] = t1;
    t1 += int64_t(LL.rows[kb]) * lay.gcols[kb];
  }
  for (int kb = 0; kb < Bl.nsec(); ++kb) {
    if (LL.rows[kb] == 0 || lay.gcols[kb] == 0) continue;
    g1.add(t1off[kb], LL.rows[kb], LL.rows[kb], lay.gcols[kb], 1.0, 0.0);
    g1.seg(LL.goff[kb], LL.rows[kb], lay.goff[kb], Bl.dim[kb], Bl.dim[kb]);
  }
  // non-zeros grouped by (t, w')
  std::vector<std::vector<const MPOSite::El*>> byTW(size_t(d) * wr);
  for (const auto& e : ms.nz) byTW[size_t(e.t) * wr + e.w2].push_back(&e);

  struct Out { int kbp, w2, rows; int64_t off; std::vector<int> ka, roff; };
  std::vector<Out> outs;
  int64_t& t2 = sp.t2;
  t2 = 0;
  for (int kbp = 0; kbp < Br.nsec(); ++kbp)
    for (int w2 = 0; w2 < wr; ++w2) {
      const int kap = LN.other[kbp * wr + w2];
      if (kap < 0) continue;
      Out o{kbp, w2, 0, t2, std::vector<int>(d, -1), std::vector<int>(d, 0)};
      for (int t = 0; t < d; ++t) {
        const int ka = Bl.find(Br.q[kap] - ms.p[t]);
        if (ka < 0 || lay.kb[ka * d + t] != kap) continue;
        o.ka[t] = ka;
        o.roff[t] = o.rows;
        o.rows += Bl.dim[ka];
      }
      t2 += int64_t(o.rows) * Br.dim[kbp];
      outs.push_back(std::move(o));
    }
  for (const Out& o : outs) {
    for (int t = 0; t < d; ++t) {
      const int ka = o.ka[t];
      if (ka < 0) continue;
      mx.add(o.off + o.roff[t], o.rows, Bl.dim[ka], Br.dim[o.kbp]);
      for (const MPOSite::El* e : byTW[size_t(t) * wr + o.w2]) {
        const int kb = Bl.find(Bl.q[ka] + ms.rl[e->w]);
        if (kb < 0 || LL.other[kb * wl + e->w] != ka) continue;
        if (lay.kb[kb * d + e->s] != o.kbp) continue;
        const int64_t colA = (lay.off[kb * d + e->s] - lay.goff[kb]) / Bl.dim[kb];
        mx.term(t1off[kb] + LL.rowoff[kb * wl + e->w] + colA * LL.rows[kb], LL.rows[kb], e->v);
      }
    }
  }
  for (const Out& o : outs) {
    const int kap = LN.other[o.kbp * wr + o.w2];
    g3.add(LN.goff[o.kbp] + LN.rowoff[o.kbp * wr + o.w2], LN.rows[o.kbp], Br.dim[kap],
           Br.dim[o.kbp], 1.0, 0.0);
    for (int t = 0; t < d; ++t) {
      const int ka = o.ka[t];
      if (ka < 0) continue;
      g3.seg(lay.off[ka * d + t], Bl.dim[ka], o.off + o.roff[t], o.rows, Bl.dim[ka]);
    }
  }
}

void plan_right_step(const Bond& Bl, const Bond& Br, const MPOSite& ms, const SiteLayout& lay,
                     const EnvLayout& RL, StepPlan& sp) {
  sp.out = make_right_env_layout(Bl, ms.rl);
  const EnvLayout& RN = sp.out;
  const int d = ms.d, wl = ms.wl, wr = ms.wr;

  GemmList& g1 = sp.g1;
  GemmList& g3 = sp.g3;
  MixList& mx = sp.mx;
  g1.clear();
  g3.clear();
  mx.clear();
  g1.tB = true;
  std::vector<int64_t> t1off(size_t(Bl.nsec()) * d, -1);
  int64_t& t1 = sp.t1;
  t1 = 0;
  for (int ka = 0; ka < Bl.nsec(); ++ka)
    for (int t = 0; t < d; ++t) {
      const int kap = lay.kb[ka * d + t];
      if (kap < 0) continue;
      t1off[ka * d + t] = t1;
      t1 += int64_t(RL.rows[kap]) * Bl.dim[ka];
    }
  for (int ka = 0; ka < Bl.nsec(); ++ka)
    for (int t = 0; t < d; ++t) {
      const int kap = lay.kb[ka * d + t];
      if (kap < 0 || RL.rows[kap] == 0) continue;
      g1.add(t1off[ka * d + t], RL.rows[kap], RL.rows[kap], Bl.dim[ka], 1.0, 0.0);
      g1.seg(RL.goff[kap], RL.rows[kap], lay.off[ka * d + t], Bl.dim[ka], Br.dim[kap]);
    }
  std::vector<std::vector<const MPOSite::El*>> byWS(size_t(wl) * d);
  for (const auto& e : ms.nz) byWS[size_t(e.w) * d + e.s].push_back(&e);

  std::vector<int64_t> t2off(size_t(Bl.nsec()) * wl, -1);
  int64_t& t2 = sp.t2;
  t2 = 0;
  for (int ka = 0; ka < Bl.nsec(); ++ka)
    for (int w = 0; w < wl; ++w) {
      const int kb = RN.other[ka * wl + w];
      if (kb < 0) continue;
      t2off[ka * wl + w] = t2;
      t2 += int64_t(lay.gcols[kb]) * Bl.dim[ka];
    }
  for (int ka = 0; ka < Bl.nsec(); ++ka)
    for (int w = 0; w < wl; ++w) {
      const int kb = RN.other[ka * wl + w];
      if (kb < 0) continue;
      for (int s = 0; s < d; ++s) {
        const int kbp = lay.kb[kb * d + s];
        if (kbp < 0) continue;
        const int64_t colA = (lay.off[kb * d + s] - lay.goff[kb]) / Bl.dim[kb];
        mx.add(t2off[ka * wl + w] + colA, lay.gcols[kb], Br.dim[kbp], Bl.dim[ka]);
        for (const MPOSite::El* e : byWS[size_t(w) * d + s]) {
          const int kap = lay.kb[ka * d + e->t];
          if (kap < 0 || RL.rows[kap] == 0) continue;
          if (RL.other[kap * wr + e->w2] != kbp) continue;
          mx.term(t1off[ka * d + e->t] + RL.rowoff[kap * wr + e->w2], RL.rows[kap], e->v);
        }
      }
    }
  for (int ka = 0; ka < Bl.nsec(); ++ka)
    for (int w = 0; w < wl; ++w) {
      const int kb = RN.other[ka * wl + w];
      if (kb < 0) continue;
      g3.add(RN.goff[ka] + RN.rowoff[ka * wl + w], RN.rows[ka], Bl.dim[kb], Bl.dim[ka], 1.0, 0.0);
      if (lay.gcols[kb] > 0)
        g3.seg(lay.goff[kb], Bl.dim[kb], t2off[ka * wl + w], lay.gcols[kb], lay.gcols[kb]);
    }
}

void put_step(Upload& u, StepPlan& sp, int split) {
  u.put(sp.g1);
  u.put(sp.mx);
  u.put(sp.g3);
  sp.split = split;
  if (split) {
    sp.g1t = retile(sp.g1, TF32_TILE_M, split_tile_n(sp.g1));
    sp.g3t = retile(sp.g3, TF32_TILE_M, split_tile_n(sp.g3));
    u.put(sp.g1t);
    u.put(sp.g3t);
  }
}

void run_step(dmrg_ctx* c, const StepPlan& sp, char* db, const double* env_in, int64_t n_in,
              const DBuf& A, double* env_out, int64_t n_out, const DBuf* bra) {
  if (c->T1.n < sp.t1 || c->T2.n < sp.t2 || n_out < sp.out.size)
    fail(DMRG_ERR_ARG, "internal plan check failed: environment step scratch too small");
  // the left step reads the ket tensor first (L psi) and the bra tensor last (conj(dual)^T T2);
  // the right step the other way round (R dual^T, then psi T2)
  const DBuf& B = bra ? *bra : A;
  const bool left = sp.g3.tA;
  const DBuf& first = left ? A : B;
  const DBuf& last = left ? B : A;
  if (sp.split)
    run_gemm_split(c, sp.g1t, db, env_in, n_in, first.p, first.n, c->T1.p, c->T1.n, sp.split);
  else
    run_gemm(c, sp.g1, db, env_in, n_in, first.p, first.n, c->T1.p, c->T1.n);
  run_mix(c, sp.mx, db, c->T1.p, c->T1.n, c->T2.p, c->T2.n);
  if (sp.split)
    run_gemm_split(c, sp.g3t, db, last.p, last.n, c->T2.p, c->T2.n, env_out, n_out, sp.split);
  else
    run_gemm(c, sp.g3, db, last.p, last.n, c->T2.p, c->T2.n, env_out, n_out);
}

void env_step_dense(dmrg_ctx* c, bool left, int ml, int d, int mr, int wl, int wr,
                    const double* env_in, const double* dual, const double* psi, const double* W,
                    double* env_out) {
  if (ml <= 0 || d <= 0 || mr <= 0 || wl <= 0 || wr <= 0)
    fail(DMRG_ERR_SHAPE, "env step: every dimension must be positive");
  // dense tensors: every bond and physical state carries charge 0 (one sector per bond)
  Bond Bl, Br;
  Bl.q = {QN()}; Bl.dim = {ml};
  Br.q = {QN()}; Br.dim = {mr};
  MPOSite ms;
  ms.wl = wl; ms.d = d; ms.wr = wr;
  ms.rl.assign(wl, QN());
  ms.rr.assign(wr, QN());
  ms.p.assign(d, QN());
  ms.dense.assign(W, W + size_t(wl) * d * d * wr);
  for (int w2 = 0; w2 < wr; ++w2)
    for (int t = 0; t < d; ++t)
      for (int s = 0; s < d; ++s)
        for (int w = 0; w < wl; ++w) {
          const double v = W[w + size_t(wl) * (s + size_t(d) * (t + size_t(d) * w2))];
          if (v != 0.0) ms.nz.push_back({w, s, t, w2, v});
        }
  const SiteLayout lay = make_site_layout(Bl, ms.p, Br);
  // site [ml, d, mr] column-major -> blocks (s) of [ml x mr], s-major
  std::vector<double> hA(size_t(ml) * d * mr), hB(hA.size());
  for (int s = 0; s < d; ++s)
    for (int b = 0; b < mr; ++b)
      for (int a = 0; a < ml; ++a) {
        const size_t src = a + size_t(ml) * (s + size_t(d) * b);
        const size_t dst = size_t(lay.off[s]) + a + size_t(ml) * b;
        hA[dst] = psi[src];
        hB[dst] = dual[src];
      }
  StepPlan sp;
  EnvLayout in_lay;
  if (left) {
    in_lay = make_left_env_layout(Bl, ms.rl);
    plan_left_step(Bl, Br, ms, lay, in_lay, sp);
  } else {
    in_lay = make_right_env_layout(Br, ms.rr);
    plan_right_step(Bl, Br, ms, lay, in_lay, sp);
  }
  // a dense environment [m, w, m] column-major is exactly the one-sector block layout
  Upload u;
  put_step(u, sp);
  char* db = u.send(c, 2);
  DBuf dA, dB, din, dout;
  try {
    dalloc(c, dA, int64_t(hA.size()));
    dalloc(c, dB, int64_t(hB.size()));
    dalloc(c, din, std::max<int64_t>(in_lay.size, 1));
    dalloc(c, dout, std::max<int64_t>(sp.out.size, 1));
    ensure(c, c->T1, std::max<int64_t>(sp.t1, 1));
    ensure(c, c->T2, std::max<int64_t>(sp.t2, 1));
    cuda_check(cudaMemcpyAsync(dA.p, hA.data(), hA.size() * 8, cudaMemcpyHostToDevice, c->stream),
               "env step psi");
    cuda_check(cudaMemcpyAsync(dB.p, hB.data(), hB.size() * 8, cudaMemcpyHostToDevice, c->stream),
               "env step dual");
    cuda_check(cudaMemcpyAsync(din.p, env_in, size_t(in_lay.size) * 8, cudaMemcpyHostToDevice,
                               c->stream), "env step input");
    run_step(c, sp, db, din.p, din.n, dA, dout.p, dout.n, &dB);
    cuda_check(cudaMemcpyAsync(env_out, dout.p, size_t(sp.out.size) * 8, cudaMemcpyDeviceToHost,
                               c->stream), "env step output");
    cuda_check(cudaStreamSynchronize(c->stream), "env step sync");
  } catch (...) {
    dfree(c, dA); dfree(c, dB); dfree(c, din); dfree(c, dout);
    throw;
  }
  dfree(c, dA); dfree(c, dB); dfree(c, din); dfree(c, dout);
}

void lupdate(dmrg_state* st, int i, double* flops, int precision) {
  dmrg_ctx* c = st->ctx;
  if (i < 0 || i + 1 >= st->L) fail(DMRG_ERR_ARG, "lupdate: site out of range");
  if (!st->Lvalid[i]) fail(DMRG_ERR_STATE, "lupdate: Lenv[site] has not been built");
  StepPlan sp;
  plan_left_step(st->bond[i], st->bond[i + 1], st->mpo->site[i], st->lay[i], st->Llay[i], sp);
  tune_gemm(c, sp.g1);
  tune_gemm(c, sp.g3);
  Upload u;
  put_step(u, sp, split_form(precision));
  char* db = u.send(c, 2);
  ensure(c, c->T1, std::max<int64_t>(sp.t1, 1));
  ensure(c, c->T2, std::max<int64_t>(sp.t2, 1));
  st->Llay[i + 1] = sp.out;
  dalloc(c, st->Lenv[i + 1], std::max<int64_t>(sp.out.size, 1));
  run_step(c, sp, db, st->Lenv[i].p, st->Lenv[i].n, st->A[i], st->Lenv[i + 1].p,
           st->Lenv[i + 1].n);
  st->Lvalid[i + 1] = 1;
  if (flops) *flops += sp.flops();
}

void rupdate(dmrg_state* st, int i, double* flops, int precision) {
  dmrg_ctx* c = st->ctx;
  if (i <= 0 || i >= st->L) fail(DMRG_ERR_ARG, "rupdate: site out of range");
  if (!st->Rvalid[i]) fail(DMRG_ERR_STATE, "rupdate: Renv[site] has not been built");
  StepPlan sp;
  plan_right_step(st->bond[i], st->bond[i + 1], st->mpo->site[i], st->lay[i], st->Rlay[i], sp);
  tune_gemm(c, sp.g1);
  tune_gemm(c, sp.g3);
  Upload u;
  put_step(u, sp, split_form(precision));
  char* db = u.send(c, 2);
  ensure(c, c->T1, std::max<int64_t>(sp.t1, 1));
  ensure(c, c->T2, std::max<int64_t>(sp.t2, 1));
  st->Rlay[i - 1] = sp.out;
  dalloc(c, st->Renv[i - 1], std::max<int64_t>(sp.out.size, 1));
  run_step(c, sp, db, st->Renv[i].p, st->Renv[i].n, st->A[i], st->Renv[i - 1].p,
           st->Renv[i - 1].n);
  st->Rvalid[i - 1] = 1;
  if (flops) *flops += sp.flops();
}

}  // namespace dmrg
