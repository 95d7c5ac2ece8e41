// engine_meas.cpp -- measurements of a device MPS.
//
// expect (lib/MPO_MPS/expect.jl:19-56): <psi|H|psi> for an MPO H over the same sites, as a chain
// of left environment steps from the boundary to the last bond. Not normalised, as in the
// reference.
//
// correlationmatrix (lib/MPO_MPS/correlationmatrix.jl:21-56): for single-site operators Cc, Ca
// and an optional trail F (a Jordan-Wigner string),
//   rho[i,j] = <psi|(Cc F)_i F_{i+1} ... F_{j-1} Ca_j|psi> / <psi|psi>   (i < j),
//   rho[j,i] = rho[i,j],   rho[i,i] = <psi|(Cc Ca)_i|psi> / <psi|psi>.
// The reference moves the orthogonality centre to each i and contracts locally, relying on the
// canonical form. The values are gauge-invariant, so the device leaves the centre where it is and
// contracts with identity transfers from both ends instead:
//   EL[b]  left identity environment at bond b,  ER[b]  right identity environment at bond b,
//   RC[j]  right step of ER[j+1] through Ca at site j,
//   row i: X = left step of EL[i] through (Cc F) at site i; for j > i, rho[i,j] = <X | RC[j]> at
//          bond j, then X = left step of X through F at site j.
// Operators are d x d column-major with the reference's orientation O[bra, ket] and act on the
// ket (contract(O, 2, psi[i], 2)). As an MPO site W[0, s(ket), t(bra), 0] = O[t, s]; under
// charge conservation an operator must change the charge by one fixed amount, which becomes the
// label of the w = 1 environment bond (r(w') = r(w) + p(ket) - p(bra)).
//
// correlation (lib/MPO_MPS/correlation.jl:98-237, dualpsi = psi): for operators 1..n, operator g
// a product of len_g single-site factors on consecutive sites starting at p_g, and optional
// trails F_g,
//   omega[p_1, ..., p_n] = <psi| prod_s O(s) |psi>,   O(s) = A_1(s) A_2(s) ... A_n(s),
// A_g(s) = F_g for s < p_g, factor s - p_g of operator g on its sites, the identity elsewhere (the
// order in which the reference applies them to its copy of the ket). Not normalised. The device
// runs one column (positions of operators 2..n) at a time: right environments R[s] through
// A_2..A_n from the right end, the left chain X[s] through A_1's trail and A_2..A_n, and at each
// position of operator 1 the chain through its factors contracted with R. Steps that share site,
// operator and charge label share one plan.
//
// Every step of a measurement is planned on the host and uploaded in one descriptor copy; the
// launches then run back to back on the context stream and the results are read back once.
#include <algorithm>
#include <cmath>
#include <deque>
#include <map>
#include <tuple>

#include "engine.hpp"

namespace dmrg {
namespace {

constexpr int MEAS_SLOT = 7;   // descriptor slot of the measurement plans (unused by the sweep)

// O[bra, ket] as a one-state MPO site. `label` is the left label (left_known) or the right one.
MPOSite op_site(const std::vector<double>& O, int d, const std::vector<QN>& p, QN label,
                bool left_known) {
  MPOSite ms;
  ms.wl = ms.wr = 1;
  ms.d = d;
  ms.p = p;
  ms.dense.assign(size_t(d) * d, 0.0);
  bool have = false;
  QN delta;
  for (int s = 0; s < d; ++s)
    for (int t = 0; t < d; ++t) {
      const double v = O[size_t(t) + size_t(s) * d];
      if (v == 0.0) continue;
      const QN dq = p[t] - p[s];   // charge added by the operator: p(bra) - p(ket)
      if (have && dq != delta)
        fail(DMRG_ERR_QN, "operator does not change the charge by one fixed amount");
      delta = dq;
      have = true;
      ms.nz.push_back({0, s, t, 0, v});
      ms.dense[size_t(s) + size_t(t) * d] = v;
    }
  if (left_known) {
    ms.rl = {label};
    ms.rr = {label - delta};
  } else {
    ms.rr = {label};
    ms.rl = {label + delta};
  }
  return ms;
}

std::vector<double> matmul(const std::vector<double>& A, const std::vector<double>& B, int d) {
  std::vector<double> C(size_t(d) * d, 0.0);
  for (int j = 0; j < d; ++j)
    for (int k = 0; k < d; ++k) {
      const double b = B[size_t(k) + size_t(j) * d];
      if (b == 0.0) continue;
      for (int i = 0; i < d; ++i) C[size_t(i) + size_t(j) * d] += A[size_t(i) + size_t(k) * d] * b;
    }
  return C;
}

// Pair contraction at bond B of an L-type environment X and an R-type environment Y, both w = 1.
struct PairPlan {
  std::vector<PairTask> t;
  int64_t total = 0;
  size_t off = 0;
};

PairPlan plan_pair(const Bond& B, const EnvLayout& X, const EnvLayout& Y) {
  PairPlan pp;
  if (X.w != 1 || Y.w != 1) fail(DMRG_ERR_ARG, "pair contraction needs one-state environments");
  for (int k = 0; k < B.nsec(); ++k) {   // ket sector
    const int kx = X.other[k];           // bra sector of X's block
    if (kx < 0 || Y.other[kx] != k) continue;
    PairTask t;
    t.x_off = X.goff[k] + X.rowoff[k];
    t.y_off = Y.goff[kx] + Y.rowoff[kx];
    t.rows = B.dim[kx];
    t.cols = B.dim[k];
    t.e0 = pp.total;
    if (int64_t(t.rows) * t.cols == 0) continue;
    pp.total += int64_t(t.rows) * t.cols;
    pp.t.push_back(t);
  }
  return pp;
}

void check_pair(const PairPlan& pp, int64_t nX, int64_t nY) {
  for (const PairTask& t : pp.t) {
    const int64_t last = int64_t(t.rows) * t.cols - 1;
    if (t.x_off < 0 || t.y_off < 0 || t.x_off + last >= nX || t.y_off + last >= nY)
      fail(DMRG_ERR_ARG, "internal plan check failed: pair contraction out of bounds");
  }
}

void run_pair(dmrg_ctx* c, const PairPlan& pp, char* db, const DBuf& X, const DBuf& Y,
              double* out) {
  check_pair(pp, X.n, Y.n);
  launch_pair_dot(c->stream, X.p, Y.p, reinterpret_cast<const PairTask*>(db + pp.off),
                  int(pp.t.size()), pp.total, c->d_partial, out);
}

// `sp` repeated for `nrows` environments stored back to back: copy r reads env_in + r*in_stride,
// writes env_out + r*out_stride and uses the scratch T1 + r*sp.t1, T2 + r*sp.t2; the site tensor
// is shared by every copy.
StepPlan replicate_step(const StepPlan& sp, int nrows, int64_t in_stride, int64_t out_stride) {
  StepPlan b;
  b.g1.tA = sp.g1.tA;
  b.g1.tB = sp.g1.tB;
  b.g3.tA = sp.g3.tA;
  b.g3.tB = sp.g3.tB;
  for (int r = 0; r < nrows; ++r) {
    for (const GemmTask& t : sp.g1.tasks) {       // env_in x site -> T1
      b.g1.add(t.c_off + r * sp.t1, t.ldc, t.M, t.N, t.alpha, t.beta);
      for (int k = t.seg0; k < t.seg0 + t.nseg; ++k) {
        const GemmSeg& g = sp.g1.segs[k];
        b.g1.seg(g.a_off + r * in_stride, g.lda, g.b_off, g.ldb, g.K);
      }
    }
    for (const MixTask& t : sp.mx.tasks) {        // T1 -> T2
      b.mx.add(t.out_off + r * sp.t2, t.ld, t.rows, t.cols);
      for (int k = t.term0; k < t.term0 + t.nterm; ++k) {
        const MixTerm& m = sp.mx.terms[k];
        b.mx.term(m.in_off + r * sp.t1, m.ld, m.coef);
      }
    }
    for (const GemmTask& t : sp.g3.tasks) {       // site x T2 -> env_out
      b.g3.add(t.c_off + r * out_stride, t.ldc, t.M, t.N, t.alpha, t.beta);
      for (int k = t.seg0; k < t.seg0 + t.nseg; ++k) {
        const GemmSeg& g = sp.g3.segs[k];
        b.g3.seg(g.a_off, g.lda, g.b_off + r * sp.t2, g.ldb, g.K);
      }
    }
  }
  b.out = sp.out;
  b.t1 = sp.t1 * nrows;
  b.t2 = sp.t2 * nrows;
  return b;
}

// out[r * out_stride] = pair contraction of row r of X (rows of x_stride doubles) with Y.
void run_pair_rows(dmrg_ctx* c, const PairPlan& pp, char* db, const DBuf& X, int nrows,
                   int64_t x_stride, const DBuf& Y, double* out, int64_t out_stride) {
  check_pair(pp, x_stride, Y.n);
  if (int64_t(nrows) * x_stride > X.n)
    fail(DMRG_ERR_ARG, "internal plan check failed: pair rows out of bounds");
  launch_pair_dot_rows(c->stream, X.p, x_stride, Y.p,
                       reinterpret_cast<const PairTask*>(db + pp.off), int(pp.t.size()), nrows,
                       out, out_stride);
}

void set_one(dmrg_ctx* c, DBuf& b) {
  static const double one = 1.0;
  cuda_check(cudaMemcpyAsync(b.p, &one, sizeof(double), cudaMemcpyHostToDevice, c->stream),
             "measurement boundary");
}

int64_t plan_scratch(const StepPlan& sp, int64_t& t1, int64_t& t2) {
  t1 = std::max(t1, sp.t1);
  t2 = std::max(t2, sp.t2);
  return sp.out.size;
}

void check_edges(const dmrg_state* st) {
  const Bond& b0 = st->bond[0];
  const Bond& bL = st->bond[st->L];
  if (b0.nsec() != 1 || b0.dim[0] != 1 || bL.nsec() != 1 || bL.dim[0] != 1)
    fail(DMRG_ERR_SHAPE, "edge bonds of the MPS must be one-dimensional");
}

}  // namespace

double measure_expect(dmrg_state* st, const dmrg_mpo* H, double* flops) {
  dmrg_ctx* c = st->ctx;
  const int L = st->L;
  if (!H || H->L != L) fail(DMRG_ERR_SHAPE, "expect: MPO length differs from the state's");
  if (H->nsym != st->nsym) fail(DMRG_ERR_QN, "expect: MPO and state carry different charges");
  for (int i = 0; i < L; ++i) {
    const MPOSite& a = H->site[i];
    const MPOSite& b = st->mpo->site[i];
    if (a.d != b.d) fail(DMRG_ERR_SHAPE, "expect: physical dimension differs at a site");
    for (int s = 0; s < a.d; ++s)
      if (a.p[s] != b.p[s]) fail(DMRG_ERR_QN, "expect: physical charges differ at a site");
  }
  if (H->site[0].wl != 1 || H->site[L - 1].wr != 1)
    fail(DMRG_ERR_SHAPE, "edge bonds of the MPO must be one-dimensional");
  check_edges(st);

  std::vector<StepPlan> sp(L);
  EnvLayout E0 = make_left_env_layout(st->bond[0], H->site[0].rl);
  if (E0.other[0] != 0) fail(DMRG_ERR_QN, "MPO edge labels do not connect the MPS edge sectors");
  int64_t t1 = 1, t2 = 1, emax = 1;
  Upload u;
  for (int i = 0; i < L; ++i) {
    plan_left_step(st->bond[i], st->bond[i + 1], H->site[i], st->lay[i], i ? sp[i - 1].out : E0,
                   sp[i]);
    emax = std::max(emax, plan_scratch(sp[i], t1, t2));
    put_step(u, sp[i]);
  }
  char* db = u.send(c, MEAS_SLOT);
  ensure(c, c->T1, t1);
  ensure(c, c->T2, t2);
  DBuf P[2];
  double value = 0.0;
  try {
    dalloc(c, P[0], emax);
    dalloc(c, P[1], emax);
    set_one(c, P[1]);
    double fl = 0.0;
    for (int i = 0; i < L; ++i) {
      const DBuf& in = P[(i + 1) & 1];
      DBuf& out = P[i & 1];
      run_step(c, sp[i], db, in.p, in.n, st->A[i], out.p, out.n);
      fl += sp[i].flops();
    }
    cuda_check(cudaGetLastError(), "expect launches");
    const EnvLayout& EL = sp[L - 1].out;
    if (EL.size >= 1)
      cuda_check(cudaMemcpyAsync(c->h_scal, P[(L - 1) & 1].p, sizeof(double),
                                 cudaMemcpyDeviceToHost, c->stream), "expect download");
    cuda_check(cudaStreamSynchronize(c->stream), "expect sync");
    value = EL.size >= 1 ? c->h_scal[0] : 0.0;
    if (flops) *flops = fl;
  } catch (...) {
    dfree(c, P[0]);
    dfree(c, P[1]);
    throw;
  }
  dfree(c, P[0]);
  dfree(c, P[1]);
  return value;
}

void measure_correlation(dmrg_state* st, int d, const double* Cc_, const double* Ca_,
                         const double* F_, double* rho, double* flops, double* norm_out) {
  dmrg_ctx* c = st->ctx;
  const int L = st->L;
  for (int i = 0; i < L; ++i)
    if (st->mpo->site[i].d != d)
      fail(DMRG_ERR_SHAPE, "correlationmatrix: operator dimension differs from a site's");
  check_edges(st);
  const size_t dd = size_t(d) * d;
  std::vector<double> Cc(Cc_, Cc_ + dd), Ca(Ca_, Ca_ + dd), Id(dd, 0.0);
  for (int a = 0; a < d; ++a) Id[size_t(a) * (d + 1)] = 1.0;
  std::vector<double> F = F_ ? std::vector<double>(F_, F_ + dd) : Id;
  const std::vector<double> FCc = matmul(Cc, F, d);      // contract(Cc, 2, trail, 1)
  const std::vector<double> onsite = matmul(Cc, Ca, d);  // contract(Cc, 2, Ca, 1)
  const QN zero;

  // ---- plans
  std::vector<EnvLayout> ELl(L + 1), ERl(L + 1);
  std::vector<StepPlan> spL(L), spR(L), spC(L);
  ELl[0] = make_left_env_layout(st->bond[0], {zero});
  ERl[L] = make_right_env_layout(st->bond[L], {zero});
  if (ELl[0].other[0] != 0 || ERl[L].other[0] != 0)
    fail(DMRG_ERR_QN, "edge sectors of the MPS do not connect");
  int64_t t1 = 1, t2 = 1;
  Upload u;
  for (int i = 0; i < L; ++i) {
    const MPOSite id = op_site(Id, d, st->mpo->site[i].p, zero, true);
    plan_left_step(st->bond[i], st->bond[i + 1], id, st->lay[i], ELl[i], spL[i]);
    ELl[i + 1] = spL[i].out;
    plan_scratch(spL[i], t1, t2);
    put_step(u, spL[i]);
  }
  for (int i = L - 1; i >= 0; --i) {
    const MPOSite id = op_site(Id, d, st->mpo->site[i].p, zero, true);
    plan_right_step(st->bond[i], st->bond[i + 1], id, st->lay[i], ERl[i + 1], spR[i]);
    ERl[i] = spR[i].out;
    plan_scratch(spR[i], t1, t2);
    put_step(u, spR[i]);
  }
  for (int j = 1; j < L; ++j) {
    const MPOSite ca = op_site(Ca, d, st->mpo->site[j].p, zero, false);
    plan_right_step(st->bond[j], st->bond[j + 1], ca, st->lay[j], ERl[j + 1], spC[j]);
    plan_scratch(spC[j], t1, t2);
    put_step(u, spC[j]);
  }
  // diagonal: (Cc Ca) at site i between EL[i] and ER[i+1]
  std::vector<StepPlan> spD(L);
  std::vector<PairPlan> ppD(L);
  int64_t dmax = 1;
  for (int i = 0; i < L; ++i) {
    const MPOSite on = op_site(onsite, d, st->mpo->site[i].p, zero, true);
    plan_left_step(st->bond[i], st->bond[i + 1], on, st->lay[i], ELl[i], spD[i]);
    dmax = std::max(dmax, plan_scratch(spD[i], t1, t2));
    put_step(u, spD[i]);
    ppD[i] = plan_pair(st->bond[i + 1], spD[i].out, ERl[i + 1]);
    ppD[i].off = u.put(ppD[i].t);
  }
  // off-diagonal, one bond (column) j at a time: the rows i < j hold X_i at bond j back to back
  // (one layout per bond, since every row carries the same charge label); X_{j-1} starts from
  // EL[j-1] through (Cc F) at site j-1, the older rows move through F at site j-1 in one
  // replicated step, and one launch contracts every row with RC[j].
  std::vector<StepPlan> spS(L), spF(L);     // [j]: start of row j-1 / batched F step into bond j
  std::vector<PairPlan> ppC(L);
  std::vector<int64_t> xs(L, 0);            // X layout size at bond j
  int64_t xmax = 1;
  QN label;
  for (int j = 1; j < L; ++j) {
    const MPOSite fc = op_site(FCc, d, st->mpo->site[j - 1].p, zero, true);
    label = fc.rr[0];
    plan_left_step(st->bond[j - 1], st->bond[j], fc, st->lay[j - 1], ELl[j - 1], spS[j]);
    plan_scratch(spS[j], t1, t2);
    put_step(u, spS[j]);
    xs[j] = spS[j].out.size;
    if (j >= 2) {
      const MPOSite f = op_site(F, d, st->mpo->site[j - 1].p, label, true);
      StepPlan one;
      plan_left_step(st->bond[j - 1], st->bond[j], f, st->lay[j - 1], spS[j - 1].out, one);
      if (one.out.size != xs[j]) fail(DMRG_ERR_ARG, "internal plan check failed: row layouts differ");
      spF[j] = replicate_step(one, j - 1, xs[j - 1], xs[j]);
      plan_scratch(spF[j], t1, t2);
      put_step(u, spF[j]);
    }
    xmax = std::max(xmax, int64_t(j) * std::max<int64_t>(xs[j], 1));
    ppC[j] = plan_pair(st->bond[j], spS[j].out, spC[j].out);
    ppC[j].off = u.put(ppC[j].t);
  }
  PairPlan norm = plan_pair(st->bond[L], ELl[L], ERl[L]);
  norm.off = u.put(norm.t);

  // ---- device buffers and launches
  std::vector<DBuf> EL(L + 1), ER(L + 1), RC(L);
  DBuf D, X[2], out;
  auto release = [&] {
    for (auto& b : EL) dfree(c, b);
    for (auto& b : ER) dfree(c, b);
    for (auto& b : RC) dfree(c, b);
    dfree(c, D);
    dfree(c, X[0]);
    dfree(c, X[1]);
    dfree(c, out);
  };
  try {
    char* db = u.send(c, MEAS_SLOT);
    ensure(c, c->T1, t1);
    ensure(c, c->T2, t2);
    for (int b = 0; b <= L; ++b) {
      dalloc(c, EL[b], std::max<int64_t>(ELl[b].size, 1));
      dalloc(c, ER[b], std::max<int64_t>(ERl[b].size, 1));
    }
    for (int j = 1; j < L; ++j) dalloc(c, RC[j], std::max<int64_t>(spC[j].out.size, 1));
    dalloc(c, D, dmax);
    dalloc(c, X[0], xmax);
    dalloc(c, X[1], xmax);
    dalloc(c, out, int64_t(L) * L + 1);
    cuda_check(cudaMemsetAsync(out.p, 0, sizeof(double) * (size_t(L) * L + 1), c->stream),
               "correlation clear");
    set_one(c, EL[0]);
    set_one(c, ER[L]);
    double fl = 0.0;
    for (int i = 0; i < L; ++i) {
      run_step(c, spL[i], db, EL[i].p, EL[i].n, st->A[i], EL[i + 1].p, EL[i + 1].n);
      fl += spL[i].flops();
    }
    for (int i = L - 1; i >= 0; --i) {
      run_step(c, spR[i], db, ER[i + 1].p, ER[i + 1].n, st->A[i], ER[i].p, ER[i].n);
      fl += spR[i].flops();
    }
    for (int j = 1; j < L; ++j) {
      run_step(c, spC[j], db, ER[j + 1].p, ER[j + 1].n, st->A[j], RC[j].p, RC[j].n);
      fl += spC[j].flops();
    }
    for (int i = 0; i < L; ++i) {
      run_step(c, spD[i], db, EL[i].p, EL[i].n, st->A[i], D.p, D.n);
      run_pair(c, ppD[i], db, D, ER[i + 1], out.p + i + int64_t(i) * L);
      fl += spD[i].flops() + 2.0 * ppD[i].total;
    }
    for (int j = 1; j < L; ++j) {
      DBuf& xo = X[j & 1];
      const DBuf& xi = X[(j - 1) & 1];
      if (j >= 2) {
        run_step(c, spF[j], db, xi.p, xi.n, st->A[j - 1], xo.p, xo.n);
        fl += spF[j].flops();
      }
      const int64_t at = int64_t(j - 1) * xs[j];
      run_step(c, spS[j], db, EL[j - 1].p, EL[j - 1].n, st->A[j - 1], xo.p + at, xo.n - at);
      fl += spS[j].flops();
      run_pair_rows(c, ppC[j], db, xo, j, xs[j], RC[j], out.p + int64_t(j) * L, 1);
      fl += 2.0 * ppC[j].total * j;
    }
    run_pair(c, norm, db, EL[L], ER[L], out.p + int64_t(L) * L);
    cuda_check(cudaGetLastError(), "correlation launches");
    std::vector<double> h(size_t(L) * L + 1);
    cuda_check(cudaMemcpyAsync(h.data(), out.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost,
                               c->stream), "correlation download");
    cuda_check(cudaStreamSynchronize(c->stream), "correlation sync");
    const double nrm = h[size_t(L) * L];
    if (!(nrm > 0.0) || !std::isfinite(nrm))
      fail(DMRG_ERR_STATE, "correlationmatrix: <psi|psi> is not positive");
    if (norm_out) *norm_out = nrm;
    for (int i = 0; i < L; ++i) {
      rho[i + size_t(i) * L] = h[i + size_t(i) * L] / nrm;
      for (int j = i + 1; j < L; ++j) {
        const double v = h[i + size_t(j) * L] / nrm;
        rho[i + size_t(j) * L] = v;
        rho[j + size_t(i) * L] = v;
      }
    }
    if (flops) *flops = fl;
  } catch (...) {
    release();
    throw;
  }
  release();
}

void measure_correlation_n(dmrg_state* st, int d, int n, const int* lens, const double* ops,
                           const int* nsites, const int* sites, const double* trails,
                           double* omega, double* flops) {
  dmrg_ctx* c = st->ctx;
  const int L = st->L;
  if (n < 1 || n > 8) fail(DMRG_ERR_ARG, "correlation: between 1 and 8 operators");
  for (int i = 0; i < L; ++i)
    if (st->mpo->site[i].d != d)
      fail(DMRG_ERR_SHAPE, "correlation: operator dimension differs from a site's");
  check_edges(st);
  const size_t dd = size_t(d) * d;
  std::vector<double> Id(dd, 0.0);
  for (int a = 0; a < d; ++a) Id[size_t(a) * (d + 1)] = 1.0;
  // operators, trails (an identity trail is none) and the start positions of each operator
  std::vector<std::vector<std::vector<double>>> O(n);
  std::vector<std::vector<double>> F(n);
  std::vector<std::vector<int>> pos(n);
  size_t oat = 0, sat = 0;
  int64_t total = 1;
  for (int g = 0; g < n; ++g) {
    if (lens[g] < 1 || lens[g] > L) fail(DMRG_ERR_ARG, "correlation: bad operator length");
    for (int k = 0; k < lens[g]; ++k, oat += dd) O[g].emplace_back(ops + oat, ops + oat + dd);
    if (trails) {
      std::vector<double> t(trails + size_t(g) * dd, trails + size_t(g + 1) * dd);
      if (t != Id) F[g] = t;
    }
    const int base = nsites[g] - (lens[g] - 1);
    if (nsites[g] < 1 || base < 1) fail(DMRG_ERR_ARG, "correlation: no position for an operator");
    for (int y = 0; y < base; ++y) {
      const int p = sites[sat + y];
      if (p < 0 || p + lens[g] > L) fail(DMRG_ERR_ARG, "correlation: an operator runs off the chain");
      pos[g].push_back(p);
    }
    sat += size_t(nsites[g]);
    total *= base;
    if (total > (int64_t(1) << 24)) fail(DMRG_ERR_BUDGET, "correlation: too many entries");
  }
  const int base1 = int(pos[0].size()), len1 = lens[0];
  const int64_t ncol = total / base1;

  // Two single-site operators over every site with no trail, or with one trail F, F F = I (a
  // Jordan-Wigner string): every entry is one of the batched correlation matrix's. For p1 <= p2
  // O(s) is F F = I left of p1, O1 F at p1, F between, O2 at p2: row p1, column p2 of
  // correlationmatrix(O1, O2; F); for p1 > p2 it is F O2 = (F O2 F) F at p2, F between, O1 at
  // p1: row p2, column p1 of correlationmatrix(F O2 F, O1; F). Both times <psi|psi>.
  bool every_site = n == 2 && lens[0] == 1 && lens[1] == 1 && nsites[0] == L && nsites[1] == L;
  for (int g = 0; every_site && g < 2; ++g)
    for (int y = 0; y < L; ++y) every_site = every_site && pos[g][y] == y;
  const bool same_trail = F[0] == F[1];
  bool involution = F[0].empty();
  if (!involution && same_trail) {
    const std::vector<double> FF = matmul(F[0], F[0], d);
    involution = true;
    for (size_t e = 0; e < dd; ++e) involution = involution && std::fabs(FF[e] - Id[e]) <= 1e-14;
  }
  if (every_site && same_trail && involution) {
    const double* Fp = F[0].empty() ? nullptr : F[0].data();
    std::vector<double> up(size_t(L) * L), lo(size_t(L) * L);
    double nrm = 0.0, f1 = 0.0, f2 = 0.0;
    measure_correlation(st, d, O[0][0].data(), O[1][0].data(), Fp, up.data(), &f1, &nrm);
    const std::vector<double> C2 = F[0].empty() ? O[1][0] : matmul(matmul(F[0], O[1][0], d), F[0], d);
    measure_correlation(st, d, C2.data(), O[0][0].data(), Fp, lo.data(), &f2, nullptr);
    for (int p2 = 0; p2 < L; ++p2)
      for (int p1 = 0; p1 < L; ++p1)
        omega[p1 + size_t(L) * p2] = nrm * (p1 <= p2 ? up[p1 + size_t(L) * p2] : lo[p2 + size_t(L) * p1]);
    if (flops) *flops = f1 + f2;
    return;
  }
  if (ncol * int64_t(L) > (int64_t(1) << 22))
    fail(DMRG_ERR_BUDGET, "correlation: too many positions of operators 2..n for this chain");
  const QN zero;

  // ---- plans, shared by site, direction, incoming charge label and operator
  std::deque<StepPlan> plans;            // stable references
  std::vector<QN> plan_out;              // charge label of each plan's output environment
  std::map<std::tuple<int, int, int, int, std::vector<double>>, int> memo;
  auto step = [&](bool left, int s, QN label, const std::vector<double>& M,
                  const EnvLayout& in) -> int {
    auto key = std::make_tuple(left ? 0 : 1, s, label.v[0], label.v[1], M);
    auto it = memo.find(key);
    if (it != memo.end()) return it->second;
    const MPOSite ms = op_site(M, d, st->mpo->site[s].p, label, left);
    plans.emplace_back();
    if (left) plan_left_step(st->bond[s], st->bond[s + 1], ms, st->lay[s], in, plans.back());
    else plan_right_step(st->bond[s], st->bond[s + 1], ms, st->lay[s], in, plans.back());
    plan_out.push_back(left ? ms.rr[0] : ms.rl[0]);
    memo.emplace(key, int(plans.size()) - 1);
    return int(plans.size()) - 1;
  };
  std::deque<PairPlan> pairs;
  std::map<std::tuple<int, int, int, int, int>, int> pmemo;
  auto pair = [&](int b, QN lx, const EnvLayout& X, QN ly, const EnvLayout& Y) -> int {
    auto key = std::make_tuple(b, lx.v[0], lx.v[1], ly.v[0], ly.v[1]);
    auto it = pmemo.find(key);
    if (it != pmemo.end()) return it->second;
    pairs.push_back(plan_pair(st->bond[b], X, Y));
    pmemo.emplace(key, int(pairs.size()) - 1);
    return int(pairs.size()) - 1;
  };
  const EnvLayout ELb = make_left_env_layout(st->bond[0], {zero});
  const EnvLayout ERb = make_right_env_layout(st->bond[L], {zero});
  if (ELb.other[0] != 0 || ERb.other[0] != 0)
    fail(DMRG_ERR_QN, "edge sectors of the MPS do not connect");
  std::vector<std::vector<int>> ystart(L);   // operator-1 entries y starting at each site
  int last1 = 0;
  for (int y = 0; y < base1; ++y) {
    ystart[pos[0][y]].push_back(y);
    last1 = std::max(last1, pos[0][y]);
  }
  struct Column {
    std::vector<int> R, X, Y, P;   // right chain by site, left chain by site, operator-1 factors
  };                                // (y * len1 + k), pair contraction per y
  std::vector<Column> cols(static_cast<size_t>(ncol));
  std::vector<std::vector<double>> S(L);
  std::vector<int> at(n, 0);
  for (int64_t col = 0; col < ncol; ++col) {
    int64_t r = col;
    for (int g = 1; g < n; ++g) {   // positions of operators 2..n, the first of them fastest
      at[g] = int(r % int64_t(pos[g].size()));
      r /= int64_t(pos[g].size());
    }
    for (int s = 0; s < L; ++s) {   // A_2(s) ... A_n(s)
      std::vector<double> M = Id;
      for (int g = 1; g < n; ++g) {
        const int p = pos[g][at[g]];
        if (s < p) { if (!F[g].empty()) M = matmul(M, F[g], d); }
        else if (s < p + lens[g]) M = matmul(M, O[g][s - p], d);
      }
      S[s] = M;
    }
    Column& q = cols[size_t(col)];
    std::vector<QN> rl(L + 1);
    std::vector<const EnvLayout*> rlay(L + 1);
    rl[L] = zero;
    rlay[L] = &ERb;
    q.R.assign(L, -1);
    for (int s = L - 1; s >= 0; --s) {
      const int k = step(false, s, rl[s + 1], S[s], *rlay[s + 1]);
      q.R[s] = k;
      rl[s] = plan_out[k];
      rlay[s] = &plans[k].out;
    }
    QN xl = zero;
    const EnvLayout* xlay = &ELb;
    q.X.assign(L, -1);
    q.Y.assign(size_t(base1) * len1, -1);
    q.P.assign(base1, -1);
    for (int s = 0; s <= last1; ++s) {
      for (int y : ystart[s]) {
        QN yl = xl;
        const EnvLayout* ylay = xlay;
        for (int k = 0; k < len1; ++k) {
          const int j = step(true, s + k, yl, matmul(O[0][k], S[s + k], d), *ylay);
          q.Y[size_t(y) * len1 + k] = j;
          yl = plan_out[j];
          ylay = &plans[j].out;
        }
        q.P[y] = pair(s + len1, yl, *ylay, rl[s + len1], *rlay[s + len1]);
      }
      if (s < last1) {
        const int j = step(true, s, xl, F[0].empty() ? S[s] : matmul(F[0], S[s], d), *xlay);
        q.X[s] = j;
        xl = plan_out[j];
        xlay = &plans[j].out;
      }
    }
  }

  // ---- one upload, buffers sized by the largest environment at each bond
  int64_t t1 = 1, t2 = 1, lmax = 1;
  std::vector<int64_t> rmax(L + 1, 1);
  Upload u;
  for (auto& sp : plans) {
    plan_scratch(sp, t1, t2);
    put_step(u, sp);
  }
  for (const Column& q : cols)
    for (int s = 0; s < L; ++s) rmax[s] = std::max(rmax[s], plans[q.R[s]].out.size);
  for (const StepPlan& sp : plans) lmax = std::max(lmax, sp.out.size);
  for (auto& pp : pairs) pp.off = u.put(pp.t);
  std::vector<DBuf> R(L + 1);
  DBuf XB, X[2], Y[2], out;
  auto release = [&] {
    for (auto& b : R) dfree(c, b);
    dfree(c, XB);
    for (int a = 0; a < 2; ++a) {
      dfree(c, X[a]);
      dfree(c, Y[a]);
    }
    dfree(c, out);
  };
  try {
    char* db = u.send(c, MEAS_SLOT);
    ensure(c, c->T1, t1);
    ensure(c, c->T2, t2);
    for (int b = 0; b <= L; ++b) dalloc(c, R[b], rmax[b]);
    dalloc(c, XB, 1);
    for (int a = 0; a < 2; ++a) {
      dalloc(c, X[a], lmax);
      dalloc(c, Y[a], lmax);
    }
    dalloc(c, out, total);
    cuda_check(cudaMemsetAsync(out.p, 0, sizeof(double) * size_t(total), c->stream),
               "correlation clear");
    set_one(c, R[L]);
    set_one(c, XB);
    double fl = 0.0;
    for (int64_t col = 0; col < ncol; ++col) {
      const Column& q = cols[size_t(col)];
      for (int s = L - 1; s >= 0; --s) {
        const StepPlan& sp = plans[q.R[s]];
        run_step(c, sp, db, R[s + 1].p, R[s + 1].n, st->A[s], R[s].p, R[s].n);
        fl += sp.flops();
      }
      const DBuf* xin = &XB;
      for (int s = 0; s <= last1; ++s) {
        for (int y : ystart[s]) {
          const DBuf* yin = xin;
          for (int k = 0; k < len1; ++k) {
            const StepPlan& sp = plans[q.Y[size_t(y) * len1 + k]];
            DBuf& yo = Y[k & 1];
            run_step(c, sp, db, yin->p, yin->n, st->A[s + k], yo.p, yo.n);
            fl += sp.flops();
            yin = &yo;
          }
          const PairPlan& pp = pairs[q.P[y]];
          if (!pp.t.empty()) {
            run_pair(c, pp, db, *yin, R[s + len1], out.p + y + int64_t(base1) * col);
            fl += 2.0 * pp.total;
          }
        }
        if (s < last1) {
          const StepPlan& sp = plans[q.X[s]];
          DBuf& xo = X[s & 1];
          run_step(c, sp, db, xin->p, xin->n, st->A[s], xo.p, xo.n);
          fl += sp.flops();
          xin = &xo;
        }
      }
    }
    cuda_check(cudaGetLastError(), "correlation launches");
    cuda_check(cudaMemcpyAsync(omega, out.p, sizeof(double) * size_t(total),
                               cudaMemcpyDeviceToHost, c->stream), "correlation download");
    cuda_check(cudaStreamSynchronize(c->stream), "correlation sync");
    if (flops) *flops = fl;
  } catch (...) {
    release();
    throw;
  }
  release();
}

}  // namespace dmrg
