// engine_eig.cpp -- batched eigensolve of the density-matrix blocks of one truncation:
// blocks with n <= 100 go to the one-CTA shared-memory Jacobi, larger ones to the block Jacobi.
#include <algorithm>

#include "engine.hpp"

namespace dmrg {

namespace {
void check_trid(const std::vector<TridTask>& ts, int64_t nbase, bool vectors) {
  for (const TridTask& t : ts) {
    const int64_t nn = int64_t(t.n) * t.n;
    if (t.n <= 0 || t.n > SYEVT_MID_NMAX || t.a_off < 0 || t.a_off + nn > nbase ||
        t.w_off < 0 || t.w_off + t.n > nbase || t.ws_off < 0 || t.ws_off + 3 * t.n > nbase)
      fail(DMRG_ERR_ARG, "internal plan check failed: tridiagonal eigensolver task");
    if (vectors && (t.keep < 0 || t.keep > t.n || t.u_off < 0 ||
                    t.u_off + int64_t(t.n) * t.keep > nbase))
      fail(DMRG_ERR_ARG, "internal plan check failed: tridiagonal eigenvector task");
  }
}
}  // namespace

void run_trid_eigvals(dmrg_ctx* c, double* base, int64_t nbase, const std::vector<TridTask>& t,
                      int slot) {
  check_trid(t, nbase, false);
  std::vector<TridTask> small, mid;
  int ns = 0, nm = 0;
  for (const TridTask& x : t) {
    if (x.n <= SYEVT_NMAX) { small.push_back(x); ns = std::max(ns, x.n); }
    else { mid.push_back(x); nm = std::max(nm, x.n); }
  }
  if (small.empty() && mid.empty()) return;
  Upload u;
  const size_t o1 = u.put(small), o2 = u.put(mid);
  char* db = u.send(c, slot);
  if (!small.empty())
    launch_trid_eigvals(c->stream, base, reinterpret_cast<const TridTask*>(db + o1),
                        int(small.size()), ns);
  if (!mid.empty())
    launch_trid_mid_eigvals(c->stream, base, reinterpret_cast<const TridTask*>(db + o2),
                            int(mid.size()), nm);
  cuda_check(cudaGetLastError(), "tridiagonal eigenvalues");
}

void run_trid_vectors(dmrg_ctx* c, double* base, int64_t nbase, std::vector<TridTask> t,
                      int slot) {
  check_trid(t, nbase, true);
  // mid-size blocks in two launches: those whose Gram matrix fits in shared memory beside the
  // block's vectors, and the rest (which then keep the whole L1 for their global-memory Gram)
  std::vector<TridTask> small, mid[2];
  int ns = 0, ks = 0, nm[2] = {0, 0}, km[2] = {0, 0};
  int nmax = 0;
  for (const TridTask& x : t)
    if (x.keep > 0 && x.n > SYEVT_NMAX) nmax = std::max(nmax, x.n);
  const int kg = nmax > 0 ? syevt_mid_gram_limit(nmax) : 0;
  int64_t xw = 0;
  for (TridTask x : t) {
    if (x.keep <= 0) continue;
    if (x.n <= SYEVT_NMAX) {
      small.push_back(x);
      ns = std::max(ns, x.n);
      ks = std::max(ks, x.keep);
    } else {
      x.x_off = xw;
      xw += syevt_mid_workspace(x.n, x.keep);
      const int g = x.keep <= kg ? 0 : 1;
      mid[g].push_back(x);
      nm[g] = std::max(nm[g], x.n);
      km[g] = std::max(km[g], x.keep);
    }
  }
  if (small.empty() && mid[0].empty() && mid[1].empty()) return;
  if (xw > 0) ensure(c, c->W, xw);
  Upload u;
  const size_t o1 = u.put(small), o2 = u.put(mid[0]), o3 = u.put(mid[1]);
  char* db = u.send(c, slot);
  if (!small.empty())
    launch_trid_vectors(c->stream, base, reinterpret_cast<const TridTask*>(db + o1),
                        int(small.size()), ns, ks);
  for (int g = 0; g < 2; ++g)
    if (!mid[g].empty())
      launch_trid_mid_vectors(c->stream, base,
                              reinterpret_cast<const TridTask*>(db + (g == 0 ? o2 : o3)),
                              int(mid[g].size()), nm[g], km[g], c->W.p);
  cuda_check(cudaGetLastError(), "tridiagonal eigenvectors");
}

int64_t eig_workspace(const std::vector<EigTask>& tasks) {
  int64_t ws = 0;
  for (const EigTask& t : tasks) {
    if (t.n <= 100) continue;
    const int64_t N = block_eig_padded(t.n);
    ws += 2 * N * N + N * 32;
  }
  return ws;
}

void run_eigs(dmrg_ctx* c, double* base, int64_t nbase, const std::vector<EigTask>& tasks,
              int64_t ws_off, int* sweeps) {
  if (sweeps) *sweeps = 0;
  if (tasks.empty()) return;   // nothing to solve: no status read, no synchronisation
  std::vector<EigTask> small;
  std::vector<BlockEigGroup> big;
  int nsmall = 0, maxN = 0, maxn = 0;
  int64_t ws = ws_off;
  for (const EigTask& t : tasks) {
    if (t.n <= 0) continue;
    if (t.n <= 100) {
      small.push_back(t);
      nsmall = std::max(nsmall, t.n);
      continue;
    }
    BlockEigGroup g{};
    g.a_off = t.a_off;
    g.w_off = t.w_off;
    g.n = t.n;
    g.N = block_eig_padded(t.n);
    g.ap_off = ws;
    g.vp_off = ws + int64_t(g.N) * g.N;
    g.q_off = ws + 2 * int64_t(g.N) * g.N;
    ws += 2 * int64_t(g.N) * g.N + int64_t(g.N) * 32;
    maxN = std::max(maxN, g.N);
    maxn = std::max(maxn, g.n);
    big.push_back(g);
  }
  check_eig(small, nbase);
  if (ws > nbase) fail(DMRG_ERR_ARG, "internal plan check failed: eigensolver workspace");
  for (const BlockEigGroup& g : big) {
    EigTask t{g.a_off, g.a_off, g.w_off, g.n, 0};
    check_eig({t}, nbase);
  }
  if (int(big.size()) > c->max_groups) fail(DMRG_ERR_SHAPE, "too many large density-matrix blocks");
  if (!small.empty()) {
    Upload u;
    const size_t off = u.put(small);
    char* db = u.send(c, 4);
    cuda_check(cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream), "status");
    launch_jacobi(c->stream, base, reinterpret_cast<const EigTask*>(db + off), int(small.size()),
                  nsmall, c->d_status);
  }
  if (!big.empty()) {
    std::vector<int2> pairs;
    std::vector<int4> tiles;
    for (int gi = 0; gi < int(big.size()); ++gi) {
      const int nb = big[gi].N / 16, np = nb / 2;
      for (int k = 0; k < np; ++k) pairs.push_back(make_int2(gi, k));
      for (int P = 0; P < np; ++P)
        for (int Q = 0; Q < np; ++Q) tiles.push_back(make_int4(gi, 0, P, Q));
      for (int rc = 0; rc < big[gi].N / 32; ++rc)
        for (int P = 0; P < np; ++P) tiles.push_back(make_int4(gi, 1, rc, P));
    }
    Upload u;
    const size_t go = u.put(big), po = u.put(pairs), to = u.put(tiles);
    char* db = u.send(c, 5);
    BlockEigPlan pl{};
    pl.groups = reinterpret_cast<const BlockEigGroup*>(db + go);
    pl.ngroups = int(big.size());
    pl.pairs = reinterpret_cast<const int2*>(db + po);
    pl.npairs = int(pairs.size());
    pl.tiles = reinterpret_cast<const int4*>(db + to);
    pl.ntiles = int(tiles.size());
    pl.maxN = maxN;
    pl.maxn = maxn;
    pl.max_sweeps = 30;
    int sw = 0;
    cuda_check(cudaGetLastError(), "block Jacobi set-up");
    launch_block_jacobi(c->stream, base, pl, c->d_flags, c->h_flags, c->d_floors, &sw);
    cuda_check(cudaGetLastError(), "block Jacobi");
    if (sweeps) *sweeps = sw;
    if (sw >= pl.max_sweeps) fail(DMRG_ERR_CUDA, "block Jacobi eigensolver did not converge");
  }
  int stat = 0;
  cuda_check(cudaMemcpyAsync(&stat, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream),
             "status");
  cuda_check(cudaStreamSynchronize(c->stream), "eigen sync");
  cuda_check(cudaGetLastError(), "eigensolve");
  if (!small.empty() && stat != 0) fail(DMRG_ERR_CUDA, "Jacobi eigensolver did not converge");
}

}  // namespace dmrg
