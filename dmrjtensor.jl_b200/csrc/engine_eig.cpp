// engine_eig.cpp -- batched eigensolve of the density-matrix blocks of one truncation:
// blocks with n <= 100 go to the one-CTA shared-memory Jacobi, larger ones to the block Jacobi.
#include <algorithm>

#include "engine.hpp"

namespace dmrg {

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
