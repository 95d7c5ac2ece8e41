// engine_step.hpp -- pieces shared by the bond steps of the two-site sweep (engine_sweep.cpp) and
// the single-site sweep with subspace expansion (engine_3s.cpp): phase timing, the global
// truncation rule, the Krylov solve, and the reduced-density-matrix eigensolve per charge group.
#pragma once
#include <vector>

#include "engine.hpp"

namespace dmrg {

// Truncation, global over all charge groups (fsvd!, algs/DMRG.jl:387): the weights of every group
// sorted descending together (ties by group, then index); k_c = the smallest k whose discarded
// weight is at most cutoff x total (total = mag, or the sum of the weights when mag = 0); keep
// k = min(maxm, max(minm, k_c)) (maxm > 0), at least 1; with degen_rtol > 0 the cut moves back out
// of a degenerate multiplet. truncerr = the discarded weight; total = the sum of all weights.
struct Sel {
  std::vector<int> keep;
  double truncerr = 0.0;
  double total = 0.0;
};
Sel select_kept(const std::vector<std::vector<double>>& vals, int maxm, int minm, double cutoff,
                double mag, double degen_rtol);

// Phase timing with CUDA events from the context's persistent pool (profile != 0 only). Events
// are read once, after the sweep's final synchronisation.
struct Timing {
  dmrg_ctx* c;
  bool on;
  int used = 0;
  struct Span { int a, b, cat; };
  std::vector<Span> spans;
  double acc[4] = {0, 0, 0, 0};   // heff, env, eig, vec
  GemmProfile gemm;
  Timing(dmrg_ctx* ctx, bool enabled) : c(ctx), on(enabled) {}
  int record();
  cudaEvent_t event(int i) const { return c->tev[i]; }
  int begin() { return on ? record() : -1; }
  void end(int a, int cat) {
    if (on && a >= 0) spans.push_back({a, record(), cat});
  }
  void flush();   // call after a stream sync
};

struct StepOut {
  double energy = 0, truncerr = 0, wait = 0;
  int m = 0, nmv = 0;
  std::vector<double> D;       // kept singular values, descending
  double heff_flops = 0, env_flops = 0;
  int eig_max_n = 0;
};

// Krylov solve of one bond step with every scalar in device memory (no host round trip). c->K
// holds the start vector (n doubles). simple2: the reference's 2-vector step of the two-site
// update (algs/DMRG.jl:57-90: H applied to the start vector before its normalisation); otherwise
// Lanczos with max(2, krylov) vectors, full re-orthogonalisation (CGS2), start normalised. The
// Ritz vector ends in c->H. Enqueues the energy download (and, for the split forms, the MMA
// status); krylov_energy reads them after the next stream synchronisation.
struct KrylovRun {
  bool split = false;
  bool fp64_energy = false;
};
// expo: the combination is exp(tau T) e_1 instead of the lowest Ritz vector (krylovTimeEvol).
KrylovRun krylov_solve(dmrg_state* st, const dmrg_params& P, const HeffPlan& hp, int64_t n,
                       bool simple2, bool final_step, Timing& tm, StepOut& so, double tau = 0.0,
                       bool expo = false);
double krylov_energy(dmrg_ctx* c, const KrylovRun& kr);
// Makes the context's stream wait for an environment update still running on env_stream
// (a no-op when none is pending). krylov_solve calls it before its first Heff application.
void join_env(dmrg_ctx* c);

// What a bond step optimises: the ground state (DMRG), or one TDVP time step of length tau
// (Krylov exponential instead of the Ritz vector, truncation weights relative to the total).
struct StepMode {
  bool tdvp = false;
  double tau = 0.0;
};

// The two-site bond step (twostep, algs/DMRG.jl:362-405; in TDVP mode the first half of a
// tdvp_twosite step, algs/time.jl:317-353): Krylov on the two-site Heff, density-matrix
// truncation, split into psi[iL], psi[iR] (j > 0: psi[iL] = U, psi[iR] = U^T psi; j < 0:
// psi[iL] = psi V, psi[iR] = V^T).
void twostep(dmrg_state* st, const dmrg_params& P, int j, int iL, int iR, bool final_step,
             Timing& tm, StepOut& so, const StepMode& mode);

// The single-site step (engine_3s.cpp) at site i, direction j: step3S (algs/DMRG.jl:324-360,
// expansion while alpha > noise_incr) or, in TDVP mode, one step of tdvp (algs/time.jl:240-274):
// Krylov exponential at the site, truncated decomposition, the environment update across the new
// bond (done inside the step in this mode), the bond matrix evolved with the zero-site Heff, and
// its product with the neighbour. so.env_flops counts the update done inside.
struct SiteMode {
  bool tdvp = false;
  double tau = 0.0;
  double alpha = 0.0, noise_incr = 0.0;
};
void single_site_step(dmrg_state* st, const dmrg_params& P, const SiteMode& md, int j, int i,
                      bool final_step, Timing& tm, StepOut& so);

// Charge groups of a matricised centre tensor: rows and columns are pieces (sector, state) at
// offsets inside the group matrix M_g [n x np] (column-major, leading dimension n).
struct Piece { int sec, s, off; };
struct Group {
  QN q;
  int n = 0, np = 0, keep = 0, kc = -1;
  std::vector<Piece> rows, cols;
  int64_t moff = 0, roff = 0, woff = 0;
};

// The reduced density matrix of every group (rows: M M^T, else M^T M), its eigenvalues
// (tridiagonal path up to SYEVT_MID_NMAX, block Jacobi above), and their download.
// c->R layout: [rho | eigenvalues | d,e,tau | eigenvectors | block-Jacobi workspace].
struct RhoSolve {
  bool rows = true;
  int64_t mtot = 0, rtot = 0, wtot = 0, W0 = 0, WS0 = 0, U0 = 0, J0 = 0;
  std::vector<EigTask> etasks;
  std::vector<TridTask> ttasks;
  std::vector<int> tgroup;
  std::vector<int64_t> uoff;   // per group: offset of its eigenvectors (columns) in c->R
  GemmList grho;
};
// Host plan: group offsets (moff, roff, woff), eigen tasks, the rho GEMM list; ensures c->M and
// c->R. eig_max_n: the largest block.
void plan_rho(dmrg_ctx* c, std::vector<Group>& G, bool rows, RhoSolve& rs, int* eig_max_n);
// Launches (after the group matrices are in c->M and grho is uploaded at db): rho, eigenvalues,
// and the asynchronous eigenvalue download into c->h_lam.
void launch_rho(dmrg_ctx* c, RhoSolve& rs, char* db);
// After the synchronisation: eigenvalues of group g (descending).
std::vector<std::vector<double>> rho_values(dmrg_ctx* c, const std::vector<Group>& G,
                                            const RhoSolve& rs);
// Eigenvectors of the kept states (G[g].keep set) of the tridiagonal-path blocks.
void launch_rho_vectors(dmrg_ctx* c, const std::vector<Group>& G, const RhoSolve& rs);

}  // namespace dmrg
