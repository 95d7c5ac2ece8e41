// engine.hpp -- host-side structures of the device DMRG engine.
//
// Data layout in HBM (all FP64, column-major blocks, one contiguous buffer per tensor):
//  * bond b: sectors (charge q, dim) sorted by q; a dense bond is one sector of charge 0.
//  * MPS site A[a,s,b]: block (ka, s) -> kb = sector(q(ka)+p(s)) is a [dim ka x dim kb] matrix;
//    blocks are stored ka-major then s, so the blocks of one left sector form one matrix
//    [dim ka x sum_s dim kb(s)] ("left group") -- the B operand of every L*A product.
//  * two-site psi[a,s1,s2,d]: block (ka,s1,s2) -> kd, same ka-major grouping.
//  * left env L[a(bra), w, b(ket)]: one matrix per ket sector kb with rows (a in ka(w), w)
//    stacked over the MPO states w (ka = sector(q(kb) - r(w))), columns b. This is the
//    reference's L[bra,w,ket] viewed as a (bra*w) x ket matrix, restricted to one ket sector.
//  * right env R[b(ket), w, a(bra)]: one matrix per bra sector ka, rows (b in kb(w), w),
//    kb = sector(q(ka) + r(w)), columns a.
//  MPO bond labels follow r(w') = r(w) + p(ket) - p(bra) (lib/MPO/makeqMPO.jl:23-84), so an
//  environment block links ket = bra + r(w).
#pragma once
#include <cstdint>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/dmrg_b200.h"
#include "kernels.cuh"

namespace dmrg {

struct QN {
  int v[2] = {0, 0};
  QN() = default;
  QN(int a, int b) { v[0] = a; v[1] = b; }
};
inline bool operator<(const QN& a, const QN& b) {
  return a.v[0] < b.v[0] || (a.v[0] == b.v[0] && a.v[1] < b.v[1]);
}
inline bool operator==(const QN& a, const QN& b) { return a.v[0] == b.v[0] && a.v[1] == b.v[1]; }
inline bool operator!=(const QN& a, const QN& b) { return !(a == b); }
inline QN operator+(const QN& a, const QN& b) { return QN(a.v[0] + b.v[0], a.v[1] + b.v[1]); }
inline QN operator-(const QN& a, const QN& b) { return QN(a.v[0] - b.v[0], a.v[1] - b.v[1]); }

struct Bond {
  std::vector<QN> q;
  std::vector<int> dim;
  int nsec() const { return int(q.size()); }
  int find(const QN& x) const;
  int64_t total() const;
  std::vector<int64_t> offsets() const;  // dense-equivalent position of each sector
};

struct MPOSite {
  int wl = 0, d = 0, wr = 0;
  std::vector<QN> rl, rr, p;   // left/right bond labels, physical labels
  struct El { int w, s, t, w2; double v; };
  std::vector<El> nz;          // non-zeros of W[w,s,t,w2]
  std::vector<double> dense;   // [wl,d,d,wr] column-major
};

// W_L x W_R contracted over the shared bond, grouped by output (t1,t2,w'').
struct TwoSiteOp {
  struct Term { int w, s1, s2; double c; };
  int d1 = 0, d2 = 0, wl = 0, wr = 0;
  std::vector<std::vector<Term>> out;   // index ((t1*d2)+t2)*wr + w''
};

struct SiteLayout {      // A[a,s,b]
  int nl = 0, d = 0;
  std::vector<int> kb;         // [ka*d+s] right sector or -1
  std::vector<int64_t> off;    // [ka*d+s] block offset
  std::vector<int64_t> goff;   // [ka] group offset
  std::vector<int> gcols;      // [ka] group columns
  int64_t size = 0;
};

struct TwoLayout {       // psi[a,s1,s2,d]
  int nl = 0, d1 = 0, d2 = 0;
  std::vector<int> kd;         // [(ka*d1+s1)*d2+s2]
  std::vector<int64_t> off;
  std::vector<int64_t> goff;
  std::vector<int> gcols;
  int64_t size = 0;
  int idx(int ka, int s1, int s2) const { return (ka * d1 + s1) * d2 + s2; }
};

struct EnvLayout {       // L: groups by ket sector; R: groups by bra sector
  int nsec = 0, w = 0;
  std::vector<int> other;      // [k*w+wi] bra sector (L) / ket sector (R), or -1
  std::vector<int> rowoff;     // [k*w+wi]
  std::vector<int> rows;       // [k]
  std::vector<int64_t> goff;   // [k]
  int64_t size = 0;
};

struct DBuf {
  double* p = nullptr;
  int64_t n = 0;   // capacity in doubles
};

// Pinned host staging + device copy for one family of task descriptors.
struct DescSlot {
  char* h = nullptr;
  char* d = nullptr;
  size_t cap = 0;
  cudaEvent_t ev = nullptr;
};

struct GemmList {
  bool tA = false, tB = false;
  uint64_t tune_key = 0;         // block-size histogram signature (0: not tuned)
  int tune_trial = 0;            // 1: this launch is timed for the tuner
  std::vector<GemmTask> tasks;
  std::vector<GemmSeg> segs;
  int tiles = 0;
  double flops = 0;
  size_t t_off = 0, s_off = 0;  // byte offsets inside the uploaded slot
  int bm = GEMM_BM;              // tile rows the tile counts refer to
  int bn = GEMM_BN;              // tile columns the tile counts refer to
  // image plan of the image-fed split form (lists retiled to TF32_TILE_N_IMAGE or
  // TF32_TILE_N_WIDE): the distinct A and B operand windows as panels, and the image chunks of
  // every segment
  std::vector<ImgPanel> pa, pb;
  std::vector<SegImg> si;
  int64_t img_a = 0, img_b = 0;  // image chunks of A and of B
  size_t pa_off = 0, pb_off = 0, si_off = 0;
  void clear() {
    tasks.clear(); segs.clear(); pa.clear(); pb.clear(); si.clear();
    tiles = 0; flops = 0; img_a = img_b = 0;
  }
  void add(int64_t c_off, int ldc, int M, int N, double alpha, double beta);
  void seg(int64_t a_off, int lda, int64_t b_off, int ldb, int K);
};
// The same products tiled for the split-precision kernel (TF32_TILE_M x bn tiles); with
// bn = TF32_TILE_N_IMAGE or TF32_TILE_N_WIDE also the image plan.
GemmList retile(const GemmList& g, int bm, int bn);

struct MixList {
  std::vector<MixTask> tasks;
  std::vector<MixTerm> terms;
  int tiles = 0;
  double flops = 0;
  size_t t_off = 0, m_off = 0;
  void clear() { tasks.clear(); terms.clear(); tiles = 0; flops = 0; }
  void add(int64_t out_off, int ld, int rows, int cols);
  void term(int64_t in_off, int ld, double c);
};

struct CopyList {
  std::vector<CopyTask> tasks;
  int tiles = 0;
  size_t t_off = 0;
  void clear() { tasks.clear(); tiles = 0; }
  void add(int64_t src_off, int lds, int64_t dst_off, int ldd, int rows, int cols, int trans,
           double scale);
};

}  // namespace dmrg

namespace dmrg {
struct HeffBatcher;   // shared Heff launches of a server's solves (batch.cpp)
// Tile-shape autotuner of the FP64 grouped GEMM. A list's signature quantises its block-size
// histogram (FLOP-weighted mean M, N and K, task count, total FLOPs, transposes, in half-octave
// buckets). The first launches of a new signature are timed once in each tile shape (64 x 64 and
// 32 x 32) with CUDA events; from then on the faster shape is used for that signature (64 x 64
// unless 32 x 32 is more than 3% faster). Both shapes give bit-identical results, so the choice
// never changes a number, only the time. The table lives in the context (one device).
struct GemmTuner {
  struct Entry {
    int trials[2] = {0, 0};       // [0] 64 x 64, [1] 32 x 32
    double best[2] = {1e30, 1e30};
    int choice = -1;
  };
  struct Pending {
    uint64_t key;
    int variant;
    cudaEvent_t a, b;
  };
  std::map<uint64_t, Entry> table;
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> free_events;
  ~GemmTuner();
};
}  // namespace dmrg

struct dmrg_ctx {
  int device = 0;
  bool tune = true;              // FP64 GEMM tile autotuner on (dmrg_params.tune of the sweep)
  dmrg::HeffBatcher* batch = nullptr;   // server contexts: the shared Heff batcher
  cudaGraphExec_t gexec = nullptr;       // the Krylov step's executable graph (dmrg_params.graph)
  bool capturing = false;                // inside a stream capture: no timed tuner trials
  long long graph_launches = 0;
  bool batch_on = false;         // inside a served solve's sweeps: Heff goes to the batcher
  dmrg::GemmTuner tuner;
  cudaStream_t stream = nullptr;
  size_t budget = 0, in_use = 0, peak = 0;
  std::string err;
  int nsm = 148;
  dmrg::DescSlot slot[10];     // descriptor upload slots, one per family (see Upload::send)
  double* d_scal = nullptr;      // small scalar workspace (256 doubles)
  double* d_partial = nullptr;   // reduction partials (16 * 296 doubles)
  int* d_status = nullptr;
  double* h_scal = nullptr;      // pinned mirror of d_scal
  double* h_lam = nullptr;       // pinned eigenvalue download buffer (grow-only)
  size_t h_lam_cap = 0;
  double* dv_scal = nullptr;     // device addresses of h_scal / h_lam (null: not mapped, the
  double* dv_lam = nullptr;      // downloads then use a copy engine)
  cudaEvent_t ev[8] = {};
  std::vector<cudaEvent_t> tev;  // phase-timing events, reused across sweeps
  int max_groups = 4096;
  int* d_flags = nullptr;        // block-Jacobi per-group flags
  int* h_flags = nullptr;        // pinned
  double* d_floors = nullptr;    // block-Jacobi per-group thresholds
  // growable scratch buffers
  dmrg::DBuf X, Y, K, H, M, R, W, T1, T2;
  dmrg::DBuf SA, SB;             // chunk images of the split GEMM's operands (scratch)
  dmrg::DBuf SL, SR;             // chunk images of the Heff's environments (one plan at a time)
  uint64_t sl_key = 0, sr_key = 0;   // which plan and form SL / SR hold (0: none)
  std::map<void*, size_t> sizes;
  // Two-site sweeps run each environment update on env_stream, forked from `stream` once the
  // new site tensor is written (env_fork) and joined before the next Krylov solve (env_join),
  // so that it overlaps the split GEMM, the next centre normalisation and the next AA product.
  cudaStream_t env_stream = nullptr;
  cudaEvent_t env_fork = nullptr, env_join = nullptr;
  bool env_overlap = false;      // inside such a sweep: twostep records env_fork
  bool env_pending = false;      // env_join recorded and not yet waited on by `stream`
};

struct dmrg_mpo {
  dmrg_ctx* ctx = nullptr;
  int L = 0, nsym = 0;
  std::vector<dmrg::MPOSite> site;
  std::vector<dmrg::TwoSiteOp> two;   // per bond (iL, iL+1)
  std::vector<dmrg::TwoSiteOp> one;   // per site, for the single-site Heff
};

struct dmrg_state {
  dmrg_ctx* ctx = nullptr;
  const dmrg_mpo* mpo = nullptr;
  int L = 0, nsym = 0, oc = 0, dir = 1;
  std::vector<dmrg::Bond> bond;                 // L+1
  std::vector<dmrg::SiteLayout> lay;            // L
  std::vector<dmrg::DBuf> A;                    // L
  std::vector<dmrg::EnvLayout> Llay, Rlay;      // L
  std::vector<dmrg::DBuf> Lenv, Renv;           // L
  std::vector<char> Lvalid, Rvalid;
  bool env_built = false;
  // dmrgcvg bookkeeping (algs/DMRG.jl:610-652): set at the first sweep with goal > 0 after an
  // environment build (the start of a dmrg call), then updated after every sweep
  bool have_last = false;
  double last_energy = 0.0, last_entropy = 0.0;
};

namespace dmrg {

// ---- errors: thrown inside the library, converted to status codes at the ABI
struct Error {
  int code;
  std::string msg;
};
[[noreturn]] void fail(int code, const std::string& msg);
void cuda_check(cudaError_t e, const char* what);

// ---- memory
void dalloc(dmrg_ctx* c, DBuf& b, int64_t n);      // (re)allocate to exactly n doubles
void dfree(dmrg_ctx* c, DBuf& b);
void ensure(dmrg_ctx* c, DBuf& b, int64_t n);      // grow-only scratch

// ---- layouts (engine_layout.cpp)
SiteLayout make_site_layout(const Bond& Bl, const std::vector<QN>& p, const Bond& Br);
TwoLayout make_two_layout(const Bond& Bl, const std::vector<QN>& p1, const std::vector<QN>& p2,
                          const Bond& Br);
EnvLayout make_left_env_layout(const Bond& B, const std::vector<QN>& r);
EnvLayout make_right_env_layout(const Bond& B, const std::vector<QN>& r);
TwoSiteOp make_two_site_op(const MPOSite& a, const MPOSite& b);
// One MPO site in the two-site form with a trivial second site (d2 = 1): out[t * wr + w'].
TwoSiteOp make_one_site_op(const MPOSite& a);

// Device-to-host transfer of `bytes` (a multiple of 4) into pinned host memory at dst: written by
// a kernel through view, dst's device address, when there is one; else an asynchronous copy.
void to_host(dmrg_ctx* c, void* dst, void* view, const void* src, size_t bytes, const char* what);
// The device address of pinned host memory h, or null when the device cannot address it.
double* device_view(double* h);

// ---- descriptor upload
struct Upload {
  std::vector<char> bytes;
  template <class T>
  size_t put(const std::vector<T>& v) {
    size_t off = (bytes.size() + 15) / 16 * 16;
    bytes.resize(off + v.size() * sizeof(T));
    if (!v.empty()) std::memcpy(bytes.data() + off, v.data(), v.size() * sizeof(T));
    return off;
  }
  void put(GemmList& g) {
    g.t_off = put(g.tasks);
    g.s_off = put(g.segs);
    if (!g.si.empty()) {
      g.pa_off = put(g.pa);
      g.pb_off = put(g.pb);
      g.si_off = put(g.si);
    }
  }
  void put(MixList& m) { m.t_off = put(m.tasks); m.m_off = put(m.terms); }
  void put(CopyList& c) { c.t_off = put(c.tasks); }
  char* send(dmrg_ctx* c, int slot);   // returns the device base of the copied bytes
};

// Launch wrappers. Every launch first checks on the host that each task's extent lies inside
// the sizes (in doubles) of the buffers it addresses; a violation is a DMRG_ERR_ARG, never a
// device fault.
void run_gemm(dmrg_ctx* c, const GemmList& g, char* dbase, const double* A, int64_t nA,
              const double* B, int64_t nB, double* C, int64_t nC);
// The launch wrappers' bounds checks alone (DMRG_ERR_ARG on a violation).
void check_gemm_list(const GemmList& g, int64_t nA, int64_t nB, int64_t nC);
void check_mix_list(const MixList& m, int64_t nin, int64_t nout);
// Picks the FP64 tile shape of a list (before its upload): retiles it to 32 x 32 when the tuner
// says so or while that shape is on trial, and marks trial launches for timing.
void tune_gemm(dmrg_ctx* c, GemmList& g);
// Folds the timings of completed trial launches into the tuner (no synchronisation).
void tuner_collect(dmrg_ctx* c);
// The same list on a split-precision tcgen05 kernel (form SPLIT_TF32X3 or SPLIT_BF16X9); the list
// must be retiled. Lists of at least SPLIT_IMAGE_FLOPS take the image-fed form: their operand
// windows are converted once into chunk images first.
constexpr double SPLIT_IMAGE_FLOPS = 1e9;
// Tile width of a list's split form: TF32_TILE_N_DIRECT below SPLIT_IMAGE_FLOPS, else the
// image-fed width (TF32_TILE_N_IMAGE or TF32_TILE_N_WIDE) whose schedule the cost model
// finishes first.
int split_tile_n(const GemmList& g);
// Options of the image-fed form: an operand's images in a persistent buffer, packed only when
// *key differs from want (an environment, fixed over the applications of one Heff plan); and A
// given as the MPO mixing's input (the plan's fused covers) instead of the mixed blocks.
struct HeffPlan;
struct ImgCache {
  DBuf* buf = nullptr;
  uint64_t* key = nullptr;
  uint64_t want = 0;
};
struct SplitOpts {
  ImgCache a, b;
  const HeffPlan* fuse = nullptr;
};
void run_gemm_split(dmrg_ctx* c, const GemmList& g, char* dbase, const double* A, int64_t nA,
                    const double* B, int64_t nB, double* C, int64_t nC, int form,
                    const SplitOpts* opts = nullptr);
// The split form of a precision (0 for DMRG_PREC_FP64).
inline int split_form(int precision) {
  return precision == DMRG_PREC_3XTF32 ? SPLIT_TF32X3
         : precision == DMRG_PREC_BF16X9 ? SPLIT_BF16X9 : 0;
}
void run_mix(dmrg_ctx* c, const MixList& m, char* dbase, const double* in, int64_t nin,
             double* out, int64_t nout);
void run_copy(dmrg_ctx* c, const CopyList& l, char* dbase, const double* src, int64_t nsrc,
              double* dst, int64_t ndst);
void check_eig(const std::vector<EigTask>& t, int64_t nbase);

// Optional per-launch timing of GEMM launches (CUDA events on the context stream).
struct GemmProfile {
  std::vector<cudaEvent_t> pool;
  std::vector<std::pair<int, double>> pending;   // (event index of the start, flops)
  int used = 0;
  double flops = 0, seconds = 0;
  int launches = 0;
  void begin(cudaStream_t s, double fl);
  void end(cudaStream_t s);
  void flush();
  ~GemmProfile();
};

// ---- contractions (engine_contract.cpp)
struct HeffPlan {
  int le = 0, re = 0;            // the environments it reads: Lenv[le], Renv[re]
  uint64_t gen = 0;              // unique per plan (keys the environment images of the split form)
  TwoLayout tl;
  GemmList g1, g3;
  GemmList g1t, g3t;             // retiled copies for the split-precision kernel (when used)
  bool split = false;
  MixList mix;
  // split form with g3t image-fed: the mixing fused into the pack of g3t's A panels (per panel
  // its covers' range; the covers' terms are mix.terms)
  bool fused = false;
  std::vector<int2> fuse_range;
  std::vector<MixCover> fuse_cover;
  size_t fr_off = 0, fc_off = 0;
  int64_t x_size = 0, y_size = 0;
  double flops = 0;
  char* dbase = nullptr;
};
void plan_heff(const dmrg_state* st, int iL, HeffPlan& hp);
// The zero-site Heff of a bond matrix C[a, d] (OC_update, algs/time.jl:205-209):
// sum L[a,w,b] C[b,c] R[c,w,d] with Lenv[le] on bond Bl and Renv[re] on bond Br (the MPO bond
// between sites re and le); the same three launches with two trivial sites. C's layout: one
// block per sector of Bl, against the sector of Br with the same charge.
void plan_heff_bond(const dmrg_state* st, int le, int re, const Bond& Bl, const Bond& Br,
                    HeffPlan& hp);
// The single-site Heff at site i (singlesite_update, algs/optimizeMPS.jl:503-511): the same three
// launches with a second site of dimension one (charge zero), reading Lenv[i] and Renv[i]; its
// vector layout is the site layout of A[i].
void plan_heff1(const dmrg_state* st, int i, HeffPlan& hp);
// Uploads the Heff task lists (tuning the FP64 lists first); with a split precision also the
// retiled copies.
void upload_heff(dmrg_ctx* c, HeffPlan& hp, int slot, int precision = DMRG_PREC_FP64);
// Adds the Heff lists to an upload (the split lists and the fused mixing's covers when prepared).
void put_heff(Upload& u, HeffPlan& hp);
// Adds the retiled split-precision lists to a plan (before its upload), and the fused mixing's
// covers when the second GEMM is image-fed.
void prepare_split(HeffPlan& hp);
// y = Heff x for vectors in the tl layout (device pointers); reads Lenv[hp.le] and Renv[hp.re].
// Fails (DMRG_ERR_TIMEOUT) if a split-precision GEMM reported an MMA wait that gave up since the
// last check, and clears the flag. Synchronous read; call after a stream synchronisation.
void check_mma_status(dmrg_ctx* c);
void apply_heff(dmrg_state* st, int iL, const HeffPlan& hp, const double* x, double* y,
                int precision, GemmProfile* prof = nullptr);

// ---- shared Heff launches across the solves of a server (batch.cpp)
HeffBatcher* batcher_create(int device);
void batcher_destroy(HeffBatcher* b);
void batcher_enter(HeffBatcher* b);   // a solve starts its sweeps
void batcher_leave(HeffBatcher* b);   // ... and ends them
void batcher_stats(HeffBatcher* b, long long* batches, long long* contributions);
// y = Heff x of one solve, run inside the batcher's next shared launch.
void batched_heff(dmrg_ctx* c, dmrg_state* st, int iL, const HeffPlan& hp, const double* x,
                  double* y, int precision);

// Heff with every intermediate in the library's fixed device array (noalloc.cu).
void heff_apply_noalloc(dmrg_state* st, int iL, const double* in_dev, double* out_dev);

// One environment step through one site (lib/MPO_MPS/Lupdate.jl:17-26, Rupdate.jl:17-26):
// g1 (env_in, A) -> T1, mix T1 -> T2 (the MPO site), g3 (A, T2) -> env_out in layout `out`.
struct StepPlan {
  GemmList g1, g3;
  GemmList g1t, g3t;        // retiled copies for the split-precision kernel (split != 0)
  int split = 0;            // split form of the two GEMMs, 0 = FP64
  MixList mx;
  EnvLayout out;
  int64_t t1 = 0, t2 = 0;   // scratch sizes in doubles
  double flops() const { return g1.flops + g3.flops + mx.flops; }
};
void plan_left_step(const Bond& Bl, const Bond& Br, const MPOSite& ms, const SiteLayout& lay,
                    const EnvLayout& LL, StepPlan& sp);
void plan_right_step(const Bond& Bl, const Bond& Br, const MPOSite& ms, const SiteLayout& lay,
                     const EnvLayout& RL, StepPlan& sp);
// Uploads the step's lists; with split = true also their split-precision retilings (the step then
// runs its two GEMMs on the 3xTF32 tensor-core kernel; the MPO mixing stays FP64).
void put_step(Upload& u, StepPlan& sp, int split = 0);
// Launches an uploaded step; c->T1 / c->T2 must hold sp.t1 / sp.t2 doubles. `bra` (optional)
// is the conjugated tensor when it differs from the ket tensor A (the dualpsi argument of
// Lupdate/Rupdate); both share A's layout.
void run_step(dmrg_ctx* c, const StepPlan& sp, char* db, const double* env_in, int64_t n_in,
              const DBuf& A, double* env_out, int64_t n_out, const DBuf* bra = nullptr);
// Lupdate(Lenv, dualpsi, psi, mpo) / Rupdate(...) as a pure function of dense host tensors.
void env_step_dense(dmrg_ctx* c, bool left, int ml, int d, int mr, int wl, int wr,
                    const double* env_in, const double* dual, const double* psi, const double* W,
                    double* env_out);

void env_boundaries(dmrg_state* st);
void lupdate(dmrg_state* st, int i, double* flops, int precision = DMRG_PREC_FP64);
void rupdate(dmrg_state* st, int i, double* flops, int precision = DMRG_PREC_FP64);

// ---- measurements (engine_meas.cpp)
// <psi|H|psi> for an MPO over the same sites and physical charges (not normalised).
double measure_expect(dmrg_state* st, const dmrg_mpo* H, double* flops);
// rho (L x L, column-major): two-point correlations of Cc and Ca with an optional trail F
// (d x d column-major operators [bra, ket]; F may be null), normalised by <psi|psi>.
// correlation(psi, ops...; sites, trail) with dualpsi = psi: operator g has lens[g] d x d factors
// (packed in `ops`), start positions sites[..] (nsites[g] entries, 0-based; the last lens[g] - 1
// are not used as starts, as in the reference) and an optional trail (trails: n matrices or
// null); omega has prod_g (nsites[g] - lens[g] + 1) entries, the first operator's index fastest.
void measure_correlation_n(dmrg_state* st, int d, int n, const int* lens, const double* ops,
                           const int* nsites, const int* sites, const double* trails,
                           double* omega, double* flops);
// (norm, optional: receives <psi|psi>, by which rho was divided)
void measure_correlation(dmrg_state* st, int d, const double* Cc, const double* Ca,
                         const double* F, double* rho, double* flops, double* norm = nullptr);

// ---- eigensolves (engine_eig.cpp)
// Tridiagonal-path eigenvalues of every task (n <= SYEVT_MID_NMAX; small and mid-size blocks in
// one launch each), then the kept eigenvectors (tasks with keep > 0; mid-size blocks use c->W
// as workspace). Offsets are checked against nbase before any launch.
void run_trid_eigvals(dmrg_ctx* c, double* base, int64_t nbase, const std::vector<TridTask>& t,
                      int slot);
void run_trid_vectors(dmrg_ctx* c, double* base, int64_t nbase, std::vector<TridTask> t,
                      int slot);
int64_t eig_workspace(const std::vector<EigTask>& tasks);
void run_eigs(dmrg_ctx* c, double* base, int64_t nbase, const std::vector<EigTask>& tasks,
              int64_t ws_off, int* sweeps);

// ---- sweep (engine_sweep.cpp)
void do_sweep(dmrg_state* st, const dmrg_params& p, dmrg_sweep_stats& out);
// ---- single-site sweep with subspace expansion (engine_3s.cpp). `noise` is alpha (in: the
// current value, out: after the sweep's last alpha_update); last_energy is the lastEnergy of
// alpha_update (the previous sweep's energy, or the starting energy).
void do_sweep3s(dmrg_state* st, const dmrg_params& p, const dmrg_noise& nz, double* noise,
                double last_energy, dmrg_sweep_stats& out);
// ---- TDVP with a real prefactor (engine_tdvp.cpp): one call of tdvp_twosite (twosite) or tdvp
void do_tdvp(dmrg_state* st, const dmrg_params& p, double prefactor, bool twosite,
             dmrg_sweep_stats& out);

}  // namespace dmrg
