// engine_layout.cpp -- block layouts, device memory, descriptor upload, launch wrappers.
#include <algorithm>
#include <cmath>
#include <map>
#include <tuple>

#include "engine.hpp"

namespace dmrg {

[[noreturn]] void fail(int code, const std::string& msg) { throw Error{code, msg}; }

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    int code = (e == cudaErrorMemoryAllocation) ? DMRG_ERR_OOM : DMRG_ERR_CUDA;
    fail(code, std::string(what) + ": " + cudaGetErrorString(e));
  }
}

int Bond::find(const QN& x) const {
  auto it = std::lower_bound(q.begin(), q.end(), x);
  if (it == q.end() || !(*it == x)) return -1;
  return int(it - q.begin());
}

int64_t Bond::total() const {
  int64_t t = 0;
  for (int d : dim) t += d;
  return t;
}

std::vector<int64_t> Bond::offsets() const {
  std::vector<int64_t> o(dim.size());
  int64_t t = 0;
  for (size_t i = 0; i < dim.size(); ++i) { o[i] = t; t += dim[i]; }
  return o;
}

// ------------------------------------------------------------------ memory

void dalloc(dmrg_ctx* c, DBuf& b, int64_t n) {
  dfree(c, b);
  if (n <= 0) return;
  size_t bytes = size_t(n) * sizeof(double);
  if (c->budget && c->in_use + bytes > c->budget)
    fail(DMRG_ERR_BUDGET, "device allocation of " + std::to_string(bytes) +
                              " bytes exceeds the context's HBM budget");
  void* p = nullptr;
  cudaError_t e = cudaMallocAsync(&p, bytes, c->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    fail(DMRG_ERR_OOM, "cudaMallocAsync(" + std::to_string(bytes) + "): " + cudaGetErrorString(e));
  }
  b.p = static_cast<double*>(p);
  b.n = n;
  c->in_use += bytes;
  c->peak = std::max(c->peak, c->in_use);
  c->sizes[p] = bytes;
}

void dfree(dmrg_ctx* c, DBuf& b) {
  if (!b.p) return;
  auto it = c->sizes.find(b.p);
  if (it != c->sizes.end()) {
    c->in_use -= it->second;
    c->sizes.erase(it);
  }
  cudaFreeAsync(b.p, c->stream);
  b.p = nullptr;
  b.n = 0;
}

void ensure(dmrg_ctx* c, DBuf& b, int64_t n) {
  if (n <= b.n) return;
  int64_t want = std::max<int64_t>(n, b.n + b.n / 4);
  dalloc(c, b, want);
}

// ------------------------------------------------------------------ layouts

SiteLayout make_site_layout(const Bond& Bl, const std::vector<QN>& p, const Bond& Br) {
  SiteLayout L;
  L.nl = Bl.nsec();
  L.d = int(p.size());
  L.kb.assign(size_t(L.nl) * L.d, -1);
  L.off.assign(size_t(L.nl) * L.d, 0);
  L.goff.assign(L.nl, 0);
  L.gcols.assign(L.nl, 0);
  int64_t off = 0;
  for (int ka = 0; ka < L.nl; ++ka) {
    L.goff[ka] = off;
    for (int s = 0; s < L.d; ++s) {
      int kb = Br.find(Bl.q[ka] + p[s]);
      L.kb[ka * L.d + s] = kb;
      if (kb < 0) continue;
      L.off[ka * L.d + s] = off;
      off += int64_t(Bl.dim[ka]) * Br.dim[kb];
      L.gcols[ka] += Br.dim[kb];
    }
  }
  L.size = off;
  return L;
}

TwoLayout make_two_layout(const Bond& Bl, const std::vector<QN>& p1, const std::vector<QN>& p2,
                          const Bond& Br) {
  TwoLayout T;
  T.nl = Bl.nsec();
  T.d1 = int(p1.size());
  T.d2 = int(p2.size());
  const size_t nb = size_t(T.nl) * T.d1 * T.d2;
  T.kd.assign(nb, -1);
  T.off.assign(nb, 0);
  T.goff.assign(T.nl, 0);
  T.gcols.assign(T.nl, 0);
  int64_t off = 0;
  for (int ka = 0; ka < T.nl; ++ka) {
    T.goff[ka] = off;
    for (int s1 = 0; s1 < T.d1; ++s1)
      for (int s2 = 0; s2 < T.d2; ++s2) {
        int kd = Br.find(Bl.q[ka] + p1[s1] + p2[s2]);
        int id = T.idx(ka, s1, s2);
        T.kd[id] = kd;
        if (kd < 0) continue;
        T.off[id] = off;
        off += int64_t(Bl.dim[ka]) * Br.dim[kd];
        T.gcols[ka] += Br.dim[kd];
      }
  }
  T.size = off;
  return T;
}

// Left env on bond B with MPO labels r: ket sector kb, MPO state w -> bra sector q(kb) - r(w).
EnvLayout make_left_env_layout(const Bond& B, const std::vector<QN>& r) {
  EnvLayout E;
  E.nsec = B.nsec();
  E.w = int(r.size());
  E.other.assign(size_t(E.nsec) * E.w, -1);
  E.rowoff.assign(size_t(E.nsec) * E.w, 0);
  E.rows.assign(E.nsec, 0);
  E.goff.assign(E.nsec, 0);
  int64_t off = 0;
  for (int kb = 0; kb < E.nsec; ++kb) {
    int rows = 0;
    for (int w = 0; w < E.w; ++w) {
      int ka = B.find(B.q[kb] - r[w]);
      E.other[kb * E.w + w] = ka;
      E.rowoff[kb * E.w + w] = rows;
      if (ka >= 0) rows += B.dim[ka];
    }
    E.rows[kb] = rows;
    E.goff[kb] = off;
    off += int64_t(rows) * B.dim[kb];
  }
  E.size = off;
  return E;
}

// Right env on bond B with MPO labels r: bra sector ka, MPO state w -> ket sector q(ka) + r(w).
EnvLayout make_right_env_layout(const Bond& B, const std::vector<QN>& r) {
  EnvLayout E;
  E.nsec = B.nsec();
  E.w = int(r.size());
  E.other.assign(size_t(E.nsec) * E.w, -1);
  E.rowoff.assign(size_t(E.nsec) * E.w, 0);
  E.rows.assign(E.nsec, 0);
  E.goff.assign(E.nsec, 0);
  int64_t off = 0;
  for (int ka = 0; ka < E.nsec; ++ka) {
    int rows = 0;
    for (int w = 0; w < E.w; ++w) {
      int kb = B.find(B.q[ka] + r[w]);
      E.other[ka * E.w + w] = kb;
      E.rowoff[ka * E.w + w] = rows;
      if (kb >= 0) rows += B.dim[kb];
    }
    E.rows[ka] = rows;
    E.goff[ka] = off;
    off += int64_t(rows) * B.dim[ka];
  }
  E.size = off;
  return E;
}

// ops[w,s1,t1,s2,t2,w''] = sum_w' WL[w,s1,t1,w'] WR[w',s2,t2,w''] (contract(mpoL,4,mpoR,1),
// algs/DMRG.jl:70), kept sparse and grouped by the output channel (t1,t2,w'').
TwoSiteOp make_two_site_op(const MPOSite& a, const MPOSite& b) {
  TwoSiteOp op;
  op.d1 = a.d;
  op.d2 = b.d;
  op.wl = a.wl;
  op.wr = b.wr;
  op.out.assign(size_t(a.d) * b.d * b.wr, {});
  std::vector<std::vector<const MPOSite::El*>> byw(b.wl);
  for (const auto& e : b.nz) byw[e.w].push_back(&e);
  std::map<std::tuple<int, int, int, int, int, int>, double> acc;
  for (const auto& ea : a.nz)
    for (const MPOSite::El* eb : byw[ea.w2])
      acc[{ea.t, eb->t, eb->w2, ea.w, ea.s, eb->s}] += ea.v * eb->v;
  for (const auto& kv : acc) {
    if (kv.second == 0.0) continue;
    auto [t1, t2, w2, w, s1, s2] = kv.first;
    op.out[(size_t(t1) * b.d + t2) * b.wr + w2].push_back({w, s1, s2, kv.second});
  }
  return op;
}

TwoSiteOp make_one_site_op(const MPOSite& a) {
  TwoSiteOp op;
  op.d1 = a.d;
  op.d2 = 1;
  op.wl = a.wl;
  op.wr = a.wr;
  op.out.assign(size_t(a.d) * a.wr, {});
  for (const auto& e : a.nz)
    if (e.v != 0.0) op.out[size_t(e.t) * a.wr + e.w2].push_back({e.w, e.s, 0, e.v});
  return op;
}

// ------------------------------------------------------------------ task lists

void GemmList::add(int64_t c_off, int ldc, int M, int N, double alpha, double beta) {
  GemmTask t{};
  t.c_off = c_off;
  t.ldc = ldc;
  t.M = M;
  t.N = N;
  t.seg0 = int(segs.size());
  t.nseg = 0;
  t.tiles_m = (M + bm - 1) / bm;
  t.tile0 = tiles;
  t.alpha = alpha;
  t.beta = beta;
  if (M <= 0 || N <= 0) { t.tiles_m = 0; }
  tiles += t.tiles_m * ((N + GEMM_BN - 1) / GEMM_BN);
  tasks.push_back(t);
}

// The image plan of a list retiled to TF32_TILE_M x g.bn (image-fed form): one panel per
// distinct operand window (offset, leading dimension, rows, K), its chunk images after those of
// the panels before it; A row tiles of SPLIT_IMG_ROWS rows, B row tiles of g.bn rows.
static void plan_images(GemmList& g) {
  using Key = std::tuple<int64_t, int, int, int>;
  std::map<Key, int> ia, ib;
  g.pa.clear();
  g.pb.clear();
  g.si.assign(g.segs.size(), SegImg{});
  g.img_a = g.img_b = 0;
  auto panel = [](std::map<Key, int>& idx, std::vector<ImgPanel>& ps, int64_t& total,
                  int64_t off, int ld, int rows, int K, int kcontig, int tile_rows) {
    const Key k{off, ld, rows, K};
    auto it = idx.find(k);
    if (it == idx.end()) {
      ImgPanel p{};
      p.off = off;
      p.ld = ld;
      p.rows = rows;
      p.K = K;
      p.kcontig = kcontig;
      p.kchunks = (K + SPLIT_IMG_K - 1) / SPLIT_IMG_K;
      p.img0 = total;
      total += int64_t((rows + tile_rows - 1) / tile_rows) * p.kchunks;
      it = idx.emplace(k, int(ps.size())).first;
      ps.push_back(p);
    }
    return ps[it->second];
  };
  for (const GemmTask& t : g.tasks) {
    if (t.M <= 0 || t.N <= 0) continue;
    for (int q = 0; q < t.nseg; ++q) {
      const GemmSeg& s = g.segs[t.seg0 + q];
      if (s.K <= 0) continue;
      SegImg& m = g.si[t.seg0 + q];
      // op(A) is M x K: K contiguous when A is stored transposed; op(B) is K x N, read as the
      // N x K window of B^T: K contiguous when B is stored untransposed
      const ImgPanel a =
          panel(ia, g.pa, g.img_a, s.a_off, s.lda, t.M, s.K, g.tA ? 1 : 0, SPLIT_IMG_ROWS);
      const ImgPanel b = panel(ib, g.pb, g.img_b, s.b_off, s.ldb, t.N, s.K, g.tB ? 0 : 1, g.bn);
      m.a_img = a.img0;
      m.a_kchunks = a.kchunks;
      m.b_img = b.img0;
      m.b_kchunks = b.kchunks;
    }
  }
}

GemmList retile(const GemmList& g, int bm, int bn) {
  GemmList r;
  r.tA = g.tA;
  r.tB = g.tB;
  r.bm = bm;
  r.bn = bn;
  r.segs = g.segs;
  r.flops = g.flops;
  r.tasks = g.tasks;
  r.tiles = 0;
  for (GemmTask& t : r.tasks) {
    t.tiles_m = (t.M <= 0 || t.N <= 0) ? 0 : (t.M + bm - 1) / bm;
    t.tile0 = r.tiles;
    r.tiles += t.tiles_m * ((t.N + bn - 1) / bn);
  }
  if (bm == TF32_TILE_M && (bn == TF32_TILE_N_IMAGE || bn == TF32_TILE_N_WIDE)) plan_images(r);
  return r;
}

// A 256-column tile runs its MMAs at about this many times the rate of a 128-column one: per
// TF32 product it reads 12 KB of operands from shared memory in 128 cycles against 8 KB in 64.
constexpr double WIDE_TILE_RATE = 1.3;

int split_tile_n(const GemmList& g) {
  if (g.flops < SPLIT_IMAGE_FLOPS) return TF32_TILE_N_DIRECT;
  // the image-fed kernel runs one CTA per SM and hands out tiles round-robin: the makespan of
  // each width is the largest CTA load (tile work = columns x K chunks) over its rate
  const int P = std::max(device_sm_count(), 1);
  double best = 0;
  int pick = TF32_TILE_N_IMAGE;
  for (int bn : {TF32_TILE_N_IMAGE, TF32_TILE_N_WIDE}) {
    int64_t ntiles = 0;
    for (const GemmTask& t : g.tasks)
      if (t.M > 0 && t.N > 0)
        ntiles += int64_t((t.M + TF32_TILE_M - 1) / TF32_TILE_M) * ((t.N + bn - 1) / bn);
    const int grid = int(std::min<int64_t>(ntiles, P));
    if (grid == 0) return TF32_TILE_N_IMAGE;
    std::vector<double> load(grid, 0.0);
    int64_t tile = 0;
    for (const GemmTask& t : g.tasks) {
      if (t.M <= 0 || t.N <= 0) continue;
      double kch = 0;
      for (int q = 0; q < t.nseg; ++q) {
        const int K = g.segs[t.seg0 + q].K;
        if (K > 0) kch += (K + SPLIT_IMG_K - 1) / SPLIT_IMG_K;
      }
      const int64_t n = int64_t((t.M + TF32_TILE_M - 1) / TF32_TILE_M) * ((t.N + bn - 1) / bn);
      for (int64_t i = 0; i < n; ++i, ++tile) load[tile % grid] += bn * kch;
    }
    const double span = *std::max_element(load.begin(), load.end()) /
                        (bn == TF32_TILE_N_WIDE ? WIDE_TILE_RATE : 1.0);
    if (bn == TF32_TILE_N_IMAGE || span < best) {
      best = span;
      pick = bn;
    }
  }
  return pick;
}

void GemmList::seg(int64_t a_off, int lda, int64_t b_off, int ldb, int K) {
  if (K <= 0) return;
  GemmSeg s{};
  s.a_off = a_off;
  s.b_off = b_off;
  s.lda = lda;
  s.ldb = ldb;
  s.K = K;
  segs.push_back(s);
  GemmTask& t = tasks.back();
  t.nseg += 1;
  flops += 2.0 * t.M * double(t.N) * K;
}

void MixList::add(int64_t out_off, int ld, int rows, int cols) {
  MixTask t{};
  t.out_off = out_off;
  t.ld = ld;
  t.rows = rows;
  t.cols = cols;
  t.term0 = int(terms.size());
  t.nterm = 0;
  t.tile0 = tiles;
  t.ntiles = (rows > 0 && cols > 0) ? (cols + 31) / 32 : 0;
  tiles += t.ntiles;
  tasks.push_back(t);
}

void MixList::term(int64_t in_off, int ld, double c) {
  MixTerm m{};
  m.in_off = in_off;
  m.ld = ld;
  m.coef = c;
  terms.push_back(m);
  MixTask& t = tasks.back();
  t.nterm += 1;
  flops += 2.0 * t.rows * double(t.cols);
}

void CopyList::add(int64_t src_off, int lds, int64_t dst_off, int ldd, int rows, int cols,
                   int trans, double scale) {
  if (rows <= 0 || cols <= 0) return;
  CopyTask t{};
  t.src_off = src_off;
  t.dst_off = dst_off;
  t.lds = lds;
  t.ldd = ldd;
  t.rows = rows;
  t.cols = cols;
  t.trans = trans;
  t.tile0 = tiles;
  t.ntiles = (cols + 31) / 32;
  t.scale = scale;
  tiles += t.ntiles;
  tasks.push_back(t);
}

void to_host(dmrg_ctx* c, void* dst, void* view, const void* src, size_t bytes,
             const char* what) {
  if (view && bytes % 4 == 0) {
    launch_to_host(c->stream, src, view, bytes);
    cuda_check(cudaGetLastError(), what);
  } else {
    cuda_check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream), what);
  }
}

double* device_view(double* h) {
  void* d = nullptr;
  if (!h || cudaHostGetDevicePointer(&d, h, 0) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return static_cast<double*>(d);
}

char* Upload::send(dmrg_ctx* c, int slot) {
  DescSlot& s = c->slot[slot];
  size_t need = bytes.size() < 16 ? 16 : bytes.size();
  // Lists that fit a kernel's parameter block travel with a launch (no staging, no copy
  // engine); stream order keeps the slot's previous readers ahead of the write. The launch
  // writes whole 16-byte words, so the slot must hold the rounded-up size.
  if ((need + 15) / 16 * 16 <= s.cap && launch_upload(c->stream, bytes.data(), bytes.size(), s.d))
    return s.d;
  if (s.ev) cuda_check(cudaEventSynchronize(s.ev), "descriptor slot wait");
  if (need > s.cap) {
    size_t cap = (std::max(need, s.cap * 2) + 15) / 16 * 16;
    if (s.h) cudaFreeHost(s.h);
    if (s.d) cudaFreeAsync(s.d, c->stream);
    cuda_check(cudaMallocHost(reinterpret_cast<void**>(&s.h), cap), "cudaMallocHost(desc)");
    cuda_check(cudaMallocAsync(reinterpret_cast<void**>(&s.d), cap, c->stream), "cudaMalloc(desc)");
    s.cap = cap;
  }
  if (!bytes.empty()) {
    std::memcpy(s.h, bytes.data(), bytes.size());
    cuda_check(cudaMemcpyAsync(s.d, s.h, bytes.size(), cudaMemcpyHostToDevice, c->stream),
               "descriptor upload");
  }
  if (!s.ev) cuda_check(cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming), "event");
  cuda_check(cudaEventRecord(s.ev, c->stream), "event record");
  return s.d;
}

namespace {
inline bool in_range(int64_t off, int64_t last, int64_t n) { return off >= 0 && off + last < n; }
[[noreturn]] void bad_plan(const char* what) {
  fail(DMRG_ERR_ARG, std::string("internal plan check failed: ") + what + " out of bounds");
}
}  // namespace

void check_gemm_list(const GemmList& g, int64_t nA, int64_t nB, int64_t nC) {
  for (const GemmTask& t : g.tasks) {
    if (t.M <= 0 || t.N <= 0) continue;
    if (t.ldc < t.M || !in_range(t.c_off, (t.M - 1) + int64_t(t.N - 1) * t.ldc, nC)) bad_plan("gemm C");
    for (int q = 0; q < t.nseg; ++q) {
      const GemmSeg& s = g.segs[t.seg0 + q];
      const int64_t ea = g.tA ? (s.K - 1) + int64_t(t.M - 1) * s.lda : (t.M - 1) + int64_t(s.K - 1) * s.lda;
      const int64_t eb = g.tB ? (t.N - 1) + int64_t(s.K - 1) * s.ldb : (s.K - 1) + int64_t(t.N - 1) * s.ldb;
      if (s.lda < (g.tA ? s.K : t.M) || !in_range(s.a_off, ea, nA)) bad_plan("gemm A");
      if (s.ldb < (g.tB ? t.N : s.K) || !in_range(s.b_off, eb, nB)) bad_plan("gemm B");
    }
  }
}

void check_mix_list(const MixList& m, int64_t nin, int64_t nout) {
  for (const MixTask& t : m.tasks) {
    if (t.rows <= 0 || t.cols <= 0) continue;
    const int64_t ext = (t.rows - 1) + int64_t(t.cols - 1) * t.ld;
    if (t.ld < t.rows || !in_range(t.out_off, ext, nout)) bad_plan("mix out");
    for (int q = 0; q < t.nterm; ++q) {
      const MixTerm& tm = m.terms[t.term0 + q];
      if (tm.ld < t.rows || !in_range(tm.in_off, (t.rows - 1) + int64_t(t.cols - 1) * tm.ld, nin))
        bad_plan("mix in");
    }
  }
}

void run_gemm(dmrg_ctx* c, const GemmList& g, char* dbase, const double* A, int64_t nA,
              const double* B, int64_t nB, double* C, int64_t nC) {
  if (g.tiles == 0) return;
  check_gemm_list(g, nA, nB, nC);
  if ((g.bm != GEMM_BM || g.bn != GEMM_BN) &&
      (g.bm != GEMM_SMALL_TILE || g.bn != GEMM_SMALL_TILE))
    bad_plan("gemm tiling");
  GemmTuner::Pending tp{};
  const bool timed = g.tune_trial && g.tune_key != 0 && !c->capturing;
  if (timed) {
    for (cudaEvent_t* e : {&tp.a, &tp.b}) {
      if (!c->tuner.free_events.empty()) {
        *e = c->tuner.free_events.back();
        c->tuner.free_events.pop_back();
      } else {
        cuda_check(cudaEventCreate(e), "tuner event");
      }
    }
    tp.key = g.tune_key;
    tp.variant = g.bm == GEMM_SMALL_TILE ? 1 : 0;
    cudaEventRecord(tp.a, c->stream);
  }
  launch_gemm_f64(c->stream, g.bm, g.tA, g.tB, A, B, C,
                  reinterpret_cast<const GemmTask*>(dbase + g.t_off), int(g.tasks.size()),
                  reinterpret_cast<const GemmSeg*>(dbase + g.s_off), g.tiles, c->nsm * 4);
  if (timed) {
    cudaEventRecord(tp.b, c->stream);
    c->tuner.pending.push_back(tp);
  }
}

GemmTuner::~GemmTuner() {
  for (auto& p : pending) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
  for (cudaEvent_t e : free_events) cudaEventDestroy(e);
}

namespace {
int half_octave(double x) { return x <= 1.0 ? 0 : int(std::floor(2.0 * std::log2(x))) + 1; }
}  // namespace

void tune_gemm(dmrg_ctx* c, GemmList& g) {
  g.tune_key = 0;
  g.tune_trial = 0;
  if (!c->tune || g.tasks.empty() || g.flops <= 0) return;
  double wm = 0, wn = 0, wk = 0, w = 0;
  for (const GemmTask& t : g.tasks) {
    if (t.M <= 0 || t.N <= 0) continue;
    for (int q = 0; q < t.nseg; ++q) {
      const GemmSeg& s = g.segs[t.seg0 + q];
      const double f = double(t.M) * t.N * s.K;
      wm += f * t.M; wn += f * t.N; wk += f * s.K; w += f;
    }
  }
  if (w <= 0) return;
  uint64_t key = 1;
  for (int v : {int(g.tA), int(g.tB), half_octave(wm / w), half_octave(wn / w), half_octave(wk / w),
                half_octave(double(g.tasks.size())), half_octave(g.flops)})
    key = key * 131 + uint64_t(v & 0xff);
  g.tune_key = key;
  GemmTuner::Entry& e = c->tuner.table[key];
  int v = e.choice;
  if (v < 0) {   // on trial: the shape with fewer finished or pending trials
    int pend[2] = {0, 0};
    for (const auto& p : c->tuner.pending)
      if (p.key == key) pend[p.variant] += 1;
    v = (e.trials[0] + pend[0] <= e.trials[1] + pend[1]) ? 0 : 1;
    g.tune_trial = 1;
  }
  if (v == 1) g = [&] {
    GemmList r = retile(g, GEMM_SMALL_TILE, GEMM_SMALL_TILE);
    r.tune_key = g.tune_key;
    r.tune_trial = g.tune_trial;
    return r;
  }();
}

void tuner_collect(dmrg_ctx* c) {
  auto& P = c->tuner.pending;
  size_t keep = 0;
  for (size_t i = 0; i < P.size(); ++i) {
    GemmTuner::Pending& p = P[i];
    if (cudaEventQuery(p.b) != cudaSuccess) {
      cudaGetLastError();     // not ready is not an error
      P[keep++] = p;
      continue;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, p.a, p.b);
    GemmTuner::Entry& e = c->tuner.table[p.key];
    e.trials[p.variant] += 1;
    e.best[p.variant] = std::min(e.best[p.variant], double(ms));
    if (e.choice < 0 && e.trials[0] > 0 && e.trials[1] > 0)
      e.choice = (e.best[1] < 0.97 * e.best[0]) ? 1 : 0;
    c->tuner.free_events.push_back(p.a);
    c->tuner.free_events.push_back(p.b);
  }
  P.resize(keep);
}

void run_gemm_split(dmrg_ctx* c, const GemmList& g, char* dbase, const double* A, int64_t nA,
                    const double* B, int64_t nB, double* C, int64_t nC, int form,
                    const SplitOpts* opts) {
  if (form != SPLIT_TF32X3 && form != SPLIT_BF16X9) bad_plan("split gemm form");
  if (g.tiles == 0) return;
  if (g.bm != TF32_TILE_M || (g.bn != TF32_TILE_N_DIRECT && g.bn != TF32_TILE_N_IMAGE &&
                              g.bn != TF32_TILE_N_WIDE))
    bad_plan("split gemm tiling");
  for (const GemmTask& t : g.tasks) {
    if (t.M <= 0 || t.N <= 0) continue;
    if (t.ldc < t.M || !in_range(t.c_off, (t.M - 1) + int64_t(t.N - 1) * t.ldc, nC)) bad_plan("gemm C");
    for (int q = 0; q < t.nseg; ++q) {
      const GemmSeg& s = g.segs[t.seg0 + q];
      const int64_t ea = g.tA ? (s.K - 1) + int64_t(t.M - 1) * s.lda : (t.M - 1) + int64_t(s.K - 1) * s.lda;
      const int64_t eb = g.tB ? (t.N - 1) + int64_t(s.K - 1) * s.ldb : (s.K - 1) + int64_t(t.N - 1) * s.ldb;
      if (s.lda < (g.tA ? s.K : t.M) || !in_range(s.a_off, ea, nA)) bad_plan("gemm A");
      if (s.ldb < (g.tB ? t.N : s.K) || !in_range(s.b_off, eb, nB)) bad_plan("gemm B");
    }
  }
  const GemmTask* tasks = reinterpret_cast<const GemmTask*>(dbase + g.t_off);
  const GemmSeg* segs = reinterpret_cast<const GemmSeg*>(dbase + g.s_off);
  if (g.bn != TF32_TILE_N_DIRECT) {   // image-fed form (large lists)
    // every chunk a segment's tiles copy lies inside the images, and every panel the pack pass
    // reads lies inside its operand
    if (g.si.size() != g.segs.size()) bad_plan("split gemm images");
    for (const GemmTask& t : g.tasks) {
      if (t.M <= 0 || t.N <= 0) continue;
      const int64_t tiles_n = (t.N + g.bn - 1) / g.bn;
      for (int q = 0; q < t.nseg; ++q) {
        const GemmSeg& s = g.segs[t.seg0 + q];
        if (s.K <= 0) continue;
        const SegImg& m = g.si[t.seg0 + q];
        const int kch = (s.K + SPLIT_IMG_K - 1) / SPLIT_IMG_K;
        if (m.a_kchunks != kch || m.b_kchunks != kch || m.a_img < 0 || m.b_img < 0 ||
            m.a_img + int64_t(t.tiles_m) * kch > g.img_a || m.b_img + tiles_n * kch > g.img_b)
          bad_plan("split gemm images");
      }
    }
    auto check_panels = [](const std::vector<ImgPanel>& ps, int64_t total, int64_t n,
                           int tile_rows, bool extent) {
      int64_t next = 0;
      for (const ImgPanel& p : ps) {
        if (p.rows <= 0 || p.K <= 0 || p.img0 != next ||
            p.kchunks != (p.K + SPLIT_IMG_K - 1) / SPLIT_IMG_K)
          bad_plan("split gemm panels");
        const int64_t last = p.kcontig ? (p.K - 1) + int64_t(p.rows - 1) * p.ld
                                       : (p.rows - 1) + int64_t(p.K - 1) * p.ld;
        if (extent && (p.ld < (p.kcontig ? p.K : p.rows) || !in_range(p.off, last, n)))
          bad_plan("split gemm panels");
        next += int64_t((p.rows + tile_rows - 1) / tile_rows) * p.kchunks;
      }
      if (next != total) bad_plan("split gemm panels");
    };
    const HeffPlan* fuse = opts ? opts->fuse : nullptr;
    if (fuse) {
      // A is the mixing input: the covers of every A panel tile its columns, and every term a
      // cover sums reads inside the input
      const MixList& mx = fuse->mix;
      if (!fuse->fused || fuse->fuse_range.size() != g.pa.size()) bad_plan("split gemm mixing");
      for (size_t i = 0; i < g.pa.size(); ++i) {
        const ImgPanel& p = g.pa[i];
        const int2 r = fuse->fuse_range[i];
        if (p.kcontig || r.y < 1 || r.x < 0 || size_t(r.x) + r.y > fuse->fuse_cover.size())
          bad_plan("split gemm mixing");
        int next = 0;
        for (int j = r.x; j < r.x + r.y; ++j) {
          const MixCover& cv = fuse->fuse_cover[j];
          if (cv.col0 != next || cv.ncols <= 0 || cv.term0 < 0 || cv.nterm < 0 ||
              size_t(cv.term0) + cv.nterm > mx.terms.size())
            bad_plan("split gemm mixing");
          next += cv.ncols;
          for (int q = cv.term0; q < cv.term0 + cv.nterm; ++q) {
            const MixTerm& tm = mx.terms[q];
            if (tm.ld < p.rows ||
                !in_range(tm.in_off, (p.rows - 1) + int64_t(cv.ncols - 1) * tm.ld, nA))
              bad_plan("split gemm mixing");
          }
        }
        if (next != p.K) bad_plan("split gemm mixing");
      }
    }
    check_panels(g.pa, g.img_a, nA, SPLIT_IMG_ROWS, fuse == nullptr);
    check_panels(g.pb, g.img_b, nB, g.bn, true);
    const int64_t cba = split_image_chunk_bytes(form, SPLIT_IMG_ROWS);
    const int64_t cbb = split_image_chunk_bytes(form, g.bn);
    // an operand's images: the scratch buffer, or a cache that is packed when its key differs
    // (a cache that has to grow loses its contents)
    auto images = [&](const ImgCache* cache, DBuf& scratch, int64_t bytes, bool& pack) {
      const int64_t n = std::max<int64_t>((bytes + 7) / 8, 1);
      pack = true;
      if (!cache || !cache->buf) {
        ensure(c, scratch, n);
        return reinterpret_cast<unsigned char*>(scratch.p);
      }
      if (cache->buf->n < n) {
        *cache->key = 0;
        ensure(c, *cache->buf, n);
      }
      pack = *cache->key != cache->want;
      *cache->key = cache->want;
      return reinterpret_cast<unsigned char*>(cache->buf->p);
    };
    bool pack_a = true, pack_b = true;
    unsigned char* ia = images(opts ? &opts->a : nullptr, c->SA, g.img_a * cba, pack_a);
    unsigned char* ib = images(opts ? &opts->b : nullptr, c->SB, g.img_b * cbb, pack_b);
    const ImgPanel* pa = reinterpret_cast<const ImgPanel*>(dbase + g.pa_off);
    if (pack_a && fuse)
      launch_pack_mix_images(form, c->stream, A, ia, pa,
                             reinterpret_cast<const int2*>(fuse->dbase + fuse->fr_off),
                             reinterpret_cast<const MixCover*>(fuse->dbase + fuse->fc_off),
                             reinterpret_cast<const MixTerm*>(fuse->dbase + fuse->mix.m_off),
                             int(g.pa.size()), g.img_a, SPLIT_IMG_ROWS);
    else if (pack_a)
      launch_pack_images(form, c->stream, A, ia, pa, int(g.pa.size()), g.img_a, SPLIT_IMG_ROWS);
    if (pack_b)
      launch_pack_images(form, c->stream, B, ib,
                         reinterpret_cast<const ImgPanel*>(dbase + g.pb_off), int(g.pb.size()),
                         g.img_b, g.bn);
    launch_gemm_split_images(form, g.bn, c->stream, ia, ib, C, tasks, int(g.tasks.size()), segs,
                             reinterpret_cast<const SegImg*>(dbase + g.si_off), g.tiles, c->nsm,
                             c->d_status + STATUS_MMA);
    return;
  }
  if (opts && opts->fuse) bad_plan("split gemm mixing");   // fused mixing needs the image form
  launch_gemm_split(form, c->stream, g.tA, g.tB, A, B, C, tasks, int(g.tasks.size()), segs,
                    g.tiles, c->nsm * 3, c->d_status + STATUS_MMA);
}

void run_mix(dmrg_ctx* c, const MixList& m, char* dbase, const double* in, int64_t nin,
             double* out, int64_t nout) {
  if (m.tiles == 0) return;
  check_mix_list(m, nin, nout);
  launch_mix(c->stream, in, out, reinterpret_cast<const MixTask*>(dbase + m.t_off),
             int(m.tasks.size()), reinterpret_cast<const MixTerm*>(dbase + m.m_off), m.tiles);
}

void run_copy(dmrg_ctx* c, const CopyList& l, char* dbase, const double* src, int64_t nsrc,
              double* dst, int64_t ndst) {
  if (l.tiles == 0) return;
  for (const CopyTask& t : l.tasks) {
    const int64_t es = t.trans ? (t.cols - 1) + int64_t(t.rows - 1) * t.lds
                               : (t.rows - 1) + int64_t(t.cols - 1) * t.lds;
    if (!in_range(t.src_off, es, nsrc)) bad_plan("copy src");
    if (t.ldd < t.rows || !in_range(t.dst_off, (t.rows - 1) + int64_t(t.cols - 1) * t.ldd, ndst))
      bad_plan("copy dst");
  }
  launch_copy(c->stream, src, dst, reinterpret_cast<const CopyTask*>(dbase + l.t_off),
              int(l.tasks.size()), l.tiles);
}

void check_eig(const std::vector<EigTask>& ts, int64_t nbase) {
  for (const EigTask& t : ts) {
    const int64_t nn = int64_t(t.n) * t.n;
    if (t.n <= 0 || !in_range(t.a_off, nn - 1, nbase) || !in_range(t.v_off, nn - 1, nbase) ||
        !in_range(t.w_off, t.n - 1, nbase))
      bad_plan("eigensolver task");
    if (t.n > 4096) fail(DMRG_ERR_SHAPE, "density-matrix block larger than 4096");
  }
}

}  // namespace dmrg
