// abi.cpp -- extern "C" entry points of libdmrgb200.so (declared in include/dmrg_b200.h).
// Exceptions (dmrg::Error) never cross this boundary: each entry point returns a status code
// and records the message in the context (dmrg_last_error).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <cmath>
#include <map>
#include <numeric>

#include "engine.hpp"

using namespace dmrg;

namespace {

thread_local std::string g_noctx_err;

template <class F>
int guarded(dmrg_ctx* c, F&& f) {
  try {
    f();
    if (c) {
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) fail(DMRG_ERR_CUDA, std::string("CUDA: ") + cudaGetErrorString(e));
      c->err.clear();
    }
    return DMRG_OK;
  } catch (const Error& e) {
    if (c) c->err = e.msg; else g_noctx_err = e.msg;
    return e.code;
  } catch (const std::exception& e) {
    if (c) c->err = e.what(); else g_noctx_err = e.what();
    return DMRG_ERR_ARG;
  }
}

QN qn_from(const int* p, int nsym) {
  QN q;
  for (int k = 0; k < nsym; ++k) q.v[k] = p[k];
  return q;
}

void set_device(dmrg_ctx* c) { cuda_check(cudaSetDevice(c->device), "cudaSetDevice"); }

// Groups bond states by charge: sectors ascending, perm[k] = original states of sector k.
Bond group_bond(const std::vector<QN>& lab, std::vector<std::vector<int>>& perm) {
  std::map<QN, std::vector<int>> m;
  for (int i = 0; i < int(lab.size()); ++i) m[lab[i]].push_back(i);
  Bond b;
  perm.clear();
  for (auto& kv : m) {
    b.q.push_back(kv.first);
    b.dim.push_back(int(kv.second.size()));
    perm.push_back(kv.second);
  }
  return b;
}

void upload_site(dmrg_ctx* c, DBuf& buf, const std::vector<double>& h) {
  dalloc(c, buf, std::max<int64_t>(int64_t(h.size()), 1));
  if (!h.empty())
    cuda_check(cudaMemcpyAsync(buf.p, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice,
                               c->stream), "MPS upload");
  cuda_check(cudaStreamSynchronize(c->stream), "MPS upload sync");
}


dmrg_state* new_state(dmrg_ctx* c, const dmrg_mpo* mpo, int oc) {
  const int L = mpo->L;
  if (oc < 0 || oc >= L) fail(DMRG_ERR_ARG, "orthogonality centre out of range");
  auto* st = new dmrg_state();
  st->ctx = c;
  st->mpo = mpo;
  st->L = L;
  st->nsym = mpo->nsym;
  st->oc = oc;
  st->dir = (oc == L - 1 && L > 1) ? -1 : 1;
  st->bond.resize(L + 1);
  st->lay.resize(L);
  st->A.resize(L);
  st->Llay.resize(L);
  st->Rlay.resize(L);
  st->Lenv.resize(L);
  st->Renv.resize(L);
  st->Lvalid.assign(L, 0);
  st->Rvalid.assign(L, 0);
  return st;
}

void free_envs(dmrg_state* st) {
  for (auto& b : st->Lenv) dfree(st->ctx, b);
  for (auto& b : st->Renv) dfree(st->ctx, b);
  st->Lvalid.assign(st->L, 0);
  st->Rvalid.assign(st->L, 0);
  st->env_built = false;
}

}  // namespace

extern "C" {

int dmrg_abi_version(void) { return DMRG_ABI_VERSION; }

long long dmrg_kernel_launches(void) { return launch_count(); }

void dmrg_params_default(dmrg_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->maxm = 0;
  p->minm = 2;
  p->cutoff = 0.0;
  p->krylov = 2;
  p->precision = DMRG_PREC_FP64;
  p->svnbond = 0;
  p->degen_rtol = 0.0;
  p->betatest = 1e-10;
  p->fp64_final = 1;
  p->cvgE = 1;
  p->goal = 0.0;
  p->tune = 1;
  p->graph = 0;
}

const char* dmrg_last_error(const dmrg_ctx* ctx) {
  return ctx ? ctx->err.c_str() : g_noctx_err.c_str();
}

int dmrg_ctx_create(int device, size_t hbm_budget_bytes, dmrg_ctx** out) {
  return guarded(nullptr, [&] {
    if (!out) fail(DMRG_ERR_ARG, "null output handle");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      fail(DMRG_ERR_NOCUDA, "no CUDA device available");
    }
    if (device < 0 || device >= ndev) fail(DMRG_ERR_ARG, "device index out of range");
    auto* c = new dmrg_ctx();
    c->device = device;
    c->budget = hbm_budget_bytes;
    try {
      set_device(c);
      cuda_check(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream");
      cudaMemPool_t pool;
      cuda_check(cudaDeviceGetDefaultMemPool(&pool, device), "mempool");
      uint64_t thr = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
      c->nsm = device_sm_count();
      cuda_check(cudaMalloc(&c->d_scal, 256 * sizeof(double)), "scalars");
      // 16 rows of 296 reduction partials, then the last-block reduction counter (zeroed)
      cuda_check(cudaMalloc(&c->d_partial, (16 * 296 + 1) * sizeof(double)), "partials");
      cuda_check(cudaMemsetAsync(c->d_partial, 0, (16 * 296 + 1) * sizeof(double), c->stream),
                 "partials clear");
      cuda_check(cudaMalloc(&c->d_status, 16 * sizeof(int)), "status");
      cuda_check(cudaMemsetAsync(c->d_status, 0, 16 * sizeof(int), c->stream), "status clear");
      cuda_check(cudaMallocHost(&c->h_scal, 256 * sizeof(double)), "pinned scalars");
      c->dv_scal = device_view(c->h_scal);
      cuda_check(cudaMalloc(&c->d_flags, c->max_groups * sizeof(int)), "flags");
      cuda_check(cudaMallocHost(&c->h_flags, c->max_groups * sizeof(int)), "pinned flags");
      cuda_check(cudaMalloc(&c->d_floors, c->max_groups * sizeof(double)), "floors");
    } catch (...) {
      delete c;
      throw;
    }
    *out = c;
  });
}

int dmrg_ctx_destroy(dmrg_ctx* c) {
  if (!c) return DMRG_ERR_ARG;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  for (DBuf* b : {&c->X, &c->Y, &c->K, &c->H, &c->M, &c->R, &c->W, &c->T1, &c->T2, &c->SA,
                  &c->SB})
    dfree(c, *b);
  for (auto& s : c->slot) {
    if (s.h) cudaFreeHost(s.h);
    if (s.d) cudaFreeAsync(s.d, c->stream);
    if (s.ev) cudaEventDestroy(s.ev);
  }
  cudaStreamSynchronize(c->stream);
  for (cudaEvent_t e : c->tev) cudaEventDestroy(e);
  cudaFree(c->d_scal);
  cudaFree(c->d_partial);
  cudaFree(c->d_status);
  cudaFreeHost(c->h_scal);
  if (c->h_lam) cudaFreeHost(c->h_lam);
  cudaFree(c->d_flags);
  cudaFreeHost(c->h_flags);
  cudaFree(c->d_floors);
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  if (c->env_stream) {
    cudaStreamSynchronize(c->env_stream);
    cudaStreamDestroy(c->env_stream);
    cudaEventDestroy(c->env_fork);
    cudaEventDestroy(c->env_join);
  }
  cudaStreamDestroy(c->stream);
  delete c;
  return DMRG_OK;
}

int dmrg_ctx_tuner(dmrg_ctx* c, int* signatures, int* decided, int* small) {
  if (!c) return DMRG_ERR_ARG;
  return guarded(c, [&] {
    set_device(c);
    tuner_collect(c);
    int n = 0, d = 0, s = 0;
    for (const auto& kv : c->tuner.table) {
      ++n;
      if (kv.second.choice >= 0) ++d;
      if (kv.second.choice == 1) ++s;
    }
    if (signatures) *signatures = n;
    if (decided) *decided = d;
    if (small) *small = s;
  });
}

int dmrg_ctx_memory(const dmrg_ctx* c, size_t* in_use, size_t* peak) {
  if (!c) return DMRG_ERR_ARG;
  if (in_use) *in_use = c->in_use;
  if (peak) *peak = c->peak;
  return DMRG_OK;
}

int dmrg_mpo_upload(dmrg_ctx* c, int L, int nsym, const int* d, const int* wl, const int* wr,
                    const double* const* W, const int* const* phys_qn,
                    const int* const* bond_qn, dmrg_mpo** out) {
  if (!c) return DMRG_ERR_ARG;
  return guarded(c, [&] {
    if (!out || !d || !wl || !wr || !W) fail(DMRG_ERR_ARG, "null argument");
    if (L < 1) fail(DMRG_ERR_ARG, "L must be positive");
    if (nsym < 0 || nsym > 2) fail(DMRG_ERR_ARG, "nsym must be 0, 1 or 2");
    if (nsym > 0 && !phys_qn) fail(DMRG_ERR_ARG, "physical labels required when nsym > 0");
    auto* m = new dmrg_mpo();
    m->ctx = c;
    m->L = L;
    m->nsym = nsym;
    m->site.resize(L);
    try {
      for (int i = 0; i < L; ++i) {
        MPOSite& s = m->site[i];
        s.wl = wl[i];
        s.d = d[i];
        s.wr = wr[i];
        if (s.wl <= 0 || s.d <= 0 || s.wr <= 0 || !W[i]) fail(DMRG_ERR_SHAPE, "bad MPO dims");
        if (i + 1 < L && wr[i] != wl[i + 1]) fail(DMRG_ERR_SHAPE, "MPO bond dims do not match");
        if (i + 1 < L && d[i] <= 0) fail(DMRG_ERR_SHAPE, "bad physical dim");
        const size_t n = size_t(s.wl) * s.d * s.d * s.wr;
        s.dense.assign(W[i], W[i] + n);
        s.p.assign(s.d, QN());
        if (nsym > 0)
          for (int a = 0; a < s.d; ++a) s.p[a] = qn_from(phys_qn[i] + a * nsym, nsym);
        for (int w2 = 0; w2 < s.wr; ++w2)
          for (int t = 0; t < s.d; ++t)
            for (int ss = 0; ss < s.d; ++ss)
              for (int w = 0; w < s.wl; ++w) {
                const double v = s.dense[w + size_t(s.wl) * (ss + size_t(s.d) * (t + size_t(s.d) * w2))];
                if (v != 0.0) s.nz.push_back({w, ss, t, w2, v});
              }
      }
      // bond labels: given, or derived with the makeqMPO largest-weight rule
      std::vector<std::vector<QN>> r(L + 1);
      r[0].assign(wl[0], QN());
      if (bond_qn && nsym > 0) {
        for (int b = 0; b <= L; ++b) {
          const int nb = b < L ? wl[b] : wr[L - 1];
          r[b].resize(nb);
          for (int k = 0; k < nb; ++k) r[b][k] = qn_from(bond_qn[b] + k * nsym, nsym);
        }
      } else {
        for (int i = 0; i < L; ++i) {
          const MPOSite& s = m->site[i];
          r[i + 1].assign(s.wr, QN());
          if (nsym == 0) continue;
          for (int w2 = 0; w2 < s.wr; ++w2) {
            std::vector<std::pair<QN, double>> tot;   // first-appearance order
            for (int t = 0; t < s.d; ++t)
              for (int ss = 0; ss < s.d; ++ss)
                for (int w = 0; w < s.wl; ++w) {
                  const QN q = r[i][w] + s.p[ss] - s.p[t];
                  const double v = s.dense[w + size_t(s.wl) * (ss + size_t(s.d) * (t + size_t(s.d) * w2))];
                  const double wgt = v * v * v * v;
                  auto it = std::find_if(tot.begin(), tot.end(), [&](auto& e) { return e.first == q; });
                  if (it == tot.end()) tot.push_back({q, wgt}); else it->second += wgt;
                }
            int best = 0;
            for (int k = 1; k < int(tot.size()); ++k)
              if (tot[k].second > tot[best].second) best = k;
            r[i + 1][w2] = (tot.empty() || tot[best].second == 0.0) ? QN() : tot[best].first;
          }
        }
      }
      for (int i = 0; i < L; ++i) {
        MPOSite& s = m->site[i];
        s.rl = r[i];
        s.rr = r[i + 1];
        for (const auto& e : s.nz)
          if (!(s.rr[e.w2] == s.rl[e.w] + s.p[e.s] - s.p[e.t]))
            fail(DMRG_ERR_QN, "MPO element breaks charge conservation at site " + std::to_string(i));
      }
      m->two.resize(std::max(L - 1, 0));
      for (int i = 0; i + 1 < L; ++i) m->two[i] = make_two_site_op(m->site[i], m->site[i + 1]);
      m->one.resize(L);
      for (int i = 0; i < L; ++i) m->one[i] = make_one_site_op(m->site[i]);
    } catch (...) {
      delete m;
      throw;
    }
    *out = m;
  });
}

int dmrg_mpo_destroy(dmrg_mpo* m) {
  if (!m) return DMRG_ERR_ARG;
  delete m;
  return DMRG_OK;
}

int dmrg_mps_upload(dmrg_ctx* c, const dmrg_mpo* mpo, const int* ml, const int* mr,
                    const double* const* A, const int* const* bond_qn, int oc, dmrg_state** out) {
  if (!c) return DMRG_ERR_ARG;
  return guarded(c, [&] {
    if (!mpo || !ml || !mr || !A || !out) fail(DMRG_ERR_ARG, "null argument");
    set_device(c);
    const int L = mpo->L, nsym = mpo->nsym;
    for (int i = 0; i < L; ++i) {
      if (ml[i] <= 0 || mr[i] <= 0 || !A[i]) fail(DMRG_ERR_SHAPE, "bad MPS dims");
      if (i + 1 < L && mr[i] != ml[i + 1]) fail(DMRG_ERR_SHAPE, "MPS bond dims do not match");
    }
    // bond labels
    std::vector<std::vector<QN>> q(L + 1);
    q[0].assign(ml[0], QN());
    if (bond_qn && nsym > 0) {
      for (int b = 0; b <= L; ++b) {
        const int nb = b < L ? ml[b] : mr[L - 1];
        q[b].resize(nb);
        for (int k = 0; k < nb; ++k) q[b][k] = qn_from(bond_qn[b] + k * nsym, nsym);
      }
    } else {
      for (int i = 0; i < L; ++i) {
        const int a_n = ml[i], d = mpo->site[i].d, b_n = mr[i];
        q[i + 1].assign(b_n, QN());
        if (nsym == 0) continue;
        for (int b = 0; b < b_n; ++b) {       // assignflux!: label of the largest element
          double best = 0.0;
          for (int a = 0; a < a_n; ++a)
            for (int s = 0; s < d; ++s) {
              const double v = std::fabs(A[i][a + size_t(a_n) * (s + size_t(d) * b)]);
              if (v > best) { best = v; q[i + 1][b] = q[i][a] + mpo->site[i].p[s]; }
            }
        }
      }
    }
    dmrg_state* st = new_state(c, mpo, oc);
    try {
      std::vector<std::vector<std::vector<int>>> perm(L + 1);
      for (int b = 0; b <= L; ++b) st->bond[b] = group_bond(q[b], perm[b]);
      for (int i = 0; i < L; ++i) {
        const Bond& Bl = st->bond[i];
        const Bond& Br = st->bond[i + 1];
        const MPOSite& ms = mpo->site[i];
        if (ms.d <= 0) fail(DMRG_ERR_SHAPE, "bad physical dim");
        st->lay[i] = make_site_layout(Bl, ms.p, Br);
        const SiteLayout& lay = st->lay[i];
        std::vector<double> h(lay.size, 0.0);
        const int a_n = ml[i], d = ms.d;
        double amax = 0.0;
        for (size_t e = 0; e < size_t(a_n) * d * mr[i]; ++e) amax = std::max(amax, std::fabs(A[i][e]));
        // forbidden elements must vanish
        std::vector<int> seca(a_n), secb(mr[i]);
        for (int k = 0; k < Bl.nsec(); ++k) for (int x : perm[i][k]) seca[x] = k;
        for (int k = 0; k < Br.nsec(); ++k) for (int x : perm[i + 1][k]) secb[x] = k;
        for (int b = 0; b < mr[i]; ++b)
          for (int s = 0; s < d; ++s)
            for (int a = 0; a < a_n; ++a) {
              const double v = A[i][a + size_t(a_n) * (s + size_t(d) * b)];
              if (v == 0.0) continue;
              if (lay.kb[seca[a] * d + s] != secb[b] && std::fabs(v) > 1e-12 * amax)
                fail(DMRG_ERR_QN, "MPS element in a charge-forbidden block at site " + std::to_string(i));
            }
        for (int ka = 0; ka < Bl.nsec(); ++ka)
          for (int s = 0; s < d; ++s) {
            const int kb = lay.kb[ka * d + s];
            if (kb < 0) continue;
            const int64_t off = lay.off[ka * d + s];
            const int ra = Bl.dim[ka];
            for (int cb = 0; cb < Br.dim[kb]; ++cb)
              for (int ca = 0; ca < ra; ++ca) {
                const int a = perm[i][ka][ca], b = perm[i + 1][kb][cb];
                h[off + ca + int64_t(cb) * ra] = A[i][a + size_t(a_n) * (s + size_t(d) * b)];
              }
          }
        upload_site(c, st->A[i], h);
      }
    } catch (...) {
      for (auto& b : st->A) dfree(c, b);
      delete st;
      throw;
    }
    *out = st;
  });
}

int dmrg_mps_upload_blocks(dmrg_ctx* c, const dmrg_mpo* mpo, const int* nsec,
                           const int* const* sec_qn, const int* const* sec_dim,
                           const double* const* data, int oc, dmrg_state** out) {
  if (!c) return DMRG_ERR_ARG;
  return guarded(c, [&] {
    if (!mpo || !nsec || !sec_dim || !data || !out) fail(DMRG_ERR_ARG, "null argument");
    if (mpo->nsym > 0 && !sec_qn) fail(DMRG_ERR_ARG, "sector charges required when nsym > 0");
    set_device(c);
    const int L = mpo->L, nsym = mpo->nsym;
    dmrg_state* st = new_state(c, mpo, oc);
    try {
      for (int b = 0; b <= L; ++b) {
        Bond& B = st->bond[b];
        for (int k = 0; k < nsec[b]; ++k) {
          B.q.push_back(nsym > 0 ? qn_from(sec_qn[b] + k * nsym, nsym) : QN());
          B.dim.push_back(sec_dim[b][k]);
          if (sec_dim[b][k] <= 0) fail(DMRG_ERR_SHAPE, "sector dims must be positive");
          if (k > 0 && !(B.q[k - 1] < B.q[k]))
            fail(DMRG_ERR_ARG, "sector charges must be strictly increasing");
        }
      }
      // every site straight from the caller's arrays (a copy from pageable memory returns once
      // the driver has staged it), one synchronisation at the end
      for (int i = 0; i < L; ++i) {
        st->lay[i] = make_site_layout(st->bond[i], mpo->site[i].p, st->bond[i + 1]);
        const size_t n = size_t(st->lay[i].size);
        dalloc(c, st->A[i], std::max<int64_t>(int64_t(n), 1));
        if (n)
          cuda_check(cudaMemcpyAsync(st->A[i].p, data[i], n * sizeof(double),
                                     cudaMemcpyHostToDevice, c->stream), "MPS upload");
      }
      cuda_check(cudaStreamSynchronize(c->stream), "MPS upload sync");
    } catch (...) {
      for (auto& b : st->A) dfree(c, b);
      delete st;
      throw;
    }
    *out = st;
  });
}

// ---- checkpoints: one little-endian binary file per state
//   "DMRGCKP1", int32 version, L, nsym, oc, dir
//   per bond b = 0..L: int32 nsec, then per sector int32 charge[nsym], int32 dim
//   per site: int32 d, int64 n, n doubles (the site's blocks in canonical order)
//   uint64 FNV-1a of every preceding byte
namespace {

constexpr char CKP_MAGIC[8] = {'D', 'M', 'R', 'G', 'C', 'K', 'P', '1'};
constexpr int32_t CKP_VERSION = 1;

struct CkpWriter {
  std::FILE* f = nullptr;
  uint64_t h = 1469598103934665603ull;
  void put(const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t k = 0; k < n; ++k) h = (h ^ b[k]) * 1099511628211ull;
    if (std::fwrite(p, 1, n, f) != n) fail(DMRG_ERR_ARG, "checkpoint: write failed");
  }
  void i32(int32_t v) { put(&v, 4); }
};

struct CkpReader {
  const std::vector<unsigned char>& buf;
  size_t pos = 0;
  explicit CkpReader(const std::vector<unsigned char>& b) : buf(b) {}
  const unsigned char* take(size_t n) {
    if (n > buf.size() - pos) fail(DMRG_ERR_ARG, "checkpoint: file is truncated");
    const unsigned char* p = buf.data() + pos;
    pos += n;
    return p;
  }
  int32_t i32() { int32_t v; std::memcpy(&v, take(4), 4); return v; }
  int64_t i64() { int64_t v; std::memcpy(&v, take(8), 8); return v; }
};

}  // namespace

int dmrg_state_save(dmrg_state* st, const char* path) {
  if (!st || !path) return DMRG_ERR_ARG;
  dmrg_ctx* c = st->ctx;
  return guarded(c, [&] {
    set_device(c);
    CkpWriter w;
    w.f = std::fopen(path, "wb");
    if (!w.f) fail(DMRG_ERR_ARG, std::string("checkpoint: cannot open ") + path);
    try {
      w.put(CKP_MAGIC, 8);
      w.i32(CKP_VERSION);
      w.i32(st->L);
      w.i32(st->nsym);
      w.i32(st->oc);
      w.i32(st->dir);
      for (int b = 0; b <= st->L; ++b) {
        const Bond& B = st->bond[b];
        w.i32(B.nsec());
        for (int k = 0; k < B.nsec(); ++k) {
          for (int a = 0; a < st->nsym; ++a) w.i32(B.q[k].v[a]);
          w.i32(B.dim[k]);
        }
      }
      std::vector<double> h;
      for (int i = 0; i < st->L; ++i) {
        const int64_t n = st->lay[i].size;
        h.resize(size_t(n));
        if (n > 0) {
          cuda_check(cudaMemcpyAsync(h.data(), st->A[i].p, sizeof(double) * size_t(n),
                                     cudaMemcpyDeviceToHost, c->stream), "checkpoint download");
          cuda_check(cudaStreamSynchronize(c->stream), "checkpoint download sync");
        }
        w.i32(st->mpo->site[i].d);
        w.put(&n, 8);
        w.put(h.data(), sizeof(double) * size_t(n));
      }
      const uint64_t sum = w.h;
      if (std::fwrite(&sum, 1, 8, w.f) != 8) fail(DMRG_ERR_ARG, "checkpoint: write failed");
      if (std::fclose(w.f) != 0) {
        w.f = nullptr;
        fail(DMRG_ERR_ARG, "checkpoint: close failed");
      }
      w.f = nullptr;
    } catch (...) {
      if (w.f) std::fclose(w.f);
      throw;
    }
  });
}

int dmrg_state_load(dmrg_ctx* c, const dmrg_mpo* mpo, const char* path, dmrg_state** out) {
  if (!c) return DMRG_ERR_ARG;
  std::vector<int> nsec;
  std::vector<std::vector<int>> qn, dims;
  std::vector<const double*> data;
  std::vector<std::vector<double>> sites;   // aligned copies of the site data
  std::vector<unsigned char> buf;
  int oc = 0, dir = 1;
  const int rc = guarded(c, [&] {
    if (!mpo || !path || !out) fail(DMRG_ERR_ARG, "null argument");
    std::FILE* f = std::fopen(path, "rb");
    if (!f) fail(DMRG_ERR_ARG, std::string("checkpoint: cannot open ") + path);
    std::fseek(f, 0, SEEK_END);
    const long len = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (len < 8 + 8) {
      std::fclose(f);
      fail(DMRG_ERR_ARG, "checkpoint: file is truncated");
    }
    buf.resize(size_t(len));
    const size_t got = std::fread(buf.data(), 1, buf.size(), f);
    std::fclose(f);
    if (got != buf.size()) fail(DMRG_ERR_ARG, "checkpoint: read failed");
    uint64_t h = 1469598103934665603ull, sum;
    for (size_t k = 0; k < buf.size() - 8; ++k) h = (h ^ buf[k]) * 1099511628211ull;
    std::memcpy(&sum, buf.data() + buf.size() - 8, 8);
    if (h != sum) fail(DMRG_ERR_ARG, "checkpoint: checksum mismatch (corrupt file)");
    buf.resize(buf.size() - 8);
    CkpReader r(buf);
    if (std::memcmp(r.take(8), CKP_MAGIC, 8) != 0) fail(DMRG_ERR_ARG, "checkpoint: not a checkpoint");
    if (r.i32() != CKP_VERSION) fail(DMRG_ERR_ARG, "checkpoint: unsupported version");
    const int L = r.i32(), nsym = r.i32();
    oc = r.i32();
    dir = r.i32();
    if (L != mpo->L) fail(DMRG_ERR_SHAPE, "checkpoint: chain length differs from the MPO's");
    if (nsym != mpo->nsym) fail(DMRG_ERR_QN, "checkpoint: charges differ from the MPO's");
    if (oc < 0 || oc >= L || (dir != 1 && dir != -1)) fail(DMRG_ERR_ARG, "checkpoint: bad centre");
    nsec.resize(L + 1);
    qn.resize(L + 1);
    dims.resize(L + 1);
    std::vector<Bond> bonds(L + 1);
    for (int b = 0; b <= L; ++b) {
      nsec[b] = r.i32();
      if (nsec[b] < 0 || nsec[b] > (1 << 24)) fail(DMRG_ERR_ARG, "checkpoint: bad sector count");
      for (int k = 0; k < nsec[b]; ++k) {
        int q[2] = {0, 0};
        for (int a = 0; a < nsym; ++a) {
          q[a] = r.i32();
          qn[b].push_back(q[a]);
        }
        dims[b].push_back(r.i32());
        bonds[b].q.push_back(QN(q[0], q[1]));
        bonds[b].dim.push_back(dims[b].back());
        if (dims[b].back() <= 0) fail(DMRG_ERR_SHAPE, "checkpoint: sector dims must be positive");
      }
    }
    data.resize(L);
    sites.resize(L);
    for (int i = 0; i < L; ++i) {
      const int d = r.i32();
      const int64_t n = r.i64();
      if (d != mpo->site[i].d) fail(DMRG_ERR_SHAPE, "checkpoint: physical dimension differs");
      for (int k = 1; k < bonds[i].nsec(); ++k)
        if (!(bonds[i].q[k - 1] < bonds[i].q[k]))
          fail(DMRG_ERR_ARG, "checkpoint: sector charges must be strictly increasing");
      const SiteLayout lay = make_site_layout(bonds[i], mpo->site[i].p, bonds[i + 1]);
      if (n != lay.size) fail(DMRG_ERR_SHAPE, "checkpoint: site data does not match its sectors");
      sites[i].resize(size_t(n));
      if (n > 0) std::memcpy(sites[i].data(), r.take(sizeof(double) * size_t(n)),
                             sizeof(double) * size_t(n));
      data[i] = sites[i].data();
    }
    if (r.pos != buf.size()) fail(DMRG_ERR_ARG, "checkpoint: trailing bytes");
  });
  if (rc != DMRG_OK) return rc;
  buf.clear();
  buf.shrink_to_fit();
  std::vector<const int*> qp(nsec.size()), dp(nsec.size());
  for (size_t b = 0; b < nsec.size(); ++b) {
    qp[b] = qn[b].data();
    dp[b] = dims[b].data();
  }
  const int rc2 = dmrg_mps_upload_blocks(c, mpo, nsec.data(), mpo->nsym ? qp.data() : nullptr,
                                         dp.data(), data.data(), oc, out);
  if (rc2 == DMRG_OK) (*out)->dir = dir;
  return rc2;
}

int dmrg_state_destroy(dmrg_state* st) {
  if (!st) return DMRG_ERR_ARG;
  dmrg_ctx* c = st->ctx;
  cudaSetDevice(c->device);
  for (auto& b : st->A) dfree(c, b);
  free_envs(st);
  cudaStreamSynchronize(c->stream);
  delete st;
  return DMRG_OK;
}

int dmrg_state_oc(const dmrg_state* st, int* oc) {
  if (!st || !oc) return DMRG_ERR_ARG;
  *oc = st->oc;
  return DMRG_OK;
}

int dmrg_bond_info(const dmrg_state* st, int bond, int* nsec, int* qn, int* dims) {
  if (!st || !nsec) return DMRG_ERR_ARG;
  if (bond < 0 || bond > st->L) return DMRG_ERR_ARG;
  const Bond& B = st->bond[bond];
  *nsec = B.nsec();
  for (int k = 0; k < B.nsec(); ++k) {
    if (qn) for (int a = 0; a < st->nsym; ++a) qn[k * st->nsym + a] = B.q[k].v[a];
    if (dims) dims[k] = B.dim[k];
  }
  return DMRG_OK;
}

int dmrg_site_size(const dmrg_state* st, int site, int64_t* n) {
  if (!st || !n || site < 0 || site >= st->L) return DMRG_ERR_ARG;
  *n = st->lay[site].size;
  return DMRG_OK;
}

int dmrg_mps_download_blocks(dmrg_state* st, int site, double* out) {
  if (!st) return DMRG_ERR_ARG;
  dmrg_ctx* c = st->ctx;
  return guarded(c, [&] {
    if (site < 0 || site >= st->L || !out) fail(DMRG_ERR_ARG, "bad site or null output");
    set_device(c);
    cuda_check(cudaMemcpyAsync(out, st->A[site].p, sizeof(double) * st->lay[site].size,
                               cudaMemcpyDeviceToHost, c->stream), "MPS download");
    cuda_check(cudaStreamSynchronize(c->stream), "MPS download sync");
  });
}

int dmrg_mps_download_all_blocks(dmrg_state* st, double* out, int64_t* sizes) {
  if (!st) return DMRG_ERR_ARG;
  dmrg_ctx* c = st->ctx;
  return guarded(c, [&] {
    size_t total = 0;
    for (int i = 0; i < st->L; ++i) {
      if (sizes) sizes[i] = st->lay[i].size;
      total += size_t(st->lay[i].size);
    }
    if (!out) return;
    set_device(c);
    size_t at = 0;
    for (int i = 0; i < st->L; ++i) {
      const size_t n = size_t(st->lay[i].size);
      if (n)
        cuda_check(cudaMemcpyAsync(out + at, st->A[i].p, n * sizeof(double), cudaMemcpyDeviceToHost,
                                   c->stream), "MPS download");
      at += n;
    }
    cuda_check(cudaStreamSynchronize(c->stream), "MPS download sync");
  });
}

int dmrg_bonds_info(const dmrg_state* st, int* nsec, int* qn, int* dims) {
  if (!st || !nsec) return DMRG_ERR_ARG;
  size_t k = 0;
  for (int b = 0; b <= st->L; ++b) {
    const Bond& B = st->bond[b];
    nsec[b] = B.nsec();
    for (int j = 0; j < B.nsec(); ++j, ++k) {
      if (dims) dims[k] = B.dim[j];
      if (qn)
        for (int a = 0; a < st->nsym; ++a) qn[k * st->nsym + a] = B.q[j].v[a];
    }
  }
  return DMRG_OK;
}

int dmrg_mps_download(dmrg_state* st, int site, double* out, int* mlo, int* mro) {
  if (!st) return DMRG_ERR_ARG;
  dmrg_ctx* c = st->ctx;
  return guarded(c, [&] {
    if (site < 0 || site >= st->L) fail(DMRG_ERR_ARG, "bad site");
    const Bond& Bl = st->bond[site];
    const Bond& Br = st->bond[site + 1];
    const int ml = int(Bl.total()), mr = int(Br.total()), d = st->mpo->site[site].d;
    if (mlo) *mlo = ml;
    if (mro) *mro = mr;
    if (!out) return;
    set_device(c);
    const SiteLayout& lay = st->lay[site];
    std::vector<double> h(lay.size);
    cuda_check(cudaMemcpyAsync(h.data(), st->A[site].p, sizeof(double) * lay.size,
                               cudaMemcpyDeviceToHost, c->stream), "MPS download");
    cuda_check(cudaStreamSynchronize(c->stream), "MPS download sync");
    std::fill(out, out + size_t(ml) * d * mr, 0.0);
    const auto ol = Bl.offsets(), orr = Br.offsets();
    for (int ka = 0; ka < Bl.nsec(); ++ka)
      for (int s = 0; s < d; ++s) {
        const int kb = lay.kb[ka * d + s];
        if (kb < 0) continue;
        const int64_t off = lay.off[ka * d + s];
        for (int cb = 0; cb < Br.dim[kb]; ++cb)
          for (int ca = 0; ca < Bl.dim[ka]; ++ca)
            out[(ol[ka] + ca) + size_t(ml) * (s + size_t(d) * (orr[kb] + cb))] =
                h[off + ca + int64_t(cb) * Bl.dim[ka]];
      }
  });
}

int dmrg_env_build(dmrg_state* st, const dmrg_mpo* mpo) {
  if (!st) return DMRG_ERR_ARG;
  dmrg_ctx* c = st->ctx;
  return guarded(c, [&] {
    if (mpo != st->mpo) fail(DMRG_ERR_ARG, "state was uploaded with a different MPO");
    set_device(c);
    free_envs(st);
    env_boundaries(st);
    for (int i = 0; i < st->oc; ++i) lupdate(st, i, nullptr);
    for (int i = st->L - 1; i > st->oc; --i) rupdate(st, i, nullptr);
    cuda_check(cudaStreamSynchronize(c->stream), "env build sync");
    st->env_built = true;
    st->have_last = false;
  });
}

int dmrg_lupdate(dmrg_state* st, const dmrg_mpo* mpo, int site) {
  if (!st) return DMRG_ERR_ARG;
  dmrg_ctx* c = st->ctx;
  return guarded(c, [&] {
    if (mpo != st->mpo) fail(DMRG_ERR_ARG, "state was uploaded with a different MPO");
    set_device(c);
    lupdate(st, site, nullptr);
    cuda_check(cudaStreamSynchronize(c->stream), "lupdate sync");
  });
}

int dmrg_rupdate(dmrg_state* st, const dmrg_mpo* mpo, int site) {
  if (!st) return DMRG_ERR_ARG;
  dmrg_ctx* c = st->ctx;
  return guarded(c, [&] {
    if (mpo != st->mpo) fail(DMRG_ERR_ARG, "state was uploaded with a different MPO");
    set_device(c);
    rupdate(st, site, nullptr);
    cuda_check(cudaStreamSynchronize(c->stream), "rupdate sync");
  });
}

int dmrg_env_step(dmrg_ctx* c, int left, int ml, int d, int mr, int wl, int wr,
                  const double* env_in, const double* dual, const double* psi, const double* W,
                  double* env_out) {
  if (!c) return DMRG_ERR_ARG;
  return guarded(c, [&] {
    if (!env_in || !psi || !W || !env_out) fail(DMRG_ERR_ARG, "env step: null array");
    set_device(c);
    env_step_dense(c, left != 0, ml, d, mr, wl, wr, env_in, dual ? dual : psi, psi, W, env_out);
  });
}

int dmrg_expect(dmrg_state* st, const dmrg_mpo* H, double* value) {
  if (!st || !H || !value) return DMRG_ERR_ARG;
  dmrg_ctx* c = st->ctx;
  return guarded(c, [&] {
    if (H->ctx != c) fail(DMRG_ERR_ARG, "MPO belongs to a different context");
    set_device(c);
    *value = measure_expect(st, H, nullptr);
  });
}

int dmrg_correlationmatrix(dmrg_state* st, int d, const double* Cc, const double* Ca,
                           const double* trail, double* rho) {
  if (!st || !Cc || !Ca || !rho || d <= 0) return DMRG_ERR_ARG;
  dmrg_ctx* c = st->ctx;
  return guarded(c, [&] {
    set_device(c);
    measure_correlation(st, d, Cc, Ca, trail, rho, nullptr);
  });
}

int dmrg_correlation(dmrg_state* st, int d, int nops, const int* oplen, const double* ops,
                     const int* nsites, const int* sites, const double* trails, double* omega) {
  if (!st || d <= 0 || nops <= 0 || !oplen || !ops || !nsites || !sites || !omega)
    return DMRG_ERR_ARG;
  dmrg_ctx* c = st->ctx;
  return guarded(c, [&] {
    set_device(c);
    measure_correlation_n(st, d, nops, oplen, ops, nsites, sites, trails, omega, nullptr);
  });
}

int dmrg_env_get(dmrg_state* st, int site, int left, double* out, int* dims) {
  if (!st) return DMRG_ERR_ARG;
  dmrg_ctx* c = st->ctx;
  return guarded(c, [&] {
    if (site < 0 || site >= st->L) fail(DMRG_ERR_ARG, "bad site");
    const bool isL = left != 0;
    if (!(isL ? st->Lvalid[site] : st->Rvalid[site])) fail(DMRG_ERR_STATE, "environment not built");
    const Bond& B = isL ? st->bond[site] : st->bond[site + 1];
    const EnvLayout& E = isL ? st->Llay[site] : st->Rlay[site];
    const int m = int(B.total()), w = E.w;
    if (dims) { dims[0] = m; dims[1] = w; dims[2] = m; }
    if (!out) return;
    set_device(c);
    std::vector<double> h(std::max<int64_t>(E.size, 1));
    const DBuf& buf = isL ? st->Lenv[site] : st->Renv[site];
    cuda_check(cudaMemcpyAsync(h.data(), buf.p, sizeof(double) * E.size, cudaMemcpyDeviceToHost,
                               c->stream), "env download");
    cuda_check(cudaStreamSynchronize(c->stream), "env download sync");
    std::fill(out, out + size_t(m) * w * m, 0.0);
    const auto o = B.offsets();
    for (int k = 0; k < E.nsec; ++k)       // k = ket sector (L) / bra sector (R)
      for (int wi = 0; wi < w; ++wi) {
        const int ko = E.other[k * w + wi];
        if (ko < 0) continue;
        for (int col = 0; col < B.dim[k]; ++col)
          for (int r = 0; r < B.dim[ko]; ++r) {
            const double v = h[E.goff[k] + E.rowoff[k * w + wi] + r + int64_t(col) * E.rows[k]];
            // L[bra, w, ket]: rows are bra (ko), cols ket (k); R[ket, w, bra]: rows ket (ko), cols bra (k)
            out[(o[ko] + r) + size_t(m) * (wi + size_t(w) * (o[k] + col))] = v;
          }
      }
  });
}

int dmrg_twosite_dims(const dmrg_state* st, const dmrg_mpo* mpo, int iL, int* dims) {
  if (!st || !mpo || !dims || iL < 0 || iL + 1 >= st->L) return DMRG_ERR_ARG;
  dims[0] = int(st->bond[iL].total());
  dims[1] = mpo->site[iL].d;
  dims[2] = mpo->site[iL + 1].d;
  dims[3] = int(st->bond[iL + 2].total());
  return DMRG_OK;
}

// psi_out = Heff psi_in (dense-equivalent host arrays), the last of `reps` applications of one
// plan to the same vector
static int heff_apply_reps(dmrg_state* st, const dmrg_mpo* mpo, int iL, const double* psi_in,
                           double* psi_out, int precision, int reps) {
  if (!st) return DMRG_ERR_ARG;
  dmrg_ctx* c = st->ctx;
  return guarded(c, [&] {
    if (mpo != st->mpo) fail(DMRG_ERR_ARG, "state was uploaded with a different MPO");
    if (iL < 0 || iL + 1 >= st->L || !psi_in || !psi_out || reps < 1)
      fail(DMRG_ERR_ARG, "bad arguments");
    if (!st->Lvalid[iL] || !st->Rvalid[iL + 1]) fail(DMRG_ERR_STATE, "environments not built");
    set_device(c);
    HeffPlan hp;
    plan_heff(st, iL, hp);
    upload_heff(c, hp, 0, precision);
    const TwoLayout& tl = hp.tl;
    const Bond& Bl = st->bond[iL];
    const Bond& Br = st->bond[iL + 2];
    const int ml = int(Bl.total()), mr = int(Br.total()), d1 = tl.d1, d2 = tl.d2;
    const auto ol = Bl.offsets(), orr = Br.offsets();
    std::vector<double> h(std::max<int64_t>(tl.size, 1), 0.0);
    auto at = [&](int a, int s1, int s2, int b) {
      return size_t(a) + size_t(ml) * (s1 + size_t(d1) * (s2 + size_t(d2) * b));
    };
    for (int ka = 0; ka < tl.nl; ++ka)
      for (int s1 = 0; s1 < d1; ++s1)
        for (int s2 = 0; s2 < d2; ++s2) {
          const int id = tl.idx(ka, s1, s2), kd = tl.kd[id];
          if (kd < 0) continue;
          for (int cb = 0; cb < Br.dim[kd]; ++cb)
            for (int ca = 0; ca < Bl.dim[ka]; ++ca)
              h[tl.off[id] + ca + int64_t(cb) * Bl.dim[ka]] = psi_in[at(ol[ka] + ca, s1, s2, orr[kd] + cb)];
        }
    ensure(c, c->K, int64_t(h.size()));
    ensure(c, c->H, int64_t(h.size()));
    cuda_check(cudaMemcpyAsync(c->K.p, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice,
                               c->stream), "psi upload");
    for (int r = 0; r < reps; ++r) apply_heff(st, iL, hp, c->K.p, c->H.p, precision);
    cuda_check(cudaMemcpyAsync(h.data(), c->H.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost,
                               c->stream), "psi download");
    cuda_check(cudaStreamSynchronize(c->stream), "heff sync");
    check_mma_status(c);
    std::fill(psi_out, psi_out + size_t(ml) * d1 * d2 * mr, 0.0);
    for (int ka = 0; ka < tl.nl; ++ka)
      for (int s1 = 0; s1 < d1; ++s1)
        for (int s2 = 0; s2 < d2; ++s2) {
          const int id = tl.idx(ka, s1, s2), kd = tl.kd[id];
          if (kd < 0) continue;
          for (int cb = 0; cb < Br.dim[kd]; ++cb)
            for (int ca = 0; ca < Bl.dim[ka]; ++ca)
              psi_out[at(ol[ka] + ca, s1, s2, orr[kd] + cb)] = h[tl.off[id] + ca + int64_t(cb) * Bl.dim[ka]];
        }
  });
}


int dmrg_heff_apply(dmrg_state* st, const dmrg_mpo* mpo, int iL, const double* psi_in,
                    double* psi_out, int precision) {
  return heff_apply_reps(st, mpo, iL, psi_in, psi_out, precision, 1);
}

int dmrg_test_heff_apply_repeat(dmrg_state* st, const dmrg_mpo* mpo, int iL,
                                const double* psi_in, double* psi_out, int precision, int reps) {
  return heff_apply_reps(st, mpo, iL, psi_in, psi_out, precision, reps);
}

int dmrg_test_heff_time(dmrg_state* st, const dmrg_mpo* mpo, int iL, int precision, int reps,
                        double* seconds, double* flops) {
  if (!st) return DMRG_ERR_ARG;
  dmrg_ctx* c = st->ctx;
  return guarded(c, [&] {
    if (mpo != st->mpo) fail(DMRG_ERR_ARG, "state was uploaded with a different MPO");
    if (iL < 0 || iL + 1 >= st->L || reps < 1 || !seconds) fail(DMRG_ERR_ARG, "bad arguments");
    if (!st->Lvalid[iL] || !st->Rvalid[iL + 1]) fail(DMRG_ERR_STATE, "environments not built");
    set_device(c);
    HeffPlan hp;
    plan_heff(st, iL, hp);
    upload_heff(c, hp, 0, precision);
    const int64_t n = std::max<int64_t>(hp.tl.size, 1);
    ensure(c, c->K, n);
    ensure(c, c->H, n);
    // a fixed non-zero vector (zero operands would run the tensor pipe at lower power)
    std::vector<double> v(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i) v[size_t(i)] = std::sin(0.37 * double(i) + 0.1);
    cuda_check(cudaMemcpyAsync(c->K.p, v.data(), size_t(n) * sizeof(double),
                               cudaMemcpyHostToDevice, c->stream), "vector");
    cuda_check(cudaStreamSynchronize(c->stream), "vector");
    apply_heff(st, iL, hp, c->K.p, c->H.p, precision);   // warm-up (packs the environments)
    cudaEvent_t e0, e1;
    cuda_check(cudaEventCreate(&e0), "event");
    cuda_check(cudaEventCreate(&e1), "event");
    cudaEventRecord(e0, c->stream);
    for (int r = 0; r < reps; ++r) apply_heff(st, iL, hp, c->K.p, c->H.p, precision);
    cudaEventRecord(e1, c->stream);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    check_mma_status(c);
    *seconds = ms * 1e-3 / reps;
    if (flops) *flops = hp.flops;
  });
}

int dmrg_heff_apply_noalloc(dmrg_state* st, const dmrg_mpo* mpo, int iL, const double* psi_in,
                            double* psi_out, int precision) {
  if (!st) return DMRG_ERR_ARG;
  dmrg_ctx* c = st->ctx;
  return guarded(c, [&] {
    if (mpo != st->mpo) fail(DMRG_ERR_ARG, "state was uploaded with a different MPO");
    if (iL < 0 || iL + 1 >= st->L || !psi_in || !psi_out) fail(DMRG_ERR_ARG, "bad arguments");
    if (precision != DMRG_PREC_FP64) fail(DMRG_ERR_ARG, "dmrg_heff_apply_noalloc computes in FP64");
    if (!st->Lvalid[iL] || !st->Rvalid[iL + 1]) fail(DMRG_ERR_STATE, "environments not built");
    set_device(c);
    heff_apply_noalloc(st, iL, psi_in, psi_out);
  });
}

int dmrg_sweep(dmrg_state* st, const dmrg_mpo* mpo, const dmrg_params* p, dmrg_sweep_stats* out) {
  if (!st) return DMRG_ERR_ARG;
  dmrg_ctx* c = st->ctx;
  return guarded(c, [&] {
    if (mpo != st->mpo) fail(DMRG_ERR_ARG, "state was uploaded with a different MPO");
    if (!p || !out) fail(DMRG_ERR_ARG, "null params/stats");
    set_device(c);
    // dmrgcvg (algs/DMRG.jl:610-652): the first comparison is against the starting energy
    // (startval, algs/optimizeMPS.jl:365-371; <psi|H|psi> of the canonical input) or entropy 0
    if (p->goal > 0 && !st->have_last) {
      if (!st->env_built) fail(DMRG_ERR_STATE, "call dmrg_env_build before dmrg_sweep");
      st->last_energy = p->cvgE ? measure_expect(st, st->mpo, nullptr) : 0.0;
      st->last_entropy = 0.0;
      st->have_last = true;
    }
    do_sweep(st, *p, *out);
    if (p->goal > 0) {
      const double chk = p->cvgE ? std::fabs(out->energy - st->last_energy)
                                 : std::fabs(st->last_entropy - out->entropy);
      out->cvg_check = chk;
      out->converged = chk < p->goal ? 1 : 0;
      if (!out->converged) {
        st->last_energy = out->energy;
        st->last_entropy = out->entropy;
      }
    }
  });
}

void dmrg_noise_default(dmrg_noise* nz) {
  if (!nz) return;
  std::memset(nz, 0, sizeof(*nz));
  nz->noise = 1.0;
  nz->noise_goal = 0.3;
  nz->noise_incr = 0.01;
}

int dmrg_sweep3s(dmrg_state* st, const dmrg_mpo* mpo, const dmrg_params* p, dmrg_noise* nz,
                 dmrg_sweep_stats* out) {
  if (!st) return DMRG_ERR_ARG;
  dmrg_ctx* c = st->ctx;
  return guarded(c, [&] {
    if (mpo != st->mpo) fail(DMRG_ERR_ARG, "state was uploaded with a different MPO");
    if (!p || !out || !nz) fail(DMRG_ERR_ARG, "null params/noise/stats");
    set_device(c);
    // lastenergy starts at startval (algs/optimizeMPS.jl:365-371), <psi|H|psi> of the input
    if (!st->have_last) {
      if (!st->env_built) fail(DMRG_ERR_STATE, "call dmrg_env_build before dmrg_sweep3s");
      st->last_energy = measure_expect(st, st->mpo, nullptr);
      st->last_entropy = 0.0;
      st->have_last = true;
    }
    double alpha = nz->noise;
    do_sweep3s(st, *p, *nz, &alpha, st->last_energy, *out);
    nz->noise = alpha;
    // dmrgcvg (algs/DMRG.jl:626-652): with cvgE the last energy moves on unless converged
    const double chk = p->cvgE ? std::fabs(out->energy - st->last_energy)
                               : std::fabs(st->last_entropy - out->entropy);
    out->cvg_check = p->goal > 0 ? chk : 0.0;
    out->converged = (p->goal > 0 && chk < p->goal) ? 1 : 0;
    if (!out->converged) {
      if (p->cvgE) st->last_energy = out->energy;
      else st->last_entropy = out->entropy;
    }
  });
}

int dmrg_tdvp(dmrg_state* st, const dmrg_mpo* mpo, const dmrg_params* p, double prefactor,
              int twosite, dmrg_sweep_stats* out) {
  if (!st) return DMRG_ERR_ARG;
  dmrg_ctx* c = st->ctx;
  return guarded(c, [&] {
    if (mpo != st->mpo) fail(DMRG_ERR_ARG, "state was uploaded with a different MPO");
    if (!p || !out) fail(DMRG_ERR_ARG, "null params/stats");
    set_device(c);
    do_tdvp(st, *p, prefactor, twosite != 0, *out);
  });
}

int dmrg_test_syevt(dmrg_ctx* c, int nmat, const int* n, const int* k, double* A, double* w,
                    double* U) {
  if (!c) return DMRG_ERR_ARG;
  return guarded(c, [&] {
    if (nmat <= 0 || !n || !k || !A || !w || !U) fail(DMRG_ERR_ARG, "bad syevt arguments");
    set_device(c);
    int64_t ta = 0, tw = 0, tu = 0;
    int mn = 0, mk = 0;
    for (int i = 0; i < nmat; ++i) {
      if (n[i] <= 0 || n[i] > SYEVT_MID_NMAX || k[i] < 0 || k[i] > n[i])
        fail(DMRG_ERR_SHAPE, "bad size");
      ta += int64_t(n[i]) * n[i];
      tw += n[i];
      tu += int64_t(n[i]) * k[i];
      mn = std::max(mn, n[i]);
      mk = std::max(mk, k[i]);
    }
    std::vector<TridTask> tasks;
    int64_t oa = 0, ow = ta, ows = ta + tw, ou = ta + 4 * tw;
    for (int i = 0; i < nmat; ++i) {
      TridTask t{oa, ow, ows, ou, n[i], k[i], 0};
      tasks.push_back(t);
      oa += int64_t(n[i]) * n[i];
      ow += n[i];
      ows += 3 * n[i];
      ou += int64_t(n[i]) * k[i];
    }
    DBuf buf;
    dalloc(c, buf, ta + 4 * tw + tu);
    cuda_check(cudaMemcpyAsync(buf.p, A, ta * 8, cudaMemcpyHostToDevice, c->stream), "A");
    run_trid_eigvals(c, buf.p, buf.n, tasks, 8);
    if (mk > 0) run_trid_vectors(c, buf.p, buf.n, tasks, 6);
    cuda_check(cudaMemcpyAsync(w, buf.p + ta, tw * 8, cudaMemcpyDeviceToHost, c->stream), "w");
    cuda_check(cudaMemcpyAsync(U, buf.p + ta + 4 * tw, tu * 8, cudaMemcpyDeviceToHost, c->stream), "U");
    cuda_check(cudaStreamSynchronize(c->stream), "syevt sync");
    dfree(c, buf);
  });
}

}  // extern "C"

extern "C" {

int dmrg_test_gemm(dmrg_ctx* c, int transA, int transB, int M, int N, int K, const double* A,
                   int lda, const double* B, int ldb, double* C, int ldc) {
  if (!c) return DMRG_ERR_ARG;
  return guarded(c, [&] {
    if (M <= 0 || N <= 0 || K < 0 || !A || !B || !C) fail(DMRG_ERR_ARG, "bad gemm arguments");
    set_device(c);
    const int64_t nA = transA ? int64_t(lda) * M : int64_t(lda) * std::max(K, 1);
    const int64_t nB = transB ? int64_t(ldb) * std::max(K, 1) : int64_t(ldb) * N;
    const int64_t nC = int64_t(ldc) * N;
    DBuf a, b, cc;
    dalloc(c, a, nA);
    dalloc(c, b, nB);
    dalloc(c, cc, nC);
    cuda_check(cudaMemcpyAsync(a.p, A, nA * 8, cudaMemcpyHostToDevice, c->stream), "A");
    cuda_check(cudaMemcpyAsync(b.p, B, nB * 8, cudaMemcpyHostToDevice, c->stream), "B");
    cuda_check(cudaMemcpyAsync(cc.p, C, nC * 8, cudaMemcpyHostToDevice, c->stream), "C");
    GemmList g;
    g.tA = transA != 0;
    g.tB = transB != 0;
    g.add(0, ldc, M, N, 1.0, 0.0);
    g.seg(0, lda, 0, ldb, K);
    Upload u;
    u.put(g);
    char* db = u.send(c, 0);
    run_gemm(c, g, db, a.p, a.n, b.p, b.n, cc.p, cc.n);
    cuda_check(cudaMemcpyAsync(C, cc.p, nC * 8, cudaMemcpyDeviceToHost, c->stream), "C D2H");
    cuda_check(cudaStreamSynchronize(c->stream), "gemm sync");
    dfree(c, a);
    dfree(c, b);
    dfree(c, cc);
  });
}

int dmrg_test_eigh(dmrg_ctx* c, int nmat, const int* n, double* A, double* w) {
  if (!c) return DMRG_ERR_ARG;
  return guarded(c, [&] {
    if (nmat <= 0 || !n || !A || !w) fail(DMRG_ERR_ARG, "bad eigh arguments");
    set_device(c);
    int64_t tot = 0, totw = 0;
    for (int i = 0; i < nmat; ++i) { tot += int64_t(n[i]) * n[i]; totw += n[i]; }
    std::vector<EigTask> tasks;
    int64_t off = 0, woff = 0;
    for (int i = 0; i < nmat; ++i) {
      EigTask t{};
      t.a_off = off;
      t.v_off = off;
      t.w_off = tot + woff;
      t.n = n[i];
      off += int64_t(n[i]) * n[i];
      woff += n[i];
      tasks.push_back(t);
    }
    const int64_t ws = eig_workspace(tasks);
    DBuf buf;
    dalloc(c, buf, tot + totw + ws);
    cuda_check(cudaMemcpyAsync(buf.p, A, tot * 8, cudaMemcpyHostToDevice, c->stream), "A");
    int sweeps = 0;
    run_eigs(c, buf.p, buf.n, tasks, tot + totw, &sweeps);
    cuda_check(cudaMemcpyAsync(A, buf.p, tot * 8, cudaMemcpyDeviceToHost, c->stream), "V D2H");
    cuda_check(cudaMemcpyAsync(w, buf.p + tot, totw * 8, cudaMemcpyDeviceToHost, c->stream), "w");
    cuda_check(cudaStreamSynchronize(c->stream), "eigh sync");
    dfree(c, buf);
  });
}

}  // extern "C"
