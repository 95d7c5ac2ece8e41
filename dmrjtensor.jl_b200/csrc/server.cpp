// server.cpp -- serving loop: independent two-site DMRG solves submitted asynchronously and run
// concurrently on one GPU (declared in include/dmrg_b200.h, "serving").
//
// Each worker thread owns one context (one CUDA stream) and runs one solve at a time through the
// library's own entry points: MPO and MPS upload, environment build, the sweeps, download. The
// bond steps of a solve are latency-bound (small blocks, one host round trip per step), so
// several solves on separate streams fill the GPU that one solve leaves idle. Admission is
// first come first served: the head of the queue starts when a worker is free and its
// worst-case device footprint fits in what the running solves leave of the HBM budget (or
// nothing is running). Every context has its own buffers, scalars and descriptor slots and the
// kernels are deterministic, so a solve gives the same bits alone and in a mix.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "engine.hpp"

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
  long long ticket = 0;
  // request copy
  int L = 0, nsym = 0, oc = 0, sweeps = 0;
  dmrg_params params{};
  std::vector<int> d, wl, wr, ml, mr;
  std::vector<std::vector<double>> W, A;
  std::vector<std::vector<int>> pq;
  size_t footprint = 0;
  // result
  int status = DMRG_REQ_QUEUED;
  int error = DMRG_OK;
  std::string message;
  double energy = 0, truncerr = 0, entropy = 0;
  int biggest_m = 0, sweeps_done = 0, final_oc = 0;
  Clock::time_point t_submit, t_start, t_done;
  std::vector<std::vector<double>> site;   // final MPS, dense-equivalent
  std::vector<int> sml, smr;
};

// Worst-case device bytes of a solve: dense-equivalent MPS, environments, and the two-site
// working set (Krylov vectors, Heff intermediates, density matrices) at the largest bond.
size_t footprint(const Job& j) {
  const int L = j.L;
  const double cap = 1e9;
  std::vector<double> m(L + 1, 1.0);
  const double maxm = j.params.maxm > 0 ? double(j.params.maxm) : cap;
  std::vector<double> left(L + 1, 1.0), right(L + 1, 1.0);
  for (int b = 1; b <= L; ++b) left[b] = std::min(cap, left[b - 1] * j.d[b - 1]);
  for (int b = L - 1; b >= 0; --b) right[b] = std::min(cap, right[b + 1] * j.d[b]);
  for (int b = 0; b <= L; ++b) {
    double mb = std::min({maxm, left[b], right[b]});
    if (b < L) mb = std::max(mb, double(j.ml[b]));
    if (b > 0) mb = std::max(mb, double(j.mr[b - 1]));
    m[b] = mb;
  }
  double mps = 0, env = 0, n2 = 0, rho = 0, wmax = 1;
  for (int i = 0; i < L; ++i) {
    mps += m[i] * j.d[i] * m[i + 1];
    env += 2.0 * m[i] * m[i] * j.wl[i];
    wmax = std::max(wmax, double(std::max(j.wl[i], j.wr[i])));
    if (i + 1 < L) {
      n2 = std::max(n2, m[i] * j.d[i] * j.d[i + 1] * m[i + 2]);
      const double side = std::max(m[i] * j.d[i], j.d[i + 1] * m[i + 2]);
      rho = std::max(rho, side * side);
    }
  }
  const int kdim = std::max(2, std::min(j.params.krylov, 16));
  const double doubles = mps + env + (kdim + 3) * n2 + 4 * wmax * n2 + 4 * rho + 2.5e5;
  return size_t(std::min(8.0 * doubles, 1.8e19));
}

}  // namespace

struct dmrg_server {
  int device = 0;
  size_t budget = 0;
  dmrg::HeffBatcher* batch = nullptr;   // shared Heff launches (null: every solve on its own)
  std::vector<dmrg_ctx*> ctx;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv;          // queue changes, admissions, completions
  std::deque<std::shared_ptr<Job>> queue;
  std::map<long long, std::shared_ptr<Job>> jobs;
  long long next_ticket = 1;
  size_t used = 0;
  int running = 0;
  bool stop = false;
  std::string err;
};

namespace {

double seconds(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double>(b - a).count();
}

// Runs one solve in context c through the public entry points; fills the job's result fields
// (the caller publishes them by setting the status under the server lock). Returns false on error.
bool run_job(dmrg_ctx* c, Job& j) {
  dmrg_mpo* mpo = nullptr;
  dmrg_state* st = nullptr;
  auto failed = [&](int code) {
    j.error = code;
    j.message = dmrg_last_error(c);
    return true;
  };
  std::vector<const double*> Wp(j.L), Ap(j.L);
  std::vector<const int*> qp(j.L, nullptr);
  for (int i = 0; i < j.L; ++i) {
    Wp[i] = j.W[i].data();
    Ap[i] = j.A[i].data();
    if (j.nsym > 0) qp[i] = j.pq[i].data();
  }
  int code = dmrg_mpo_upload(c, j.L, j.nsym, j.d.data(), j.wl.data(), j.wr.data(), Wp.data(),
                             j.nsym > 0 ? qp.data() : nullptr, nullptr, &mpo);
  bool bad = code != DMRG_OK && failed(code);
  if (!bad) {
    code = dmrg_mps_upload(c, mpo, j.ml.data(), j.mr.data(), Ap.data(), nullptr, j.oc, &st);
    bad = code != DMRG_OK && failed(code);
  }
  if (!bad) {
    code = dmrg_env_build(st, mpo);
    bad = code != DMRG_OK && failed(code);
  }
  // inside the sweeps the solve's Heff applications join the server's shared launches
  struct Batched {
    dmrg_ctx* c;
    explicit Batched(dmrg_ctx* x) : c(x) {
      if (c->batch) { batcher_enter(c->batch); c->batch_on = true; }
    }
    ~Batched() {
      if (c->batch) { c->batch_on = false; batcher_leave(c->batch); }
    }
  };
  std::unique_ptr<Batched> batched(bad ? nullptr : new Batched(c));
  for (int s = 0; !bad && s < j.sweeps; ++s) {
    dmrg_sweep_stats ss;
    code = dmrg_sweep(st, mpo, &j.params, &ss);
    if (code != DMRG_OK) { bad = failed(code); break; }
    j.energy = ss.energy;
    j.truncerr = ss.max_truncerr;
    j.entropy = ss.entropy;
    j.biggest_m = ss.biggest_m;
    j.sweeps_done = s + 1;
    if (ss.converged) break;     // dmrgcvg's goal test (algs/DMRG.jl:610-652)
  }
  batched.reset();
  if (!bad) {
    j.site.resize(j.L);
    j.sml.resize(j.L);
    j.smr.resize(j.L);
    for (int i = 0; i < j.L && !bad; ++i) {
      int a = 0, b = 0;
      code = dmrg_mps_download(st, i, nullptr, &a, &b);
      if (code == DMRG_OK) {
        j.site[i].assign(size_t(a) * j.d[i] * b, 0.0);
        code = dmrg_mps_download(st, i, j.site[i].data(), &a, &b);
      }
      if (code != DMRG_OK) bad = failed(code);
      j.sml[i] = a;
      j.smr[i] = b;
    }
    if (!bad) dmrg_state_oc(st, &j.final_oc);
  }
  if (st) dmrg_state_destroy(st);
  if (mpo) dmrg_mpo_destroy(mpo);
  return !bad;
}

void worker(dmrg_server* s, int w) {
  for (;;) {
    std::shared_ptr<Job> j;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv.wait(lk, [&] {
        if (s->queue.empty()) return s->stop;
        const size_t fp = s->queue.front()->footprint;
        return s->running == 0 || s->budget == 0 || s->used + fp <= s->budget;
      });
      if (s->queue.empty()) return;   // stop requested and nothing left to run
      j = s->queue.front();
      s->queue.pop_front();
      s->used += j->footprint;
      s->running += 1;
      j->status = DMRG_REQ_RUNNING;
      j->t_start = Clock::now();
    }
    s->cv.notify_all();
    const bool ok = run_job(s->ctx[w], *j);
    {
      std::lock_guard<std::mutex> lk(s->mu);
      j->status = ok ? DMRG_REQ_DONE : DMRG_REQ_FAILED;
      j->t_done = Clock::now();
      s->used -= j->footprint;
      s->running -= 1;
      // the request copy is not needed any more
      j->W.clear(); j->A.clear(); j->pq.clear();
    }
    s->cv.notify_all();
  }
}

int server_fail(dmrg_server* s, int code, const std::string& msg) {
  std::lock_guard<std::mutex> lk(s->mu);
  s->err = msg;
  return code;
}

}  // namespace

extern "C" {

int dmrg_server_create(const dmrg_server_config* cfg, dmrg_server** out) {
  if (!cfg || !out) return DMRG_ERR_ARG;
  *out = nullptr;
  if (cfg->slots < 1 || cfg->slots > 256) return DMRG_ERR_ARG;
  auto* s = new dmrg_server();
  s->device = cfg->device;
  s->budget = cfg->hbm_budget_bytes;
  for (int w = 0; w < cfg->slots; ++w) {
    dmrg_ctx* c = nullptr;
    const int code = dmrg_ctx_create(cfg->device, 0, &c);
    if (code != DMRG_OK) {
      for (dmrg_ctx* x : s->ctx) dmrg_ctx_destroy(x);
      delete s;
      return code;
    }
    s->ctx.push_back(c);
  }
  if (!cfg->unbatched) {
    try {
      s->batch = dmrg::batcher_create(cfg->device);
    } catch (const dmrg::Error& e) {
      for (dmrg_ctx* x : s->ctx) dmrg_ctx_destroy(x);
      delete s;
      return e.code;
    }
    for (dmrg_ctx* c : s->ctx) c->batch = s->batch;
  }
  for (int w = 0; w < cfg->slots; ++w) s->workers.emplace_back(worker, s, w);
  *out = s;
  return DMRG_OK;
}

int dmrg_server_submit(dmrg_server* s, const dmrg_request* r, long long* ticket) {
  if (!s || !r || !ticket) return DMRG_ERR_ARG;
  if (r->L < 2 || r->nsym < 0 || r->nsym > 2 || r->sweeps < 0 || !r->d || !r->wl || !r->wr ||
      !r->W || !r->ml || !r->mr || !r->A || (r->nsym > 0 && !r->phys_qn))
    return server_fail(s, DMRG_ERR_ARG, "dmrg_server_submit: bad request");
  auto j = std::make_shared<Job>();
  j->L = r->L;
  j->nsym = r->nsym;
  j->oc = r->oc;
  j->sweeps = r->sweeps;
  j->params = r->params;
  j->d.assign(r->d, r->d + r->L);
  j->wl.assign(r->wl, r->wl + r->L);
  j->wr.assign(r->wr, r->wr + r->L);
  j->ml.assign(r->ml, r->ml + r->L);
  j->mr.assign(r->mr, r->mr + r->L);
  for (int i = 0; i < r->L; ++i) {
    if (j->d[i] < 1 || j->wl[i] < 1 || j->wr[i] < 1 || j->ml[i] < 1 || j->mr[i] < 1 || !r->W[i] ||
        !r->A[i] || (r->nsym > 0 && !r->phys_qn[i]))
      return server_fail(s, DMRG_ERR_ARG, "dmrg_server_submit: bad site " + std::to_string(i));
    j->W.emplace_back(r->W[i], r->W[i] + size_t(j->wl[i]) * j->d[i] * j->d[i] * j->wr[i]);
    j->A.emplace_back(r->A[i], r->A[i] + size_t(j->ml[i]) * j->d[i] * j->mr[i]);
    if (r->nsym > 0) j->pq.emplace_back(r->phys_qn[i], r->phys_qn[i] + j->d[i] * r->nsym);
  }
  j->footprint = footprint(*j);
  if (s->budget > 0 && j->footprint > s->budget)
    return server_fail(s, DMRG_ERR_BUDGET,
                       "dmrg_server_submit: the solve needs up to " + std::to_string(j->footprint) +
                           " bytes, the budget is " + std::to_string(s->budget));
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) {
      s->err = "dmrg_server_submit: server is shutting down";
      return DMRG_ERR_STATE;
    }
    j->ticket = s->next_ticket++;
    j->t_submit = Clock::now();
    s->jobs[j->ticket] = j;
    s->queue.push_back(j);
    *ticket = j->ticket;
  }
  s->cv.notify_all();
  return DMRG_OK;
}

int dmrg_server_poll(dmrg_server* s, long long ticket, int wait_ms, dmrg_result* out) {
  if (!s || !out) return DMRG_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->jobs.find(ticket);
  if (it == s->jobs.end()) {
    s->err = "dmrg_server_poll: unknown ticket";
    return DMRG_ERR_ARG;
  }
  std::shared_ptr<Job> j = it->second;
  auto finished = [&] { return j->status == DMRG_REQ_DONE || j->status == DMRG_REQ_FAILED; };
  if (wait_ms < 0) s->cv.wait(lk, finished);
  else if (wait_ms > 0) s->cv.wait_for(lk, std::chrono::milliseconds(wait_ms), finished);
  std::memset(out, 0, sizeof(*out));
  out->status = j->status;
  out->footprint_bytes = j->footprint;
  if (finished()) {   // result fields are written by the worker before it publishes the status
    out->error = j->error;
    out->energy = j->energy;
    out->max_truncerr = j->truncerr;
    out->entropy = j->entropy;
    out->biggest_m = j->biggest_m;
    out->sweeps_done = j->sweeps_done;
  }
  const auto now = Clock::now();
  if (j->status == DMRG_REQ_QUEUED) {
    out->queue_seconds = seconds(j->t_submit, now);
  } else {
    out->queue_seconds = seconds(j->t_submit, j->t_start);
    out->run_seconds = seconds(j->t_start, finished() ? j->t_done : now);
  }
  if (j->status == DMRG_REQ_FAILED) s->err = j->message;
  return DMRG_OK;
}

int dmrg_server_fetch_site(dmrg_server* s, long long ticket, int site, double* out, int* ml,
                           int* d, int* mr, int* oc) {
  if (!s) return DMRG_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(ticket);
  if (it == s->jobs.end()) {
    s->err = "dmrg_server_fetch_site: unknown ticket";
    return DMRG_ERR_ARG;
  }
  const Job& j = *it->second;
  if (j.status != DMRG_REQ_DONE) {
    s->err = "dmrg_server_fetch_site: the solve has not finished successfully";
    return DMRG_ERR_STATE;
  }
  if (site < 0 || site >= j.L) {
    s->err = "dmrg_server_fetch_site: bad site";
    return DMRG_ERR_ARG;
  }
  if (ml) *ml = j.sml[site];
  if (d) *d = j.d[site];
  if (mr) *mr = j.smr[site];
  if (oc) *oc = j.final_oc;
  if (out) std::copy(j.site[site].begin(), j.site[site].end(), out);
  return DMRG_OK;
}

int dmrg_server_release(dmrg_server* s, long long ticket) {
  if (!s) return DMRG_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(ticket);
  if (it == s->jobs.end()) return DMRG_ERR_ARG;
  if (it->second->status != DMRG_REQ_DONE && it->second->status != DMRG_REQ_FAILED) {
    s->err = "dmrg_server_release: the solve has not finished";
    return DMRG_ERR_STATE;
  }
  s->jobs.erase(it);
  return DMRG_OK;
}

int dmrg_server_destroy(dmrg_server* s) {
  if (!s) return DMRG_ERR_ARG;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv.notify_all();
  for (auto& t : s->workers) t.join();
  for (dmrg_ctx* c : s->ctx) dmrg_ctx_destroy(c);
  dmrg::batcher_destroy(s->batch);
  delete s;
  return DMRG_OK;
}

int dmrg_server_stats(dmrg_server* s, long long* batches, long long* contributions) {
  if (!s) return DMRG_ERR_ARG;
  if (batches) *batches = 0;
  if (contributions) *contributions = 0;
  if (s->batch) dmrg::batcher_stats(s->batch, batches, contributions);
  return DMRG_OK;
}

const char* dmrg_server_last_error(const dmrg_server* s) {
  return s ? s->err.c_str() : "null server";
}

}  // extern "C"
