// batch.cpp -- shared Heff launches across the solves of the serving loop (continuous batching).
//
// Every solve of a server runs in its own host thread, context and CUDA stream. Inside its
// sweeps, each Heff application (the L.psi GEMM, the MPO mixing, the Y.R GEMM; the hot path of
// the Lanczos step) is not launched on the solve's own stream: the solve hands its three task
// lists to the server's batcher, which concatenates the lists of every solve that is at a Heff
// application at that moment and runs them as ONE launch per phase on the batcher's stream,
// ordered after each contributor's stream (events) and before its next work. The grouped kernels
// already take arbitrary task lists; the batched lists address every operand by its absolute
// device address (element offsets from address 0), so blocks of different solves sit in one
// launch.
//
// A round fires when every solve that is inside its sweeps has contributed, or when the previous
// round has finished on the GPU and a contributor has waited BATCH_COLLECT_US for others, or at
// the latest BATCH_WAIT_US after a contributor arrived (a solve busy with host work or with a
// larger step does not hold the others up for long), or when a solve leaves its sweeps. While a
// round runs on the GPU the arriving requests collect for the next one: the GPU is never idle
// for a request that waits. Each task's tiles are computed exactly as in a launch of its own
// (tiles are independent; FP64 lists use 64 x 64 tiles, split lists the direct form), so a
// solve's numbers do not depend on the solves it is batched with.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <condition_variable>
#include <cstdint>
#include <mutex>

#include "engine.hpp"

namespace dmrg {

namespace {
constexpr int BATCH_WAIT_US = 1000;
constexpr int BATCH_COLLECT_US = 60;
constexpr int BATCH_POLL_US = 15;
}  // namespace

struct HeffBatcher {
  struct Req {
    GemmList g1, g3;
    MixList mix;
    int form = 0;                  // 0 = FP64, else the split form
    int* mma_status = nullptr;     // the contributor's status word (split timeouts)
    cudaEvent_t ready = nullptr;   // contributor's stream: operands ready
    bool fired = false;
    bool failed = false;
    std::string error;
    cudaEvent_t done = nullptr;    // batcher's stream: results written
  };
  int device = 0, nsm = 148;
  cudaStream_t stream = nullptr;
  std::mutex mu;
  std::condition_variable cv;
  int active = 0;                  // solves inside their sweeps
  std::vector<Req*> pending;
  // descriptor uploads (pinned host + device), two slots used in turn; a slot is reused once its
  // previous copy has completed
  struct Slot {
    char* h = nullptr;
    char* d = nullptr;
    size_t cap = 0;
    cudaEvent_t ev = nullptr;
  } slot[2];
  int next_slot = 0;
  int* d_err = nullptr;            // split-kernel timeout flag of the batched launches (sticky)
  cudaEvent_t last = nullptr;      // recorded after the last round's launches
  std::vector<cudaEvent_t> free_events;
  long long batches = 0, contributions = 0;
};

namespace {

int64_t addr(const void* p) { return int64_t(reinterpret_cast<uintptr_t>(p) / sizeof(double)); }

// src with every operand offset made absolute (bases A, B, C), appended to dst.
void append_gemm(GemmList& dst, const GemmList& src, const double* A, const double* B,
                 const double* C) {
  const int seg_base = int(dst.segs.size());
  for (GemmSeg s : src.segs) {
    s.a_off += addr(A);
    s.b_off += addr(B);
    dst.segs.push_back(s);
  }
  for (GemmTask t : src.tasks) {
    t.c_off += addr(C);
    t.seg0 += seg_base;
    t.tile0 += dst.tiles;
    dst.tasks.push_back(t);
  }
  dst.tiles += src.tiles;
  dst.flops += src.flops;
  dst.tA = src.tA;
  dst.tB = src.tB;
  dst.bm = src.bm;
  dst.bn = src.bn;
}

void append_mix(MixList& dst, const MixList& src, const double* in, const double* out) {
  const int term_base = int(dst.terms.size());
  for (MixTerm m : src.terms) {
    m.in_off += addr(in);
    dst.terms.push_back(m);
  }
  for (MixTask t : src.tasks) {
    t.out_off += addr(out);
    t.term0 += term_base;
    t.tile0 += dst.tiles;
    dst.tasks.push_back(t);
  }
  dst.tiles += src.tiles;
  dst.flops += src.flops;
}

cudaEvent_t take_event(HeffBatcher* b) {
  if (!b->free_events.empty()) {
    cudaEvent_t e = b->free_events.back();
    b->free_events.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "batch event");
  return e;
}

// Runs every pending request as one launch per phase and form. Called with b->mu held.
void fire(HeffBatcher* b) {
  std::vector<HeffBatcher::Req*> reqs;
  reqs.swap(b->pending);
  if (reqs.empty()) return;
  try {
    cuda_check(cudaSetDevice(b->device), "cudaSetDevice");
    struct Merged { GemmList g1, g3; MixList mix; size_t o[6] = {}; bool used = false; };
    Merged fm[3];                                   // by form: FP64, 3xTF32, BF16x9
    for (HeffBatcher::Req* r : reqs) {
      Merged& m = fm[r->form];
      m.used = true;
      append_gemm(m.g1, r->g1, nullptr, nullptr, nullptr);
      append_mix(m.mix, r->mix, nullptr, nullptr);
      append_gemm(m.g3, r->g3, nullptr, nullptr, nullptr);
      cuda_check(cudaStreamWaitEvent(b->stream, r->ready, 0), "batch wait");
    }
    Upload u;
    for (Merged& m : fm) {
      if (!m.used) continue;
      m.o[0] = u.put(m.g1.tasks); m.o[1] = u.put(m.g1.segs);
      m.o[2] = u.put(m.mix.tasks); m.o[3] = u.put(m.mix.terms);
      m.o[4] = u.put(m.g3.tasks); m.o[5] = u.put(m.g3.segs);
    }
    HeffBatcher::Slot& sl = b->slot[b->next_slot];
    b->next_slot ^= 1;
    if (sl.ev) cuda_check(cudaEventSynchronize(sl.ev), "batch descriptor slot");
    const size_t need = std::max<size_t>(u.bytes.size(), 16);
    if (need > sl.cap) {
      const size_t cap = std::max(need, sl.cap * 2);
      if (sl.h) cudaFreeHost(sl.h);
      if (sl.d) cudaFreeAsync(sl.d, b->stream);
      sl.h = nullptr;
      sl.d = nullptr;
      sl.cap = 0;
      cuda_check(cudaMallocHost(reinterpret_cast<void**>(&sl.h), cap), "batch descriptors");
      cuda_check(cudaMallocAsync(reinterpret_cast<void**>(&sl.d), cap, b->stream),
                 "batch descriptors");
      sl.cap = cap;
    }
    std::memcpy(sl.h, u.bytes.data(), u.bytes.size());
    cuda_check(cudaMemcpyAsync(sl.d, sl.h, u.bytes.size(), cudaMemcpyHostToDevice, b->stream),
               "batch descriptor upload");
    if (!sl.ev) cuda_check(cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming), "event");
    cuda_check(cudaEventRecord(sl.ev, b->stream), "event record");
    char* dbase = sl.d;
    for (int f = 0; f < 3; ++f) {
      Merged& m = fm[f];
      if (!m.used) continue;
      const auto* t1 = reinterpret_cast<const GemmTask*>(dbase + m.o[0]);
      const auto* s1 = reinterpret_cast<const GemmSeg*>(dbase + m.o[1]);
      const auto* mt = reinterpret_cast<const MixTask*>(dbase + m.o[2]);
      const auto* mm = reinterpret_cast<const MixTerm*>(dbase + m.o[3]);
      const auto* t3 = reinterpret_cast<const GemmTask*>(dbase + m.o[4]);
      const auto* s3 = reinterpret_cast<const GemmSeg*>(dbase + m.o[5]);
      if (f == 0) {
        launch_gemm_f64(b->stream, GEMM_BM, m.g1.tA, m.g1.tB, nullptr, nullptr, nullptr, t1,
                        int(m.g1.tasks.size()), s1, m.g1.tiles, b->nsm * 4);
      } else {
        launch_gemm_split(f, b->stream, m.g1.tA, m.g1.tB, nullptr, nullptr, nullptr, t1,
                          int(m.g1.tasks.size()), s1, m.g1.tiles, b->nsm * 3, b->d_err);
      }
      if (m.mix.tiles > 0)
        launch_mix(b->stream, nullptr, nullptr, mt, int(m.mix.tasks.size()), mm, m.mix.tiles);
      if (f == 0) {
        launch_gemm_f64(b->stream, GEMM_BM, m.g3.tA, m.g3.tB, nullptr, nullptr, nullptr, t3,
                        int(m.g3.tasks.size()), s3, m.g3.tiles, b->nsm * 4);
      } else {
        launch_gemm_split(f, b->stream, m.g3.tA, m.g3.tB, nullptr, nullptr, nullptr, t3,
                          int(m.g3.tasks.size()), s3, m.g3.tiles, b->nsm * 3, b->d_err);
      }
    }
    cuda_check(cudaGetLastError(), "batched Heff launch");
    for (HeffBatcher::Req* r : reqs) {
      if (r->form != 0 && r->mma_status)   // the batched launches' timeout flag, to the solve
        cuda_check(cudaMemcpyAsync(r->mma_status, b->d_err, sizeof(int), cudaMemcpyDeviceToDevice,
                                   b->stream), "batch status");
      r->done = take_event(b);
      cuda_check(cudaEventRecord(r->done, b->stream), "batch done");
    }
    if (!b->last) cuda_check(cudaEventCreateWithFlags(&b->last, cudaEventDisableTiming), "event");
    cuda_check(cudaEventRecord(b->last, b->stream), "batch round end");
    b->batches += 1;
    b->contributions += int64_t(reqs.size());
  } catch (const Error& e) {
    for (HeffBatcher::Req* r : reqs) {
      r->failed = true;
      r->error = e.msg;
    }
  }
  for (HeffBatcher::Req* r : reqs) r->fired = true;
  b->cv.notify_all();
}

}  // namespace

HeffBatcher* batcher_create(int device) {
  auto* b = new HeffBatcher();
  b->device = device;
  try {
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    cuda_check(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "batch stream");
    cuda_check(cudaMalloc(reinterpret_cast<void**>(&b->d_err), sizeof(int)), "batch flag");
    cuda_check(cudaMemset(b->d_err, 0, sizeof(int)), "batch flag");
    b->nsm = device_sm_count();
  } catch (...) {
    batcher_destroy(b);
    throw;
  }
  return b;
}

void batcher_destroy(HeffBatcher* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (cudaEvent_t e : b->free_events) cudaEventDestroy(e);
  for (auto& sl : b->slot) {
    if (sl.ev) cudaEventDestroy(sl.ev);
    if (sl.h) cudaFreeHost(sl.h);
    if (sl.d) cudaFree(sl.d);
  }
  if (b->d_err) cudaFree(b->d_err);
  if (b->last) cudaEventDestroy(b->last);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

void batcher_enter(HeffBatcher* b) {
  std::lock_guard<std::mutex> lk(b->mu);
  b->active += 1;
}

void batcher_leave(HeffBatcher* b) {
  std::lock_guard<std::mutex> lk(b->mu);
  b->active -= 1;
  // the solves still inside their sweeps may all be waiting now
  if (!b->pending.empty() && int(b->pending.size()) >= b->active) fire(b);
}

void batcher_stats(HeffBatcher* b, long long* batches, long long* contributions) {
  std::lock_guard<std::mutex> lk(b->mu);
  if (batches) *batches = b->batches;
  if (contributions) *contributions = b->contributions;
}

void batched_heff(dmrg_ctx* c, dmrg_state* st, int iL, const HeffPlan& hp, const double* x,
                  double* y, int precision) {
  HeffBatcher* b = c->batch;
  ensure(c, c->X, std::max<int64_t>(hp.x_size, 1));
  ensure(c, c->Y, std::max<int64_t>(hp.y_size, 1));
  const int64_t n = hp.tl.size;
  const int form = split_form(precision);
  if (precision != DMRG_PREC_FP64 && !form)
    fail(DMRG_ERR_ARG, "precision: FP64, 3xTF32 and BF16x9 are the built forms");
  (void)iL;
  const DBuf& Le = st->Lenv[hp.le];
  const DBuf& Re = st->Renv[hp.re];
  // the solve's own lists, tiled for the batched launch, checked against its own buffers
  const GemmList g1 = form ? retile(hp.g1, TF32_TILE_M, TF32_TILE_N_DIRECT)
                           : retile(hp.g1, GEMM_BM, GEMM_BN);
  const GemmList g3 = form ? retile(hp.g3, TF32_TILE_M, TF32_TILE_N_DIRECT)
                           : retile(hp.g3, GEMM_BM, GEMM_BN);
  check_gemm_list(g1, Le.n, n, c->X.n);
  check_mix_list(hp.mix, c->X.n, c->Y.n);
  check_gemm_list(g3, c->Y.n, Re.n, n);
  HeffBatcher::Req r;
  r.form = form;
  r.mma_status = c->d_status + STATUS_MMA;
  append_gemm(r.g1, g1, Le.p, x, c->X.p);
  append_mix(r.mix, hp.mix, c->X.p, c->Y.p);
  append_gemm(r.g3, g3, c->Y.p, Re.p, y);
  {
    std::lock_guard<std::mutex> lk(b->mu);
    r.ready = take_event(b);
  }
  cuda_check(cudaEventRecord(r.ready, c->stream), "batch ready");
  std::unique_lock<std::mutex> lk(b->mu);
  b->pending.push_back(&r);
  if (int(b->pending.size()) >= b->active) fire(b);
  const auto t0 = std::chrono::steady_clock::now();
  const auto collect = t0 + std::chrono::microseconds(BATCH_COLLECT_US);
  const auto deadline = t0 + std::chrono::microseconds(BATCH_WAIT_US);
  while (!r.fired) {
    b->cv.wait_for(lk, std::chrono::microseconds(BATCH_POLL_US));
    if (r.fired) break;
    const auto now = std::chrono::steady_clock::now();
    bool idle = true;   // no round in flight on the batcher's stream
    if (b->last) {
      const cudaError_t q = cudaEventQuery(b->last);
      idle = q != cudaErrorNotReady;
      if (q != cudaSuccess) cudaGetLastError();
    }
    if (now >= deadline || (idle && now >= collect)) fire(b);
  }
  b->free_events.push_back(r.ready);   // the batcher stream's wait has been enqueued
  if (r.failed) fail(DMRG_ERR_CUDA, "batched Heff launch: " + r.error);
  cudaEvent_t done = r.done;
  lk.unlock();
  const cudaError_t e = cudaStreamWaitEvent(c->stream, done, 0);
  lk.lock();
  b->free_events.push_back(done);      // this solve's wait on it has been enqueued
  lk.unlock();
  cuda_check(e, "batch join");
}

}  // namespace dmrg
