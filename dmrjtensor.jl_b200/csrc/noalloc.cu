// noalloc.cu -- the two-site effective Hamiltonian applied without any device allocation.
//
// Some callers cannot allocate device memory at the point where they apply Heff: a host
// framework whose caching allocator already owns all free HBM (so a cudaMalloc from this library
// would fail or fragment the pool), or an iterative solver loop whose latency budget forbids
// allocator calls. dmrg_heff_apply_noalloc serves them: the caller passes device input/output
// vectors, and every intermediate of the contraction (the block-layout copies of the vectors,
// the step-1 and step-2 intermediates, and the task descriptors) lives in one file-scope
// __device__ array of fixed size. Nothing here calls cudaMalloc, cudaFree or an allocating
// library routine.
//
// The array is part of the library image: every GPU that loads the library holds it until the
// process exits. All calls share it and it keeps the previous call's contents; every region a
// call reads is written earlier in the same call, so nothing needs clearing. Calls that overlap
// on the GPU (two host threads, or two contexts on one device) race on the array.
#include <mutex>

#include "engine.hpp"

namespace dmrg {
namespace {

constexpr int64_t NOALLOC_DOUBLES = int64_t(1) << 20;       // 8 MiB of FP64 intermediates
constexpr int64_t NOALLOC_DESC_BYTES = int64_t(1) << 20;    // 1 MiB of task descriptors
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_DOUBLES + NOALLOC_DESC_BYTES / 8];

double* g_scratch_dev[kMaxDevices] = {};
std::mutex g_scratch_mu;

// Device address of the array on `device` (the current device). Host code cannot use the
// array's name as a device address, so the address is looked up once per device.
double* scratch_address(int device) {
  if (device < 0 || device >= kMaxDevices) fail(DMRG_ERR_ARG, "device index out of range");
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_dev[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      fail(DMRG_ERR_CUDA, std::string("cudaGetSymbolAddress of the no-allocation scratch: ") +
                              cudaGetErrorString(e));
    }
    g_scratch_dev[device] = static_cast<double*>(p);
  }
  return g_scratch_dev[device];
}

}  // namespace

void heff_apply_noalloc(dmrg_state* st, int iL, const double* in, double* out) {
  dmrg_ctx* c = st->ctx;
  HeffPlan hp;
  plan_heff(st, iL, hp);                       // host memory only
  const TwoLayout& tl = hp.tl;
  const Bond& Bl = st->bond[iL];
  const Bond& Br = st->bond[iL + 2];
  const int64_t ml = Bl.total(), mr = Br.total(), d1 = tl.d1, d2 = tl.d2;
  const int64_t ndense = ml * d1 * d2 * mr;
  const int64_t need = 2 * tl.size + std::max<int64_t>(hp.x_size, 1) + std::max<int64_t>(hp.y_size, 1);
  if (need > NOALLOC_DOUBLES)
    fail(DMRG_ERR_BUDGET, "dmrg_heff_apply_noalloc: this two-site space needs " +
                              std::to_string(need) + " doubles of scratch, the fixed maximum is " +
                              std::to_string(NOALLOC_DOUBLES) + " (use dmrg_heff_apply)");
  // dense-equivalent [ml, d1, d2, mr] <-> block layout
  const auto ol = Bl.offsets(), orr = Br.offsets();
  const int64_t ldd = ml * d1 * d2;
  CopyList gin, gout;
  for (int ka = 0; ka < tl.nl; ++ka)
    for (int s1 = 0; s1 < d1; ++s1)
      for (int s2 = 0; s2 < d2; ++s2) {
        const int id = tl.idx(ka, s1, s2), kd = tl.kd[id];
        if (kd < 0) continue;
        const int64_t doff = ol[ka] + ml * (s1 + d1 * s2) + orr[kd] * ldd;
        gin.add(doff, int(ldd), tl.off[id], Bl.dim[ka], Bl.dim[ka], Br.dim[kd], 0, 1.0);
        gout.add(tl.off[id], Bl.dim[ka], doff, int(ldd), Bl.dim[ka], Br.dim[kd], 0, 1.0);
      }
  Upload u;
  u.put(hp.g1);
  u.put(hp.mix);
  u.put(hp.g3);
  u.put(gin);
  u.put(gout);
  if (int64_t(u.bytes.size()) > NOALLOC_DESC_BYTES)
    fail(DMRG_ERR_BUDGET, "dmrg_heff_apply_noalloc: the task list needs " +
                              std::to_string(u.bytes.size()) + " bytes, the fixed maximum is " +
                              std::to_string(NOALLOC_DESC_BYTES) + " (use dmrg_heff_apply)");
  double* S = scratch_address(c->device);
  char* desc = reinterpret_cast<char*>(S + NOALLOC_DOUBLES);
  double* bin = S;
  double* bout = bin + tl.size;
  double* X = bout + tl.size;
  double* Y = X + std::max<int64_t>(hp.x_size, 1);
  // pageable host source: the copy is complete before the host vector goes out of scope
  cuda_check(cudaMemcpyAsync(desc, u.bytes.data(), u.bytes.size(), cudaMemcpyHostToDevice,
                             c->stream), "no-allocation descriptor copy");
  hp.dbase = desc;
  // the whole input is gathered into the block layout before the output is touched, so psi_in
  // and psi_out may be the same (or overlapping) device buffers
  run_copy(c, gin, desc, in, ndense, bin, tl.size);
  cuda_check(cudaMemsetAsync(out, 0, size_t(ndense) * sizeof(double), c->stream), "output clear");
  run_gemm(c, hp.g1, desc, st->Lenv[iL].p, st->Lenv[iL].n, bin, tl.size, X, hp.x_size);
  run_mix(c, hp.mix, desc, X, hp.x_size, Y, hp.y_size);
  run_gemm(c, hp.g3, desc, Y, hp.y_size, st->Renv[iL + 1].p, st->Renv[iL + 1].n, bout, tl.size);
  run_copy(c, gout, desc, bout, tl.size, out, ndense);
  cuda_check(cudaStreamSynchronize(c->stream), "no-allocation Heff");
}

}  // namespace dmrg
