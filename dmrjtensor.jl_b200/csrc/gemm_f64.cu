// gemm_f64.cu -- persistent grouped FP64 GEMM on the FP64 tensor-core path (DMMA, m8n8k4).
//
// One launch executes every block product of one contraction step (all QN block triples), as
// a flat list of 64x64 output tiles; each CTA walks tiles with a stride of gridDim.x. A tile
// accumulates over the K-segments of its task (stacked MPO channels, physical states) through a
// 3-stage cp.async pipeline. Operands may be transposed (NN, NT, TN) so that no permute copies
// are needed anywhere in the sweep. B200 has no tcgen05 FP64 kind; mma.sync f64 is the FP64
// tensor-core instruction on sm_100a.
#include <atomic>
#include <map>
#include <mutex>
#include <utility>

#include "kernels.cuh"
#include "launch.cuh"

namespace dmrg {
namespace {

constexpr int BK = GEMM_BK;
constexpr int STAGES = 3, PAD = 4, THREADS = 128;

template <int BM, int BN>
struct F64Tile {
  static constexpr int LDS_A = BM + PAD;   // k-slices of A / B in shared memory, padded rows
  static constexpr int LDS_B = BN + PAD;
  static constexpr size_t SMEM = size_t(STAGES) * BK * (LDS_A + LDS_B) * sizeof(double);
  static constexpr int MI = BM / 16, NI = BN / 16;   // m8n8 fragments per warp (2 x 2 warps)
  static constexpr int A_PER = BM * BK / THREADS, B_PER = BN * BK / THREADS;
};

__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, bool pred) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  int sz = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// D(8x8) += A(8x4, row) * B(4x8, col). Lane l holds A[l>>2][l&3], B[l&3][l>>2],
// D[l>>2][2*(l&3) + {0,1}].
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

template <int BM, int BN, bool TA, bool TB>
__global__ void __launch_bounds__(THREADS)
k_gemm_f64(const double* __restrict__ A, const double* __restrict__ B, double* __restrict__ C,
           const GemmTask* __restrict__ tasks, int ntasks, const GemmSeg* __restrict__ segs,
           int total_tiles) {
  grid_entry();
  using TL = F64Tile<BM, BN>;
  constexpr int LDS_A = TL::LDS_A, LDS_B = TL::LDS_B, MI = TL::MI, NI = TL::NI;
  constexpr int A_PER = TL::A_PER, B_PER = TL::B_PER;
  extern __shared__ double smem[];
  double* As = smem;
  double* Bs = smem + STAGES * BK * LDS_A;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp & 1, wn = warp >> 1;
  const int g = lane >> 2, t = lane & 3;

  for (int tile = blockIdx.x; tile < total_tiles; tile += gridDim.x) {
    int lo = 0, hi = ntasks - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (tasks[mid].tile0 <= tile) lo = mid; else hi = mid - 1;
    }
    const GemmTask tk = tasks[lo];
    const int local = tile - tk.tile0;
    const int m0 = (local % tk.tiles_m) * BM;
    const int n0 = (local / tk.tiles_m) * BN;
    int nsteps = 0;
    for (int q = 0; q < tk.nseg; ++q) nsteps += (segs[tk.seg0 + q].K + BK - 1) / BK;

    double acc[MI][NI][2];
#pragma unroll
    for (int i = 0; i < MI; ++i)
#pragma unroll
      for (int j = 0; j < NI; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    int p_seg = 0, p_k = 0;  // producer cursor
    auto issue = [&](int stage) {
      while (segs[tk.seg0 + p_seg].K <= p_k) { ++p_seg; p_k = 0; }
      const GemmSeg sg = segs[tk.seg0 + p_seg];
      const double* Ab = A + sg.a_off;
      const double* Bb = B + sg.b_off;
      double* as = As + stage * BK * LDS_A;
      double* bs = Bs + stage * BK * LDS_B;
      // thread e = tid + THREADS r covers element (i, k) of the A slice (rows fastest unless A is
      // stored K-contiguous) and (k, j) of the B slice (K fastest unless B is stored N-contiguous)
#pragma unroll
      for (int r = 0; r < A_PER; ++r) {
        const int e = tid + THREADS * r;
        const int i = TA ? e / BK : e % BM, k = TA ? e % BK : e / BM;
        const int gi = m0 + i, gk = p_k + k;
        const bool ok = gi < tk.M && gk < sg.K;
        const double* src = TA ? Ab + gk + int64_t(gi) * sg.lda : Ab + gi + int64_t(gk) * sg.lda;
        cp_async8(&as[k * LDS_A + i], ok ? src : Ab, ok);
      }
#pragma unroll
      for (int r = 0; r < B_PER; ++r) {
        const int e = tid + THREADS * r;
        const int j = TB ? e % BN : e / BK, k = TB ? e / BN : e % BK;
        const int gj = n0 + j, gk = p_k + k;
        const bool ok = gj < tk.N && gk < sg.K;
        const double* src = TB ? Bb + gj + int64_t(gk) * sg.ldb : Bb + gk + int64_t(gj) * sg.ldb;
        cp_async8(&bs[k * LDS_B + j], ok ? src : Bb, ok);
      }
      p_k += BK;
    };

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
      if (s < nsteps) issue(s);
      cp_commit();
    }
    for (int step = 0; step < nsteps; ++step) {
      cp_wait<STAGES - 2>();
      __syncthreads();
      const int nxt = step + STAGES - 1;
      if (nxt < nsteps) issue(nxt % STAGES);
      cp_commit();
      const double* as = As + (step % STAGES) * BK * LDS_A;
      const double* bs = Bs + (step % STAGES) * BK * LDS_B;
#pragma unroll
      for (int kk = 0; kk < BK; kk += 4) {
        double a[MI], b[NI];
#pragma unroll
        for (int mi = 0; mi < MI; ++mi) a[mi] = as[(kk + t) * LDS_A + wm * (BM / 2) + mi * 8 + g];
#pragma unroll
        for (int ni = 0; ni < NI; ++ni) b[ni] = bs[(kk + t) * LDS_B + wn * (BN / 2) + ni * 8 + g];
#pragma unroll
        for (int mi = 0; mi < MI; ++mi)
#pragma unroll
          for (int ni = 0; ni < NI; ++ni) dmma(acc[mi][ni][0], acc[mi][ni][1], a[mi], b[ni]);
      }
    }
    cp_wait<0>();
    __syncthreads();

    double* Cb = C + tk.c_off;
#pragma unroll
    for (int mi = 0; mi < MI; ++mi) {
      const int row = m0 + wm * (BM / 2) + mi * 8 + g;
      if (row >= tk.M) continue;
#pragma unroll
      for (int ni = 0; ni < NI; ++ni) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int col = n0 + wn * (BN / 2) + ni * 8 + 2 * t + e;
          if (col < tk.N) {
            const int64_t idx = row + int64_t(col) * tk.ldc;
            double v = tk.alpha * acc[mi][ni][e];
            if (tk.beta != 0.0) v += tk.beta * Cb[idx];
            Cb[idx] = v;
          }
        }
      }
    }
  }
}

template <int BM, int BN, bool TA, bool TB>
void launch_variant(cudaStream_t s, const double* A, const double* B, double* C,
                    const GemmTask* tasks, int ntasks, const GemmSeg* segs, int total_tiles,
                    int grid_cap) {
  constexpr size_t SM = F64Tile<BM, BN>::SMEM;
  raise_smem_limit(reinterpret_cast<const void*>(k_gemm_f64<BM, BN, TA, TB>), SM);
  int grid = total_tiles < grid_cap ? total_tiles : grid_cap;
  launch_k(k_gemm_f64<BM, BN, TA, TB>, grid, THREADS, SM, s, A, B, C, tasks, ntasks, segs,
           total_tiles);
  count_launch();
}

template <int BM, int BN>
void dispatch_f64(cudaStream_t s, bool transA, bool transB, const double* A, const double* B,
                  double* C, const GemmTask* tasks, int ntasks, const GemmSeg* segs,
                  int total_tiles, int grid_cap) {
  if (!transA && !transB)
    launch_variant<BM, BN, false, false>(s, A, B, C, tasks, ntasks, segs, total_tiles, grid_cap);
  else if (!transA && transB)
    launch_variant<BM, BN, false, true>(s, A, B, C, tasks, ntasks, segs, total_tiles, grid_cap);
  else if (transA && !transB)
    launch_variant<BM, BN, true, false>(s, A, B, C, tasks, ntasks, segs, total_tiles, grid_cap);
  else
    launch_variant<BM, BN, true, true>(s, A, B, C, tasks, ntasks, segs, total_tiles, grid_cap);
}

}  // namespace

void launch_gemm_f64(cudaStream_t s, int tile, bool transA, bool transB, const double* A,
                     const double* B, double* C, const GemmTask* tasks, int ntasks,
                     const GemmSeg* segs, int total_tiles, int grid_cap) {
  if (total_tiles <= 0 || ntasks <= 0) return;
  if (tile == 32)
    dispatch_f64<32, 32>(s, transA, transB, A, B, C, tasks, ntasks, segs, total_tiles, grid_cap);
  else
    dispatch_f64<64, 64>(s, transA, transB, A, B, C, tasks, ntasks, segs, total_tiles, grid_cap);
}

// Raises (never lowers) the dynamic shared-memory limit of a kernel on the current device. The
// limit is a property of the kernel shared by every host thread, so launchers on different
// threads (one context each) must never lower it below what another thread launches with.
void raise_smem_limit(const void* func, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> cur;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  size_t& c = cur[{dev, func}];
  if (bytes > c &&
      cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)) ==
          cudaSuccess)
    c = bytes;
}

static std::atomic<long long> g_launches{0};
void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

int device_sm_count() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n;
}

}  // namespace dmrg
