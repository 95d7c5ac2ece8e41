// vec_kernels.cu -- memory-bound kernels of the sweep: sparse MPO mixing of block lists,
// strided block copies (gathers/scatters), and the Lanczos vector operations with deterministic
// two-stage warp-shuffle reductions (fixed grid, fixed order: bit-identical from run to run).
#include "kernels.cuh"

namespace dmrg {
namespace {

constexpr int MIX_COLS = 32;      // columns per mixing / copy tile
constexpr int RED_BLOCKS = 296;   // 2 x 148 SMs
constexpr int RED_THREADS = 256;
constexpr int MAXK = 16;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__global__ void k_mix(const double* __restrict__ in, double* __restrict__ out,
                      const MixTask* __restrict__ tasks, int ntasks,
                      const MixTerm* __restrict__ terms, int total_tiles) {
  for (int tile = blockIdx.x; tile < total_tiles; tile += gridDim.x) {
    int lo = 0, hi = ntasks - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (tasks[mid].tile0 <= tile) lo = mid; else hi = mid - 1;
    }
    const MixTask tk = tasks[lo];
    const int c0 = (tile - tk.tile0) * MIX_COLS;
    const int ncol = min(MIX_COLS, tk.cols - c0);
    const int nel = ncol * tk.rows;
    for (int e = threadIdx.x; e < nel; e += blockDim.x) {
      const int r = e % tk.rows, c = c0 + e / tk.rows;
      double acc = 0.0;
      for (int q = 0; q < tk.nterm; ++q) {
        const MixTerm tm = terms[tk.term0 + q];
        acc += tm.coef * in[tm.in_off + r + int64_t(c) * tm.ld];
      }
      out[tk.out_off + r + int64_t(c) * tk.ld] = acc;
    }
  }
}

__global__ void k_copy(const double* __restrict__ src, double* __restrict__ dst,
                       const CopyTask* __restrict__ tasks, int ntasks, int total_tiles) {
  for (int tile = blockIdx.x; tile < total_tiles; tile += gridDim.x) {
    int lo = 0, hi = ntasks - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (tasks[mid].tile0 <= tile) lo = mid; else hi = mid - 1;
    }
    const CopyTask tk = tasks[lo];
    const int c0 = (tile - tk.tile0) * MIX_COLS;
    const int ncol = min(MIX_COLS, tk.cols - c0);
    const int nel = ncol * tk.rows;
    for (int e = threadIdx.x; e < nel; e += blockDim.x) {
      const int r = e % tk.rows, c = c0 + e / tk.rows;
      const double v = tk.trans ? src[tk.src_off + c + int64_t(r) * tk.lds]
                                : src[tk.src_off + r + int64_t(c) * tk.lds];
      dst[tk.dst_off + r + int64_t(c) * tk.ldd] = tk.scale * v;
    }
  }
}

// partial[j*gridDim + b] = sum over this block's share of X_j . y
__global__ void k_mdot_partial(const double* __restrict__ X, int64_t ldx, int k,
                               const double* __restrict__ y, int64_t n, double* partial) {
  double acc[MAXK];
#pragma unroll
  for (int j = 0; j < MAXK; ++j) acc[j] = 0.0;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double yi = y[i];
#pragma unroll
    for (int j = 0; j < MAXK; ++j)
      if (j < k) acc[j] += X[j * ldx + i] * yi;
  }
  __shared__ double red[MAXK][RED_THREADS / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < MAXK; ++j) {
    if (j < k) {
      double v = warp_sum(acc[j]);
      if (lane == 0) red[j][wid] = v;
    }
  }
  __syncthreads();
  if (threadIdx.x < k) {
    double s = 0.0;
    for (int w = 0; w < RED_THREADS / 32; ++w) s += red[threadIdx.x][w];
    partial[threadIdx.x * gridDim.x + blockIdx.x] = s;
  }
}

__global__ void k_reduce_rows(const double* __restrict__ partial, int nb, double* out) {
  const int j = blockIdx.x;
  double s = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partial[j * nb + b];
  s = warp_sum(s);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (blockDim.x + 31) / 32; ++w) t += red[w];
    out[j] = t;
  }
}

__global__ void k_axpby(int64_t n, double a, const double* ap, double asign,
                        const double* __restrict__ x, double b, const double* bp, double bsign,
                        double* y, int b_recip) {
  double aa = a, bb = b;
  if (ap) aa = asign * (*ap);
  if (bp) bb = bsign * (b_recip ? 1.0 / (*bp) : (*bp));
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double xv = x ? x[i] : 0.0;
    y[i] = (bb == 0.0) ? aa * xv : aa * xv + bb * y[i];   // y is not read when bb == 0
  }
}

__global__ void k_msub(const double* __restrict__ X, int64_t ldx, int k,
                       const double* __restrict__ c, double* y, int64_t n) {
  double cc[MAXK];
#pragma unroll
  for (int j = 0; j < MAXK; ++j) cc[j] = j < k ? c[j] : 0.0;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    double v = y[i];
#pragma unroll
    for (int j = 0; j < MAXK; ++j)
      if (j < k) v -= cc[j] * X[j * ldx + i];
    y[i] = v;
  }
}

__global__ void k_scale(double* x, int64_t n, double a) {
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) x[i] *= a;
}

int grid_for(int64_t n) {
  int64_t b = (n + RED_THREADS - 1) / RED_THREADS;
  if (b > 4 * RED_BLOCKS) b = 4 * RED_BLOCKS;
  if (b < 1) b = 1;
  return int(b);
}

}  // namespace

void launch_mix(cudaStream_t s, const double* in, double* out, const MixTask* tasks, int ntasks,
                const MixTerm* terms, int total_tiles) {
  if (total_tiles <= 0) return;
  int grid = total_tiles < 4096 ? total_tiles : 4096;
  k_mix<<<grid, 256, 0, s>>>(in, out, tasks, ntasks, terms, total_tiles);
  count_launch();
}

void launch_copy(cudaStream_t s, const double* src, double* dst, const CopyTask* tasks,
                 int ntasks, int total_tiles) {
  if (total_tiles <= 0) return;
  int grid = total_tiles < 4096 ? total_tiles : 4096;
  k_copy<<<grid, 256, 0, s>>>(src, dst, tasks, ntasks, total_tiles);
  count_launch();
}

void launch_mdot(cudaStream_t s, const double* X, int64_t ldx, int k, const double* y, int64_t n,
                 double* partial, double* out) {
  k_mdot_partial<<<RED_BLOCKS, RED_THREADS, 0, s>>>(X, ldx, k, y, n, partial);
  k_reduce_rows<<<k, 256, 0, s>>>(partial, RED_BLOCKS, out);
  count_launch(2);
}

void launch_axpby(cudaStream_t s, int64_t n, double a, const double* ap, double asign,
                  const double* x, double b, const double* bp, double bsign, double* y,
                  int b_recip) {
  if (n <= 0) return;
  k_axpby<<<grid_for(n), RED_THREADS, 0, s>>>(n, a, ap, asign, x, b, bp, bsign, y, b_recip);
  count_launch();
}

void launch_msub(cudaStream_t s, const double* X, int64_t ldx, int k, const double* c, double* y,
                 int64_t n) {
  if (n <= 0 || k <= 0) return;
  k_msub<<<grid_for(n), RED_THREADS, 0, s>>>(X, ldx, k, c, y, n);
  count_launch();
}

void launch_scale(cudaStream_t s, double* x, int64_t n, double a) {
  if (n <= 0) return;
  k_scale<<<grid_for(n), RED_THREADS, 0, s>>>(x, n, a);
  count_launch();
}

void launch_zero(cudaStream_t s, double* x, int64_t n) {
  if (n <= 0) return;
  cudaMemsetAsync(x, 0, size_t(n) * sizeof(double), s);
}

}  // namespace dmrg
