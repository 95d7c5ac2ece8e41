// vec_kernels.cu -- memory-bound kernels of the sweep: sparse MPO mixing of block lists,
// strided block copies (gathers/scatters), and the Lanczos vector operations with deterministic
// two-stage warp-shuffle reductions (fixed grid, fixed order: bit-identical from run to run).
#include <algorithm>
#include <cstring>

#include "kernels.cuh"
#include "launch.cuh"

namespace dmrg {
namespace {

constexpr int MIX_COLS = 32;      // columns per mixing / copy tile
constexpr int MIX_TALL = 64;      // mixing blocks of at least this many rows: a warp per column
constexpr int MIX_ROWS_PER_LANE = 4;
constexpr int RED_BLOCKS = 296;   // 2 x 148 SMs
constexpr int RED_THREADS = 256;
constexpr int MAXK = 16;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Last-block reduction: every block has written its row partials; the block that arrives last
// (atomic counter, after a fence) sums them in the fixed order of a separate reduction kernel,
// writes out[0..k), and resets the counter for the next kernel on the stream.
__device__ __forceinline__ bool arrive_last(unsigned* counter) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  return last;
}

__device__ void finish_rows(const double* partial, int nb, int k, double* out, unsigned* counter) {
  __shared__ double red[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) / 32;
  __threadfence();
  for (int j = 0; j < k; ++j) {
    double s = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) s += __ldcg(partial + j * nb + b);
    s = warp_sum(s);
    if (lane == 0) red[wid] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < nw; ++w) t += red[w];
      out[j] = t;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *counter = 0u;
}

__global__ void k_mix(const double* __restrict__ in, double* __restrict__ out,
                      const MixTask* __restrict__ tasks, int ntasks,
                      const MixTerm* __restrict__ terms, int total_tiles) {
  grid_entry();
  for (int tile = blockIdx.x; tile < total_tiles; tile += gridDim.x) {
    int lo = 0, hi = ntasks - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (tasks[mid].tile0 <= tile) lo = mid; else hi = mid - 1;
    }
    const MixTask tk = tasks[lo];
    const int c0 = (tile - tk.tile0) * MIX_COLS;
    const int ncol = min(MIX_COLS, tk.cols - c0);
    if (tk.rows >= MIX_TALL) {
      // tall blocks: a warp per column, MIX_ROWS_PER_LANE rows per lane (rows lane + 32 j of a
      // 128-row slab), so that every thread has that many independent loads of a term in flight
      const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
      for (int cc = warp; cc < ncol; cc += nwarp) {
        const int64_t c = c0 + cc;
        for (int r0 = 0; r0 < tk.rows; r0 += 32 * MIX_ROWS_PER_LANE) {
          double acc[MIX_ROWS_PER_LANE];
#pragma unroll
          for (int j = 0; j < MIX_ROWS_PER_LANE; ++j) acc[j] = 0.0;
#pragma unroll 2
          for (int q = 0; q < tk.nterm; ++q) {
            const MixTerm tm = terms[tk.term0 + q];
            const double* src = in + tm.in_off + c * tm.ld;
            double v[MIX_ROWS_PER_LANE];
#pragma unroll
            for (int j = 0; j < MIX_ROWS_PER_LANE; ++j) {
              const int r = r0 + lane + 32 * j;
              v[j] = r < tk.rows ? src[r] : 0.0;
            }
#pragma unroll
            for (int j = 0; j < MIX_ROWS_PER_LANE; ++j) acc[j] += tm.coef * v[j];
          }
#pragma unroll
          for (int j = 0; j < MIX_ROWS_PER_LANE; ++j) {
            const int r = r0 + lane + 32 * j;
            if (r < tk.rows) out[tk.out_off + r + c * tk.ld] = acc[j];
          }
        }
      }
      continue;
    }
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
  grid_entry();
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

// partial[j*gridDim + b] = sum over this block's share of X_j . y; the last block to finish
// writes out[j] = sum_b partial[j*gridDim + b].
__global__ void k_mdot_partial(const double* __restrict__ X, int64_t ldx, int k,
                               const double* __restrict__ y, int64_t n, double* partial,
                               double* out, unsigned* counter) {
  grid_entry();
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
  if (arrive_last(counter)) finish_rows(partial, gridDim.x, k, out, counter);
}

__global__ void k_pair_dot(const double* __restrict__ X, const double* __restrict__ Y,
                           const PairTask* __restrict__ tasks, int ntasks, int64_t total,
                           double* partial, double* out, unsigned* counter) {
  grid_entry();
  double acc = 0.0;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += stride) {
    int lo = 0, hi = ntasks - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (tasks[mid].e0 <= e) lo = mid; else hi = mid - 1;
    }
    const PairTask tk = tasks[lo];
    const int64_t q = e - tk.e0;
    const int64_t r = q % tk.rows, c = q / tk.rows;
    acc += X[tk.x_off + q] * Y[tk.y_off + c + r * tk.cols];
  }
  __shared__ double red[RED_THREADS / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  acc = warp_sum(acc);
  if (lane == 0) red[wid] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < RED_THREADS / 32; ++w) t += red[w];
    partial[blockIdx.x] = t;
  }
  if (arrive_last(counter)) finish_rows(partial, gridDim.x, 1, out, counter);
}

__global__ void k_pair_dot_rows(const double* __restrict__ X, int64_t x_stride,
                                const double* __restrict__ Y, const PairTask* __restrict__ tasks,
                                int ntasks, double* out, int64_t out_stride) {
  grid_entry();
  const double* Xr = X + int64_t(blockIdx.x) * x_stride;
  double acc = 0.0;
  for (int k = 0; k < ntasks; ++k) {
    const PairTask tk = tasks[k];
    const int64_t n = int64_t(tk.rows) * tk.cols;
    for (int64_t q = threadIdx.x; q < n; q += blockDim.x) {
      const int64_t r = q % tk.rows, c = q / tk.rows;
      acc += Xr[tk.x_off + q] * Y[tk.y_off + c + r * tk.cols];
    }
  }
  __shared__ double red[RED_THREADS / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  acc = warp_sum(acc);
  if (lane == 0) red[wid] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < RED_THREADS / 32; ++w) t += red[w];
    out[int64_t(blockIdx.x) * out_stride] = t;
  }
}

__global__ void k_axpby(int64_t n, double a, const double* ap, double asign,
                        const double* __restrict__ x, double b, const double* bp, double bsign,
                        double* y, int b_recip) {
  grid_entry();
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
  grid_entry();
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
  grid_entry();
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) x[i] *= a;
}

// x *= 1/sqrt(*nrm2) when *nrm2 > 0 (normalisation by a device-resident squared norm)
__global__ void k_scale_rsqrt(double* x, int64_t n, const double* nrm2) {
  grid_entry();
  const double v = *nrm2;
  const double a = (v > 0.0) ? 1.0 / sqrt(v) : 1.0;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) x[i] *= a;
}

// partial rows 0/1: this block's share of <x,x> and <x,y>
__global__ void k_dot2_partial(const double* __restrict__ x, const double* __restrict__ y,
                               int64_t n, double* partial, double* out, unsigned* counter) {
  grid_entry();
  double sxx = 0.0, sxy = 0.0;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double xv = x[i];
    sxx += xv * xv;
    sxy += xv * y[i];
  }
  __shared__ double red[2][RED_THREADS / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  sxx = warp_sum(sxx);
  sxy = warp_sum(sxy);
  if (lane == 0) { red[0][wid] = sxx; red[1][wid] = sxy; }
  __syncthreads();
  if (threadIdx.x < 2) {
    double s = 0.0;
    for (int w = 0; w < RED_THREADS / 32; ++w) s += red[threadIdx.x][w];
    partial[threadIdx.x * gridDim.x + blockIdx.x] = s;
  }
  if (arrive_last(counter)) finish_rows(partial, gridDim.x, 2, out, counter);
}

// First half of the reference 2-vector Krylov step, from s[KK] = <K,K> and s[KH] = <K,HK>:
// K <- K / |K|, a1 = <K,HK> / |K| (stored at s[ALPHA]), H <- H - a1 K, and this block's share
// of <H,H> in partial row 0.
__global__ void k_lanczos2_orth(double* K, double* H, int64_t n, double* s, double* partial,
                                unsigned* counter) {
  grid_entry();
  const double nn = sqrt(s[lz::KK]);
  const double inv = 1.0 / nn;
  const double a1 = s[lz::KH] / nn;
  double shh = 0.0;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double k = K[i] * inv;
    const double h = H[i] - a1 * k;
    K[i] = k;
    H[i] = h;
    shh += h * h;
  }
  __shared__ double red[RED_THREADS / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  shh = warp_sum(shh);
  if (lane == 0) red[wid] = shh;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < RED_THREADS / 32; ++w) t += red[w];
    partial[blockIdx.x] = t;
    if (blockIdx.x == 0) s[lz::ALPHA] = a1;
  }
  if (arrive_last(counter)) finish_rows(partial, gridDim.x, 1, s + lz::B2, counter);
}

// Next Krylov vector K_{j+1} = H / beta_j with beta_j = sqrt(s[B2+j]), or 0 once the recursion
// has broken down (beta_j <= betatest, or an earlier breakdown: s[ACT+j] == 0). Every thread
// takes the decision from the same read-only inputs; thread 0 records beta_j (0 on breakdown)
// and the activity of K_{j+1}.
__global__ void k_next_vector(const double* __restrict__ H, double* __restrict__ Kn, int64_t n,
                              double* s, int j, double betatest) {
  grid_entry();
  const bool act = (j == 0) || (s[lz::ACT + j] != 0.0);
  const double b = sqrt(s[lz::B2 + j]);
  const bool ok = act && (b > betatest);
  const double r = ok ? 1.0 / b : 0.0;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    Kn[i] = ok ? r * H[i] : 0.0;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    s[lz::BETA + j] = ok ? b : 0.0;
    s[lz::ACT + j + 1] = ok ? 1.0 : 0.0;
  }
}

// Ritz step of the Krylov solve, one warp: T = tridiag(alpha, beta) of the m active vectors
// (m = 1 + number of leading non-zero beta_j, at most kdim), cyclic Jacobi (serial rotation
// order; lanes own the rows/columns of one rotation) until the off-diagonal is at the rounding
// level of the diagonal, lowest
// eigenvalue -> s[EN], its eigenvector -> s[COEF + j] (0 for j >= m).
// expo = 0: the lowest Ritz pair (s[EN], s[COEF + j]). expo = 1: s[COEF + j] = (exp(tau T) e_1)_j
// (krylovTimeEvol, algs/time.jl:182-203: the Krylov vectors are orthonormal, so these are the
// coefficients of exp(tau H) applied to the normalised start vector), from the eigenpairs of T;
// when they sum to exactly zero, the first column of I + T instead. s[EN] = lowest eigenvalue.
__global__ void k_ritz(double* s, int kdim, double tau, int expo) {
  grid_entry();
  __shared__ double A[MAXK * MAXK], V[MAXK * MAXK];
  const int lane = threadIdx.x;
  int m = 1;
  while (m < kdim && s[lz::BETA + m - 1] > 0.0) ++m;
  for (int e = lane; e < m * m; e += 32) {
    const int r = e % m, c = e / m;
    double v = 0.0;
    if (r == c) v = s[lz::ALPHA + r];
    else if (r == c + 1) v = s[lz::BETA + c];
    else if (c == r + 1) v = s[lz::BETA + r];
    A[e] = v;
    V[e] = (r == c) ? 1.0 : 0.0;
  }
  __syncwarp();
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, dg = 0.0;
    for (int p = 0; p < m; ++p) {
      dg += A[p + p * m] * A[p + p * m];
      for (int q = p + 1; q < m; ++q) off += A[p + q * m] * A[p + q * m];
    }
    if (off < 1e-300 || off <= 1e-32 * dg) break;   // off-diagonal at the rounding level
    for (int p = 0; p < m; ++p)
      for (int q = p + 1; q < m; ++q) {
        const double apq = A[p + q * m];
        if (fabs(apq) < 1e-300) continue;
        const double theta = (A[q + q * m] - A[p + p * m]) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
        __syncwarp();
        if (lane < m) {   // rows p, q
          const double ap = A[p + lane * m], aq = A[q + lane * m];
          A[p + lane * m] = c * ap - sn * aq;
          A[q + lane * m] = sn * ap + c * aq;
        }
        __syncwarp();
        if (lane < m) {   // columns p, q
          const double ap = A[lane + p * m], aq = A[lane + q * m];
          A[lane + p * m] = c * ap - sn * aq;
          A[lane + q * m] = sn * ap + c * aq;
          const double vp = V[lane + p * m], vq = V[lane + q * m];
          V[lane + p * m] = c * vp - sn * vq;
          V[lane + q * m] = sn * vp + c * vq;
        }
        __syncwarp();
      }
  }
  int o = 0;
  for (int k = 1; k < m; ++k)
    if (A[k + k * m] < A[o + o * m]) o = k;   // lowest; ties keep the lower index
  if (lane == 0) s[lz::EN] = A[o + o * m];
  if (!expo) {
    for (int k = lane; k < kdim; k += 32) s[lz::COEF + k] = (k < m) ? V[k + o * m] : 0.0;
    return;
  }
  // c_k = sum_j V[k,j] exp(tau lambda_j) V[0,j]; every lane forms the sum of all c_k itself (the
  // same fixed order in each lane) for the zero test
  double tot = 0.0, mine = 0.0;
  for (int k = 0; k < m; ++k) {
    double ck = 0.0;
    for (int jj = 0; jj < m; ++jj) ck += V[k + jj * m] * exp(tau * A[jj + jj * m]) * V[jj * m];
    tot += ck;
    if (k == lane) mine = ck;
  }
  if (tot == 0.0) {   // (I + T) e_1
    mine = lane == 0 ? 1.0 + s[lz::ALPHA] : (lane == 1 && m > 1 ? s[lz::BETA] : 0.0);
  }
  for (int k = lane; k < kdim; k += 32) s[lz::COEF + k] = (k < m) ? mine : 0.0;
}

// y = sum_j c[j] * X_j (y not read), j < k, c in device memory
__global__ void k_lincomb(const double* __restrict__ X, int64_t ldx, int k,
                          const double* __restrict__ c, double* __restrict__ y, int64_t n) {
  grid_entry();
  double cc[MAXK];
#pragma unroll
  for (int j = 0; j < MAXK; ++j) cc[j] = j < k ? c[j] : 0.0;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    double v = cc[0] * X[i];
#pragma unroll
    for (int j = 1; j < MAXK; ++j)
      if (j < k) v += cc[j] * X[j * ldx + i];
    y[i] = v;
  }
}

// The context's partial array holds MAXK rows of RED_BLOCKS partials followed by one unsigned
// counter for the last-block reductions.
unsigned* reduction_counter(double* partial) {
  return reinterpret_cast<unsigned*>(partial + MAXK * RED_BLOCKS);
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
  launch_k(k_mix, grid, 256, 0, s, in, out, tasks, ntasks, terms, total_tiles);
  count_launch();
}

void launch_copy(cudaStream_t s, const double* src, double* dst, const CopyTask* tasks,
                 int ntasks, int total_tiles) {
  if (total_tiles <= 0) return;
  int grid = total_tiles < 4096 ? total_tiles : 4096;
  launch_k(k_copy, grid, 256, 0, s, src, dst, tasks, ntasks, total_tiles);
  count_launch();
}

void launch_mdot(cudaStream_t s, const double* X, int64_t ldx, int k, const double* y, int64_t n,
                 double* partial, double* out) {
  launch_k(k_mdot_partial, RED_BLOCKS, RED_THREADS, 0, s, X, ldx, k, y, n, partial, out,
           reduction_counter(partial));
  count_launch();
}

void launch_axpby(cudaStream_t s, int64_t n, double a, const double* ap, double asign,
                  const double* x, double b, const double* bp, double bsign, double* y,
                  int b_recip) {
  if (n <= 0) return;
  launch_k(k_axpby, grid_for(n), RED_THREADS, 0, s, n, a, ap, asign, x, b, bp, bsign, y, b_recip);
  count_launch();
}

void launch_msub(cudaStream_t s, const double* X, int64_t ldx, int k, const double* c, double* y,
                 int64_t n) {
  if (n <= 0 || k <= 0) return;
  launch_k(k_msub, grid_for(n), RED_THREADS, 0, s, X, ldx, k, c, y, n);
  count_launch();
}

void launch_scale(cudaStream_t s, double* x, int64_t n, double a) {
  if (n <= 0) return;
  launch_k(k_scale, grid_for(n), RED_THREADS, 0, s, x, n, a);
  count_launch();
}

void launch_scale_rsqrt(cudaStream_t s, double* x, int64_t n, const double* nrm2) {
  if (n <= 0) return;
  launch_k(k_scale_rsqrt, grid_for(n), RED_THREADS, 0, s, x, n, nrm2);
  count_launch();
}

void launch_dot2(cudaStream_t s, const double* x, const double* y, int64_t n, double* partial,
                 double* out) {
  launch_k(k_dot2_partial, RED_BLOCKS, RED_THREADS, 0, s, x, y, n, partial, out,
           reduction_counter(partial));
  count_launch();
}

void launch_lanczos2_orth(cudaStream_t s, double* K, double* H, int64_t n, double* scal,
                          double* partial) {
  launch_k(k_lanczos2_orth, RED_BLOCKS, RED_THREADS, 0, s, K, H, n, scal, partial,
           reduction_counter(partial));
  count_launch();
}

void launch_pair_dot(cudaStream_t s, const double* X, const double* Y, const PairTask* tasks,
                     int ntasks, int64_t total, double* partial, double* out) {
  if (ntasks <= 0 || total <= 0) {
    cudaMemsetAsync(out, 0, sizeof(double), s);
    return;
  }
  const int grid = int(std::min<int64_t>(RED_BLOCKS, (total + RED_THREADS - 1) / RED_THREADS));
  launch_k(k_pair_dot, grid, RED_THREADS, 0, s, X, Y, tasks, ntasks, total, partial, out,
           reduction_counter(partial));
  count_launch();
}

void launch_pair_dot_rows(cudaStream_t s, const double* X, int64_t x_stride, const double* Y,
                          const PairTask* tasks, int ntasks, int nrows, double* out,
                          int64_t out_stride) {
  if (nrows <= 0) return;
  launch_k(k_pair_dot_rows, nrows, RED_THREADS, 0, s, X, x_stride, Y, tasks, ntasks, out,
           out_stride);
  count_launch();
}

void launch_next_vector(cudaStream_t s, const double* H, double* Kn, int64_t n, double* scal,
                        int j, double betatest) {
  launch_k(k_next_vector, grid_for(n), RED_THREADS, 0, s, H, Kn, n, scal, j, betatest);
  count_launch();
}

void launch_ritz(cudaStream_t s, double* scal, int kdim, double tau, bool expo) {
  launch_k(k_ritz, 1, 32, 0, s, scal, kdim, tau, expo ? 1 : 0);
  count_launch();
}

void launch_lincomb(cudaStream_t s, const double* X, int64_t ldx, int k, const double* c,
                    double* y, int64_t n) {
  if (n <= 0 || k <= 0) return;
  launch_k(k_lincomb, grid_for(n), RED_THREADS, 0, s, X, ldx, k, c, y, n);
  count_launch();
}

void launch_zero(cudaStream_t s, double* x, int64_t n) {
  if (n <= 0) return;
  cudaMemsetAsync(x, 0, size_t(n) * sizeof(double), s);
}

// Descriptor upload carried by the launch itself: the bytes travel as the kernel's parameter
// block (up to 32 KB of parameters on sm_70 and later), and the kernel writes them to the
// descriptor slot. Unlike a host-to-device copy this needs no copy engine between two kernels
// and chains with them through programmatic dependent launch.
template <int N>
struct ParamBlob {
  uint4 v[N / 16];
};

template <int N>
__global__ void __launch_bounds__(256) k_upload(const __grid_constant__ ParamBlob<N> blob,
                                                uint4* __restrict__ dst, int nvec) {
  grid_entry();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nvec) dst[i] = blob.v[i];
}

template <int N>
void upload_blob(cudaStream_t s, const void* src, size_t bytes, void* dst) {
  ParamBlob<N> b;
  const int nvec = int((bytes + 15) / 16);
  b.v[nvec - 1] = make_uint4(0u, 0u, 0u, 0u);
  std::memcpy(b.v, src, bytes);
  launch_k(k_upload<N>, (nvec + 255) / 256, 256, 0, s, b, reinterpret_cast<uint4*>(dst), nvec);
  count_launch();
}

// The reverse direction for the few words the host reads back each bond step (the energy, the
// status words, the density-matrix eigenvalues): a kernel stores them straight into pinned host
// memory through its device address, so the transfer chains with the kernels before it instead
// of waiting for a copy engine. Stream synchronisation makes the stores visible to the host.
__global__ void __launch_bounds__(256) k_to_host(const uint32_t* __restrict__ src,
                                                 uint32_t* __restrict__ dst, int64_t nwords) {
  grid_entry();
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nwords; i += stride)
    dst[i] = src[i];
}

void launch_to_host(cudaStream_t s, const void* src, void* dst_view, size_t bytes) {
  const int64_t nwords = int64_t(bytes / 4);
  if (nwords <= 0) return;
  const int grid = int(std::min<int64_t>((nwords + 255) / 256, 64));
  launch_k(k_to_host, grid, 256, 0, s, reinterpret_cast<const uint32_t*>(src),
           reinterpret_cast<uint32_t*>(dst_view), nwords);
  count_launch();
}

bool launch_upload(cudaStream_t s, const void* src, size_t bytes, void* dst) {
  if (bytes == 0 || bytes > size_t(UPLOAD_PARAM_MAX) || (reinterpret_cast<uintptr_t>(dst) & 15))
    return false;
  if (bytes <= 2048) upload_blob<2048>(s, src, bytes, dst);
  else if (bytes <= 8192) upload_blob<8192>(s, src, bytes, dst);
  else upload_blob<UPLOAD_PARAM_MAX>(s, src, bytes, dst);
  return true;
}

}  // namespace dmrg
