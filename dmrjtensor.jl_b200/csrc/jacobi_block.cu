// jacobi_block.cu -- block two-sided Jacobi for the large QN blocks of the reduced density
// matrix (n > 100), all blocks of one truncation batched into the same launches.
//
// The matrix is padded to N = nb*16 (nb even) with zero rows/columns (exactly decoupled: their
// entries stay zero, so they never rotate). A sweep runs nb-1 rounds of the round-robin
// tournament over the nb column blocks; in a round the nb/2 disjoint block pairs (I,J) are:
//   1. solved: the 32x32 pivot matrix [[A_II A_IJ];[A_JI A_JJ]] is diagonalised in shared memory
//      by cyclic Jacobi, giving an orthogonal Q_P for pair P;
//   2. applied: every 32x32 tile A[P,Q] <- Q_P^T A[P,Q] Q_Q and every V[rows,P] <- V[rows,P] Q_P,
//      one CTA per tile (the tiles of a round are independent).
// Sweeps stop when the off-diagonal norm of every matrix is below 1e-12 ||A||_F. The skip rule inside the pivot solves is
// |a_pq| <= 1e-15 sqrt(|a_pp a_qq|), or below the larger of 1e-15 ||A||_F and 1e-14 ||S||_F,
// the rounding level of the pivot matrix S's own rotations.
#include "kernels.cuh"
#include "launch.cuh"

namespace dmrg {
namespace {

constexpr int B = 16, P2 = 2 * B;  // column blocks of 16: 32 x 32 pivot matrices
constexpr int SOLVE_THREADS = 256, UPD_THREADS = (P2 / 4) * (P2 / 4);
constexpr int INNER_MAX = 4;     // pivots need not be exact: the outer sweeps converge anyway
constexpr int LDS = P2 + 1;   // padded shared leading dimension (odd: conflict-free columns)

__device__ __forceinline__ void pair_blocks(int k, int r, int nb, int& I, int& J) {
  I = (k == 0) ? 0 : ((k - 1 + r) % (nb - 1)) + 1;
  J = ((nb - 1 - k - 1 + r) % (nb - 1)) + 1;
}

// global index of local row x (0..P2-1) of pair (I,J)
__device__ __forceinline__ int64_t pidx(int x, int I, int J) {
  return x < B ? int64_t(I) * B + x : int64_t(J) * B + (x - B);
}

__global__ void k_bj_init(double* __restrict__ base, const BlockEigGroup* __restrict__ g, int ng) {
  grid_entry();
  const BlockEigGroup gr = g[blockIdx.y];
  const int64_t NN = int64_t(gr.N) * gr.N;
  for (int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < NN;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int i = int(e % gr.N), j = int(e / gr.N);
    base[gr.ap_off + e] = (i < gr.n && j < gr.n) ? base[gr.a_off + i + int64_t(j) * gr.n] : 0.0;
    base[gr.vp_off + e] = (i == j) ? 1.0 : 0.0;
  }
}

__global__ void k_bj_norm(double* __restrict__ base, const BlockEigGroup* __restrict__ g,
                          double* __restrict__ floor_out) {
  grid_entry();
  const BlockEigGroup gr = g[blockIdx.x];
  double f = 0.0;
  const int64_t nn = int64_t(gr.n) * gr.n;
  for (int64_t e = threadIdx.x; e < nn; e += blockDim.x) {
    const double v = base[gr.a_off + e];
    f += v * v;
  }
  for (int o = 16; o > 0; o >>= 1) f += __shfl_xor_sync(0xffffffffu, f, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = f;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < int(blockDim.x / 32); ++w) t += red[w];
    floor_out[blockIdx.x] = 1e-15 * sqrt(t);
  }
}

// One CTA per (group, pair) of round r.
__global__ void __launch_bounds__(SOLVE_THREADS)
k_bj_solve(double* __restrict__ base, const BlockEigGroup* __restrict__ g,
           const int2* __restrict__ pairs, int npairs, int r, const double* __restrict__ floors,
           int* __restrict__ flags) {
  grid_entry();
  const int2 pk = pairs[blockIdx.x];
  const BlockEigGroup gr = g[pk.x];
  const int nb = gr.N / B;
  if (r >= nb - 1) return;
  int I, J;
  pair_blocks(pk.y, r, nb, I, J);
  extern __shared__ double smem_solve[];
  double* S = smem_solve;             // 64 x 65
  double* Vs = smem_solve + P2 * LDS;  // 64 x 65
  __shared__ double cs[P2 / 2], sn[P2 / 2];
  __shared__ int pp[P2 / 2], qq[P2 / 2];
  __shared__ int rotated, any;
  const int tid = threadIdx.x;
  const double* Ap = base + gr.ap_off;
  for (int e = tid; e < P2 * P2; e += blockDim.x) {
    const int x = e % P2, y = e / P2;
    S[x + y * LDS] = Ap[pidx(x, I, J) + pidx(y, I, J) * gr.N];
    Vs[x + y * LDS] = (x == y) ? 1.0 : 0.0;
  }
  if (tid == 0) any = 0;
  __shared__ double red[SOLVE_THREADS / 32];
  __shared__ double floor_abs;
  {   // pivot-local floor: 1e-14 ||S||_F (the rounding level of the pivot's own rotations)
    double f = 0.0;
    for (int e = tid; e < P2 * P2; e += blockDim.x) {
      const double v = S[(e % P2) + (e / P2) * LDS];
      f += v * v;
    }
    for (int o = 16; o > 0; o >>= 1) f += __shfl_xor_sync(0xffffffffu, f, o);
    if ((tid & 31) == 0) red[tid >> 5] = f;
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
      for (int w = 0; w < SOLVE_THREADS / 32; ++w) t += red[w];
      floor_abs = fmax(1e-14 * sqrt(t), floors[pk.x]);
    }
    __syncthreads();
  }
  for (int sweep = 0; sweep < INNER_MAX; ++sweep) {
    if (tid == 0) rotated = 0;
    __syncthreads();
    for (int rr = 0; rr < P2 - 1; ++rr) {
      if (tid < P2 / 2) {
        const int k = tid;
        const int i0 = (k == 0) ? 0 : ((k - 1 + rr) % (P2 - 1)) + 1;
        const int i1 = ((P2 - 1 - k - 1 + rr) % (P2 - 1)) + 1;
        const int p = min(i0, i1), q = max(i0, i1);
        const double apq = S[p + q * LDS], app = S[p + p * LDS], aqq = S[q + q * LDS];
        double c = 1.0, s = 0.0;
        if (fabs(apq) > floor_abs && fabs(apq) > 1e-15 * sqrt(fabs(app) * fabs(aqq))) {
          const double theta = (aqq - app) / (2.0 * apq);
          const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
          c = 1.0 / sqrt(t * t + 1.0);
          s = t * c;
          rotated = 1;
        }
        pp[k] = p; qq[k] = q; cs[k] = c; sn[k] = s;
      }
      __syncthreads();
      for (int it = tid; it < (P2 / 2) * P2; it += blockDim.x) {   // rows
        const int k = it / P2, j = it % P2;
        const double s = sn[k];
        if (s == 0.0) continue;
        const int p = pp[k], q = qq[k];
        const double c = cs[k];
        const double ap = S[p + j * LDS], aq = S[q + j * LDS];
        S[p + j * LDS] = c * ap - s * aq;
        S[q + j * LDS] = s * ap + c * aq;
      }
      __syncthreads();
      for (int it = tid; it < (P2 / 2) * P2; it += blockDim.x) {   // columns
        const int k = it / P2, i = it % P2;
        const double s = sn[k];
        if (s == 0.0) continue;
        const int p = pp[k], q = qq[k];
        const double c = cs[k];
        const double ap = S[i + p * LDS], aq = S[i + q * LDS];
        S[i + p * LDS] = c * ap - s * aq;
        S[i + q * LDS] = s * ap + c * aq;
        const double vp = Vs[i + p * LDS], vq = Vs[i + q * LDS];
        Vs[i + p * LDS] = c * vp - s * vq;
        Vs[i + q * LDS] = s * vp + c * vq;
      }
      __syncthreads();
    }
    if (!rotated) break;
    if (tid == 0) any = 1;
    __syncthreads();
  }
  double* Q = base + gr.q_off + int64_t(pk.y) * P2 * P2;
  for (int e = tid; e < P2 * P2; e += blockDim.x) Q[e] = Vs[(e % P2) + (e / P2) * LDS];
  if (tid == 0 && any) flags[pk.x] = 1;
}

// One CTA per tile of round r. Tile list entries: (group, kind, a, b):
//   kind 0: A tile (P=a, Q=b);  kind 1: V tile (row chunk a of P2 rows, pair b).
__global__ void __launch_bounds__(UPD_THREADS)
k_bj_update(double* __restrict__ base, const BlockEigGroup* __restrict__ g,
            const int4* __restrict__ tiles, int r) {
  grid_entry();
  const int4 tl = tiles[blockIdx.x];
  const BlockEigGroup gr = g[tl.x];
  const int nb = gr.N / B;
  if (r >= nb - 1) return;
  extern __shared__ double sm[];
  double* X = sm;               // input tile
  double* Qs = X + P2 * LDS;    // right factor
  double* T = Qs + P2 * LDS;    // intermediate
  const int tid = threadIdx.x;
  const int tr = (tid % (P2 / 4)) * 4, tc = (tid / (P2 / 4)) * 4;   // this thread's 4x4 patch
  double* Ap = base + gr.ap_off;
  double* Vp = base + gr.vp_off;
  const double* Qb = base + gr.q_off;
  if (tl.y == 0) {
    int IP, JP, IQ, JQ;
    pair_blocks(tl.z, r, nb, IP, JP);
    pair_blocks(tl.w, r, nb, IQ, JQ);
    const double* QQ = Qb + int64_t(tl.w) * P2 * P2;
    for (int e = tid; e < P2 * P2; e += blockDim.x) {
      const int x = e % P2, y = e / P2;
      X[x + y * LDS] = Ap[pidx(x, IP, JP) + pidx(y, IQ, JQ) * gr.N];
      Qs[x + y * LDS] = QQ[e];
    }
    __syncthreads();
    double acc[4][4] = {};
    for (int k = 0; k < P2; ++k) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = X[(tr + i) + k * LDS];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Qs[k + (tc + j) * LDS];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] += a[i] * b[j];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) T[(tr + i) + (tc + j) * LDS] = acc[i][j];
    __syncthreads();
    const double* QP = Qb + int64_t(tl.z) * P2 * P2;
    for (int e = tid; e < P2 * P2; e += blockDim.x) Qs[(e % P2) + (e / P2) * LDS] = QP[e];
    __syncthreads();
    double o[4][4] = {};
    for (int k = 0; k < P2; ++k) {   // out = QP^T T: out(i,j) = sum_k QP(k,i) T(k,j)
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = Qs[k + (tr + i) * LDS];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = T[k + (tc + j) * LDS];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) o[i][j] += a[i] * b[j];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
        Ap[pidx(tr + i, IP, JP) + pidx(tc + j, IQ, JQ) * gr.N] = o[i][j];
  } else {
    int IP, JP;
    pair_blocks(tl.w, r, nb, IP, JP);
    const int row0 = tl.z * P2;
    const double* QP = Qb + int64_t(tl.w) * P2 * P2;
    for (int e = tid; e < P2 * P2; e += blockDim.x) {
      const int x = e % P2, y = e / P2;
      X[x + y * LDS] = Vp[(row0 + x) + pidx(y, IP, JP) * gr.N];
      Qs[x + y * LDS] = QP[e];
    }
    __syncthreads();
    double acc[4][4] = {};
    for (int k = 0; k < P2; ++k) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = X[(tr + i) + k * LDS];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Qs[k + (tc + j) * LDS];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] += a[i] * b[j];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) Vp[(row0 + tr + i) + pidx(tc + j, IP, JP) * gr.N] = acc[i][j];
  }
}

// off-diagonal Frobenius norm of each padded matrix: flags[g] = 1 while off(A) > tol ||A||_F
__global__ void k_bj_offnorm(const double* __restrict__ base, const BlockEigGroup* __restrict__ g,
                             const double* __restrict__ floors, int* __restrict__ flags) {
  grid_entry();
  const BlockEigGroup gr = g[blockIdx.x];
  double f = 0.0;
  const int64_t NN = int64_t(gr.N) * gr.N;
  for (int64_t e = threadIdx.x; e < NN; e += blockDim.x) {
    const int i = int(e % gr.N), j = int(e / gr.N);
    if (i != j) {
      const double v = base[gr.ap_off + e];
      f += v * v;
    }
  }
  for (int o = 16; o > 0; o >>= 1) f += __shfl_xor_sync(0xffffffffu, f, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = f;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < int(blockDim.x / 32); ++w) t += red[w];
    // floors[g] = 1e-15 ||A||_F ; converged when off(A) <= 1e-12 ||A||_F
    flags[blockIdx.x] = sqrt(t) > 1e3 * floors[blockIdx.x] ? 1 : 0;   // off(A) > 1e-12 ||A||_F
  }
}

// Sorted eigenpairs of the converged padded problem back into the caller's layout.
__global__ void k_bj_finish(double* __restrict__ base, const BlockEigGroup* __restrict__ g) {
  grid_entry();
  const BlockEigGroup gr = g[blockIdx.x];
  extern __shared__ double lam[];
  int* rank = reinterpret_cast<int*>(lam + gr.n);
  const int n = gr.n, tid = threadIdx.x;
  for (int i = tid; i < n; i += blockDim.x) lam[i] = base[gr.ap_off + i + int64_t(i) * gr.N];
  __syncthreads();
  for (int i = tid; i < n; i += blockDim.x) {
    const double li = lam[i];
    int rk = 0;
    for (int j = 0; j < n; ++j) {
      const double lj = lam[j];
      rk += (lj > li) || (lj == li && j < i);
    }
    rank[i] = rk;
  }
  __syncthreads();
  for (int i = tid; i < n; i += blockDim.x) base[gr.w_off + rank[i]] = lam[i];
  for (int64_t e = tid; e < int64_t(n) * n; e += blockDim.x) {
    const int i = int(e % n), j = int(e / n);
    base[gr.a_off + i + int64_t(rank[j]) * n] = base[gr.vp_off + i + int64_t(j) * gr.N];
  }
}

constexpr size_t UPD_SMEM = 3 * P2 * LDS * sizeof(double);
constexpr size_t SOLVE_SMEM = 2 * P2 * LDS * sizeof(double);

}  // namespace

int block_eig_padded(int n) {
  int nb = (n + B - 1) / B;
  nb += nb & 1;
  return nb * B;
}

void launch_block_jacobi(cudaStream_t s, double* base, const BlockEigPlan& pl, int* flags_dev,
                         int* flags_host, double* floors_dev, int* sweeps_done) {
  const int ng = pl.ngroups;
  if (ng == 0) { if (sweeps_done) *sweeps_done = 0; return; }
  launch_k(k_bj_init, dim3(64, ng), 256, 0, s, base, pl.groups, ng);
  launch_k(k_bj_norm, ng, 512, 0, s, base, pl.groups, floors_dev);
  count_launch(2);
  raise_smem_limit(reinterpret_cast<const void*>(k_bj_update), UPD_SMEM);
  raise_smem_limit(reinterpret_cast<const void*>(k_bj_solve), SOLVE_SMEM);
  const int nbmax = pl.maxN / B;
  int sw = 0;
  for (; sw < pl.max_sweeps; ++sw) {
    cudaMemsetAsync(flags_dev, 0, sizeof(int) * ng, s);
    for (int r = 0; r < nbmax - 1; ++r) {
      launch_k(k_bj_solve, pl.npairs, SOLVE_THREADS, SOLVE_SMEM, s, base, pl.groups, pl.pairs,
               pl.npairs, r, floors_dev, flags_dev);
      launch_k(k_bj_update, pl.ntiles, UPD_THREADS, UPD_SMEM, s, base, pl.groups, pl.tiles, r);
      count_launch(2);
    }
    launch_k(k_bj_offnorm, ng, 512, 0, s, base, pl.groups, floors_dev, flags_dev);
    count_launch();
    cudaMemcpyAsync(flags_host, flags_dev, sizeof(int) * ng, cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    bool any = false;
    for (int i = 0; i < ng; ++i) any |= flags_host[i] != 0;
    if (!any) { ++sw; break; }
  }
  if (sweeps_done) *sweeps_done = sw;
  size_t fs = sizeof(double) * pl.maxn + sizeof(int) * pl.maxn;
  raise_smem_limit(reinterpret_cast<const void*>(k_bj_finish), fs);
  launch_k(k_bj_finish, ng, 512, fs, s, base, pl.groups);
  count_launch();
}

}  // namespace dmrg
