// jacobi.cu -- batched FP64 two-sided cyclic Jacobi eigensolver for the QN blocks of the
// two-site reduced density matrix (the rho form of the truncation, algs/DMRG.jl:425-467).
//
// One CTA per block. Each sweep visits all n(n-1)/2 pivots in n-1 rounds of n/2 disjoint
// rotations (round-robin ordering), so a round is a fully parallel rotate-rows / rotate-columns
// pass. Small blocks live in shared memory; larger ones are rotated in place in global memory.
// Pivots are skipped when |a_pq| <= 1e-15*sqrt(|a_pp a_qq|) or |a_pq| <= 1e-15*||A||_F: the
// absolute floor is needed for rank-deficient density matrices, whose null-space entries are
// rounding noise that no rotation removes. The sweep loop stops
// after a sweep without rotations. Eigenvalues are returned descending, ties by index, and the
// matching eigenvectors overwrite the input matrix column by column.
#include "kernels.cuh"
#include "launch.cuh"

namespace dmrg {
namespace {

constexpr int JAC_THREADS = 512;
constexpr int JAC_MAX_SWEEPS = 40;

__global__ void __launch_bounds__(JAC_THREADS)
k_jacobi(double* __restrict__ base, const EigTask* __restrict__ tasks, int in_smem,
         int* status) {
  grid_entry();
  const EigTask tk = tasks[blockIdx.x];
  const int n = tk.n;
  if (n <= 0) return;
  const int nn = n + (n & 1), npairs = nn / 2, rounds = nn - 1;
  extern __shared__ double sm[];
  double* lam = sm;                                    // n
  double* cs = lam + nn;                               // npairs
  double* sn = cs + npairs;                            // npairs
  int* pp = reinterpret_cast<int*>(sn + npairs);       // npairs
  int* qq = pp + npairs;                               // npairs
  int* rank = qq + npairs;                             // nn
  double* tail = reinterpret_cast<double*>(rank + nn + (nn & 1));
  double* Ag = base + tk.a_off;
  double* A = in_smem ? tail : Ag;
  double* V = in_smem ? tail + int64_t(n) * n : base + tk.v_off;
  __shared__ int rotated;
  __shared__ double floor_abs;
  const int tid = threadIdx.x;

  for (int64_t e = tid; e < int64_t(n) * n; e += blockDim.x) {
    if (in_smem) A[e] = Ag[e];
    const int i = int(e % n), j = int(e / n);
    V[e] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  {   // absolute floor: 1e-15 * ||A||_F (off-diagonal rounding noise cannot go much lower)
    __shared__ double red[JAC_THREADS / 32];
    double f = 0.0;
    for (int64_t e = tid; e < int64_t(n) * n; e += blockDim.x) f += A[e] * A[e];
    for (int o = 16; o > 0; o >>= 1) f += __shfl_xor_sync(0xffffffffu, f, o);
    if ((tid & 31) == 0) red[tid >> 5] = f;
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
      for (int w = 0; w < int(blockDim.x / 32); ++w) t += red[w];
      floor_abs = 1e-15 * sqrt(t);
    }
  }
  __syncthreads();

  int sweep = 0;
  for (; sweep < JAC_MAX_SWEEPS; ++sweep) {
    if (tid == 0) rotated = 0;
    __syncthreads();
    for (int r = 0; r < rounds; ++r) {
      for (int k = tid; k < npairs; k += blockDim.x) {
        const int i0 = (k == 0) ? 0 : ((k - 1 + r) % (nn - 1)) + 1;
        const int i1 = ((nn - 1 - k - 1 + r) % (nn - 1)) + 1;
        const int p = min(i0, i1), q = max(i0, i1);
        double c = 1.0, s = 0.0;
        if (q < n) {
          const double apq = A[p + int64_t(q) * n];
          const double app = A[p + int64_t(p) * n];
          const double aqq = A[q + int64_t(q) * n];
          if (fabs(apq) > floor_abs && fabs(apq) > 1e-15 * sqrt(fabs(app) * fabs(aqq))) {
            const double theta = (aqq - app) / (2.0 * apq);
            const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            c = 1.0 / sqrt(t * t + 1.0);
            s = t * c;
            rotated = 1;
          }
        }
        pp[k] = p;
        qq[k] = (q < n) ? q : -1;
        cs[k] = c;
        sn[k] = s;
      }
      __syncthreads();
      // rows p, q  <-  J^T A : warp w owns pairs w, w+nwarps, ..; lanes walk the columns
      const int lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
      for (int k = warp; k < npairs; k += nwarps) {
        const int q = qq[k];
        const double s = sn[k];
        if (q < 0 || s == 0.0) continue;
        const int p = pp[k];
        const double c = cs[k];
        for (int j = lane; j < n; j += 32) {
          const double ap = A[p + j * n], aq = A[q + j * n];
          A[p + j * n] = c * ap - s * aq;
          A[q + j * n] = s * ap + c * aq;
        }
      }
      __syncthreads();
      // columns p, q  <-  A J, V J : lanes walk the (contiguous) rows
      for (int k = warp; k < npairs; k += nwarps) {
        const int q = qq[k];
        const double s = sn[k];
        if (q < 0 || s == 0.0) continue;
        const int p = pp[k];
        const double c = cs[k];
        double* Ap_ = A + p * n;
        double* Aq_ = A + q * n;
        double* Vp_ = V + p * n;
        double* Vq_ = V + q * n;
        for (int i = lane; i < n; i += 32) {
          const double ap = Ap_[i], aq = Aq_[i];
          Ap_[i] = c * ap - s * aq;
          Aq_[i] = s * ap + c * aq;
          const double vp = Vp_[i], vq = Vq_[i];
          Vp_[i] = c * vp - s * vq;
          Vq_[i] = s * vp + c * vq;
        }
      }
      __syncthreads();
    }
    if (!rotated) break;
    __syncthreads();
  }
  if (tid == 0 && sweep >= JAC_MAX_SWEEPS && status) atomicAdd(status, 1);

  for (int i = tid; i < n; i += blockDim.x) lam[i] = A[i + int64_t(i) * n];
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
  double* W = base + tk.w_off;
  for (int i = tid; i < n; i += blockDim.x) W[rank[i]] = lam[i];
  // sorted eigenvectors overwrite the input matrix (A is no longer needed)
  if (in_smem) {
    for (int64_t e = tid; e < int64_t(n) * n; e += blockDim.x) {
      const int i = int(e % n), j = int(e / n);
      Ag[i + int64_t(rank[j]) * n] = V[e];
    }
  } else {
    for (int64_t e = tid; e < int64_t(n) * n; e += blockDim.x) {
      const int i = int(e % n), j = int(e / n);
      Ag[i + int64_t(rank[j]) * n] = V[e];
    }
  }
}

size_t jacobi_smem(int n, bool in_smem) {
  const int nn = n + (n & 1), npairs = nn / 2;
  size_t b = sizeof(double) * (nn + 2 * npairs) + sizeof(int) * (2 * npairs + nn + (nn & 1));
  b = (b + 15) / 16 * 16;
  if (in_smem) b += sizeof(double) * 2 * size_t(n) * n;
  return b;
}

}  // namespace

// Host: tasks with n <= 100 run from shared memory, the rest in place in global memory.
void launch_jacobi(cudaStream_t s, double* base, const EigTask* tasks, int ntasks, int max_n,
                   int* status) {
  if (ntasks <= 0) return;
  const bool small = max_n <= 100;
  const size_t smem = jacobi_smem(max_n, small);
  raise_smem_limit(reinterpret_cast<const void*>(k_jacobi), smem);
  launch_k(k_jacobi, ntasks, JAC_THREADS, smem, s, base, tasks, small ? 1 : 0, status);
  count_launch();
}

}  // namespace dmrg
