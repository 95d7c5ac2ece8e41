// hestenes.cu -- one-sided (Hestenes) Jacobi on the two-site matrix of each centre-charge group.
//
// For a group with matrix X (r x c, column-major) the kernel orthogonalises the c columns by
// plane rotations, X <- X J, V <- V J, until every pair satisfies
// |x_p . x_q| <= tol |x_p||x_q| with tol = max(1e-13, 4 sqrt(r) eps) (the threshold form of
// LAPACK's dgesvj, never below the rounding level of an r-term dot product) or
// |x_p . x_q| <= 1e-32 ||X||_F^2. Then X^T X = V diag(|x_i|^2) V^T: the columns of V are the
// eigenvectors of the reduced density matrix X^T X and |x_i|^2 its eigenvalues, and the rotated X
// is the other factor of the decomposition (X V). Used with X = M^T (sweep to the right: V gives
// the new left site tensor, X^T the D.V part) or X = M (sweep to the left: V^T is the new right
// site tensor, X the U.D part), so no density matrix is formed and the split is a copy.
//
// One CTA per group, X and V resident in shared memory; a warp owns a column pair per round (dot
// products with warp shuffles, rotation, update), so a round needs a single barrier. Columns are
// returned sorted by descending |x_i|^2 (ties by index).
#include "kernels.cuh"

namespace dmrg {
namespace {

constexpr int HJ_THREADS = 1024;   // one warp per column pair for c <= 64
constexpr int HJ_MAX_SWEEPS = 40;

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __launch_bounds__(HJ_THREADS)
k_hestenes(double* __restrict__ base, const SvdTask* __restrict__ tasks, int* status) {
  const SvdTask tk = tasks[blockIdx.x];
  const int r = tk.r, c = tk.c;
  if (c <= 0) return;
  extern __shared__ double sm[];
  double* X = sm;                         // r x c
  double* V = X + int64_t(r) * c;         // c x c
  double* nrm = V + int64_t(c) * c;       // c
  int* rank = reinterpret_cast<int*>(nrm + c);
  __shared__ int rotated;
  __shared__ double floor2;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  double* Xg = base + tk.x_off;
  for (int e = tid; e < r * c; e += blockDim.x) X[e] = Xg[e];
  for (int e = tid; e < c * c; e += blockDim.x) V[e] = ((e % c) == (e / c)) ? 1.0 : 0.0;
  __syncthreads();
  if (warp == 0) {
    double f = 0.0;
    for (int e = lane; e < r * c; e += 32) f += X[e] * X[e];
    f = wsum(f);
    if (lane == 0) floor2 = 1e-32 * f;
  }
  __syncthreads();
  const int cc = c + (c & 1), npairs = cc / 2, rounds = cc - 1;
  // orthogonality target: max(1e-13, 4 sqrt(r) eps). The kept state U U^T M is exact whatever the
  // target; it only moves the kept subspace at second order.
  const double tol = fmax(1e-13, 4.0 * sqrt(double(r)) * 1.1102230246251565e-16);
  const double tol2 = tol * tol;
  int sweep = 0;
  for (; sweep < HJ_MAX_SWEEPS; ++sweep) {
    if (tid == 0) rotated = 0;
    __syncthreads();
    for (int rr = 0; rr < rounds; ++rr) {
      for (int k = warp; k < npairs; k += nwarps) {
        const int i0 = (k == 0) ? 0 : ((k - 1 + rr) % (cc - 1)) + 1;
        const int i1 = ((cc - 1 - k - 1 + rr) % (cc - 1)) + 1;
        const int p = min(i0, i1), q = max(i0, i1);
        if (q >= c) continue;
        double* xp = X + p * r;
        double* xq = X + q * r;
        double a = 0.0, b = 0.0, g = 0.0;
        for (int i = lane; i < r; i += 32) {
          const double u = xp[i], v = xq[i];
          a += u * u;
          b += v * v;
          g += u * v;
        }
        a = wsum(a);
        b = wsum(b);
        g = wsum(g);
        if (g * g <= tol2 * (a * b) || fabs(g) <= floor2) continue;
        const double zeta = (b - a) / (2.0 * g);
        const double t = copysign(1.0, zeta) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double cs = rsqrt(1.0 + t * t), sn = cs * t;
        for (int i = lane; i < r; i += 32) {
          const double u = xp[i], v = xq[i];
          xp[i] = cs * u - sn * v;
          xq[i] = sn * u + cs * v;
        }
        double* vp = V + p * c;
        double* vq = V + q * c;
        for (int i = lane; i < c; i += 32) {
          const double u = vp[i], v = vq[i];
          vp[i] = cs * u - sn * v;
          vq[i] = sn * u + cs * v;
        }
        if (lane == 0) rotated = 1;
      }
      __syncthreads();
    }
    if (!rotated) break;
    __syncthreads();
  }
  if (tid == 0 && status) {
    if (sweep >= HJ_MAX_SWEEPS) atomicAdd(status, 1);
    atomicMax(status + 1, sweep + 1);   // sweeps used (diagnostics)
  }
  for (int k = warp; k < c; k += nwarps) {
    double a = 0.0;
    for (int i = lane; i < r; i += 32) a += X[k * r + i] * X[k * r + i];
    a = wsum(a);
    if (lane == 0) nrm[k] = a;
  }
  __syncthreads();
  for (int i = tid; i < c; i += blockDim.x) {
    const double li = nrm[i];
    int rk = 0;
    for (int j = 0; j < c; ++j) rk += (nrm[j] > li) || (nrm[j] == li && j < i);
    rank[i] = rk;
  }
  __syncthreads();
  double* W = base + tk.w_off;
  double* Vg = base + tk.v_off;
  for (int i = tid; i < c; i += blockDim.x) W[rank[i]] = nrm[i];
  for (int e = tid; e < c * c; e += blockDim.x) Vg[(e % c) + int64_t(rank[e / c]) * c] = V[e];
  for (int e = tid; e < r * c; e += blockDim.x) Xg[(e % r) + int64_t(rank[e / r]) * r] = X[e];
}

}  // namespace

size_t hestenes_smem(int r, int c) {
  return sizeof(double) * (size_t(r) * c + size_t(c) * c + c) + sizeof(int) * size_t(c) + 16;
}

void launch_hestenes(cudaStream_t s, double* base, const SvdTask* tasks, int ntasks,
                     size_t smem, int* status) {
  if (ntasks <= 0) return;
  raise_smem_limit(reinterpret_cast<const void*>(k_hestenes), smem);
  k_hestenes<<<ntasks, HJ_THREADS, smem, s>>>(base, tasks, status);
  count_launch();
}

}  // namespace dmrg
