// syevt.cu -- density-matrix eigensolver for blocks up to SYEVT_NMAX: Householder
// tridiagonalisation, bisection, inverse iteration, re-orthogonalisation, back-transformation.
//
// Launch 1 (k_trid_eigvals), one CTA per block, matrix in shared memory:
//   * A = Q T Q^T by n-2 Householder reflectors (lower form, LAPACK dsytd2 order); the reflector
//     vectors are written into the strictly lower part of the caller's matrix, d/e/tau into a
//     small per-block workspace;
//   * all eigenvalues of T by bisection to an absolute width of 4 eps ||T|| (one thread per
//     eigenvalue), with a division-free Sturm count (see sturm_below).
// The host then truncates globally and asks for the top-k vectors of each block.
// Launch 2 (k_trid_vectors), one CTA per block:
//   * eigenvectors of T by inverse iteration on (T - lambda I) with partial-pivoting LU (three
//     iterations from a fixed pseudo-random start). Eigenvalues closer than 1e-10 ||T|| form a
//     cluster whose members are re-orthogonalised against each other at every iteration; kept
//     eigenvalues below 1e-13 ||T|| (numerically zero) get an orthonormal completion instead;
//   * two passes of classical Gram-Schmidt over the k vectors (largest eigenvalue first);
//   * back-transformation U = Q Z with the stored reflectors.
#include "kernels.cuh"

namespace dmrg {
namespace {

constexpr int TE_THREADS = 256;

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// block-wide sum; red has >= 32 entries; all threads get the result
__device__ double bsum(double v, double* red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = wsum(v);
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  const int nw = blockDim.x >> 5;
  for (int i = 0; i < nw; ++i) t += red[i];
  return t;
}

// Number of eigenvalues of T(d,e) strictly below x: sign changes of the leading minors
// D_j = (d_j - x) D_{j-1} - e_{j-1}^2 D_{j-2}. Only one FMA per step sits on the dependent chain
// (the products with the previous minor and d_j - x are off it); an exact zero minor counts with
// the sign opposite to its predecessor; every 8 steps the pair is renormalised by a power of two.
__device__ int sturm_below(const double* d, const double* e2, int n, double x) {
  double Dm1 = 1.0, D = d[0] - x;
  int c = (D < 0) ? 1 : 0;
  bool neg = D < 0;
  for (int j = 1; j < n; ++j) {
    const double Dn = fma(d[j] - x, D, -e2[j - 1] * Dm1);
    const bool ng = (Dn == 0.0) ? !neg : (Dn < 0);
    c += (ng != neg) ? 1 : 0;
    neg = ng;
    Dm1 = D;
    D = Dn;
    if ((j & 7) == 0) {
      const double mx = fmax(fabs(D), fabs(Dm1));
      const int ex = (mx > 0.0) ? ilogb(mx) : 0;
      D = scalbn(D, -ex);
      Dm1 = scalbn(Dm1, -ex);
    }
  }
  return c;
}

__global__ void __launch_bounds__(TE_THREADS)
k_trid_eigvals(double* __restrict__ base, const TridTask* __restrict__ tasks) {
  const TridTask tk = tasks[blockIdx.x];
  const int n = tk.n;
  if (n <= 0) return;
  extern __shared__ double sm[];
  double* A = sm;               // n x n
  double* v = A + n * n;        // n
  double* p = v + n;            // n
  double* d = p + n;            // n
  double* e = d + n;            // n
  double* e2 = e + n;           // n
  double* tau = e2 + n;         // n
  __shared__ double red[32];
  __shared__ double s_tau, s_scale, s_beta, s_K;
  const int tid = threadIdx.x;
  double* Ag = base + tk.a_off;
  for (int x = tid; x < n * n; x += blockDim.x) A[x] = Ag[x];
  __syncthreads();
  for (int k = 0; k + 2 < n; ++k) {
    const int m = n - k - 1;              // length of x = A[k+1:n, k]
    const double* col = A + k * n + k + 1;
    double part = 0.0;
    for (int i = 1 + tid; i < m; i += blockDim.x) part += col[i] * col[i];
    const double xn2 = bsum(part, red);
    if (tid == 0) {
      const double alpha = col[0];
      if (xn2 == 0.0) {
        s_tau = 0.0; s_beta = alpha; s_scale = 0.0;
      } else {
        const double beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
        s_tau = (beta - alpha) / beta;
        s_scale = 1.0 / (alpha - beta);
        s_beta = beta;
      }
      e[k] = s_beta;
      tau[k] = s_tau;
      d[k] = A[k + k * n];
    }
    __syncthreads();
    const double t = s_tau, sc = s_scale;
    for (int i = tid; i < m; i += blockDim.x) v[i] = (i == 0) ? 1.0 : col[i] * sc;
    __syncthreads();
    if (t != 0.0) {
      // p = t * B v, B = A[k+1:, k+1:] symmetric: p_i = sum_j B[j,i] v_j (contiguous column),
      // 8 lanes per column so that 32 columns reduce in parallel
      {
        const int g8 = tid >> 3, l8 = tid & 7, ng8 = blockDim.x >> 3;
        for (int ib = 0; ib < m; ib += ng8) {     // uniform trip count: shuffles stay convergent
          const int i = ib + g8;
          double s = 0.0;
          if (i < m) {
            const double* colB = A + (k + 1 + i) * n + (k + 1);
            for (int j = l8; j < m; j += 8) s += colB[j] * v[j];
          }
          s += __shfl_xor_sync(0xffffffffu, s, 4, 8);
          s += __shfl_xor_sync(0xffffffffu, s, 2, 8);
          s += __shfl_xor_sync(0xffffffffu, s, 1, 8);
          if (i < m && l8 == 0) p[i] = t * s;
        }
      }
      __syncthreads();
      double kp = 0.0;
      for (int i = tid; i < m; i += blockDim.x) kp += p[i] * v[i];
      const double K = bsum(kp, red);
      if (tid == 0) s_K = 0.5 * t * K;
      __syncthreads();
      const double hk = s_K;
      for (int i = tid; i < m; i += blockDim.x) p[i] -= hk * v[i];   // p becomes w
      __syncthreads();
      {
        const int lane = tid & 31, wp = tid >> 5, nw = blockDim.x >> 5;
        for (int j = wp; j < m; j += nw) {
          double* colB = A + (k + 1 + j) * n + (k + 1);
          const double vj = v[j], pj = p[j];
          for (int i = lane; i < m; i += 32) colB[i] -= v[i] * pj + p[i] * vj;
        }
      }
      __syncthreads();
    }
    // keep the reflector (v[1:]) in the now-unused column below the subdiagonal
    for (int i = 1 + tid; i < m; i += blockDim.x) A[k * n + k + 1 + i] = v[i];
    __syncthreads();
  }
  if (tid == 0) {
    if (n >= 2) {
      d[n - 2] = A[(n - 2) + (n - 2) * n];
      e[n - 2] = A[(n - 1) + (n - 2) * n];
      tau[n - 2] = 0.0;
    }
    d[n - 1] = A[(n - 1) + (n - 1) * n];
    e[n - 1] = 0.0;
    tau[n - 1] = 0.0;
  }
  __syncthreads();
  for (int i = tid; i < n; i += blockDim.x) e2[i] = e[i] * e[i];
  for (int x = tid; x < n * n; x += blockDim.x) Ag[x] = A[x];
  double* ws = base + tk.ws_off;          // d | e | tau
  for (int i = tid; i < n; i += blockDim.x) {
    ws[i] = d[i];
    ws[n + i] = e[i];
    ws[2 * n + i] = tau[i];
  }
  __syncthreads();
  // Gershgorin interval
  __shared__ double s_lo, s_hi;
  if (tid == 0) {
    double lo = 1e300, hi = -1e300;
    for (int i = 0; i < n; ++i) {
      const double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i + 1 < n ? fabs(e[i]) : 0.0);
      lo = fmin(lo, d[i] - r);
      hi = fmax(hi, d[i] + r);
    }
    const double pad = 2.2e-16 * fmax(fabs(lo), fabs(hi)) + 1e-300;
    s_lo = lo - pad;
    s_hi = hi + pad;
  }
  __syncthreads();
  const double tn = fmax(fabs(s_lo), fabs(s_hi));
  double* W = base + tk.w_off;
  for (int i = tid; i < n; i += blockDim.x) {       // i-th largest = (n-1-i)-th smallest
    const int target = n - 1 - i;
    double a = s_lo, b = s_hi;
    for (int it = 0; it < 128; ++it) {
      const double mid = 0.5 * (a + b);
      if (b - a <= 8.9e-16 * tn || mid == a || mid == b) break;   // converged / no progress
      if (sturm_below(d, e2, n, mid) > target) b = mid; else a = mid;
    }
    W[i] = 0.5 * (a + b);
  }
}

// pseudo-random start vector entry (fixed: results are reproducible)
__device__ __forceinline__ double prand(int i, int j) {
  unsigned h = unsigned(i) * 2654435761u ^ (unsigned(j) * 40503u + 0x9e3779b9u);
  h ^= h >> 15; h *= 2246822519u; h ^= h >> 13; h *= 3266489917u; h ^= h >> 16;
  return (double(h) / 4294967296.0) - 0.5;
}

// One thread: z <- (T - lam I)^{-1} z three times with re-orthogonalisation against Zc columns
// [c0, col) (a cluster), using partial-pivoting LU held in local arrays.
__device__ void inverse_iteration(const double* d, const double* e, int n, double lam,
                                  double* Z, int col, int c0, double tn) {
  constexpr int NM = SYEVT_NMAX;
  double u0[NM], u1[NM], u2[NM], l[NM];
  int piv[NM];
  // factor (T - lam I) = P L U with U having two superdiagonals
  double pert = 2.2e-16 * tn;
  double dk = d[0] - lam, ek = n > 1 ? e[0] : 0.0;
  for (int k = 0; k < n; ++k) {
    if (k == n - 1) {
      u0[k] = dk; u1[k] = 0.0; u2[k] = 0.0; piv[k] = 0;
      break;
    }
    const double sub = e[k];                  // T(k+1, k)
    const double dn = d[k + 1] - lam;
    const double en = (k + 2 < n) ? e[k + 1] : 0.0;
    if (fabs(dk) >= fabs(sub)) {              // no swap
      const double piv_v = (dk == 0.0) ? pert : dk;
      u0[k] = piv_v; u1[k] = ek; u2[k] = 0.0; piv[k] = 0;
      l[k] = sub / piv_v;
      dk = dn - l[k] * ek;
      ek = en;
    } else {                                  // swap rows k and k+1
      u0[k] = sub; u1[k] = dn; u2[k] = en; piv[k] = 1;
      l[k] = dk / sub;
      dk = ek - l[k] * dn;
      ek = -l[k] * en;
    }
  }
  if (u0[n - 1] == 0.0) u0[n - 1] = pert;
  for (int k = 0; k < n; ++k) u0[k] = 1.0 / u0[k];   // store reciprocals: the solves multiply
  double* z = Z + int64_t(col) * n;
  for (int it = 0; it < 3; ++it) {
    // solve P L y = z
    for (int k = 0; k + 1 < n; ++k) {
      if (piv[k]) { const double t = z[k]; z[k] = z[k + 1]; z[k + 1] = t; }
      z[k + 1] -= l[k] * z[k];
    }
    // solve U x = y
    for (int k = n - 1; k >= 0; --k) {
      double s = z[k];
      if (k + 1 < n) s -= u1[k] * z[k + 1];
      if (k + 2 < n) s -= u2[k] * z[k + 2];
      z[k] = s * u0[k];
    }
    for (int c = c0; c < col; ++c) {          // cluster re-orthogonalisation
      const double* y = Z + int64_t(c) * n;
      double dot = 0.0;
      for (int i = 0; i < n; ++i) dot += y[i] * z[i];
      for (int i = 0; i < n; ++i) z[i] -= dot * y[i];
    }
    double nr = 0.0;
    for (int i = 0; i < n; ++i) nr += z[i] * z[i];
    nr = sqrt(nr);
    if (nr == 0.0) { for (int i = 0; i < n; ++i) z[i] = prand(i, col + 7 * it); continue; }
    for (int i = 0; i < n; ++i) z[i] /= nr;
  }
}

__global__ void __launch_bounds__(TE_THREADS)
k_trid_vectors(double* __restrict__ base, const TridTask* __restrict__ tasks) {
  const TridTask tk = tasks[blockIdx.x];
  const int n = tk.n, kk = tk.keep;
  if (n <= 0 || kk <= 0) return;
  extern __shared__ double sm[];
  double* Z = sm;                 // n x kk (columns = vectors of T, then of A)
  double* d = Z + n * kk;         // n
  double* e = d + n;              // n
  double* y = e + n;              // kk (dot products)
  int* cl = reinterpret_cast<int*>(y + kk);   // cluster start of each kept index
  __shared__ double red[32];
  __shared__ double s_tn;
  const int tid = threadIdx.x;
  const double* ws = base + tk.ws_off;
  const double* W = base + tk.w_off;
  for (int i = tid; i < n; i += blockDim.x) { d[i] = ws[i]; e[i] = ws[n + i]; }
  if (tid == 0) {
    double tn = 0.0;
    for (int i = 0; i < n; ++i) tn = fmax(tn, fabs(W[i]));
    s_tn = fmax(tn, 1e-300);
    // clusters among the kept eigenvalues (descending): gap <= 1e-10 ||T||
    int c0 = 0;
    cl[0] = 0;
    for (int i = 1; i < kk; ++i) {
      if (W[i - 1] - W[i] > 1e-10 * s_tn) c0 = i;
      cl[i] = c0;
    }
  }
  __syncthreads();
  const double tn = s_tn;
  // each cluster is handled by the thread of its first member, members in order
  for (int i = tid; i < kk; i += blockDim.x) {
    if (cl[i] != i) continue;
    int j = i;
    while (j < kk && cl[j] == i) {
      double* z = Z + int64_t(j) * n;
      for (int r = 0; r < n; ++r) z[r] = prand(r, j);
      if (W[j] > 1e-13 * tn) inverse_iteration(d, e, n, W[j], Z, j, i, tn);
      ++j;
    }
  }
  __syncthreads();
  // two passes of classical Gram-Schmidt, largest eigenvalue first
  int attempt = 0;
  for (int c = 0; c < kk; ++c) {
    double* z = Z + int64_t(c) * n;
    for (int pass = 0; pass < 2; ++pass) {
      {
        const int g8 = tid >> 3, l8 = tid & 7, ng8 = blockDim.x >> 3;
        for (int qb = 0; qb < c; qb += ng8) {     // uniform trip count
          const int q = qb + g8;
          double s = 0.0;
          if (q < c) {
            const double* zq = Z + int64_t(q) * n;
            for (int r = l8; r < n; r += 8) s += zq[r] * z[r];
          }
          s += __shfl_xor_sync(0xffffffffu, s, 4, 8);
          s += __shfl_xor_sync(0xffffffffu, s, 2, 8);
          s += __shfl_xor_sync(0xffffffffu, s, 1, 8);
          if (q < c && l8 == 0) y[q] = s;
        }
      }
      __syncthreads();
      for (int r = tid; r < n; r += blockDim.x) {
        double s = z[r];
        for (int q = 0; q < c; ++q) s -= y[q] * Z[int64_t(q) * n + r];
        z[r] = s;
      }
      __syncthreads();
    }
    double part = 0.0;
    for (int r = tid; r < n; r += blockDim.x) part += z[r] * z[r];
    const double nr = sqrt(bsum(part, red));
    if (nr < 1e-8 && attempt < 8) {   // (numerically) in the span already: another start
      ++attempt;
      for (int r = tid; r < n; r += blockDim.x) z[r] = prand(r, c + 1000 * attempt);
      __syncthreads();
      --c;   // redo this column (every thread takes the same branch: nr is block-wide)
      continue;
    }
    attempt = 0;
    for (int r = tid; r < n; r += blockDim.x) z[r] /= fmax(nr, 1e-300);
    __syncthreads();
  }
  // back-transformation with the reflectors H_k = I - tau_k v_k v_k^T (rows k+1..n-1)
  const double* Ag = base + tk.a_off;
  const double* tau = ws + 2 * n;
  for (int k = n - 3; k >= 0; --k) {
    const double t = tau[k];
    if (t == 0.0) continue;
    const int m = n - k - 1;
    const double* vk = Ag + k * n + k + 1;    // vk[0] = 1 implicitly
    const int lane = tid & 31, wp = tid >> 5, nw = blockDim.x >> 5;
    {
      const int g8 = tid >> 3, l8 = tid & 7, ng8 = blockDim.x >> 3;
      for (int qb = 0; qb < kk; qb += ng8) {       // uniform trip count: shuffles stay convergent
        const int q = qb + g8;
        double s = 0.0;
        if (q < kk) {
          const double* zq = Z + int64_t(q) * n + k + 1;
          for (int r = l8; r < m; r += 8) s += (r == 0 ? 1.0 : vk[r]) * zq[r];
        }
        s += __shfl_xor_sync(0xffffffffu, s, 4, 8);
        s += __shfl_xor_sync(0xffffffffu, s, 2, 8);
        s += __shfl_xor_sync(0xffffffffu, s, 1, 8);
        if (q < kk && l8 == 0) y[q] = t * s;
      }
    }
    __syncthreads();
    for (int q = wp; q < kk; q += nw) {
      double* zq = Z + int64_t(q) * n + k + 1;
      const double yq = y[q];
      for (int r = lane; r < m; r += 32) zq[r] -= (r == 0 ? 1.0 : vk[r]) * yq;
    }
    __syncthreads();
  }
  double* U = base + tk.u_off;
  for (int x = tid; x < n * kk; x += blockDim.x) U[x] = Z[x];
}

}  // namespace

size_t syevt_smem_vals(int n) { return sizeof(double) * (size_t(n) * n + 7 * size_t(n)) + 64; }
size_t syevt_smem_vecs(int n, int k) {
  return sizeof(double) * (size_t(n) * k + 2 * size_t(n) + k) + sizeof(int) * size_t(k) + 64;
}

void launch_trid_eigvals(cudaStream_t s, double* base, const TridTask* tasks, int ntasks, int max_n) {
  if (ntasks <= 0) return;
  const size_t sm = syevt_smem_vals(max_n);
  cudaFuncSetAttribute(k_trid_eigvals, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
  k_trid_eigvals<<<ntasks, TE_THREADS, sm, s>>>(base, tasks);
  count_launch();
}

void launch_trid_vectors(cudaStream_t s, double* base, const TridTask* tasks, int ntasks,
                         int max_n, int max_k) {
  if (ntasks <= 0) return;
  const size_t sm = syevt_smem_vecs(max_n, max_k);
  cudaFuncSetAttribute(k_trid_vectors, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
  k_trid_vectors<<<ntasks, TE_THREADS, sm, s>>>(base, tasks);
  count_launch();
}

}  // namespace dmrg
