// syevt.cu -- density-matrix eigensolver for blocks up to SYEVT_NMAX: Householder
// tridiagonalisation, multisection, inverse iteration, re-orthogonalisation, back-transformation.
// One CTA per block; every phase is laid out for latency (few block barriers, no dependent
// shared- or local-memory loads on the arithmetic chains), since the blocks are small.
//
// Launch 1 (k_trid_eigvals), matrix in shared memory:
//   * A = Q T Q^T by n-2 Householder reflectors (lower form, LAPACK dsytd2 order). Per step two
//     block barriers: B v (two threads per row), then the rank-2 update, during which warp 0
//     updates the next pivot column first and builds the next reflector (look-ahead). The
//     reflector vectors are written into the strictly lower part of the caller's matrix, d/e/tau
//     into a small per-block workspace;
//   * all eigenvalues of T by multisection (2, 3, 4 or 8 threads per eigenvalue as n allows, one
//     Sturm count each per step) to an absolute width of 8.9e-16 ||T||, with a division-free
//     Sturm count (see sturm_below).
// The host then truncates globally and asks for the top-k vectors of each block.
// Launch 2 (k_trid_vectors):
//   * eigenvectors of T by inverse iteration on (T - lambda I) with partial-pivoting LU, one
//     thread per vector (three iterations from a fixed pseudo-random start; factors in shared
//     memory). Vectors of (nearly) equal eigenvalues come out as independent vectors of their
//     common eigenspace; kept eigenvalues below 1e-13 ||T|| (numerically zero) start from the
//     pseudo-random vector alone (an orthonormal completion after the next step);
//   * Cholesky QR over the k vectors (largest eigenvalue first), a second pass unless the Gram
//     matrix was already within 1e-3/k of the identity; two passes of classical Gram-Schmidt
//     with restarts instead if a Cholesky pivot shows nearly dependent vectors;
//   * back-transformation U = Q Z with the stored reflectors, in blocks of 8 (compact WY form
//     I - V T V^T, LAPACK dlarft order).
#include "kernels.cuh"
#include "launch.cuh"
#include "syevt_common.cuh"

namespace dmrg {
namespace {

constexpr int TE_THREADS = 256;   // 8 warps; two threads per row / per eigenvalue (n <= 128)
static_assert(TE_THREADS == 256, "the Householder step sums exactly 8 per-warp shares");
constexpr int TV_THREADS = 256;
constexpr int BT_NB = 8;          // reflectors per back-transformation block
// dynamic shared memory per CTA: the 227 KB opt-in maximum less room for the kernels' static
// shared memory (the dynamic limit of a kernel is the maximum minus its static part)
constexpr size_t SMEM_LIMIT = 227 * 1024 - 1024;

// Householder reflector of column k (one warp): x = A[k+1:n, k], H = I - tau v v^T with v[0] = 1
// and H x = beta e_1. Writes v (length n-k-1) to vout, stores v[1:] in place below the
// subdiagonal, and records d[k] = A[k,k], e[k] = beta, tau[k].
__device__ void householder_col(double* __restrict__ A, int n, int k, double* __restrict__ vout,
                                double* d, double* e, double* tau, int lane) {
  const int m = n - k - 1;
  double* col = A + k * n + k + 1;
  double part = 0.0;
  for (int i = 1 + lane; i < m; i += 32) part += col[i] * col[i];
  const double xn2 = wsum(part);
  const double alpha = col[0];
  double t, sc, beta;
  if (xn2 == 0.0) {
    t = 0.0; sc = 0.0; beta = alpha;
  } else {
    beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
    t = (beta - alpha) / beta;
    sc = 1.0 / (alpha - beta);
  }
  for (int i = lane; i < m; i += 32) {
    const double vi = (i == 0) ? 1.0 : col[i] * sc;
    vout[i] = vi;
    if (i > 0) col[i] = vi;
  }
  if (lane == 0) {
    e[k] = beta;
    tau[k] = t;
    d[k] = A[k + k * n];
  }
}

__global__ void __launch_bounds__(TE_THREADS)
k_trid_eigvals(double* __restrict__ base, const TridTask* __restrict__ tasks) {
  grid_entry();
  const TridTask tk = tasks[blockIdx.x];
  const int n = tk.n;
  if (n <= 0) return;
  extern __shared__ double sm[];
  double* A = sm;               // n x n
  double* vb = A + n * n;       // 2 x n: reflector of this step / of the next
  double* p = vb + 2 * n;       // n
  double* d = p + n;            // n
  double* e = d + n;            // n
  double* e2 = e + n;           // n
  double* tau = e2 + n;         // n
  __shared__ double s_lo, s_hi;
  __shared__ double kw[TE_THREADS / 32];   // per-warp shares of K
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  double* Ag = base + tk.a_off;
  for (int x = tid; x < n * n; x += blockDim.x) A[x] = Ag[x];
  __syncthreads();
  if (n >= 3 && warp == 0) householder_col(A, n, 0, vb, d, e, tau, lane);
  __syncthreads();
  for (int k = 0; k + 2 < n; ++k) {
    const int m = n - k - 1;
    const double* v = vb + (k & 1) * n;
    double* vn = vb + ((k + 1) & 1) * n;
    const double t = tau[k];
    double* B = A + (k + 1) * n + (k + 1);     // trailing matrix B[i + j*n], i, j < m
    {   // p = t B v: two threads per row (row i, half h of the columns; rows of B are read along
        // consecutive i, conflict-free), and this warp's share of K = p.v
      const int i = warp * 16 + (lane >> 1), h = lane & 1;
      const int jh = (m + 1) >> 1;
      const int j0 = h ? jh : 0, j1 = h ? m : jh;
      double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
      if (i < m) {
        const double* Bi = B + i;
        int j = j0;
        for (; j + 8 <= j1; j += 8) {
          double bb[8], ww[8];
#pragma unroll
          for (int q = 0; q < 8; ++q) { bb[q] = Bi[(j + q) * n]; ww[q] = v[j + q]; }
          s0 += bb[0] * ww[0]; s1 += bb[1] * ww[1]; s2 += bb[2] * ww[2]; s3 += bb[3] * ww[3];
          s0 += bb[4] * ww[4]; s1 += bb[5] * ww[5]; s2 += bb[6] * ww[6]; s3 += bb[7] * ww[7];
        }
        for (; j < j1; ++j) s0 += Bi[j * n] * v[j];
      }
      double sv = (s0 + s1) + (s2 + s3);
      sv += __shfl_xor_sync(FULL, sv, 1);
      double kpart = 0.0;
      if (i < m && h == 0) {
        const double pi = t * sv;
        p[i] = pi;
        kpart = pi * v[i];
      }
      kpart = wsum(kpart);
      if (lane == 0) kw[warp] = kpart;
    }
    __syncthreads();
    // K = p.v, w = p - (t K / 2) v; B -= v w^T + w v^T
    const double K = ((kw[0] + kw[1]) + (kw[2] + kw[3])) + ((kw[4] + kw[5]) + (kw[6] + kw[7]));
    const double hk = 0.5 * t * K;
    if (warp == 0) {
      // pivot column (column 0 of B, all rows; c[r] = its row lane + 32 r), then the next
      // reflector from it, without a round trip through shared memory
      const double v0 = v[0];
      const double w0 = p[0] - hk * v0;
      double c[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int i = lane + 32 * r;
        double vi = 0.0, pi = 0.0, bi = 0.0;
        if (i < m) { vi = v[i]; pi = p[i]; bi = B[i]; }
        const double wi = pi - hk * vi;
        c[r] = bi - (vi * w0 + wi * v0);
      }
      if (k + 3 < n) {
        // column k+1 of A: d[k+1] = c(0), alpha = c(1), x tail = c(2..m-1)
        double part = 0.0;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int i = lane + 32 * r;
          if (i >= 2 && i < m) part += c[r] * c[r];
        }
        const double xn2 = wsum(part);
        const double alpha = __shfl_sync(FULL, c[0], 1);
        double tn, sc, beta;
        if (xn2 == 0.0) {
          tn = 0.0; sc = 0.0; beta = alpha;
        } else {
          beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
          tn = (beta - alpha) / beta;
          sc = 1.0 / (alpha - beta);
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int i = lane + 32 * r;
          if (i >= 1 && i < m) {
            const double vi = (i == 1) ? 1.0 : c[r] * sc;
            vn[i - 1] = vi;
            if (i >= 2) B[i] = vi;             // reflector tail, below the subdiagonal
          }
        }
        if (lane == 0) {
          d[k + 1] = c[0];
          e[k + 1] = beta;
          tau[k + 1] = tn;
        }
      } else {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int i = lane + 32 * r;
          if (i < m) B[i] = c[r];
        }
      }
    } else {
      // columns 1..m-1, rows 1..m-1 (row 0 of B is never read again), two columns at a time
      double vi[4], wi[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int i = 1 + lane + 32 * r;
        vi[r] = (i < m) ? v[i] : 0.0;
        wi[r] = (i < m) ? p[i] - hk * v[i] : 0.0;
      }
      const int ow = nw - 1;
      for (int j = warp; j < m; j += 2 * ow) {
        const int j2 = j + ow;
        const bool two = j2 < m;
        const double vj = v[j], wj = p[j] - hk * vj;
        const double vj2 = two ? v[j2] : 0.0;
        const double wj2 = two ? p[j2] - hk * vj2 : 0.0;
        double* col = B + j * n;
        double* col2 = B + j2 * n;
        double b1[4], b2[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int i = 1 + lane + 32 * r;
          b1[r] = (i < m) ? col[i] : 0.0;
          b2[r] = (two && i < m) ? col2[i] : 0.0;
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int i = 1 + lane + 32 * r;
          if (i < m) {
            col[i] = b1[r] - (vi[r] * wj + wi[r] * vj);
            if (two) col2[i] = b2[r] - (vi[r] * wj2 + wi[r] * vj2);
          }
        }
      }
    }
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
  if (warp == 0) {   // Gershgorin interval
    double lo = 1e300, hi = -1e300;
    for (int i = lane; i < n; i += 32) {
      const double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i + 1 < n ? fabs(e[i]) : 0.0);
      lo = fmin(lo, d[i] - r);
      hi = fmax(hi, d[i] + r);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo = fmin(lo, __shfl_xor_sync(FULL, lo, o));
      hi = fmax(hi, __shfl_xor_sync(FULL, hi, o));
    }
    if (lane == 0) {
      const double pad = 2.2e-16 * fmax(fabs(lo), fabs(hi)) + 1e-300;
      s_lo = lo - pad;
      s_hi = hi + pad;
    }
  }
  __syncthreads();
  // multisection: a group of P lanes per eigenvalue (P = 2, 3, 4 or 8 as n allows with 256
  // threads; a group never straddles a warp: for P = 3 each warp holds ten groups, lanes 30-31
  // idle) counts at the P interior points x_g = a + (g + 1) w / (P + 1) of its interval; the
  // counts are nondecreasing in x, so the group's ballot bits read 0..01..1 and the first set bit
  // g brackets the eigenvalue in [x_(g-1), x_g] (no bit: [x_(P-1), b]). The interval shrinks by
  // P + 1 per step: ~32 steps for P = 2, ~27 for P = 3, ~22 for P = 4, ~16 for P = 8.
  const double tn = fmax(fabs(s_lo), fabs(s_hi));
  const double tol = 8.9e-16 * tn;
  const int P = n <= TE_THREADS / 8 ? 8
                : (n <= TE_THREADS / 4 ? 4 : (n <= (TE_THREADS / 32) * 10 ? 3 : 2));
  const int ei = P == 3 ? (lane < 30 ? warp * 10 + lane / 3 : n) : tid / P;
  const int h = P == 3 ? lane % 3 : tid % P;
  const int target = n - 1 - ei;           // i-th largest = (n-1-i)-th smallest
  const double frac = 1.0 / double(P + 1);
  bool done = ei >= n;
  double a = s_lo, b = s_hi;
  for (int it = 0; it < 200; ++it) {
    if (__all_sync(FULL, done)) break;
    bool below = false;
    const double w = b - a;
    if (!done) {
      const double xl = a + w * frac, xh = a + w * (double(P) * frac);
      if (w <= tol || !(a < xl && xl < xh && xh < b)) done = true;   // converged / no progress
      else below = sturm_below(d, e2, n, a + w * (double(h + 1) * frac)) > target;
    }
    const unsigned bal = __ballot_sync(FULL, below);
    if (!done) {
      const unsigned bits = (bal >> (lane - h)) & ((1u << P) - 1u);
      if (bits == 0) {
        a = a + w * (double(P) * frac);
      } else {
        const int g = __ffs(bits) - 1;
        const double xg = a + w * (double(g + 1) * frac);
        if (g > 0) a = a + w * (double(g) * frac);
        b = xg;
      }
    }
  }
  if (h == 0 && ei < n) base[tk.w_off + ei] = 0.5 * (a + b);
}

// Shared-memory layout of k_trid_vectors (doubles first, then ints).
__host__ __device__ size_t vec_union_doubles(int n, int k, int nslot) {
  size_t u = size_t(4) * nslot * n;
  if (size_t(k) * k > u) u = size_t(k) * k;
  if (size_t(n) * n > u) u = size_t(n) * n;
  return u;
}
__host__ __device__ size_t vec_layout_bytes(int n, int k, int nslot) {
  const int ldz = k | 1;
  const int nblk = n >= 3 ? (n - 2 + BT_NB - 1) / BT_NB : 0;
  const size_t dbl = 2 * size_t(n) + size_t(n) * ldz + size_t(BT_NB) * k + size_t(nblk) * 64 +
                     8 * 64 + 2 * size_t(k) + vec_union_doubles(n, k, nslot);
  return sizeof(double) * dbl + sizeof(int) * size_t(nslot) * n + 64;
}

__global__ void __launch_bounds__(TV_THREADS)
k_trid_vectors(double* __restrict__ base, const TridTask* __restrict__ tasks, int nslot) {
  grid_entry();
  const TridTask tk = tasks[blockIdx.x];
  const int n = tk.n, kk = tk.keep;
  if (n <= 0 || kk <= 0) return;
  const int ldz = kk | 1;                 // odd row stride
  const int nblk = n >= 3 ? (n - 2 + BT_NB - 1) / BT_NB : 0;
  extern __shared__ double sm[];
  double* d = sm;                         // n
  double* e = d + n;                      // n
  double* Z = e + n;                      // n x ldz: vector q of row r at Z[r*ldz + q]
  double* Y = Z + n * ldz;                // BT_NB x kk
  double* Tb = Y + BT_NB * kk;            // nblk x 64: T factor of each reflector block
  double* Sw = Tb + nblk * 64;            // 8 warps x 64: reflector Gram entries
  double* rinv = Sw + 8 * 64;             // kk: 1 / Cholesky pivot
  double* sq = rinv + kk;                 // kk: sqrt(Cholesky pivot)
  double* Un = sq + kk;                   // LU factors (nslot threads) | Gram matrix | reflectors
  int* piv = reinterpret_cast<int*>(Un + vec_union_doubles(n, kk, nslot));
  __shared__ double red[32];
  __shared__ double s_tn;
  __shared__ int s_flag, s_need2;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double* ws = base + tk.ws_off;
  const double* W = base + tk.w_off;
  const double* Ag = base + tk.a_off;
  const double* tau = ws + 2 * n;
  for (int i = tid; i < n; i += blockDim.x) { d[i] = ws[i]; e[i] = ws[n + i]; }
  if (warp == 0) {
    double tn = 0.0;
    for (int i = lane; i < n; i += 32) tn = fmax(tn, fabs(W[i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) tn = fmax(tn, __shfl_xor_sync(FULL, tn, o));
    if (lane == 0) {
      s_tn = fmax(tn, 1e-300);
      s_flag = 0;
      s_need2 = 0;
    }
  }
  __syncthreads();
  const double tn = s_tn;
  // ---- inverse iteration: one thread per kept vector, nslot vectors at a time. Vectors of
  // (nearly) equal eigenvalues come out as independent vectors of their common eigenspace and
  // are separated by the orthogonalisation below.
  for (int b0 = 0; b0 < kk; b0 += nslot) {
    const int j = b0 + tid;
    if (tid < nslot && j < kk) {
      LUSlot f{Un + tid, Un + int64_t(nslot) * n + tid, Un + int64_t(2) * nslot * n + tid,
               Un + int64_t(3) * nslot * n + tid, piv + tid, nslot};
      for (int r = 0; r < n; ++r) Z[r * ldz + j] = prand(r, j);
      if (W[j] > 1e-13 * tn) inverse_iteration(d, e, n, W[j], Z, ldz, j, tn, f);
    }
    __syncthreads();
  }
  // ---- Cholesky QR: G = Z^T Z = R^T R, Z <- Z R^{-1}; a second pass when G was not already
  // within 1e-3/k of the identity
  double* G = Un;                         // kk x kk row-major, upper triangle
  for (int pass = 0; pass < 2; ++pass) {
    for (int x = tid; x < kk * kk; x += blockDim.x) {
      const int p = x / kk, q = x - p * kk;
      if (p > q) continue;
      double s0 = 0.0, s1 = 0.0;
      int r = 0;
      for (; r + 2 <= n; r += 2) {
        s0 += Z[r * ldz + p] * Z[r * ldz + q];
        s1 += Z[(r + 1) * ldz + p] * Z[(r + 1) * ldz + q];
      }
      if (r < n) s0 += Z[r * ldz + p] * Z[r * ldz + q];
      const double g = s0 + s1;
      G[p * kk + q] = g;
      if (pass == 0 && fabs(g - (p == q ? 1.0 : 0.0)) > 1e-3 / kk) s_need2 = 1;
    }
    __syncthreads();
    for (int j = 0; j < kk; ++j) {        // outer-product elimination, row j is read-only here
      const double gjj = G[j * kk + j];
      if (!(gjj > 1e-8) && tid == 0) s_flag = 1;   // nearly dependent: Gram-Schmidt instead
      const double inv = 1.0 / fmax(gjj, 1e-300);
      const int t = kk - j - 1;
      for (int x = tid; x < t * t; x += blockDim.x) {
        const int p = j + 1 + x / t, q = j + 1 + x % t;
        if (p <= q) G[p * kk + q] -= G[j * kk + p] * G[j * kk + q] * inv;
      }
      __syncthreads();
    }
    for (int q = tid; q < kk; q += blockDim.x) {
      const double g = fmax(G[q * kk + q], 1e-300);
      rinv[q] = 1.0 / g;
      sq[q] = sqrt(g);
    }
    __syncthreads();
    if (s_flag) break;
    for (int r = tid; r < n; r += blockDim.x) {   // row r: y R' = z with y_q = x_q / sqrt(g_q)
      double* zr = Z + r * ldz;
      for (int q = 0; q < kk; ++q) {
        double s0 = zr[q], s1 = 0.0;
        int p = 0;
        for (; p + 2 <= q; p += 2) {
          s0 -= zr[p] * G[p * kk + q];
          s1 -= zr[p + 1] * G[(p + 1) * kk + q];
        }
        if (p < q) s0 -= zr[p] * G[p * kk + q];
        zr[q] = (s0 + s1) * rinv[q];
      }
      for (int q = 0; q < kk; ++q) zr[q] *= sq[q];
    }
    __syncthreads();
    if (!s_need2) break;
  }
  if (s_flag) {
    // two passes of classical Gram-Schmidt, largest eigenvalue first, with fresh starts for
    // vectors that lie (numerically) in the span of the previous ones
    int attempt = 0;
    for (int c = 0; c < kk; ++c) {
      for (int pass = 0; pass < 2; ++pass) {
        {
          const int g8 = tid >> 3, l8 = tid & 7, ng8 = blockDim.x >> 3;
          for (int qb = 0; qb < c; qb += ng8) {   // uniform trip count: shuffles stay convergent
            const int q = qb + g8;
            double s = 0.0;
            if (q < c)
              for (int r = l8; r < n; r += 8) s += Z[r * ldz + q] * Z[r * ldz + c];
            s += __shfl_xor_sync(FULL, s, 4, 8);
            s += __shfl_xor_sync(FULL, s, 2, 8);
            s += __shfl_xor_sync(FULL, s, 1, 8);
            if (q < c && l8 == 0) Y[q] = s;
          }
        }
        __syncthreads();
        for (int r = tid; r < n; r += blockDim.x) {
          double s = Z[r * ldz + c];
          for (int q = 0; q < c; ++q) s -= Y[q] * Z[r * ldz + q];
          Z[r * ldz + c] = s;
        }
        __syncthreads();
      }
      double part = 0.0;
      for (int r = tid; r < n; r += blockDim.x) part += Z[r * ldz + c] * Z[r * ldz + c];
      const double nr = sqrt(bsum(part, red));
      if (nr < 1e-8 && attempt < 8) {   // block-wide value: every thread takes the same branch
        ++attempt;
        for (int r = tid; r < n; r += blockDim.x) Z[r * ldz + c] = prand(r, c + 1000 * attempt);
        __syncthreads();
        --c;
        continue;
      }
      attempt = 0;
      for (int r = tid; r < n; r += blockDim.x) Z[r * ldz + c] /= fmax(nr, 1e-300);
      __syncthreads();
    }
  }
  // ---- back-transformation U = H_0 H_1 ... H_{n-3} Z in blocks of BT_NB reflectors:
  // H_k0 ... H_k0+nb-1 = I - V T V^T (T upper triangular, forward order). The reflectors are
  // staged in shared memory (column k holds v_k below its implicit unit entry at row k+1).
  double* V = Un;
  for (int x = tid; x < n * n; x += blockDim.x) V[x] = Ag[x];
  __syncthreads();
  for (int bb = warp; bb < nblk; bb += 8) {
    const int k0 = bb * BT_NB, nb = min(BT_NB, n - 2 - k0);
    double* S = Sw + warp * 64;
    if (lane < 28) {                      // S[c][i] = v_c . v_i, c < i
      int c = 0, i = 0, x = lane;
      for (int cc = 0; cc < BT_NB; ++cc) {
        const int cnt = BT_NB - 1 - cc;
        if (x < cnt) { c = cc; i = cc + 1 + x; break; }
        x -= cnt;
      }
      if (i < nb) {
        const int kc = k0 + c, ki = k0 + i;
        const double* vc = V + kc * n;
        const double* vi = V + ki * n;
        double s0 = vc[ki + 1], s1 = 0.0;      // v_i[ki+1] = 1
        int r = ki + 2;
        for (; r + 2 <= n; r += 2) { s0 += vc[r] * vi[r]; s1 += vc[r + 1] * vi[r + 1]; }
        if (r < n) s0 += vc[r] * vi[r];
        S[c * 8 + i] = s0 + s1;
      }
    }
    __syncwarp();
    if (lane < nb) {                      // row a of T: T[a][i] = -tau_i sum_{c=a}^{i-1} T[a][c] S[c][i]
      const int a = lane;
      double Tr[BT_NB];
#pragma unroll
      for (int i = 0; i < BT_NB; ++i) {
        double v = 0.0;
        if (i == a) {
          v = tau[k0 + a];
        } else if (i > a && i < nb) {
          double s = 0.0;
#pragma unroll
          for (int c = 0; c < BT_NB; ++c)
            if (c >= a && c < i) s += Tr[c] * S[c * 8 + i];
          v = -tau[k0 + i] * s;
        }
        Tr[i] = v;
      }
#pragma unroll
      for (int i = 0; i < BT_NB; ++i) Tb[bb * 64 + a * 8 + i] = Tr[i];
    }
    __syncwarp();
  }
  __syncthreads();
  for (int bb = nblk - 1; bb >= 0; --bb) {
    const int k0 = bb * BT_NB, nb = min(BT_NB, n - 2 - k0);
    const double* T = Tb + bb * 64;
    {   // Y = T (V^T Z): 8-lane groups, lane a = reflector, group = vector q
      const int g8 = tid >> 3, a = tid & 7, ng8 = blockDim.x >> 3;
      for (int qb = 0; qb < kk; qb += ng8) {      // uniform trip count: shuffles stay convergent
        const int q = qb + g8;
        double y = 0.0;
        if (q < kk && a < nb) {
          const int k = k0 + a;
          const double* vk = V + k * n;
          double s0 = Z[(k + 1) * ldz + q], s1 = 0.0, s2 = 0.0, s3 = 0.0;
          int r = k + 2;
          for (; r + 4 <= n; r += 4) {
            double vv[4], zz[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) { vv[u] = vk[r + u]; zz[u] = Z[(r + u) * ldz + q]; }
            s0 += vv[0] * zz[0]; s1 += vv[1] * zz[1]; s2 += vv[2] * zz[2]; s3 += vv[3] * zz[3];
          }
          for (; r < n; ++r) s0 += vk[r] * Z[r * ldz + q];
          y = (s0 + s1) + (s2 + s3);
        }
        double y2 = 0.0;
#pragma unroll
        for (int c = 0; c < BT_NB; ++c) {
          const double yc = __shfl_sync(FULL, y, c, 8);
          if (c >= a && c < nb) y2 += T[a * 8 + c] * yc;
        }
        if (q < kk && a < nb) Y[a * kk + q] = y2;
      }
    }
    __syncthreads();
    // Z -= V Y on rows r0..n-1: a thread owns row r (its reflector entries in registers) and
    // the vectors q = g, g + G, ... of its group g
    const int r0 = k0 + 1, nr = n - r0;
    const int G = max(1, int(blockDim.x) / nr);
    if (tid < G * nr) {
      const int g = tid / nr, r = r0 + (tid - g * nr);
      double va[BT_NB];
#pragma unroll
      for (int a = 0; a < BT_NB; ++a) {
        const int k = k0 + a;
        va[a] = (a >= nb) ? 0.0 : (r == k + 1) ? 1.0 : (r > k + 1 ? V[k * n + r] : 0.0);
      }
      double* zr = Z + r * ldz;
      int q = g;
      for (; q + G < kk; q += 2 * G) {
        double s0 = 0.0, s1 = 0.0;
#pragma unroll
        for (int a = 0; a < BT_NB; ++a) {
          if (a < nb) {
            s0 += va[a] * Y[a * kk + q];
            s1 += va[a] * Y[a * kk + q + G];
          }
        }
        zr[q] -= s0;
        zr[q + G] -= s1;
      }
      if (q < kk) {
        double s0 = 0.0;
#pragma unroll
        for (int a = 0; a < BT_NB; ++a)
          if (a < nb) s0 += va[a] * Y[a * kk + q];
        zr[q] -= s0;
      }
    }
    __syncthreads();
  }
  double* U = base + tk.u_off;
  for (int x = tid; x < n * kk; x += blockDim.x) {
    const int q = x / n, r = x - q * n;
    U[x] = Z[r * ldz + q];
  }
}

int vec_slots(int max_n, int max_k) {
  int nslot = max_k;
  while (nslot > 1 && vec_layout_bytes(max_n, max_k, nslot) > SMEM_LIMIT) --nslot;
  return nslot;
}

}  // namespace

size_t syevt_smem_vals(int n) { return sizeof(double) * (size_t(n) * n + 7 * size_t(n)) + 64; }
size_t syevt_smem_vecs(int n, int k) { return vec_layout_bytes(n, k, vec_slots(n, k)); }

void launch_trid_eigvals(cudaStream_t s, double* base, const TridTask* tasks, int ntasks, int max_n) {
  if (ntasks <= 0) return;
  const size_t sm = syevt_smem_vals(max_n);
  raise_smem_limit(reinterpret_cast<const void*>(k_trid_eigvals), sm);
  launch_k(k_trid_eigvals, ntasks, TE_THREADS, sm, s, base, tasks);
  count_launch();
}

void launch_trid_vectors(cudaStream_t s, double* base, const TridTask* tasks, int ntasks,
                         int max_n, int max_k) {
  if (ntasks <= 0) return;
  const int nslot = vec_slots(max_n, max_k);
  const size_t sm = vec_layout_bytes(max_n, max_k, nslot);
  raise_smem_limit(reinterpret_cast<const void*>(k_trid_vectors), sm);
  launch_k(k_trid_vectors, ntasks, TV_THREADS, sm, s, base, tasks, nslot);
  count_launch();
}

}  // namespace dmrg
