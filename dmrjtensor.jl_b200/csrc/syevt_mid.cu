// syevt_mid.cu -- density-matrix eigensolver for mid-size blocks, SYEVT_NMAX < n <= SYEVT_MID_NMAX:
// the method of syevt.cu (Householder tridiagonalisation, multisection, inverse iteration,
// Cholesky QR, blocked back-transformation), one CTA of 512 threads per block, for matrices that
// do not fit in shared memory.
//
// Launch 1 (k_trid_mid_vals): the Householder steps run on the matrix in place in global memory
// (L2-resident: a 512 x 512 block is 2 MB) until the trailing block's lower triangle fits in
// shared memory in packed form (m <= mp, about 230 beside the vectors); it is then copied there
// and the remaining steps run on the copy, which is written back at the end (its strictly lower
// part holds the last reflectors). Global steps: the product p = tau B v by columns (B is
// symmetric: p_j = tau B(:,j).v, one warp per column, four columns in flight), one block barrier,
// then the rank-2 update B -= v w^T + w v^T by the other warps while warp 0 updates the next pivot
// column first and builds the next reflector from it. Packed steps: the same with p by row pairs
// (the stored part of row a along the diagonal direction and of column a below it).
// Eigenvalues by trisection as in syevt.cu, in rounds of 256 eigenvalues.
// Launch 2 (k_trid_mid_vectors): inverse iteration (one thread per kept vector, LU factors in a
// global workspace interleaved by thread so that every factor access of a warp is one line),
// Cholesky QR (a second pass unless the Gram matrix is within 1e-3/k of the identity; classical
// Gram-Schmidt with restarts if a pivot shows nearly dependent vectors); the vectors Z of the
// tridiagonal matrix stay in the workspace.
// Launch 3 (k_trid_mid_backtransform): U = H_0 ... H_{n-3} Z in blocks of 8 reflectors (compact
// WY), one CTA per slice of 32 kept vectors with its slice of Z in shared memory, the reflectors
// read from the matrix in global memory (every slice is independent of the others).
#include "kernels.cuh"
#include "launch.cuh"
#include "syevt_common.cuh"

namespace dmrg {
namespace {

constexpr int MT = 512;             // threads per CTA
constexpr int NW = MT / 32;         // warps
constexpr int MID_BT_NB = 8;        // reflectors per back-transformation block
// columns per warp and pass in the product p = tau B v and in the rank-2 update (fewer for the
// 16-row variant, whose register budget under 512 threads is the same)
constexpr size_t MID_SMEM_LIMIT = 227 * 1024 - 2048;

// Householder reflector of x = col[0..m) (one warp): H x = beta e_1 with v[0] = 1,
// H = I - tau v v^T. Writes v to vout and v[1..m) into col[1..m); returns beta and tau.
__device__ void house_warp(double* __restrict__ col, int m, double* __restrict__ vout,
                           double& beta_o, double& tau_o, int lane) {
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
  beta_o = beta;
  tau_o = t;
}

// Packed lower-triangular storage of the trailing block once it fits in shared memory: column j
// (0-based, of the block of size m0 copied at the switch) holds rows j..m0-1 from offset pk(j).
__device__ __forceinline__ int pk(int j, int m0) { return j * m0 - (j * (j - 1)) / 2; }

// RM = register rows per lane: n <= 32 RM.
template <int RM>
__global__ void __launch_bounds__(MT, 1)
k_trid_mid_vals(double* __restrict__ base, const TridTask* __restrict__ tasks, int mp) {
  grid_entry();
  constexpr int CW = RM >= 16 ? 2 : 4;
  constexpr int CU = RM >= 16 ? 1 : 2;
  const TridTask tk = tasks[blockIdx.x];
  const int n = tk.n;
  if (n < 3 || n > 32 * RM) return;
  extern __shared__ double sm[];
  double* vb = sm;                         // 2 x n: reflector of this step / of the next
  double* p = vb + 2 * n;                  // n
  double* d = p + n;                       // n
  double* e = d + n;                       // n
  double* e2 = e + n;                      // n
  double* tau = e2 + n;                    // n
  double* S = tau + n;                     // packed trailing block, mp (mp + 1) / 2
  __shared__ double kw[NW];
  __shared__ double s_lo, s_hi;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double* Ag = base + tk.a_off;
  double* B = Ag + n + 1;                  // trailing block of step 0, A[1:, 1:]
  const int ld = n;
  if (warp == 0) {
    double be, ta;
    house_warp(Ag + 1, n - 1, vb, be, ta, lane);
    if (lane == 0) { d[0] = Ag[0]; e[0] = be; tau[0] = ta; }
  }
  __syncthreads();
  // steps on the matrix in global memory while the trailing block is larger than mp
  int k = 0;
  for (; k + 2 < n && n - k - 1 > mp; ++k) {
    const int m = n - k - 1;
    const double* v = vb + (k & 1) * n;
    double* vn = vb + ((k + 1) & 1) * n;
    const double t = tau[k];
    {   // p = t B v by columns, and this warp's share of K = p.v
      double vr[RM];
#pragma unroll
      for (int r = 0; r < RM; ++r) {
        const int i = lane + 32 * r;
        vr[r] = (i < m) ? v[i] : 0.0;
      }
      // CW columns per warp at a time: their loads are independent, so a lane keeps CW * RM
      // loads in flight instead of RM (the steps on the L2-resident matrix are latency-bound)
      double kpart = 0.0;
      for (int j0 = warp; j0 < m; j0 += CW * NW) {
        double sc[CW];
#pragma unroll
        for (int c = 0; c < CW; ++c) {
          const int j = j0 + c * NW;
          double s0 = 0.0, s1 = 0.0;
          if (j < m) {
            const double* col = B + int64_t(j) * ld;
#pragma unroll
            for (int r = 0; r < RM; r += 2) {
              const int i0 = lane + 32 * r, i1 = i0 + 32;
              if (i0 < m) s0 += col[i0] * vr[r];
              if (r + 1 < RM && i1 < m) s1 += col[i1] * vr[r + 1];
            }
          }
          sc[c] = s0 + s1;
        }
#pragma unroll
        for (int c = 0; c < CW; ++c) sc[c] = wsum(sc[c]);
        if (lane == 0) {
#pragma unroll
          for (int c = 0; c < CW; ++c) {
            const int j = j0 + c * NW;
            if (j < m) {
              const double pj = t * sc[c];
              p[j] = pj;
              kpart += pj * v[j];
            }
          }
        }
      }
      if (lane == 0) kw[warp] = kpart;
    }
    __syncthreads();
    double K = 0.0;
#pragma unroll
    for (int w = 0; w < NW; ++w) K += kw[w];
    const double hk = 0.5 * t * K;
    if (warp == 0) {
      // pivot column (column 0 of B) with the update applied, then the next reflector from it
      const double v0 = v[0];
      const double w0 = p[0] - hk * v0;
      double c[RM];
#pragma unroll
      for (int r = 0; r < RM; ++r) {
        const int i = lane + 32 * r;
        double vi = 0.0, pi = 0.0, bi = 0.0;
        if (i < m) { vi = v[i]; pi = p[i]; bi = B[i]; }
        const double wi = pi - hk * vi;
        c[r] = bi - (vi * w0 + wi * v0);
      }
      if (k + 3 < n) {
        double part = 0.0;
#pragma unroll
        for (int r = 0; r < RM; ++r) {
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
        for (int r = 0; r < RM; ++r) {
          const int i = lane + 32 * r;
          if (i >= 1 && i < m) {
            const double vi = (i == 1) ? 1.0 : c[r] * sc;
            vn[i - 1] = vi;
            if (i >= 2) B[i] = vi;         // reflector tail, below the subdiagonal
          }
        }
        if (lane == 0) {
          d[k + 1] = c[0];
          e[k + 1] = beta;
          tau[k + 1] = tn;
        }
      } else {
#pragma unroll
        for (int r = 0; r < RM; ++r) {
          const int i = lane + 32 * r;
          if (i < m) B[i] = c[r];
        }
      }
    } else {
      // columns 1..m-1, rows 1..m-1 (row 0 of B is never read again); CU columns at a time
      double vi[RM], wi[RM];
#pragma unroll
      for (int r = 0; r < RM; ++r) {
        const int i = 1 + lane + 32 * r;
        vi[r] = (i < m) ? v[i] : 0.0;
        wi[r] = (i < m) ? p[i] - hk * vi[r] : 0.0;
      }
      for (int j0 = warp; j0 < m; j0 += CU * (NW - 1)) {
        double cv[CU][RM];
#pragma unroll
        for (int c = 0; c < CU; ++c) {
          const int j = j0 + c * (NW - 1);
#pragma unroll
          for (int r = 0; r < RM; ++r) {
            const int i = 1 + lane + 32 * r;
            cv[c][r] = (j < m && i < m) ? B[int64_t(j) * ld + i] : 0.0;
          }
        }
#pragma unroll
        for (int c = 0; c < CU; ++c) {
          const int j = j0 + c * (NW - 1);
          if (j < m) {
            const double vj = v[j], wj = p[j] - hk * vj;
            double* col = B + int64_t(j) * ld;
#pragma unroll
            for (int r = 0; r < RM; ++r) {
              const int i = 1 + lane + 32 * r;
              if (i < m) col[i] = cv[c][r] - (vi[r] * wj + wi[r] * vj);
            }
          }
        }
      }
    }
    __syncthreads();
    B += ld + 1;
  }

  // the trailing block of step k_sw into shared memory (lower triangle, packed), then the
  // remaining steps there: p = tau B v by row pairs (thread 2a sums row a's stored part b <= a
  // along the diagonal direction, thread 2a+1 the column a part b > a), the rank-2 update by
  // columns, warp 0 updating the pivot column first and building the next reflector from it
  const int k_sw = k, m0 = n - k - 1;
  for (int x = tid; x < m0 * m0; x += MT) {
    const int i = x % m0, j = x / m0;
    if (i >= j) S[pk(j, m0) + i - j] = B[i + int64_t(j) * ld];
  }
  __syncthreads();
  for (; k + 2 < n; ++k) {
    const int s0 = k - k_sw, m = n - k - 1;
    const double* v = vb + (k & 1) * n;
    double* vn = vb + ((k + 1) & 1) * n;
    const double t = tau[k];
    const int pks0 = pk(s0, m0);
    {
      const int a = tid >> 1, h = tid & 1;
      double sa = 0.0, sb = 0.0;
      if (a < m) {
        if (h == 0) {                      // b = 0..a: element (a, b) in column s0 + b
          int idx = pks0 + a;
          int b = 0;
          for (; b + 1 <= a; b += 2) {
            sa += S[idx] * v[b];
            idx += m - b - 1;
            sb += S[idx] * v[b + 1];
            idx += m - b - 2;
          }
          if (b <= a) sa += S[idx] * v[b];
        } else {                           // b = a+1..m-1: element (b, a) in column s0 + a
          const double* col = S + pk(s0 + a, m0) - a;
          int b = a + 1;
          for (; b + 2 <= m; b += 2) {
            sa += col[b] * v[b];
            sb += col[b + 1] * v[b + 1];
          }
          if (b < m) sa += col[b] * v[b];
        }
      }
      double sum = sa + sb;
      sum += __shfl_xor_sync(FULL, sum, 1);
      double kpart = 0.0;
      if (a < m && h == 0) {
        const double pa = t * sum;
        p[a] = pa;
        kpart = pa * v[a];
      }
      kpart = wsum(kpart);
      if (lane == 0) kw[warp] = kpart;
    }
    __syncthreads();
    double K = 0.0;
#pragma unroll
    for (int w = 0; w < NW; ++w) K += kw[w];
    const double hk = 0.5 * t * K;
    if (warp == 0) {
      double* B0 = S + pks0;               // pivot column: rows 0..m-1
      const double v0 = v[0];
      const double w0 = p[0] - hk * v0;
      double c[RM];
#pragma unroll
      for (int r = 0; r < RM; ++r) {
        const int i = lane + 32 * r;
        double vi = 0.0, pi = 0.0, bi = 0.0;
        if (i < m) { vi = v[i]; pi = p[i]; bi = B0[i]; }
        const double wi = pi - hk * vi;
        c[r] = bi - (vi * w0 + wi * v0);
      }
      if (k + 3 < n) {
        double part = 0.0;
#pragma unroll
        for (int r = 0; r < RM; ++r) {
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
        for (int r = 0; r < RM; ++r) {
          const int i = lane + 32 * r;
          if (i >= 1 && i < m) {
            const double vi = (i == 1) ? 1.0 : c[r] * sc;
            vn[i - 1] = vi;
            if (i >= 2) B0[i] = vi;        // reflector tail, below the subdiagonal
          }
        }
        if (lane == 0) {
          d[k + 1] = c[0];
          e[k + 1] = beta;
          tau[k + 1] = tn;
        }
      } else {
#pragma unroll
        for (int r = 0; r < RM; ++r) {
          const int i = lane + 32 * r;
          if (i < m) B0[i] = c[r];
        }
      }
    } else {
      for (int j = warp; j < m; j += NW - 1) {   // columns 1..m-1, rows j..m-1
        const double vj = v[j], wj = p[j] - hk * vj;
        double* col = S + pk(s0 + j, m0) - j;
        for (int i = j + lane; i < m; i += 32) {
          const double vi = v[i], wi = p[i] - hk * vi;
          col[i] = col[i] - (vi * wj + wi * vj);
        }
      }
    }
    __syncthreads();
  }
  if (tid == 0) {   // the last 2 x 2 block: A[n-2.., n-2..] at packed column s0f - 1 and s0f
    const int s0f = (n - 2) - k_sw;
    d[n - 2] = S[pk(s0f - 1, m0)];
    e[n - 2] = S[pk(s0f - 1, m0) + 1];
    tau[n - 2] = 0.0;
    d[n - 1] = S[pk(s0f, m0)];
    e[n - 1] = 0.0;
    tau[n - 1] = 0.0;
  }
  {   // the packed block back into the caller's matrix (its reflector tails)
    double* G = Ag + int64_t(k_sw + 1) * n + (k_sw + 1);
    for (int x = tid; x < m0 * m0; x += MT) {
      const int i = x % m0, j = x / m0;
      if (i >= j) G[i + int64_t(j) * n] = S[pk(j, m0) + i - j];
    }
  }
  __syncthreads();
  for (int i = tid; i < n; i += MT) e2[i] = e[i] * e[i];
  double* ws = base + tk.ws_off;          // d | e | tau
  for (int i = tid; i < n; i += MT) {
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
  // trisection, MT/2 eigenvalues per round: threads 2i, 2i+1 count at the interval's two
  // interior points
  const double tnm = fmax(fabs(s_lo), fabs(s_hi));
  const double tol = 8.9e-16 * tnm;
  for (int e0 = 0; e0 < n; e0 += MT / 2) {
    const int ei = e0 + (tid >> 1), h = tid & 1;
    const int target = n - 1 - ei;         // i-th largest = (n-1-i)-th smallest
    bool done = ei >= n;
    double a = s_lo, b = s_hi;
    for (int it = 0; it < 200; ++it) {
      if (__all_sync(FULL, done)) break;
      double x0 = 0.0, x1 = 0.0;
      bool below = false;
      if (!done) {
        const double w = b - a;
        x0 = a + w * (1.0 / 3.0);
        x1 = a + w * (2.0 / 3.0);
        if (w <= tol || !(a < x0 && x0 < x1 && x1 < b)) done = true;
        else below = sturm_below(d, e2, n, h ? x1 : x0) > target;
      }
      const bool other = __shfl_xor_sync(FULL, below, 1);
      if (!done) {
        const bool r0 = h ? other : below, r1 = h ? below : other;
        if (r0) b = x0;
        else if (r1) { a = x0; b = x1; }
        else a = x1;
      }
    }
    if (h == 0 && ei < n) base[tk.w_off + ei] = 0.5 * (a + b);
  }
}

// Workspace of one task of k_trid_mid_vectors, in doubles from x_off: LU factors (4 n k),
// pivots (n k ints), Z (n x (k|1), row-major), Gram matrix (k x k).
__host__ __device__ inline int64_t mid_vec_workspace(int n, int k) {
  const int64_t ldz = k | 1;
  return 4 * int64_t(n) * k + (int64_t(n) * k + 1) / 2 + int64_t(n) * ldz + int64_t(k) * k + 8;
}

// Packed upper triangle by rows of a k x k matrix: row p starts at gpk(p, k).
__host__ __device__ __forceinline__ int gpk(int p, int k) { return p * k - (p * (p - 1)) / 2; }

// Shared memory of k_trid_mid_vectors: d, e (n each), rinv, sq (k each) and, for k <= kg, the
// packed Gram matrix. kg = the largest k for which all of it fits.
__host__ __device__ inline size_t mid_vec_smem_k(int n, int k, bool gram) {
  return sizeof(double) * (2 * size_t(n) + 2 * size_t(k) +
                           (gram ? size_t(k) * (k + 1) / 2 : 0)) + 64;
}
int mid_vec_kg(int max_n) {
  int kg = 0;
  while (mid_vec_smem_k(max_n, kg + 1, true) <= MID_SMEM_LIMIT) ++kg;
  return kg;
}

__global__ void __launch_bounds__(MT, 1)
k_trid_mid_vectors(double* __restrict__ base, const TridTask* __restrict__ tasks,
                   double* __restrict__ xws, int kg) {
  grid_entry();
  const TridTask tk = tasks[blockIdx.x];
  const int n = tk.n, kk = tk.keep;
  if (n < 3 || kk <= 0) return;
  const int ldz = kk | 1;
  extern __shared__ double sm[];
  double* d = sm;                          // n
  double* e = d + n;                       // n
  double* rinv = e + n;                    // kk
  double* sq = rinv + kk;                  // kk
  __shared__ double red[32];
  __shared__ double s_tn;
  __shared__ int s_flag, s_need2;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double* X = xws + tk.x_off;
  double* Un = X;                                          // 4 n kk factors
  int* piv = reinterpret_cast<int*>(X + 4 * int64_t(n) * kk);
  double* Z = X + 4 * int64_t(n) * kk + (int64_t(n) * kk + 1) / 2;   // n x ldz
  double* G = Z + int64_t(n) * ldz;                        // kk x kk row-major, upper triangle
  const double* ws = base + tk.ws_off;
  const double* W = base + tk.w_off;
  for (int i = tid; i < n; i += MT) { d[i] = ws[i]; e[i] = ws[n + i]; }
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
  // ---- inverse iteration: one thread per kept vector; factor element q of thread j at
  // [q * kk + j], so that a warp's accesses to one factor element form one line
  for (int b0 = 0; b0 < kk; b0 += MT) {
    const int j = b0 + tid;
    if (j < kk) {
      LUSlot f{Un + j, Un + int64_t(n) * kk + j, Un + 2 * int64_t(n) * kk + j,
               Un + 3 * int64_t(n) * kk + j, piv + j, kk};
      for (int r = 0; r < n; ++r) Z[int64_t(r) * ldz + j] = prand(r, j);
      if (W[j] > 1e-13 * tn) inverse_iteration(d, e, n, W[j], Z, ldz, j, tn, f);
    }
  }
  __syncthreads();
  // ---- Cholesky QR: G = Z^T Z = R^T R with R = D^(1/2) U (U unit upper), Z <- Z U^-1 D^(-1/2);
  // a second pass unless G was within 1e-3/k of the identity. When the packed upper triangle of
  // G fits in shared memory (kk <= kg) it lives there: the Gram matrix by 4 x 4 register tiles,
  // the elimination by one warp per row, the solve by one thread per row in blocks of 32
  // columns held in registers. Otherwise G stays in the global workspace.
  const bool gsm = kk <= kg;
  double* Gs = sq + kk;                    // packed: G(p, q), q >= p, at gpk(p) + q - p
  for (int pass = 0; pass < 2; ++pass) {
    if (gsm) {
      const int nb4 = (kk + 3) >> 2, ntile = nb4 * (nb4 + 1) / 2;
      for (int x = tid; x < ntile; x += MT) {
        int I = 0;
        while ((I + 1) * nb4 - ((I + 1) * I) / 2 <= x) ++I;
        const int J = I + (x - (I * nb4 - (I * (I - 1)) / 2));
        double acc[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) acc[c] = 0.0;
        for (int r = 0; r < n; ++r) {
          const double* zr = Z + int64_t(r) * ldz;
          double a[4], b[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int ca = 4 * I + u, cb = 4 * J + u;
            a[u] = ca < kk ? zr[ca] : 0.0;
            b[u] = cb < kk ? zr[cb] : 0.0;
          }
#pragma unroll
          for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int w2 = 0; w2 < 4; ++w2) acc[u * 4 + w2] += a[u] * b[w2];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int w2 = 0; w2 < 4; ++w2) {
            const int pp = 4 * I + u, q = 4 * J + w2;
            if (pp <= q && q < kk) {
              const double gv = acc[u * 4 + w2];
              Gs[gpk(pp, kk) + q - pp] = gv;
              if (pass == 0 && fabs(gv - (pp == q ? 1.0 : 0.0)) > 1e-3 / kk) s_need2 = 1;
            }
          }
      }
      __syncthreads();
      for (int j = 0; j < kk; ++j) {
        const double* rowj = Gs + gpk(j, kk) - j;      // rowj[q] = G(j, q), q >= j
        const double gjj = rowj[j];
        if (!(gjj > 1e-8) && tid == 0) s_flag = 1;
        const double inv = 1.0 / fmax(gjj, 1e-300);
        for (int pr = j + 1 + warp; pr < kk; pr += NW) {
          const double f = rowj[pr] * inv;
          double* rowp = Gs + gpk(pr, kk) - pr;
          for (int q = pr + lane; q < kk; q += 32) rowp[q] -= f * rowj[q];
        }
        __syncthreads();
      }
      for (int q = tid; q < kk; q += MT) {
        const double g = fmax(Gs[gpk(q, kk)], 1e-300);
        rinv[q] = 1.0 / g;
        sq[q] = sqrt(g);
      }
      __syncthreads();
      if (s_flag) break;
      for (int r = tid; r < n; r += MT) {
        double* zr = Z + int64_t(r) * ldz;
        for (int q0 = 0; q0 < kk; q0 += 32) {
          const int qb = min(32, kk - q0);
          double acc[32];
#pragma unroll
          for (int c = 0; c < 32; ++c) acc[c] = c < qb ? zr[q0 + c] : 0.0;
#pragma unroll 4
          for (int pp = 0; pp < q0; ++pp) {
            const double y = zr[pp];
            const double* gr = Gs + gpk(pp, kk) - pp;  // gr[q] = G(pp, q)
#pragma unroll
            for (int c = 0; c < 32; ++c)
              if (c < qb) acc[c] -= y * gr[q0 + c];
          }
#pragma unroll
          for (int c = 0; c < 32; ++c) {
            if (c < qb) {
              const double* gc = Gs + gpk(q0, kk) - q0;  // row q0, then down the block
              double sacc = acc[c];
              int off = 0;
#pragma unroll
              for (int c2 = 0; c2 < 32; ++c2) {
                if (c2 < c) sacc -= acc[c2] * gc[off + q0 + c];
                off += kk - (q0 + c2) - 1;             // gpk(p + 1) - (p + 1) - (gpk(p) - p)
              }
              acc[c] = sacc * rinv[q0 + c];
            }
          }
#pragma unroll
          for (int c = 0; c < 32; ++c)
            if (c < qb) zr[q0 + c] = acc[c];
        }
        for (int q = 0; q < kk; ++q) zr[q] *= sq[q];
      }
      __syncthreads();
      if (!s_need2) break;
      continue;
    }
    for (int x = tid; x < kk * kk; x += MT) {
      const int pp = x / kk, q = x - pp * kk;
      if (pp > q) continue;
      double s0 = 0.0, s1 = 0.0;
      int r = 0;
      for (; r + 2 <= n; r += 2) {
        s0 += Z[int64_t(r) * ldz + pp] * Z[int64_t(r) * ldz + q];
        s1 += Z[int64_t(r + 1) * ldz + pp] * Z[int64_t(r + 1) * ldz + q];
      }
      if (r < n) s0 += Z[int64_t(r) * ldz + pp] * Z[int64_t(r) * ldz + q];
      const double g = s0 + s1;
      G[int64_t(pp) * kk + q] = g;
      if (pass == 0 && fabs(g - (pp == q ? 1.0 : 0.0)) > 1e-3 / kk) s_need2 = 1;
    }
    __syncthreads();
    for (int j = 0; j < kk; ++j) {
      const double gjj = G[int64_t(j) * kk + j];
      if (!(gjj > 1e-8) && tid == 0) s_flag = 1;
      const double inv = 1.0 / fmax(gjj, 1e-300);
      const int t = kk - j - 1;
      for (int x = tid; x < t * t; x += MT) {
        const int pp = j + 1 + x / t, q = j + 1 + x % t;
        if (pp <= q)
          G[int64_t(pp) * kk + q] -= G[int64_t(j) * kk + pp] * G[int64_t(j) * kk + q] * inv;
      }
      __syncthreads();
    }
    for (int q = tid; q < kk; q += MT) {
      const double g = fmax(G[int64_t(q) * kk + q], 1e-300);
      rinv[q] = 1.0 / g;
      sq[q] = sqrt(g);
    }
    __syncthreads();
    if (s_flag) break;
    for (int r = tid; r < n; r += MT) {
      double* zr = Z + int64_t(r) * ldz;
      for (int q = 0; q < kk; ++q) {
        double s0 = zr[q], s1 = 0.0;
        int pp = 0;
        for (; pp + 2 <= q; pp += 2) {
          s0 -= zr[pp] * G[int64_t(pp) * kk + q];
          s1 -= zr[pp + 1] * G[int64_t(pp + 1) * kk + q];
        }
        if (pp < q) s0 -= zr[pp] * G[int64_t(pp) * kk + q];
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
          const int g8 = tid >> 3, l8 = tid & 7, ng8 = MT >> 3;
          for (int qb = 0; qb < c; qb += ng8) {
            const int q = qb + g8;
            double s = 0.0;
            if (q < c)
              for (int r = l8; r < n; r += 8) s += Z[int64_t(r) * ldz + q] * Z[int64_t(r) * ldz + c];
            s += __shfl_xor_sync(FULL, s, 4, 8);
            s += __shfl_xor_sync(FULL, s, 2, 8);
            s += __shfl_xor_sync(FULL, s, 1, 8);
            if (q < c && l8 == 0) G[q] = s;      // G reused as the coefficient row
          }
        }
        __syncthreads();
        for (int r = tid; r < n; r += MT) {
          double s = Z[int64_t(r) * ldz + c];
          for (int q = 0; q < c; ++q) s -= G[q] * Z[int64_t(r) * ldz + q];
          Z[int64_t(r) * ldz + c] = s;
        }
        __syncthreads();
      }
      double part = 0.0;
      for (int r = tid; r < n; r += MT) part += Z[int64_t(r) * ldz + c] * Z[int64_t(r) * ldz + c];
      const double nr = sqrt(bsum(part, red));
      if (nr < 1e-8 && attempt < 8) {
        ++attempt;
        for (int r = tid; r < n; r += MT) Z[int64_t(r) * ldz + c] = prand(r, c + 1000 * attempt);
        __syncthreads();
        --c;
        continue;
      }
      attempt = 0;
      for (int r = tid; r < n; r += MT) Z[int64_t(r) * ldz + c] /= fmax(nr, 1e-300);
      __syncthreads();
    }
  }
}

// Back-transformation U = H_0 H_1 ... H_{n-3} Z for one slice of BT_W kept vectors per CTA
// (blockIdx.y = slice): the slice of Z is staged in shared memory, the reflectors are read from
// the matrix in global memory (L2-resident, shared by the slices), applied in blocks of
// MID_BT_NB with their compact-WY T factors (built by each CTA: cheap next to the product).
constexpr int BT_W = 32;
__global__ void __launch_bounds__(MT, 1)
k_trid_mid_backtransform(double* __restrict__ base, const TridTask* __restrict__ tasks,
                         const double* __restrict__ xws) {
  grid_entry();
  const TridTask tk = tasks[blockIdx.x];
  const int n = tk.n, kk = tk.keep;
  const int q0 = blockIdx.y * BT_W;
  if (n < 3 || q0 >= kk) return;
  const int w = min(BT_W, kk - q0);
  const int ldz = kk | 1;
  const int nblk = (n - 2 + MID_BT_NB - 1) / MID_BT_NB;
  extern __shared__ double sm[];
  double* Zs = sm;                               // n x BT_W, row-major (Zs[r * BT_W + q])
  double* Wv = Zs + size_t(n) * BT_W;            // MID_BT_NB x BT_W
  double* Yv = Wv + MID_BT_NB * BT_W;            // MID_BT_NB x BT_W
  double* Tb = Yv + MID_BT_NB * BT_W;            // nblk x 64
  double* Sw = Tb + size_t(nblk) * 64;           // NW x 64
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double* X = xws + tk.x_off;
  const double* Z = X + 4 * int64_t(n) * kk + (int64_t(n) * kk + 1) / 2;
  const double* V = base + tk.a_off;             // reflector k: V[k n + r], r > k + 1
  const double* tau = base + tk.ws_off + 2 * n;
  for (int x = tid; x < n * BT_W; x += MT) {
    const int r = x / BT_W, q = x - r * BT_W;
    Zs[x] = q < w ? Z[int64_t(r) * ldz + q0 + q] : 0.0;
  }
  // T factor of every reflector block (one warp per block)
  for (int bb = warp; bb < nblk; bb += NW) {
    const int k0 = bb * MID_BT_NB, nb = min(MID_BT_NB, n - 2 - k0);
    double* Sg = Sw + warp * 64;
    if (lane < 28) {                      // Sg[c][i] = v_c . v_i, c < i
      int c = 0, i = 0, x = lane;
      for (int cc = 0; cc < MID_BT_NB; ++cc) {
        const int cnt = MID_BT_NB - 1 - cc;
        if (x < cnt) { c = cc; i = cc + 1 + x; break; }
        x -= cnt;
      }
      if (i < nb) {
        const int kc = k0 + c, ki = k0 + i;
        const double* vc = V + int64_t(kc) * n;
        const double* vi = V + int64_t(ki) * n;
        double s0 = vc[ki + 1], s1 = 0.0;      // v_i[ki+1] = 1
        int r = ki + 2;
        for (; r + 2 <= n; r += 2) { s0 += vc[r] * vi[r]; s1 += vc[r + 1] * vi[r + 1]; }
        if (r < n) s0 += vc[r] * vi[r];
        Sg[c * 8 + i] = s0 + s1;
      }
    }
    __syncwarp();
    if (lane < nb) {                      // row a of T: T[a][i] = -tau_i sum_{c=a}^{i-1} T[a][c] S[c][i]
      const int a = lane;
      double Tr[MID_BT_NB];
#pragma unroll
      for (int i = 0; i < MID_BT_NB; ++i) {
        double v = 0.0;
        if (i == a) {
          v = tau[k0 + a];
        } else if (i > a && i < nb) {
          double sacc = 0.0;
#pragma unroll
          for (int c = 0; c < MID_BT_NB; ++c)
            if (c >= a && c < i) sacc += Tr[c] * Sg[c * 8 + i];
          v = -tau[k0 + i] * sacc;
        }
        Tr[i] = v;
      }
#pragma unroll
      for (int i = 0; i < MID_BT_NB; ++i) Tb[bb * 64 + a * 8 + i] = Tr[i];
    }
    __syncwarp();
  }
  __syncthreads();
  for (int bb = nblk - 1; bb >= 0; --bb) {
    const int k0 = bb * MID_BT_NB, nb = min(MID_BT_NB, n - 2 - k0);
    const double* T = Tb + bb * 64;
    {   // W = V^T Zs: pair (a, q) with the rows split between the two halves of the block
      const int half = tid / (MT / 2), pq = tid - half * (MT / 2);
      const int a = pq / BT_W, q = pq - a * BT_W;
      double sacc = 0.0;
      if (a < nb) {
        const int k = k0 + a;
        const double* vk = V + int64_t(k) * n;
        if (half == 0) sacc = Zs[(k + 1) * BT_W + q];
        for (int r = k + 2 + half; r < n; r += 2) sacc += vk[r] * Zs[r * BT_W + q];
      }
      if (half == 1 && a < MID_BT_NB) Wv[a * BT_W + q] = sacc;
      __syncthreads();
      if (half == 0 && a < MID_BT_NB) Wv[a * BT_W + q] += sacc;
    }
    __syncthreads();
    if (tid < MID_BT_NB * BT_W) {         // Y = T W
      const int a = tid / BT_W, q = tid - a * BT_W;
      double y = 0.0;
      if (a < nb)
        for (int c = a; c < nb; ++c) y += T[a * 8 + c] * Wv[c * BT_W + q];
      Yv[a * BT_W + q] = y;
    }
    __syncthreads();
    // Zs -= V Y on rows k0+1..n-1
    for (int x = (k0 + 1) * BT_W + tid; x < n * BT_W; x += MT) {
      const int r = x / BT_W, q = x - r * BT_W;
      double sacc = 0.0;
#pragma unroll
      for (int a = 0; a < MID_BT_NB; ++a) {
        const int k = k0 + a;
        if (a < nb && r >= k + 1) {
          const double va = (r == k + 1) ? 1.0 : V[int64_t(k) * n + r];
          sacc += va * Yv[a * BT_W + q];
        }
      }
      Zs[x] -= sacc;
    }
    __syncthreads();
  }
  double* U = base + tk.u_off;
  for (int x = tid; x < n * w; x += MT) {
    const int q = x / n, r = x - q * n;
    U[int64_t(q0 + q) * n + r] = Zs[r * BT_W + q];
  }
}

int mid_mp(int max_n) {
  // largest trailing block whose packed lower triangle fits in shared memory beside the 7 n
  // vectors (at least 2: the last steps always run there)
  const size_t avail = MID_SMEM_LIMIT - sizeof(double) * 7 * size_t(max_n) - 64;
  int mp = 2;
  while (size_t(mp + 1) * (mp + 2) / 2 * sizeof(double) <= avail) ++mp;
  return mp;
}

template <int RM>
void launch_vals(cudaStream_t s, double* base, const TridTask* tasks, int ntasks, int max_n) {
  const int mp = mid_mp(max_n);
  const size_t sm = sizeof(double) * (size_t(mp) * (mp + 1) / 2 + 7 * size_t(max_n)) + 64;
  raise_smem_limit(reinterpret_cast<const void*>(k_trid_mid_vals<RM>), sm);
  launch_k(k_trid_mid_vals<RM>, ntasks, MT, sm, s, base, tasks, mp);
  count_launch();
}

}  // namespace

int64_t syevt_mid_workspace(int n, int k) { return mid_vec_workspace(n, k); }
int syevt_mid_gram_limit(int max_n) { return mid_vec_kg(max_n); }

void launch_trid_mid_eigvals(cudaStream_t s, double* base, const TridTask* tasks, int ntasks,
                             int max_n) {
  if (ntasks <= 0) return;
  if (max_n <= 256) launch_vals<8>(s, base, tasks, ntasks, max_n);
  else launch_vals<16>(s, base, tasks, ntasks, max_n);
}

void launch_trid_mid_vectors(cudaStream_t s, double* base, const TridTask* tasks, int ntasks,
                             int max_n, int max_k, double* xws) {
  if (ntasks <= 0) return;
  // the Gram matrix in shared memory only when every task's fits (callers split the tasks)
  const int kg = max_k <= mid_vec_kg(max_n) ? max_k : 0;
  const size_t sm = mid_vec_smem_k(max_n, max_k, kg > 0);
  raise_smem_limit(reinterpret_cast<const void*>(k_trid_mid_vectors), sm);
  launch_k(k_trid_mid_vectors, ntasks, MT, sm, s, base, tasks, xws, kg);
  count_launch();
  const int nblk = max_n >= 3 ? (max_n - 2 + MID_BT_NB - 1) / MID_BT_NB : 0;
  const size_t sb = sizeof(double) * (size_t(max_n) * BT_W + 2 * MID_BT_NB * BT_W +
                                      size_t(nblk) * 64 + NW * 64);
  raise_smem_limit(reinterpret_cast<const void*>(k_trid_mid_backtransform), sb);
  const dim3 grid(ntasks, (max_k + BT_W - 1) / BT_W);
  launch_k(k_trid_mid_backtransform, grid, MT, sb, s, base, tasks, xws);
  count_launch();
}

}  // namespace dmrg
