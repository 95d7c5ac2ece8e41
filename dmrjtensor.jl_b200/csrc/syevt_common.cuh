// syevt_common.cuh -- device helpers shared by the density-matrix eigensolvers (syevt.cu for
// blocks up to SYEVT_NMAX, syevt_mid.cu for blocks up to SYEVT_MID_NMAX): warp and block sums,
// the division-free Sturm count of the symmetric tridiagonal matrix, the reproducible start
// vectors and the inverse iteration of one eigenvector.
#pragma once
#include "kernels.cuh"

namespace dmrg {
namespace {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}

// Scales a pair by the power of two that brings the larger magnitude into [1, 2): exact, keeps
// the signs, and needs only exponent-field arithmetic.
__device__ __forceinline__ void rescale_pair(double& D, double& Dm1) {
  const double mx = fmax(fabs(D), fabs(Dm1));
  const int fld = (__double2hiint(mx) >> 20) & 0x7ff;
  if (fld != 0 && fld != 0x7ff) {
    const int ex = min(fld - 1023, 1022);
    const double sc = __hiloint2double((1023 - ex) << 20, 0);
    D *= sc;
    Dm1 *= sc;
  }
}

// Number of eigenvalues of T(d,e) strictly below x: sign changes of the leading minors
// D_j = (d_j - x) D_{j-1} - e_{j-1}^2 D_{j-2}. The carried pair is (D_{j-1}, t_j) with
// t_j = -e_{j-1}^2 D_{j-2}: each step is one FMA for D_j and one product t_{j+1} from D_{j-1}, two
// independent operations, so only the FMA is on the dependent chain. Groups of 8 steps load
// first, count signs after the group (an exact zero minor counts with the sign opposite to its
// predecessor), then rescale the pair by a power of two.
__device__ int sturm_below(const double* __restrict__ d, const double* __restrict__ e2, int n,
                           double x) {
  double D = d[0] - x;
  double t = -e2[0];                      // t_1 = -e_0^2 D_{-1}, D_{-1} = 1
  bool neg = D < 0.0;
  int c = neg ? 1 : 0;
  int j = 1;
  for (; j + 8 <= n; j += 8) {
    double dx[8], ee[8], Ds[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      dx[q] = d[j + q] - x;
      ee[q] = e2[j + q];                  // e2[n-1] = 0: the last product is unused
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const double Dn = fma(dx[q], D, t);
      t = -ee[q] * D;
      D = Dn;
      Ds[q] = Dn;
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const bool ng = (Ds[q] == 0.0) ? !neg : (Ds[q] < 0.0);
      c += (ng != neg) ? 1 : 0;
      neg = ng;
    }
    rescale_pair(D, t);
  }
  for (; j < n; ++j) {
    const double Dn = fma(d[j] - x, D, t);
    t = -e2[j] * D;
    D = Dn;
    const bool ng = (Dn == 0.0) ? !neg : (Dn < 0.0);
    c += (ng != neg) ? 1 : 0;
    neg = ng;
  }
  return c;
}

// pseudo-random start vector entry (fixed: results are reproducible)
__device__ __forceinline__ double prand(int i, int j) {
  unsigned h = unsigned(i) * 2654435761u ^ (unsigned(j) * 40503u + 0x9e3779b9u);
  h ^= h >> 15; h *= 2246822519u; h ^= h >> 13; h *= 3266489917u; h ^= h >> 16;
  return (double(h) / 4294967296.0) - 0.5;
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

// LU factors of one solver thread in shared memory: element k at [k * stride] (threads
// interleaved, so that neighbouring threads touch neighbouring words).
struct LUSlot {
  double *u0, *u1, *u2, *l;
  int* piv;
  int stride;
};

// One thread: z <- (T - lam I)^{-1} z three times, z = column col of the row-major Z (leading
// dimension ldz). The solves run in groups of 8 steps whose loads are issued first, so that only
// the arithmetic recurrence is on the dependent chain.
__device__ void inverse_iteration(const double* __restrict__ d, const double* __restrict__ e, int n,
                                  double lam, double* Z, int ldz, int col, double tn, LUSlot f) {
  const int S = f.stride;
  // factor (T - lam I) = P L U with U having two superdiagonals; u0 keeps reciprocal pivots
  const double pert = 2.2e-16 * tn;
  double dk = d[0] - lam, ek = n > 1 ? e[0] : 0.0;
  for (int k = 0; k + 1 < n; ++k) {
    const double sub = e[k];                  // T(k+1, k)
    const double dn = d[k + 1] - lam;
    const double en = (k + 2 < n) ? e[k + 1] : 0.0;
    if (fabs(dk) >= fabs(sub)) {              // no swap
      const double r = 1.0 / ((dk == 0.0) ? pert : dk);
      const double lk = sub * r;
      f.u0[k * S] = r; f.u1[k * S] = ek; f.u2[k * S] = 0.0; f.piv[k * S] = 0; f.l[k * S] = lk;
      dk = dn - lk * ek;
      ek = en;
    } else {                                  // swap rows k and k+1
      const double r = 1.0 / sub;
      const double lk = dk * r;
      f.u0[k * S] = r; f.u1[k * S] = dn; f.u2[k * S] = en; f.piv[k * S] = 1; f.l[k * S] = lk;
      dk = ek - lk * dn;
      ek = -lk * en;
    }
  }
  f.u0[(n - 1) * S] = 1.0 / ((dk == 0.0) ? pert : dk);
  f.u1[(n - 1) * S] = 0.0; f.u2[(n - 1) * S] = 0.0; f.piv[(n - 1) * S] = 0;
  double* z = Z + col;                        // z[r] at z[r * ldz]
  for (int it = 0; it < 3; ++it) {
    // solve P L y = z; z[k] is carried in a register. Loads of a group precede its stores, and
    // every store goes below the indices still to be loaded.
    double zk = z[0];
    int k = 0;
    for (; k + 8 < n; k += 8) {
      double zz[8], ll[8];
      int pp[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        zz[q] = z[(k + 1 + q) * ldz];
        ll[q] = f.l[(k + q) * S];
        pp[q] = f.piv[(k + q) * S];
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        double zn = zz[q];
        if (pp[q]) { const double tt = zk; zk = zn; zn = tt; }
        zn -= ll[q] * zk;
        z[(k + q) * ldz] = zk;
        zk = zn;
      }
    }
    for (; k + 1 < n; ++k) {
      double zn = z[(k + 1) * ldz];
      if (f.piv[k * S]) { const double tt = zk; zk = zn; zn = tt; }
      zn -= f.l[k * S] * zk;
      z[k * ldz] = zk;
      zk = zn;
    }
    z[(n - 1) * ldz] = zk;
    // solve U x = y (x[k+1], x[k+2] carried in registers)
    double x1 = 0.0, x2 = 0.0;
    k = n - 1;
    for (; k >= 7; k -= 8) {
      double zz[8], a0[8], a1[8], a2[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        zz[q] = z[(k - q) * ldz];
        a0[q] = f.u0[(k - q) * S];
        a1[q] = f.u1[(k - q) * S];
        a2[q] = f.u2[(k - q) * S];
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const double xk = (zz[q] - a1[q] * x1 - a2[q] * x2) * a0[q];
        z[(k - q) * ldz] = xk;
        x2 = x1;
        x1 = xk;
      }
    }
    for (; k >= 0; --k) {
      const double xk = (z[k * ldz] - f.u1[k * S] * x1 - f.u2[k * S] * x2) * f.u0[k * S];
      z[k * ldz] = xk;
      x2 = x1;
      x1 = xk;
    }
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    int i = 0;
    for (; i + 4 <= n; i += 4) {
      s0 += z[i * ldz] * z[i * ldz];
      s1 += z[(i + 1) * ldz] * z[(i + 1) * ldz];
      s2 += z[(i + 2) * ldz] * z[(i + 2) * ldz];
      s3 += z[(i + 3) * ldz] * z[(i + 3) * ldz];
    }
    for (; i < n; ++i) s0 += z[i * ldz] * z[i * ldz];
    const double nr = sqrt((s0 + s1) + (s2 + s3));
    if (nr == 0.0) {
      for (int r = 0; r < n; ++r) z[r * ldz] = prand(r, col + 7 * it);
      continue;
    }
    const double inv = 1.0 / nr;
    for (int r = 0; r < n; ++r) z[r * ldz] *= inv;
  }
}

}  // namespace
}  // namespace dmrg
