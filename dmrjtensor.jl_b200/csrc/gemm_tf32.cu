// gemm_tf32.cu -- grouped GEMM C = alpha op(A) op(B) + beta C with FP64 operands and result,
// computed as three TF32 tensor-core products on tcgen05 (the split form of the Heff GEMMs).
//
// Each FP64 operand element x is split into x_hi = tf32(x) and x_lo = tf32(x - x_hi), and
// C ~ A_hi B_hi + A_hi B_lo + A_lo B_hi is accumulated in FP32 in tensor memory: about FP32
// accuracy (relative ~1e-7 per product), with the tensor pipe doing the arithmetic. The FP64
// Krylov recursion, normalisation and the final Ritz energy stay FP64 in the caller.
//
// Same task lists as the FP64 kernel (GemmTask / GemmSeg, element offsets from base pointers),
// tiled 128 x 64 (direct form) or 128 x 128 (pre-split form); the lists are retiled to match. One CTA of 4 warps per tile at a time
// (persistent over tiles): the threads stage a K chunk of 32 of op(A) and op(B) into shared
// memory in the canonical K-major layout (8-row x 16-byte core matrices, no swizzle), one thread
// issues 4 k-steps x 3 tcgen05.mma (M=128, N=64, K=8) into a 64-column TMEM accumulator and
// commits to an mbarrier, and all threads wait (bounded) before the next chunk overwrites the
// tiles. The epilogue reads the accumulator with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 =
// rows of the tile) and writes alpha acc + beta C in FP64.
//
// Large lists use the pre-split form (PRE): one memory-bound pass writes every operand element as
// an interleaved (hi, lo) FP32 pair, and the GEMM stages the pairs without converting. In the
// direct form each tile re-splits its operands (five conversions per element on the XU pipe,
// repeated for every tile that reads the element), which bounds the kernel at large sizes; the
// pre-split pass converts each element once. Both forms round identically, so their results are
// bit-identical.
#include <type_traits>

#include "kernels.cuh"

namespace dmrg {
namespace {

constexpr int TBM = 128, TBK = 32;
constexpr int TT = 128;                          // 4 warps
constexpr int A_BYTES = TBM * TBK * 4;           // 16 KB per split part
constexpr long long WAIT_LIMIT = 1ll << 22;      // try_wait rounds before giving up
constexpr int A_QUADS = TBM * TBK / 4 / TT;      // per thread
static_assert(TF32_TILE_N_DIRECT == 64 && TF32_TILE_N_PRESPLIT == 128, "tile widths");

// Tile width by form: 128 x 64 for the direct form (small lists: narrow blocks), 128 x 128 for
// the pre-split form (each staged A tile feeds twice the products).
template <bool PRE>
struct Tile {
  static constexpr int BN = PRE ? TF32_TILE_N_PRESPLIT : TF32_TILE_N_DIRECT;
  static constexpr int B_BYTES = BN * TBK * 4;                      // per split part
  static constexpr int SMEM = 2 * A_BYTES + 2 * B_BYTES + 1024;     // + alignment slack
  static constexpr uint32_t TMEM_COLS = BN;                         // FP32 128 lanes x BN
  static constexpr int B_QUADS = BN * TBK / 4 / TT;
  // instruction descriptor: D F32 (bits 4-5 = 1), A and B TF32 (bits 7-9, 10-12 = 2), both
  // K-major (bits 15, 16 = 0), N >> 3 at bit 17, M >> 4 at bit 24
  static constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) |
                                    (uint32_t(BN >> 3) << 17) | (uint32_t(TBM >> 4) << 24);
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, K-major without swizzle: core matrices of 8 rows x 16 bytes;
// the next 4 K elements (second core matrix of a k-step) 128 bytes on (leading byte offset), the
// next 8 rows 256 bytes on (stride byte offset); descriptor version 1 at bit 46.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr) {
  uint64_t d = uint64_t((addr >> 4) & 0x3FFFu);
  d |= uint64_t(128 >> 4) << 16;
  d |= uint64_t(256 >> 4) << 32;
  d |= uint64_t(1) << 46;
  return d;
}

// byte offset of element (row, k) of a staged operand with R rows and a K chunk of TBK
__device__ __forceinline__ int soff(int R, int row, int k) {
  return (k >> 3) * (R * 32) + (row >> 3) * 256 + ((k >> 2) & 1) * 128 + (row & 7) * 16 +
         (k & 3) * 4;
}

__device__ __forceinline__ float tf32r(float f) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(f));
  return __uint_as_float(r);
}

__device__ __forceinline__ void split(double x, float& hi, float& lo) {
  hi = tf32r(float(x));
  lo = tf32r(float(x - double(hi)));
}

__device__ __forceinline__ void to_pair(double x, float& hi, float& lo) { split(x, hi, lo); }
__device__ __forceinline__ void to_pair(float2 x, float& hi, float& lo) {
  hi = x.x;
  lo = x.y;
}

__global__ void k_presplit(const double* __restrict__ x, float2* __restrict__ y, int64_t n) {
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    float h, l;
    split(x[i], h, l);
    y[i] = make_float2(h, l);
  }
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t da, uint64_t db, uint32_t acc,
                                         uint32_t idesc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ bool mbar_try(uint32_t addr, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(addr), "r"(parity)
      : "memory");
  return ok != 0;
}

// 16 accumulator columns of this thread's row; the wait carries the registers so that no use
// can be scheduled before the load has completed
__device__ __forceinline__ void tmem_ld16_wait(uint32_t addr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                 "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                 "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
               :
               : "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

template <bool TA, bool TB, bool PRE>
__global__ void __launch_bounds__(TT, 3)
k_gemm_tf32x3(const void* __restrict__ Av, const void* __restrict__ Bv, double* __restrict__ C,
              const GemmTask* __restrict__ tasks, int ntasks, const GemmSeg* __restrict__ segs,
              int total_tiles, int* err) {
  // operand elements: FP64 values (direct form) or pre-split (hi, lo) pairs
  using T = typename std::conditional<PRE, float2, double>::type;
  const T* __restrict__ A = static_cast<const T*>(Av);
  const T* __restrict__ B = static_cast<const T*>(Bv);
  constexpr int TBN = Tile<PRE>::BN, B_BYTES = Tile<PRE>::B_BYTES, B_QUADS = Tile<PRE>::B_QUADS;
  constexpr uint32_t TMEM_COLS = Tile<PRE>::TMEM_COLS, IDESC = Tile<PRE>::IDESC;
  extern __shared__ unsigned char smraw[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // 1024-byte aligned operand area: A_hi | A_lo | B_hi | B_lo
  const uint32_t raw = smem_u32(smraw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  unsigned char* sp = smraw + (base - raw);
  const uint32_t aH = base, aL = base + A_BYTES, bH = base + 2 * A_BYTES,
                 bL = base + 2 * A_BYTES + B_BYTES;
  const uint32_t mb = smem_u32(&mbar);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                 :: "r"(smem_u32(&tmem_slot)), "r"(TMEM_COLS) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" :: "r"(mb) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tmem_slot;
  uint32_t phase = 0;
  bool failed = false;

  for (int tile = blockIdx.x; tile < total_tiles; tile += gridDim.x) {
    int lo = 0, hi = ntasks - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (tasks[mid].tile0 <= tile) lo = mid; else hi = mid - 1;
    }
    const GemmTask tk = tasks[lo];
    const int local = tile - tk.tile0;
    const int m0 = (local % tk.tiles_m) * TBM, n0 = (local / tk.tiles_m) * TBN;
    // K chunks of this tile, over all its segments: (segment q, offset k0). Each thread owns
    // the elements tid + TT i of a chunk: loaded into registers in one batch (the next chunk's
    // loads are issued while the current chunk's MMAs run), then split into the staged tiles.
    bool issued = false;
    int q = 0, k0 = 0;
    while (q < tk.nseg && segs[tk.seg0 + q].K <= 0) ++q;
    // quads: 4 consecutive K elements of one row (one 16-byte unit of the staged layout).
    // Operand stored with rows contiguous: consecutive threads take consecutive rows. Stored
    // with K contiguous: 8 consecutive threads take the same quad of 8 consecutive rows (their
    // 16-byte stores land in 8 different bank groups of one 128-byte line), the next 8 the next
    // quad, so a warp still reads 8 rows x 16 contiguous K elements.
    T ra[A_QUADS][4], rb[B_QUADS][4];
    auto a_quad = [&](int i, int& r, int& kq) {
      const int e = tid + TT * i;
      if (TA) { r = (e & 7) + 8 * (e >> 6); kq = (e >> 3) & 7; } else { r = e % TBM; kq = e / TBM; }
    };
    auto b_quad = [&](int i, int& c, int& kq) {
      const int e = tid + TT * i;
      if (TB) { c = e % TBN; kq = e / TBN; } else { c = (e & 7) + 8 * (e >> 6); kq = (e >> 3) & 7; }
    };
    const T zero = T{};
    auto load_chunk = [&](int qq, int kk0) {
      const GemmSeg sg = segs[tk.seg0 + qq];
#pragma unroll
      for (int i = 0; i < A_QUADS; ++i) {
        int r, kq;
        a_quad(i, r, kq);
        const int gr = m0 + r;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int gk = kk0 + 4 * kq + j;
          ra[i][j] = (gr < tk.M && gk < sg.K)
                         ? (TA ? A[sg.a_off + gk + int64_t(gr) * sg.lda] : A[sg.a_off + gr + int64_t(gk) * sg.lda])
                         : zero;
        }
      }
#pragma unroll
      for (int i = 0; i < B_QUADS; ++i) {
        int c, kq;
        b_quad(i, c, kq);
        const int gc = n0 + c;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int gk = kk0 + 4 * kq + j;
          rb[i][j] = (gc < tk.N && gk < sg.K)
                         ? (TB ? B[sg.b_off + gc + int64_t(gk) * sg.ldb] : B[sg.b_off + gk + int64_t(gc) * sg.ldb])
                         : zero;
        }
      }
    };
    if (q < tk.nseg) load_chunk(q, k0);
    while (q < tk.nseg) {
      const int ks = min(TBK, segs[tk.seg0 + q].K - k0);
#pragma unroll
      for (int i = 0; i < A_QUADS; ++i) {
        int r, kq;
        a_quad(i, r, kq);
        float4 h, l;
        to_pair(ra[i][0], h.x, l.x);
        to_pair(ra[i][1], h.y, l.y);
        to_pair(ra[i][2], h.z, l.z);
        to_pair(ra[i][3], h.w, l.w);
        const int o = soff(TBM, r, 4 * kq);
        *reinterpret_cast<float4*>(sp + o) = h;
        *reinterpret_cast<float4*>(sp + A_BYTES + o) = l;
      }
#pragma unroll
      for (int i = 0; i < B_QUADS; ++i) {
        int c, kq;
        b_quad(i, c, kq);
        float4 h, l;
        to_pair(rb[i][0], h.x, l.x);
        to_pair(rb[i][1], h.y, l.y);
        to_pair(rb[i][2], h.z, l.z);
        to_pair(rb[i][3], h.w, l.w);
        const int o = soff(TBN, c, 4 * kq);
        *reinterpret_cast<float4*>(sp + 2 * A_BYTES + o) = h;
        *reinterpret_cast<float4*>(sp + 2 * A_BYTES + B_BYTES + o) = l;
      }
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        for (int st = 0; st * 8 < ks; ++st) {
          const uint64_t dah = sdesc(aH + st * (TBM * 32)), dal = sdesc(aL + st * (TBM * 32));
          const uint64_t dbh = sdesc(bH + st * (TBN * 32)), dbl = sdesc(bL + st * (TBN * 32));
          mma_tf32(tmem, dah, dbh, issued ? 1u : 0u, IDESC);
          issued = true;
          mma_tf32(tmem, dah, dbl, 1u, IDESC);
          mma_tf32(tmem, dal, dbh, 1u, IDESC);
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                     :: "r"(mb) : "memory");
      }
      issued = true;   // every thread: the accumulator holds this tile's partial sum
      // next chunk coordinates; its loads go out while the MMAs run
      k0 += TBK;
      if (k0 >= segs[tk.seg0 + q].K) {
        k0 = 0;
        ++q;
        while (q < tk.nseg && segs[tk.seg0 + q].K <= 0) ++q;
      }
      if (q < tk.nseg) load_chunk(q, k0);
      // the MMAs read the staged tiles: wait until they have completed (bounded)
      long long it = 0;
      bool late = false;
      while (!mbar_try(mb, phase)) {
        if (++it > WAIT_LIMIT) { late = true; break; }
      }
      phase ^= 1u;
      failed = __syncthreads_or(late) != 0;   // the same decision in every thread
      if (failed) break;
    }
    if (failed) break;
    // epilogue: row m0 + 32 warp + lane of the tile, 64 columns
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const int row = m0 + 32 * warp + lane;
    const double alpha = tk.alpha, beta = tk.beta;
#pragma unroll
    for (int c4 = 0; c4 < TBN / 16; ++c4) {
      float v[16];
      if (issued) {
        tmem_ld16_wait(tmem + (uint32_t(32 * warp) << 16) + uint32_t(16 * c4), v);
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] = 0.0f;
      }
      if (row < tk.M) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = n0 + 16 * c4 + j;
          if (col < tk.N) {
            double* cp = C + tk.c_off + row + int64_t(col) * tk.ldc;
            const double acc = alpha * double(v[j]);
            *cp = (beta == 0.0) ? acc : acc + beta * (*cp);
          }
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();   // accumulator reads done before the next tile's first MMA
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  }
  if (failed && err) atomicExch(err, 1);
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n"
                 :: "r"(tmem), "r"(TMEM_COLS) : "memory");
}

template <bool TA, bool TB, bool PRE>
void launch_tf32_variant(cudaStream_t s, const void* A, const void* B, double* C,
                         const GemmTask* tasks, int ntasks, const GemmSeg* segs, int total_tiles,
                         int grid_cap, int* err) {
  raise_smem_limit(reinterpret_cast<const void*>(k_gemm_tf32x3<TA, TB, PRE>), Tile<PRE>::SMEM);
  const int grid = total_tiles < grid_cap ? total_tiles : grid_cap;
  k_gemm_tf32x3<TA, TB, PRE><<<grid, TT, Tile<PRE>::SMEM, s>>>(A, B, C, tasks, ntasks, segs,
                                                                total_tiles, err);
  count_launch();
}

template <bool PRE>
void dispatch(cudaStream_t s, bool transA, bool transB, const void* A, const void* B, double* C,
              const GemmTask* tasks, int ntasks, const GemmSeg* segs, int total_tiles,
              int grid_cap, int* err) {
  if (!transA && !transB)
    launch_tf32_variant<false, false, PRE>(s, A, B, C, tasks, ntasks, segs, total_tiles, grid_cap, err);
  else if (!transA && transB)
    launch_tf32_variant<false, true, PRE>(s, A, B, C, tasks, ntasks, segs, total_tiles, grid_cap, err);
  else if (transA && !transB)
    launch_tf32_variant<true, false, PRE>(s, A, B, C, tasks, ntasks, segs, total_tiles, grid_cap, err);
  else
    launch_tf32_variant<true, true, PRE>(s, A, B, C, tasks, ntasks, segs, total_tiles, grid_cap, err);
}

}  // namespace

void launch_gemm_tf32x3(cudaStream_t s, bool transA, bool transB, const double* A, const double* B,
                        double* C, const GemmTask* tasks, int ntasks, const GemmSeg* segs,
                        int total_tiles, int grid_cap, int* err) {
  if (total_tiles <= 0) return;
  dispatch<false>(s, transA, transB, A, B, C, tasks, ntasks, segs, total_tiles, grid_cap, err);
}

void launch_presplit(cudaStream_t s, const double* x, float2* pairs, int64_t n) {
  if (n <= 0) return;
  const int64_t blocks = (n + 255) / 256;
  k_presplit<<<int(blocks < 1184 ? blocks : 1184), 256, 0, s>>>(x, pairs, n);
  count_launch();
}

void launch_gemm_tf32x3_presplit(cudaStream_t s, bool transA, bool transB, const float2* A,
                                 const float2* B, double* C, const GemmTask* tasks, int ntasks,
                                 const GemmSeg* segs, int total_tiles, int grid_cap, int* err) {
  if (total_tiles <= 0) return;
  dispatch<true>(s, transA, transB, A, B, C, tasks, ntasks, segs, total_tiles, grid_cap, err);
}

}  // namespace dmrg
