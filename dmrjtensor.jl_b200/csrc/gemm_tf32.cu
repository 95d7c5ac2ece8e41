// gemm_tf32.cu -- grouped GEMM C = alpha op(A) op(B) + beta C with FP64 operands and result,
// computed as several low-precision tensor-core products on tcgen05 (the split forms of the Heff
// and environment GEMMs). Two forms:
//
//  * 3xTF32: each FP64 operand element x is split into x_hi = tf32(x) and x_lo = tf32(x - x_hi),
//    and C ~ A_hi B_hi + A_hi B_lo + A_lo B_hi (tcgen05.mma kind::tf32, K = 8 per instruction);
//  * 9xBF16: x = b0 + b1 + b2 with b0 = bf16(x), b1 = bf16(x - b0), b2 = bf16(x - b0 - b1)
//    (each part rounded to nearest even from the exact remainder), and C ~ sum over all nine
//    products A_i B_j (kind::f16 with BF16 operands, K = 16 per instruction).
// Both accumulate in FP32 in tensor memory: about FP32 accuracy (relative ~1e-7 per product), with
// the tensor pipe doing the arithmetic. The FP64 Krylov recursion, normalisation and the final
// Ritz energy stay FP64 in the caller.
//
// Same task lists as the FP64 kernel (GemmTask / GemmSeg, element offsets from base pointers).
// A K chunk of 32 of op(A) and op(B) sits in shared memory in the canonical K-major layout
// (8-row x 16-byte core matrices, no swizzle; one plane per split part), one thread issues the
// chunk's MMAs into a TMEM accumulator, and the epilogue reads the accumulator with tcgen05.ld
// (a warp reads TMEM lanes 32 (warp % 4) .. + 31 = rows of the tile) and writes alpha acc +
// beta C in FP64.
//
// Small lists (direct form, tiles 128 x 64): a CTA of 4 warps per tile at a time, persistent
// over tiles; the threads load a chunk of FP64 operands into registers, split them into the
// staged planes, one thread issues the MMAs and commits to an mbarrier, and all threads wait
// (bounded) before the next chunk overwrites the tiles (the next chunk's loads are in flight
// meanwhile; several CTAs per SM overlap one another's staging and MMAs).
//
// Large lists (image-fed form, tiles 128 x 128): a pack pass converts every distinct operand
// window of the list once into chunk images (split planes in the staged layout, zero-padded to
// whole 128-row tiles and 32-element K chunks), and a persistent kernel of one CTA per SM runs
// a producer / MMA / epilogue pipeline over them: one thread moves each chunk's A and B images
// into a ring of shared-memory stages with bulk copies (cp.async.bulk, completion counted in
// bytes on the stage's mbarrier), one thread issues the MMAs of a stage as soon as it is full and
// frees it with tcgen05.commit, and four epilogue warps drain one of two TMEM accumulators while
// the MMAs of the next tile fill the other. Every wait is bounded: a wait that gives up raises
// the kernel's error flag and makes the other roles stop, the producer then waits for its own
// copies in flight, the MMA thread for its MMAs, and the CTA frees its tensor memory.
//
// Both forms stage the same split planes and issue the same MMAs in the same order, so their
// results are bit-identical.
#include "kernels.cuh"
#include "launch.cuh"

namespace dmrg {
namespace {

constexpr int TBM = 128, TBK = 32;
constexpr int TT = 128;                          // 4 warps (direct form)
constexpr long long WAIT_LIMIT = 1ll << 22;      // try_wait rounds before giving up (direct form)
static_assert(TF32_TILE_N_DIRECT == 64 && TF32_TILE_N_IMAGE == 128, "tile widths");
static_assert(SPLIT_IMG_ROWS == TBM && TF32_TILE_N_IMAGE == 128 && TF32_TILE_N_WIDE == 256,
              "image tile shapes");

// The two split forms. A 16-byte unit of a staged plane holds QE consecutive K elements of one
// row; an MMA consumes KSTEP K elements (two core matrices along K).
struct FormTF32 {
  static constexpr int PLANES = 2, EB = 4, QE = 4, KSTEP = 8, PRODUCTS = 3;
  static constexpr uint32_t KIND_BITS = (2u << 7) | (2u << 10);   // A, B = TF32
};
struct FormBF16 {
  static constexpr int PLANES = 3, EB = 2, QE = 8, KSTEP = 16, PRODUCTS = 9;
  static constexpr uint32_t KIND_BITS = (1u << 7) | (1u << 10);   // A, B = BF16
};

constexpr int IK = SPLIT_IMG_K;                  // K elements of an image chunk
static_assert(IK % FormTF32::KSTEP == 0 && IK % FormBF16::KSTEP == 0, "image chunk depth");

// instruction descriptor: D F32 (bits 4-5 = 1), A and B types, both K-major (bits 15, 16 = 0),
// N >> 3 at bit 17, M >> 4 at bit 24
template <class F, int BN>
constexpr uint32_t idesc() {
  return (1u << 4) | F::KIND_BITS | (uint32_t(BN >> 3) << 17) | (uint32_t(TBM >> 4) << 24);
}

template <class F>
struct Tile {
  static constexpr int BN = TF32_TILE_N_DIRECT;
  static constexpr int KQ = TBK / F::QE;                        // units per row and chunk
  static constexpr int A_BYTES = TBM * TBK * F::EB;             // per plane
  static constexpr int B_BYTES = BN * TBK * F::EB;
  static constexpr int SMEM = F::PLANES * (A_BYTES + B_BYTES) + 1024;   // + alignment slack
  static constexpr uint32_t TMEM_COLS = BN;                     // FP32 128 lanes x BN
  static constexpr int A_UNITS = TBM * KQ / TT;                 // per thread
  static constexpr int B_UNITS = BN * KQ / TT;
  static constexpr uint32_t IDESC = idesc<F, BN>();
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, K-major without swizzle: core matrices of 8 rows x 16 bytes;
// the second core matrix along K of a k-step 128 bytes on (leading byte offset), the next 8 rows
// 256 bytes on (stride byte offset); descriptor version 1 at bit 46.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr) {
  uint64_t d = uint64_t((addr >> 4) & 0x3FFFu);
  d |= uint64_t(128 >> 4) << 16;
  d |= uint64_t(256 >> 4) << 32;
  d |= uint64_t(1) << 46;
  return d;
}

// byte offset of the 16-byte unit (row, kq) of a staged plane with R rows: a k-step block (all
// rows, KSTEP = 2 QE elements) is R*32 bytes; inside it 8-row groups of 256 bytes, each two core
// matrices (K halves) of 128 bytes, each 8 rows of 16 bytes
__device__ __forceinline__ int uoff(int R, int row, int kq) {
  return (kq >> 1) * (R * 32) + (row >> 3) * 256 + (kq & 1) * 128 + (row & 7) * 16;
}

__device__ __forceinline__ float tf32r(float f) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(f));
  return __uint_as_float(r);
}

// bf16 bits of f, rounded to nearest (ties to even); f finite
__device__ __forceinline__ uint32_t bf16_bits(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u + 0x7FFFu + ((u >> 16) & 1u)) >> 16;
}
__device__ __forceinline__ double bf16_value(uint32_t b) { return double(__uint_as_float(b << 16)); }

// The split parts of one element as an 8-byte record: TF32 (hi, lo) as two floats; BF16
// (b0, b1, b2, 0) as four 16-bit values.
__device__ __forceinline__ uint2 split_rec(FormTF32, double x) {
  const float hi = tf32r(float(x));
  const float lo = tf32r(float(x - double(hi)));
  return make_uint2(__float_as_uint(hi), __float_as_uint(lo));
}
__device__ __forceinline__ uint2 split_rec(FormBF16, double x) {
  const uint32_t b0 = bf16_bits(float(x));
  const double r1 = x - bf16_value(b0);
  const uint32_t b1 = bf16_bits(float(r1));
  const double r2 = r1 - bf16_value(b1);
  const uint32_t b2 = bf16_bits(float(r2));
  return make_uint2(b0 | (b1 << 16), b2);
}

// stores one 16-byte unit per plane from QE records (shared or global memory)
__device__ __forceinline__ void store_unit(FormTF32, unsigned char* sp, int plane_bytes, int o,
                                           const uint2* r) {
  *reinterpret_cast<uint4*>(sp + o) = make_uint4(r[0].x, r[1].x, r[2].x, r[3].x);
  *reinterpret_cast<uint4*>(sp + plane_bytes + o) = make_uint4(r[0].y, r[1].y, r[2].y, r[3].y);
}
__device__ __forceinline__ void store_unit(FormBF16, unsigned char* sp, int plane_bytes, int o,
                                           const uint2* r) {
  uint32_t p0[4], p1[4], p2[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const uint2 a = r[2 * q], b = r[2 * q + 1];
    p0[q] = (a.x & 0xFFFFu) | (b.x << 16);
    p1[q] = (a.x >> 16) | (b.x & 0xFFFF0000u);
    p2[q] = (a.y & 0xFFFFu) | (b.y << 16);
  }
  *reinterpret_cast<uint4*>(sp + o) = make_uint4(p0[0], p0[1], p0[2], p0[3]);
  *reinterpret_cast<uint4*>(sp + plane_bytes + o) = make_uint4(p1[0], p1[1], p1[2], p1[3]);
  *reinterpret_cast<uint4*>(sp + 2 * plane_bytes + o) = make_uint4(p2[0], p2[1], p2[2], p2[3]);
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
__device__ __forceinline__ void mma_f16(uint32_t tmem, uint64_t da, uint64_t db, uint32_t acc,
                                        uint32_t idesc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

// The products of one k-step: plane descriptors of A and B (plane p at base + p * plane bytes).
// TF32: hi.hi, hi.lo, lo.hi; BF16: all nine pairs, smallest parts first.
__device__ __forceinline__ void kstep_mmas(FormTF32, uint32_t tmem, uint32_t a, uint32_t ab,
                                           uint32_t b, uint32_t bb, bool& issued, uint32_t idesc) {
  const uint64_t a0 = sdesc(a), a1 = sdesc(a + ab), b0 = sdesc(b), b1 = sdesc(b + bb);
  mma_tf32(tmem, a0, b0, issued ? 1u : 0u, idesc);
  issued = true;
  mma_tf32(tmem, a0, b1, 1u, idesc);
  mma_tf32(tmem, a1, b0, 1u, idesc);
}
__device__ __forceinline__ void kstep_mmas(FormBF16, uint32_t tmem, uint32_t a, uint32_t ab,
                                           uint32_t b, uint32_t bb, bool& issued, uint32_t idesc) {
#pragma unroll
  for (int s = 4; s >= 0; --s)        // part-index sum s = i + j, small terms first
#pragma unroll
    for (int i = 2; i >= 0; --i) {
      const int jj = s - i;
      if (jj < 0 || jj > 2) continue;
      mma_f16(tmem, sdesc(a + i * ab), sdesc(b + jj * bb), issued ? 1u : 0u, idesc);
      issued = true;
    }
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
               :: "r"(bar) : "memory");
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

// the task of a global tile index (tasks sorted by tile0)
__device__ __forceinline__ int find_task(const GemmTask* __restrict__ tasks, int ntasks, int tile) {
  int lo = 0, hi = ntasks - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tasks[mid].tile0 <= tile) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// epilogue of 16 accumulator columns of one row: C = alpha acc + beta C (beta == 0: C not read)
__device__ __forceinline__ void store16(double* __restrict__ C, const GemmTask& tk, int row,
                                        int col0, const float* v) {
  if (row >= tk.M) return;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const int col = col0 + j;
    if (col < tk.N) {
      double* cp = C + tk.c_off + row + int64_t(col) * tk.ldc;
      const double acc = tk.alpha * double(v[j]);
      *cp = (tk.beta == 0.0) ? acc : acc + tk.beta * (*cp);
    }
  }
}

// ------------------------------------------------------------------------------ direct form

template <class F, bool TA, bool TB>
__global__ void __launch_bounds__(TT, 3)
k_gemm_split(const double* __restrict__ A, const double* __restrict__ B, double* __restrict__ C,
             const GemmTask* __restrict__ tasks, int ntasks, const GemmSeg* __restrict__ segs,
             int total_tiles, int* err) {
  grid_entry();
  using TL = Tile<F>;
  constexpr int TBN = TL::BN, KQ = TL::KQ, QE = F::QE;
  constexpr int A_BYTES = TL::A_BYTES, B_BYTES = TL::B_BYTES;
  constexpr int A_UNITS = TL::A_UNITS, B_UNITS = TL::B_UNITS;
  constexpr uint32_t TMEM_COLS = TL::TMEM_COLS, IDESC = TL::IDESC;
  extern __shared__ unsigned char smraw[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // 1024-byte aligned operand area: A planes | B planes
  const uint32_t raw = smem_u32(smraw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  unsigned char* sp = smraw + (base - raw);
  const uint32_t aS = base, bS = base + F::PLANES * A_BYTES;
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
    const GemmTask tk = tasks[find_task(tasks, ntasks, tile)];
    const int local = tile - tk.tile0;
    const int m0 = (local % tk.tiles_m) * TBM, n0 = (local / tk.tiles_m) * TBN;
    // K chunks of this tile, over all its segments: (segment q, offset k0). Each thread owns
    // the 16-byte units tid + TT i of a chunk (QE consecutive K elements of one row): loaded into
    // registers in one batch (the next chunk's loads are issued while the current chunk's MMAs
    // run), then split into the staged planes. Operand stored with rows contiguous: consecutive
    // threads take consecutive rows. Stored with K contiguous: 8 consecutive threads take the
    // same unit of 8 consecutive rows (their 16-byte stores land in 8 different bank groups of
    // one 128-byte line), the next 8 the next unit.
    bool issued = false;
    int q = 0, k0 = 0;
    while (q < tk.nseg && segs[tk.seg0 + q].K <= 0) ++q;
    double ra[A_UNITS][QE], rb[B_UNITS][QE];
    auto a_unit = [&](int i, int& r, int& kq) {
      const int e = tid + TT * i;
      if (TA) { r = (e & 7) + 8 * (e / (8 * KQ)); kq = (e >> 3) % KQ; } else { r = e % TBM; kq = e / TBM; }
    };
    auto b_unit = [&](int i, int& c, int& kq) {
      const int e = tid + TT * i;
      if (TB) { c = e % TBN; kq = e / TBN; } else { c = (e & 7) + 8 * (e / (8 * KQ)); kq = (e >> 3) % KQ; }
    };
    auto load_chunk = [&](int qq, int kk0) {
      const GemmSeg sg = segs[tk.seg0 + qq];
#pragma unroll
      for (int i = 0; i < A_UNITS; ++i) {
        int r, kq;
        a_unit(i, r, kq);
        const int gr = m0 + r;
#pragma unroll
        for (int j = 0; j < QE; ++j) {
          const int gk = kk0 + QE * kq + j;
          ra[i][j] = (gr < tk.M && gk < sg.K)
                         ? (TA ? A[sg.a_off + gk + int64_t(gr) * sg.lda] : A[sg.a_off + gr + int64_t(gk) * sg.lda])
                         : 0.0;
        }
      }
#pragma unroll
      for (int i = 0; i < B_UNITS; ++i) {
        int c, kq;
        b_unit(i, c, kq);
        const int gc = n0 + c;
#pragma unroll
        for (int j = 0; j < QE; ++j) {
          const int gk = kk0 + QE * kq + j;
          rb[i][j] = (gc < tk.N && gk < sg.K)
                         ? (TB ? B[sg.b_off + gc + int64_t(gk) * sg.ldb] : B[sg.b_off + gk + int64_t(gc) * sg.ldb])
                         : 0.0;
        }
      }
    };
    if (q < tk.nseg) load_chunk(q, k0);
    while (q < tk.nseg) {
      const int ks = min(TBK, segs[tk.seg0 + q].K - k0);
#pragma unroll
      for (int i = 0; i < A_UNITS; ++i) {
        int r, kq;
        a_unit(i, r, kq);
        uint2 rec[QE];
#pragma unroll
        for (int j = 0; j < QE; ++j) rec[j] = split_rec(F{}, ra[i][j]);
        store_unit(F{}, sp, A_BYTES, uoff(TBM, r, kq), rec);
      }
#pragma unroll
      for (int i = 0; i < B_UNITS; ++i) {
        int c, kq;
        b_unit(i, c, kq);
        uint2 rec[QE];
#pragma unroll
        for (int j = 0; j < QE; ++j) rec[j] = split_rec(F{}, rb[i][j]);
        store_unit(F{}, sp + F::PLANES * A_BYTES, B_BYTES, uoff(TBN, c, kq), rec);
      }
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        for (int st = 0; st * F::KSTEP < ks; ++st)
          kstep_mmas(F{}, tmem, aS + st * (TBM * 32), A_BYTES, bS + st * (TBN * 32), B_BYTES,
                     issued, IDESC);
        mma_commit(mb);
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
    // epilogue: row m0 + 32 warp + lane of the tile
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const int row = m0 + 32 * warp + lane;
#pragma unroll
    for (int c4 = 0; c4 < TBN / 16; ++c4) {
      float v[16];
      if (issued) {
        tmem_ld16_wait(tmem + (uint32_t(32 * warp) << 16) + uint32_t(16 * c4), v);
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] = 0.0f;
      }
      store16(C, tk, row, n0 + 16 * c4, v);
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

// --------------------------------------------------------------------------- image-fed form

constexpr int IMG_THREADS = 192;   // warp 0 producer, warp 1 MMA issuer, warps 2-5 epilogue
constexpr int PACK_THREADS = 256;
// a wait of the image-fed kernel gives up after this long (ns); the longest legitimate wait
// (an epilogue warp waiting for a whole tile's MMAs) is well under a millisecond
constexpr unsigned long long IMG_WAIT_NS = 1000000000ull;

// bytes of one chunk image of R rows (planes of R x IK elements)
template <class F>
constexpr int chunk_bytes(int R) { return F::PLANES * R * IK * F::EB; }

// tiles of TBM x BN: a stage holds the A chunk (TBM rows) and the B chunk (BN rows)
template <class F, int BN_>
struct Img {
  static constexpr int BN = BN_;
  static constexpr int A_PLANE = TBM * IK * F::EB, B_PLANE = BN * IK * F::EB;
  static constexpr int A_CHUNK = chunk_bytes<F>(TBM), B_CHUNK = chunk_bytes<F>(BN);
  static constexpr int STAGE = A_CHUNK + B_CHUNK;
  static constexpr int STAGES = (196 * 1024) / STAGE;
  static constexpr int SMEM = STAGES * STAGE + 1024;             // + alignment slack
  static constexpr uint32_t TMEM_COLS = 2 * BN;                  // two accumulators
  static constexpr uint32_t IDESC = idesc<F, BN>();
  static_assert(STAGES >= 2 && SMEM <= 227 * 1024, "image stages fit in shared memory");
  static_assert(STAGE < (1 << 20), "transaction count of one stage");
  static_assert(TMEM_COLS == 256 || TMEM_COLS == 512, "tensor memory allocation");
};

// One CTA per image chunk (grid-stride), R rows per chunk: unit u of a plane (in image order) is
// the 16-byte unit (row, kq) with u * 16 = uoff(R, row, kq); its QE elements are read from the
// panel's window
// (zero outside it), split, and written to every plane of the chunk. Consecutive threads write
// consecutive units; they read consecutive rows (rows contiguous) or 32/64-byte runs of one row
// each (K contiguous).
template <class F>
__global__ void __launch_bounds__(PACK_THREADS)
k_pack_images(const double* __restrict__ x, unsigned char* __restrict__ img,
              const ImgPanel* __restrict__ panels, int npanels, int64_t total_chunks, int R) {
  grid_entry();
  const int plane = R * IK * F::EB, units = R * (IK / F::QE);
  for (int64_t ch = blockIdx.x; ch < total_chunks; ch += gridDim.x) {
    int lo = 0, hi = npanels - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (panels[mid].img0 <= ch) lo = mid; else hi = mid - 1;
    }
    const ImgPanel p = panels[lo];
    const int local = int(ch - p.img0);
    const int rt = local / p.kchunks, kc = local - (local / p.kchunks) * p.kchunks;
    unsigned char* dst = img + ch * int64_t(F::PLANES) * plane;
    for (int u = threadIdx.x; u < units; u += PACK_THREADS) {
      const int kstep = u / (2 * R), w = u - kstep * (2 * R);
      const int row = (w >> 4) * 8 + (w & 7), kq = 2 * kstep + ((w >> 3) & 1);
      const int gr = rt * R + row;
      uint2 rec[F::QE];
#pragma unroll
      for (int j = 0; j < F::QE; ++j) {
        const int gk = kc * IK + kq * F::QE + j;
        double v = 0.0;
        if (gr < p.rows && gk < p.K)
          v = p.kcontig ? x[p.off + gk + int64_t(gr) * p.ld] : x[p.off + gr + int64_t(gk) * p.ld];
        rec[j] = split_rec(F{}, v);
      }
      store_unit(F{}, dst, plane, u * 16, rec);
    }
  }
}

// The pack of an operand that is the MPO mixing of x (see MixCover): the same units as
// k_pack_images, each element summed over its cover's terms in term order (the sums of the
// mixing kernel, bit for bit). A unit's QE columns usually share one cover: then the term loop
// is outside and each term's QE loads go out together.
template <class F>
__global__ void __launch_bounds__(PACK_THREADS)
k_pack_mix_images(const double* __restrict__ x, unsigned char* __restrict__ img,
                  const ImgPanel* __restrict__ panels, const int2* __restrict__ ranges,
                  const MixCover* __restrict__ covers, const MixTerm* __restrict__ terms,
                  int npanels, int64_t total_chunks, int R) {
  grid_entry();
  constexpr int QE = F::QE;
  const int plane = R * IK * F::EB, units = R * (IK / QE);
  for (int64_t ch = blockIdx.x; ch < total_chunks; ch += gridDim.x) {
    int lo = 0, hi = npanels - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (panels[mid].img0 <= ch) lo = mid; else hi = mid - 1;
    }
    const ImgPanel p = panels[lo];
    const int2 rg = ranges[lo];
    const int local = int(ch - p.img0);
    const int rt = local / p.kchunks, kc = local - (local / p.kchunks) * p.kchunks;
    unsigned char* dst = img + ch * int64_t(F::PLANES) * plane;
    for (int u = threadIdx.x; u < units; u += PACK_THREADS) {
      const int kstep = u / (2 * R), w = u - kstep * (2 * R);
      const int row = (w >> 4) * 8 + (w & 7), kq = 2 * kstep + ((w >> 3) & 1);
      const int gr = rt * R + row;
      const int k0 = kc * IK + kq * QE;
      double v[QE];
#pragma unroll
      for (int j = 0; j < QE; ++j) v[j] = 0.0;
      if (gr < p.rows && k0 < p.K) {
        int ci = rg.x;
        while (ci < rg.x + rg.y - 1 && k0 >= covers[ci].col0 + covers[ci].ncols) ++ci;
        const MixCover cv = covers[ci];
        if (k0 + QE <= min(p.K, cv.col0 + cv.ncols)) {
#pragma unroll 2
          for (int q = 0; q < cv.nterm; ++q) {
            const MixTerm tm = terms[cv.term0 + q];
            const double* src = x + tm.in_off + gr + int64_t(k0 - cv.col0) * tm.ld;
            double t[QE];
#pragma unroll
            for (int j = 0; j < QE; ++j) t[j] = src[int64_t(j) * tm.ld];
#pragma unroll
            for (int j = 0; j < QE; ++j) v[j] += tm.coef * t[j];
          }
        } else {
          // the unit straddles two covers or the panel's last column
#pragma unroll
          for (int j = 0; j < QE; ++j) {
            const int gk = k0 + j;
            if (gk >= p.K) continue;
            int cj = rg.x;
            while (cj < rg.x + rg.y - 1 && gk >= covers[cj].col0 + covers[cj].ncols) ++cj;
            const MixCover cw = covers[cj];
            double acc = 0.0;
            for (int q = 0; q < cw.nterm; ++q) {
              const MixTerm tm = terms[cw.term0 + q];
              acc += tm.coef * x[tm.in_off + gr + int64_t(gk - cw.col0) * tm.ld];
            }
            v[j] = acc;
          }
        }
      }
      uint2 rec[QE];
#pragma unroll
      for (int j = 0; j < QE; ++j) rec[j] = split_rec(F{}, v[j]);
      store_unit(F{}, dst, plane, u * 16, rec);
    }
  }
}

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait for the completion of the phase of parity `parity`. Gives up (false) when the
// abort flag is up (check_abort) or after IMG_WAIT_NS, raising the flag.
__device__ __noinline__ bool img_wait_slow(uint32_t bar, uint32_t parity, volatile int* abort_flag,
                                           bool check_abort) {
  const unsigned long long t0 = globaltimer();
  for (uint32_t it = 0;; ++it) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 31u) == 31u) {
      if (check_abort && *abort_flag) return false;
      if (globaltimer() - t0 > IMG_WAIT_NS || it > (1u << 30)) {
        *abort_flag = 1;
        return false;
      }
    }
  }
}
__device__ __forceinline__ bool img_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag,
                                         bool check_abort) {
  return mbar_try(bar, parity) || img_wait_slow(bar, parity, abort_flag, check_abort);
}

template <class F, int BN>
__global__ void __launch_bounds__(IMG_THREADS, 1)
k_gemm_img(const unsigned char* __restrict__ imgA, const unsigned char* __restrict__ imgB,
           double* __restrict__ C, const GemmTask* __restrict__ tasks, int ntasks,
           const GemmSeg* __restrict__ segs, const SegImg* __restrict__ simg, int total_tiles,
           int* err) {
  grid_entry();
  using I = Img<F, BN>;
  constexpr int S = I::STAGES;
  extern __shared__ unsigned char smraw[];
  // full[S] | empty[S] | acc_full[2] | acc_empty[2] | drain
  __shared__ __align__(8) uint64_t bars[2 * S + 5];
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_word;
  volatile int* abort_flag = &abort_word;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t raw = smem_u32(smraw);
  const uint32_t base = (raw + 1023u) & ~1023u;   // stage s: A chunk, B chunk
  auto full = [&](int s) { return smem_u32(&bars[s]); };
  auto empty = [&](int s) { return smem_u32(&bars[S + s]); };
  auto acc_full = [&](int b) { return smem_u32(&bars[2 * S + b]); };
  auto acc_empty = [&](int b) { return smem_u32(&bars[2 * S + 2 + b]); };
  const uint32_t drain = smem_u32(&bars[2 * S + 4]);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                 :: "r"(smem_u32(&tmem_slot)), "r"(I::TMEM_COLS) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (tid == 0) {
    abort_word = 0;
    for (int i = 0; i < 2 * S + 5; ++i) {
      // acc_empty: one arrival per epilogue warp; the others: one arrival (or the commit)
      const int count = (i >= 2 * S + 2 && i < 2 * S + 4) ? 4 : 1;
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n"
                   :: "r"(smem_u32(&bars[i])), "r"(count) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tmem_slot;

  if (warp == 0) {
    // ---- producer: chunk c of this CTA goes to stage c % S (its (c / S)-th use)
    if (lane == 0) {
      int c = 0;
      bool ok = true;
      for (int tile = blockIdx.x; ok && tile < total_tiles; tile += gridDim.x) {
        const GemmTask tk = tasks[find_task(tasks, ntasks, tile)];
        const int local = tile - tk.tile0;
        const int mt = local % tk.tiles_m, nt = local / tk.tiles_m;
        for (int q = 0; ok && q < tk.nseg; ++q) {
          const int K = segs[tk.seg0 + q].K;
          if (K <= 0) continue;
          const SegImg im = simg[tk.seg0 + q];
          const unsigned char* ga = imgA + (im.a_img + int64_t(mt) * im.a_kchunks) * I::A_CHUNK;
          const unsigned char* gb = imgB + (im.b_img + int64_t(nt) * im.b_kchunks) * I::B_CHUNK;
          const int nk = (K + IK - 1) / IK;
          for (int kc = 0; kc < nk; ++kc, ++c) {
            const int s = c % S, n = c / S;
            if (n > 0 && !img_wait(empty(s), uint32_t(n - 1) & 1u, abort_flag, true)) {
              ok = false;
              break;
            }
            const uint32_t sa = base + uint32_t(s) * I::STAGE, sb = sa + I::A_CHUNK;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n"
                         :: "r"(full(s)), "r"(I::STAGE) : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                :: "r"(sa), "l"(ga + int64_t(kc) * I::A_CHUNK), "r"(I::A_CHUNK), "r"(full(s))
                : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                :: "r"(sb), "l"(gb + int64_t(kc) * I::B_CHUNK), "r"(I::B_CHUNK), "r"(full(s))
                : "memory");
          }
        }
      }
      // copies in flight land before the CTA exits: wait for the last fill of every stage
      for (int s = 0; s < S && s < c; ++s)
        img_wait(full(s), uint32_t((c - 1 - s) / S) & 1u, abort_flag, false);
    }
    __syncwarp();
  } else if (warp == 1) {
    // ---- MMA issuer: tile t of this CTA accumulates into TMEM columns (t & 1) * BN
    if (lane == 0) {
      int c = 0, t = 0;
      bool ok = true;
      for (int tile = blockIdx.x; ok && tile < total_tiles; tile += gridDim.x, ++t) {
        const GemmTask tk = tasks[find_task(tasks, ntasks, tile)];
        const int b = t & 1, u = t >> 1;
        if (u > 0 && !img_wait(acc_empty(b), uint32_t(u - 1) & 1u, abort_flag, true)) break;
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const uint32_t acc = tmem + uint32_t(b * I::BN);
        bool issued = false;
        for (int q = 0; ok && q < tk.nseg; ++q) {
          const int K = segs[tk.seg0 + q].K;
          if (K <= 0) continue;
          const int nk = (K + IK - 1) / IK;
          for (int kc = 0; kc < nk; ++kc, ++c) {
            const int s = c % S, n = c / S;
            if (!img_wait(full(s), uint32_t(n) & 1u, abort_flag, true)) {
              ok = false;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t sa = base + uint32_t(s) * I::STAGE, sb = sa + I::A_CHUNK;
            const int ks = min(IK, K - kc * IK);
            for (int st = 0; st * F::KSTEP < ks; ++st)
              kstep_mmas(F{}, acc, sa + st * (TBM * 32), I::A_PLANE, sb + st * (BN * 32),
                         I::B_PLANE, issued, I::IDESC);
            mma_commit(empty(s));   // the stage is free once these MMAs have read it
          }
        }
        if (ok) mma_commit(acc_full(b));
      }
      // every MMA issued has completed before the tensor memory is freed
      mma_commit(drain);
      img_wait(drain, 0u, abort_flag, false);
    }
    __syncwarp();
  } else {
    // ---- epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 = rows of the tile
    const int wq = warp & 3;
    int t = 0;
    for (int tile = blockIdx.x; tile < total_tiles; tile += gridDim.x, ++t) {
      const GemmTask tk = tasks[find_task(tasks, ntasks, tile)];
      const int local = tile - tk.tile0;
      const int m0 = (local % tk.tiles_m) * TBM, n0 = (local / tk.tiles_m) * I::BN;
      bool has = false;   // whether any MMA wrote the accumulator
      for (int q = 0; q < tk.nseg && !has; ++q) has = segs[tk.seg0 + q].K > 0;
      const int b = t & 1, u = t >> 1;
      int ok = 1;
      if (lane == 0) ok = img_wait(acc_full(b), uint32_t(u) & 1u, abort_flag, true) ? 1 : 0;
      ok = __shfl_sync(0xffffffffu, ok, 0);   // one decision per warp (tcgen05.ld is warp-wide)
      if (!ok) break;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const int row = m0 + 32 * wq + lane;
#pragma unroll 1
      for (int c4 = 0; c4 < I::BN / 16; ++c4) {
        float v[16];
        if (has) {
          tmem_ld16_wait(tmem + (uint32_t(32 * wq) << 16) + uint32_t(b * I::BN + 16 * c4), v);
        } else {
#pragma unroll
          for (int j = 0; j < 16; ++j) v[j] = 0.0f;
        }
        store16(C, tk, row, n0 + 16 * c4, v);
      }
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      __syncwarp();
      if (lane == 0)
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" :: "r"(acc_empty(b)) : "memory");
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (tid == 0 && abort_word != 0 && err) atomicExch(err, 1);
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n"
                 :: "r"(tmem), "r"(I::TMEM_COLS) : "memory");
}

// ------------------------------------------------------------------------------- launchers

template <class F, bool TA, bool TB>
void launch_variant(cudaStream_t s, const double* A, const double* B, double* C,
                    const GemmTask* tasks, int ntasks, const GemmSeg* segs, int total_tiles,
                    int grid_cap, int* err) {
  raise_smem_limit(reinterpret_cast<const void*>(k_gemm_split<F, TA, TB>), Tile<F>::SMEM);
  const int grid = total_tiles < grid_cap ? total_tiles : grid_cap;
  launch_k(k_gemm_split<F, TA, TB>, grid, TT, Tile<F>::SMEM, s, A, B, C, tasks, ntasks, segs,
           total_tiles, err);
  count_launch();
}

template <class F>
void dispatch(cudaStream_t s, bool transA, bool transB, const double* A, const double* B,
              double* C, const GemmTask* tasks, int ntasks, const GemmSeg* segs, int total_tiles,
              int grid_cap, int* err) {
  if (!transA && !transB)
    launch_variant<F, false, false>(s, A, B, C, tasks, ntasks, segs, total_tiles, grid_cap, err);
  else if (!transA && transB)
    launch_variant<F, false, true>(s, A, B, C, tasks, ntasks, segs, total_tiles, grid_cap, err);
  else if (transA && !transB)
    launch_variant<F, true, false>(s, A, B, C, tasks, ntasks, segs, total_tiles, grid_cap, err);
  else
    launch_variant<F, true, true>(s, A, B, C, tasks, ntasks, segs, total_tiles, grid_cap, err);
}

template <class F>
void launch_pack(cudaStream_t s, const double* x, unsigned char* img, const ImgPanel* panels,
                 int npanels, int64_t total_chunks, int rows) {
  const int grid = int(total_chunks < 4096 ? total_chunks : 4096);
  launch_k(k_pack_images<F>, grid, PACK_THREADS, 0, s, x, img, panels, npanels, total_chunks, rows);
  count_launch();
}

template <class F>
void launch_pack_mix(cudaStream_t s, const double* x, unsigned char* img, const ImgPanel* panels,
                     const int2* ranges, const MixCover* covers, const MixTerm* terms,
                     int npanels, int64_t total_chunks, int rows) {
  const int grid = int(total_chunks < 4096 ? total_chunks : 4096);
  launch_k(k_pack_mix_images<F>, grid, PACK_THREADS, 0, s, x, img, panels, ranges, covers, terms,
           npanels, total_chunks, rows);
  count_launch();
}

template <class F, int BN>
void launch_img(cudaStream_t s, const unsigned char* imgA, const unsigned char* imgB, double* C,
                const GemmTask* tasks, int ntasks, const GemmSeg* segs, const SegImg* simg,
                int total_tiles, int grid_cap, int* err) {
  using I = Img<F, BN>;
  raise_smem_limit(reinterpret_cast<const void*>(k_gemm_img<F, BN>), I::SMEM);
  const int grid = total_tiles < grid_cap ? total_tiles : grid_cap;
  launch_k(k_gemm_img<F, BN>, grid, IMG_THREADS, I::SMEM, s, imgA, imgB, C, tasks, ntasks, segs,
           simg, total_tiles, err);
  count_launch();
}

template <class F>
void launch_img_bn(int bn, cudaStream_t s, const unsigned char* imgA, const unsigned char* imgB,
                   double* C, const GemmTask* tasks, int ntasks, const GemmSeg* segs,
                   const SegImg* simg, int total_tiles, int grid_cap, int* err) {
  if (bn == TF32_TILE_N_WIDE)
    launch_img<F, TF32_TILE_N_WIDE>(s, imgA, imgB, C, tasks, ntasks, segs, simg, total_tiles,
                                    grid_cap, err);
  else
    launch_img<F, TF32_TILE_N_IMAGE>(s, imgA, imgB, C, tasks, ntasks, segs, simg, total_tiles,
                                        grid_cap, err);
}

}  // namespace

void launch_gemm_split(int form, cudaStream_t s, bool transA, bool transB, const double* A,
                       const double* B, double* C, const GemmTask* tasks, int ntasks,
                       const GemmSeg* segs, int total_tiles, int grid_cap, int* err) {
  if (total_tiles <= 0) return;
  if (form == SPLIT_BF16X9)
    dispatch<FormBF16>(s, transA, transB, A, B, C, tasks, ntasks, segs, total_tiles, grid_cap, err);
  else
    dispatch<FormTF32>(s, transA, transB, A, B, C, tasks, ntasks, segs, total_tiles, grid_cap, err);
}

int64_t split_image_chunk_bytes(int form, int rows) {
  return form == SPLIT_BF16X9 ? chunk_bytes<FormBF16>(rows) : chunk_bytes<FormTF32>(rows);
}

void launch_pack_images(int form, cudaStream_t s, const double* x, unsigned char* img,
                        const ImgPanel* panels, int npanels, int64_t total_chunks, int rows) {
  if (total_chunks <= 0 || npanels <= 0) return;
  if (rows != SPLIT_IMG_ROWS && rows != TF32_TILE_N_WIDE) return;
  if (form == SPLIT_BF16X9) launch_pack<FormBF16>(s, x, img, panels, npanels, total_chunks, rows);
  else launch_pack<FormTF32>(s, x, img, panels, npanels, total_chunks, rows);
}

void launch_pack_mix_images(int form, cudaStream_t s, const double* x, unsigned char* img,
                            const ImgPanel* panels, const int2* ranges, const MixCover* covers,
                            const MixTerm* terms, int npanels, int64_t total_chunks, int rows) {
  if (total_chunks <= 0 || npanels <= 0) return;
  if (rows != SPLIT_IMG_ROWS && rows != TF32_TILE_N_WIDE) return;
  if (form == SPLIT_BF16X9)
    launch_pack_mix<FormBF16>(s, x, img, panels, ranges, covers, terms, npanels, total_chunks, rows);
  else
    launch_pack_mix<FormTF32>(s, x, img, panels, ranges, covers, terms, npanels, total_chunks, rows);
}

void launch_gemm_split_images(int form, int bn, cudaStream_t s, const unsigned char* imgA,
                              const unsigned char* imgB, double* C, const GemmTask* tasks,
                              int ntasks, const GemmSeg* segs, const SegImg* simg,
                              int total_tiles, int grid_cap, int* err) {
  if (total_tiles <= 0) return;
  if (form == SPLIT_BF16X9)
    launch_img_bn<FormBF16>(bn, s, imgA, imgB, C, tasks, ntasks, segs, simg, total_tiles,
                            grid_cap, err);
  else
    launch_img_bn<FormTF32>(bn, s, imgA, imgB, C, tasks, ntasks, segs, simg, total_tiles,
                            grid_cap, err);
}

}  // namespace dmrg
