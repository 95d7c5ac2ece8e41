// kernels.cuh -- device kernels of the two-site DMRG engine (sm_100a).
//
// Every contraction of the hot path (Heff steps, environment updates, density matrices, the
// split back into site tensors) is a list of independent dense block products C = op(A) op(B)
// whose operands are sub-matrices of a few device buffers. The host plans the lists; one
// persistent grouped-GEMM launch executes a whole list. Offsets are element offsets from the
// launch's base pointers, so one plan serves every Lanczos vector.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace dmrg {

// One K-segment of a block product: C += op(A_seg) op(B_seg), A_seg is M x K, B_seg is K x N.
struct GemmSeg {
  int64_t a_off, b_off;
  int lda, ldb, K, pad;
};

// One output block C (M x N, column-major, leading dimension ldc) = alpha * sum_seg + beta * C.
struct GemmTask {
  int64_t c_off;
  int ldc, M, N;
  int seg0, nseg;
  int tiles_m;      // ceil(M / BM)
  int tile0;        // first global tile index of this task
  int pad;
  double alpha, beta;
};

// out block (rows x cols, ld) = sum_t coef_t * in_t (same shape, own ld); sparse MPO mixing.
struct MixTerm {
  int64_t in_off;
  int ld, pad;
  double coef;
};
struct MixTask {
  int64_t out_off;
  int ld, rows, cols;
  int term0, nterm;
  int tile0;        // first tile (tiles of 32 columns x all rows)
  int ntiles;
  int pad;
};

// dst (rows x cols, ldd) = scale * src (or src^T when trans), src leading dimension lds.
struct CopyTask {
  int64_t src_off, dst_off;
  int lds, ldd, rows, cols;
  int trans, tile0, ntiles, pad;
  double scale;
};

// One block pair of an environment contraction across a bond: sum_{r,c} X[x_off + r + c*rows] *
// Y[y_off + c + r*cols] (an L-type block [bra x ket] against the R-type block [ket x bra]).
// Tasks are sorted by e0, the first element of the task in the flattened element range.
struct PairTask {
  int64_t x_off, y_off, e0;
  int rows, cols;
};

// Symmetric eigenproblem of an n x n column-major matrix at a_off (leading dim n); eigenvalues
// go to w_off (n doubles, descending) and eigenvectors (columns, same order) to v_off (n x n).
struct EigTask {
  int64_t a_off, v_off, w_off;
  int n, pad;
};

// Tridiagonal eigensolver for density-matrix blocks with n <= SYEVT_NMAX (syevt.cu, shared
// memory) and SYEVT_NMAX < n <= SYEVT_MID_NMAX (syevt_mid.cu, global memory + shared memory).
constexpr int SYEVT_NMAX = 112;
constexpr int SYEVT_MID_NMAX = 512;
struct TridTask {
  int64_t a_off;   // n x n matrix (column-major, ld n); reflectors are stored in its lower part
  int64_t w_off;   // n eigenvalues, descending
  int64_t ws_off;  // 3n workspace: d, e, tau
  int64_t u_off;   // n x keep eigenvectors (launch 2)
  int n, keep;
  int64_t x_off;   // mid-size launches 2-3: workspace offset (syevt_mid_workspace(n, keep) doubles)
};
size_t syevt_smem_vals(int n);
size_t syevt_smem_vecs(int n, int k);
void launch_trid_eigvals(cudaStream_t s, double* base, const TridTask* tasks, int ntasks, int max_n);
void launch_trid_vectors(cudaStream_t s, double* base, const TridTask* tasks, int ntasks,
                         int max_n, int max_k);
int64_t syevt_mid_workspace(int n, int k);
// Largest kept count whose Gram matrix the mid-size vector kernel holds in shared memory for
// blocks up to max_n (tasks above it take the global-memory path; launch them separately).
int syevt_mid_gram_limit(int max_n);
void launch_trid_mid_eigvals(cudaStream_t s, double* base, const TridTask* tasks, int ntasks,
                             int max_n);
// xws: workspace base of the tasks' x_off
void launch_trid_mid_vectors(cudaStream_t s, double* base, const TridTask* tasks, int ntasks,
                             int max_n, int max_k, double* xws);

constexpr int GEMM_BM = 64, GEMM_BN = 64, GEMM_BK = 16;
constexpr int GEMM_SMALL_TILE = 32;   // the second tile shape of the FP64 GEMM (32 x 32)

// Persistent grouped FP64 GEMM (DMMA m8n8k4 tensor-core path), square tiles of `tile` = 64 or
// 32 (the task list's tile counts must match). Every output element accumulates its K products
// in the same order for both tile shapes, so the results are bit-identical.
void launch_gemm_f64(cudaStream_t s, int tile, bool transA, bool transB, const double* A,
                     const double* B, double* C, const GemmTask* tasks, int ntasks,
                     const GemmSeg* segs, int total_tiles, int grid_cap);

// Split-precision grouped GEMM on tcgen05 (FP32 accumulation in TMEM, FP64 in/out), direct form
// with tiles of TF32_TILE_M x TF32_TILE_N_DIRECT: form SPLIT_TF32X3 = three TF32 products,
// SPLIT_BF16X9 = nine BF16 products; err[0] is set when an MMA completion wait gave up.
constexpr int SPLIT_TF32X3 = 1, SPLIT_BF16X9 = 2;
constexpr int TF32_TILE_M = 128;
constexpr int TF32_TILE_N_DIRECT = 64, TF32_TILE_N_IMAGE = 128, TF32_TILE_N_WIDE = 256;
void launch_gemm_split(int form, cudaStream_t s, bool transA, bool transB, const double* A,
                       const double* B, double* C, const GemmTask* tasks, int ntasks,
                       const GemmSeg* segs, int total_tiles, int grid_cap, int* err);
// Image-fed form for large lists (tiles TF32_TILE_M x bn, bn = TF32_TILE_N_IMAGE or
// TF32_TILE_N_WIDE). Every distinct operand window of the list (an ImgPanel: element (r, k) at
// off + r + k*ld, or off + k + r*ld when kcontig) is converted once into chunk images: row tiles
// (SPLIT_IMG_ROWS rows for A, bn rows for B) x K chunks of SPLIT_IMG_K, each chunk the split
// planes of the tile in the MMA's shared-memory layout, zero outside the window. Chunk (rt, kc)
// of a panel is image chunk img0 + rt * kchunks + kc. The GEMM then moves whole chunks with bulk
// copies; a segment finds its chunks through its SegImg.
constexpr int SPLIT_IMG_ROWS = 128, SPLIT_IMG_K = 32;
struct ImgPanel {
  int64_t off, img0;
  int ld, rows, K, kcontig;
  int kchunks, pad;
};
struct SegImg {
  int64_t a_img, b_img;      // first image chunk of the segment's A and B panels
  int a_kchunks, b_kchunks;  // chunks per row tile of those panels
};
// bytes of one chunk image with `rows` rows (SPLIT_IMG_ROWS or TF32_TILE_N_WIDE)
int64_t split_image_chunk_bytes(int form, int rows);
// writes the chunk images (`rows` rows each) of panels[0, npanels) (total_chunks in all) from x
void launch_pack_images(int form, cudaStream_t s, const double* x, unsigned char* img,
                        const ImgPanel* panels, int npanels, int64_t total_chunks, int rows);
// The MPO mixing fused into the image pack of an operand (the mixed blocks are never written):
// columns [col0, col0 + ncols) of a panel are sum_t coef_t * x[in_off_t + r + (k - col0) * ld_t]
// over the mixing terms [term0, term0 + nterm) (MixTerm); a panel's covers (ranges[panel] =
// first cover, count) are sorted by col0 and tile its K columns.
struct MixCover {
  int col0, ncols, term0, nterm;
};
void launch_pack_mix_images(int form, cudaStream_t s, const double* x, unsigned char* img,
                            const ImgPanel* panels, const int2* ranges, const MixCover* covers,
                            const MixTerm* terms, int npanels, int64_t total_chunks, int rows);
void launch_gemm_split_images(int form, int bn, cudaStream_t s, const unsigned char* imgA,
                              const unsigned char* imgB, double* C, const GemmTask* tasks,
                              int ntasks, const GemmSeg* segs, const SegImg* simg,
                              int total_tiles, int grid_cap, int* err);
// slot of the context's status words that the split-precision GEMM sets on a timeout
constexpr int STATUS_MMA = 8;

void launch_mix(cudaStream_t s, const double* in, double* out, const MixTask* tasks, int ntasks,
                const MixTerm* terms, int total_tiles);

void launch_copy(cudaStream_t s, const double* src, double* dst, const CopyTask* tasks,
                 int ntasks, int total_tiles);

// Deterministic reductions: out[j] = <x_j, y> for j < k (x_j = X + j*ldx), written to device memory.
void launch_mdot(cudaStream_t s, const double* X, int64_t ldx, int k, const double* y, int64_t n,
                 double* partial, double* out);
// y = a*x + b*y with a, b either immediate (ap == nullptr) or read from device pointers.
void launch_axpby(cudaStream_t s, int64_t n, double a, const double* ap, double asign,
                  const double* x, double b, const double* bp, double bsign, double* y,
                  int b_recip);
// y -= sum_j c[j] * X_j  (c in device memory), j < k.
void launch_msub(cudaStream_t s, const double* X, int64_t ldx, int k, const double* c,
                 double* y, int64_t n);
void launch_scale(cudaStream_t s, double* x, int64_t n, double a);
void launch_zero(cudaStream_t s, double* x, int64_t n);
// Descriptor bytes [src, src + bytes) to the device address dst (16-byte aligned) as one launch
// whose parameter block carries them; false (nothing launched) above UPLOAD_PARAM_MAX bytes.
constexpr int UPLOAD_PARAM_MAX = 32704;
bool launch_upload(cudaStream_t s, const void* src, size_t bytes, void* dst);
// bytes (a multiple of 4) from device memory to pinned host memory whose device address is
// dst_view (cudaHostGetDevicePointer), written by one launch.
void launch_to_host(cudaStream_t s, const void* src, void* dst_view, size_t bytes);

// Device-resident Krylov scalars: slots of the context's 256-double scalar array. The Krylov
// solve of a bond step runs without host round trips; the host reads only the energy (EN).
namespace lz {
constexpr int CGS = 0;      // [0, 16): Gram-Schmidt coefficients
constexpr int KK = 16;      // <K,K>      (KK and KH adjacent: written by one dot2)
constexpr int KH = 17;      // <K,HK>
constexpr int NRM = 18;     // squared norm of the centre site tensor
constexpr int EN = 19;      // Ritz energy
constexpr int COEF = 32;    // [32, 48): Ritz vector coefficients
constexpr int ALPHA = 48;   // [48, 64): alpha_j
constexpr int B2 = 64;      // [64, 80): |r_j|^2
constexpr int BETA = 80;    // [80, 96): beta_j (0 after a breakdown)
constexpr int ACT = 96;     // [96, 113): 1 while K_j is an active Krylov vector
}  // namespace lz
// x *= 1/sqrt(*nrm2) when *nrm2 > 0
void launch_scale_rsqrt(cudaStream_t s, double* x, int64_t n, const double* nrm2);
// out[0] = <x,x>, out[1] = <x,y>
void launch_dot2(cudaStream_t s, const double* x, const double* y, int64_t n, double* partial,
                 double* out);
// reference 2-vector step: K /= |K|, H -= a1 K, s[ALPHA] = a1, s[B2] = <H,H>
void launch_lanczos2_orth(cudaStream_t s, double* K, double* H, int64_t n, double* scal,
                          double* partial);
// K_{j+1} = H / beta_j, or 0 after a breakdown (beta_j <= betatest)
void launch_next_vector(cudaStream_t s, const double* H, double* Kn, int64_t n, double* scal,
                        int j, double betatest);
// lowest Ritz pair of the Krylov tridiagonal: s[EN], s[COEF + j]; with expo the coefficients of
// exp(tau T) e_1 instead (s[EN] still the lowest eigenvalue)
void launch_ritz(cudaStream_t s, double* scal, int kdim, double tau, bool expo);
// out[0] = sum over the pair tasks (total elements `total`; deterministic order)
void launch_pair_dot(cudaStream_t s, const double* X, const double* Y, const PairTask* tasks,
                     int ntasks, int64_t total, double* partial, double* out);
// out[r * out_stride] = sum over the pair tasks with X shifted by r * x_stride, r < nrows (one
// block per row; fixed order)
void launch_pair_dot_rows(cudaStream_t s, const double* X, int64_t x_stride, const double* Y,
                          const PairTask* tasks, int ntasks, int nrows, double* out,
                          int64_t out_stride);
// y = sum_j c[j] X_j, j < k
void launch_lincomb(cudaStream_t s, const double* X, int64_t ldx, int k, const double* c,
                    double* y, int64_t n);

// Block Jacobi for large blocks (n > 100): padded to N = 16*nb (nb even).
struct BlockEigGroup {
  int64_t a_off, w_off;          // caller's matrix (n x n) / eigenvalues (n), as in EigTask
  int64_t ap_off, vp_off, q_off; // workspace: padded A (N x N), V (N x N), pair rotations
  int n, N;
};
struct BlockEigPlan {
  const BlockEigGroup* groups;   // device arrays
  int ngroups;
  const int2* pairs;             // (group, pair index) for every block pair of a round
  int npairs;
  const int4* tiles;             // (group, kind 0 = A tile / 1 = V tile, a, b)
  int ntiles;
  int maxN, maxn, max_sweeps;
};
int block_eig_padded(int n);
// Runs the sweeps (host loop with one flag read per sweep). flags/floors: >= ngroups entries.
void launch_block_jacobi(cudaStream_t s, double* base, const BlockEigPlan& plan, int* flags_dev,
                         int* flags_host, double* floors_dev, int* sweeps_done);

// Batched cyclic Jacobi: one CTA per task. Overwrites the matrices.
void launch_jacobi(cudaStream_t s, double* base, const EigTask* tasks, int ntasks, int max_n,
                   int* status);

int device_sm_count();
// Raises (never lowers) a kernel's dynamic shared-memory limit on the current device; safe when
// several host threads launch the same kernel with different sizes.
void raise_smem_limit(const void* func, size_t bytes);
// Process-wide count of kernel launches issued by this library.
void count_launch(int n = 1);
long long launch_count();

}  // namespace dmrg
