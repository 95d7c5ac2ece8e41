/*
 * dmrg_b200.h -- C ABI of libdmrgb200.so, a B200 (sm_100a) two-site DMRG engine.
 *
 * The library is the device side of a drop-in for DMRJtensor.jl's two-site path:
 *   dmrg(psi::MPS, mpo::MPO; m, minm, sweeps, cutoff)          algs/DMRG.jl:549-588
 *     -> dmrg_twosite -> optmps -> twostep                      algs/DMRG.jl:675-691,362-405
 *                                                              algs/optimizeMPS.jl:759-849
 *   makeEnv(psi, mpo) / Lupdate / Rupdate / Lupdate! / Rupdate!  lib/Env/makeEnv.jl:196-246
 *                                                              lib/MPO_MPS/Lupdate.jl:17-37
 *                                                              lib/MPO_MPS/Rupdate.jl:17-37
 * A Julia host binds these with ccall; Python tests bind them with ctypes. Plain C types only.
 *
 * Conventions
 *  - Host arrays are column-major with the reference's index order:
 *      MPS site   A[ml, d, mr]            (lib/types.jl:84-101)
 *      MPO site   W[wl, d, d, wr]         ket = index 2, bra = index 3 (lib/MPO/makeMPO.jl:76)
 *      left env   L[m(bra), w, m(ket)]    right env R[m(ket), w, m(bra)]  (lib/Env/makeEnv.jl:17-26)
 *  - Sites and bonds are 0-based: site i in [0, L); bond b in [0, L] is left of site b.
 *  - Quantum numbers: nsym in {0,1,2} int32 charges per state (0 = dense, no symmetry).
 *    A physical label array has d*nsym ints (state-major). Abelian U(1)^nsym fusion by addition.
 *    MPS bond labels obey q(right) = q(left) + p(s); MPO bond labels obey
 *    r(right) = r(left) + p(ket) - p(bra) (the makeqMPO rule of lib/MPO/makeqMPO.jl:23-84).
 *    Inside the library each bond basis is grouped by charge (a permutation = a gauge change);
 *    downloads report the grouped order and its labels.
 *  - Every function returns 0 (DMRG_OK) or an error code; dmrg_last_error() gives the text.
 *    No C++ exception crosses this boundary. A context is used by one host thread at a time.
 *  - Caller-owned host buffers are read/written only during the call. Device objects belong to
 *    their handles and are released by the matching *_destroy.
 */
#ifndef DMRG_B200_H
#define DMRG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DMRG_ABI_VERSION 3

#if defined(__GNUC__)
#define DMRG_API __attribute__((visibility("default")))
#else
#define DMRG_API
#endif

enum dmrg_status {
  DMRG_OK = 0,
  DMRG_ERR_ARG = 1,      /* bad argument / null handle */
  DMRG_ERR_SHAPE = 2,    /* inconsistent dimensions */
  DMRG_ERR_QN = 3,       /* data in a block that the quantum numbers forbid */
  DMRG_ERR_OOM = 4,      /* device allocation failed */
  DMRG_ERR_BUDGET = 5,   /* request exceeds the context's HBM budget */
  DMRG_ERR_TIMEOUT = 6,  /* a bounded device wait gave up */
  DMRG_ERR_CUDA = 7,     /* CUDA runtime error */
  DMRG_ERR_STATE = 8,    /* object not in a usable state (e.g. environments not built) */
  DMRG_ERR_NOCUDA = 9    /* no CUDA device */
};

enum dmrg_precision {
  DMRG_PREC_FP64 = 0,    /* plain form: every contraction in FP64 (DMMA) */
  DMRG_PREC_3XTF32 = 1,  /* chosen form: the Heff and environment-update GEMMs as 3 TF32
                            tensor-core products (FP32-accurate); with fp64_final the environments
                            of the sweep's second half are FP64 so that the reported energy is the
                            exact FP64 Rayleigh quotient of the final Ritz vector */
  DMRG_PREC_BF16X9 = 2   /* chosen form with BF16 parts: every FP64 operand split into three BF16
                            values, the nine products on the BF16 tensor cores (kind::f16, FP32
                            accumulation); same FP64 parts and fp64_final rule as 3XTF32 */
};

typedef struct dmrg_ctx dmrg_ctx;
typedef struct dmrg_mpo dmrg_mpo;
typedef struct dmrg_state dmrg_state;

/* Parameters of one sweep: the two-site subset of algvars (algs/optimizeMPS.jl:36-106,514-577). */
typedef struct dmrg_params {
  int maxm;          /* `m` keyword; <= 0 means unlimited                      */
  int minm;          /* default 2                                              */
  double cutoff;     /* discarded weight bound, mag = 1 (algs/DMRG.jl:387)      */
  int krylov;        /* 2 = the reference's 2-vector step (algs/DMRG.jl:57-90); k>2 Lanczos with
                        full re-orthogonalisation                               */
  int precision;     /* enum dmrg_precision                                    */
  int svnbond;       /* bond whose entropy is reported (1-based, cld(L,2) by default; 0 = default) */
  double degen_rtol; /* >0: never split a cluster of equal weights at the cut  */
  double betatest;   /* Krylov breakdown threshold, 1e-10 (algs/DMRG.jl:57)     */
  int fp64_final;    /* chosen forms: 1 = re-evaluate the Ritz energy with one FP64 matvec */
  int profile;       /* 1 = time every Heff GEMM launch with CUDA events (gemm_* stats)  */
  int cvgE;          /* convergence test of dmrgcvg (algs/DMRG.jl:610-652): 1 = energy, 0 = entropy */
  int tune;          /* 1 (default): FP64 GEMM tile shapes picked per block-size histogram by the
                        context's autotuner (timed trials, bit-identical results); 0: 64 x 64 */
  double goal;       /* > 0: the sweep reports `converged` when |E - E_last| < goal (cvgE = 1) or
                        |S - S_last| < goal (cvgE = 0); E_last starts at <psi|H|psi> of the state
                        the environments were built for (startval, algs/optimizeMPS.jl:255-258,
                        365-371), S_last at 0. 0 (the default) never converges: all sweeps run */
  int graph;         /* 1: the Lanczos step after its first Heff runs as one CUDA graph (captured
                        per step, the context's executable updated in place); 0 (default): plain
                        launches, chained by programmatic dependent launch, which measure as fast
                        or faster. Same numbers either way */
  int halfsweep;     /* 1: a sweep is L-1 bond steps in the current direction (halfsweep of
                        algs/DMRG.jl:253), the direction carrying over to the next call; 0
                        (default): 2(L-1) steps, back and forth. With a split precision and
                        fp64_final every environment update of a half sweep is FP64 */
} dmrg_params;

/* Per-sweep record (what dmrgcvg prints, algs/DMRG.jl:610-652, plus timings). */
typedef struct dmrg_sweep_stats {
  double energy;        /* energy of the last bond step of the sweep          */
  double max_truncerr;  /* maxtrunc over the sweep                            */
  int biggest_m;        /* largest kept bond dimension in the sweep           */
  int n_matvec;         /* Heff applications in the sweep                     */
  double entropy;       /* -sum D^2 log D^2 at bond svnbond, leftward step    */
  double seconds;       /* device-timed sweep duration                        */
  double heff_flops;    /* algorithmic FLOPs of all Heff applications         */
  double heff_seconds;  /* device time inside Heff applications               */
  double env_flops;     /* algorithmic FLOPs of the environment updates       */
  double env_seconds;
  double eig_seconds;   /* density-matrix formation + eigensolve + split      */
  double vec_seconds;   /* Lanczos vector operations                          */
  double d_top[8];      /* largest singular values at bond svnbond            */
  double gemm_flops;    /* profile = 1: algorithmic FLOPs of the Heff GEMM launches */
  double gemm_seconds;  /* profile = 1: their summed device time                     */
  int gemm_launches;    /* profile = 1: their number                                  */
  int eig_max_n;        /* largest density-matrix block of the sweep                  */
  double host_seconds;  /* host wall time of the sweep call                           */
  double wait_seconds;  /* of which blocked in the per-step eigenvalue synchronisation */
  int converged;        /* goal > 0 and the dmrgcvg test passed: the caller stops sweeping */
  int graph_launches;   /* graph = 1: Krylov steps that ran as one CUDA graph launch       */
  double cvg_check;     /* the tested difference (energy or entropy) when goal > 0        */
} dmrg_sweep_stats;

/* ---------------------------------------------------------------- context */
DMRG_API int dmrg_abi_version(void);
/* Creates a context on `device` (one CUDA stream). hbm_budget_bytes = 0: no budget. */
DMRG_API int dmrg_ctx_create(int device, size_t hbm_budget_bytes, dmrg_ctx** out);
DMRG_API int dmrg_ctx_destroy(dmrg_ctx* ctx);
DMRG_API const char* dmrg_last_error(const dmrg_ctx* ctx);
/* Number of kernel launches this library has issued in this process (all contexts). */
DMRG_API long long dmrg_kernel_launches(void);
/* Bytes currently allocated on the device by this context, and its peak. */
DMRG_API int dmrg_ctx_memory(const dmrg_ctx* ctx, size_t* in_use, size_t* peak);
/* The FP64 GEMM tile autotuner of the context (no reference counterpart): *signatures = block-size
 * histograms seen, *decided = of which both tile shapes were timed, *small = of which 32 x 32
 * tiles won. Any pointer may be NULL. */
DMRG_API int dmrg_ctx_tuner(dmrg_ctx* ctx, int* signatures, int* decided, int* small);

/* ---------------------------------------------------------------- MPO (MPO(...), makeMPO, makeqMPO)
 * W[i]: column-major [wl[i], d[i], d[i], wr[i]] doubles (lib/MPO/makeMPO.jl:59-92 layout).
 * phys_qn[i]: d[i]*nsym ints or NULL when nsym = 0.
 * bond_qn: NULL (labels derived with the makeqMPO largest-weight rule) or L+1 arrays of
 *          (bond dim)*nsym ints. Replaces makeqMPO (lib/MPO/makeqMPO.jl:23-84). */
DMRG_API int dmrg_mpo_upload(dmrg_ctx* ctx, int L, int nsym, const int* d, const int* wl, const int* wr,
                    const double* const* W, const int* const* phys_qn, const int* const* bond_qn,
                    dmrg_mpo** out);
DMRG_API int dmrg_mpo_destroy(dmrg_mpo* mpo);

/* ---------------------------------------------------------------- MPS
 * Dense-equivalent upload (MPS(...) / makeqMPS, lib/MPS/MPS.jl:17-37, lib/MPS/makeqMPS.jl:26-102):
 * A[i] column-major [ml[i], d[i], mr[i]] (mr[i] == ml[i+1]). bond_qn: NULL (labels from the
 * largest-magnitude element, the assignflux! rule of lib/MPS/MPS.jl:206-219) or L+1 arrays.
 * oc: 0-based orthogonality centre (psi.oc - 1). Elements in QN-forbidden positions must be 0. */
DMRG_API int dmrg_mps_upload(dmrg_ctx* ctx, const dmrg_mpo* mpo, const int* ml, const int* mr,
                    const double* const* A, const int* const* bond_qn, int oc, dmrg_state** out);
/* Block-form upload: bond b has nsec[b] sectors with charges sec_qn[b] (nsec[b]*nsym ints,
 * strictly increasing lexicographically) and sizes sec_dim[b]. data[i] holds site i's blocks in
 * canonical order: for each left sector ka (ascending), for each physical state s, if the right
 * sector with q = q(ka)+p(s) exists, the column-major block [dim ka, dim kb]. */
DMRG_API int dmrg_mps_upload_blocks(dmrg_ctx* ctx, const dmrg_mpo* mpo, const int* nsec,
                           const int* const* sec_qn, const int* const* sec_dim,
                           const double* const* data, int oc, dmrg_state** out);
/* Checkpoint of a device state (the persistence of largeMPS / loadMPS, lib/MPS/largeMPS.jl:19-81,
 * in one file instead of one file per tensor): the bond sectors, the centre, the sweep direction
 * and every site's blocks, with a checksum. Environments are not stored: after dmrg_state_load
 * call dmrg_env_build (the rebuilt environments equal the ones a sweep leaves, bit for bit, so a
 * resumed run continues exactly as an uninterrupted one). */
DMRG_API int dmrg_state_save(dmrg_state* st, const char* path);
/* Reads a checkpoint into a new state for `mpo` (same length, charges and physical dimensions as
 * the state that was saved; DMRG_ERR_SHAPE / DMRG_ERR_QN otherwise, DMRG_ERR_ARG for a corrupt or
 * truncated file). */
DMRG_API int dmrg_state_load(dmrg_ctx* ctx, const dmrg_mpo* mpo, const char* path,
                             dmrg_state** out);
DMRG_API int dmrg_state_destroy(dmrg_state* st);
DMRG_API int dmrg_state_oc(const dmrg_state* st, int* oc);
/* Sector structure of bond b: *nsec; if qn/dims are non-NULL they receive nsec*nsym / nsec ints. */
DMRG_API int dmrg_bond_info(const dmrg_state* st, int bond, int* nsec, int* qn, int* dims);
/* Number of doubles of site i in block form. */
DMRG_API int dmrg_site_size(const dmrg_state* st, int site, int64_t* n_blocks_doubles);
DMRG_API int dmrg_mps_download_blocks(dmrg_state* st, int site, double* out);
/* Every site's blocks at once, back to back (site 0 first), with one synchronisation; sizes
 * (L entries, optional) gets each site's count in doubles, and a NULL
 * `out` only fills sizes. No counterpart in the reference: the download side of the state copy
 * that dmrg() makes (the per-site dmrg_mps_download_blocks, batched). */
DMRG_API int dmrg_mps_download_all_blocks(dmrg_state* st, double* out, int64_t* sizes);
/* Every bond's sectors at once: nsec[b] for b = 0..L, and (optional) the sectors' charges
 * (nsym ints each) and dims, bond 0 first. The batched form of dmrg_bond_info. */
DMRG_API int dmrg_bonds_info(const dmrg_state* st, int* nsec, int* qn, int* dims);
/* Dense-equivalent download of site i: out [ml, d, mr] column-major in the grouped bond order;
 * ml/mr receive the bond sizes (out may be NULL to query them). */
DMRG_API int dmrg_mps_download(dmrg_state* st, int site, double* out, int* ml, int* mr);

/* ---------------------------------------------------------------- environments
 * makeEnv(psi, mpo) (lib/Env/makeEnv.jl:196-221): boundary ones(1,1,1), Lenv[0..oc], Renv[oc..L-1]. */
DMRG_API int dmrg_env_build(dmrg_state* st, const dmrg_mpo* mpo);
/* Lupdate!(i, Lenv, psi, mpo): Lenv[i+1] = Lupdate(Lenv[i], psi[i], psi[i], mpo[i])
 * (lib/MPO_MPS/Lupdate.jl:17-37). Requires Lenv[i]. */
DMRG_API int dmrg_lupdate(dmrg_state* st, const dmrg_mpo* mpo, int site);
/* Rupdate!(i, Renv, psi, mpo): Renv[i-1] = Rupdate(Renv[i], ...) (lib/MPO_MPS/Rupdate.jl:17-37). */
DMRG_API int dmrg_rupdate(dmrg_state* st, const dmrg_mpo* mpo, int site);
/* Lupdate(Lenv, dualpsi, psi, mpo) / Rupdate(Renv, dualpsi, psi, mpo) as pure functions of dense
 * host tensors (lib/MPO_MPS/Lupdate.jl:17-26, lib/MPO_MPS/Rupdate.jl:17-26), computed on the device:
 *   left = 1: env_in = L[ml(bra), wl, ml(ket)], env_out = L'[mr(bra), wr, mr(ket)]
 *   left = 0: env_in = R[mr(ket), wr, mr(bra)], env_out = R'[ml(ket), wl, ml(bra)]
 * psi and dual are [ml, d, mr] sites (dual = NULL: the same tensor as psi), W is [wl, d, d, wr];
 * all column-major. */
DMRG_API int dmrg_env_step(dmrg_ctx* ctx, int left, int ml, int d, int mr, int wl, int wr,
                           const double* env_in, const double* dual, const double* psi,
                           const double* W, double* env_out);
/* Lenv[i] (left=1) or Renv[i] (left=0) as a dense-equivalent column-major [m, w, m] array
 * (L[bra,w,ket] / R[ket,w,bra]). dims receives the 3 sizes; out may be NULL to query them. */
DMRG_API int dmrg_env_get(dmrg_state* st, int site, int left, double* out, int* dims);

/* ---------------------------------------------------------------- contractions (tests / Env API)
 * Two-site effective Hamiltonian on sites (iL, iL+1) applied to a dense-equivalent vector
 * psi_in [ml, d1, d2, mr] (make2site / inline Heff, algs/DMRG.jl:48-54,69-73), psi_out same shape.
 * Uses Lenv[iL] and Renv[iL+1]. precision: enum dmrg_precision. */
DMRG_API int dmrg_heff_apply(dmrg_state* st, const dmrg_mpo* mpo, int iL, const double* psi_in,
                    double* psi_out, int precision);
/* Same product as dmrg_heff_apply for callers that cannot allocate device memory at this point
 * (for example a host framework whose caching allocator already owns all free HBM, or a solver
 * loop that must not call the allocator). No reference counterpart: the reference allocates every
 * intermediate itself. psi_in and psi_out are DEVICE pointers to dense-equivalent
 * [ml, d1, d2, mr] column-major vectors; every intermediate lives in one fixed device array inside
 * the library (9 MiB per GPU that loads the library, kept until exit), limited to 2^20 doubles of
 * vector/intermediate data and 1 MiB of task descriptors: larger two-site spaces are rejected with
 * DMRG_ERR_BUDGET. Nothing is allocated, no cudaMalloc/cudaFree is called. The call runs on the context's own stream, which is not ordered after the caller's streams:
 * finish writing psi_in first (for example synchronise the stream that produced it). psi_in and
 * psi_out may be the same buffer (the input is read completely before the output is written).
 * Calls share the array: calls that overlap on the GPU race. Returns after the result is written. */
DMRG_API int dmrg_heff_apply_noalloc(dmrg_state* st, const dmrg_mpo* mpo, int iL,
                                     const double* psi_in, double* psi_out, int precision);
/* Dense-equivalent dims of the two-site space at (iL, iL+1): dims[4] = {ml, d1, d2, mr}. */
DMRG_API int dmrg_twosite_dims(const dmrg_state* st, const dmrg_mpo* mpo, int iL, int* dims);

/* ---------------------------------------------------------------- measurements
 * expect(psi, H) (lib/MPO_MPS/expect.jl:19-56): *value = <psi|H|psi> for an MPO H over the same
 * sites and physical charges as the state's own MPO (H may differ from it), not normalised, as in
 * the reference. The state's environments and centre are left as they are. */
DMRG_API int dmrg_expect(dmrg_state* st, const dmrg_mpo* H, double* value);
/* correlationmatrix(psi, Cc, Ca; trail) (lib/MPO_MPS/correlationmatrix.jl:21-83): rho [L, L]
 * column-major with rho[i,j] = <psi|(Cc F)_i F_{i+1}..F_{j-1} Ca_j|psi> / <psi|psi> for i < j,
 * rho[j,i] = rho[i,j] and rho[i,i] = <psi|(Cc Ca)_i|psi> / <psi|psi>. Cc, Ca and the trail F are
 * d x d column-major operators O[bra, ket] applied on every site (every site must have physical
 * dimension d); trail may be NULL (no string). Under charge conservation each operator must change
 * the charge by one fixed amount (DMRG_ERR_QN otherwise). The reference moves the orthogonality
 * centre to each site as a side effect; this call leaves the centre where it is (the values are
 * gauge-invariant and agree with the reference's for a normalised state). */
DMRG_API int dmrg_correlationmatrix(dmrg_state* st, int d, const double* Cc, const double* Ca,
                                    const double* trail, double* rho);

/* correlation(psi, ops...; sites, trail) (lib/MPO_MPS/correlation.jl:98-237) with dualpsi = psi:
 * omega[p_1, ..., p_n] = <psi| prod_s O(s) |psi>, not normalised, with O(s) = A_1(s) ... A_n(s)
 * and A_g(s) = trail_g left of operator g, factor s - p_g of operator g on its oplen[g]
 * consecutive sites, the identity elsewhere (the order in which the reference applies them).
 * ops: the factors of every operator, d x d column-major O[bra, ket], operator 1 first; sites:
 * nsites[g] 0-based start candidates of operator g, concatenated, of which the first
 * nsites[g] - oplen[g] + 1 are used (as in the reference); trails: nops matrices or NULL (an
 * identity trail is none). omega: prod_g (nsites[g] - oplen[g] + 1) values, operator 1's index
 * fastest. The reference indexes its result by the site numbers themselves, so the two agree
 * when every sites list is 0, 1, ...; for three or more operators the reference reuses right
 * environments of an earlier position combination (its Renv array is updated in place from the
 * rightmost operator of the current combination, which can lie left of the previous one's), and
 * its values there differ from the definition above, which this computes. */
DMRG_API int dmrg_correlation(dmrg_state* st, int d, int nops, const int* oplen,
                              const double* ops, const int* nsites, const int* sites,
                              const double* trails, double* omega);

/* ---------------------------------------------------------------- the sweep
 * One optmps sweep (algs/optimizeMPS.jl:790-835): 2(L-1) twostep calls, each followed by an
 * environment update; the centre reverses at the edges. Requires dmrg_env_build first. */
DMRG_API int dmrg_sweep(dmrg_state* st, const dmrg_mpo* mpo, const dmrg_params* p, dmrg_sweep_stats* out);

/* Noise schedule of the single-site sweep with subspace expansion (method "3S"): the
 * noise / noise_goal / noise_incr fields of algvars (algs/optimizeMPS.jl:528-532). */
typedef struct dmrg_noise {
  double noise;       /* alpha, the weight of the expansion term (default 1.0): in = its value at the
                         start of the sweep, out = after the sweep's last alpha_update           */
  double noise_goal;  /* default 0.3: the site condition of alpha_update (algs/DMRG.jl:289-302) */
  double noise_incr;  /* default 0.01: alpha's relative step; the centre is expanded while
                         alpha > noise_incr (alpha_condition, algs/DMRG.jl:335)                */
  double reserved;
} dmrg_noise;

/* Fills *nz with the reference defaults (noise 1.0, noise_goal 0.3, noise_incr 0.01). */
DMRG_API void dmrg_noise_default(dmrg_noise* nz);

/* One optmps sweep with step3S (algs/DMRG.jl:324-360, dmrg3S :655-671): 2(L-1) single-site steps
 * (Krylov solve of the single-site Heff with max(2, krylov) vectors, expansion by Lexpand /
 * Rexpand while alpha > noise_incr, truncated move of the centre with weights relative to the
 * total (moveR! / moveL! with condition, lib/MPS/move.jl:124-199), alpha_update), each followed
 * by an environment update. p: maxm, minm, cutoff, krylov, precision, svnbond, degen_rtol,
 * betatest, fp64_final, profile, tune, graph, goal and cvgE as for dmrg_sweep. The lastEnergy of
 * alpha_update is the previous sweep's energy (the starting energy <psi|H|psi> for the first
 * sweep after dmrg_env_build); with cvgE = 0 it stays the starting energy (dmrgcvg,
 * algs/DMRG.jl:626-652). max_truncerr is relative to the total weight of each step. */
DMRG_API int dmrg_sweep3s(dmrg_state* st, const dmrg_mpo* mpo, const dmrg_params* p,
                          dmrg_noise* nz, dmrg_sweep_stats* out);

/* One call of tdvp_twosite (twosite = 1, algs/time.jl:288-363) or tdvp (twosite = 0, :211-286)
 * with a real prefactor: L-1 steps from the centre (rightward from the left edge or an interior
 * centre, leftward from the right edge), turning at the edge. Each step applies exp(tau H) by
 * krylovTimeEvol (:182-203: Lanczos with max(2, krylov) vectors, the combination exp(tau T) e_1;
 * tau = prefactor / (L-1) / 2 two-site, prefactor / L / 2 single-site) to the two-site tensor and
 * then to the site left as centre (two-site), or to the site and then to the bond matrix through
 * the zero-site Heff (single-site), with a truncated move (maxm, minm, cutoff, weights relative to
 * the total) and the environment update between; the new centre is normalised.
 * p: maxm (the `m` keyword), minm, cutoff, krylov (`r`), precision, degen_rtol, betatest, tune,
 * graph, profile. out->energy = En of the last Krylov call (the lowest eigenvalue of its
 * tridiagonal), out->max_truncerr / biggest_m / timings as for a sweep.
 * The single-site reference runs L steps and its last one reads past the chain's end (its turn
 * test compares the centre with L+1); this call stops at the edge instead. A complex prefactor
 * (real-time evolution) needs complex tensors and is not available. Requires dmrg_env_build. */
DMRG_API int dmrg_tdvp(dmrg_state* st, const dmrg_mpo* mpo, const dmrg_params* p,
                       double prefactor, int twosite, dmrg_sweep_stats* out);
/* ---------------------------------------------------------------- kernel test hooks
 * No reference counterpart: these expose single device kernels to the parity tests.
 * C[M,N] = op(A) op(B) with the grouped FP64 GEMM (one task, one K segment), host arrays,
 * column-major with leading dimensions lda/ldb/ldc; op = transpose when trans* != 0. */
DMRG_API int dmrg_test_gemm(dmrg_ctx* ctx, int transA, int transB, int M, int N, int K,
                            const double* A, int lda, const double* B, int ldb, double* C, int ldc);
/* Batched symmetric eigensolve (the truncation's Jacobi kernel): nmat column-major matrices of
 * sizes n[i] packed back to back in A; eigenvalues (descending) packed into w and eigenvectors
 * (columns) overwrite A. */
DMRG_API int dmrg_test_eigh(dmrg_ctx* ctx, int nmat, const int* n, double* A, double* w);

/* Tridiagonal-path eigensolver (n[i] <= 512; blocks above 112 take the mid-size kernels): all
 * eigenvalues (descending, packed in w) and the
 * eigenvectors of the k[i] largest (packed n[i] x k[i] column-major in U). A is overwritten. */
DMRG_API int dmrg_test_syevt(dmrg_ctx* ctx, int nmat, const int* n, const int* k, double* A,
                             double* w, double* U);

/* Device time of the two-site Heff at (iL, iL+1) in the given precision: `reps` applications to
 * a device-resident vector timed with CUDA events on the context's stream (no host copies).
 * *seconds = time per application, *flops = its algorithmic FLOPs (block GEMMs + MPO mixing). */
DMRG_API int dmrg_test_heff_time(dmrg_state* st, const dmrg_mpo* mpo, int iL, int precision,
                                 int reps, double* seconds, double* flops);

/* Test hook (no counterpart in the reference): dmrg_heff_apply's result after `reps` >= 1
 * applications of one Heff plan to psi_in. From the second application on, the split forms reuse
 * the environment images the first one packed, as the Lanczos iterations of a bond step do; the
 * result equals one application's bit for bit. */
DMRG_API int dmrg_test_heff_apply_repeat(dmrg_state* st, const dmrg_mpo* mpo, int iL,
                                         const double* psi_in, double* psi_out, int precision,
                                         int reps);

/* Fills *p with the reference defaults (minm 2, krylov 2, betatest 1e-10, ...). */
DMRG_API void dmrg_params_default(dmrg_params* p);

/* ---------------------------------------------------------------- serving
 * Many independent ground-state solves on one GPU: each request is what one call of
 * dmrg(psi, mpo; m, minm, sweeps, cutoff) computes (algs/DMRG.jl:549-588), submitted
 * asynchronously. The server runs up to `slots` solves at once, one host worker thread and one
 * context (CUDA stream) each, so that the latency-bound bond steps of different solves overlap on
 * the GPU; a request starts as soon as a slot is free and its worst-case device footprint fits
 * in what the running solves leave of `hbm_budget_bytes` (continuous admission, first come first
 * served). Inside their sweeps the solves' Heff applications are gathered into shared grouped
 * launches (one per phase for all solves at a Lanczos step). A solve's results do not depend on
 * the other solves running beside it: every block is computed as in a launch of its own. */
typedef struct dmrg_server dmrg_server;

typedef struct dmrg_server_config {
  int device;
  int slots;                 /* concurrent solves, >= 1 */
  size_t hbm_budget_bytes;   /* 0: no budget (slots alone limit admission) */
  int unbatched;             /* 0 (default): the Heff applications of all solves inside their
                                sweeps share grouped launches (continuous batching); 1: every
                                solve launches its own */
  int reserved[7];
} dmrg_server_config;

/* One solve. Same arrays and conventions as dmrg_mpo_upload / dmrg_mps_upload (dense-equivalent
 * column-major tensors, physical charges per site or NULL for nsym = 0, bond labels derived).
 * The server copies everything during dmrg_server_submit. */
typedef struct dmrg_request {
  int L, nsym;
  const int* d;                      /* [L] physical dimensions */
  const int* wl; const int* wr;      /* [L] MPO bond dimensions */
  const double* const* W;            /* [L] MPO sites [wl, d, d, wr] */
  const int* const* phys_qn;         /* [L] d*nsym charges, or NULL when nsym = 0 */
  const int* ml; const int* mr;      /* [L] MPS bond dimensions */
  const double* const* A;            /* [L] MPS sites [ml, d, mr] */
  int oc;                            /* 0-based orthogonality centre */
  int sweeps;
  dmrg_params params;
} dmrg_request;

enum dmrg_request_status {
  DMRG_REQ_QUEUED = 0, DMRG_REQ_RUNNING = 1, DMRG_REQ_DONE = 2, DMRG_REQ_FAILED = 3
};

typedef struct dmrg_result {
  int status;                 /* enum dmrg_request_status */
  int error;                  /* dmrg_status of a failed solve */
  double energy;              /* last bond step of the last sweep (what dmrg returns) */
  double max_truncerr;        /* of the last sweep */
  double entropy;             /* of the last sweep, bond SvNbond */
  int biggest_m;
  int sweeps_done;
  double queue_seconds;       /* submit -> start */
  double run_seconds;         /* start -> done (upload, sweeps, download) */
  size_t footprint_bytes;     /* admission estimate */
} dmrg_result;

DMRG_API int dmrg_server_create(const dmrg_server_config* cfg, dmrg_server** out);
/* Copies the request and queues it; *ticket identifies it. Rejects (DMRG_ERR_BUDGET) a request
 * whose footprint alone exceeds the budget. */
DMRG_API int dmrg_server_submit(dmrg_server* s, const dmrg_request* req, long long* ticket);
/* Status and statistics of a ticket, waiting up to wait_ms milliseconds for it to finish
 * (0: no wait, < 0: until it finishes). */
DMRG_API int dmrg_server_poll(dmrg_server* s, long long ticket, int wait_ms, dmrg_result* out);
/* Final MPS site of a finished ticket, dense-equivalent [ml, d, mr] in the grouped bond order
 * (out NULL: sizes only), as dmrg_mps_download; *oc receives the final centre when non-NULL. */
DMRG_API int dmrg_server_fetch_site(dmrg_server* s, long long ticket, int site, double* out,
                                    int* ml, int* d, int* mr, int* oc);
/* Forgets a finished ticket (its host copy of the final MPS). */
DMRG_API int dmrg_server_release(dmrg_server* s, long long ticket);
/* Finishes the queued and running solves, then stops the workers. */
DMRG_API int dmrg_server_destroy(dmrg_server* s);
DMRG_API const char* dmrg_server_last_error(const dmrg_server* s);
/* Shared-launch statistics since the server started: *batches = rounds of shared Heff launches
 * (each one launch per phase and form), *contributions = Heff applications they carried
 * (contributions / batches = mean number of solves per shared launch). */
DMRG_API int dmrg_server_stats(dmrg_server* s, long long* batches, long long* contributions);

#ifdef __cplusplus
}
#endif
#endif /* DMRG_B200_H */
