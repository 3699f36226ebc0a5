/*
 * dmrg_b200.h - C ABI of libdmrg_b200, the sm_100a implementation of the
 * dmrgcc DMRG hot path (block-sparse H_eff*psi, environment updates, Lanczos,
 * per-sector SVD truncation).
 *
 * The reference (jiandong94/dmrgcc) has no FFI: its hot path is reached through
 * C++ member functions whose numeric work bottoms out in MKL.  Each entry point
 * below names the reference member it stands in for.  All arguments are plain
 * pointers and sizes.  Every call returns 0 on success or a negative DMRG_E*
 * code; dmrg_last_error() gives the message.  No entry point exits the process.
 *
 * Storage conventions (identical to the reference's):
 *   - a block list ("RealMatrixBlock") is an ordered list of dense blocks, each
 *     row-major, packed back to back in list order (VectorizeMatrixBlock,
 *     src/tensor/real_matrix_block.cc:173-194).  A site tensor's packed storage
 *     IS the Lanczos vector;
 *   - an environment is one block list per MPO bond index, packed index-major;
 *   - the MPO site tensor W is dense [left_bond][right_bond][d][d] (row p1,
 *     column p2), as RealTensorOperator::tensor_operator_[l][r](p1, p2).
 * Device pointers ("_dev") are CUDA global memory on the context's device;
 * host pointers ("_host") are ordinary (optionally pinned) host memory.
 */
#ifndef DMRG_B200_H_
#define DMRG_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DMRG_OK 0
#define DMRG_E_ARG (-1)      /* invalid argument / inconsistent block shapes */
#define DMRG_E_CUDA (-2)     /* a CUDA runtime call failed */
#define DMRG_E_NOMEM (-3)    /* device allocation failed */
#define DMRG_E_NUMERIC (-4)  /* an iterative device routine hit its iteration cap */
#define DMRG_E_STATE (-5)    /* call made in the wrong state */
#define DMRG_E_IO (-6)       /* a file could not be opened, read or written, or is malformed */

/* Arithmetic of the block GEMMs.  FP64: plain double (FP64 tensor path).
 * TF32X3 / BF16X3: 5th-generation tensor cores (tcgen05): every FP64 operand is
 * split into hi + lo parts (TF32 after rounding to FP32, or BF16), each product
 * is taken as hi*hi + hi*lo + lo*hi with FP32 accumulation in tensor memory,
 * the terms of a block sum are added in FP64 and results are stored as FP64
 * (relative error of a block sum ~1e-6 for TF32X3, ~1e-5 for BF16X3). */
#define DMRG_PREC_FP64 0
#define DMRG_PREC_BF16X3 1
#define DMRG_PREC_TF32X3 2

typedef struct dmrg_ctx_s* dmrg_ctx_t;
typedef struct dmrg_heff_s* dmrg_heff_t;
typedef struct dmrg_env_s* dmrg_env_t;
typedef struct dmrg_canon_s* dmrg_canon_t;
typedef struct dmrg_run_s* dmrg_run_t;
typedef struct dmrg_model_s* dmrg_model_t;

/* Shape of one block list: block k has sector indices (left[k], right[k]) and a
 * rows[k] x cols[k] row-major matrix.  Stands in for RealMatrixBlock's
 * left_index_/right_index_/matrix_block_ (src/tensor/real_matrix_block.h:6-40). */
typedef struct {
    int nblocks;
    const int* left;
    const int* right;
    const int* rows;
    const int* cols;
} dmrg_blocks_t;

/* ---- context --------------------------------------------------------------- */
const char* dmrg_version(void);
/* Last error message of this thread (never NULL). */
const char* dmrg_last_error(void);
/* Creates a context on CUDA device `device` with its own non-blocking stream. */
int dmrg_ctx_create(int device, dmrg_ctx_t* out);
int dmrg_ctx_destroy(dmrg_ctx_t ctx);
/* Replaces the context's stream (a cudaStream_t passed as void*; NULL = own). */
int dmrg_ctx_set_stream(dmrg_ctx_t ctx, void* stream);
void* dmrg_ctx_stream(dmrg_ctx_t ctx);
int dmrg_ctx_sync(dmrg_ctx_t ctx);
/* Device memory helpers for callers without their own allocator. */
int dmrg_malloc(dmrg_ctx_t ctx, size_t bytes, void** dev);
int dmrg_free(dmrg_ctx_t ctx, void* dev);
int dmrg_memcpy_h2d(dmrg_ctx_t ctx, void* dst_dev, const void* src_host, size_t bytes);
int dmrg_memcpy_d2h(dmrg_ctx_t ctx, void* dst_host, const void* src_dev, size_t bytes);
int dmrg_memset(dmrg_ctx_t ctx, void* dev, int value, size_t bytes);
/* Seeded synthetic values for benchmarks and tests: dev[i] = element start+i of
 * the splitmix64 stream seeded with `seed`, mapped to [-1, 1).  No reference
 * counterpart (the reference draws its random tensors from glibc rand()). */
int dmrg_fill_uniform(dmrg_ctx_t ctx, double* dev, int64_t n, uint64_t seed, int64_t start);
/* FP64 throughput of this GPU, measured by a register-only loop of DMMA
 * (mode 0) or DFMA (mode 1) instructions on all SMs: the roofline denominator
 * of the FP64 block GEMMs.  No reference counterpart. */
int dmrg_fp64_peak(dmrg_ctx_t ctx, int mode, int iters, double* tflops);
/* Number of kernels this library has launched in this process, on any context
 * (for launch accounting in benchmarks).  No reference counterpart. */
int dmrg_launch_count(int64_t* count);

/* ---- a1: H_eff * psi --------------------------------------------------------
 * Replaces RealTensorContraction::MultiplyEffectHamilton(RealTensorLattice*,
 * RealTensorOperator*, double* state)
 * (src/dmrg/realdmrg/real_tensor_contraction.h:91-92, .cc:1223-1291).
 *
 * dmrg_heff_create builds the block-product schedule once per site from the
 * site tensor's block list `ket` (sector pair of each block and its physics
 * index physics_index[num_left_sector * num_right_sector], -1 = no block),
 * the dense MPO tensor W and the block structure of the left environment
 * L[0..left_bond) and right environment R[0..right_bond) (L blocks are
 * (bra, ket) sector pairs, R blocks (ket, bra), as in the reference).
 * precision: DMRG_PREC_*. */
int dmrg_heff_create(dmrg_ctx_t ctx, int num_left_sector, int num_right_sector,
                     const int* physics_index, const dmrg_blocks_t* ket, int physics_dim,
                     int left_bond, int right_bond, const double* W, const dmrg_blocks_t* L,
                     const dmrg_blocks_t* R, int precision, dmrg_heff_t* out);
/* The same operator for a tensor whose blocks carry their own physics index
 * (block_phys[ket->nblocks], each in [0, physics_dim)) instead of one index per
 * sector pair; blocks may then share a sector pair.  This is the two-site
 * effective Hamiltonian: the two-site tensor Theta(k, p1, p2, l) has one block
 * per (left sector k, middle sector m, right sector l) with combined index
 * p1 * d + p2, and W is the two-site MPO W_j W_{j+1} contracted over their
 * shared bond ([left_bond][right_bond][d*d][d*d]).  The reference is
 * single-site only (MultiplyEffectHamilton, real_tensor_contraction.cc:
 * 1223-1291, is this operator with one site's W); there is no counterpart. */
int dmrg_heff_create_blocks(dmrg_ctx_t ctx, int num_left_sector, int num_right_sector,
                            const int* block_phys, const dmrg_blocks_t* ket, int physics_dim,
                            int left_bond, int right_bond, const double* W, const dmrg_blocks_t* L,
                            const dmrg_blocks_t* R, int precision, dmrg_heff_t* out);
int dmrg_heff_destroy(dmrg_heff_t h);
/* Number of doubles of the packed site tensor / left env / right env. */
int dmrg_heff_sizes(dmrg_heff_t h, int64_t* psi_dim, int64_t* left_env_size,
                    int64_t* right_env_size);
/* FLOPs of one application: `algorithmic` counts the reference loop's GEMMs
 * (real_tensor_contraction.cc:1243-1285), `executed` what the schedule runs. */
int dmrg_heff_flops(dmrg_heff_t h, double* algorithmic, double* executed);
/* Points the operator at device-resident environments (packed as above).  The
 * pointers must stay valid while the operator is used. */
int dmrg_heff_set_env(dmrg_heff_t h, const double* L_dev, const double* R_dev);
/* out_dev (+)= H_eff * psi_dev on the context stream (accumulate != 0 adds into
 * out_dev like the reference's `state +=`; 0 overwrites).  Asynchronous. */
int dmrg_heff_apply(dmrg_heff_t h, const double* psi_dev, double* out_dev, int accumulate);
/* Same with host buffers: copies psi in, applies, copies the result out, and
 * waits.  This is the drop-in for the reference call on a host `state`. */
int dmrg_heff_apply_host(dmrg_heff_t h, const double* psi_host, double* out_host, int accumulate);
/* One accumulating application with CUDA events between its two grouped
 * launches (K*R products, then L*(KR) sums); waits and returns each launch's
 * duration in milliseconds.  For roofline accounting; no reference counterpart. */
int dmrg_heff_profile(dmrg_heff_t h, const double* psi_dev, double* out_dev, double* ms_stage_a,
                      double* ms_stage_b);

/* The same H_eff * psi for callers that cannot call cudaMalloc (for example a
 * host framework that owns every device allocation under a fixed budget).  No
 * reference counterpart: the reference has no device code.  It allocates
 * nothing: it takes the block structure directly (as dmrg_heff_create) plus the
 * device environments, psi and out, and keeps its schedule and the K*R
 * intermediate in one static device array of 16 MiB per GPU that loads the
 * library (held until exit).  Problems needing more return DMRG_E_ARG with the
 * size required.  All calls share that array: calls that overlap on the GPU
 * race (calls from different host threads are serialised by a lock held until
 * the call's own stream synchronisation, so only work queued on the GPU by other
 * means can overlap).  The first call on a device looks up the array's device
 * address and keeps it for the life of the process; make it before any stream
 * capture, and do not use the library across a cudaDeviceReset.  Every table is
 * validated on the host first (sectors in range, each ket block's physics index
 * in [0, physics_dim)); a malformed one returns DMRG_E_ARG before any CUDA
 * call.  Runs on `stream` (a cudaStream_t; NULL = the legacy default stream) and
 * returns after the work is queued and the schedule copied (it synchronises
 * `stream`). */
int dmrg_heff_apply_noalloc(int num_left_sector, int num_right_sector, const int* physics_index,
                            const dmrg_blocks_t* ket, int physics_dim, int left_bond, int right_bond,
                            const double* W, const dmrg_blocks_t* L, const dmrg_blocks_t* R,
                            const double* L_dev, const double* R_dev, const double* psi_dev,
                            double* out_dev, int accumulate, void* stream);

/* ---- a4/a5: Lanczos ground state of H_eff ----------------------------------
 * Replaces RealTensorLanczos::LanczosMethod(int num_iter, int site, double& result)
 * (src/dmrg/realdmrg/real_tensor_lanczos.h:23, .cc:14-201).  psi_dev holds the
 * start vector (the site tensor, packed; used as is, like the reference) and
 * receives the ground vector.  Stops like the reference: beta < zero_tol,
 * |E_i - E_{i-1}| < precision (the reference hard-codes both at 1e-15), or
 * niter iterations.  psi_dim < 100 uses the reference's dense exact
 * diagonalisation branch (.cc:34-56).  *iters = Krylov dimension (0 for the
 * dense branch).  niter <= 512.  Synchronous. */
int dmrg_lanczos(dmrg_heff_t h, double* psi_dev, int niter, double precision, double zero_tol,
                 double* energy, int* iters);
/* For a split-precision operator (DMRG_PREC_TF32X3 / BF16X3), dmrg_lanczos runs
 * a Krylov phase on split-precision matvecs and then an FP64 Krylov run from its
 * Ritz vector, when psi_dim >= min_psi_dim (default 200000: below it the split
 * matvec is not enough faster to pay for two phases and the FP64 run is used
 * alone).  No reference counterpart (the reference has FP64 only). */
int dmrg_heff_set_split_threshold(dmrg_heff_t h, int64_t min_psi_dim);
/* Length of that FP64 run, process-wide: iters > 0 (default 4) FP64 matvecs,
 * whose lowest Ritz value is the energy (its error quadratic in the split
 * vector's) and whose Ritz vector the state; iters <= 0: the FP64 Lanczos to the
 * reference's own convergence. */
int dmrg_lanczos_set_polish(int iters);
/* Krylov dimension of the split phase of the last dmrg_lanczos call (0 when it
 * ran FP64 only). */
int dmrg_heff_split_iters(dmrg_heff_t h, int* iters);
/* enable != 0 (the default; environment variable DMRG_LANCZOS_GRAPH=0 changes
 * it for new operators): dmrg_lanczos runs its Krylov loop as one CUDA graph
 * launch, a conditional WHILE node whose body is one iteration (matvec, the
 * recurrence, the tridiagonal step and convergence test, the
 * reorthogonalisation) with the iteration index kept on the device, captured on
 * first use and relaunched while niter and the stopping constants stay the
 * same; the host reads the result once per run.  0: one launch per kernel and
 * a host read of the convergence flag every few iterations.  Both give
 * bit-identical results.  Replaces the iteration loop of
 * RealTensorLanczos::LanczosMethod (real_tensor_lanczos.cc:57-185). */
int dmrg_heff_set_graph(dmrg_heff_t h, int enable);

/* ---- the complex path (complex128) -------------------------------------------
 * Complex values are interleaved (re, im) doubles, the layout of the reference's
 * Complex (src/tensor/complex.h:15-16) and of cuDoubleComplex; offsets and
 * sizes count complex elements.
 *
 * dmrg_zheff_*: ComplexTensorContraction::MultiplyEffectHamilton
 * (src/dmrg/complexdmrg/complex_tensor_contraction.cc:1244-1312): the same
 * arguments as dmrg_heff_create with a complex MPO W ([lb][rb][d][d] complex);
 * products on the FP64 tensor path as four real products per complex product.
 * dmrg_zlanczos: ComplexTensorLanczos::LanczosMethod (complex_tensor_lanczos.cc:
 * 14-160; the conjugated inner product, :162-169), same stopping rule and
 * dense branch (psi_dim < 100) as dmrg_lanczos.  *flops: real FLOPs of one
 * application over the reference loop. */
typedef struct dmrg_zheff_s* dmrg_zheff_t;
int dmrg_zheff_create(dmrg_ctx_t ctx, int num_left_sector, int num_right_sector, const int* physics_index,
                      const dmrg_blocks_t* ket, int physics_dim, int left_bond, int right_bond,
                      const double* W, const dmrg_blocks_t* L, const dmrg_blocks_t* R, dmrg_zheff_t* out);
int dmrg_zheff_destroy(dmrg_zheff_t h);
int dmrg_zheff_sizes(dmrg_zheff_t h, int64_t* psi_dim, int64_t* left_env_size, int64_t* right_env_size,
                     double* flops);
int dmrg_zheff_set_env(dmrg_zheff_t h, const double* L_dev, const double* R_dev);
int dmrg_zheff_apply(dmrg_zheff_t h, const double* psi_dev, double* out_dev, int accumulate);
int dmrg_zlanczos(dmrg_zheff_t h, double* psi_dev, int niter, double precision, double zero_tol,
                  double* energy, int* iters);
/* Complex environment update: ComplexTensorContraction::Left/Right
 * ComputeTensorContraction (complex_tensor_contraction.cc:800-975, 977-1150;
 * the bra block Hermitian-conjugated, :929, :1113).  Same arguments as
 * dmrg_env_create with a complex MPO W; the handle answers dmrg_env_out_info /
 * _out_blocks / _flops (real FLOPs) and is applied by dmrg_zenv_apply on
 * complex ket and environments.  Released by dmrg_env_destroy. */
int dmrg_zenv_create(dmrg_ctx_t ctx, int side, int num_left_sector, int num_right_sector,
                     const int* physics_index, const dmrg_blocks_t* ket, int physics_dim, int left_bond,
                     int right_bond, const double* W, const dmrg_blocks_t* env_in, dmrg_env_t* out);
int dmrg_zenv_apply(dmrg_env_t e, const double* ket_dev, const double* env_in_dev, double* env_out_dev);
/* Complex canonicalisation: ComplexTensorLattice::Left/RightCanonicalTensorLattice
 * (src/dmrg/complexdmrg/complex_tensor_lattice.cc; per-sector zgesdd through
 * ComplexMatrix::SVDMatrix, src/tensor/complex_matrix.cc:601-638, and
 * ComputeTruncateDim).  The same calls as dmrg_canon_* on complex data: each
 * sector's SVD runs on the device as the batched Jacobi SVD of its real form
 * [[Re A, -Im A], [Im A, Re A]], whose complex singular triplets are recovered
 * on the host; the new ket takes U (side 0) or V^H (side 1), the canonical
 * tensor S V^H or U S.  Singular-vector phases are free, as with zgesdd. */
typedef struct dmrg_zcanon_s* dmrg_zcanon_t;
int dmrg_zcanon_create(dmrg_ctx_t ctx, int side, int num_left_sector, int num_right_sector,
                       const int* left_dim, const int* right_dim, const dmrg_blocks_t* ket,
                       dmrg_zcanon_t* out);
int dmrg_zcanon_destroy(dmrg_zcanon_t c);
int dmrg_zcanon_run(dmrg_zcanon_t c, const double* ket_dev, int max_dim, double canpre, int* tdim_out,
                    double* discarded);
int dmrg_zcanon_out_info(dmrg_zcanon_t c, int64_t* ket_size, int64_t* canonical_size, int* sweeps);
int dmrg_zcanon_out_blocks(dmrg_zcanon_t c, int* ket_rows, int* ket_cols, int* canon_rows,
                           int* canon_cols, int* match_dim);
int dmrg_zcanon_singular_values(dmrg_zcanon_t c, int sector, int cap, double* values, int* count);
int dmrg_zcanon_write(dmrg_zcanon_t c, const double* ket_dev, double* new_ket_dev, double* canonical_dev);

/* ---- a2/a3: environment update ---------------------------------------------
 * side 0 replaces RealTensorContraction::LeftComputeTensorContraction
 * (real_tensor_contraction.cc:782-940): env_in = L[0..left_bond) of this site,
 * result = L[0..right_bond) of the next site.  side 1 replaces
 * RightComputeTensorContraction (:959-1119): env_in = R[0..right_bond), result =
 * R[0..left_bond) of the previous site.  The result's block structure (the
 * reference's zero_flag pass, :797-883 / :974-1060) is decided at create time
 * and can be read back with dmrg_env_out_blocks. */
int dmrg_env_create(dmrg_ctx_t ctx, int side, int num_left_sector, int num_right_sector,
                    const int* physics_index, const dmrg_blocks_t* ket, int physics_dim,
                    int left_bond, int right_bond, const double* W, const dmrg_blocks_t* env_in,
                    int precision, dmrg_env_t* out);
int dmrg_env_destroy(dmrg_env_t e);
/* Output bond count and total packed size (doubles). */
int dmrg_env_out_info(dmrg_env_t e, int* out_bond, int64_t* out_size);
/* Block structure of output bond index o: arrays of capacity `cap`;
 * *nblocks receives the count. */
int dmrg_env_out_blocks(dmrg_env_t e, int o, int cap, int* nblocks, int* left, int* right,
                        int* rows, int* cols);
int dmrg_env_flops(dmrg_env_t e, double* algorithmic, double* executed);
/* env_out_dev = updated environment (overwritten).  Asynchronous. */
int dmrg_env_apply(dmrg_env_t e, const double* ket_dev, const double* env_in_dev,
                   double* env_out_dev);

/* ---- a6/a7: canonicalisation by per-sector SVD + truncation ---------------
 * side 0 replaces RealTensorLattice::LeftCanonicalTensorLattice(int max_dim,
 * double canonical_precision) (src/dmrg/realdmrg/real_tensor_lattice.h:186,
 * .cc:558-676); side 1 replaces RightCanonicalTensorLattice (:194, .cc:794-911).
 * left_dim[num_left_sector], right_dim[num_right_sector] are the lattice's
 * sector dimensions; `ket` the site tensor's block list.  Three steps:
 *   dmrg_canon_run: stacks each sector's blocks on the device, batched one-sided
 *     Jacobi SVD, truncation exactly as ComputeTruncateDim (:501-555) -> the kept
 *     dimension of every sector (tdim_out[num sectors]: right sectors for side 0,
 *     left sectors for side 1) and the discarded weight (sum of dropped sigma^2,
 *     which the reference does not report);
 *   dmrg_canon_out_info / _out_blocks: sizes of the new ket (block order kept)
 *     and of the canonical tensor (one block per sector; match_dim as the
 *     reference's match_dim_);
 *   dmrg_canon_write: new ket blocks (U or V^T slices) and canonical blocks
 *     (S V^T or U S) into caller-allocated device buffers. */
int dmrg_canon_create(dmrg_ctx_t ctx, int side, int num_left_sector, int num_right_sector,
                      const int* left_dim, const int* right_dim, const dmrg_blocks_t* ket,
                      dmrg_canon_t* out);
int dmrg_canon_destroy(dmrg_canon_t c);
int dmrg_canon_run(dmrg_canon_t c, const double* ket_dev, int max_dim, double canpre, int* tdim_out,
                   double* discarded);
int dmrg_canon_out_info(dmrg_canon_t c, int64_t* ket_size, int64_t* canonical_size, int* sweeps);
int dmrg_canon_out_blocks(dmrg_canon_t c, int* ket_rows, int* ket_cols, int* canon_rows,
                          int* canon_cols, int* match_dim);
int dmrg_canon_singular_values(dmrg_canon_t c, int sector, int cap, double* values, int* count);
int dmrg_canon_write(dmrg_canon_t c, const double* ket_dev, double* new_ket_dev, double* canonical_dev);
/* The Jacobi pair solve's rotation schedule (diagnostic; no reference
 * counterpart): out[63 * 32], entry (step r, lane) = a | b << 6 | flip << 12 |
 * j << 13 | jflip << 18 with (a, b), a < b, the pair of the pair's 64 columns
 * that the lane rotates in step r, flip = the lane addresses b first, j = the
 * seat lane holding the pair (seats j and 63 - j; at step r seat 0 holds column
 * 0 and seat s >= 1 column ((s - 1 - r) mod 63) + 1) and jflip = the column in
 * seat j is not the one addressed first.  Every two columns share one step;
 * within each half-warp the first (and the second) columns are distinct mod 16. */
int dmrg_svd_pair_schedule(unsigned int* out);
/* The rounds a Jacobi sweep visits for one sector of `cols` columns (diagnostic;
 * no reference counterpart): bm holds the block-pair measures of its 32-column
 * blocks (bi <= bj, row-major over bi: nb (nb + 1) / 2 values), tol the
 * convergence threshold.  pairs[k] = round << 16 | bi << 8 | bj for the block
 * pairs the sweep solves (bj may be the empty block that pads an odd count);
 * *n_pairs and *n_rounds are set, DMRG_E_ARG when more than cap pairs. */
int dmrg_svd_plan_rounds(int cols, const double* bm, double tol, int cap, int* pairs, int* n_pairs,
                         int* n_rounds);
/* Cap on the Jacobi sweeps of every later canonicalisation in this process
 * (sweeps <= 0: the default, 40).  A canonicalisation that does not converge
 * within the cap returns DMRG_E_NUMERIC, as the reference treats a failed
 * dgesvd (src/tensor/real_matrix.cc:615-619) - but without exiting.  For
 * fault-injection tests of that path; no reference counterpart. */
int dmrg_svd_set_max_sweeps(int sweeps);

/* ---- whole runs: the sweep engine ------------------------------------------
 * dmrg_run_create reads a reference input file (the model keys of
 * model/real_spinless_bose_square_model.cc:11-35 plus the RealTensorRundmrg keys
 * and sweep table, real_tensor_rundmrg.cc:3-113), builds the quantum-number
 * tables and the MPO on the host, and the initial MPS on the device
 * (RealTensorSpace::DefineTensorSpace, glibc rand() seeded with opt->seed, 1 =
 * the reference's implicit seed).  dmrg_run_execute replaces
 * RealTensorRundmrg::Run (:115-245): every site step (Lanczos, subspace
 * expansion, SVD truncation, environment update, merge) runs on the device.
 * model: "real_spinless_bose_square" (NULL = that), "complex_spinless_bose_square"
 * (its complex twin, model/complex_spinless_bose_square_model.cc),
 * "real_spinful_bose_square" or "complex_spinful_bose_square". */
typedef struct {
    int precision;              /* DMRG_PREC_FP64, or DMRG_PREC_TF32X3: Lanczos
                                   matvecs first in split precision, then the
                                   FP64 Lanczos from that vector (dmrg_lanczos) */
    int verbose;                /* 1: print like the reference */
    unsigned seed;              /* 0 or 1: the reference's stream */
    int stop_after_half_sweeps; /* -1: the whole table */
    double lanczos_precision;   /* 0: the reference's 1e-15 */
    int two_site;               /* 0: the reference's single-site sweeps with
                                   subspace expansion; 1: two-site sweeps over the
                                   same sweep table (maxm, niter, canpre per
                                   half-sweep; no expansion): per bond the
                                   two-site tensor, its Lanczos ground state
                                   (dmrg_heff_create_blocks), a per-middle-sector
                                   SVD truncated to maxm, the environment update.
                                   No reference counterpart. */
    int lanczos_graph;          /* 0: the default (each Lanczos call one CUDA
                                   graph launch in a single run, launch by
                                   launch in dmrg_run_execute_many); 1: graphs
                                   always; -1: never */
} dmrg_run_options_t;
/* The run options an input file asks for (host only, no GPU needed): the
 * defaults (FP64, verbose 1, seed 1, every half-sweep, the reference's Lanczos
 * tolerance, single-site, default graph use), changed by the optional keys of
 * the file's input group: precision = fp64 | tf32x3 | bf16x3, mode = onesite |
 * twosite, seed = <int >= 0>, lanczos_tol = <double >= 0, 0 = 1e-15>,
 * lanczos_graph = -1 | 0 | 1.  The reference reads none of these keys, so its
 * own input files give its behaviour.  DMRG_E_ARG for an unreadable file or a
 * value outside these sets. */
int dmrg_run_options_from_input(const char* input_path, dmrg_run_options_t* opt);
int dmrg_run_create(dmrg_ctx_t ctx, const char* input_path, const char* model,
                    const dmrg_run_options_t* opt, dmrg_run_t* out);
int dmrg_run_execute(dmrg_run_t r);
/* Executes n independent runs side by side (for example a U/t scan): `threads`
 * host threads (<= 0: one per hardware thread, at most n) take the runs in
 * order, each on its own context's stream, so the kernels of different runs
 * overlap on the GPU.  Every run must have a context (stream) of its own.
 * Their Lanczos calls run launch by launch (the per-call graph capture and
 * instantiation serialise across host threads on one device).
 * status[i] receives run i's return code; the call returns the first failure.
 * The reference runs one instance per process
 * (model/real_spinless_bose_square_model.cc:11-42). */
int dmrg_run_execute_many(dmrg_run_t* runs, int n, int threads, int* status);
int dmrg_run_destroy(dmrg_run_t r);
/* Energy after each half-sweep (the reference's "right/left energy =" lines)
 * and its wall time. */
int dmrg_run_half_sweeps(dmrg_run_t r, int cap, double* energies, double* seconds, int* count);
/* One record per site step: half-sweep index, site, Lanczos energy, Krylov
 * dimension, discarded weight of the truncation, psi_dim, seconds. */
int dmrg_run_steps(dmrg_run_t r, int cap, int* half_sweep, int* site, double* energy, int* lanczos_dim,
                   double* discarded, int64_t* psi_dim, double* seconds, int* count);
/* Where each half-sweep's time went (no reference counterpart; the reference
 * prints only totals): seconds[5*i + k] for phase k of half-sweep i, k = 0
 * Lanczos, 1 subspace expansion, 2 canonicalisation (SVD + truncation), 3
 * environment update, 4 match + merge; svd_sweeps[i] = Jacobi sweeps summed over
 * the half-sweep's canonicalisations. */
int dmrg_run_phases(dmrg_run_t r, int cap, double* seconds, int* svd_sweeps, int* count);

/* ---- model layer (host only) -----------------------------------------------
 * The MPO of RealSpinlessBoseSquareHamiltonian::DefineTensorHamiltonian
 * (model/hamiltonian/real_spinless_bose_square_hamiltonian.cc:171-228) and the
 * quantum tables (which 0: MPS bonds, RealTensorSpace; 1: MPO bonds,
 * RealTensorHamiltonian), built from an input file without a GPU.
 * dmrg_model_create returns DMRG_E_ARG, with the reason, for a missing or
 * malformed input file (the reference prints and exits), an unknown model, and
 * sizes no model can be built for: num_site_x or num_site_y below 1,
 * physics_dim below 2, or a boson number outside [0, (physics_dim - 1) * sites].
 * The array outputs take a capacity `cap` and receive at most cap values; the
 * sizes (*left_bond, *right_bond, *rows) are always set, so a call with cap 0
 * returns them.  which: 0 or 1. */
int dmrg_model_create(const char* input_path, const char* model, dmrg_model_t* out);
int dmrg_model_destroy(dmrg_model_t m);
int dmrg_model_info(dmrg_model_t m, int* num_site, int* physics_dim, int* num_quantum);
int dmrg_model_mpo(dmrg_model_t m, int site, int* left_bond, int* right_bond, int cap, double* W);
/* model "complex_spinful_bose_square" (the reference's
 * ComplexSpinfulBoseSquareHamiltonian, Peierls phases included) builds a complex
 * MPO: *is_complex = 1 and dmrg_model_mpo writes interleaved (re, im) values
 * (cap counts doubles).  A run of such a model sweeps with complex tensors
 * (ComplexTensorRundmrg), single-site FP64. */
int dmrg_model_is_complex(dmrg_model_t m, int* is_complex);
int dmrg_model_quantum_table(dmrg_model_t m, int which, int bond, int cap, int* values, int* rows);

/* ---- host bookkeeping helpers (no device work) ----------------------------
 * dmrg_quicksort_index: the reference's QuickSort with index
 * (src/util/general.ih:7-65), same tie order; descending != 0 for flag 0.
 * dmrg_truncate_dims: ComputeTruncateDim over nsec sectors whose singular values
 * are concatenated in `values` (counts[i] each; modified in place like the
 * reference's array). */
int dmrg_quicksort_index(double* values, int* index, int n, int descending);
int dmrg_truncate_dims(int nsec, const int* counts, double* values, int max_dim, double canpre,
                       int* tdim_out);
/* dmrg_rand_stream: the first n values of the stream that srand(seed) + rand()
 * give with glibc (the reference's random source: RandomMatrix,
 * src/tensor/real_matrix.cc:201-208), from the engine's own generator. */
int dmrg_rand_stream(unsigned seed, int n, int* out);

#ifdef __cplusplus
}
#endif

#endif /* DMRG_B200_H_ */
