/*
 * blco.h -- C ABI of the B200 BLCO engine (libblco_b200.so).
 *
 * The reference (jeewhanchoi/blocked-linearized-coordinate) has no FFI: its
 * boundary is the cpd64 CLI plus three in-process C++ entry points.  Each
 * function below replaces one of them with plain pointers, sizes and status
 * codes; the citation names the reference interface it stands in for.
 *
 * Conventions
 *   - Every function returns a blco_status (0 = BLCO_OK).  The reference
 *     exits the process on any CUDA error (src/utils.cu:131-137); here the
 *     error is returned and blco_last_error() gives the message of the
 *     calling thread's last failure.
 *   - Factor matrices are row-major dims[n] x rank FP64, as KruskalModel::U
 *     (include/kruskal_model.hpp:8-16).
 *   - BLCO coordinates are uint64 with mode n in bits
 *     [mode_pos[n], mode_pos[n] + bits_n), in ALTO order, exactly as
 *     gen_blcotensor_host<uint64> produces them (include/blco.hpp:196-331).
 *   - "d_" pointers are device (HBM) pointers, others are host pointers.
 *   - A tensor handle may be used from one host thread at a time.
 */
#ifndef BLCO_B200_H_
#define BLCO_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BLCO_MAX_MODES 5 /* MAX_NUM_MODES, config.mk:19 */

typedef enum blco_status {
    BLCO_OK = 0,
    BLCO_ERR_INVALID = 1,     /* bad argument (mode, rank, sizes, pointers) */
    BLCO_ERR_UNSUPPORTED = 2, /* valid input outside what this build handles */
    BLCO_ERR_CUDA = 3,        /* a CUDA runtime call or kernel failed */
    BLCO_ERR_NOMEM = 4,       /* device or pinned allocation failed */
    BLCO_ERR_TIMEOUT = 5,     /* a bounded device-side wait gave up */
    BLCO_ERR_IO = 6,          /* file could not be read or parsed */
    BLCO_ERR_STATE = 7        /* handle used in a state that does not allow it */
} blco_status;

/* MTTKRP kernel ids, the values of the reference -k flag
 * (src/alto_dev.cu:1974-2011).  The reference variants are re-designed for
 * B200, keeping each id's role:
 *   1  register/segmented conflict resolution (lvl1)
 *   2  lvl1 + shared-memory privatisation of heavy output rows (lvl2 role)
 *   3  shared-memory partial output matrix, for short modes (lvl3 role)
 *   4  compressed fibres (no reference counterpart): the mode's copy of the
 *      stream grouped by (output row, index of the shortest other mode),
 *      that mode's factor row gathered once per fibre and single-nonzero
 *      fibres in a second stream; resident tensors with 64-bit keys, 3-5
 *      modes, every mode below 2^31, rank * element size 32 bytes times a
 *      power of two up to 1024 bytes, 32-byte aligned factors (the copy is
 *      built on first use; other calls take the automatic rule)
 *   10 automatic selection: 3 when the mode's output fits in shared
 *      memory, else 4 where it applies, else 2 when the mode has at least
 *      2^18 nonzeros in heavy rows (heavy-row chunk 128 / 512 / 2048 below
 *      2^20 / below 2^23 / above, cold tiles round-robin), else 1 (the
 *      reference's rule, src/alto_dev.cu:1975,1996-2001, is 3 for at most
 *      100 rows, else 1)
 *   11, 12 one launch over all blocks (always the case here; mapped to 1)
 *   13 one atomic per (nonzero, column)
 *   20 tuned: the fastest schedule of the autotuner's sweep on this tensor
 *      and mode (swept on first use, then cached in the tensor)
 *   21 learned: the schedule the selector network proposes (set with
 *      blco_selector_set); the sweep when no network is set or when no
 *      other schedule group is predicted slower by the margin (schedules
 *      that differ only in tile order form a group)
 * 20 and 21 are no reference flags; they apply to resident tensors.      */
enum {
    BLCO_KERNEL_AUTO = 10,
    BLCO_KERNEL_LVL1 = 1,
    BLCO_KERNEL_LVL2 = 2,
    BLCO_KERNEL_LVL3 = 3,
    BLCO_KERNEL_FIBRE = 4,
    BLCO_KERNEL_BATCHED = 11,
    BLCO_KERNEL_BATCHED_V2 = 12,
    BLCO_KERNEL_ATOMIC = 13,
    BLCO_KERNEL_TUNED = 20,
    BLCO_KERNEL_LEARNED = 21
};

/* Schedules of the autotuner's space, and the selector network's inputs. */
#define BLCO_TUNE_CONFIGS 14
#define BLCO_MLP_FEATURES 25

/* Numeric form. */
enum {
    BLCO_PRECISION_FP64 = 0,      /* plain form: all values and factors FP64 */
    BLCO_PRECISION_MIXED = 1,     /* chosen form: FP32 values, factors and
                                     accumulation; FP64 Grams, solve, lambda, fit */
    BLCO_PRECISION_MIXED_BF16 = 2 /* as MIXED, with BF16 factor-row gathers */
};

/* The R x R solve of CP-ALS (blco_opts.solve). */
enum {
    BLCO_SOLVE_AUTO = 0,
    BLCO_SOLVE_PINV = 1
};
#define BLCO_GUARD_COND 3e4

/* Element types of factor/output arrays for blco_mttkrp_ex. */
enum {
    BLCO_DTYPE_F64 = 0,
    BLCO_DTYPE_F32 = 1,
    BLCO_DTYPE_BF16 = 2
};

/* Options shared by the MTTKRP and CP-ALS entry points; the fields mirror
 * the reference flags (src/main.cpp:70-96).  Fill with blco_opts_init. */
typedef struct blco_opts {
    int kernel;            /* -k, default 10 */
    int nprtn;             /* -n: partial matrices for kernel 3; 0 = auto */
    int thread_cf;         /* --thread-cf: tiles per warp step, default 2 */
    int stream_data;       /* --stream-data: blocks stay in pinned host memory */
    int precision;         /* BLCO_PRECISION_* */
    int verbose;           /* print the reference's progress lines */
    int device;            /* --device */
    uint64_t residency_bytes; /* device budget for streamed blocks; 0 = 8 GiB */
    void* stream;          /* cudaStream_t to run on; NULL = the default stream */
    int gram_tensor_cores; /* mixed forms' Grams (blco_gram_f32's two
                              engines): 0 (default) or 1 = on the tensor
                              cores (tcgen05, exact integer digit products)
                              up to rank 64, FP64 on the CUDA cores above;
                              -1 = on the CUDA cores */
    int solve;             /* BLCO_SOLVE_AUTO: Cholesky of the R x R system,
                              the pseudoinverse when it is not positive
                              definite; BLCO_SOLVE_PINV: the reference's
                              pseudoinverse (eigen-decomposition, values at
                              or below R * ulp(max) dropped,
                              src/cpd_gpu.cu:452-532) in every case */
    double guard_cond;     /* mixed forms: a plan whose R x R system has a
                              condition estimate above this continues in
                              FP64 (the FP32 working set's rounding grows
                              with the condition number); 0 = the default
                              (BLCO_GUARD_COND), negative = never */
} blco_opts;

typedef struct blco_tensor blco_tensor; /* opaque */

typedef struct blco_tensor_info {
    int nmodes;
    uint64_t dims[BLCO_MAX_MODES];
    uint64_t nnz;
    uint64_t block_count;
    uint64_t max_block_size;
    uint64_t mode_masks[BLCO_MAX_MODES]; /* (1 << bits_n) - 1 */
    int mode_pos[BLCO_MAX_MODES];        /* field offsets */
    uint64_t alto_masks[BLCO_MAX_MODES]; /* interleaved ALTO masks */
    int alto_bits;                       /* sum of bits_n */
    int device;
    int resident; /* 1: stream in HBM; 0: pinned host blocks (streamed) */
    /* Keys above 64 bits (alto_bits > 64, the reference's 128-bit build,
     * ALTO_MASK_LENGTH=128): alto_masks holds the low key word and
     * alto_masks_hi the upper one; mode_masks / mode_pos then cover each
     * mode's low-word bits only, and the rest of a coordinate is its
     * block's block_coords (include/blco.hpp:222-233, 301-319). */
    uint64_t alto_masks_hi[BLCO_MAX_MODES];
} blco_tensor_info;

/* ---- library ------------------------------------------------------------ */

void blco_opts_init(blco_opts* opts);
const char* blco_status_string(int status);
/* Message of the calling thread's last failed call ("" if none). */
const char* blco_last_error(void);
/* Library version string. */
const char* blco_version(void);

/* ---- encoder ------------------------------------------------------------ */

/* Encode a COO tensor into BLCO on the GPU.
 * Replaces gen_blcotensor_host<LIT> (include/blco.hpp:196) followed by
 * gen_blcotensor_device + send_blcotensor_over (src/blco.cu:12, 120): the
 * linearization, ALTO sort, re-linearization and block split all run as
 * sm_100a kernels and the result matches the reference bit for bit.
 * Coordinates of up to 64 key bits give the 64-bit build's encoding (cpd64,
 * LIT = uint64); 65 to 128 bits give the 128-bit build's (cpd128, LIT =
 * unsigned __int128): one block per distinct upper key word, split into
 * max_block_size slices, with non-zero block_coords.  Keys above 64 bits
 * are resident only (opts->stream_data gives BLCO_ERR_UNSUPPORTED).
 *   cidx[n] (host): nnz 0-based coordinates of mode n; vals (host): nnz values.
 *   max_block_size: the --max-block-size of the reference (0 = nnz).
 *   opts->stream_data: keep the encoded blocks in pinned host memory instead
 *   of HBM, for the streamed out-of-memory path; a streamed tensor of more
 *   than opts->residency_bytes / (8 * nmodes + 40) nonzeros is encoded in
 *   chunks of that size (the COO is never whole on the device), with the
 *   same result.
 * Ties between equal coordinates keep input order. */
int blco_encode(int nmodes, const uint64_t* dims, uint64_t nnz,
                const uint64_t* const* cidx, const double* vals,
                uint64_t max_block_size, const blco_opts* opts,
                blco_tensor** out);

/* Same, with the COO arrays already in device memory (d_cidx[n], d_vals). */
int blco_encode_device(int nmodes, const uint64_t* dims, uint64_t nnz,
                       const uint64_t* const* d_cidx, const double* d_vals,
                       uint64_t max_block_size, const blco_opts* opts,
                       blco_tensor** out);

/* Allocation-free encoder.  No counterpart in the reference: it exists for
 * callers that cannot allocate device memory while they encode, for example
 * code whose device memory is owned by another allocator (a framework's
 * memory pool, a service with a fixed budget) or that must not call
 * cudaMalloc, which can synchronise the device and fail.
 * Encodes nnz nonzeros (COO in device memory: d_cidx[n], d_vals) into the
 * caller's device arrays d_coords_out / d_vals_out (nnz entries each), with
 * the same bits as blco_encode; no tensor handle, no heavy-row tables.
 * Scratch: a fixed 32 MiB device array inside the library, held by every GPU
 * that loads it until the process exits; this function calls no cudaMalloc,
 * cudaFree or allocating library routine.
 *   - nnz above BLCO_NOALLOC_MAX_NNZ, and coordinates needing more than 64
 *     key bits (their block coordinates have no output array here), are
 *     rejected with BLCO_ERR_UNSUPPORTED;
 *   - every call on a device shares that one array: calls that overlap on
 *     the GPU (other streams or host threads) race, so serialise them;
 *   - the first call on a device does the library's set-up there (loading
 *     its device code, looking up the array's address): make that first
 *     call before any stream capture.
 * Runs on `stream` (NULL = default stream) and synchronises it twice: after
 * copying the encoder's tables from pageable host memory, and to read back
 * the coordinate-range check, so it returns after the encode has finished.
 * A device reset (cudaDeviceReset) between calls is allowed: every call
 * looks up the array's address again. */
#define BLCO_NOALLOC_MAX_NNZ 1900000ull
int blco_encode_device_noalloc(int nmodes, const uint64_t* dims, uint64_t nnz,
                               const uint64_t* const* d_cidx, const double* d_vals,
                               uint64_t* d_coords_out, double* d_vals_out, void* stream);

/* Free a tensor.  Replaces delete_blcotensor_host/_device
 * (src/blco.cu:61-91). */
int blco_tensor_free(blco_tensor* t);

int blco_tensor_get_info(const blco_tensor* t, blco_tensor_info* info);

/* Copy the encoded arrays to host memory: coords/values (nnz entries, the
 * reference's blcotensor::coords / ::values), block_offsets (block_count + 1
 * entries: start of every block, then nnz) and block_coords
 * (block_count * nmodes, blco_block::block_coords).  Any pointer may be
 * NULL to skip that array. */
int blco_tensor_copy_out(const blco_tensor* t, uint64_t* coords, double* values,
                         uint64_t* block_offsets, uint64_t* block_coords);

/* Device pointers of the resident stream (BLCO_ERR_STATE if streamed). */
int blco_tensor_device_arrays(const blco_tensor* t, const uint64_t** d_coords,
                              const double** d_values);
/* Statistics of the compressed-fibre copy of `mode` (kernel id 4), building
 * it if needed: stats[0] fibre mode, [1] nonzeros in fibres of two or more,
 * [2] single-nonzero fibres, [3] fibres of two or more, [4] factor rows one
 * MTTKRP of the mode gathers ((nmodes - 2) per fibred nonzero, one per
 * fibre, nmodes - 1 per single-nonzero fibre).  BLCO_ERR_UNSUPPORTED where
 * kernel 4 does not apply.  No counterpart in the reference. */
int blco_tensor_fibre_stats(blco_tensor* t, int mode, uint64_t* stats);

/* ---- MTTKRP ------------------------------------------------------------- */

/* d_out += MTTKRP of mode `mode` (row-major dims[mode] x rank) using device
 * factor matrices d_factors[n] (row-major dims[n] x rank; d_factors[mode]
 * is not read).  Replaces mttkrp_alto_dev_onemode<IType>
 * (src/alto_dev.cu:1955-2032), which also accumulates into its output.
 * Runs on opts->stream; returns after enqueueing (streamed tensors: after
 * the last block is enqueued). */
int blco_mttkrp(blco_tensor* t, int mode, int rank, const double* const* d_factors,
                double* d_out, const blco_opts* opts);

/* Mixed-precision MTTKRP (the chosen form's kernel): d_out (FP32,
 * dims[mode] x rank) += MTTKRP computed from the tensor's values rounded to
 * FP32, factor rows of type factor_dtype (BLCO_DTYPE_F32 or
 * BLCO_DTYPE_BF16, row-major dims[n] x rank) and FP32 accumulation.
 * BLCO_DTYPE_F64 factors with an FP64 output is the same as blco_mttkrp.
 * No reference counterpart (the reference is FP64 only). */
int blco_mttkrp_ex(blco_tensor* t, int mode, int rank, int factor_dtype,
                   const void* const* d_factors, void* d_out, const blco_opts* opts);

/* Host-pointer form: out (host) += MTTKRP, factors are host arrays.  The
 * role of the reference -p benchmark driver mttkrp_alto_dev
 * (src/alto_dev.cu:1857-1952) for one call; synchronous. */
int blco_mttkrp_host(blco_tensor* t, int mode, int rank, const double* const* factors,
                     double* out, const blco_opts* opts);

/* ---- CP-ALS ------------------------------------------------------------- */

/* CP-ALS with host factors.  Replaces cpals_blco_dev (src/cpd_gpu.cu:21-242)
 * and keeps its arithmetic: modes in descending length order, pseudoinverse
 * of the Hadamard product of Grams with the n*ulp(s_max) cut-off, column
 * L2 scaling with lambda_c <- sqrt(lambda_c + ||u_c||^2) (lambda is not
 * reset, as in the reference), fit as kruskal_fit_gpu, stop when
 * |fit - fit_old| < tol or the fit is NaN.  factors (host, dims[n] x rank)
 * and lambda (host, rank) are read and updated in place.
 *   fit_out: last fit; fits (may be NULL): one entry per executed
 *   iteration (maxiter entries must fit); iters_out: iterations executed.
 * A streamed tensor (encoded with opts->stream_data) runs every form: each
 * MTTKRP copies its blocks through a ring of device buffers of at most
 * opts->residency_bytes; the mixed forms copy 4-byte values (from a pinned
 * FP32 copy of the values made on first use). */
int blco_cpals(blco_tensor* t, int rank, double* const* factors, double* lambda,
               int maxiter, double tol, const blco_opts* opts, double* fit_out,
               double* fits, int* iters_out);

/* Re-usable CP-ALS state over device factors: set-up (||X||, Grams and
 * workspace) once, then run iterations.  d_factors and d_lambda stay owned
 * by the caller and must outlive the plan. */
typedef struct blco_cpals_plan blco_cpals_plan;

int blco_cpals_plan_create(blco_tensor* t, int rank, double* const* d_factors,
                           double* d_lambda, const blco_opts* opts,
                           blco_cpals_plan** out);
/* Run up to `iters` iterations (the convergence test uses tol and the fit
 * of the previous call).  fits: host array of `iters` entries or NULL. */
int blco_cpals_plan_iterate(blco_cpals_plan* p, int iters, double tol, double* fits,
                            int* iters_done);
/* Milliseconds of device time spent in MTTKRP per mode over all iterations
 * run so far (CUDA events on the plan's stream); ms has nmodes entries. */
int blco_cpals_plan_mttkrp_ms(const blco_cpals_plan* p, double* ms, int* calls);
/* The condition estimate of every mode's last R x R solve (cond: nmodes
 * entries; the squared ratio of the extreme Cholesky pivots, or the ratio
 * of the extreme kept eigenvalues) and whether a mixed plan runs in FP64
 * (promoted: 1 when an estimate exceeded guard_cond, at plan creation or
 * after an iteration).  No counterpart in the reference. */
int blco_cpals_plan_condition(const blco_cpals_plan* p, double* cond, int* promoted);
/* Device bytes the plan holds: the caller's FP64 factors and lambda, its
 * workspace and, for a streamed tensor, the ring of block buffers, which is
 * sized so that the total stays within opts.residency_bytes.  No
 * counterpart in the reference. */
int blco_cpals_plan_device_bytes(const blco_cpals_plan* p, uint64_t* bytes);
int blco_cpals_plan_destroy(blco_cpals_plan* p);

/* Sharded CP-ALS (several processes, one GPU each, each holding a share of
 * the nonzeros of one tensor and the same factors).  No reference
 * counterpart: the reference decomposes on one GPU.  The partition of the
 * nonzeros is free (the MTTKRP is a sum over nonzeros); the one exchange is
 * a sum of every mode's MTTKRP over the ranks.
 *   blco_cpals_plan_set_reduce: after each mode's MTTKRP the plan calls
 *   fn(ctx, d_buf, count, dtype, stream) from the thread that runs
 *   blco_cpals_plan_iterate, with the MTTKRP output (count elements of
 *   BLCO_DTYPE_F64 or _F32 in device memory) and the plan's stream; fn
 *   must enqueue a sum over the ranks into d_buf on that stream (for
 *   instance ncclAllReduce) and return 0 (else the iteration stops with
 *   BLCO_ERR_CUDA).  Every rank must get identical sums: every later step
 *   is deterministic, so all ranks then compute the same factors and fits
 *   and take the same convergence decision.  fn = NULL removes the hook.
 *   blco_cpals_plan_set_norm_sq: the sum over the ranks of their tensors'
 *   squared values (||X||^2 of the whole tensor, for the fit). */
typedef int (*blco_reduce_fn)(void* ctx, void* d_buf, uint64_t count, int dtype, void* stream);
int blco_cpals_plan_set_reduce(blco_cpals_plan* p, blco_reduce_fn fn, void* ctx);
int blco_cpals_plan_set_norm_sq(blco_cpals_plan* p, double norm_sq);

/* Batched CP-ALS of many independent resident tensors (no counterpart in the
 * reference, which decomposes one tensor per run).  Tensors may differ in
 * nnz, order (1..5) and rank (ranks[t] in 1..64); up to 4096 tensors, all on
 * one device.  Each iteration is one sweep over every unconverged tensor:
 * the MTTKRP of mode slot k (a tensor's k-th longest mode) of all tensors
 * is one persistent launch, the dense steps are one launch per step over
 * all tensors, and the fit and the convergence test (|fit - fit_old| < tol,
 * or NaN, per tensor) run on the device.  The sweep is captured once as a
 * CUDA graph and replayed per iteration.  The arithmetic is FP64 and the
 * algorithm is that of blco_cpals, tensor by tensor.
 *   d_factors[t][n]: device FP64 dims[n] x ranks[t] row-major, updated in
 *   place; d_lambdas[t]: device FP64 ranks[t], updated in place.  Both stay
 *   owned by the caller and must outlive the batch.  opts->verbose < 0
 *   disables the graph (each sweep is enqueued launch by launch). */
typedef struct blco_batch blco_batch;

int blco_batch_create(int count, blco_tensor* const* tensors, const int* ranks,
                      double* const* const* d_factors, double* const* d_lambdas,
                      double tol, const blco_opts* opts, blco_batch** out);
/* Run `iters` sweeps (0..4096).  fits (may be NULL): host array of
 * iters x count, entry [i * count + t] the fit of tensor t after sweep i of
 * this call (a converged tensor keeps its last value there).  iters_done
 * (may be NULL): per tensor, iterations executed since creation. */
int blco_batch_iterate(blco_batch* b, int iters, double* fits, int* iters_done);
int blco_batch_destroy(blco_batch* b);
/* Device time (CUDA events on the batch's stream) of the sweeps run by the
 * last blco_batch_iterate call, in milliseconds. */
int blco_batch_last_ms(const blco_batch* b, double* ms);
/* Device time of one sweep's MTTKRP launches alone (the persistent batched
 * MTTKRP of every mode slot, outside the graph; the batch's state is
 * unchanged: the MTTKRP results are recomputed by every sweep), in
 * milliseconds.  Synchronous on the batch's stream. */
int blco_batch_mttkrp_ms(blco_batch* b, double* ms);

/* ---- MTTKRP schedule selection (no counterpart in the reference, which
 * has the fixed -k 10 rule, src/alto_dev.cu:1975,1996-2001). */

/* One schedule: kernel id (1, 2, 3, 4 or 13), heavy-row chunk (kernel 2:
 * the positions of one warp task of the heavy-row kernel; 0 otherwise) and
 * tile order (kernels 1-3 and 13: 1 = tiles dealt round-robin over the
 * grid's warps, 0 = a contiguous range of tiles per CTA; kernel 4: 1 = warp
 * tasks taken in stream order, 0 = in a strided order that spreads
 * concurrent tasks over the stream). */
typedef struct blco_tune_config {
    int kernel;
    int hot_chunk;
    int interleave;
} blco_tune_config;

/* The BLCO_TUNE_CONFIGS schedules of the autotuner's space, in index order. */
int blco_tune_space(blco_tune_config* configs);

/* The exhaustive sweep: times every schedule (CUDA events, `reps` runs after
 * one warm-up) for this tensor, mode, rank and factor dtype on synthetic
 * factors.  ms[k] (BLCO_TUNE_CONFIGS entries, may be NULL): milliseconds
 * per MTTKRP, -1 for schedules that do not apply (kernel 3 when the mode's
 * output does not fit in shared memory).  best (may be NULL): index of the
 * fastest.  The result is cached in the tensor (kernel id 20 uses it). */
int blco_autotune(blco_tensor* t, int mode, int rank, int factor_dtype, int reps,
                  const blco_opts* opts, float* ms, int* best);

/* The selector's BLCO_MLP_FEATURES inputs for one mode: sizes (log2 nnz,
 * order, rank, dtype, mode length, factor and output bytes, factor bytes
 * over L2), row statistics of the mode (row occupancy, mean and longest
 * fibre, heavy-row share and count, nonzero share by fibre-length bucket),
 * whether kernel 3 applies, and the block count. */
int blco_tune_features(const blco_tensor* t, int mode, int rank, int factor_dtype,
                       float* features);

/* The selector network: BLCO_MLP_FEATURES -> hidden (ReLU) -> hidden (ReLU)
 * -> BLCO_TUNE_CONFIGS, FP32, trained and run by this library's kernels.
 * Output k predicts log2(time of schedule k / time of the best schedule).
 * Parameters (flat, in this order): W1[hidden][F] b1[hidden]
 * W2[hidden][hidden] b2[hidden] W3[K][hidden] b3[K], row-major. */
typedef struct blco_mlp blco_mlp;

int blco_mlp_create(int hidden, uint64_t seed, int device, blco_mlp** out);
int blco_mlp_num_params(const blco_mlp* net, int* n);
int blco_mlp_set_params(blco_mlp* net, const float* params, int n);
int blco_mlp_get_params(const blco_mlp* net, float* params, int n);
/* X: n x F (host), out: n x K (host). */
int blco_mlp_predict(blco_mlp* net, const float* X, int n, float* out);
/* Loss (mean over the entries with mask 1 of (out - Y)^2) and its gradient
 * with respect to the parameters (host array of num_params), for host
 * arrays X (n x F), Y and mask (n x K). */
int blco_mlp_grad(blco_mlp* net, const float* X, const float* Y, const float* mask, int n,
                  float* grad, float* loss);
/* Adam (0.9, 0.999, 1e-8) over shuffled mini-batches for `epochs` epochs;
 * loss (may be NULL): the loss over all n rows afterwards. */
int blco_mlp_train(blco_mlp* net, const float* X, const float* Y, const float* mask, int n,
                   int epochs, int batch, float lr, uint64_t seed, float* loss);
int blco_mlp_destroy(blco_mlp* net);

/* The network kernel id 21 uses (NULL: none, the sweep decides), and the
 * margin in predicted log2 time: when the best schedule's prediction is not
 * below every other group's by the margin, the sweep runs instead.  The
 * network must outlive its use. */
int blco_selector_set(blco_mlp* net, float margin);

/* The schedule index that kernel id 21 would use with this network and
 * margin (net NULL: the sweep); used_sweep (may be NULL) is set to 1 when
 * the sweep decided. */
int blco_select(blco_tensor* t, int mode, int rank, int factor_dtype, blco_mlp* net,
                float margin, const blco_opts* opts, int* config, int* used_sweep);

/* G = U^T U for a device FP32 matrix U (I x rank, row-major, rank 1..64),
 * G (device, rank x rank FP64).  tensor_cores 1: products on the tensor
 * cores (per 64-row tile and column, a power-of-two scale and four 8-bit
 * integer digits per value, exact integer sums in the FP32 accumulator,
 * FP64 beyond the tile; each value to within 2^-33 of its tile column's
 * largest magnitude; U 16-byte aligned); 0: FP64 products on the CUDA
 * cores.  The Gram of the
 * reference's ata_gpu (src/cpd_gpu.cu:547-568) for the mixed form's FP32
 * factors.  Synchronous on `stream` (NULL: default stream). */
int blco_gram_f32(const float* d_U, uint64_t I, int rank, double* d_G, int tensor_cores, int device,
                  void* stream);

/* Self-check of the tensor-core Gram's bounded wait on its MMA completion
 * barrier: one launch that issues no MMA and no commit, so that its wait
 * runs out (after 64 polls), then an ordinary launch.  *timeout_status
 * receives the first launch's status (BLCO_ERR_TIMEOUT when the kernel
 * reported the timeout), *after_status the second's (BLCO_OK when it ran
 * and its Gram was exact: the first freed its tensor memory).  Returns an
 * error only when the check itself could not run. */
int blco_gram_tc_timeout_check(int device, int* timeout_status, int* after_status);

/* ---- .tns text loading on the GPU (the reference's read_tns_dims /
 * read_tns_data, src/sptensor.cpp:74-160, feeding the encoder directly). */

typedef struct blco_tns_info {
    int nmodes;                     /* fields of the first data line minus one */
    uint64_t dims[BLCO_MAX_MODES];  /* largest 1-based index per mode */
    uint64_t nnz;                   /* data lines */
    uint64_t lines;                 /* lines in the file */
    uint64_t host_parsed;           /* lines the device left to strtoull / strtod */
} blco_tns_info;

/* Reads a FROSTT .tns file, parses it on the GPU (same line rules, indices
 * and values as the host loader: every value is the double strtod gives)
 * and encodes it as blco_encode_device does; the coordinates never exist on
 * the host.  info (may be NULL) receives the mode count, lengths, nnz and
 * line counts.  Errors: BLCO_ERR_IO (open / read), BLCO_ERR_INVALID
 * (malformed line or index 0, with the line number in blco_last_error()). */
int blco_encode_tns(const char* path, uint64_t max_block_size, const blco_opts* opts,
                    blco_tensor** out, blco_tns_info* info);

/* The loader's decimal-to-double conversion run on the host (the code the
 * GPU runs): parses s[0..len) with strtod's decimal syntax.  Returns 0 with
 * *out set when it decides the correctly rounded value, 1 when it leaves the
 * number to strtod (over 19 significant digits, halfway cases, subnormal or
 * overflowing values, hex / inf / nan), 2 when there is no number;
 * *consumed = characters used. */
int blco_parse_decimal(const char* s, int len, double* out, int* consumed);

/* Number of this library's kernels launched by the calling thread since the
 * last reset (for reporting launch counts). */
uint64_t blco_launch_count(int reset);

#ifdef __cplusplus
}
#endif

#endif /* BLCO_B200_H_ */
