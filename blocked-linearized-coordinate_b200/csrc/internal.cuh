// internal.cuh -- shared declarations of the BLCO engine (not part of the ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "blco.h"

namespace blco {

// ---------------------------------------------------------------- errors --

void set_error(const std::string& msg);
const char* last_error();

// Records a CUDA failure and yields BLCO_ERR_CUDA (or BLCO_ERR_NOMEM).
int cuda_fail(cudaError_t e, const char* what, const char* file, int line);

#define BLCO_CUDA(call)                                                        \
    do {                                                                       \
        cudaError_t _e = (call);                                               \
        if (_e != cudaSuccess) return ::blco::cuda_fail(_e, #call, __FILE__, __LINE__); \
    } while (0)

#define BLCO_TRY(call)                                                         \
    do {                                                                       \
        int _s = (call);                                                       \
        if (_s != BLCO_OK) return _s;                                          \
    } while (0)

#define BLCO_CHECK_LAUNCH(name)                                                \
    do {                                                                       \
        ::blco::count_launch();                                                \
        cudaError_t _e = cudaGetLastError();                                   \
        if (_e != cudaSuccess) return ::blco::cuda_fail(_e, name, __FILE__, __LINE__); \
    } while (0)

int fail(int status, const std::string& msg);
void count_launch();
// Adds n (may be negative) to the calling thread's launch counter.
void add_launches(long long n);
unsigned long long launches_so_far();

// ----------------------------------------------------------- device info --

struct DeviceInfo {
    int device = 0;
    int sm_count = 148;
    size_t smem_optin = 227 * 1024;
    size_t l2_bytes = 126ull << 20;
};
int device_info(int device, DeviceInfo* out);

// ------------------------------------------------------------ bit layout --

// Per-tensor layout constants, passed by value to kernels.
//
// Wide keys (alto_bits > 64, the reference's 128-bit build): the ALTO key
// has a low word (alto_masks) and an upper word (alto_masks_hi).  A BLCO
// coordinate holds each mode's low-word bits only (low_bits[n] of them,
// mode_masks/mode_pos as the reference computes them), and the rest of the
// coordinate is the block coordinate.  The engine keeps the block
// coordinates of every nonzero as one 64-bit block field,
//   field = OR_n (c_n >> low_bits[n]) << bpos[n],
// so that row_n = ((coord >> mode_pos[n]) & mode_masks[n])
//               | (((field >> bpos[n]) & bmask[n]) << low_bits[n]).
struct Layout {
    int nmodes;
    uint64_t dims[BLCO_MAX_MODES];
    uint64_t mode_masks[BLCO_MAX_MODES];
    int mode_pos[BLCO_MAX_MODES];
    uint64_t alto_masks[BLCO_MAX_MODES];
    int alto_bits;
    int wide;                              // alto_bits > 64
    uint64_t alto_masks_hi[BLCO_MAX_MODES]; // upper key word (wide only)
    int low_bits[BLCO_MAX_MODES];          // popcount(alto_masks[n])
    int bpos[BLCO_MAX_MODES];              // block field offsets (wide only)
    uint64_t bmask[BLCO_MAX_MODES];        // (1 << (bits_n - low_bits[n])) - 1
};

// Computes masks/positions from dims (include/alto.hpp:597-695,
// include/blco.hpp:221-233).  Keys of up to 128 bits; returns BLCO_OK,
// BLCO_ERR_INVALID or BLCO_ERR_UNSUPPORTED.
int make_layout(int nmodes, const uint64_t* dims, Layout* out);

__host__ __device__ __forceinline__ uint64_t wide_row(const Layout& L, int n, uint64_t coord, uint64_t field)
{
    return ((coord >> L.mode_pos[n]) & L.mode_masks[n]) | (((field >> L.bpos[n]) & L.bmask[n]) << L.low_bits[n]);
}

// ---------------------------------------------------------------- tensor --

// Per-mode heavy-row table: open-addressing hash of the rows that receive
// the most nonzeros, used by the MTTKRP kernels to keep those rows'
// partial sums in shared memory.
struct HotTable {
    uint32_t* d_keys = nullptr; // hash_size entries: row + 1, 0 = empty
    uint32_t* d_slot = nullptr; // hash_size entries: slot in the smem table
    uint32_t* d_rows = nullptr; // nhot entries: slot -> row (slots by descending nnz)
    int hash_size = 0;          // power of two (0 = no table)
    int nhot = 0;               // number of rows in the table
    uint64_t hot_nnz = 0;       // nonzeros that fall on hot rows
    // CSR copy of the hot rows' nonzeros: entries d_ptr[s] .. d_ptr[s+1] of
    // d_hcoords / d_hvals are the nonzeros of hot row slot s, in ALTO order
    // (a row-grouped copy of part of the stream, read contiguously).
    uint32_t* d_ptr = nullptr;  // nhot + 1 entries
    uint64_t* d_hcoords = nullptr;
    double* d_hvals = nullptr;
    float* d_hvals32 = nullptr; // mixed form, made on first use
    double* d_acc = nullptr;    // mixed form: FP64 sums of the hot rows (nhot x acc_rank)
    int acc_rank = 0;
    // The remaining (cold) nonzeros of this mode, by row (ALTO order inside a row).
    uint64_t cold_nnz = 0;
    uint64_t* d_ccoords = nullptr;
    double* d_cvals = nullptr;
    float* d_cvals32 = nullptr; // mixed form, made on first use
};

// One MTTKRP schedule of the autotuner's space.
struct TuneCfg {
    int kernel;     // BLCO_KERNEL_LVL1 / LVL2 / LVL3 / ATOMIC
    int hot_chunk;  // LVL2: positions per warp task of the heavy-row kernel
    int interleave; // tile kernel: round-robin tile order
};
extern const TuneCfg TUNE_SPACE[BLCO_TUNE_CONFIGS];

// Autotuner timings of one (mode, factor dtype) of a tensor.
struct TuneCache {
    bool valid = false;
    int rank = 0;
    float ms[BLCO_TUNE_CONFIGS] = {}; // -1: schedule not valid here
};

// Compressed-fibre copy of the stream for one mode (fibre.cu, kernel id 4):
// nonzeros grouped by (row of the mode, index of the fibre mode), fibres of
// two or more nonzeros in the fibred stream, single-nonzero fibres in the
// loose stream.  Built on first use; resident 64-bit-key tensors only.
struct FibreCopy {
    bool built = false;
    int fmode = -1;                      // fibre mode (shortest other mode)
    int ninner = 0;                      // other modes besides it
    int inner[BLCO_MAX_MODES] = {};
    uint64_t nf = 0, nl = 0;             // fibred / loose nonzeros
    uint64_t nfib = 0, nrows_f = 0, nrows_l = 0;
    uint32_t* d_fw[3] = {};              // fibred: inner indices (bit 31 of [0]: fibre start)
    double* d_fv = nullptr;
    float* d_fv32 = nullptr;             // mixed forms, made on first use
    uint32_t* d_fib = nullptr;           // fibre-mode index per fibre (bit 31: row start)
    uint32_t* d_frows = nullptr;         // output row per row run
    uint32_t* d_fctab = nullptr;         // (fibre, row run) at every 256th position
    uint32_t* d_lw[4] = {};              // loose: fibre-mode index (bit 31: row start), inner indices
    double* d_lv = nullptr;
    float* d_lv32 = nullptr;
    uint32_t* d_lrows = nullptr;
    uint32_t* d_lctab = nullptr;         // row run at every 256th position
    uint32_t* d_counter = nullptr;       // task counter of a launch (calls on one mode run in stream order)
};

struct ModeStats {
    uint64_t max_row_nnz = 0;
    uint64_t nonempty_rows = 0;
    uint64_t log2_hist[40] = {}; // rows with nnz in [2^b, 2^(b+1))
};

} // namespace blco

struct blco_cpals_plan;
struct blco_batch;
struct blco_mlp;

struct blco_tensor {
    blco::Layout layout;
    uint64_t nnz = 0;
    uint64_t max_block_size = 0;
    uint64_t block_count = 0;
    int device = 0;
    bool resident = true;
    // resident stream (HBM)
    uint64_t* d_coords = nullptr;
    double* d_values = nullptr;
    float* d_values_f32 = nullptr; // mixed form, created on first use
    // streamed blocks (pinned host)
    uint64_t* h_coords = nullptr;
    double* h_values = nullptr;
    float* h_values32 = nullptr; // mixed forms of a streamed tensor, made on first use
    // wide keys: per-nonzero block field (see Layout) and the blocks
    // (block_count + 1 offsets, block_count x nmodes block coordinates)
    uint64_t* d_bfield = nullptr;
    std::vector<uint64_t> block_offsets;
    std::vector<uint64_t> block_coords;
    // wide keys: per mode, the stream sorted by that mode's row (key order
    // inside a row), read by that mode's MTTKRP
    struct WideCopy {
        uint64_t* d_coords = nullptr;
        uint64_t* d_field = nullptr;
        double* d_vals = nullptr;
        float* d_vals32 = nullptr; // mixed form, made on first use
    } wide_copy[BLCO_MAX_MODES];
    // heavy-row tables, one per mode, built at encode time
    blco::HotTable hot[BLCO_MAX_MODES];
    blco::FibreCopy fib[BLCO_MAX_MODES];
    blco::ModeStats stats[BLCO_MAX_MODES];
    double norm_sq = 0.0; // sum of squared values
    blco::TuneCache tune[BLCO_MAX_MODES][3];
};

namespace blco {

cudaStream_t pick_stream(const blco_tensor* t, const blco_opts* opts);

// encode.cu
int encode_impl(int nmodes, const uint64_t* dims, uint64_t nnz,
                const uint64_t* const* d_cidx, const double* d_vals,
                uint64_t max_block_size, const blco_opts* opts, blco_tensor** out);
int build_hot_tables(blco_tensor* t, cudaStream_t s);
// Nonzeros per chunk of the chunked encoder of streamed tensors (from the
// residency budget); larger streamed tensors are encoded chunk by chunk.
uint64_t stream_chunk_nnz(const blco_opts* opts, int nmodes);
int sort_stream_by_mode(const blco_tensor* t, int mode, uint64_t* d_coords, double* d_vals, uint64_t* tmp_k,
                        double* tmp_v, cudaStream_t s);
// Stable LSD radix sort of (key, payload) pairs by key bits [0, end_bit);
// *in_alt: the result is in (k1, v1).
int radix_sort_pairs_u64(uint64_t* k0, uint64_t* v0, uint64_t* k1, uint64_t* v1, uint64_t n, int end_bit,
                         cudaStream_t s, bool* in_alt);
// In-place exclusive scan of n uint32 values; sums holds n / 4096 + 2 entries.
int scan_u32_ext(uint32_t* a, uint64_t n, uint32_t* sums, cudaStream_t s);
int encode_noalloc_impl(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* const* d_cidx,
                        const double* d_vals, uint64_t* d_coords_out, double* d_vals_out, cudaStream_t s);

// mttkrp.cu
// factor_dtype selects the precision policy: BLCO_DTYPE_F64 (FP64 values,
// factors and output) or BLCO_DTYPE_F32 / BLCO_DTYPE_BF16 (FP32 values and
// output, FP32 or BF16 factors).
struct MttkrpArgs {
    const uint64_t* coords;
    const void* vals;
    uint64_t nnz;
    int mode;
    int rank;
    const void* factors[BLCO_MAX_MODES];
    void* out;
    int factor_dtype;
    int kernel;
    int thread_cf;
    int hot_chunk;  // positions per warp task of the heavy-row kernel (0: 512)
    int interleave; // tile kernel: 1 deals tiles round-robin to the grid's warps
    int out64;      // wide keys, FP32 factors: out is FP64 (sums of heavy rows stay FP64)
};
int mttkrp_launch(const blco_tensor* t, const MttkrpArgs& a, cudaStream_t s);
// fibre.cu: the compressed-fibre schedule (kernel id 4).
bool fibre_eligible(const blco_tensor* t, int mode);
int fibre_lanes(int rank, int dtype); // lanes per factor row, 0 = no kernel for this rank
// Scratch of a fibre-copy build: sort keys and stream positions (a pair of
// each for the radix sort's ping-pong), two flag/scan arrays and the scans'
// block sums, 40 bytes per nonzero.  Taken with cudaMalloc, not from the
// stream-ordered pool: the pool hands its memory back at every
// synchronisation, so a build per mode mapped and unmapped all of it again
// (about 90 ms per mode at 200M nonzeros, against a few ms here).  One
// scratch serves the builds of all modes of a plan.
struct FibScratch {
    uint64_t *k0 = nullptr, *k1 = nullptr, *i0 = nullptr, *i1 = nullptr;
    uint32_t *sa = nullptr, *sb = nullptr, *sums = nullptr;
    uint64_t cap = 0; // nonzeros the buffers hold
};
int fib_scratch_reserve(FibScratch& sc, uint64_t n);
void fib_scratch_free(FibScratch& sc); // waits for the device (cudaFree)
// Builds the mode's copy once (no-op when built); sc = nullptr: a scratch of
// its own, freed before it returns.
int build_fibre_copy(blco_tensor* t, int mode, cudaStream_t s, FibScratch* sc = nullptr);
// encode.cu: the mode's heavy-row and cold stream copies (HotTable), built
// on first use by the heavy-row schedule (no-op when built, not resident,
// or the mode has no heavy rows).
int build_mode_copies(blco_tensor* t, int mode, cudaStream_t s);
// The fibre kernel can serve this call (resident stream, rank, alignment).
bool fibre_usable(const blco_tensor* t, const MttkrpArgs& a);
// The call takes the fibre kernel: kernel id 4, or the automatic rule
// choosing it, and fibre_usable.
bool fibre_route(const blco_tensor* t, const MttkrpArgs& a);
void fibre_free(FibreCopy& f);
int mttkrp_fibre_launch(blco_tensor* t, const MttkrpArgs& a, cudaStream_t s);
// Wide-key tensors: FP64 MTTKRP over the BLCO stream in key order.
int mttkrp_wide_launch(const blco_tensor* t, const MttkrpArgs& a, cudaStream_t s);
int mttkrp_select_kernel(const blco_tensor* t, int mode, int rank, int requested, int factor_dtype);
// Automatic rule: the heavy-row path needs at least this many heavy nonzeros.
constexpr uint64_t AUTO_HOT_MIN_NNZ = 1ull << 18;
uint32_t auto_hot_chunk(uint64_t hot_nnz);
// Streamed blocks: a reusable ring of device buffers and a copy stream.
struct StreamRing;
int stream_ring_create(const blco_tensor* t, uint64_t residency_bytes, StreamRing** out);
int stream_ring_destroy(StreamRing* r);
uint64_t stream_ring_bytes(const StreamRing* r);
int mttkrp_streamed_ring(const blco_tensor* t, const MttkrpArgs& base, StreamRing* r, cudaStream_t s);
// FP32 copy of the resident values (created on first use).
int values_f32(blco_tensor* t, cudaStream_t s, const float** out);
// Pinned FP32 copy of a streamed tensor's values (made once, on the host).
int host_values_f32(blco_tensor* t);

// cpals.cu
int plan_create(blco_tensor* t, int rank, double* const* d_factors, double* d_lambda, const blco_opts* opts,
                blco_cpals_plan** out);
int plan_iterate(blco_cpals_plan* p, int iters, double tol, double* fits, int* iters_done, bool verbose);
int plan_destroy(blco_cpals_plan* p);
int plan_mttkrp_ms(const blco_cpals_plan* p, double* ms, int* calls);
int plan_condition(const blco_cpals_plan* p, double* cond, int* promoted);
int plan_device_bytes(const blco_cpals_plan* p, uint64_t* bytes);
int plan_set_reduce(blco_cpals_plan* p, blco_reduce_fn fn, void* ctx);
int plan_set_norm_sq(blco_cpals_plan* p, double norm_sq);

int batch_create(int T, blco_tensor* const* tensors, const int* ranks, double* const* const* d_factors,
                 double* const* d_lambdas, double tol, const blco_opts* opts, blco_batch** out);
int batch_iterate(blco_batch* b, int iters, double* fits, int* iters_done);
int batch_destroy(blco_batch* b);
double batch_last_ms(const blco_batch* b);
int batch_mttkrp_ms(blco_batch* b, double* ms);
int cpals_host(blco_tensor* t, int rank, double* const* factors, double* lambda, int maxiter,
               double tol, const blco_opts* opts, double* fit_out, double* fits, int* iters_out);

// gram_tc.cu: the mixed form's Gram (and optional scale / BF16 copy) on the
// tensor cores; writes *nparts FP64 R x R partials (at most
// gram_tc_max_ctas(sm)), sets *d_err when an MMA completion wait times out.
// spin_max: polls per wait (0: the default, 2^24); no_commit (self-test of
// the timeout path only): issue no MMA and no commit, so the first wait runs
// out.
int gram_tc_max_ctas(int sm);
int gram_tc_launch(float* U, uint64_t I, int R, const double* inv, uint16_t* bf16_out, double* partials, int sm,
                   int* d_err, cudaStream_t s, int* nparts, uint32_t spin_max = 0, int no_commit = 0);
int gram_tc_timeout_check(int device, int* timeout_status, int* after_status);

// cpals.cu: standalone Gram of a device FP32 matrix (tensor or CUDA cores).
int gram_f32(float* U, uint64_t I, int R, double* G, bool tensor_cores, int sm, cudaStream_t s);

// tns_parse.cu
int encode_tns_impl(const char* path, uint64_t max_block_size, const blco_opts* opts, blco_tensor** out,
                    blco_tns_info* info);
int parse_decimal_host(const char* s, int len, double* out, int* consumed);

// tune.cu
int tune_features(const blco_tensor* t, int mode, int rank, int dtype, float* f);
int tune_sweep(blco_tensor* t, int mode, int rank, int dtype, int reps, cudaStream_t s, float* ms_out);
int tune_best(const float* ms);
int mlp_create(int hidden, uint64_t seed, int device, blco_mlp** out);
int mlp_set_params(blco_mlp* m, const float* params, int n);
int mlp_get_params(const blco_mlp* m, float* params, int n);
int mlp_num_params(const blco_mlp* m);
int mlp_predict(blco_mlp* m, const float* X, int n, float* out);
int mlp_grad(blco_mlp* m, const float* X, const float* Y, const float* Mk, int n, float* grad, float* loss);
int mlp_train(blco_mlp* m, const float* X, const float* Y, const float* Mk, int n, int epochs, int batch, float lr,
              uint64_t seed, float* loss_out);
int mlp_destroy(blco_mlp* m);
int selector_set(blco_mlp* net, float margin);
int select_config(blco_tensor* t, int mode, int rank, int dtype, blco_mlp* net, float margin, cudaStream_t s,
                  int* cfg, int* used_sweep);
// Fills a->kernel / hot_chunk / interleave for the requested kernel id
// (BLCO_KERNEL_TUNED and BLCO_KERNEL_LEARNED resolve to a schedule).
int resolve_schedule(blco_tensor* t, int mode, int rank, int dtype, int requested, cudaStream_t s, MttkrpArgs* a);

} // namespace blco
