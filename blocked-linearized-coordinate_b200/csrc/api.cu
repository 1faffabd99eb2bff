// api.cu -- the extern "C" boundary of libblco_b200 (include/blco.h).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "internal.cuh"

namespace blco {

static thread_local std::string g_last_error;
static thread_local uint64_t g_launches = 0;

void set_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }
void count_launch() { g_launches++; }
void add_launches(long long n) { g_launches += (uint64_t)n; }
unsigned long long launches_so_far() { return g_launches; }

int fail(int status, const std::string& msg)
{
    g_last_error = msg;
    return status;
}

int cuda_fail(cudaError_t e, const char* what, const char* file, int line)
{
    char buf[512];
    snprintf(buf, sizeof(buf), "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
    g_last_error = buf;
    return e == cudaErrorMemoryAllocation ? BLCO_ERR_NOMEM : BLCO_ERR_CUDA;
}

int device_info(int device, DeviceInfo* out)
{
    static std::mutex mu;
    static DeviceInfo cache[64];
    static bool have[64] = {};
    if (device < 0 || device >= 64) return fail(BLCO_ERR_INVALID, "bad device ordinal");
    std::lock_guard<std::mutex> g(mu);
    if (!have[device]) {
        DeviceInfo d;
        d.device = device;
        BLCO_CUDA(cudaDeviceGetAttribute(&d.sm_count, cudaDevAttrMultiProcessorCount, device));
        int optin = 0;
        BLCO_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
        d.smem_optin = (size_t)optin;
        int major = 0;
        BLCO_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
        if (major != 10)
            return fail(BLCO_ERR_UNSUPPORTED, "this library is built for sm_100a (B200) only");
        cache[device] = d;
        have[device] = true;
    }
    *out = cache[device];
    return BLCO_OK;
}

cudaStream_t pick_stream(const blco_tensor*, const blco_opts* opts)
{
    // NULL selects the default stream, so work is ordered with the caller's
    // other default-stream work.
    return opts ? (cudaStream_t)opts->stream : (cudaStream_t)0;
}

// Streamed MTTKRP: the blocks stay in pinned host memory; they are copied
// into a ring of device buffers on a copy stream while the compute stream
// runs the kernel on the previous block (the --stream-data path,
// src/alto_dev.cu:1979-2012, with events instead of one stream per block).
static int mttkrp_streamed(blco_tensor* t, const MttkrpArgs& base, const blco_opts* opts, cudaStream_t s)
{
    // the ring holds what the residency budget leaves after the caller's
    // factors and output
    const uint64_t budget = opts && opts->residency_bytes ? opts->residency_bytes : (8ull << 30);
    const uint64_t eb = base.factor_dtype == BLCO_DTYPE_F64 ? 8 : base.factor_dtype == BLCO_DTYPE_F32 ? 4 : 2;
    uint64_t held = t->layout.dims[base.mode] * (uint64_t)base.rank * (base.factor_dtype == BLCO_DTYPE_F64 ? 8 : 4);
    for (int m = 0; m < t->layout.nmodes; m++) held += t->layout.dims[m] * (uint64_t)base.rank * eb;
    if (budget <= held + 32) return fail(BLCO_ERR_NOMEM, "the residency budget does not cover the factors and output");
    StreamRing* ring = nullptr;
    BLCO_TRY(stream_ring_create(t, budget - held, &ring));
    const int st = mttkrp_streamed_ring(t, base, ring, s);
    const int st2 = stream_ring_destroy(ring);
    return st != BLCO_OK ? st : st2;
}

} // namespace blco

using namespace blco;

extern "C" {

void blco_opts_init(blco_opts* o)
{
    if (!o) return;
    memset(o, 0, sizeof(*o));
    o->kernel = BLCO_KERNEL_AUTO;
    o->nprtn = 0;
    o->thread_cf = 2;
    o->precision = BLCO_PRECISION_FP64;
}

const char* blco_status_string(int s)
{
    switch (s) {
    case BLCO_OK: return "ok";
    case BLCO_ERR_INVALID: return "invalid argument";
    case BLCO_ERR_UNSUPPORTED: return "unsupported";
    case BLCO_ERR_CUDA: return "CUDA error";
    case BLCO_ERR_NOMEM: return "out of memory";
    case BLCO_ERR_TIMEOUT: return "device wait timed out";
    case BLCO_ERR_IO: return "I/O error";
    case BLCO_ERR_STATE: return "invalid state";
    default: return "unknown status";
    }
}

const char* blco_last_error(void) { return blco::last_error(); }

const char* blco_version(void) { return "blco_b200 0.1.0 (sm_100a)"; }

uint64_t blco_launch_count(int reset)
{
    uint64_t v = blco::g_launches;
    if (reset) blco::g_launches = 0;
    return v;
}

int blco_encode_device(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* const* d_cidx,
                       const double* d_vals, uint64_t max_block_size, const blco_opts* opts, blco_tensor** out)
{
    if (!out) return fail(BLCO_ERR_INVALID, "null output handle");
    return encode_impl(nmodes, dims, nnz, d_cidx, d_vals, max_block_size, opts, out);
}

int blco_encode(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* const* cidx, const double* vals,
                uint64_t max_block_size, const blco_opts* opts, blco_tensor** out)
{
    if (!out) return fail(BLCO_ERR_INVALID, "null output handle");
    *out = nullptr;
    if (nmodes < 1 || nmodes > BLCO_MAX_MODES) return fail(BLCO_ERR_INVALID, "nmodes must be 1..5");
    if (!dims || (nnz && (!cidx || !vals))) return fail(BLCO_ERR_INVALID, "null argument");
    int device = opts ? opts->device : 0;
    BLCO_CUDA(cudaSetDevice(device));
    DeviceInfo di;
    BLCO_TRY(device_info(device, &di));
    // A streamed tensor larger than one chunk is encoded chunk by chunk
    // straight from the host arrays: the COO never sits whole on the device.
    if (opts && opts->stream_data && nnz > stream_chunk_nnz(opts, nmodes)) {
        for (int n = 0; n < nmodes; n++)
            if (!cidx[n]) return fail(BLCO_ERR_INVALID, "null coordinate array");
        return encode_impl(nmodes, dims, nnz, cidx, vals, max_block_size, opts, out);
    }
    const uint64_t n_alloc = nnz ? nnz : 1;
    uint64_t* dc[BLCO_MAX_MODES] = {};
    double* dv = nullptr;
    int st = BLCO_OK;
    cudaStream_t s = opts && opts->stream ? (cudaStream_t)opts->stream : nullptr;
    auto cleanup = [&]() {
        if (s) cudaStreamSynchronize(s);
        else cudaDeviceSynchronize();
        for (int n = 0; n < nmodes; n++) cudaFree(dc[n]);
        cudaFree(dv);
    };
    for (int n = 0; n < nmodes && st == BLCO_OK; n++) {
        if (nnz && !cidx[n]) st = fail(BLCO_ERR_INVALID, "null coordinate array");
        cudaError_t e = cudaMalloc(&dc[n], n_alloc * 8);
        if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(dc[n], cidx[n], nnz * 8, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess && st == BLCO_OK) st = cuda_fail(e, "coordinate upload", __FILE__, __LINE__);
    }
    if (st == BLCO_OK) {
        cudaError_t e = cudaMalloc(&dv, n_alloc * 8);
        if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(dv, vals, nnz * 8, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) st = cuda_fail(e, "value upload", __FILE__, __LINE__);
    }
    if (st == BLCO_OK) {
        if (s) st = cudaStreamSynchronize(s) == cudaSuccess ? BLCO_OK : fail(BLCO_ERR_CUDA, "upload sync failed");
        else st = cudaDeviceSynchronize() == cudaSuccess ? BLCO_OK : fail(BLCO_ERR_CUDA, "upload sync failed");
    }
    if (st == BLCO_OK) st = encode_impl(nmodes, dims, nnz, dc, dv, max_block_size, opts, out);
    cleanup();
    return st;
}

int blco_encode_device_noalloc(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* const* d_cidx,
                               const double* d_vals, uint64_t* d_coords_out, double* d_vals_out, void* stream)
{
    return encode_noalloc_impl(nmodes, dims, nnz, d_cidx, d_vals, d_coords_out, d_vals_out, (cudaStream_t)stream);
}

int blco_tensor_free(blco_tensor* t)
{
    if (!t) return BLCO_OK;
    cudaSetDevice(t->device);
    cudaDeviceSynchronize();
    cudaFree(t->d_coords);
    cudaFree(t->d_values);
    cudaFree(t->d_values_f32);
    cudaFree(t->d_bfield);
    for (auto& w : t->wide_copy) {
        cudaFree(w.d_coords);
        cudaFree(w.d_field);
        cudaFree(w.d_vals);
        cudaFree(w.d_vals32);
    }
    if (t->h_coords) cudaFreeHost(t->h_coords);
    if (t->h_values) cudaFreeHost(t->h_values);
    if (t->h_values32) cudaFreeHost(t->h_values32);
    for (int n = 0; n < BLCO_MAX_MODES; n++) {
        cudaFree(t->hot[n].d_keys);
        cudaFree(t->hot[n].d_slot);
        cudaFree(t->hot[n].d_rows);
        cudaFree(t->hot[n].d_ptr);
        cudaFree(t->hot[n].d_hcoords);
        cudaFree(t->hot[n].d_hvals);
        cudaFree(t->hot[n].d_hvals32);
        cudaFree(t->hot[n].d_acc);
        cudaFree(t->hot[n].d_ccoords);
        cudaFree(t->hot[n].d_cvals);
        cudaFree(t->hot[n].d_cvals32);
        blco::fibre_free(t->fib[n]);
    }
    delete t;
    return BLCO_OK;
}

int blco_tensor_get_info(const blco_tensor* t, blco_tensor_info* info)
{
    if (!t || !info) return fail(BLCO_ERR_INVALID, "null argument");
    memset(info, 0, sizeof(*info));
    info->nmodes = t->layout.nmodes;
    for (int n = 0; n < t->layout.nmodes; n++) {
        info->dims[n] = t->layout.dims[n];
        info->mode_masks[n] = t->layout.mode_masks[n];
        info->mode_pos[n] = t->layout.mode_pos[n];
        info->alto_masks[n] = t->layout.alto_masks[n];
        info->alto_masks_hi[n] = t->layout.alto_masks_hi[n];
    }
    info->nnz = t->nnz;
    info->block_count = t->block_count;
    info->max_block_size = t->max_block_size;
    info->alto_bits = t->layout.alto_bits;
    info->device = t->device;
    info->resident = t->resident ? 1 : 0;
    return BLCO_OK;
}

int blco_tensor_copy_out(const blco_tensor* t, uint64_t* coords, double* values, uint64_t* block_offsets,
                         uint64_t* block_coords)
{
    if (!t) return fail(BLCO_ERR_INVALID, "null tensor");
    BLCO_CUDA(cudaSetDevice(t->device));
    if (t->nnz) {
        if (t->resident) {
            if (coords) BLCO_CUDA(cudaMemcpy(coords, t->d_coords, t->nnz * 8, cudaMemcpyDeviceToHost));
            if (values) BLCO_CUDA(cudaMemcpy(values, t->d_values, t->nnz * 8, cudaMemcpyDeviceToHost));
        } else {
            if (coords) memcpy(coords, t->h_coords, t->nnz * 8);
            if (values) memcpy(values, t->h_values, t->nnz * 8);
        }
    }
    if (t->layout.wide) {
        if (block_offsets) memcpy(block_offsets, t->block_offsets.data(), (t->block_count + 1) * sizeof(uint64_t));
        if (block_coords) memcpy(block_coords, t->block_coords.data(), t->block_coords.size() * sizeof(uint64_t));
        return BLCO_OK;
    }
    const uint64_t B = t->max_block_size ? t->max_block_size : t->nnz;
    if (block_offsets) {
        for (uint64_t b = 0; b < t->block_count; b++) block_offsets[b] = b * B;
        block_offsets[t->block_count] = t->nnz;
    }
    if (block_coords) memset(block_coords, 0, t->block_count * t->layout.nmodes * sizeof(uint64_t));
    return BLCO_OK;
}

int blco_tensor_device_arrays(const blco_tensor* t, const uint64_t** d_coords, const double** d_values)
{
    if (!t) return fail(BLCO_ERR_INVALID, "null tensor");
    if (!t->resident) return fail(BLCO_ERR_STATE, "tensor blocks are streamed from host memory");
    if (d_coords) *d_coords = t->d_coords;
    if (d_values) *d_values = t->d_values;
    return BLCO_OK;
}

int blco_mttkrp(blco_tensor* t, int mode, int rank, const double* const* d_factors, double* d_out,
                const blco_opts* opts)
{
    if (!t || !d_factors || !d_out) return fail(BLCO_ERR_INVALID, "null argument");
    if (mode < 0 || mode >= t->layout.nmodes) return fail(BLCO_ERR_INVALID, "mode out of range");
    if (rank < 1) return fail(BLCO_ERR_INVALID, "rank must be positive");
    if (opts && opts->precision != BLCO_PRECISION_FP64)
        return fail(BLCO_ERR_UNSUPPORTED, "blco_mttkrp takes FP64 factors; use the mixed-precision entry point");
    for (int m = 0; m < t->layout.nmodes; m++)
        if (m != mode && !d_factors[m]) return fail(BLCO_ERR_INVALID, "null factor matrix");
    BLCO_CUDA(cudaSetDevice(t->device));
    cudaStream_t s = pick_stream(t, opts);
    MttkrpArgs a;
    memset(&a, 0, sizeof(a));
    a.nnz = t->nnz;
    a.mode = mode;
    a.rank = rank;
    for (int m = 0; m < t->layout.nmodes; m++) a.factors[m] = d_factors[m];
    a.out = d_out;
    a.factor_dtype = BLCO_DTYPE_F64;
    a.thread_cf = opts ? opts->thread_cf : 2;
    BLCO_TRY(resolve_schedule(t, mode, rank, BLCO_DTYPE_F64, opts ? opts->kernel : BLCO_KERNEL_AUTO, s, &a));
    if (!t->resident) return mttkrp_streamed(t, a, opts, s);
    a.coords = t->d_coords;
    a.vals = t->d_values;
    return mttkrp_launch(t, a, s);
}

int blco_mttkrp_ex(blco_tensor* t, int mode, int rank, int factor_dtype, const void* const* d_factors,
                   void* d_out, const blco_opts* opts)
{
    if (factor_dtype == BLCO_DTYPE_F64)
        return blco_mttkrp(t, mode, rank, reinterpret_cast<const double* const*>(d_factors),
                           reinterpret_cast<double*>(d_out), opts);
    if (!t || !d_factors || !d_out) return fail(BLCO_ERR_INVALID, "null argument");
    if (factor_dtype != BLCO_DTYPE_F32 && factor_dtype != BLCO_DTYPE_BF16)
        return fail(BLCO_ERR_INVALID, "factor_dtype must be BLCO_DTYPE_F32 or BLCO_DTYPE_BF16");
    if (mode < 0 || mode >= t->layout.nmodes) return fail(BLCO_ERR_INVALID, "mode out of range");
    if (rank < 1) return fail(BLCO_ERR_INVALID, "rank must be positive");
    if (t->layout.wide && factor_dtype == BLCO_DTYPE_BF16)
        return fail(BLCO_ERR_UNSUPPORTED, "keys above 64 bits: FP64 or FP32 factors (no BF16 gathers)");
    for (int m = 0; m < t->layout.nmodes; m++)
        if (m != mode && !d_factors[m]) return fail(BLCO_ERR_INVALID, "null factor matrix");
    BLCO_CUDA(cudaSetDevice(t->device));
    cudaStream_t s = pick_stream(t, opts);
    const float* v32 = nullptr;
    if (t->resident) BLCO_TRY(values_f32(t, s, &v32));
    else BLCO_TRY(host_values_f32(t));
    MttkrpArgs a;
    memset(&a, 0, sizeof(a));
    a.coords = t->d_coords;
    a.vals = v32;
    a.nnz = t->nnz;
    a.mode = mode;
    a.rank = rank;
    for (int m = 0; m < t->layout.nmodes; m++) a.factors[m] = d_factors[m];
    a.out = d_out;
    a.factor_dtype = factor_dtype;
    a.thread_cf = opts ? opts->thread_cf : 2;
    BLCO_TRY(resolve_schedule(t, mode, rank, factor_dtype, opts ? opts->kernel : BLCO_KERNEL_AUTO, s, &a));
    if (!t->resident) return mttkrp_streamed(t, a, opts, s);
    return mttkrp_launch(t, a, s);
}

int blco_mttkrp_host(blco_tensor* t, int mode, int rank, const double* const* factors, double* out,
                     const blco_opts* opts)
{
    if (!t || !factors || !out) return fail(BLCO_ERR_INVALID, "null argument");
    if (mode < 0 || mode >= t->layout.nmodes) return fail(BLCO_ERR_INVALID, "mode out of range");
    if (rank < 1) return fail(BLCO_ERR_INVALID, "rank must be positive");
    BLCO_CUDA(cudaSetDevice(t->device));
    cudaStream_t s = pick_stream(t, opts);
    const int N = t->layout.nmodes;
    double* df[BLCO_MAX_MODES] = {};
    int st = BLCO_OK;
    for (int m = 0; m < N && st == BLCO_OK; m++) {
        size_t b = t->layout.dims[m] * (size_t)rank * sizeof(double);
        cudaError_t e = cudaMalloc(&df[m], b);
        const double* src = m == mode ? out : factors[m];
        if (e == cudaSuccess && src) e = cudaMemcpyAsync(df[m], src, b, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) st = cuda_fail(e, "factor upload", __FILE__, __LINE__);
    }
    if (st == BLCO_OK) st = blco_mttkrp(t, mode, rank, df, df[mode], opts);
    if (st == BLCO_OK) {
        cudaError_t e = cudaMemcpyAsync(out, df[mode], t->layout.dims[mode] * (size_t)rank * sizeof(double),
                                        cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_fail(e, "MTTKRP download", __FILE__, __LINE__);
    }
    cudaStreamSynchronize(s);
    for (int m = 0; m < N; m++) cudaFree(df[m]);
    return st;
}

int blco_cpals(blco_tensor* t, int rank, double* const* factors, double* lambda, int maxiter, double tol,
               const blco_opts* opts, double* fit_out, double* fits, int* iters_out)
{
    if (!t) return fail(BLCO_ERR_INVALID, "null tensor");
    if (maxiter < 0) return fail(BLCO_ERR_INVALID, "maxiter must be >= 0");
    BLCO_CUDA(cudaSetDevice(t->device));
    return cpals_host(t, rank, factors, lambda, maxiter, tol, opts, fit_out, fits, iters_out);
}

int blco_cpals_plan_create(blco_tensor* t, int rank, double* const* d_factors, double* d_lambda,
                           const blco_opts* opts, blco_cpals_plan** out)
{
    if (!out) return fail(BLCO_ERR_INVALID, "null output handle");
    if (!t) return fail(BLCO_ERR_INVALID, "null tensor");
    BLCO_CUDA(cudaSetDevice(t->device));
    return plan_create(t, rank, d_factors, d_lambda, opts, out);
}

int blco_cpals_plan_iterate(blco_cpals_plan* p, int iters, double tol, double* fits, int* iters_done)
{
    if (!p) return fail(BLCO_ERR_INVALID, "null plan");
    return plan_iterate(p, iters, tol, fits, iters_done, false);
}

int blco_cpals_plan_mttkrp_ms(const blco_cpals_plan* p, double* ms, int* calls) { return plan_mttkrp_ms(p, ms, calls); }

int blco_tensor_fibre_stats(blco_tensor* t, int mode, uint64_t* stats)
{
    if (!t || !stats) return fail(BLCO_ERR_INVALID, "null argument");
    if (!fibre_eligible(t, mode)) return fail(BLCO_ERR_UNSUPPORTED, "no fibre copy for this tensor and mode");
    cudaSetDevice(t->device);
    BLCO_TRY(build_fibre_copy(t, mode, pick_stream(t, nullptr)));
    const FibreCopy& f = t->fib[mode];
    stats[0] = (uint64_t)f.fmode;
    stats[1] = f.nf;
    stats[2] = f.nl;
    stats[3] = f.nfib;
    stats[4] = f.nf * (uint64_t)f.ninner + f.nfib + f.nl * (uint64_t)(f.ninner + 1);
    return BLCO_OK;
}

int blco_cpals_plan_condition(const blco_cpals_plan* p, double* cond, int* promoted)
{
    return plan_condition(p, cond, promoted);
}

int blco_cpals_plan_device_bytes(const blco_cpals_plan* p, uint64_t* bytes) { return plan_device_bytes(p, bytes); }

int blco_cpals_plan_destroy(blco_cpals_plan* p) { return plan_destroy(p); }

int blco_cpals_plan_set_reduce(blco_cpals_plan* p, blco_reduce_fn fn, void* ctx) { return plan_set_reduce(p, fn, ctx); }

int blco_cpals_plan_set_norm_sq(blco_cpals_plan* p, double norm_sq) { return plan_set_norm_sq(p, norm_sq); }

int blco_batch_create(int count, blco_tensor* const* tensors, const int* ranks, double* const* const* d_factors,
                      double* const* d_lambdas, double tol, const blco_opts* opts, blco_batch** out)
{
    if (!out) return fail(BLCO_ERR_INVALID, "null output handle");
    return batch_create(count, tensors, ranks, d_factors, d_lambdas, tol, opts, out);
}

int blco_batch_iterate(blco_batch* b, int iters, double* fits, int* iters_done)
{
    if (!b) return fail(BLCO_ERR_INVALID, "null batch");
    return batch_iterate(b, iters, fits, iters_done);
}

int blco_batch_destroy(blco_batch* b) { return batch_destroy(b); }

int blco_tune_space(blco_tune_config* configs)
{
    if (!configs) return fail(BLCO_ERR_INVALID, "null argument");
    for (int k = 0; k < BLCO_TUNE_CONFIGS; k++) {
        configs[k].kernel = TUNE_SPACE[k].kernel;
        configs[k].hot_chunk = TUNE_SPACE[k].hot_chunk;
        configs[k].interleave = TUNE_SPACE[k].interleave;
    }
    return BLCO_OK;
}

int blco_autotune(blco_tensor* t, int mode, int rank, int factor_dtype, int reps, const blco_opts* opts, float* ms,
                  int* best)
{
    if (!t) return fail(BLCO_ERR_INVALID, "null tensor");
    BLCO_CUDA(cudaSetDevice(t->device));
    float local[BLCO_TUNE_CONFIGS];
    BLCO_TRY(tune_sweep(t, mode, rank, factor_dtype, reps, pick_stream(t, opts), local));
    if (ms) memcpy(ms, local, sizeof(local));
    if (best) *best = tune_best(local);
    return BLCO_OK;
}

int blco_tune_features(const blco_tensor* t, int mode, int rank, int factor_dtype, float* features)
{
    if (!t || !features) return fail(BLCO_ERR_INVALID, "null argument");
    if (rank < 1) return fail(BLCO_ERR_INVALID, "rank must be positive");
    return tune_features(t, mode, rank, factor_dtype, features);
}

int blco_mlp_create(int hidden, uint64_t seed, int device, blco_mlp** out)
{
    if (!out) return fail(BLCO_ERR_INVALID, "null output handle");
    return mlp_create(hidden, seed, device, out);
}

int blco_mlp_num_params(const blco_mlp* net, int* n)
{
    if (!net || !n) return fail(BLCO_ERR_INVALID, "null argument");
    *n = mlp_num_params(net);
    return BLCO_OK;
}

int blco_mlp_set_params(blco_mlp* net, const float* params, int n)
{
    if (!net || !params) return fail(BLCO_ERR_INVALID, "null argument");
    return mlp_set_params(net, params, n);
}

int blco_mlp_get_params(const blco_mlp* net, float* params, int n)
{
    if (!net || !params) return fail(BLCO_ERR_INVALID, "null argument");
    return mlp_get_params(net, params, n);
}

int blco_mlp_predict(blco_mlp* net, const float* X, int n, float* out)
{
    if (!net || (n > 0 && (!X || !out))) return fail(BLCO_ERR_INVALID, "null argument");
    return mlp_predict(net, X, n, out);
}

int blco_mlp_grad(blco_mlp* net, const float* X, const float* Y, const float* mask, int n, float* grad, float* loss)
{
    if (!net || !X || !Y || !mask) return fail(BLCO_ERR_INVALID, "null argument");
    return mlp_grad(net, X, Y, mask, n, grad, loss);
}

int blco_mlp_train(blco_mlp* net, const float* X, const float* Y, const float* mask, int n, int epochs, int batch,
                   float lr, uint64_t seed, float* loss)
{
    if (!net || !X || !Y || !mask) return fail(BLCO_ERR_INVALID, "null argument");
    return mlp_train(net, X, Y, mask, n, epochs, batch, lr, seed, loss);
}

int blco_mlp_destroy(blco_mlp* net) { return mlp_destroy(net); }

int blco_selector_set(blco_mlp* net, float margin) { return selector_set(net, margin); }

int blco_select(blco_tensor* t, int mode, int rank, int factor_dtype, blco_mlp* net, float margin,
                const blco_opts* opts, int* config, int* used_sweep)
{
    if (!t || !config) return fail(BLCO_ERR_INVALID, "null argument");
    if (!t->resident) return fail(BLCO_ERR_UNSUPPORTED, "schedule selection needs a resident tensor");
    if (mode < 0 || mode >= t->layout.nmodes) return fail(BLCO_ERR_INVALID, "mode out of range");
    BLCO_CUDA(cudaSetDevice(t->device));
    int swept = 0;
    BLCO_TRY(select_config(t, mode, rank, factor_dtype, net, margin, pick_stream(t, opts), config, &swept));
    if (used_sweep) *used_sweep = swept;
    return BLCO_OK;
}

int blco_gram_f32(const float* d_U, uint64_t I, int rank, double* d_G, int tensor_cores, int device, void* stream)
{
    if (!d_U || !d_G) return fail(BLCO_ERR_INVALID, "null argument");
    if (rank < 1 || rank > 64) return fail(BLCO_ERR_UNSUPPORTED, "rank must be 1..64");
    BLCO_CUDA(cudaSetDevice(device));
    DeviceInfo di;
    BLCO_TRY(device_info(device, &di));
    return gram_f32(const_cast<float*>(d_U), I, rank, d_G, tensor_cores != 0, di.sm_count,
                    static_cast<cudaStream_t>(stream));
}

int blco_gram_tc_timeout_check(int device, int* timeout_status, int* after_status)
{
    if (!timeout_status || !after_status) return fail(BLCO_ERR_INVALID, "null argument");
    *timeout_status = *after_status = -1;
    return gram_tc_timeout_check(device, timeout_status, after_status);
}

int blco_encode_tns(const char* path, uint64_t max_block_size, const blco_opts* opts, blco_tensor** out,
                    blco_tns_info* info)
{
    if (!path || !out) return fail(BLCO_ERR_INVALID, "null argument");
    return encode_tns_impl(path, max_block_size, opts, out, info);
}

int blco_parse_decimal(const char* s, int len, double* out, int* consumed)
{
    if (!s || !out || len < 0) return 2;
    return parse_decimal_host(s, len, out, consumed);
}

int blco_batch_last_ms(const blco_batch* b, double* ms)
{
    if (!b || !ms) return fail(BLCO_ERR_INVALID, "null argument");
    *ms = batch_last_ms(b);
    return BLCO_OK;
}

int blco_batch_mttkrp_ms(blco_batch* b, double* ms)
{
    if (!b || !ms) return fail(BLCO_ERR_INVALID, "null argument");
    return batch_mttkrp_ms(b, ms);
}

} // extern "C"
