// tune.cu -- MTTKRP schedule selection: the exhaustive autotuner sweep, the
// per-mode features, and the learned selector (a small MLP trained and run
// by the kernels in this file).
//
// The reference picks an MTTKRP kernel with a fixed rule (-k 10,
// src/alto_dev.cu:1975,1996-2001: lvl3 when the target mode has at most 100
// rows, else lvl1).  Here a schedule is one of BLCO_TUNE_CONFIGS entries of
// TUNE_SPACE (kernel variant x heavy-row chunk x tile order).  The sweep
// times every valid entry on the tensor itself; the selector predicts, from
// per-mode statistics, log2(time / best time) of every entry and takes the
// smallest, falling back to the sweep when no other schedule group (the
// schedules that differ only in tile order form a group) is predicted to be
// slower by at least a margin.
//
// Network: F inputs -> H (ReLU) -> H (ReLU) -> K outputs, FP32.  Parameters
// are one flat array: W1[H][F] b1[H] W2[H][H] b2[H] W3[K][H] b3[K].  Loss:
// masked mean squared error over the valid entries.  Every reduction runs in
// a fixed order (no atomics), so training is deterministic for a seed.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "internal.cuh"

namespace blco {

const TuneCfg TUNE_SPACE[BLCO_TUNE_CONFIGS] = {
    {BLCO_KERNEL_LVL1, 0, 0},    {BLCO_KERNEL_LVL1, 0, 1},    {BLCO_KERNEL_LVL2, 512, 0},
    {BLCO_KERNEL_LVL2, 512, 1},  {BLCO_KERNEL_LVL2, 2048, 0}, {BLCO_KERNEL_LVL2, 2048, 1},
    {BLCO_KERNEL_LVL2, 128, 0},  {BLCO_KERNEL_LVL2, 128, 1},  {BLCO_KERNEL_LVL3, 0, 0},
    {BLCO_KERNEL_LVL3, 0, 1},    {BLCO_KERNEL_ATOMIC, 0, 0},  {BLCO_KERNEL_ATOMIC, 0, 1},
    {BLCO_KERNEL_FIBRE, 0, 0},   {BLCO_KERNEL_FIBRE, 0, 1},
};

namespace {

size_t dtype_bytes(int dtype) { return dtype == BLCO_DTYPE_F64 ? 8 : dtype == BLCO_DTYPE_F32 ? 4 : 2; }

bool cfg_valid(const blco_tensor* t, int mode, int rank, int dtype, int k)
{
    if (TUNE_SPACE[k].kernel == BLCO_KERNEL_LVL3)
        return mttkrp_select_kernel(t, mode, rank, BLCO_KERNEL_LVL3, dtype) == BLCO_KERNEL_LVL3;
    if (TUNE_SPACE[k].kernel == BLCO_KERNEL_FIBRE)
        return fibre_eligible(t, mode) && fibre_lanes(rank, dtype) > 0;
    return true;
}

// ------------------------------------------------------------ MLP kernels

constexpr int ML_THREADS = 256;

// Z = X W^T + b (n x out), A = relu(Z) or Z.
__global__ void k_mlp_fwd(const float* __restrict__ X, int n, int in, const float* __restrict__ W,
                          const float* __restrict__ b, int out, int relu, float* __restrict__ A)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * out) return;
    const int i = e / out, o = e % out;
    float z = b[o];
    for (int j = 0; j < in; j++) z = fmaf(X[(size_t)i * in + j], W[(size_t)o * in + j], z);
    A[e] = relu ? fmaxf(z, 0.f) : z;
}

// dOut = 2 * mask * (Out - Y) * inv_count; per-block partial losses.
__global__ void k_mlp_loss(const float* __restrict__ Out, const float* __restrict__ Y, const float* __restrict__ Mk,
                           int total, float inv_count, float* __restrict__ dOut, float* __restrict__ part)
{
    __shared__ float red[ML_THREADS];
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.f;
    if (e < total) {
        const float d = Mk[e] * (Out[e] - Y[e]);
        dOut[e] = 2.f * d * inv_count;
        l = d * d * inv_count;
    }
    red[threadIdx.x] = l;
    __syncthreads();
    for (int s = ML_THREADS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void k_mlp_sum(const float* __restrict__ part, int n, float* __restrict__ out)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        float s = 0.f;
        for (int i = 0; i < n; i++) s += part[i];
        *out = s;
    }
}

// dW[o][j] = sum_i dZ[i][o] X[i][j]; db[o] = sum_i dZ[i][o] (thread per weight).
__global__ void k_mlp_bwd_w(const float* __restrict__ dZ, const float* __restrict__ X, int n, int in, int out,
                            float* __restrict__ dW, float* __restrict__ db)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= out * (in + 1)) return;
    const int o = e / (in + 1), j = e % (in + 1);
    float s = 0.f;
    if (j < in) {
        for (int i = 0; i < n; i++) s = fmaf(dZ[(size_t)i * out + o], X[(size_t)i * in + j], s);
        dW[(size_t)o * in + j] = s;
    } else {
        for (int i = 0; i < n; i++) s += dZ[(size_t)i * out + o];
        db[o] = s;
    }
}

// dX[i][j] = (sum_o dZ[i][o] W[o][j]) * (Aprev[i][j] > 0): the gradient at
// the previous layer's pre-activation (its ReLU derivative applied).
__global__ void k_mlp_bwd_x(const float* __restrict__ dZ, const float* __restrict__ W, int n, int in, int out,
                            const float* __restrict__ Aprev, float* __restrict__ dX)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * in) return;
    const int i = e / in, j = e % in;
    float s = 0.f;
    for (int o = 0; o < out; o++) s = fmaf(dZ[(size_t)i * out + o], W[(size_t)o * in + j], s);
    dX[e] = Aprev[e] > 0.f ? s : 0.f;
}

__global__ void k_mlp_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                           float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const float gi = g[e];
    const float mi = b1 * m[e] + (1.f - b1) * gi;
    const float vi = b2 * v[e] + (1.f - b2) * gi * gi;
    m[e] = mi;
    v[e] = vi;
    p[e] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void k_mlp_gather(const float* __restrict__ src, const int* __restrict__ idx, int n, int width,
                             float* __restrict__ dst)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * width) return;
    dst[e] = src[(size_t)idx[e / width] * width + e % width];
}

inline unsigned blocks_for(size_t n) { return (unsigned)std::max<size_t>(1, (n + ML_THREADS - 1) / ML_THREADS); }

uint64_t splitmix(uint64_t& s)
{
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

} // namespace
} // namespace blco

struct blco_mlp {
    int F = BLCO_MLP_FEATURES, H = 64, K = BLCO_TUNE_CONFIGS;
    int nparams = 0;
    int device = 0;
    int cap = 0; // rows the work buffers hold
    float* d_params = nullptr;
    float* d_grad = nullptr;
    float* d_m = nullptr;
    float* d_v = nullptr;
    float *X = nullptr, *A1 = nullptr, *A2 = nullptr, *Out = nullptr, *Y = nullptr, *Mk = nullptr;
    float *dOut = nullptr, *dA2 = nullptr, *dA1 = nullptr, *part = nullptr, *loss = nullptr;
    int adam_t = 0;
    cudaStream_t s = nullptr;
};

namespace blco {
namespace {

struct PView {
    float *W1, *b1, *W2, *b2, *W3, *b3;
};

PView view(const blco_mlp* m, float* base)
{
    PView v;
    v.W1 = base;
    v.b1 = v.W1 + m->H * m->F;
    v.W2 = v.b1 + m->H;
    v.b2 = v.W2 + m->H * m->H;
    v.W3 = v.b2 + m->H;
    v.b3 = v.W3 + m->K * m->H;
    return v;
}

void mlp_free_work(blco_mlp* m)
{
    for (float** p : {&m->X, &m->A1, &m->A2, &m->Out, &m->Y, &m->Mk, &m->dOut, &m->dA2, &m->dA1, &m->part}) {
        cudaFree(*p);
        *p = nullptr;
    }
    m->cap = 0;
}

int mlp_reserve(blco_mlp* m, int n)
{
    if (n <= m->cap) return BLCO_OK;
    mlp_free_work(m);
    const size_t N = (size_t)n;
    cudaError_t e = cudaMalloc(&m->X, N * m->F * 4);
    if (e == cudaSuccess) e = cudaMalloc(&m->A1, N * m->H * 4);
    if (e == cudaSuccess) e = cudaMalloc(&m->A2, N * m->H * 4);
    if (e == cudaSuccess) e = cudaMalloc(&m->Out, N * m->K * 4);
    if (e == cudaSuccess) e = cudaMalloc(&m->Y, N * m->K * 4);
    if (e == cudaSuccess) e = cudaMalloc(&m->Mk, N * m->K * 4);
    if (e == cudaSuccess) e = cudaMalloc(&m->dOut, N * m->K * 4);
    if (e == cudaSuccess) e = cudaMalloc(&m->dA2, N * m->H * 4);
    if (e == cudaSuccess) e = cudaMalloc(&m->dA1, N * m->H * 4);
    if (e == cudaSuccess) e = cudaMalloc(&m->part, (N * m->K / ML_THREADS + 2) * 4);
    if (e != cudaSuccess) {
        mlp_free_work(m);
        return cuda_fail(e, "MLP work buffers", __FILE__, __LINE__);
    }
    m->cap = n;
    return BLCO_OK;
}

// Forward pass of the rows already in m->X.
int mlp_forward(blco_mlp* m, int n)
{
    PView p = view(m, m->d_params);
    k_mlp_fwd<<<blocks_for((size_t)n * m->H), ML_THREADS, 0, m->s>>>(m->X, n, m->F, p.W1, p.b1, m->H, 1, m->A1);
    BLCO_CHECK_LAUNCH("k_mlp_fwd");
    k_mlp_fwd<<<blocks_for((size_t)n * m->H), ML_THREADS, 0, m->s>>>(m->A1, n, m->H, p.W2, p.b2, m->H, 1, m->A2);
    BLCO_CHECK_LAUNCH("k_mlp_fwd");
    k_mlp_fwd<<<blocks_for((size_t)n * m->K), ML_THREADS, 0, m->s>>>(m->A2, n, m->H, p.W3, p.b3, m->K, 0, m->Out);
    BLCO_CHECK_LAUNCH("k_mlp_fwd");
    return BLCO_OK;
}

// Loss and gradient (into m->d_grad) of the rows in m->X / Y / Mk.
int mlp_backward(blco_mlp* m, int n, float inv_count)
{
    PView p = view(m, m->d_params);
    PView g = view(m, m->d_grad);
    const int total = n * m->K;
    const unsigned lb = blocks_for(total);
    k_mlp_loss<<<lb, ML_THREADS, 0, m->s>>>(m->Out, m->Y, m->Mk, total, inv_count, m->dOut, m->part);
    BLCO_CHECK_LAUNCH("k_mlp_loss");
    k_mlp_sum<<<1, 32, 0, m->s>>>(m->part, (int)lb, m->loss);
    BLCO_CHECK_LAUNCH("k_mlp_sum");
    k_mlp_bwd_w<<<blocks_for((size_t)m->K * (m->H + 1)), ML_THREADS, 0, m->s>>>(m->dOut, m->A2, n, m->H, m->K, g.W3,
                                                                               g.b3);
    BLCO_CHECK_LAUNCH("k_mlp_bwd_w");
    k_mlp_bwd_x<<<blocks_for((size_t)n * m->H), ML_THREADS, 0, m->s>>>(m->dOut, p.W3, n, m->H, m->K, m->A2, m->dA2);
    BLCO_CHECK_LAUNCH("k_mlp_bwd_x");
    k_mlp_bwd_w<<<blocks_for((size_t)m->H * (m->H + 1)), ML_THREADS, 0, m->s>>>(m->dA2, m->A1, n, m->H, m->H, g.W2,
                                                                               g.b2);
    BLCO_CHECK_LAUNCH("k_mlp_bwd_w");
    k_mlp_bwd_x<<<blocks_for((size_t)n * m->H), ML_THREADS, 0, m->s>>>(m->dA2, p.W2, n, m->H, m->H, m->A1, m->dA1);
    BLCO_CHECK_LAUNCH("k_mlp_bwd_x");
    k_mlp_bwd_w<<<blocks_for((size_t)m->H * (m->F + 1)), ML_THREADS, 0, m->s>>>(m->dA1, m->X, n, m->F, m->H, g.W1,
                                                                               g.b1);
    BLCO_CHECK_LAUNCH("k_mlp_bwd_w");
    return BLCO_OK;
}

float masked_inv_count(const float* Mk, size_t total)
{
    double c = 0.0;
    for (size_t i = 0; i < total; i++) c += Mk[i];
    return c > 0.0 ? (float)(1.0 / c) : 0.f;
}

} // namespace

// -------------------------------------------------------------- features

int tune_features(const blco_tensor* t, int mode, int rank, int dtype, float* f)
{
    const Layout& L = t->layout;
    if (mode < 0 || mode >= L.nmodes) return fail(BLCO_ERR_INVALID, "mode out of range");
    if (L.wide) return fail(BLCO_ERR_UNSUPPORTED, "keys above 64 bits have one MTTKRP schedule (nothing to select)");
    for (int i = 0; i < BLCO_MLP_FEATURES; i++) f[i] = 0.f;
    auto lg = [](double x) { return (float)std::log2(std::max(1.0, x)); };
    const double nnz = (double)t->nnz;
    const double sf = (double)dtype_bytes(dtype), so = dtype == BLCO_DTYPE_F64 ? 8.0 : 4.0;
    double other = 0.0;
    for (int m = 0; m < L.nmodes; m++)
        if (m != mode) other += (double)L.dims[m] * rank * sf;
    const double It = (double)L.dims[mode];
    const ModeStats& ms = t->stats[mode];
    const HotTable& ht = t->hot[mode];
    DeviceInfo di;
    BLCO_TRY(device_info(t->device, &di));
    f[0] = lg(nnz) / 32.f;
    f[1] = L.nmodes / 5.f;
    f[2] = lg(rank) / 8.f;
    f[3 + std::min(2, std::max(0, dtype))] = 1.f;
    f[6] = lg(It) / 32.f;
    f[7] = lg(other) / 40.f;
    f[8] = lg(It * rank * so) / 40.f;
    f[9] = (float)std::max(-4.0, std::min(4.0, std::log2(std::max(1.0, other) / (double)di.l2_bytes))) / 4.f;
    f[10] = It > 0 ? (float)(ms.nonempty_rows / It) : 0.f;
    f[11] = lg(nnz / std::max<double>(1.0, (double)ms.nonempty_rows)) / 16.f;
    f[12] = lg((double)ms.max_row_nnz) / 32.f;
    f[13] = nnz > 0 ? (float)(ht.hot_nnz / nnz) : 0.f;
    f[14] = ht.nhot / 4096.f;
    // share of the nonzeros in rows of length [1,2) [2,4) [4,16) [16,64)
    // [64,256) [256,4K) [4K,64K) [64K,...), from the log2 row-length counts
    // (a row in bucket b is taken to hold 1.5 * 2^b nonzeros, b > 0)
    static const int edges[9] = {0, 1, 2, 4, 6, 8, 12, 16, 40};
    double tot = 0.0, bucket[8] = {};
    for (int b = 0; b < 40; b++) {
        const double w = (double)ms.log2_hist[b] * (b == 0 ? 1.0 : 1.5 * std::ldexp(1.0, b));
        int k = 0;
        while (k < 7 && b >= edges[k + 1]) k++;
        bucket[k] += w;
        tot += w;
    }
    for (int k = 0; k < 8; k++) f[15 + k] = tot > 0 ? (float)(bucket[k] / tot) : 0.f;
    f[23] = mttkrp_select_kernel(t, mode, rank, BLCO_KERNEL_LVL3, dtype) == BLCO_KERNEL_LVL3 ? 1.f : 0.f;
    f[24] = lg((double)t->block_count) / 16.f;
    return BLCO_OK;
}

// ------------------------------------------------------------ the sweep

int tune_sweep(blco_tensor* t, int mode, int rank, int dtype, int reps, cudaStream_t s, float* ms_out)
{
    const Layout& L = t->layout;
    if (!t->resident) return fail(BLCO_ERR_UNSUPPORTED, "the autotuner needs a resident tensor");
    if (L.wide) return fail(BLCO_ERR_UNSUPPORTED, "keys above 64 bits have one MTTKRP schedule (nothing to tune)");
    if (mode < 0 || mode >= L.nmodes) return fail(BLCO_ERR_INVALID, "mode out of range");
    if (rank < 1 || rank > 256) return fail(BLCO_ERR_UNSUPPORTED, "rank must be 1..256");
    if (dtype < BLCO_DTYPE_F64 || dtype > BLCO_DTYPE_BF16) return fail(BLCO_ERR_INVALID, "unknown factor dtype");
    reps = std::max(1, reps);
    TuneCache& tc = t->tune[mode][dtype];
    if (tc.valid && tc.rank == rank) {
        if (ms_out) memcpy(ms_out, tc.ms, sizeof(tc.ms));
        return BLCO_OK;
    }
    const size_t fb = dtype_bytes(dtype), ob = dtype == BLCO_DTYPE_F64 ? 8 : 4;
    void* fac[BLCO_MAX_MODES] = {};
    void* out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int st = BLCO_OK;
    cudaError_t e = cudaSuccess;
    for (int m = 0; m < L.nmodes && e == cudaSuccess; m++) {
        const size_t bytes = L.dims[m] * (size_t)rank * fb;
        e = cudaMalloc(&fac[m], bytes);
        // any finite pattern times the same as real factors: 0x3f bytes are
        // 4.8e-4 in FP64, 0.75 in FP32 / BF16 halves
        if (e == cudaSuccess) e = cudaMemsetAsync(fac[m], 0x3f, bytes, s);
    }
    if (e == cudaSuccess) e = cudaMalloc(&out, L.dims[mode] * (size_t)rank * ob);
    if (e == cudaSuccess) e = cudaMemsetAsync(out, 0, L.dims[mode] * (size_t)rank * ob, s);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e != cudaSuccess) st = cuda_fail(e, "autotuner buffers", __FILE__, __LINE__);
    const void* vals = t->d_values;
    if (st == BLCO_OK && dtype != BLCO_DTYPE_F64) {
        const float* v32 = nullptr;
        st = values_f32(t, s, &v32);
        vals = v32;
    }
    float ms[BLCO_TUNE_CONFIGS];
    for (int k = 0; k < BLCO_TUNE_CONFIGS && st == BLCO_OK; k++) {
        ms[k] = -1.f;
        if (!cfg_valid(t, mode, rank, dtype, k)) continue;
        MttkrpArgs a;
        memset(&a, 0, sizeof(a));
        a.coords = t->d_coords;
        a.vals = vals;
        a.nnz = t->nnz;
        a.mode = mode;
        a.rank = rank;
        for (int m = 0; m < L.nmodes; m++) a.factors[m] = fac[m];
        a.out = out;
        a.factor_dtype = dtype;
        a.kernel = TUNE_SPACE[k].kernel;
        a.thread_cf = 2;
        a.hot_chunk = TUNE_SPACE[k].hot_chunk;
        a.interleave = TUNE_SPACE[k].interleave;
        if ((st = mttkrp_launch(t, a, s)) != BLCO_OK) break; // warm-up
        if ((e = cudaEventRecord(e0, s)) != cudaSuccess) break;
        for (int r = 0; r < reps && st == BLCO_OK; r++) st = mttkrp_launch(t, a, s);
        if (st != BLCO_OK) break;
        if ((e = cudaEventRecord(e1, s)) != cudaSuccess) break;
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess) break;
        float el = 0.f;
        if ((e = cudaEventElapsedTime(&el, e0, e1)) != cudaSuccess) break;
        ms[k] = el / reps;
    }
    if (st == BLCO_OK && e != cudaSuccess) st = cuda_fail(e, "autotuner timing", __FILE__, __LINE__);
    cudaStreamSynchronize(s);
    for (void* p : fac) cudaFree(p);
    cudaFree(out);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st != BLCO_OK) return st;
    memcpy(tc.ms, ms, sizeof(ms));
    tc.rank = rank;
    tc.valid = true;
    if (ms_out) memcpy(ms_out, ms, sizeof(ms));
    return BLCO_OK;
}

int tune_best(const float* ms)
{
    int best = -1;
    for (int k = 0; k < BLCO_TUNE_CONFIGS; k++)
        if (ms[k] >= 0.f && (best < 0 || ms[k] < ms[best])) best = k;
    return best;
}

// ------------------------------------------------------------------ MLP

int mlp_create(int hidden, uint64_t seed, int device, blco_mlp** out)
{
    *out = nullptr;
    if (hidden < 1 || hidden > 1024) return fail(BLCO_ERR_INVALID, "hidden width must be 1..1024");
    BLCO_CUDA(cudaSetDevice(device));
    DeviceInfo di;
    BLCO_TRY(device_info(device, &di));
    blco_mlp* m = new blco_mlp();
    m->H = hidden;
    m->device = device;
    m->nparams = m->H * m->F + m->H + m->H * m->H + m->H + m->K * m->H + m->K;
    cudaError_t e = cudaStreamCreateWithFlags(&m->s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&m->d_params, m->nparams * 4);
    if (e == cudaSuccess) e = cudaMalloc(&m->d_grad, m->nparams * 4);
    if (e == cudaSuccess) e = cudaMalloc(&m->d_m, m->nparams * 4);
    if (e == cudaSuccess) e = cudaMalloc(&m->d_v, m->nparams * 4);
    if (e == cudaSuccess) e = cudaMalloc(&m->loss, 4);
    if (e != cudaSuccess) {
        mlp_destroy(m);
        return cuda_fail(e, "MLP parameters", __FILE__, __LINE__);
    }
    // uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights, zero biases
    std::vector<float> h(m->nparams, 0.f);
    PView v = view(m, h.data());
    uint64_t st = seed;
    auto fill = [&](float* w, int rows, int fan_in) {
        const float a = 1.f / std::sqrt((float)fan_in);
        for (int i = 0; i < rows * fan_in; i++)
            w[i] = a * (2.f * (float)((splitmix(st) >> 11) * (1.0 / 9007199254740992.0)) - 1.f);
    };
    fill(v.W1, m->H, m->F);
    fill(v.W2, m->H, m->H);
    fill(v.W3, m->K, m->H);
    int rc = mlp_set_params(m, h.data(), m->nparams);
    if (rc != BLCO_OK) {
        mlp_destroy(m);
        return rc;
    }
    *out = m;
    return BLCO_OK;
}

int mlp_set_params(blco_mlp* m, const float* params, int n)
{
    if (n != m->nparams) return fail(BLCO_ERR_INVALID, "parameter count does not match the network");
    BLCO_CUDA(cudaSetDevice(m->device));
    BLCO_CUDA(cudaMemcpyAsync(m->d_params, params, n * 4, cudaMemcpyHostToDevice, m->s));
    BLCO_CUDA(cudaMemsetAsync(m->d_m, 0, n * 4, m->s));
    BLCO_CUDA(cudaMemsetAsync(m->d_v, 0, n * 4, m->s));
    BLCO_CUDA(cudaStreamSynchronize(m->s));
    m->adam_t = 0;
    return BLCO_OK;
}

int mlp_get_params(const blco_mlp* m, float* params, int n)
{
    if (n != m->nparams) return fail(BLCO_ERR_INVALID, "parameter count does not match the network");
    BLCO_CUDA(cudaSetDevice(m->device));
    BLCO_CUDA(cudaMemcpyAsync(params, m->d_params, n * 4, cudaMemcpyDeviceToHost, m->s));
    BLCO_CUDA(cudaStreamSynchronize(m->s));
    return BLCO_OK;
}

int mlp_num_params(const blco_mlp* m) { return m->nparams; }

int mlp_predict(blco_mlp* m, const float* X, int n, float* out)
{
    if (n < 0) return fail(BLCO_ERR_INVALID, "negative row count");
    if (n == 0) return BLCO_OK;
    BLCO_CUDA(cudaSetDevice(m->device));
    BLCO_TRY(mlp_reserve(m, n));
    BLCO_CUDA(cudaMemcpyAsync(m->X, X, (size_t)n * m->F * 4, cudaMemcpyHostToDevice, m->s));
    BLCO_TRY(mlp_forward(m, n));
    BLCO_CUDA(cudaMemcpyAsync(out, m->Out, (size_t)n * m->K * 4, cudaMemcpyDeviceToHost, m->s));
    BLCO_CUDA(cudaStreamSynchronize(m->s));
    return BLCO_OK;
}

int mlp_grad(blco_mlp* m, const float* X, const float* Y, const float* Mk, int n, float* grad, float* loss)
{
    if (n < 1) return fail(BLCO_ERR_INVALID, "need at least one row");
    BLCO_CUDA(cudaSetDevice(m->device));
    BLCO_TRY(mlp_reserve(m, n));
    const size_t nk = (size_t)n * m->K;
    BLCO_CUDA(cudaMemcpyAsync(m->X, X, (size_t)n * m->F * 4, cudaMemcpyHostToDevice, m->s));
    BLCO_CUDA(cudaMemcpyAsync(m->Y, Y, nk * 4, cudaMemcpyHostToDevice, m->s));
    BLCO_CUDA(cudaMemcpyAsync(m->Mk, Mk, nk * 4, cudaMemcpyHostToDevice, m->s));
    BLCO_TRY(mlp_forward(m, n));
    BLCO_TRY(mlp_backward(m, n, masked_inv_count(Mk, nk)));
    if (grad) BLCO_CUDA(cudaMemcpyAsync(grad, m->d_grad, m->nparams * 4, cudaMemcpyDeviceToHost, m->s));
    if (loss) BLCO_CUDA(cudaMemcpyAsync(loss, m->loss, 4, cudaMemcpyDeviceToHost, m->s));
    BLCO_CUDA(cudaStreamSynchronize(m->s));
    return BLCO_OK;
}

int mlp_train(blco_mlp* m, const float* X, const float* Y, const float* Mk, int n, int epochs, int batch, float lr,
              uint64_t seed, float* loss_out)
{
    if (n < 1 || epochs < 0 || batch < 1) return fail(BLCO_ERR_INVALID, "bad training sizes");
    BLCO_CUDA(cudaSetDevice(m->device));
    batch = std::min(batch, n);
    float *dX = nullptr, *dY = nullptr, *dM = nullptr;
    int* didx = nullptr;
    const size_t nk = (size_t)n * m->K;
    cudaError_t e = cudaMalloc(&dX, (size_t)n * m->F * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dY, nk * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dM, nk * 4);
    if (e == cudaSuccess) e = cudaMalloc(&didx, (size_t)n * epochs * sizeof(int) + sizeof(int));
    int st = e == cudaSuccess ? BLCO_OK : cuda_fail(e, "training buffers", __FILE__, __LINE__);
    if (st == BLCO_OK) st = mlp_reserve(m, batch);
    // the shuffled order of every epoch, made on the host from the seed
    std::vector<int> order((size_t)n * std::max(1, epochs));
    uint64_t rs = seed;
    for (int ep = 0; ep < epochs; ep++) {
        int* o = order.data() + (size_t)ep * n;
        for (int i = 0; i < n; i++) o[i] = i;
        for (int i = n - 1; i > 0; i--) std::swap(o[i], o[splitmix(rs) % (uint64_t)(i + 1)]);
    }
    if (st == BLCO_OK) {
        e = cudaMemcpyAsync(dX, X, (size_t)n * m->F * 4, cudaMemcpyHostToDevice, m->s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dY, Y, nk * 4, cudaMemcpyHostToDevice, m->s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dM, Mk, nk * 4, cudaMemcpyHostToDevice, m->s);
        if (e == cudaSuccess && epochs > 0)
            e = cudaMemcpyAsync(didx, order.data(), (size_t)n * epochs * sizeof(int), cudaMemcpyHostToDevice, m->s);
        if (e != cudaSuccess) st = cuda_fail(e, "training data", __FILE__, __LINE__);
    }
    // per-batch masked counts (host, from the same order)
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int ep = 0; ep < epochs && st == BLCO_OK; ep++) {
        for (int i0 = 0; i0 < n && st == BLCO_OK; i0 += batch) {
            const int nb = std::min(batch, n - i0);
            const int* idx = didx + (size_t)ep * n + i0;
            double cnt = 0.0;
            const int* ho = order.data() + (size_t)ep * n + i0;
            for (int i = 0; i < nb; i++)
                for (int k = 0; k < m->K; k++) cnt += Mk[(size_t)ho[i] * m->K + k];
            k_mlp_gather<<<blocks_for((size_t)nb * m->F), ML_THREADS, 0, m->s>>>(dX, idx, nb, m->F, m->X);
            k_mlp_gather<<<blocks_for((size_t)nb * m->K), ML_THREADS, 0, m->s>>>(dY, idx, nb, m->K, m->Y);
            k_mlp_gather<<<blocks_for((size_t)nb * m->K), ML_THREADS, 0, m->s>>>(dM, idx, nb, m->K, m->Mk);
            count_launch();
            count_launch();
            BLCO_CHECK_LAUNCH("k_mlp_gather");
            if ((st = mlp_forward(m, nb)) != BLCO_OK) break;
            if ((st = mlp_backward(m, nb, cnt > 0 ? (float)(1.0 / cnt) : 0.f)) != BLCO_OK) break;
            m->adam_t++;
            const float c1 = 1.f - std::pow(b1, (float)m->adam_t), c2 = 1.f - std::pow(b2, (float)m->adam_t);
            k_mlp_adam<<<blocks_for(m->nparams), ML_THREADS, 0, m->s>>>(m->d_params, m->d_grad, m->d_m, m->d_v,
                                                                       m->nparams, lr, b1, b2, eps, c1, c2);
            BLCO_CHECK_LAUNCH("k_mlp_adam");
        }
    }
    // loss over the whole set with the final parameters
    if (st == BLCO_OK && loss_out) {
        float total = 0.f;
        for (int i0 = 0; i0 < n && st == BLCO_OK; i0 += batch) {
            const int nb = std::min(batch, n - i0);
            e = cudaMemcpyAsync(m->X, dX + (size_t)i0 * m->F, (size_t)nb * m->F * 4, cudaMemcpyDeviceToDevice, m->s);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(m->Y, dY + (size_t)i0 * m->K, (size_t)nb * m->K * 4, cudaMemcpyDeviceToDevice, m->s);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(m->Mk, dM + (size_t)i0 * m->K, (size_t)nb * m->K * 4, cudaMemcpyDeviceToDevice,
                                    m->s);
            if (e != cudaSuccess) {
                st = cuda_fail(e, "loss evaluation", __FILE__, __LINE__);
                break;
            }
            if ((st = mlp_forward(m, nb)) != BLCO_OK) break;
            if ((st = mlp_backward(m, nb, masked_inv_count(Mk, nk))) != BLCO_OK) break;
            float l = 0.f;
            if ((e = cudaMemcpyAsync(&l, m->loss, 4, cudaMemcpyDeviceToHost, m->s)) != cudaSuccess ||
                (e = cudaStreamSynchronize(m->s)) != cudaSuccess) {
                st = cuda_fail(e, "loss evaluation", __FILE__, __LINE__);
                break;
            }
            total += l;
        }
        *loss_out = total;
    }
    cudaStreamSynchronize(m->s);
    cudaFree(dX);
    cudaFree(dY);
    cudaFree(dM);
    cudaFree(didx);
    return st;
}

int mlp_destroy(blco_mlp* m)
{
    if (!m) return BLCO_OK;
    if (m->s) cudaStreamSynchronize(m->s);
    mlp_free_work(m);
    cudaFree(m->d_params);
    cudaFree(m->d_grad);
    cudaFree(m->d_m);
    cudaFree(m->d_v);
    cudaFree(m->loss);
    if (m->s) cudaStreamDestroy(m->s);
    delete m;
    return BLCO_OK;
}

// ------------------------------------------------------------ selection

namespace {
std::mutex g_sel_mu;
blco_mlp* g_selector = nullptr;
float g_margin = 0.1f;
} // namespace

int selector_set(blco_mlp* net, float margin)
{
    std::lock_guard<std::mutex> lk(g_sel_mu);
    g_selector = net;
    g_margin = margin;
    return BLCO_OK;
}

int select_config(blco_tensor* t, int mode, int rank, int dtype, blco_mlp* net, float margin, cudaStream_t s,
                  int* cfg, int* used_sweep)
{
    *used_sweep = 0;
    if (net) {
        float f[BLCO_MLP_FEATURES], pred[BLCO_TUNE_CONFIGS];
        BLCO_TRY(tune_features(t, mode, rank, dtype, f));
        BLCO_TRY(mlp_predict(net, f, 1, pred));
        // best valid schedule, and the best of the other groups (schedules
        // differing only in tile order form a group: 2k, 2k + 1)
        int b0 = -1;
        for (int k = 0; k < BLCO_TUNE_CONFIGS; k++)
            if (cfg_valid(t, mode, rank, dtype, k) && (b0 < 0 || pred[k] < pred[b0])) b0 = k;
        int b1 = -1;
        for (int k = 0; k < BLCO_TUNE_CONFIGS; k++)
            if (k / 2 != b0 / 2 && cfg_valid(t, mode, rank, dtype, k) && (b1 < 0 || pred[k] < pred[b1])) b1 = k;
        if (b0 >= 0 && (b1 < 0 || pred[b1] - pred[b0] >= margin)) {
            *cfg = b0;
            return BLCO_OK;
        }
    }
    float ms[BLCO_TUNE_CONFIGS];
    BLCO_TRY(tune_sweep(t, mode, rank, dtype, 3, s, ms));
    *used_sweep = 1;
    *cfg = tune_best(ms);
    if (*cfg < 0) return fail(BLCO_ERR_UNSUPPORTED, "no valid MTTKRP schedule");
    return BLCO_OK;
}

int resolve_schedule(blco_tensor* t, int mode, int rank, int dtype, int requested, cudaStream_t s, MttkrpArgs* a)
{
    a->kernel = requested;
    if (requested != BLCO_KERNEL_TUNED && requested != BLCO_KERNEL_LEARNED) return BLCO_OK;
    if (t->layout.wide) {
        a->kernel = BLCO_KERNEL_LVL1; // keys above 64 bits have one kernel
        return BLCO_OK;
    }
    if (!t->resident) {
        a->kernel = BLCO_KERNEL_AUTO; // streamed blocks: the heuristic
        return BLCO_OK;
    }
    blco_mlp* net = nullptr;
    float margin = 0.f;
    if (requested == BLCO_KERNEL_LEARNED) {
        std::lock_guard<std::mutex> lk(g_sel_mu);
        net = g_selector;
        margin = g_margin;
    }
    int cfg = -1, swept = 0;
    BLCO_TRY(select_config(t, mode, rank, dtype, net, margin, s, &cfg, &swept));
    a->kernel = TUNE_SPACE[cfg].kernel;
    a->hot_chunk = TUNE_SPACE[cfg].hot_chunk;
    a->interleave = TUNE_SPACE[cfg].interleave;
    return BLCO_OK;
}

} // namespace blco
