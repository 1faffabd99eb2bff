// gather_ceiling.cu -- the rate at which this GPU gathers random factor rows,
// the ceiling of the MTTKRP kernels (bench.py's roofline reports each
// MTTKRP's gathered rows per second against it).
//
//   bin/gather_ceiling [--rows N] [--gathers G] [--zipf S] [--inflight U] [--ctas-per-sm C]
//
// A gather is one factor row of 128 bytes (rank 32 in FP32) loaded by 8
// lanes with one 16-byte load each, U rows in flight per lane group (4, the
// MTTKRP kernels' step), C CTAs of 8 warps per SM (4: 32 warps, the MTTKRP
// kernels' occupancy); other U and C measure how the rate scales.  Row indices are
// drawn on the GPU: Zipf(S) over N rows by inverse CDF (the workload's
// per-mode distribution), and uniform over a 256k-row (32 MB, L2-resident)
// factor.  Prints one JSON line with G rows/s for each; best of 5 timed
// launches after one warm-up (CUDA events).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#define CK(x)                                                                  \
    do {                                                                       \
        cudaError_t e_ = (x);                                                  \
        if (e_ != cudaSuccess) {                                               \
            fprintf(stderr, "gather_ceiling: %s (%s:%d)\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
            return 1;                                                          \
        }                                                                      \
    } while (0)

__device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// idx[i]: Zipf by binary search of u in cdf (n entries), or uniform in [0, n) when cdf is null.
__global__ void k_draw(uint32_t* idx, uint64_t count, const double* cdf, uint32_t n, uint64_t seed)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = mix64(seed ^ (i * 0x2545f4914f6cdd1dull));
        if (!cdf) {
            idx[i] = (uint32_t)(r % n);
            continue;
        }
        const double u = (double)(r >> 11) * (1.0 / 9007199254740992.0);
        uint32_t lo = 0, hi = n - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (cdf[mid] < u) lo = mid + 1;
            else hi = mid;
        }
        idx[i] = lo;
    }
}

template <int U>
__global__ void __launch_bounds__(256) k_gather(const float4* __restrict__ F, const uint32_t* __restrict__ idx,
                                                uint64_t count, float4* __restrict__ sink)
{
    const int sub = threadIdx.x & 7;
    const uint64_t g = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 3;
    const uint64_t G = (gridDim.x * (uint64_t)blockDim.x) >> 3;
    const uint64_t per = count / G, a = g * per, b = a + per;
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    for (uint64_t q = a; q + U <= b; q += U) {
        float4 v[U];
#pragma unroll
        for (int u = 0; u < U; u++) v[u] = __ldg(F + (uint64_t)__ldg(idx + q + u) * 8 + sub);
#pragma unroll
        for (int u = 0; u < U; u++) acc.x += v[u].x, acc.y += v[u].y, acc.z += v[u].z, acc.w += v[u].w;
    }
    sink[blockIdx.x * (uint64_t)blockDim.x + threadIdx.x] = acc;
}

int main(int argc, char** argv)
{
    uint32_t rows = 2000000;
    uint64_t count = 64ull << 20;
    double s = 1.1;
    int inflight = 4, per_sm = 4;
    for (int i = 1; i + 1 < argc; i += 2) {
        if (!strcmp(argv[i], "--rows")) rows = (uint32_t)strtoul(argv[i + 1], nullptr, 10);
        else if (!strcmp(argv[i], "--gathers")) count = strtoull(argv[i + 1], nullptr, 10);
        else if (!strcmp(argv[i], "--zipf")) s = strtod(argv[i + 1], nullptr);
        else if (!strcmp(argv[i], "--inflight")) inflight = atoi(argv[i + 1]);
        else if (!strcmp(argv[i], "--ctas-per-sm")) per_sm = atoi(argv[i + 1]);
    }
    if (inflight != 1 && inflight != 2 && inflight != 4 && inflight != 8 && inflight != 16) {
        fprintf(stderr, "gather_ceiling: --inflight takes 1, 2, 4, 8 or 16\n");
        return 1;
    }
    if (per_sm < 1 || per_sm > 8) {
        fprintf(stderr, "gather_ceiling: --ctas-per-sm takes 1..8\n");
        return 1;
    }
    void (*kern)(const float4*, const uint32_t*, uint64_t, float4*) =
        inflight == 1 ? k_gather<1> : inflight == 2 ? k_gather<2> : inflight == 4 ? k_gather<4>
                                    : inflight == 8 ? k_gather<8> : k_gather<16>;
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0));
    const uint32_t l2rows = 262144;
    const uint32_t frows = std::max(rows, l2rows);
    float4* F = nullptr;
    uint32_t* idx = nullptr;
    float4* sink = nullptr;
    double* dcdf = nullptr;
    CK(cudaMalloc(&F, (size_t)frows * 128));
    CK(cudaMemset(F, 0, (size_t)frows * 128));
    CK(cudaMalloc(&idx, count * sizeof(uint32_t)));
    const int blocks = sms * per_sm;
    CK(cudaMalloc(&sink, (size_t)blocks * 256 * sizeof(float4)));
    std::vector<double> cdf(rows);
    double acc = 0.0;
    for (uint32_t k = 0; k < rows; k++) cdf[k] = (acc += std::pow((double)(k + 1), -s));
    for (auto& c : cdf) c /= acc;
    CK(cudaMalloc(&dcdf, rows * sizeof(double)));
    CK(cudaMemcpy(dcdf, cdf.data(), rows * sizeof(double), cudaMemcpyHostToDevice));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    double rate[2];
    for (int which = 0; which < 2; which++) {
        k_draw<<<sms * 8, 256>>>(idx, count, which == 0 ? dcdf : nullptr, which == 0 ? rows : l2rows, 12345u + which);
        CK(cudaGetLastError());
        kern<<<blocks, 256>>>(F, idx, count, sink);
        CK(cudaGetLastError());
        float best = 1e30f;
        for (int r = 0; r < 5; r++) {
            CK(cudaEventRecord(e0));
            kern<<<blocks, 256>>>(F, idx, count, sink);
            CK(cudaEventRecord(e1));
            CK(cudaEventSynchronize(e1));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            best = std::min(best, ms);
        }
        rate[which] = (double)count / (best * 1e-3) / 1e9;
    }
    printf("{\"zipf\": %.3f, \"rows\": %u, \"grows_per_s_zipf\": %.2f, \"grows_per_s_l2_resident\": %.2f, "
           "\"gathers\": %llu, \"row_bytes\": 128, \"sms\": %d, \"inflight\": %d, \"ctas_per_sm\": %d}\n",
           s, rows, rate[0], rate[1], (unsigned long long)count, sms, inflight, per_sm);
    cudaFree(F);
    cudaFree(idx);
    cudaFree(sink);
    cudaFree(dcdf);
    return 0;
}
