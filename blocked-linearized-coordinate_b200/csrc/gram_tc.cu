// gram_tc.cu -- the mixed form's Gram U^T U on the 5th-generation tensor
// cores (tcgen05.mma, accumulator in TMEM), as a split-BF16 product.
//
// U is I x R FP32, row-major (R <= 64).  Each FP32 value is split into two
// BF16 values, hi = bf16(u) and lo = bf16(u - hi) (hi + lo keeps 16
// mantissa bits).  A tile of 64 rows of U is written to shared memory as the
// K-major operand S (128 x 64 BF16): row m < R holds column m of hi, row
// R + m column m of lo, rows >= 2R zero.  One MMA chain computes
// D = S S^T (M = 128, N = 2R rounded up to 16, K = 64 per tile), whose four
// R x R blocks are hi.hi, hi.lo, lo.hi and lo.lo; their sum is the Gram of
// (hi + lo).  D accumulates in FP32 in TMEM over one tile (64 rows, 4
// MMAs); the CTA then reads it back (tcgen05.ld) and adds it to FP64
// accumulators in shared memory.  The tensor cores' FP32 accumulation is not
// round-to-nearest (it leans low, about 4e-7 relative over 512-row spans),
// and that bias reaches the CP-ALS fit through the Grams, so the FP32 spans
// are kept to one tile.
// Each CTA writes its R x R FP64 partial; the partials are summed in FP64
// in a fixed order.
//
// The same pass optionally scales U by inv (columns, written back) and
// writes the BF16 gather copy, as the CUDA-core Gram does.
//
// Shared memory operand layout (the tcgen05 "no swizzle" K-major canonical
// layout): element (m, k) of a tile at byte ((k / 8) * 128 + m) * 16 +
// (k % 8) * 2, i.e. 8 x 16-byte core matrices; the descriptor's leading
// byte offset (between the two 8-element K halves of one MMA) is 2048 and
// its stride byte offset (between 8-row groups) is 128.
//
// Every wait on the MMA completion barrier is bounded; on timeout the CTA
// sets *err, stops issuing work, still frees its TMEM and returns.
#include <cstdint>

#include "internal.cuh"

namespace blco {
namespace {

constexpr int TG_THREADS = 128;   // 4 warps: one TMEM lane quarter each
constexpr int TG_KT = 64;         // rows of U per tile (4 MMAs of K = 16)
constexpr int TG_FLUSH = 1;       // tiles per FP32 accumulation period
constexpr int TG_CHUNKS = TG_KT / 8;
constexpr uint32_t TG_SPIN_MAX = 1u << 24;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr)
{
    const uint64_t lbo = 2048 >> 4, sbo = 128 >> 4;
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | (lbo << 16) | (sbo << 32) | (1ull << 46);
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    for (uint32_t it = 0; it < TG_SPIN_MAX; it++) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(bar), "r"(parity)
                     : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ uint16_t bf16_bits_rn(float x)
{
    const uint32_t u = __float_as_uint(x);
    return (uint16_t)((u + 0x7fffu + ((u >> 16) & 1u)) >> 16);
}

__device__ __forceinline__ float bf16_to_f32(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }

template <bool SCALE, bool BF16OUT>
__global__ void __launch_bounds__(TG_THREADS) k_gram_tc(float* __restrict__ U, uint64_t I, int R,
                                                        const double* __restrict__ inv,
                                                        uint16_t* __restrict__ bf16_out, uint64_t rows_per_cta,
                                                        int ncols, double* __restrict__ partials,
                                                        int* __restrict__ err)
{
    __shared__ __align__(1024) uint4 S[TG_CHUNKS * 128]; // 16 KB operand tile
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    extern __shared__ __align__(16) double gacc[];       // [2R][R + 1] FP64 sums of D rows
    const int tid = threadIdx.x, warp = tid >> 5;
    const int N = ((2 * R + 15) / 16) * 16;
    const uint64_t r_beg = (uint64_t)blockIdx.x * rows_per_cta;
    const uint64_t r_end = min(I, r_beg + rows_per_cta);
    const int ntiles = r_beg < r_end ? (int)((r_end - r_beg + TG_KT - 1) / TG_KT) : 0;

    for (int i = tid; i < TG_CHUNKS * 128; i += TG_THREADS) S[i] = make_uint4(0, 0, 0, 0);
    for (int i = tid; i < 2 * R * (R + 1); i += TG_THREADS) gacc[i] = 0.0;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(ncols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    const uint32_t bar = smem_u32(&mbar);
    const uint32_t s_addr = smem_u32(S);
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((128u >> 4) << 24);
    const int items = TG_CHUNKS * R; // (chunk j, column c) pairs of one tile

    uint32_t phase = 0;   // completed commits so far
    bool ok = true;
    bool fresh = true;    // the next MMA overwrites D
    for (int t = 0; t < ntiles && ok; t++) {
        const uint64_t k0 = r_beg + (uint64_t)t * TG_KT;
        // Load and split this tile's values (column c of rows k0 + 8j .. +7)
        // while the previous tile's MMAs run; then wait for them before
        // overwriting S.
        uint4 hi_w[4], lo_w[4];
        int my_items = 0;
        uint16_t hb[4][8], lb[4][8];
        for (int it = tid, n = 0; it < items && n < 4; it += TG_THREADS, n++) {
            const int j = it / R, c = it % R;
#pragma unroll
            for (int e = 0; e < 8; e++) {
                const uint64_t row = k0 + 8 * j + e;
                float v = 0.f;
                if (row < r_end) {
                    v = U[row * R + c];
                    if (SCALE) v = (float)((double)v * inv[c]);
                    if constexpr (BF16OUT) {
                        const uint16_t b = bf16_bits_rn(v);
                        v = bf16_to_f32(b);
                        bf16_out[row * R + c] = b;
                    }
                    if (SCALE || BF16OUT) U[row * R + c] = v;
                }
                const uint16_t h = bf16_bits_rn(v);
                hb[n][e] = h;
                lb[n][e] = bf16_bits_rn(v - bf16_to_f32(h));
            }
            my_items = n + 1;
        }
#pragma unroll
        for (int n = 0; n < 4; n++) {
            hi_w[n] = make_uint4(hb[n][0] | ((uint32_t)hb[n][1] << 16), hb[n][2] | ((uint32_t)hb[n][3] << 16),
                                 hb[n][4] | ((uint32_t)hb[n][5] << 16), hb[n][6] | ((uint32_t)hb[n][7] << 16));
            lo_w[n] = make_uint4(lb[n][0] | ((uint32_t)lb[n][1] << 16), lb[n][2] | ((uint32_t)lb[n][3] << 16),
                                 lb[n][4] | ((uint32_t)lb[n][5] << 16), lb[n][6] | ((uint32_t)lb[n][7] << 16));
        }
        if (t > 0) {
            if (!mbar_wait(bar, (phase - 1) & 1)) {
                ok = false;
                atomicExch(err, 1);
            }
        }
        // every TG_FLUSH tiles: fold D into the FP64 sums (after the wait
        // above, all MMAs issued so far are complete)
        if (ok && t > 0 && t % TG_FLUSH == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int m = tid; // this thread's D row (TMEM lane)
            for (int c0 = 0; c0 < N; c0 += 16) {
                uint32_t d[16];
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                             : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]),
                               "=r"(d[7]), "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]),
                               "=r"(d[13]), "=r"(d[14]), "=r"(d[15])
                             : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (m < 2 * R) {
#pragma unroll
                    for (int x = 0; x < 16; x++) {
                        const int col = c0 + x;
                        if (col < 2 * R) gacc[m * (R + 1) + (col < R ? col : col - R)] += (double)__uint_as_float(d[x]);
                    }
                }
            }
            fresh = true;
        }
        if (!ok) break;
        for (int n = 0; n < my_items; n++) {
            const int it = tid + n * TG_THREADS;
            const int j = it / R, c = it % R;
            S[j * 128 + c] = hi_w[n];
            S[j * 128 + R + c] = lo_w[n];
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int kk = 0; kk < TG_KT / 16; kk++) {
                const uint64_t da = umma_desc(s_addr + kk * 2 * 2048);
                const uint32_t acc = (fresh && kk == 0) ? 0u : 1u;
                asm volatile("{\n\t.reg .pred p;\n\t"
                             "setp.ne.b32 p, %4, 0;\n\t"
                             "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                             :
                             : "r"(tmem), "l"(da), "l"(da), "r"(idesc), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                         : "memory");
        }
        fresh = false;
        phase++;
    }
    // last fold
    if (ok && ntiles > 0) {
        if (!mbar_wait(bar, (phase - 1) & 1)) {
            ok = false;
            atomicExch(err, 1);
        } else {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int m = tid;
            for (int c0 = 0; c0 < N; c0 += 16) {
                uint32_t d[16];
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                             : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]),
                               "=r"(d[7]), "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]),
                               "=r"(d[13]), "=r"(d[14]), "=r"(d[15])
                             : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (m < 2 * R) {
#pragma unroll
                    for (int x = 0; x < 16; x++) {
                        const int col = c0 + x;
                        if (col < 2 * R) gacc[m * (R + 1) + (col < R ? col : col - R)] += (double)__uint_as_float(d[x]);
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
    }
    // G_cta[a][c] = (hi_a + lo_a) . (hi_c + lo_c): rows a (hi) and R + a (lo)
    for (int e = tid; e < R * R; e += TG_THREADS) {
        const int a = e / R, c = e % R;
        partials[(size_t)blockIdx.x * R * R + e] = gacc[a * (R + 1) + c] + gacc[(R + a) * (R + 1) + c];
    }
}

} // namespace

int gram_tc_max_ctas(int sm) { return sm * 8; }

int gram_tc_launch(float* U, uint64_t I, int R, const double* inv, uint16_t* bf16_out, double* partials, int sm,
                   int* d_err, cudaStream_t s, int* nparts)
{
    if (R < 1 || R > 64) return fail(BLCO_ERR_UNSUPPORTED, "tensor-core Gram takes rank 1..64");
    const int N = ((2 * R + 15) / 16) * 16;
    int ncols = 32;
    while (ncols < N) ncols *= 2;
    // rows per CTA: whole tiles, at most 8 CTAs per SM
    const uint64_t tiles = (I + TG_KT - 1) / TG_KT;
    const uint64_t maxc = (uint64_t)gram_tc_max_ctas(sm);
    const uint64_t tiles_per = std::max<uint64_t>(1, (tiles + maxc - 1) / maxc);
    const uint64_t rows_per = tiles_per * TG_KT;
    const int grid = (int)std::max<uint64_t>(1, (I + rows_per - 1) / rows_per);
    const size_t smem = (size_t)2 * R * (R + 1) * sizeof(double);
    void (*fn)(float*, uint64_t, int, const double*, uint16_t*, uint64_t, int, double*, int*);
    if (bf16_out) fn = inv ? k_gram_tc<true, true> : k_gram_tc<false, true>;
    else fn = inv ? k_gram_tc<true, false> : k_gram_tc<false, false>;
    BLCO_CUDA(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    fn<<<grid, TG_THREADS, smem, s>>>(U, I, R, inv, bf16_out, rows_per, ncols, partials, d_err);
    BLCO_CHECK_LAUNCH("k_gram_tc");
    *nparts = grid;
    return BLCO_OK;
}

} // namespace blco
