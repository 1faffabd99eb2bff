// gram_tc.cu -- the mixed form's Gram U^T U on the 5th-generation tensor
// cores (tcgen05.mma, accumulator in TMEM), exact in the accumulator.
//
// U is I x R FP32, row-major (R <= 64).  Rows are taken 64 at a time (a
// tile).  In a tile every column c gets a power-of-two scale 2^e_c with
// max |u_c| < 2^e_c, and every value becomes three integer digits:
//   x = u * 2^(8 - e_c)  (|x| < 256),  d2 = rint(x),
//   d1 = rint(256 (x - d2)),  d0 = rint(256 (256 (x - d2) - d1)),
// so u = 2^(e_c - 8) (d2 + d1 / 2^8 + d0 / 2^16) to within 2^(e_c - 25)
// (FP32's own precision at the tile's largest value).  The digits are
// integers in [-256, 256], exact in BF16, and their products (at most 2^16)
// summed over the 64 rows stay below 2^22: every partial sum the tensor
// cores form in their FP32 accumulator is an integer below 2^24, hence
// exact, whatever the accumulator's rounding.  (A split into BF16 hi + lo
// parts, the usual scheme, is not exact there: the tensor cores' FP32
// accumulation leans low, and that bias reached the CP-ALS fit.)
//
// The digit rows form the K-major operand S of one tile: row i * RB + c
// holds digit i of column c (RB = R rounded up to 8, 16, 32 or 64; rows of
// padding columns are zero).  One MMA chain per 128-row group of S computes
// D = S S^T over the tile (M = 128, N = 3 RB rounded up to 16, K = 64 in 4
// MMAs); D[i RB + a][j RB + c] = sum over the tile of d_i(a) d_j(c).  The
// CTA reads D back (tcgen05.ld) and adds
//   2^(e_a - 8 - 8 i) 2^(e_c - 8 - 8 j) D[i RB + a][j RB + c]
// for i + j <= 2 (the terms of i + j >= 3 are below 2^-24 of the leading
// one) to FP64 sums: registers for RB <= 32, shared memory for RB = 64.
// The next tile's loads and digits overlap the previous tile's MMAs.  Each
// CTA writes its R x R FP64 partial; the partials are summed in FP64 in a
// fixed order.
//
// The same pass optionally scales U by inv (columns, written back) and
// writes the BF16 gather copy, as the CUDA-core Gram does; the Gram is then
// that of the values written back.
//
// Shared memory operand layout (the tcgen05 "no swizzle" K-major canonical
// layout): element (m, k) of S at byte ((k / 8) * ROWS + m) * 16 + (k % 8) *
// 2, ROWS = 128 per row group: 8 x 16-byte core matrices; the descriptor's
// leading byte offset (between the two 8-element K halves of one MMA) is
// ROWS * 16 and its stride byte offset (between 8-row groups) is 128.
//
// Every wait on the MMA completion barrier is bounded, and the decision is
// the CTA's (__syncthreads_or over the threads' waits): on timeout the CTA
// sets *err, stops issuing, waits once more (bounded) for the MMAs of the
// commit it gave up on, frees its TMEM and returns.  If that second wait
// also runs out, the TMEM is freed with those MMAs possibly still running;
// the host reports BLCO_ERR_TIMEOUT either way.
#include <cstdint>

#include "internal.cuh"

namespace blco {

namespace {

constexpr int TG_THREADS = 128;   // 4 warps: one TMEM lane quarter each
constexpr int TG_KT = 64;         // rows of U per tile (4 MMAs of K = 16)
constexpr int TG_CHUNKS = TG_KT / 8;
constexpr uint32_t TG_SPIN_MAX = 1u << 24;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// sm100 shared-memory matrix descriptor: no swizzle, K-major, start address,
// leading byte offset lbo, stride byte offset 128, descriptor version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)(128 >> 4) << 32) | (1ull << 46);
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, uint32_t limit)
{
    for (uint32_t it = 0; it < limit; it++) {
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

// Every thread waits (bounded) for the barrier phase; true on every thread
// of the CTA when any thread's wait ran out.  Also a CTA barrier.
__device__ __forceinline__ bool cta_wait_late(uint32_t bar, uint32_t parity, uint32_t limit)
{
    const int late = mbar_wait(bar, parity, limit) ? 0 : 1;
    return __syncthreads_or(late) != 0;
}

__device__ __forceinline__ uint16_t bf16_bits_rn(float x)
{
    const uint32_t u = __float_as_uint(x);
    return (uint16_t)((u + 0x7fffu + ((u >> 16) & 1u)) >> 16);
}

__device__ __forceinline__ float bf16_to_f32(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }

// e with m 2^e == x, m in [0.5, 1) (0 for x == 0), for x >= 0 given as bits.
__device__ __forceinline__ int exponent_of(uint32_t bits)
{
    if (bits >= 0x00800000u && bits < 0x7f800000u) return (int)(bits >> 23) - 126;
    int e = 0;
    frexpf(__uint_as_float(bits), &e); // zero, subnormal, inf, NaN
    return e;
}

// x * 2^k, exact for the |result| < 256 used here.
__device__ __forceinline__ float scale_pow2(float x, int k)
{
    if (k >= -126 && k <= 127) return x * __int_as_float((127 + k) << 23);
    return ldexpf(x, k);
}

// 2^k as a double (k within the normal range: |k| < 1000 here).
__device__ __forceinline__ double pow2_f64(int k) { return __longlong_as_double((long long)(1023 + k) << 52); }

// BF16 bits of an integer-valued float of magnitude <= 256 (exact: its low
// 16 bits are zero).
__device__ __forceinline__ uint32_t digit_bits(float d) { return __float_as_uint(d) >> 16; }

// 16 consecutive TMEM columns of this warp's 32 lanes.
__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&d)[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
                   "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]),
                   "=r"(d[15])
                 : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

template <int RB>
struct GramShape {
    static constexpr int MG = 3 * RB > 128 ? 2 : 1;    // 128-row groups of S
    static constexpr int ROWS = 128 * MG;               // rows of S per K chunk
    static constexpr int N = (3 * RB + 15) / 16 * 16;   // MMA N: digit rows of B
    static constexpr int NCOLS = MG == 2 ? 512 : N <= 32 ? 32 : N <= 64 ? 64 : 128;
    static constexpr int NI = (TG_CHUNKS * RB + TG_THREADS - 1) / TG_THREADS; // (chunk, column) items per thread
    static constexpr bool REG = RB <= 32;               // digit-row sums in registers
};

// Adds one tile's D (scales sd[j RB + c] = 2^(e_c - 8 - 8 j)) to this
// thread's digit-row sums: acc (registers, RB <= 32) or gsm (RB = 64).
template <int RB>
__device__ __forceinline__ void fold_tile(uint32_t tmem, int warp, int tid, const double* sd,
                                          double (&acc)[GramShape<RB>::REG ? RB : 1], double* gsm)
{
    using G = GramShape<RB>;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
    for (int g = 0; g < G::MG; g++) {
        const int q = g * 128 + tid;
        const bool act = q < 3 * RB;
        const int i = act ? q / RB : 3;
        const double wa = act ? sd[q] : 0.0;
#pragma unroll
        for (int c0 = 0; c0 < G::N; c0 += 16) {
            uint32_t d[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(g * 256 + c0), d);
#pragma unroll
            for (int x = 0; x < 16; x++) {
                const int n = c0 + x;
                if (n >= 3 * RB) continue;
                const int j = n / RB, c = n % RB;
                if (i + j <= 2) {
                    const double v = (double)__uint_as_float(d[x]) * sd[n]; // exact: D times a power of two
                    if constexpr (G::REG) acc[c] = fma(wa, v, acc[c]);
                    else gsm[q * (RB + 1) + c] = fma(wa, v, gsm[q * (RB + 1) + c]);
                }
            }
        }
    }
}

template <int RB, bool SCALE, bool BF16OUT>
__global__ void __launch_bounds__(TG_THREADS) k_gram_tc(float* __restrict__ U, uint64_t I, int R,
                                                        const double* __restrict__ inv,
                                                        uint16_t* __restrict__ bf16_out, uint64_t rows_per_cta,
                                                        double* __restrict__ partials, int* __restrict__ err,
                                                        uint32_t spin_max, int no_commit)
{
    using G = GramShape<RB>;
    __shared__ __align__(1024) uint4 S[TG_CHUNKS * G::ROWS];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    __shared__ uint32_t cmax[2][RB];   // per tile (double-buffered): largest |u| of each column, as bits
    __shared__ double sdj[2][3 * RB];  // per tile: 2^(e_c - 8 - 8 j) at j RB + c
    extern __shared__ __align__(16) double gsm[]; // [3 RB][RB + 1] FP64 digit-row sums
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint64_t r_beg = (uint64_t)blockIdx.x * rows_per_cta;
    const uint64_t r_end = min(I, r_beg + rows_per_cta);
    const int ntiles = r_beg < r_end ? (int)((r_end - r_beg + TG_KT - 1) / TG_KT) : 0;
    const int items = TG_CHUNKS * R;

    for (int i = tid; i < TG_CHUNKS * G::ROWS; i += TG_THREADS) S[i] = make_uint4(0, 0, 0, 0);
    for (int i = tid; i < 2 * RB; i += TG_THREADS) (&cmax[0][0])[i] = 0u;
    if constexpr (!G::REG)
        for (int i = tid; i < 3 * RB * (RB + 1); i += TG_THREADS) gsm[i] = 0.0;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(G::NCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    const uint32_t bar = smem_u32(&mbar);
    const uint32_t s_addr = smem_u32(S);
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(G::N >> 3) << 17) | ((128u >> 4) << 24);

    double acc[G::REG ? RB : 1];
#pragma unroll
    for (int c = 0; c < (G::REG ? RB : 1); c++) acc[c] = 0.0;

    uint32_t phase = 0; // commits issued (or, in the self-test, skipped)
    bool late = false;  // the same on every thread
    for (int t = 0; t < ntiles; t++) {
        const int b = t & 1;
        const uint64_t k0 = r_beg + (uint64_t)t * TG_KT;
        // item (j, c): column c of rows k0 + 8j .. +7
        float v[G::NI][8];
#pragma unroll
        for (int n = 0; n < G::NI; n++) {
            const int it = tid + n * TG_THREADS;
            float amax = 0.f;
#pragma unroll
            for (int e = 0; e < 8; e++) v[n][e] = 0.f;
            if (it < items) {
                const int j = it / R, c = it % R;
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const uint64_t row = k0 + 8 * j + e;
                    if (row < r_end) {
                        float x = U[row * R + c];
                        if (SCALE) x = (float)((double)x * inv[c]);
                        if constexpr (BF16OUT) {
                            const uint16_t h = bf16_bits_rn(x);
                            x = bf16_to_f32(h);
                            bf16_out[row * R + c] = h;
                        }
                        if (SCALE || BF16OUT) U[row * R + c] = x;
                        v[n][e] = x;
                        amax = fmaxf(amax, fabsf(x));
                    }
                }
                atomicMax(&cmax[b][c], __float_as_uint(amax));
            }
        }
        // the next tile's maxima (last read before the previous MMA issue)
        if (tid < RB) cmax[b ^ 1][tid] = 0u;
        __syncthreads();
        // digits of this tile, and its scales for the fold
        uint4 w[G::NI][3];
#pragma unroll
        for (int n = 0; n < G::NI; n++) {
            const int it = tid + n * TG_THREADS;
            const int c = it < items ? it % R : 0;
            const int ex = exponent_of(cmax[b][c]);
            uint32_t h[3][4];
#pragma unroll
            for (int e = 0; e < 8; e += 2) {
                uint32_t lohi[3][2];
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    const float x = scale_pow2(v[n][e + u], 8 - ex);
                    const float d2 = rintf(x);
                    const float r1 = (x - d2) * 256.f;
                    const float d1 = rintf(r1);
                    const float d0 = rintf((r1 - d1) * 256.f);
                    lohi[0][u] = digit_bits(d2);
                    lohi[1][u] = digit_bits(d1);
                    lohi[2][u] = digit_bits(d0);
                }
#pragma unroll
                for (int i = 0; i < 3; i++) h[i][e / 2] = lohi[i][0] | (lohi[i][1] << 16);
            }
#pragma unroll
            for (int i = 0; i < 3; i++) w[n][i] = make_uint4(h[i][0], h[i][1], h[i][2], h[i][3]);
        }
        for (int k = tid; k < 3 * RB; k += TG_THREADS) {
            const int j = k / RB, c = k % RB;
            sdj[b][k] = pow2_f64(exponent_of(cmax[b][c]) - 8 - 8 * j);
        }
        // the previous tile's MMAs: complete before S is rewritten and D read
        if (t > 0 && cta_wait_late(bar, (phase - 1) & 1, spin_max)) {
            late = true;
            break;
        }
#pragma unroll
        for (int n = 0; n < G::NI; n++) {
            const int it = tid + n * TG_THREADS;
            if (it < items) {
                const int j = it / R, c = it % R;
#pragma unroll
                for (int i = 0; i < 3; i++) S[j * G::ROWS + i * RB + c] = w[n][i];
            }
        }
        if (t > 0) fold_tile<RB>(tmem, warp, tid, sdj[b ^ 1], acc, gsm);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (tid == 0 && !no_commit) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int kk = 0; kk < TG_KT / 16; kk++) {
                const uint32_t kb = s_addr + (uint32_t)(kk * 2 * G::ROWS * 16);
                const uint64_t db = umma_desc(kb, G::ROWS * 16);
#pragma unroll
                for (int g = 0; g < G::MG; g++) {
                    const uint64_t da = umma_desc(kb + (uint32_t)(g * 128 * 16), G::ROWS * 16);
                    asm volatile("{\n\t.reg .pred p;\n\t"
                                 "setp.ne.b32 p, %4, 0;\n\t"
                                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                                 :
                                 : "r"(tmem + (uint32_t)(g * 256)), "l"(da), "l"(db), "r"(idesc), "r"(kk));
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                         : "memory");
        }
        phase++;
    }
    // the last tile
    if (!late && ntiles > 0) {
        if (cta_wait_late(bar, (phase - 1) & 1, spin_max)) late = true;
        else fold_tile<RB>(tmem, warp, tid, sdj[(ntiles - 1) & 1], acc, gsm);
    }
    if (late) {
        if (tid == 0) atomicExch(err, 1);
        // the MMAs of the commit given up on may still run: wait for them
        // once more before their TMEM is freed
        if (!no_commit) (void)cta_wait_late(bar, (phase - 1) & 1, spin_max);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(G::NCOLS));
    }
    if constexpr (G::REG) {
        if (tid < 3 * RB)
#pragma unroll
            for (int c = 0; c < RB; c++) gsm[tid * (RB + 1) + c] = acc[c];
        __syncthreads();
    }
    // G_cta[a][c] = sum over digits i of the rows i RB + a
    for (int e = tid; e < R * R; e += TG_THREADS) {
        const int a = e / R, c = e % R;
        partials[(size_t)blockIdx.x * R * R + e] =
            gsm[a * (RB + 1) + c] + gsm[(RB + a) * (RB + 1) + c] + gsm[(2 * RB + a) * (RB + 1) + c];
    }
}

template <int RB>
int gram_tc_dispatch(float* U, uint64_t I, int R, const double* inv, uint16_t* bf16_out, double* partials, int sm,
                     int* d_err, cudaStream_t s, int* nparts, uint32_t spin_max, int no_commit)
{
    using G = GramShape<RB>;
    // CTAs per SM: at most 8, and as many as TMEM holds (512 columns)
    const uint64_t per_sm = (uint64_t)std::min(8, 512 / G::NCOLS);
    const uint64_t tiles = (I + TG_KT - 1) / TG_KT;
    const uint64_t maxc = std::min<uint64_t>((uint64_t)sm * per_sm, (uint64_t)gram_tc_max_ctas(sm));
    const uint64_t tiles_per = std::max<uint64_t>(1, (tiles + maxc - 1) / maxc);
    const uint64_t rows_per = tiles_per * TG_KT;
    const int grid = (int)std::max<uint64_t>(1, (I + rows_per - 1) / rows_per);
    const size_t smem = (size_t)3 * RB * (RB + 1) * sizeof(double);
    void (*fn)(float*, uint64_t, int, const double*, uint16_t*, uint64_t, double*, int*, uint32_t, int);
    if (bf16_out) fn = inv ? k_gram_tc<RB, true, true> : k_gram_tc<RB, false, true>;
    else fn = inv ? k_gram_tc<RB, true, false> : k_gram_tc<RB, false, false>;
    BLCO_CUDA(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    fn<<<grid, TG_THREADS, smem, s>>>(U, I, R, inv, bf16_out, rows_per, partials, d_err, spin_max, no_commit);
    BLCO_CHECK_LAUNCH("k_gram_tc");
    *nparts = grid;
    return BLCO_OK;
}

} // namespace

int gram_tc_max_ctas(int sm) { return sm * 8; }

int gram_tc_launch(float* U, uint64_t I, int R, const double* inv, uint16_t* bf16_out, double* partials, int sm,
                   int* d_err, cudaStream_t s, int* nparts, uint32_t spin_max, int no_commit)
{
    if (R < 1 || R > 64) return fail(BLCO_ERR_UNSUPPORTED, "tensor-core Gram takes rank 1..64");
    if (spin_max == 0) spin_max = TG_SPIN_MAX;
    if (R <= 8) return gram_tc_dispatch<8>(U, I, R, inv, bf16_out, partials, sm, d_err, s, nparts, spin_max, no_commit);
    if (R <= 16)
        return gram_tc_dispatch<16>(U, I, R, inv, bf16_out, partials, sm, d_err, s, nparts, spin_max, no_commit);
    if (R <= 32)
        return gram_tc_dispatch<32>(U, I, R, inv, bf16_out, partials, sm, d_err, s, nparts, spin_max, no_commit);
    return gram_tc_dispatch<64>(U, I, R, inv, bf16_out, partials, sm, d_err, s, nparts, spin_max, no_commit);
}

} // namespace blco
