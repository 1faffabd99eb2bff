// gram_tc.cu -- the mixed form's Gram U^T U on the 5th-generation tensor
// cores (tcgen05.mma, accumulator in TMEM), exact in the accumulator.
//
// U is I x R FP32, row-major (R <= 64).  Rows are taken 256 at a time (a
// super-tile), staged in shared memory.  In a
// super-tile every column c gets a power-of-two scale 2^e_c with
// max |u_c| < 2^e_c, and every value becomes four integer digits, most
// significant first:
//   x = u * 2^(8 - e_c)  (|x| < 256),  d_0 = rint(x),
//   d_k = rint(256^k x - sum_{l<k} 256^(k-l) d_l)  (k = 1, 2, 3),
// so u = 2^(e_c - 8) sum_k d_k / 256^k to within 2^(e_c - 33): exact for
// every value above 2^-9 of the column's largest in the super-tile (FP32
// keeps 24 bits), and within 2^-33 of that largest value below it (the Gram
// of a column whose magnitudes span many decades within a few hundred rows,
// as Zipf-skewed factor rows do, needs those low digits).  The digits are
// integers in [-256, 256], exact in BF16, and their products (at most 2^16)
// summed over at most 256 rows stay at or below 2^24: every partial sum the
// tensor cores form in their FP32 accumulator is an integer of at most
// 2^24, hence exact, whatever the accumulator's rounding.  (A split into
// BF16 hi + lo parts, the usual scheme, is not exact there: the tensor
// cores' FP32 accumulation leans low, and that bias reached the CP-ALS fit.)
//
// The digit rows form the K-major operand S of one super-tile: row k * RB +
// c holds digit k of column c (RB = R rounded up to 8, 16, 32 or 64; rows of
// padding columns are zero).  One MMA chain per 128-row group of S computes
// D = S S^T over the super-tile (M = 128, N = 4 RB, K = 256 in 16 MMAs);
// D[i RB + a][j RB + c] = sum over the super-tile of d_i(a) d_j(c).  The CTA
// reads D back (tcgen05.ld) and adds
//   2^(e_a - 8 - 8 i) 2^(e_c - 8 - 8 j) D[i RB + a][j RB + c]
// for every digit pair (i, j) to FP64 sums in registers.  (Dropping the
// small pairs would bias the diagonal: there the dropped products are
// squares.)  The CTA has 8 warps, two on each TMEM lane quarter, each
// folding half of D's columns.  Ranks above 32 split the columns in two
// halves (k_gram_tc_halves below).
// The next super-tile's loads overlap the previous one's MMAs.  Each CTA
// writes its R x R FP64 partial; the partials are summed in FP64 in a fixed
// order.
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
#include <algorithm>
#include <cstdint>

#include "internal.cuh"

namespace blco {

namespace {

constexpr int TG_LANES = 128;     // TMEM lanes: D rows, one quarter per warp (warp id mod 4)
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
    static_assert(RB == 8 || RB == 16 || RB == 32, "ranks above 32 take k_gram_tc_halves");
    static constexpr int ND = 4;                        // digits per value
    static constexpr int ROWS = 128;                    // rows of S per K chunk (M = 128)
    static constexpr int N = ND * RB;                   // MMA N: digit rows of B (32..128)
    static constexpr int NCOLS = N <= 32 ? 32 : N <= 64 ? 64 : 128;
    static constexpr int KS = 256;                      // rows per fold (a super-tile)
    static constexpr int CH = KS / 8;                   // K chunks of S
    // 8 warps: two per TMEM lane quarter, each pair splitting D's columns in halves
    static constexpr int THREADS = 256;
    static constexpr int HALVES = THREADS / TG_LANES;
    static constexpr int NV = (KS * RB / 4 + THREADS - 1) / THREADS; // float4 loads per thread
    static constexpr int MINB = 2;                      // CTAs per SM the registers must allow
    static constexpr size_t S_BYTES = (size_t)CH * ROWS * 16;
    static constexpr size_t STAGE_BYTES = (size_t)KS * RB * 4;
    static constexpr size_t GSM_BYTES = (size_t)ND * RB * (RB + 1) * 8;
    // dynamic shared memory: S and the staged rows; the FP64 sums reuse that
    // space once the last fold is done
    static constexpr size_t SMEM = S_BYTES + STAGE_BYTES > GSM_BYTES ? S_BYTES + STAGE_BYTES : GSM_BYTES;
};

// Adds one super-tile's D (scales sd[j RB + c] = 2^(e_c - 8 - 8 j)) to this
// thread's digit-row sums acc.
template <int RB>
__device__ __forceinline__ void fold_tile(uint32_t tmem, int warp, int tid, const double* sd, double (&acc)[RB])
{
    using G = GramShape<RB>;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int q = tid % TG_LANES, half = tid / TG_LANES;
    const uint32_t quarter = (uint32_t)(warp % 4) * 32;
    const bool act = q < G::ND * RB;
    const double wa = act ? sd[q] : 0.0;
#pragma unroll
    for (int c0 = 0; c0 < G::N / G::HALVES; c0 += 16) {
        const int cb = half * (G::N / G::HALVES) + c0; // this half's columns of D
        uint32_t d[16];
        tmem_ld16(tmem + (quarter << 16) + (uint32_t)cb, d);
#pragma unroll
        for (int x = 0; x < 16; x++) {
            const int n = cb + x;
            const int c = n % RB;
            if (act) {
                const double v = (double)__uint_as_float(d[x]) * sd[n]; // exact: D times a power of two
                acc[c] = fma(wa, v, acc[c]);
            }
        }
    }
}

template <int RB, bool SCALE, bool BF16OUT>
__global__ void __launch_bounds__(GramShape<RB>::THREADS, GramShape<RB>::MINB) k_gram_tc(float* __restrict__ U, uint64_t I, int R,
                                                        const double* __restrict__ inv,
                                                        uint16_t* __restrict__ bf16_out, uint64_t rows_per_cta,
                                                        double* __restrict__ partials, int* __restrict__ err,
                                                        uint32_t spin_max, int no_commit)
{
    using G = GramShape<RB>;
    extern __shared__ __align__(1024) unsigned char dsm[];
    uint4* S = reinterpret_cast<uint4*>(dsm);                          // [CH][ROWS] operand chunks
    float* stage = reinterpret_cast<float*>(dsm + G::S_BYTES);         // [KS][R] rows of U
    double* gsm = reinterpret_cast<double*>(dsm);                      // sums, after the last fold
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    __shared__ uint32_t cmax[2][RB];      // per super-tile (double-buffered): largest |u| per column, as bits
    __shared__ double sdj[2][G::ND * RB]; // per super-tile: 2^(e_c - 8 - 8 j) at j RB + c
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint64_t r_beg = (uint64_t)blockIdx.x * rows_per_cta;
    const uint64_t r_end = min(I, r_beg + rows_per_cta);
    const int nsup = r_beg < r_end ? (int)((r_end - r_beg + G::KS - 1) / G::KS) : 0;
    const int items = G::CH * R;          // (chunk j, column c): column c of 8 staged rows

    for (int i = tid; i < G::CH * G::ROWS; i += G::THREADS) S[i] = make_uint4(0, 0, 0, 0);
    for (int i = tid; i < 2 * RB; i += G::THREADS) (&cmax[0][0])[i] = 0u;
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

    double acc[RB];
#pragma unroll
    for (int c = 0; c < RB; c++) acc[c] = 0.0;

    uint32_t phase = 0; // commits issued (or, in the self-test, skipped)
    bool late = false;  // the same on every thread
    for (int t = 0; t < nsup; t++) {
        const int b = t & 1;
        const uint64_t k0 = r_beg + (uint64_t)t * G::KS;
        // stage rows k0 .. k0 + KS - 1 (contiguous in U; 16-byte aligned as
        // k0 is a multiple of 4), scaled / rounded and written back as asked
        {
            const uint64_t base = k0 * (uint64_t)R;                 // first element
            const uint64_t valid = (min(r_end, k0 + G::KS) - k0) * (uint64_t)R;
            const int nv4 = G::KS * R / 4;
            float4 buf[G::NV];
#pragma unroll
            for (int k = 0; k < G::NV; k++) {
                const int f = tid + k * G::THREADS;
                const uint64_t e0 = 4 * (uint64_t)f;
                float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                if (f < nv4 && e0 < valid) {
                    if (e0 + 4 <= valid) {
                        v = *reinterpret_cast<const float4*>(U + base + e0);
                    } else { // the last rows' ragged end (at most 3 elements)
                        v.x = U[base + e0];
                        if (e0 + 1 < valid) v.y = U[base + e0 + 1];
                        if (e0 + 2 < valid) v.z = U[base + e0 + 2];
                    }
                }
                buf[k] = v;
            }
#pragma unroll
            for (int k = 0; k < G::NV; k++) {
                const int f = tid + k * G::THREADS;
                if (f >= nv4) continue;
                if (SCALE || BF16OUT) {
                    const uint64_t e0 = 4 * (uint64_t)f;
                    float x[4] = {buf[k].x, buf[k].y, buf[k].z, buf[k].w};
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        if (e0 + u >= valid) continue;
                        const uint64_t gi = base + e0 + u;
                        float y = x[u];
                        if (SCALE) y = (float)((double)y * inv[(int)(gi % (uint64_t)R)]);
                        if constexpr (BF16OUT) {
                            const uint16_t h = bf16_bits_rn(y);
                            y = bf16_to_f32(h);
                            bf16_out[gi] = h;
                        }
                        x[u] = y;
                    }
                    buf[k] = make_float4(x[0], x[1], x[2], x[3]);
                    if (e0 + 4 <= valid) {
                        *reinterpret_cast<float4*>(U + base + e0) = buf[k];
                    } else if (e0 < valid) {
                        U[base + e0] = x[0];
                        if (e0 + 1 < valid) U[base + e0 + 1] = x[1];
                        if (e0 + 2 < valid) U[base + e0 + 2] = x[2];
                    }
                }
                reinterpret_cast<float4*>(stage)[f] = buf[k];
            }
        }
        // the next super-tile's maxima (last read before the previous MMA issue)
        if (tid < RB) cmax[b ^ 1][tid] = 0u;
        __syncthreads();
        for (int it = tid; it < items; it += G::THREADS) {
            const int j = it / R, c = it % R;
            float m = 0.f;
#pragma unroll
            for (int e = 0; e < 8; e++) m = fmaxf(m, fabsf(stage[(8 * j + e) * R + c]));
            atomicMax(&cmax[b][c], __float_as_uint(m));
        }
        __syncthreads();
        for (int k = tid; k < G::ND * RB; k += G::THREADS)
            sdj[b][k] = pow2_f64(exponent_of(cmax[b][k % RB]) - 8 - 8 * (k / RB));
        // the previous super-tile's MMAs: complete before S is rewritten and D read
        if (t > 0 && cta_wait_late(bar, (phase - 1) & 1, spin_max)) {
            late = true;
            break;
        }
        // digits of this super-tile into S
        for (int it = tid; it < items; it += G::THREADS) {
            const int j = it / R, c = it % R;
            const int ex = exponent_of(cmax[b][c]);
            uint32_t h[G::ND][4];
#pragma unroll
            for (int e = 0; e < 8; e += 2) {
                uint32_t lohi[G::ND][2];
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    // every step exact: x has 24 significant bits, the
                    // remainders shrink by 2^8 and stay in [-0.5, 0.5] * 2^8
                    float r = scale_pow2(stage[(8 * j + e + u) * R + c], 8 - ex);
#pragma unroll
                    for (int k = 0; k < G::ND; k++) {
                        const float d = rintf(r);
                        lohi[k][u] = digit_bits(d);
                        r = (r - d) * 256.f;
                    }
                }
#pragma unroll
                for (int k = 0; k < G::ND; k++) h[k][e / 2] = lohi[k][0] | (lohi[k][1] << 16);
            }
#pragma unroll
            for (int k = 0; k < G::ND; k++) S[j * G::ROWS + k * RB + c] = make_uint4(h[k][0], h[k][1], h[k][2], h[k][3]);
        }
        if (t > 0) fold_tile<RB>(tmem, warp, tid, sdj[b ^ 1], acc);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (tid == 0 && !no_commit) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll 1
            for (int kk = 0; kk < G::KS / 16; kk++) {
                const uint64_t dd = umma_desc(s_addr + (uint32_t)(kk * 2 * G::ROWS * 16), G::ROWS * 16);
                asm volatile("{\n\t.reg .pred p;\n\t"
                             "setp.ne.b32 p, %4, 0;\n\t"
                             "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                             :
                             : "r"(tmem), "l"(dd), "l"(dd), "r"(idesc), "r"(kk));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                         : "memory");
        }
        phase++;
    }
    // the last super-tile
    if (!late && nsup > 0) {
        if (cta_wait_late(bar, (phase - 1) & 1, spin_max)) late = true;
        else fold_tile<RB>(tmem, warp, tid, sdj[(nsup - 1) & 1], acc);
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
    {
        // S and the staged rows are no longer read (barrier above): the sums
        // go there, the second half of the CTA adding its columns' share
        const int q = tid % TG_LANES;
#pragma unroll
        for (int h = 0; h < G::HALVES; h++) {
            if (tid / TG_LANES == h && q < G::ND * RB)
#pragma unroll
                for (int c = 0; c < RB; c++) gsm[q * (RB + 1) + c] = (h ? gsm[q * (RB + 1) + c] : 0.0) + acc[c];
            __syncthreads();
        }
    }
    // G_cta[a][c] = sum over digits i of the rows i RB + a
    for (int e = tid; e < R * R; e += G::THREADS) {
        const int a = e / R, c = e % R;
        double g = 0.0;
#pragma unroll
        for (int i = 0; i < G::ND; i++) g += gsm[(i * RB + a) * (RB + 1) + c];
        partials[(size_t)blockIdx.x * R * R + e] = g;
    }
}

template <int RB>
int gram_tc_dispatch(float* U, uint64_t I, int R, const double* inv, uint16_t* bf16_out, double* partials, int sm,
                     int* d_err, cudaStream_t s, int* nparts, uint32_t spin_max, int no_commit)
{
    using G = GramShape<RB>;
    const size_t smem = G::SMEM;
    void (*fn)(float*, uint64_t, int, const double*, uint16_t*, uint64_t, double*, int*, uint32_t, int);
    if (bf16_out) fn = inv ? k_gram_tc<RB, true, true> : k_gram_tc<RB, false, true>;
    else fn = inv ? k_gram_tc<RB, true, false> : k_gram_tc<RB, false, false>;
    BLCO_CUDA(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    BLCO_CUDA(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                   (int)cudaSharedmemCarveoutMaxShared));
    // CTAs per SM: as many as the registers, the shared memory and TMEM
    // (512 columns) hold at once, at most 8: one wave
    cudaFuncAttributes fa;
    BLCO_CUDA(cudaFuncGetAttributes(&fa, (const void*)fn));
    int dev = 0, regs_sm = 65536, smem_sm = 0, smem_rsv = 0;
    BLCO_CUDA(cudaGetDevice(&dev));
    BLCO_CUDA(cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev));
    BLCO_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    BLCO_CUDA(cudaDeviceGetAttribute(&smem_rsv, cudaDevAttrReservedSharedMemoryPerBlock, dev));
    const int by_regs = regs_sm / (std::max(1, fa.numRegs) * G::THREADS);
    const int by_smem = smem_sm / (int)(smem + fa.sharedSizeBytes + (size_t)smem_rsv);
    const uint64_t per_sm = (uint64_t)std::max(1, std::min({8, 512 / G::NCOLS, by_regs, by_smem}));
    const uint64_t sups = (I + G::KS - 1) / G::KS;
    const uint64_t maxc = std::min<uint64_t>((uint64_t)sm * per_sm, (uint64_t)gram_tc_max_ctas(sm));
    const uint64_t sups_per = std::max<uint64_t>(1, (sups + maxc - 1) / maxc);
    const uint64_t rows_per = sups_per * G::KS;
    const int grid = (int)std::max<uint64_t>(1, (I + rows_per - 1) / rows_per);
    fn<<<grid, G::THREADS, smem, s>>>(U, I, R, inv, bf16_out, rows_per, partials, d_err, spin_max, no_commit);
    BLCO_CHECK_LAUNCH("k_gram_tc");
    *nparts = grid;
    return BLCO_OK;
}

// Ranks 33..64: the columns in two halves, A = columns 0..31 and B = the
// rest (zero-padded to 32), each with its own 128 digit rows (four digits of
// 32 columns), so every MMA keeps M = N = 128 and the sums stay in
// registers.  Per super-tile three MMA chains fill three TMEM regions:
// A A^T, A B^T and B B^T (B A^T is the transpose of A B^T); warps 0-3 fold
// the digit rows of A (the AA and AB regions), warps 4-7 those of B (BB).
constexpr int TH_THREADS = 256;
constexpr int TH_KS = 256;               // rows per super-tile
constexpr int TH_CH = TH_KS / 8;         // K chunks of S
constexpr int TH_NV = (TH_KS * 64 / 4 + TH_THREADS - 1) / TH_THREADS; // float4 loads per thread
constexpr size_t TH_S_BYTES = (size_t)TH_CH * 128 * 16; // one half's operand
constexpr size_t TH_STAGE_BYTES = (size_t)TH_KS * 64 * 4;
constexpr size_t TH_SMEM = 2 * TH_S_BYTES + TH_STAGE_BYTES;
constexpr size_t TH_GSM_BYTES = (size_t)3 * 128 * 33 * 8;  // sums, over S once the last fold is done
static_assert(TH_GSM_BYTES <= TH_SMEM, "tensor-core Gram: the sums must fit the operand space");

// Adds region d (128 columns: digit j of column c at j * 32 + c) of one
// super-tile to acc[c]: weights wa (this row's scale) and sd[j * 64 + off + c].
__device__ __forceinline__ void fold_half(uint32_t taddr, double wa, const double* sd, int off, double (&acc)[32])
{
#pragma unroll
    for (int c0 = 0; c0 < 128; c0 += 16) {
        uint32_t d[16];
        tmem_ld16(taddr + (uint32_t)c0, d);
#pragma unroll
        for (int x = 0; x < 16; x++) {
            const int n = c0 + x, j = n / 32, c = n % 32;
            const double v = (double)__uint_as_float(d[x]) * sd[j * 64 + off + c]; // exact: D times a power of two
            acc[c] = fma(wa, v, acc[c]);
        }
    }
}

template <bool SCALE, bool BF16OUT>
__global__ void __launch_bounds__(TH_THREADS, 1) k_gram_tc_halves(float* __restrict__ U, uint64_t I, int R,
                                                                const double* __restrict__ inv,
                                                                uint16_t* __restrict__ bf16_out, uint64_t rows_per_cta,
                                                                double* __restrict__ partials, int* __restrict__ err,
                                                                uint32_t spin_max, int no_commit)
{
    extern __shared__ __align__(1024) unsigned char dsm[];
    uint4* SA = reinterpret_cast<uint4*>(dsm);                        // [CH][128]
    uint4* SB = reinterpret_cast<uint4*>(dsm + TH_S_BYTES);           // [CH][128]
    float* stage = reinterpret_cast<float*>(dsm + 2 * TH_S_BYTES);    // [KS][R]
    double* gsm = reinterpret_cast<double*>(dsm);                     // [3][128][33] at the end
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    __shared__ uint32_t cmax[2][64];
    __shared__ double sdj[2][4 * 64];  // per super-tile: 2^(e_c - 8 - 8 j) at j 64 + c
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint64_t r_beg = (uint64_t)blockIdx.x * rows_per_cta;
    const uint64_t r_end = min(I, r_beg + rows_per_cta);
    const int nsup = r_beg < r_end ? (int)((r_end - r_beg + TH_KS - 1) / TH_KS) : 0;
    const int items = TH_CH * R;

    for (int i = tid; i < 2 * TH_CH * 128; i += TH_THREADS) SA[i] = make_uint4(0, 0, 0, 0); // SA and SB
    for (int i = tid; i < 2 * 64; i += TH_THREADS) (&cmax[0][0])[i] = 0u;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    const uint32_t bar = smem_u32(&mbar);
    const uint32_t sa_addr = smem_u32(SA), sb_addr = smem_u32(SB);
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(128 >> 3) << 17) | ((128u >> 4) << 24);
    const bool rows_a = warp < 4;  // this warp folds A's digit rows (else B's)
    const int q = (warp % 4) * 32 + lane; // digit row: digit q / 32 of column q % 32 of the half
    const uint32_t trow = tmem + ((uint32_t)((warp % 4) * 32) << 16);

    double acc0[32], acc1[32]; // A rows: AA and AB sums; B rows: BB sums in acc0
#pragma unroll
    for (int c = 0; c < 32; c++) acc0[c] = 0.0, acc1[c] = 0.0;
    auto fold = [&](const double* sd) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int i = q / 32, a = q % 32;
        if (rows_a) {
            const double wa = sd[i * 64 + a];
            fold_half(trow + 0, wa, sd, 0, acc0);     // A A^T
            fold_half(trow + 128, wa, sd, 32, acc1);  // A B^T
        } else {
            const double wb = sd[i * 64 + 32 + a];
            fold_half(trow + 256, wb, sd, 32, acc0);  // B B^T
        }
    };

    uint32_t phase = 0;
    bool late = false;
    for (int t = 0; t < nsup; t++) {
        const int b = t & 1;
        const uint64_t k0 = r_beg + (uint64_t)t * TH_KS;
        {
            const uint64_t base = k0 * (uint64_t)R;
            const uint64_t valid = (min(r_end, k0 + TH_KS) - k0) * (uint64_t)R;
            const int nv4 = TH_KS * R / 4;
            float4 buf[TH_NV];
#pragma unroll
            for (int k = 0; k < TH_NV; k++) {
                const int f = tid + k * TH_THREADS;
                const uint64_t e0 = 4 * (uint64_t)f;
                float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                if (f < nv4 && e0 < valid) {
                    if (e0 + 4 <= valid) {
                        v = *reinterpret_cast<const float4*>(U + base + e0);
                    } else {
                        v.x = U[base + e0];
                        if (e0 + 1 < valid) v.y = U[base + e0 + 1];
                        if (e0 + 2 < valid) v.z = U[base + e0 + 2];
                    }
                }
                buf[k] = v;
            }
#pragma unroll
            for (int k = 0; k < TH_NV; k++) {
                const int f = tid + k * TH_THREADS;
                if (f >= nv4) continue;
                if (SCALE || BF16OUT) {
                    const uint64_t e0 = 4 * (uint64_t)f;
                    float x[4] = {buf[k].x, buf[k].y, buf[k].z, buf[k].w};
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        if (e0 + u >= valid) continue;
                        const uint64_t gi = base + e0 + u;
                        float y = x[u];
                        if (SCALE) y = (float)((double)y * inv[(int)(gi % (uint64_t)R)]);
                        if constexpr (BF16OUT) {
                            const uint16_t h = bf16_bits_rn(y);
                            y = bf16_to_f32(h);
                            bf16_out[gi] = h;
                        }
                        x[u] = y;
                    }
                    buf[k] = make_float4(x[0], x[1], x[2], x[3]);
                    if (e0 + 4 <= valid) {
                        *reinterpret_cast<float4*>(U + base + e0) = buf[k];
                    } else if (e0 < valid) {
                        U[base + e0] = x[0];
                        if (e0 + 1 < valid) U[base + e0 + 1] = x[1];
                        if (e0 + 2 < valid) U[base + e0 + 2] = x[2];
                    }
                }
                reinterpret_cast<float4*>(stage)[f] = buf[k];
            }
        }
        if (tid < 64) cmax[b ^ 1][tid] = 0u;
        __syncthreads();
        for (int it = tid; it < items; it += TH_THREADS) {
            const int j = it / R, c = it % R;
            float m = 0.f;
#pragma unroll
            for (int e = 0; e < 8; e++) m = fmaxf(m, fabsf(stage[(8 * j + e) * R + c]));
            atomicMax(&cmax[b][c], __float_as_uint(m));
        }
        __syncthreads();
        for (int k = tid; k < 4 * 64; k += TH_THREADS)
            sdj[b][k] = pow2_f64(exponent_of(cmax[b][k % 64]) - 8 - 8 * (k / 64));
        if (t > 0 && cta_wait_late(bar, (phase - 1) & 1, spin_max)) {
            late = true;
            break;
        }
        for (int it = tid; it < items; it += TH_THREADS) {
            const int j = it / R, c = it % R;
            const int ex = exponent_of(cmax[b][c]);
            uint32_t h[4][4];
#pragma unroll
            for (int e = 0; e < 8; e += 2) {
                uint32_t lohi[4][2];
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    float r = scale_pow2(stage[(8 * j + e + u) * R + c], 8 - ex);
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        const float d = rintf(r);
                        lohi[k][u] = digit_bits(d);
                        r = (r - d) * 256.f;
                    }
                }
#pragma unroll
                for (int k = 0; k < 4; k++) h[k][e / 2] = lohi[k][0] | (lohi[k][1] << 16);
            }
            uint4* S = c < 32 ? SA : SB;
            const int cc = c % 32;
#pragma unroll
            for (int k = 0; k < 4; k++) S[j * 128 + k * 32 + cc] = make_uint4(h[k][0], h[k][1], h[k][2], h[k][3]);
        }
        if (t > 0) fold(sdj[b ^ 1]);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (tid == 0 && !no_commit) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll 1
            for (int kk = 0; kk < TH_KS / 16; kk++) {
                const uint32_t off = (uint32_t)(kk * 2 * 128 * 16);
                const uint64_t da = umma_desc(sa_addr + off, 128 * 16);
                const uint64_t db = umma_desc(sb_addr + off, 128 * 16);
                asm volatile("{\n\t.reg .pred p;\n\t"
                             "setp.ne.b32 p, %4, 0;\n\t"
                             "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                             :
                             : "r"(tmem), "l"(da), "l"(da), "r"(idesc), "r"(kk));
                asm volatile("{\n\t.reg .pred p;\n\t"
                             "setp.ne.b32 p, %4, 0;\n\t"
                             "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                             :
                             : "r"(tmem + 128u), "l"(da), "l"(db), "r"(idesc), "r"(kk));
                asm volatile("{\n\t.reg .pred p;\n\t"
                             "setp.ne.b32 p, %4, 0;\n\t"
                             "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                             :
                             : "r"(tmem + 256u), "l"(db), "l"(db), "r"(idesc), "r"(kk));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                         : "memory");
        }
        phase++;
    }
    if (!late && nsup > 0) {
        if (cta_wait_late(bar, (phase - 1) & 1, spin_max)) late = true;
        else fold(sdj[(nsup - 1) & 1]);
    }
    if (late) {
        if (tid == 0) atomicExch(err, 1);
        if (!no_commit) (void)cta_wait_late(bar, (phase - 1) & 1, spin_max);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
    }
    // sums into shared memory (over the operands, no longer read): AA and AB
    // rows of A, BB rows of B
    double* gAA = gsm;
    double* gAB = gsm + 128 * 33;
    double* gBB = gsm + 2 * 128 * 33;
#pragma unroll
    for (int c = 0; c < 32; c++) {
        if (rows_a) {
            gAA[q * 33 + c] = acc0[c];
            gAB[q * 33 + c] = acc1[c];
        } else {
            gBB[q * 33 + c] = acc0[c];
        }
    }
    __syncthreads();
    // G_cta: sum over digits i of the rows i * 32 + a of the right block
    for (int e = tid; e < R * R; e += TH_THREADS) {
        const int a = e / R, c = e % R;
        double g = 0.0;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            if (a < 32 && c < 32) g += gAA[(i * 32 + a) * 33 + c];
            else if (a < 32) g += gAB[(i * 32 + a) * 33 + (c - 32)];
            else if (c < 32) g += gAB[(i * 32 + c) * 33 + (a - 32)];
            else g += gBB[(i * 32 + a - 32) * 33 + (c - 32)];
        }
        partials[(size_t)blockIdx.x * R * R + e] = g;
    }
}

int gram_tc_halves_launch(float* U, uint64_t I, int R, const double* inv, uint16_t* bf16_out, double* partials,
                          int sm, int* d_err, cudaStream_t s, int* nparts, uint32_t spin_max, int no_commit)
{
    void (*fn)(float*, uint64_t, int, const double*, uint16_t*, uint64_t, double*, int*, uint32_t, int);
    if (bf16_out) fn = inv ? k_gram_tc_halves<true, true> : k_gram_tc_halves<false, true>;
    else fn = inv ? k_gram_tc_halves<true, false> : k_gram_tc_halves<false, false>;
    BLCO_CUDA(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TH_SMEM));
    // one CTA per SM: it holds the whole TMEM (three 128-column regions)
    const uint64_t sups = (I + TH_KS - 1) / TH_KS;
    const uint64_t maxc = std::min<uint64_t>((uint64_t)sm, (uint64_t)gram_tc_max_ctas(sm));
    const uint64_t sups_per = std::max<uint64_t>(1, (sups + maxc - 1) / maxc);
    const uint64_t rows_per = sups_per * TH_KS;
    const int grid = (int)std::max<uint64_t>(1, (I + rows_per - 1) / rows_per);
    fn<<<grid, TH_THREADS, TH_SMEM, s>>>(U, I, R, inv, bf16_out, rows_per, partials, d_err, spin_max, no_commit);
    BLCO_CHECK_LAUNCH("k_gram_tc_halves");
    *nparts = grid;
    return BLCO_OK;
}

} // namespace

int gram_tc_max_ctas(int sm) { return sm * 8; }

int gram_tc_launch(float* U, uint64_t I, int R, const double* inv, uint16_t* bf16_out, double* partials, int sm,
                   int* d_err, cudaStream_t s, int* nparts, uint32_t spin_max, int no_commit)
{
    if (R < 1 || R > 64) return fail(BLCO_ERR_UNSUPPORTED, "tensor-core Gram takes rank 1..64");
    if (reinterpret_cast<uintptr_t>(U) % 16)
        return fail(BLCO_ERR_UNSUPPORTED, "tensor-core Gram stages rows with 16-byte loads: U must be 16-byte aligned");
    if (spin_max == 0) spin_max = TG_SPIN_MAX;
    if (R <= 8) return gram_tc_dispatch<8>(U, I, R, inv, bf16_out, partials, sm, d_err, s, nparts, spin_max, no_commit);
    if (R <= 16)
        return gram_tc_dispatch<16>(U, I, R, inv, bf16_out, partials, sm, d_err, s, nparts, spin_max, no_commit);
    if (R <= 32)
        return gram_tc_dispatch<32>(U, I, R, inv, bf16_out, partials, sm, d_err, s, nparts, spin_max, no_commit);
    return gram_tc_halves_launch(U, I, R, inv, bf16_out, partials, sm, d_err, s, nparts, spin_max, no_commit);
}

} // namespace blco
