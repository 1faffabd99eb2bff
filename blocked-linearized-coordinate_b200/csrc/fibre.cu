// fibre.cu -- MTTKRP over compressed-fibre copies of the stream (kernel id 4).
//
//   out[i_t, :] += sum over nonzeros x of x * prod_{m != t} U_m[i_m, :]
//
// The reference's kernels (src/alto_dev.cu:31-1847) gather every other
// mode's factor row for every nonzero.  On B200 a random 128-byte row gather
// runs at ~134 G rows/s from a 2M-row Zipf-accessed factor (~200 G rows/s
// from L1), so at 200M nonzeros two gathers per nonzero cost more than the
// whole HBM budget of the mode.  A mode-t copy here is grouped by
// (row of t, index of the fibre mode f), f being the shortest other mode:
//
//   out[i_t] += sum_fibres U_f[i_f] (.) ( sum_{nonzeros of the fibre} x * prod_inner U_m[i_m] )
//
// so U_f's row is gathered once per fibre instead of once per nonzero.
// Fibres of one nonzero gain nothing from that and go to a second, "loose"
// stream that gathers every row per nonzero without fibre bookkeeping.
//
// Layout of a mode's copy (FibreCopy, all 32-bit indices, so every mode
// length must be below 2^31):
//   fibred stream  fw[m][q]  index of inner mode m (bit 31 of m = 0: the
//                            nonzero starts a fibre), fv[q] value;
//                  fib[k]    U_f row of fibre k (bit 31: the fibre starts a row);
//                  frows[r]  output row of the r-th row run;
//                  fctab     (fibre, row run) at every 256th position;
//   loose stream   lw[0][q]  U_f row (bit 31: the nonzero starts a row),
//                  lw[1+m][q] inner indices, lv[q] value, lrows, lctab.
// Arrays are padded to a multiple of 4 positions (plus one step), zeros.
//
// Kernel: a group of L lanes holds one R-wide row, 16 bytes per lane
// (L = R * element bytes / 16: 8 lanes for FP32 at R = 32, 16 for FP64).
// Work comes in tasks of 256 positions per lane group (32 / L groups per
// warp), fibred tasks first; warps take tasks from a counter in a strided
// order (consecutive takers land far apart in the stream, so concurrent
// warps share few output rows), or in stream order.  A group walks its 256
// positions four nonzeros per step, with all of a step's gathers issued
// before any product and the next step's index words loaded ahead.  The
// fibre sum s, the row sum and the fibre row c stay in registers; the next
// fibre's row is gathered one fibre ahead.  A row's sum goes to the output
// with atomics when the row run ends (tasks overlap rows only at their
// ends).  Partial sums in the mixed forms are FP32 over one step (at most
// four products) and are folded into FP64 registers after every step, so a
// heavy row's millions of terms are summed in FP64.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "internal.cuh"

namespace blco {
namespace {

constexpr uint32_t FB_FLAG = 0x80000000u;
constexpr uint32_t FB_IDX = 0x7fffffffu;
constexpr int FB_CHUNK = 256;    // chunk-table granularity (positions)
constexpr int FB_SUB = 256;      // positions a lane group walks per task (a multiple of FB_CHUNK)
constexpr int FB_THREADS = 256;
constexpr int FB_U = 4;          // nonzeros per lane-group step (their gathers are issued together)
// Bytes of factor row per lane: one 128-bit load.  (256-bit loads gather
// rows at the same rate on B200 but double the per-lane state: measured no
// faster for FP32 rows and slower for FP64 rows.)
constexpr int fb_vb(int) { return 16; }

// Element types of one numeric form: value, factor, partial sum, and the
// columns one lane holds (16 bytes of factor row).
struct FibF64 {
    typedef double TV;
    typedef double TS;
    static constexpr int V = 2; // columns per 16 bytes
    static constexpr int VB = 16;
};
struct FibF32 {
    typedef float TV;
    typedef float TS;
    static constexpr int V = 4;
    static constexpr int VB = 16;
};
struct FibBF16 {
    typedef float TV;
    typedef float TS;
    static constexpr int V = 8;
    static constexpr int VB = 16;
};

struct FibParams {
    // fibred stream
    const uint32_t* fw[3];
    const void* fv;
    const uint32_t* fib;
    const uint32_t* frows;
    const uint32_t* fctab;
    uint64_t nf;
    // loose stream
    const uint32_t* lw[4];
    const void* lv;
    const uint32_t* lrows;
    const uint32_t* lctab;
    uint64_t nl;
    // factors: the fibre mode's and the inner modes' (in FibreCopy::inner order)
    const void* ff;
    const void* fi[3];
    void* out;
    // work: tasks of (32 / L) * FB_SUB positions, one per warp, fibred ones
    // first, taken from *counter in the order k -> k * stride mod ntasks
    // (stride coprime to ntasks)
    uint32_t* counter;
    uint64_t ntask_f, ntasks, stride;
};

// A numeric form with VB bytes of factor row per lane (16: one 128-bit
// load, 32: one 256-bit load); V columns per lane.
template <class B, int VBYTES>
struct Lanes : B {
    static constexpr int VB = VBYTES;
    static constexpr int V = B::V * VBYTES / 16;
};

// One 16-byte piece of a factor row into E partial-type columns.
template <class T, int E>
__device__ __forceinline__ void unpack16(const uint4 r, typename T::TS* o)
{
    if constexpr (E == 2) {
        o[0] = __hiloint2double((int)r.y, (int)r.x);
        o[1] = __hiloint2double((int)r.w, (int)r.z);
    } else if constexpr (E == 4) {
        o[0] = __uint_as_float(r.x);
        o[1] = __uint_as_float(r.y);
        o[2] = __uint_as_float(r.z);
        o[3] = __uint_as_float(r.w);
    } else {
        const uint32_t w[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            o[2 * k] = __uint_as_float(w[k] << 16);
            o[2 * k + 1] = __uint_as_float(w[k] & 0xffff0000u);
        }
    }
}

// This lane's VB bytes of factor row `row` (rows of L * VB bytes).
template <class T>
__device__ __forceinline__ void gather(const void* F, uint32_t row, int lanes, int sub, typename T::TS (&o)[T::V])
{
    constexpr int E = T::V * 16 / T::VB; // columns per 16 bytes
    const char* ptr = reinterpret_cast<const char*>(F) + ((size_t)row * lanes + sub) * T::VB;
    if constexpr (T::VB == 16) {
        unpack16<T, E>(__ldg(reinterpret_cast<const uint4*>(ptr)), o);
    } else {
        uint4 a, b;
        asm("ld.global.nc.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
            : "=r"(a.x), "=r"(a.y), "=r"(a.z), "=r"(a.w), "=r"(b.x), "=r"(b.y), "=r"(b.z), "=r"(b.w)
            : "l"(ptr));
        unpack16<T, E>(a, o);
        unpack16<T, E>(b, o + E);
    }
}

// Values of positions q..q+U-1 (q a multiple of U).
template <int U, typename TV>
__device__ __forceinline__ void load_vals(const void* v, uint64_t q, TV (&x)[U])
{
    if constexpr (sizeof(TV) == 8) {
#pragma unroll
        for (int k = 0; k < U / 2; k++) {
            const double2 a = __ldg(reinterpret_cast<const double2*>(v) + (q >> 1) + k);
            x[2 * k] = a.x, x[2 * k + 1] = a.y;
        }
    } else {
#pragma unroll
        for (int k = 0; k < U / 4; k++) {
            const float4 a = __ldg(reinterpret_cast<const float4*>(v) + (q >> 2) + k);
            x[4 * k] = a.x, x[4 * k + 1] = a.y, x[4 * k + 2] = a.z, x[4 * k + 3] = a.w;
        }
    }
}

// Adds one lane's columns of a finished FP64 row sum to the output.
template <int V, typename TO>
__device__ __forceinline__ void flush_row(TO* o, const double (&a)[V])
{
    if constexpr (sizeof(TO) == 4 && V % 4 == 0) {
#pragma unroll
        for (int j = 0; j < V; j += 4)
            atomicAdd(reinterpret_cast<float4*>(o + j),
                      make_float4((float)a[j], (float)a[j + 1], (float)a[j + 2], (float)a[j + 3]));
    } else {
#pragma unroll
        for (int j = 0; j < V; j++) atomicAdd(o + j, (TO)a[j]);
    }
}

// This lane's columns of row `row` of a factor; b is the factor's address
// plus this lane's byte offset, ROWB the bytes of a row.
template <class T, int ROWB>
__device__ __forceinline__ void gather_at(const char* b, uint32_t row, typename T::TS (&o)[T::V])
{
    constexpr int E = T::V * 16 / T::VB; // columns per 16 bytes
    const char* ptr = b + (size_t)row * ROWB;
    if constexpr (T::VB == 16) {
        unpack16<T, E>(__ldg(reinterpret_cast<const uint4*>(ptr)), o);
    } else {
        uint4 u, w;
        asm("ld.global.nc.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
            : "=r"(u.x), "=r"(u.y), "=r"(u.z), "=r"(u.w), "=r"(w.x), "=r"(w.y), "=r"(w.z), "=r"(w.w)
            : "l"(ptr));
        unpack16<T, E>(u, o);
        unpack16<T, E>(w, o + E);
    }
}

// Index words of one FB_U-position step.
template <int NW>
struct StepIn {
    uint32_t w[NW][FB_U];
};

template <int NW>
__device__ __forceinline__ void load_words(StepIn<NW>& in, const uint32_t* const (&wp)[NW], uint32_t i)
{
#pragma unroll
    for (int m = 0; m < NW; m++)
#pragma unroll
        for (int k = 0; k < FB_U / 4; k++) {
            const uint4 u = __ldg(reinterpret_cast<const uint4*>(wp[m] + (size_t)i * FB_U) + k);
            in.w[m][4 * k] = u.x, in.w[m][4 * k + 1] = u.y, in.w[m][4 * k + 2] = u.z, in.w[m][4 * k + 3] = u.w;
        }
}

// One lane's walk over a range of the fibred stream.  s: the current
// fibre's sum over this step's nonzeros; c / cn: the current and the next
// fibre's U_f row; a: the FP64 row sum.  In the mixed forms s is FP32 over at
// most the FB_U nonzeros of a step and is folded into a after every step
// (fibres longer than a step contribute one s * c per step).
template <int NM, int L, class T, typename TO>
struct FibredWalk {
    typedef typename T::TS TS;
    typedef typename T::TV TV;
    static constexpr int V = T::V, R = L * V, NI = NM - 2, ROWB = L * T::VB;
    const FibParams& p;
    const char* fb;
    const char* ib[NI];
    TO* out;
    const uint32_t* wp[NI];
    const TV* vp;
    uint32_t fi, ri, fwn, fwnn, row, rown;
    TS s[V], c[V], cn[V];
    double a[V];

    __device__ __forceinline__ FibredWalk(const FibParams& p_, int sub, uint64_t first) : p(p_)
    {
        fb = reinterpret_cast<const char*>(p.ff) + sub * T::VB;
#pragma unroll
        for (int m = 0; m < NI; m++) {
            ib[m] = reinterpret_cast<const char*>(p.fi[m]) + sub * T::VB;
            wp[m] = p.fw[m] + first;
        }
        out = reinterpret_cast<TO*>(p.out) + sub * V;
        vp = reinterpret_cast<const TV*>(p.fv) + first;
        fi = p.fctab[2 * (first / FB_CHUNK)];
        ri = p.fctab[2 * (first / FB_CHUNK) + 1];
        fwn = p.fib[fi + 1];
        fwnn = p.fib[fi + 2];
        row = p.frows[ri];
        rown = p.frows[ri + 1];
        gather_at<T, ROWB>(fb, p.fib[fi] & FB_IDX, c);
        gather_at<T, ROWB>(fb, fwn & FB_IDX, cn);
#pragma unroll
        for (int v = 0; v < V; v++) s[v] = TS(0), a[v] = 0.0;
    }

    __device__ __forceinline__ void flush()
    {
        flush_row<V, TO>(out + (size_t)row * R, a);
#pragma unroll
        for (int v = 0; v < V; v++) a[v] = 0.0;
    }

    // s * c joins the row sum
    __device__ __forceinline__ void take()
    {
#pragma unroll
        for (int v = 0; v < V; v++) {
            if constexpr (sizeof(TS) == 4) a[v] += (double)(s[v] * c[v]);
            else a[v] = fma(s[v], c[v], a[v]);
            s[v] = TS(0);
        }
    }

    // Fibre fi ends; the next fibre's row is already in cn, the one after it
    // is gathered now.
    __device__ __forceinline__ void close_fibre()
    {
        take();
#pragma unroll
        for (int v = 0; v < V; v++) c[v] = cn[v];
        fi++;
        const uint32_t fw = fwn;
        fwn = fwnn;
        fwnn = p.fib[fi + 2];
        gather_at<T, ROWB>(fb, fwn & FB_IDX, cn);
        if (fw & FB_FLAG) { // the new fibre starts a new row run
            flush();
            row = rown;
            ri++;
            rown = p.frows[ri + 1];
        }
    }

    typedef StepIn<NI> In;

    __device__ __forceinline__ void load(In& in, uint32_t i) const { load_words<NI>(in, wp, i); }

    // Step i (positions FB_U*i.. of the range, whose words are in `in`;
    // values are loaded here, beside the gathers).  With TAIL, positions at
    // or past n are padding and take no part.
    template <bool TAIL>
    __device__ __forceinline__ void process(In& in, uint32_t i, uint32_t n)
    {
        if (i == 0) in.w[0][0] &= FB_IDX; // a range's first nonzero continues the fibre it starts in
        TV x[FB_U];
        load_vals<FB_U, TV>(vp, (uint64_t)FB_U * i, x);
        TS b[FB_U][V];
#pragma unroll
        for (int q = 0; q < FB_U; q++) {
            if (!TAIL || FB_U * i + q < n) {
                gather_at<T, ROWB>(ib[0], in.w[0][q] & FB_IDX, b[q]);
            } else {
                x[q] = TV(0);
                in.w[0][q] = 0;
#pragma unroll
                for (int v = 0; v < V; v++) b[q][v] = TS(0);
            }
        }
#pragma unroll
        for (int m = 1; m < NI; m++) {
            TS e[FB_U][V];
#pragma unroll
            for (int q = 0; q < FB_U; q++) {
                if (!TAIL || FB_U * i + q < n) gather_at<T, ROWB>(ib[m], in.w[m][q], e[q]);
                else {
#pragma unroll
                    for (int v = 0; v < V; v++) e[q][v] = TS(0);
                }
            }
#pragma unroll
            for (int q = 0; q < FB_U; q++)
#pragma unroll
                for (int v = 0; v < V; v++) b[q][v] *= e[q][v];
        }
        uint32_t any = 0;
#pragma unroll
        for (int q = 0; q < FB_U; q++) any |= in.w[0][q];
        any &= FB_FLAG;
        if (!any) {
#pragma unroll
            for (int q = 0; q < FB_U; q++)
#pragma unroll
                for (int v = 0; v < V; v++) s[v] = fma((TS)x[q], b[q][v], s[v]);
        } else {
#pragma unroll
            for (int q = 0; q < FB_U; q++) {
                if (in.w[0][q] & FB_FLAG) close_fibre();
#pragma unroll
                for (int v = 0; v < V; v++) s[v] = fma((TS)x[q], b[q][v], s[v]);
            }
        }
        if constexpr (sizeof(TS) == 4) take();
    }

    __device__ __forceinline__ void finish()
    {
        take();
        flush();
    }
};

// One lane's walk over a range of the loose stream: every nonzero is a
// fibre of its own, so x * U_f row * inner rows goes straight into the row
// sum (FP32 over a step in the mixed forms, then FP64).
template <int NM, int L, class T, typename TO>
struct LooseWalk {
    typedef typename T::TS TS;
    typedef typename T::TV TV;
    static constexpr int V = T::V, R = L * V, NI = NM - 2, ROWB = L * T::VB;
    const FibParams& p;
    const char* fb;
    const char* ib[NI];
    TO* out;
    const uint32_t* wp[NI + 1];
    const TV* vp;
    uint32_t ri, row, rown;
    TS acc[V];
    double a[V];

    __device__ __forceinline__ LooseWalk(const FibParams& p_, int sub, uint64_t first) : p(p_)
    {
        fb = reinterpret_cast<const char*>(p.ff) + sub * T::VB;
#pragma unroll
        for (int m = 0; m < NI; m++) ib[m] = reinterpret_cast<const char*>(p.fi[m]) + sub * T::VB;
#pragma unroll
        for (int m = 0; m <= NI; m++) wp[m] = p.lw[m] + first;
        out = reinterpret_cast<TO*>(p.out) + sub * V;
        vp = reinterpret_cast<const TV*>(p.lv) + first;
        ri = p.lctab[first / FB_CHUNK];
        row = p.lrows[ri];
        rown = p.lrows[ri + 1];
#pragma unroll
        for (int v = 0; v < V; v++) acc[v] = TS(0), a[v] = 0.0;
    }

    __device__ __forceinline__ void fold()
    {
#pragma unroll
        for (int v = 0; v < V; v++) {
            a[v] += (double)acc[v];
            acc[v] = TS(0);
        }
    }

    __device__ __forceinline__ void flush()
    {
        fold();
        flush_row<V, TO>(out + (size_t)row * R, a);
#pragma unroll
        for (int v = 0; v < V; v++) a[v] = 0.0;
    }

    typedef StepIn<NI + 1> In;

    __device__ __forceinline__ void load(In& in, uint32_t i) const { load_words<NI + 1>(in, wp, i); }

    template <bool TAIL>
    __device__ __forceinline__ void process(In& in, uint32_t i, uint32_t n)
    {
        if (i == 0) in.w[0][0] &= FB_IDX;
        TV x[FB_U];
        load_vals<FB_U, TV>(vp, (uint64_t)FB_U * i, x);
        TS b[FB_U][V];
#pragma unroll
        for (int q = 0; q < FB_U; q++) {
            if (!TAIL || FB_U * i + q < n) {
                gather_at<T, ROWB>(fb, in.w[0][q] & FB_IDX, b[q]);
            } else {
                x[q] = TV(0);
                in.w[0][q] = 0;
#pragma unroll
                for (int v = 0; v < V; v++) b[q][v] = TS(0);
            }
        }
#pragma unroll
        for (int m = 0; m < NI; m++) {
            TS e[FB_U][V];
#pragma unroll
            for (int q = 0; q < FB_U; q++) {
                if (!TAIL || FB_U * i + q < n) gather_at<T, ROWB>(ib[m], in.w[m + 1][q], e[q]);
                else {
#pragma unroll
                    for (int v = 0; v < V; v++) e[q][v] = TS(0);
                }
            }
#pragma unroll
            for (int q = 0; q < FB_U; q++)
#pragma unroll
                for (int v = 0; v < V; v++) b[q][v] *= e[q][v];
        }
        uint32_t any = 0;
#pragma unroll
        for (int q = 0; q < FB_U; q++) any |= in.w[0][q];
        any &= FB_FLAG;
        if (!any) {
#pragma unroll
            for (int q = 0; q < FB_U; q++)
#pragma unroll
                for (int v = 0; v < V; v++) acc[v] = fma((TS)x[q], b[q][v], acc[v]);
        } else {
#pragma unroll
            for (int q = 0; q < FB_U; q++) {
                if (in.w[0][q] & FB_FLAG) { // a new row run starts here
                    flush();
                    row = rown;
                    ri++;
                    rown = p.lrows[ri + 1];
                }
#pragma unroll
                for (int v = 0; v < V; v++) acc[v] = fma((TS)x[q], b[q][v], acc[v]);
            }
        }
        if constexpr (sizeof(TS) == 4) fold();
    }

    __device__ __forceinline__ void finish() { flush(); }
};

// Walks the n positions of a range FB_U per step; the next step's index
// words are loaded while this step's rows are gathered, so a step waits on
// one memory latency (the gathers), not two.  The last step may hold padding
// (arrays are padded by at least one step).
template <class W>
__device__ __forceinline__ void walk(W& wk, uint32_t n)
{
    typename W::In cur, nxt;
    wk.load(cur, 0);
    const uint32_t full = n / FB_U;
    uint32_t i = 0;
    for (; i < full; i++) {
        if (FB_U * (i + 1) < n) wk.load(nxt, i + 1);
        wk.template process<false>(cur, i, n);
        cur = nxt;
    }
    if (FB_U * i < n) wk.template process<true>(cur, i, n);
    wk.finish();
}

// Resident CTAs per SM the register budget is sized for.  The kernel is
// bound by the gathers in flight, which the register file limits: for
// 3-mode tensors with up to 4 columns per lane, four CTAs (32 warps, 64
// registers) measured fastest (2.85 ms per FP32 mode of the 200M-nonzero
// workload, against 3.06 ms with three CTAs and 4.1 ms with two, whatever
// the extra gathers a wider step puts in flight); larger states take two.
template <int NM, class T>
constexpr int fib_min_blocks() { return (NM == 3 && T::V <= 4) ? 4 : 2; }

template <int NM, int L, class T, typename TO>
__global__ void __launch_bounds__(FB_THREADS, fib_min_blocks<NM, T>()) k_mttkrp_fib(const FibParams p)
{
    constexpr int GPW = 32 / L; // lane groups per warp
    const int lane = threadIdx.x & 31, grp = lane / L, sub = lane % L;
    // A warp takes one task of GPW * FB_SUB positions; group g walks the g-th
    // FB_SUB of it, so the groups of a warp run the same loop in step and
    // diverge only where a fibre or row run ends.
    for (;;) {
        uint32_t k = 0;
        if (lane == 0) k = atomicAdd(p.counter, 1u);
        k = __shfl_sync(0xffffffffu, k, 0);
        if (k >= p.ntasks) break;
        const uint64_t task = (uint64_t)k * p.stride % p.ntasks;
        if (task < p.ntask_f) {
            const uint64_t first = (task * GPW + grp) * FB_SUB;
            if (first < p.nf) {
                FibredWalk<NM, L, T, TO> wk(p, sub, first);
                walk(wk, (uint32_t)min((uint64_t)FB_SUB, p.nf - first));
            }
        } else {
            const uint64_t first = ((task - p.ntask_f) * GPW + grp) * FB_SUB;
            if (first < p.nl) {
                LooseWalk<NM, L, T, TO> wk(p, sub, first);
                walk(wk, (uint32_t)min((uint64_t)FB_SUB, p.nl - first));
            }
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------- building --

// key = (row of mode t) << bits_f | (index of mode f); idx = stream position.
__global__ void k_fib_keys(const uint64_t* __restrict__ coords, uint64_t n, int pos_t, uint64_t mask_t, int pos_f,
                           uint64_t mask_f, int bits_f, uint64_t* __restrict__ keys, uint64_t* __restrict__ idx)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = coords[i];
        keys[i] = (((c >> pos_t) & mask_t) << bits_f) | ((c >> pos_f) & mask_f);
        idx[i] = i;
    }
}

// flag[p] = 1 when sorted position p belongs to a fibre of two or more
// nonzeros; flag[n] = 0 (the exclusive scan then ends with the total).
__global__ void k_fib_multi(const uint64_t* __restrict__ k, uint64_t n, uint32_t* __restrict__ flag)
{
    for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p <= n; p += (uint64_t)gridDim.x * blockDim.x) {
        if (p == n) {
            flag[p] = 0;
            continue;
        }
        const bool first = p == 0 || k[p] != k[p - 1];
        const bool last = p + 1 == n || k[p + 1] != k[p];
        flag[p] = (first && last) ? 0u : 1u;
    }
}

// Stable split: fibred positions to [0, nf), loose ones to [nf, n).
__global__ void k_fib_split(const uint64_t* __restrict__ k, const uint64_t* __restrict__ idx, uint64_t n,
                            const uint32_t* __restrict__ excl, uint64_t nf, uint64_t* __restrict__ ko,
                            uint64_t* __restrict__ io)
{
    for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < n; p += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t e = excl[p];
        const bool multi = excl[p + 1] != e;
        const uint64_t d = multi ? e : nf + (p - e);
        ko[d] = k[p];
        io[d] = idx[p];
    }
}

// Fibre-start and row-start flags of a (sorted) key run; flag[n] = 0.
__global__ void k_fib_starts(const uint64_t* __restrict__ k, uint64_t n, int bits_f, uint32_t* __restrict__ fs,
                             uint32_t* __restrict__ rs)
{
    for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q <= n; q += (uint64_t)gridDim.x * blockDim.x) {
        if (q == n) {
            if (fs) fs[q] = 0;
            rs[q] = 0;
            continue;
        }
        if (fs) fs[q] = (q == 0 || k[q] != k[q - 1]) ? 1u : 0u;
        rs[q] = (q == 0 || (k[q] >> bits_f) != (k[q - 1] >> bits_f)) ? 1u : 0u;
    }
}

struct FibWrite {
    const uint64_t* coords;
    const double* vals;
    const uint64_t* k;   // sorted keys of this stream
    const uint64_t* idx; // their stream positions
    const uint32_t* fsx; // exclusive scan of fibre starts (fibred) / null (loose)
    const uint32_t* rsx; // exclusive scan of row starts
    uint64_t n;
    int bits_f;
    uint64_t mask_f;
    int ninner;
    int ipos[3];
    uint64_t imask[3];
    uint32_t* w[4];
    double* v;
    uint32_t* fib;
    uint32_t* rows;
    uint32_t* ctab;
};

__global__ void k_fib_write(const FibWrite f)
{
    for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < f.n; q += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t key = f.k[q];
        const uint64_t i = f.idx[q];
        const uint64_t c = f.coords[i];
        const uint32_t rstart = f.rsx[q + 1] != f.rsx[q];
        const uint32_t ridx = f.rsx[q];
        const uint32_t fidx = (uint32_t)(key & f.mask_f);
        const uint32_t row = (uint32_t)(key >> f.bits_f);
        f.v[q] = f.vals[i];
        if (f.fsx) { // fibred stream
            const uint32_t fstart = f.fsx[q + 1] != f.fsx[q];
            for (int m = 0; m < f.ninner; m++) {
                uint32_t w = (uint32_t)((c >> f.ipos[m]) & f.imask[m]);
                if (m == 0 && fstart) w |= FB_FLAG;
                f.w[m][q] = w;
            }
            if (fstart) f.fib[f.fsx[q]] = fidx | (rstart ? FB_FLAG : 0u);
            if (q % FB_CHUNK == 0) {
                f.ctab[2 * (q / FB_CHUNK)] = f.fsx[q] + fstart - 1;
                f.ctab[2 * (q / FB_CHUNK) + 1] = ridx + rstart - 1;
            }
        } else { // loose stream
            f.w[0][q] = fidx | (rstart ? FB_FLAG : 0u);
            for (int m = 0; m < f.ninner; m++) f.w[m + 1][q] = (uint32_t)((c >> f.ipos[m]) & f.imask[m]);
            if (q % FB_CHUNK == 0) f.ctab[q / FB_CHUNK] = ridx + rstart - 1;
        }
        if (rstart) f.rows[ridx] = row;
    }
}

__global__ void k_fib_to_f32(const double* __restrict__ in, float* __restrict__ out, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

// Stream arrays hold a multiple of 8 positions plus one 8-position step of
// zero padding, so a step may load whole vectors past the end.
inline uint64_t pad4(uint64_t n) { return ((n + 7) & ~7ull) + 8; }

// A stride coprime to n near n * 0.618: consecutive task numbers land far
// apart in the streams, so lane groups working at the same time rarely share
// an output row (whose flushes would contend) and the order still visits
// every task once.
uint64_t task_stride(uint64_t n)
{
    if (n <= 2) return 1;
    uint64_t st = std::max<uint64_t>(1, (uint64_t)(n * 0.6180339887));
    auto gcd = [](uint64_t a, uint64_t b) { while (b) { uint64_t t = a % b; a = b; b = t; } return a; };
    while (gcd(st, n) != 1) st++;
    return st;
}

int elem_bytes(int dtype) { return dtype == BLCO_DTYPE_F64 ? 8 : dtype == BLCO_DTYPE_F32 ? 4 : 2; }

typedef void (*FibFn)(FibParams);

template <int NM, class B, typename TO>
FibFn pick_fib_nm(int L)
{
    typedef Lanes<B, B::VB> T;
    switch (L) {
    case 1: return k_mttkrp_fib<NM, 1, T, TO>;
    case 2: return k_mttkrp_fib<NM, 2, T, TO>;
    case 4: return k_mttkrp_fib<NM, 4, T, TO>;
    case 8: return k_mttkrp_fib<NM, 8, T, TO>;
    case 16: return k_mttkrp_fib<NM, 16, T, TO>;
    case 32: return k_mttkrp_fib<NM, 32, T, TO>;
    default: return nullptr;
    }
}

template <class T, typename TO>
FibFn pick_fib(int nm, int L)
{
    switch (nm) {
    case 3: return pick_fib_nm<3, T, TO>(L);
    case 4: return pick_fib_nm<4, T, TO>(L);
    case 5: return pick_fib_nm<5, T, TO>(L);
    default: return nullptr;
    }
}

} // namespace

bool fibre_eligible(const blco_tensor* t, int mode)
{
    const Layout& L = t->layout;
    if (!t->resident || L.wide || L.nmodes < 3 || t->nnz == 0 || t->nnz >= (1ull << 32)) return false;
    if (mode < 0 || mode >= L.nmodes) return false;
    for (int m = 0; m < L.nmodes; m++)
        if (L.dims[m] >= (1ull << 31)) return false;
    return true;
}

int fibre_lanes(int rank, int dtype)
{
    const int bytes = rank * elem_bytes(dtype), vb = fb_vb(dtype);
    if (bytes % vb) return 0;
    const int L = bytes / vb;
    return (L == 1 || L == 2 || L == 4 || L == 8 || L == 16 || L == 32) ? L : 0;
}

void fibre_free(FibreCopy& f)
{
    for (int m = 0; m < 3; m++) cudaFree(f.d_fw[m]);
    for (int m = 0; m < 4; m++) cudaFree(f.d_lw[m]);
    cudaFree(f.d_fv);
    cudaFree(f.d_fv32);
    cudaFree(f.d_fib);
    cudaFree(f.d_frows);
    cudaFree(f.d_fctab);
    cudaFree(f.d_lv);
    cudaFree(f.d_lv32);
    cudaFree(f.d_lrows);
    cudaFree(f.d_lctab);
    cudaFree(f.d_counter);
    f = FibreCopy();
}

void fib_scratch_free(FibScratch& sc)
{
    cudaFree(sc.k0);
    cudaFree(sc.k1);
    cudaFree(sc.i0);
    cudaFree(sc.i1);
    cudaFree(sc.sa);
    cudaFree(sc.sb);
    cudaFree(sc.sums);
    sc = FibScratch();
}

int fib_scratch_reserve(FibScratch& sc, uint64_t n)
{
    if (sc.k0 && sc.cap >= n) return BLCO_OK;
    fib_scratch_free(sc);
    cudaError_t e = cudaMalloc(&sc.k0, n * 8);
    if (e == cudaSuccess) e = cudaMalloc(&sc.k1, n * 8);
    if (e == cudaSuccess) e = cudaMalloc(&sc.i0, n * 8);
    if (e == cudaSuccess) e = cudaMalloc(&sc.i1, n * 8);
    if (e == cudaSuccess) e = cudaMalloc(&sc.sa, (n + 1) * 4);
    if (e == cudaSuccess) e = cudaMalloc(&sc.sb, (n + 1) * 4);
    if (e == cudaSuccess) e = cudaMalloc(&sc.sums, ((n + 1) / 4096 + 2) * 4);
    if (e != cudaSuccess) {
        fib_scratch_free(sc);
        return cuda_fail(e, "fibre-copy scratch", __FILE__, __LINE__);
    }
    sc.cap = n;
    return BLCO_OK;
}

int build_fibre_copy(blco_tensor* t, int mode, cudaStream_t s, FibScratch* sc)
{
    FibreCopy& fc = t->fib[mode];
    if (fc.built) return BLCO_OK;
    if (!fibre_eligible(t, mode)) return fail(BLCO_ERR_UNSUPPORTED, "fibre copies need a resident tensor of 3-5 modes, "
                                                                     "64-bit keys, modes below 2^31 and nnz below 2^32");
    const Layout& L = t->layout;
    const int N = L.nmodes;
    const uint64_t n = t->nnz;
    DeviceInfo di;
    BLCO_TRY(device_info(t->device, &di));
    FibreCopy f;
    // fibre mode: the shortest other mode (most repeated indices), ties by index
    int fm = -1;
    for (int m = 0; m < N; m++)
        if (m != mode && (fm < 0 || L.dims[m] < L.dims[fm])) fm = m;
    f.fmode = fm;
    for (int m = 0; m < N; m++)
        if (m != mode && m != fm) f.inner[f.ninner++] = m;
    const int bits_t = __builtin_popcountll(L.mode_masks[mode]);
    const int bits_f = __builtin_popcountll(L.mode_masks[fm]);

    FibScratch own;
    FibScratch& S = sc ? *sc : own;
    int st = BLCO_OK;
    auto cleanup = [&]() {
        if (!sc) fib_scratch_free(own);
    };
#define FB_CUDA(call)                                                          \
    do {                                                                       \
        cudaError_t _e = (call);                                               \
        if (_e != cudaSuccess) {                                               \
            st = cuda_fail(_e, #call, __FILE__, __LINE__);                     \
            cleanup();                                                         \
            fibre_free(f);                                                     \
            return st;                                                         \
        }                                                                      \
    } while (0)
#define FB_TRY(call)                                                           \
    do {                                                                       \
        if ((st = (call)) != BLCO_OK) {                                        \
            cleanup();                                                         \
            fibre_free(f);                                                     \
            return st;                                                         \
        }                                                                      \
    } while (0)
    FB_TRY(fib_scratch_reserve(S, n));
    uint64_t *k0 = S.k0, *k1 = S.k1, *i0 = S.i0, *i1 = S.i1;
    uint32_t *sa = S.sa, *sb = S.sb, *sums = S.sums;
    const int grid = (int)std::min<uint64_t>((n + 255) / 256, (uint64_t)di.sm_count * 16);
    k_fib_keys<<<grid, 256, 0, s>>>(t->d_coords, n, L.mode_pos[mode], L.mode_masks[mode], L.mode_pos[fm],
                                    L.mode_masks[fm], bits_f, k0, i0);
    count_launch();
    bool alt = false;
    FB_TRY(radix_sort_pairs_u64(k0, i0, k1, i1, n, bits_t + bits_f, s, &alt));
    uint64_t *ks = alt ? k1 : k0, *is = alt ? i1 : i0; // sorted
    uint64_t *kt = alt ? k0 : k1, *it = alt ? i0 : i1; // free pair
    k_fib_multi<<<grid, 256, 0, s>>>(ks, n, sa);
    count_launch();
    FB_TRY(scan_u32_ext(sa, n + 1, sums, s));
    uint32_t nf32 = 0;
    FB_CUDA(cudaMemcpyAsync(&nf32, sa + n, 4, cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaStreamSynchronize(s));
    const uint64_t nf = nf32, nl = n - nf;
    k_fib_split<<<grid, 256, 0, s>>>(ks, is, n, sa, nf, kt, it);
    count_launch();
    f.nf = nf;
    f.nl = nl;

    // fibred stream
    uint32_t tot[3] = {0, 0, 0};
    if (nf) {
        k_fib_starts<<<grid, 256, 0, s>>>(kt, nf, bits_f, sa, sb);
        count_launch();
        FB_TRY(scan_u32_ext(sa, nf + 1, sums, s));
        FB_TRY(scan_u32_ext(sb, nf + 1, sums, s));
        FB_CUDA(cudaMemcpyAsync(&tot[0], sa + nf, 4, cudaMemcpyDeviceToHost, s));
        FB_CUDA(cudaMemcpyAsync(&tot[1], sb + nf, 4, cudaMemcpyDeviceToHost, s));
        FB_CUDA(cudaStreamSynchronize(s));
        f.nfib = tot[0];
        f.nrows_f = tot[1];
        const uint64_t np = pad4(nf);
        for (int m = 0; m < f.ninner; m++) {
            FB_CUDA(cudaMalloc(&f.d_fw[m], np * 4));
            FB_CUDA(cudaMemsetAsync(f.d_fw[m] + nf, 0, (np - nf) * 4, s)); // k_fib_write fills [0, nf)
        }
        FB_CUDA(cudaMalloc(&f.d_fv, np * 8));
        FB_CUDA(cudaMemsetAsync(f.d_fv + nf, 0, (np - nf) * 8, s));
        FB_CUDA(cudaMalloc(&f.d_fib, (f.nfib + 3) * 4));
        FB_CUDA(cudaMemsetAsync(f.d_fib, 0, (f.nfib + 3) * 4, s));
        FB_CUDA(cudaMalloc(&f.d_frows, (f.nrows_f + 2) * 4));
        FB_CUDA(cudaMemsetAsync(f.d_frows, 0, (f.nrows_f + 2) * 4, s));
        FB_CUDA(cudaMalloc(&f.d_fctab, (2 * ((nf + FB_CHUNK - 1) / FB_CHUNK) + 2) * 4));
        FibWrite w;
        memset(&w, 0, sizeof(w));
        w.coords = t->d_coords;
        w.vals = t->d_values;
        w.k = kt;
        w.idx = it;
        w.fsx = sa;
        w.rsx = sb;
        w.n = nf;
        w.bits_f = bits_f;
        w.mask_f = L.mode_masks[fm];
        w.ninner = f.ninner;
        for (int m = 0; m < f.ninner; m++) {
            w.ipos[m] = L.mode_pos[f.inner[m]];
            w.imask[m] = L.mode_masks[f.inner[m]];
            w.w[m] = f.d_fw[m];
        }
        w.v = f.d_fv;
        w.fib = f.d_fib;
        w.rows = f.d_frows;
        w.ctab = f.d_fctab;
        k_fib_write<<<grid, 256, 0, s>>>(w);
        count_launch();
    }
    // loose stream
    if (nl) {
        k_fib_starts<<<grid, 256, 0, s>>>(kt + nf, nl, bits_f, nullptr, sb);
        count_launch();
        FB_TRY(scan_u32_ext(sb, nl + 1, sums, s));
        FB_CUDA(cudaMemcpyAsync(&tot[2], sb + nl, 4, cudaMemcpyDeviceToHost, s));
        FB_CUDA(cudaStreamSynchronize(s));
        f.nrows_l = tot[2];
        const uint64_t np = pad4(nl);
        for (int m = 0; m <= f.ninner; m++) {
            FB_CUDA(cudaMalloc(&f.d_lw[m], np * 4));
            FB_CUDA(cudaMemsetAsync(f.d_lw[m] + nl, 0, (np - nl) * 4, s)); // k_fib_write fills [0, nl)
        }
        FB_CUDA(cudaMalloc(&f.d_lv, np * 8));
        FB_CUDA(cudaMemsetAsync(f.d_lv + nl, 0, (np - nl) * 8, s));
        FB_CUDA(cudaMalloc(&f.d_lrows, (f.nrows_l + 2) * 4));
        FB_CUDA(cudaMemsetAsync(f.d_lrows, 0, (f.nrows_l + 2) * 4, s));
        FB_CUDA(cudaMalloc(&f.d_lctab, ((nl + FB_CHUNK - 1) / FB_CHUNK + 1) * 4));
        FibWrite w;
        memset(&w, 0, sizeof(w));
        w.coords = t->d_coords;
        w.vals = t->d_values;
        w.k = kt + nf;
        w.idx = it + nf;
        w.fsx = nullptr;
        w.rsx = sb;
        w.n = nl;
        w.bits_f = bits_f;
        w.mask_f = L.mode_masks[fm];
        w.ninner = f.ninner;
        for (int m = 0; m < f.ninner; m++) {
            w.ipos[m] = L.mode_pos[f.inner[m]];
            w.imask[m] = L.mode_masks[f.inner[m]];
        }
        for (int m = 0; m <= f.ninner; m++) w.w[m] = f.d_lw[m];
        w.v = f.d_lv;
        w.rows = f.d_lrows;
        w.ctab = f.d_lctab;
        k_fib_write<<<grid, 256, 0, s>>>(w);
        count_launch();
    }
    FB_CUDA(cudaMalloc(&f.d_counter, sizeof(uint32_t)));
    FB_CUDA(cudaGetLastError());
    FB_CUDA(cudaStreamSynchronize(s));
    cleanup();
#undef FB_CUDA
#undef FB_TRY
    f.built = true;
    fc = f;
    return BLCO_OK;
}

int fibre_values_f32(blco_tensor* t, int mode, cudaStream_t s)
{
    FibreCopy& f = t->fib[mode];
    if (f.nf && !f.d_fv32) {
        const uint64_t np = pad4(f.nf);
        BLCO_CUDA(cudaMalloc(&f.d_fv32, np * 4));
        k_fib_to_f32<<<1024, 256, 0, s>>>(f.d_fv, f.d_fv32, np);
        BLCO_CHECK_LAUNCH("k_fib_to_f32");
    }
    if (f.nl && !f.d_lv32) {
        const uint64_t np = pad4(f.nl);
        BLCO_CUDA(cudaMalloc(&f.d_lv32, np * 4));
        k_fib_to_f32<<<1024, 256, 0, s>>>(f.d_lv, f.d_lv32, np);
        BLCO_CHECK_LAUNCH("k_fib_to_f32");
    }
    return BLCO_OK;
}

bool fibre_usable(const blco_tensor* t, const MttkrpArgs& a)
{
    if (!fibre_eligible(t, a.mode) || !fibre_lanes(a.rank, a.factor_dtype)) return false;
    for (int m = 0; m < t->layout.nmodes; m++)
        if (m != a.mode && ((uintptr_t)a.factors[m] & (fb_vb(a.factor_dtype) - 1))) return false;
    return ((uintptr_t)a.out & 15u) == 0;
}

int mttkrp_fibre_launch(blco_tensor* t, const MttkrpArgs& a, cudaStream_t s)
{
    const Layout& L = t->layout;
    const int lanes = fibre_lanes(a.rank, a.factor_dtype);
    if (!fibre_usable(t, a))
        return fail(BLCO_ERR_UNSUPPORTED, "the fibre schedule needs rank * element size of 32 bytes times a power "
                                          "of two up to 1024, 32-byte aligned factors, a 16-byte aligned output and a "
                                          "resident "
                                          "tensor with 64-bit keys");
    BLCO_TRY(build_fibre_copy(t, a.mode, s));
    FibreCopy& f = t->fib[a.mode];
    const bool f64 = a.factor_dtype == BLCO_DTYPE_F64;
    if (!f64) BLCO_TRY(fibre_values_f32(t, a.mode, s));
    DeviceInfo di;
    BLCO_TRY(device_info(t->device, &di));
    FibParams p;
    memset(&p, 0, sizeof(p));
    for (int m = 0; m < f.ninner; m++) {
        p.fw[m] = f.d_fw[m];
        p.fi[m] = a.factors[f.inner[m]];
    }
    for (int m = 0; m <= f.ninner; m++) p.lw[m] = f.d_lw[m];
    p.fv = f64 ? (const void*)f.d_fv : (const void*)f.d_fv32;
    p.lv = f64 ? (const void*)f.d_lv : (const void*)f.d_lv32;
    p.fib = f.d_fib;
    p.frows = f.d_frows;
    p.fctab = f.d_fctab;
    p.nf = f.nf;
    p.lrows = f.d_lrows;
    p.lctab = f.d_lctab;
    p.nl = f.nl;
    p.ff = a.factors[f.fmode];
    p.out = a.out;
    const uint64_t task = (uint64_t)(32 / lanes) * FB_SUB;
    p.ntask_f = (f.nf + task - 1) / task;
    p.ntasks = p.ntask_f + (f.nl + task - 1) / task;
    p.stride = a.interleave ? 1 : task_stride(p.ntasks); // 1: tasks in stream order
    p.counter = f.d_counter;
    BLCO_CUDA(cudaMemsetAsync(f.d_counter, 0, sizeof(uint32_t), s));
    FibFn fn = nullptr;
    const bool out64 = f64 || a.out64;
    switch (a.factor_dtype) {
    case BLCO_DTYPE_F64: fn = pick_fib<FibF64, double>(L.nmodes, lanes); break;
    case BLCO_DTYPE_F32:
        fn = out64 ? pick_fib<FibF32, double>(L.nmodes, lanes) : pick_fib<FibF32, float>(L.nmodes, lanes);
        break;
    default: fn = out64 ? pick_fib<FibBF16, double>(L.nmodes, lanes) : pick_fib<FibBF16, float>(L.nmodes, lanes); break;
    }
    if (!fn) return fail(BLCO_ERR_UNSUPPORTED, "no fibre kernel for this order and rank");
    int per_sm = 0;
    BLCO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fn, FB_THREADS, 0));
    const int grid = di.sm_count * std::max(1, per_sm);
    fn<<<grid, FB_THREADS, 0, s>>>(p);
    BLCO_CHECK_LAUNCH("k_mttkrp_fib");
    return BLCO_OK;
}

} // namespace blco
