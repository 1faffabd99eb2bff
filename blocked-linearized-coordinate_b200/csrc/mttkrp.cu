// mttkrp.cu -- sparse MTTKRP over the BLCO stream (64-bit keys; keys of up to
// 128 bits in the wide-key section).
//
//   out[r_t(i), :] += val_i * prod_{m != t} U_m[r_m(i), :]
//
// The reference computes this with one-warp CTAs over 32-nonzero tiles
// (mttkrp_lvl1/lvl2/lvl3/atomic, src/alto_dev.cu:31-1847).  This file keeps
// the tile-level conflict resolution idea but is laid out for B200:
//   * persistent CTAs, one per SM (grid = SM count), 24 warps per CTA, each
//     CTA owning one contiguous slice of a stream (or the tiles dealt
//     round-robin over the grid's warps);
//   * the tile kernel (k_mttkrp_vec): a warp takes 32 nonzeros, decodes rows
//     with shifts and masks (alt_pext, src/alto_dev.cu:13-16), groups equal
//     output rows with __match_any_sync and writes the tile in row order
//     into a per-warp shared staging area as packed 32-byte records (two
//     16-byte loads per record; the slot ranges are offset by 16 bytes so
//     concurrent slots hit different banks);
//   * factor rows are gathered with 128-bit loads: R/VEC lanes per nonzero
//     (VEC = 2 FP64, 4 FP32 or 8 BF16 columns per load), several nonzeros in
//     flight per warp;
//   * runs of equal output rows are summed in registers and flushed once:
//     into a per-CTA FP64 shared-memory accumulator when the mode is short
//     enough to fit (the lvl3 role) or for heavy rows without a row-grouped
//     copy, otherwise with global atomics (FP64 red, or 4-wide FP32 vector
//     red);
//   * the heavy-row kernel (k_mttkrp_hot) walks a mode's row-grouped copy of
//     its heaviest rows, keeping FP64 sums in registers until the row
//     changes; the tile kernel then runs on the mode's cold copy, which is
//     ordered by row so that a tile spans few rows.
// Precision policies:
//   PolicyF64   plain form: FP64 values, factors, accumulation and output;
//   PolicyF32   mixed form: FP32 values, FP32 factor gathers, FP32 output;
//   PolicyBF16  mixed form: FP32 values, BF16 factor gathers, FP32 output.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>

#include <vector>

#include <thread>

#include "internal.cuh"

namespace blco {
namespace {

constexpr int MT_THREADS = 768; // 24 warps, one CTA per SM
constexpr int MT_WARPS = MT_THREADS / 32;
constexpr int REC_BYTES = 32;

__global__ void k_to_f32(const double* __restrict__ in, float* __restrict__ out, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

// VEC: columns per 16-byte gather; UNROLL: nonzeros whose gathers are in
// flight per slot (bounded by the registers the gathered values take).
struct PolicyF64 {
    typedef double TV;
    typedef double TF;
    typedef double TA;
    static constexpr int VEC = 2;
    static constexpr int UNROLL = 4;
};
struct PolicyF32 {
    typedef float TV;
    typedef float TF;
    typedef float TA;
    static constexpr int VEC = 4;
    static constexpr int UNROLL = 4;
};
struct PolicyBF16 {
    typedef float TV;
    typedef __nv_bfloat16 TF;
    typedef float TA;
    static constexpr int VEC = 8;
    static constexpr int UNROLL = 2;
};

struct MtParams {
    const uint64_t* coords;
    const void* vals;
    uint64_t nnz;
    const void* f[BLCO_MAX_MODES];
    void* out;
    uint64_t mask[BLCO_MAX_MODES];
    int pos[BLCO_MAX_MODES];
    int mode;
    int rank;
    // heavy-row privatisation
    const uint32_t* hot_keys;  // hash_size entries (row + 1, 0 = empty)
    const uint32_t* hot_slot;  // hash_size entries
    const uint32_t* hot_rows;  // slot -> row
    int hash_size;             // 0: no table
    int nhot;                  // slots kept in shared memory (slot < nhot)
    int direct;                // 1: every row of the target mode is a slot (slot = row)
    int nacc;                  // rows held in the shared accumulator
    int merge;                 // 0: flush every nonzero on its own (kernel 13)
    int interleave;            // 1: tiles dealt round-robin to the grid's warps; 0: a contiguous range per CTA
    uint64_t tiles_per_cta;
};

// The row-grouped copy of a mode's hot rows (HotTable::d_hcoords / d_hvals).
struct HotParams {
    const uint64_t* coords; // grouped by slot, ALTO order inside a slot
    const void* vals;       // same order, TV of the policy
    const uint32_t* ptr;    // nhot + 1 offsets
    const uint32_t* rows;   // slot -> row
    double* acc;            // non-null: FP64 per-slot sums (nhot x R) instead of the output
    int nhot;
    uint32_t total;         // ptr[nhot]
    uint32_t chunk;         // positions per warp task (multiple of 32)
};

__device__ __forceinline__ uint32_t hot_hash(uint32_t r) { return (r * 2654435761u) >> 7; }

// Slot of `row` in the shared accumulator, or -1.
__device__ __forceinline__ int hot_lookup(const MtParams& p, const uint32_t* skeys, const uint32_t* sslot,
                                          uint32_t row)
{
    if (p.direct) return (int)row;
    if (p.hash_size == 0) return -1;
    uint32_t h = hot_hash(row) & (p.hash_size - 1);
    for (int probe = 0; probe < p.hash_size; probe++) {
        uint32_t k = skeys[h];
        if (k == row + 1) {
            int s = (int)sslot[h];
            return s < p.nhot ? s : -1;
        }
        if (k == 0) return -1;
        h = (h + 1) & (p.hash_size - 1);
    }
    return -1;
}

// Per-thread copy of the target/other mode fields, resolved once with
// compile-time indices so the hot loop keeps them in registers.
template <int NM>
struct ModeSel {
    static constexpr int NO = NM > 1 ? NM - 1 : 1;
    int tpos;
    uint64_t tmask;
    int opos[NO];
    uint64_t omask[NO];
    const void* of[NO];

    __device__ __forceinline__ explicit ModeSel(const MtParams& p)
    {
        tpos = p.pos[0];
        tmask = p.mask[0];
#pragma unroll
        for (int m = 1; m < NM; m++)
            if (m == p.mode) {
                tpos = p.pos[m];
                tmask = p.mask[m];
            }
#pragma unroll
        for (int k = 0; k < NO; k++) {
            opos[k] = 0;
            omask[k] = 0;
            of[k] = nullptr;
        }
#pragma unroll
        for (int k = 0; k < NM - 1; k++) {
            // k-th mode other than the target: k if k < mode, else k + 1
            opos[k] = p.pos[k];
            omask[k] = p.mask[k];
            of[k] = p.f[k];
            if (k >= p.mode) {
                opos[k] = p.pos[k + 1];
                omask[k] = p.mask[k + 1];
                of[k] = p.f[k + 1];
            }
        }
    }
};

// Packed staging record (32 bytes):
//   a = {row_t, slot, oth0, oth1}, b = {oth2, oth3, value (FP64 bits, or FP32 in .z)}
struct Rec {
    uint4 a;
    uint4 b;
};

template <int PER>
__device__ __forceinline__ int rec_offset(int p)
{
    return p * REC_BYTES + (p / PER) * 16;
}

template <typename TV>
__device__ __forceinline__ TV rec_val(const uint4& b);
template <>
__device__ __forceinline__ double rec_val<double>(const uint4& b)
{
    return __hiloint2double((int)b.w, (int)b.z);
}
template <>
__device__ __forceinline__ float rec_val<float>(const uint4& b)
{
    return __uint_as_float(b.z);
}

template <typename TV>
__device__ __forceinline__ void rec_set_val(uint4& b, TV v);
template <>
__device__ __forceinline__ void rec_set_val<double>(uint4& b, double v)
{
    b.z = (uint32_t)__double2loint(v);
    b.w = (uint32_t)__double2hiint(v);
}
template <>
__device__ __forceinline__ void rec_set_val<float>(uint4& b, float v)
{
    b.z = __float_as_uint(v);
    b.w = 0;
}

__device__ __forceinline__ uint32_t rec_oth(const Rec& r, int k)
{
    return k == 0 ? r.a.z : k == 1 ? r.a.w : k == 2 ? r.b.x : r.b.y;
}

// Sorts the warp's tile by output row into the staging area.  Returns the
// number of valid entries and the bitmask of positions that end a run.
template <int NM, int PER, typename TV>
__device__ __forceinline__ int stage_tile(const MtParams& p, const ModeSel<NM>& ms, const uint32_t* skeys,
                                          const uint32_t* sslot, uint64_t i0, unsigned char* st, uint32_t& ends)
{
    const int lane = threadIdx.x & 31;
    const uint64_t i = i0 + lane;
    const bool valid = i < p.nnz;
    uint64_t c = valid ? __ldcs(p.coords + i) : 0;
    TV v = valid ? __ldcs(reinterpret_cast<const TV*>(p.vals) + i) : TV(0);
    uint32_t rt = (uint32_t)((c >> ms.tpos) & ms.tmask);
    uint32_t ro[4] = {0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < NM - 1; k++) ro[k] = (uint32_t)((c >> ms.opos[k]) & ms.omask[k]);
    int slot = valid ? hot_lookup(p, skeys, sslot, rt) : -1;
    // Entries past the end are ordered after the working ones.
    const bool work = valid;
    const uint32_t wmask = __ballot_sync(0xffffffffu, work);
    uint32_t key = work ? rt : 0xffffffffu;
    uint32_t peers = __match_any_sync(0xffffffffu, key);
    const uint32_t lt = (1u << lane) - 1;
    int leader = __ffs(peers) - 1;
    uint32_t x = (lane == leader && work) ? (uint32_t)__popc(peers) : 0u;
    uint32_t inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    uint32_t start = __shfl_sync(0xffffffffu, inc - x, leader);
    const int count = __popc(wmask);
    int sp = work ? (int)start + __popc(peers & lt) : count + __popc(~wmask & lt);
    bool last = work && (peers >> lane) == 1u;
    ends = __reduce_or_sync(0xffffffffu, last ? (1u << sp) : 0u);
    Rec r;
    r.a = make_uint4(rt, (uint32_t)slot, ro[0], ro[1]);
    r.b = make_uint4(ro[2], ro[3], 0u, 0u);
    rec_set_val<TV>(r.b, v);
    uint4* dst = reinterpret_cast<uint4*>(st + rec_offset<PER>(sp));
    dst[0] = r.a;
    dst[1] = r.b;
    __syncwarp();
    return count;
}

// 16-byte gather of VEC factor entries, widened to the accumulator type.
template <class P>
struct Gather;
template <>
struct Gather<PolicyF64> {
    static __device__ __forceinline__ void load(const void* base, uint32_t row, int R, int q, double (&g)[2])
    {
        double2 v = __ldg(reinterpret_cast<const double2*>(base) + ((size_t)row * R) / 2 + q);
        g[0] = v.x;
        g[1] = v.y;
    }
};
template <>
struct Gather<PolicyF32> {
    static __device__ __forceinline__ void load(const void* base, uint32_t row, int R, int q, float (&g)[4])
    {
        float4 v = __ldg(reinterpret_cast<const float4*>(base) + ((size_t)row * R) / 4 + q);
        g[0] = v.x;
        g[1] = v.y;
        g[2] = v.z;
        g[3] = v.w;
    }
};
template <>
struct Gather<PolicyBF16> {
    static __device__ __forceinline__ void load(const void* base, uint32_t row, int R, int q, float (&g)[8])
    {
        uint4 v = __ldg(reinterpret_cast<const uint4*>(base) + ((size_t)row * R) / 8 + q);
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int j = 0; j < 4; j++) {
            // bf16 -> fp32 is exact: the bf16 bits are the high half of the fp32.
            g[2 * j] = __uint_as_float(w[j] << 16);
            g[2 * j + 1] = __uint_as_float(w[j] & 0xffff0000u);
        }
    }
};

template <class P>
__device__ __forceinline__ void flush_global(void* out, uint32_t row, int R, int q,
                                             const typename P::TA (&a)[P::VEC])
{
    constexpr int VEC = P::VEC;
    typename P::TA* o = reinterpret_cast<typename P::TA*>(out) + (size_t)row * R + VEC * q;
    if constexpr (sizeof(typename P::TA) == 8) {
#pragma unroll
        for (int j = 0; j < VEC; j++) atomicAdd(o + j, a[j]);
    } else {
#pragma unroll
        for (int j = 0; j < VEC; j += 4)
            atomicAdd(reinterpret_cast<float4*>(o + j), make_float4(a[j], a[j + 1], a[j + 2], a[j + 3]));
    }
}

template <int NM, int R, class P>
__global__ void __launch_bounds__(MT_THREADS, 1) k_mttkrp_vec(MtParams p)
{
    typedef typename P::TV TV;
    typedef typename P::TA TA;
    typedef double TS; // shared accumulators are FP64 in every form
    constexpr int VEC = P::VEC;
    constexpr int LPN = R / VEC;
    constexpr int SLOTS = 32 / LPN;
    constexpr int PER = 32 / SLOTS;
    constexpr int STAGE = 32 * REC_BYTES + SLOTS * 16;
    constexpr int MT_UNROLL = P::UNROLL;
    extern __shared__ __align__(16) unsigned char smem[];
    uint32_t* skeys = reinterpret_cast<uint32_t*>(smem);
    uint32_t* sslot = skeys + p.hash_size;
    TS* sacc = reinterpret_cast<TS*>(smem + 8 * (size_t)p.hash_size);
    const int nacc = p.nacc;
    unsigned char* stages = reinterpret_cast<unsigned char*>(sacc + (size_t)nacc * R);
    stages = reinterpret_cast<unsigned char*>(((uintptr_t)stages + 15) & ~(uintptr_t)15);

    for (int i = threadIdx.x; i < p.hash_size; i += blockDim.x) {
        skeys[i] = p.hot_keys[i];
        sslot[i] = p.hot_slot[i];
    }
    for (size_t i = threadIdx.x; i < (size_t)nacc * R; i += blockDim.x) sacc[i] = TS(0);
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int slot = lane / LPN, q = lane % LPN;
    unsigned char* st = stages + (size_t)warp * STAGE;
    const uint64_t ntiles = (p.nnz + 31) / 32;
    const uint64_t t_beg = p.interleave ? (uint64_t)blockIdx.x * MT_WARPS : (uint64_t)blockIdx.x * p.tiles_per_cta;
    const uint64_t t_end = p.interleave ? ntiles : min(ntiles, t_beg + p.tiles_per_cta);
    const uint64_t t_step = p.interleave ? (uint64_t)gridDim.x * MT_WARPS : (uint64_t)MT_WARPS;
    const ModeSel<NM> ms(p);

    for (uint64_t tile = t_beg + warp; tile < t_end; tile += t_step) {
        uint32_t ends;
        const int count = stage_tile<NM, PER, TV>(p, ms, skeys, sslot, tile * 32, st, ends);
        if (!p.merge) ends = 0xffffffffu;
        const int pb = slot * PER, pe = min(pb + PER, count);
        TA acc[VEC];
#pragma unroll
        for (int j = 0; j < VEC; j++) acc[j] = TA(0);
        for (int p0 = pb; p0 < pe; p0 += MT_UNROLL) {
            TA g[MT_UNROLL][NM > 1 ? NM - 1 : 1][VEC];
            Rec rec[MT_UNROLL];
#pragma unroll
            for (int u = 0; u < MT_UNROLL; u++) {
                int pp = p0 + u;
                if (pp < pe) {
                    const uint4* src = reinterpret_cast<const uint4*>(st + rec_offset<PER>(pp));
                    rec[u].a = src[0];
                    rec[u].b = src[1];
#pragma unroll
                    for (int k = 0; k < NM - 1; k++) Gather<P>::load(ms.of[k], rec_oth(rec[u], k), R, q, g[u][k]);
                }
            }
#pragma unroll
            for (int u = 0; u < MT_UNROLL; u++) {
                int pp = p0 + u;
                if (pp < pe) {
                    const TA v = (TA)rec_val<TV>(rec[u].b);
#pragma unroll
                    for (int j = 0; j < VEC; j++) {
                        TA prod = v;
#pragma unroll
                        for (int k = 0; k < NM - 1; k++) prod *= g[u][k][j];
                        acc[j] += prod;
                    }
                    if (((ends >> pp) & 1u) || pp == pe - 1) {
                        const int s = (int)rec[u].a.y;
                        if (s >= 0) {
                            TS* d = sacc + (size_t)s * R + VEC * q;
#pragma unroll
                            for (int j = 0; j < VEC; j++) atomicAdd(d + j, (TS)acc[j]);
                        } else {
                            flush_global<P>(p.out, rec[u].a.x, R, q, acc);
                        }
#pragma unroll
                        for (int j = 0; j < VEC; j++) acc[j] = TA(0);
                    }
                }
            }
        }
        __syncwarp();
    }
    __syncthreads();
    // Write the privatised rows back once.
    TA* out = reinterpret_cast<TA*>(p.out);
    for (size_t i = threadIdx.x; i < (size_t)nacc * R; i += blockDim.x) {
        TS v = sacc[i];
        if (v != TS(0)) {
            size_t s = i / R;
            uint32_t row = p.direct ? (uint32_t)s : p.hot_rows[s];
            atomicAdd(out + (size_t)row * R + (i % R), (TA)v);
        }
    }
}

// Hot-row kernel: walks the CSR view of the mode's heaviest rows.  Warp
// tasks are chunks of `chunk` consecutive positions; inside a chunk the
// nonzeros come grouped by row, so each lane group keeps its partial sum in
// registers across the whole chunk and flushes it (global atomics) only when
// its row changes and at the chunk end.  No shared-memory accumulators and
// no sorting are needed.
template <int NM, int R, class P>
__global__ void __launch_bounds__(MT_THREADS, 1) k_mttkrp_hot(MtParams p, HotParams h)
{
    typedef typename P::TV TV;
    typedef typename P::TA TA;
    constexpr int VEC = P::VEC;
    constexpr int LPN = R / VEC;
    constexpr int GROUPS = 32 / LPN;
    constexpr int PER = 32 / GROUPS;
    constexpr int STAGE = 32 * REC_BYTES + GROUPS * 16;
    constexpr int MT_UNROLL = P::UNROLL;
    extern __shared__ __align__(16) unsigned char smem[];
    uint32_t* sptr = reinterpret_cast<uint32_t*>(smem);   // nhot + 1
    uint32_t* srows = sptr + h.nhot + 1;                    // nhot
    unsigned char* stages =
        reinterpret_cast<unsigned char*>(((uintptr_t)(srows + h.nhot) + 15) & ~(uintptr_t)15);
    for (int i = threadIdx.x; i <= h.nhot; i += blockDim.x) sptr[i] = h.ptr[i];
    for (int i = threadIdx.x; i < h.nhot; i += blockDim.x) srows[i] = h.rows[i];
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = lane / LPN, q = lane % LPN;
    unsigned char* st = stages + (size_t)warp * STAGE;
    const ModeSel<NM> ms(p);
    const uint32_t nchunks = (h.total + h.chunk - 1) / h.chunk;
    const uint32_t nw = gridDim.x * MT_WARPS;
    // Partial sums run over up to `chunk` nonzeros: kept in FP64 in every form.
    double acc[VEC];
    int acc_slot = -1;
    auto flush = [&](int slot_id) {
        if (h.acc) {
            double* d = h.acc + (size_t)slot_id * R + VEC * q;
#pragma unroll
            for (int j = 0; j < VEC; j++) atomicAdd(d + j, acc[j]);
        } else {
            TA a[VEC];
#pragma unroll
            for (int j = 0; j < VEC; j++) a[j] = (TA)acc[j];
            flush_global<P>(p.out, srows[slot_id], R, q, a);
        }
    };
    for (uint32_t c = blockIdx.x * MT_WARPS + warp; c < nchunks; c += nw) {
        const uint32_t j0 = c * h.chunk, j1 = min(h.total, j0 + h.chunk);
        // slot holding position j0: the last s with sptr[s] <= j0
        int lo = 0, hi = h.nhot - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (sptr[mid] <= j0) lo = mid;
            else hi = mid - 1;
        }
        int cur = lo;
#pragma unroll
        for (int j = 0; j < VEC; j++) acc[j] = 0.0;
        acc_slot = -1;
        for (uint32_t sub = j0; sub < j1; sub += 32) {
            while (cur < h.nhot - 1 && sptr[cur + 1] <= sub) cur++;
            const uint32_t jj = sub + lane;
            const bool valid = jj < j1;
            int ls = cur;
            if (valid)
                while (ls < h.nhot - 1 && sptr[ls + 1] <= jj) ls++;
            const uint64_t cc = valid ? __ldcs(h.coords + jj) : 0ull;
            const TV v = valid ? __ldcs(reinterpret_cast<const TV*>(h.vals) + jj) : TV(0);
            uint32_t ro[4] = {0, 0, 0, 0};
#pragma unroll
            for (int k = 0; k < NM - 1; k++) ro[k] = (uint32_t)((cc >> ms.opos[k]) & ms.omask[k]);
            Rec r;
            r.a = make_uint4(0u, (uint32_t)ls, ro[0], ro[1]);
            r.b = make_uint4(ro[2], ro[3], 0u, 0u);
            rec_set_val<TV>(r.b, v);
            uint4* dst = reinterpret_cast<uint4*>(st + rec_offset<PER>(lane));
            dst[0] = r.a;
            dst[1] = r.b;
            __syncwarp();
            const int count = (int)min(32u, j1 - sub);
            const int pb = grp * PER, pe = min(pb + PER, count);
            for (int p0 = pb; p0 < pe; p0 += MT_UNROLL) {
                TA g[MT_UNROLL][NM > 1 ? NM - 1 : 1][VEC];
                Rec rec[MT_UNROLL];
#pragma unroll
                for (int u = 0; u < MT_UNROLL; u++) {
                    int pp = p0 + u;
                    if (pp < pe) {
                        const uint4* src = reinterpret_cast<const uint4*>(st + rec_offset<PER>(pp));
                        rec[u].a = src[0];
                        rec[u].b = src[1];
#pragma unroll
                        for (int k = 0; k < NM - 1; k++)
                            Gather<P>::load(ms.of[k], rec_oth(rec[u], k), R, q, g[u][k]);
                    }
                }
#pragma unroll
                for (int u = 0; u < MT_UNROLL; u++) {
                    int pp = p0 + u;
                    if (pp < pe) {
                        const int s = (int)rec[u].a.y;
                        if (s != acc_slot) {
                            if (acc_slot >= 0) flush(acc_slot);
#pragma unroll
                            for (int j = 0; j < VEC; j++) acc[j] = 0.0;
                            acc_slot = s;
                        }
                        const TA vv = (TA)rec_val<TV>(rec[u].b);
#pragma unroll
                        for (int j = 0; j < VEC; j++) {
                            TA prod = vv;
#pragma unroll
                            for (int k = 0; k < NM - 1; k++) prod *= g[u][k][j];
                            acc[j] += (double)prod;
                        }
                    }
                }
            }
            __syncwarp();
        }
        if (acc_slot >= 0) flush(acc_slot);
        acc_slot = -1;
    }
}

// out[rows[s]] += (float)acc[s] for the mixed form's hot rows (one rounding).
__global__ void k_merge_hot(const double* __restrict__ acc, const uint32_t* __restrict__ rows, int nhot, int R,
                            float* __restrict__ out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nhot * R; i += gridDim.x * blockDim.x) {
        const int s = i / R, c = i % R;
        float* o = out + (size_t)rows[s] * R + c;
        *o = (float)((double)*o + acc[i]);
    }
}

// Generic kernel: any R up to 256, a whole warp per nonzero, columns
// lane, lane+32, ...  Used for ranks the vectorised kernels do not cover and
// for factor pointers that are not 16-byte aligned.
constexpr int GEN_MAXC = 8;

template <int NM, class P>
__global__ void __launch_bounds__(MT_THREADS, 1) k_mttkrp_gen(MtParams p)
{
    typedef typename P::TV TV;
    typedef typename P::TF TF;
    typedef typename P::TA TA;
    typedef double TS;
    constexpr int PER = 32;
    constexpr int STAGE = 32 * REC_BYTES + 16;
    extern __shared__ __align__(16) unsigned char smem[];
    uint32_t* skeys = reinterpret_cast<uint32_t*>(smem);
    uint32_t* sslot = skeys + p.hash_size;
    TS* sacc = reinterpret_cast<TS*>(smem + 8 * (size_t)p.hash_size);
    const int R = p.rank;
    const int nacc = p.nacc;
    unsigned char* stages = reinterpret_cast<unsigned char*>(sacc + (size_t)nacc * R);
    stages = reinterpret_cast<unsigned char*>(((uintptr_t)stages + 15) & ~(uintptr_t)15);
    for (int i = threadIdx.x; i < p.hash_size; i += blockDim.x) {
        skeys[i] = p.hot_keys[i];
        sslot[i] = p.hot_slot[i];
    }
    for (size_t i = threadIdx.x; i < (size_t)nacc * R; i += blockDim.x) sacc[i] = TS(0);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* st = stages + (size_t)warp * STAGE;
    const uint64_t ntiles = (p.nnz + 31) / 32;
    const uint64_t t_beg = p.interleave ? (uint64_t)blockIdx.x * MT_WARPS : (uint64_t)blockIdx.x * p.tiles_per_cta;
    const uint64_t t_end = p.interleave ? ntiles : min(ntiles, t_beg + p.tiles_per_cta);
    const uint64_t t_step = p.interleave ? (uint64_t)gridDim.x * MT_WARPS : (uint64_t)MT_WARPS;
    const ModeSel<NM> ms(p);
    const int ncol = (R + 31) / 32;
    for (uint64_t tile = t_beg + warp; tile < t_end; tile += t_step) {
        uint32_t ends;
        const int count = stage_tile<NM, PER, TV>(p, ms, skeys, sslot, tile * 32, st, ends);
        if (!p.merge) ends = 0xffffffffu;
        TA acc[GEN_MAXC];
#pragma unroll
        for (int j = 0; j < GEN_MAXC; j++) acc[j] = TA(0);
        for (int pp = 0; pp < count; pp++) {
            const uint4* src = reinterpret_cast<const uint4*>(st + rec_offset<PER>(pp));
            Rec rec;
            rec.a = src[0];
            rec.b = src[1];
            const TA v = (TA)rec_val<TV>(rec.b);
#pragma unroll
            for (int j = 0; j < GEN_MAXC; j++) {
                int c = lane + 32 * j;
                if (j < ncol && c < R) {
                    TA prod = v;
#pragma unroll
                    for (int k = 0; k < NM - 1; k++)
                        prod *= (TA)reinterpret_cast<const TF*>(ms.of[k])[(size_t)rec_oth(rec, k) * R + c];
                    acc[j] += prod;
                }
            }
            if (((ends >> pp) & 1u) || pp == count - 1) {
                const uint32_t row = rec.a.x;
                const int s = (int)rec.a.y;
#pragma unroll
                for (int j = 0; j < GEN_MAXC; j++) {
                    int c = lane + 32 * j;
                    if (j < ncol && c < R) {
                        if (s >= 0) atomicAdd(sacc + (size_t)s * R + c, (TS)acc[j]);
                        else atomicAdd(reinterpret_cast<TA*>(p.out) + (size_t)row * R + c, acc[j]);
                    }
                    acc[j] = TA(0);
                }
            }
        }
        __syncwarp();
    }
    __syncthreads();
    TA* out = reinterpret_cast<TA*>(p.out);
    for (size_t i = threadIdx.x; i < (size_t)nacc * R; i += blockDim.x) {
        TS v = sacc[i];
        if (v != TS(0)) {
            size_t s = i / R;
            uint32_t row = p.direct ? (uint32_t)s : p.hot_rows[s];
            atomicAdd(out + (size_t)row * R + (i % R), (TA)v);
        }
    }
}

typedef void (*KernelFn)(MtParams);

template <int NM, class P>
KernelFn pick_vec(int R)
{
    constexpr int V = P::VEC;
    switch (R) {
    case 2: if constexpr (V <= 2) return k_mttkrp_vec<NM, 2, P>; else return nullptr;
    case 4: if constexpr (V <= 4) return k_mttkrp_vec<NM, 4, P>; else return nullptr;
    case 8: return k_mttkrp_vec<NM, 8, P>;
    case 16: return k_mttkrp_vec<NM, 16, P>;
    case 32: return k_mttkrp_vec<NM, 32, P>;
    case 64: return k_mttkrp_vec<NM, 64, P>;
    case 128: if constexpr (V >= 4) return k_mttkrp_vec<NM, 128, P>; else return nullptr;
    default: return nullptr;
    }
}

typedef void (*HotFn)(MtParams, HotParams);

template <int NM, class P>
HotFn pick_hot_nm(int R)
{
    constexpr int V = P::VEC;
    switch (R) {
    case 8: return k_mttkrp_hot<NM, 8, P>;
    case 16: return k_mttkrp_hot<NM, 16, P>;
    case 32: return k_mttkrp_hot<NM, 32, P>;
    case 64: return k_mttkrp_hot<NM, 64, P>;
    case 128: if constexpr (V >= 4) return k_mttkrp_hot<NM, 128, P>; else return nullptr;
    default: return nullptr;
    }
}

template <class P>
HotFn pick_hot(int nm, int R)
{
    switch (nm) {
    case 2: return pick_hot_nm<2, P>(R);
    case 3: return pick_hot_nm<3, P>(R);
    case 4: return pick_hot_nm<4, P>(R);
    case 5: return pick_hot_nm<5, P>(R);
    default: return nullptr;
    }
}

template <class P>
KernelFn pick_generic(int nm)
{
    switch (nm) {
    case 1: return k_mttkrp_gen<1, P>;
    case 2: return k_mttkrp_gen<2, P>;
    case 3: return k_mttkrp_gen<3, P>;
    case 4: return k_mttkrp_gen<4, P>;
    default: return k_mttkrp_gen<5, P>;
    }
}

template <class P>
KernelFn pick_kernel(int nm, int R, bool aligned16)
{
    KernelFn f = nullptr;
    if (aligned16) {
        switch (nm) {
        case 1: f = pick_vec<1, P>(R); break;
        case 2: f = pick_vec<2, P>(R); break;
        case 3: f = pick_vec<3, P>(R); break;
        case 4: f = pick_vec<4, P>(R); break;
        case 5: f = pick_vec<5, P>(R); break;
        }
    }
    return f ? f : pick_generic<P>(nm);
}

// Per-CTA staging bytes: 32 records per warp plus one 16-byte pad per slot
// range (slots = 32 lanes / lanes per nonzero).
size_t stage_bytes(int rank, int vec)
{
    int lpn = rank / vec;
    int slots = (lpn >= 1 && lpn <= 32 && rank % vec == 0) ? 32 / lpn : 1;
    return (size_t)MT_WARPS * (32 * REC_BYTES + slots * 16) + 16;
}

int policy_vec(int dtype) { return dtype == BLCO_DTYPE_F64 ? 2 : dtype == BLCO_DTYPE_F32 ? 4 : 8; }

// Shared-memory accumulators are FP64 in every form: a heavy row collects
// up to millions of contributions per CTA, too many to sum in FP32.
size_t acc_elem_bytes(int) { return 8; }

} // namespace

int mttkrp_select_kernel(const blco_tensor* t, int mode, int rank, int requested, int factor_dtype)
{
    if (t->layout.wide) return BLCO_KERNEL_LVL1; // one kernel for keys above 64 bits
    DeviceInfo di;
    if (device_info(t->device, &di) != BLCO_OK) return BLCO_KERNEL_LVL1;
    size_t budget = di.smem_optin - stage_bytes(rank, policy_vec(factor_dtype)) - 2 * sizeof(uint32_t) * 4096 - 1024;
    bool fits_direct = t->layout.dims[mode] * (uint64_t)rank * acc_elem_bytes(factor_dtype) <= budget;
    const bool fibre_ok = fibre_eligible(t, mode) && fibre_lanes(rank, factor_dtype) > 0;
    const int tiles = t->hot[mode].nhot > 0 && t->hot[mode].hot_nnz >= AUTO_HOT_MIN_NNZ ? BLCO_KERNEL_LVL2
                                                                                      : BLCO_KERNEL_LVL1;
    switch (requested) {
    case BLCO_KERNEL_LVL1:
    case BLCO_KERNEL_BATCHED:
    case BLCO_KERNEL_BATCHED_V2: return BLCO_KERNEL_LVL1;
    case BLCO_KERNEL_LVL2: return BLCO_KERNEL_LVL2;
    case BLCO_KERNEL_LVL3: return fits_direct ? BLCO_KERNEL_LVL3 : BLCO_KERNEL_LVL2;
    case BLCO_KERNEL_ATOMIC: return BLCO_KERNEL_ATOMIC;
    case BLCO_KERNEL_FIBRE: return fibre_ok ? BLCO_KERNEL_FIBRE : fits_direct ? BLCO_KERNEL_LVL3 : tiles;
    default:
        if (fits_direct) return BLCO_KERNEL_LVL3;
        return fibre_ok ? BLCO_KERNEL_FIBRE : tiles;
    }
}

bool fibre_route(const blco_tensor* t, const MttkrpArgs& a)
{
    if (a.kernel != BLCO_KERNEL_FIBRE && a.kernel != BLCO_KERNEL_AUTO) return false;
    if (a.coords != t->d_coords || !fibre_usable(t, a)) return false;
    return mttkrp_select_kernel(t, a.mode, a.rank, a.kernel, a.factor_dtype) == BLCO_KERNEL_FIBRE;
}

// Heavy-row chunk of the automatic rule: few heavy nonzeros need small
// chunks to give every warp of the grid work (128 below 1M, 512 below 8M,
// else 2048, from autotuner sweeps over skewed tensors of 1e5..2e8 nnz).
uint32_t auto_hot_chunk(uint64_t hot_nnz) { return hot_nnz < (1u << 20) ? 128u : hot_nnz < (8u << 20) ? 512u : 2048u; }

int values_f32(blco_tensor* t, cudaStream_t s, const float** out)
{
    if (!t->d_values_f32 && t->nnz) {
        if (!t->resident) return fail(BLCO_ERR_STATE, "FP32 values of a streamed tensor are made per block");
        BLCO_CUDA(cudaMalloc(&t->d_values_f32, t->nnz * sizeof(float)));
        k_to_f32<<<1024, 256, 0, s>>>(t->d_values, t->d_values_f32, t->nnz);
        BLCO_CHECK_LAUNCH("k_to_f32");
    }
    *out = t->d_values_f32;
    return BLCO_OK;
}

int host_values_f32(blco_tensor* t)
{
    if (t->h_values32 || !t->nnz) return BLCO_OK;
    if (!t->h_values) return fail(BLCO_ERR_STATE, "tensor has no host values");
    float* h = nullptr;
    BLCO_CUDA(cudaMallocHost(&h, t->nnz * sizeof(float)));
    const unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    for (unsigned w = 0; w < nt; w++)
        th.emplace_back([&, w]() {
            const uint64_t a = t->nnz * w / nt, b = t->nnz * (w + 1) / nt;
            for (uint64_t i = a; i < b; i++) h[i] = (float)t->h_values[i];
        });
    for (auto& x : th) x.join();
    t->h_values32 = h;
    return BLCO_OK;
}

// --------------------------------------------------------- wide keys --
//
// MTTKRP of a tensor whose keys need more than 64 bits (the reference's
// 128-bit build).  The reference reads the stream in key order
// (src/alto_dev.cu:31-306, alt_pext adding the block coordinate, :13-16);
// here mode n reads its own copy of the stream sorted by the row of mode n
// (built at encode time), and a row index is field | block coordinate,
// taken from the per-nonzero block field.  A group of G lanes (G = 8, 16 or
// 32 columns wide) walks a contiguous run of 4G nonzeros: lane k of the
// group loads nonzero k of each batch of G (coalesced) and decodes its
// rows, then the group takes the batch's nonzeros one by one through
// shuffles, gathers the other modes' factor rows (G consecutive columns per
// load), and keeps the running sum of an output row in registers until the
// row changes, when it adds the sum to the output with FP64 atomics; in
// row order that is about once per row and warp task.

namespace {

struct WideParams {
    const uint64_t* coords;
    const uint64_t* field;
    const void* vals;             // T
    uint64_t nnz;
    Layout L;
    const void* f[BLCO_MAX_MODES]; // T
    void* out;                     // T
    int mode;
    int rank;
    int col0; // first column of this launch's column slab
};

constexpr int WIDE_THREADS = 256;
constexpr int WIDE_BATCHES = 4; // batches of G nonzeros per group task

// T: element type of values, factors and output (FP64, or FP32 for the
// mixed form); run sums are FP64 in both.
template <typename T, typename TO, int G, int CPL>
__global__ __launch_bounds__(WIDE_THREADS) void k_mttkrp_wide(const WideParams p)
{
    const T* __restrict__ vals = static_cast<const T*>(p.vals);
    TO* __restrict__ out = static_cast<TO*>(p.out);
    const int lane = threadIdx.x & 31;
    const int sub = lane % G;
    const int grp = lane / G;
    constexpr uint64_t WARP_TASK = (uint64_t)32 * WIDE_BATCHES;
    const uint64_t nwarps = (uint64_t)gridDim.x * (WIDE_THREADS / 32);
    const uint64_t wid = (uint64_t)blockIdx.x * (WIDE_THREADS / 32) + (threadIdx.x >> 5);
    const int nm = p.L.nmodes;
    const int R = p.rank;
    const uint64_t ntasks = (p.nnz + WARP_TASK - 1) / WARP_TASK;
    for (uint64_t task = wid; task < ntasks; task += nwarps) {
        const uint64_t g0 = task * WARP_TASK + (uint64_t)grp * (G * WIDE_BATCHES);
        uint64_t cur = ~0ull;
        double acc[CPL];
#pragma unroll
        for (int k = 0; k < CPL; k++) acc[k] = 0.0;
        for (int b = 0; b < WIDE_BATCHES; b++) {
            const uint64_t i = g0 + (uint64_t)b * G + sub;
            const bool ok = i < p.nnz;
            uint32_t row[BLCO_MAX_MODES];
            double v = 0.0;
            {
                const uint64_t c = ok ? __ldg(p.coords + i) : 0;
                const uint64_t fld = ok ? __ldg(p.field + i) : 0;
                v = ok ? (double)__ldg(vals + i) : 0.0;
#pragma unroll
                for (int n = 0; n < BLCO_MAX_MODES; n++)
                    row[n] = n < nm ? (uint32_t)wide_row(p.L, n, c, fld) : 0u;
            }
            const uint32_t okmask = __ballot_sync(0xffffffffu, ok);
#pragma unroll 4
            for (int j = 0; j < G; j++) {
                const int src = grp * G + j;
                const bool vj = (okmask >> src) & 1u;
                uint32_t r[BLCO_MAX_MODES];
#pragma unroll
                for (int n = 0; n < BLCO_MAX_MODES; n++) r[n] = __shfl_sync(0xffffffffu, row[n], j, G);
                const double vv = __shfl_sync(0xffffffffu, v, j, G);
                if (!vj) continue;
                const uint64_t rt = r[p.mode];
                if (rt != cur) {
                    if (cur != ~0ull) {
#pragma unroll
                        for (int k = 0; k < CPL; k++) {
                            const int col = p.col0 + sub + k * G;
                            if (col < R) atomicAdd(out + cur * R + col, (TO)acc[k]);
                            acc[k] = 0.0;
                        }
                    }
                    cur = rt;
                }
#pragma unroll
                for (int k = 0; k < CPL; k++) {
                    const int col = p.col0 + sub + k * G;
                    if (col < R) {
                        T prod = (T)vv;
#pragma unroll
                        for (int n = 0; n < BLCO_MAX_MODES; n++)
                            if (n < nm && n != p.mode)
                                prod *= __ldg(static_cast<const T*>(p.f[n]) + (uint64_t)r[n] * R + col);
                        acc[k] += (double)prod;
                    }
                }
            }
        }
        if (cur != ~0ull) {
#pragma unroll
            for (int k = 0; k < CPL; k++) {
                const int col = p.col0 + sub + k * G;
                if (col < R) atomicAdd(out + cur * R + col, (TO)acc[k]);
            }
        }
    }
}

// The same walk with two columns per lane (16-byte gathers of FP64 pairs),
// the mode count fixed at compile time and every row decoded once, when
// its batch is loaded: L = R/2 lanes per nonzero (R even, 2L >= R, column
// slab of up to 64), 32/L nonzeros in flight per warp instruction.
// OFF32: factor offsets row * R + col fit in 32 bits.
struct WideParams2 {
    const uint64_t* coords;
    const uint64_t* field;
    const double* vals;
    uint64_t nnz;
    Layout L;
    const double* fo[BLCO_MAX_MODES - 1]; // factors of the other modes, in mode order
    int other[BLCO_MAX_MODES - 1];        // their mode numbers
    double* out;
    int mode;
    int rank;
    int col0;
};

template <int NM, int L, bool OFF32>
__global__ __launch_bounds__(WIDE_THREADS) void k_mttkrp_wide2(const WideParams2 p)
{
    constexpr int NO = NM - 1;
    const int lane = threadIdx.x & 31;
    const int sub = lane % L;
    const int grp = lane / L;
    constexpr uint64_t WARP_TASK = (uint64_t)32 * WIDE_BATCHES;
    const uint64_t nwarps = (uint64_t)gridDim.x * (WIDE_THREADS / 32);
    const uint64_t wid = (uint64_t)blockIdx.x * (WIDE_THREADS / 32) + (threadIdx.x >> 5);
    const int R = p.rank;
    const int col = p.col0 + 2 * sub;
    const bool cok = col < R; // col + 1 < R too: R is even
    const uint64_t ntasks = (p.nnz + WARP_TASK - 1) / WARP_TASK;
    for (uint64_t task = wid; task < ntasks; task += nwarps) {
        const uint64_t g0 = task * WARP_TASK + (uint64_t)grp * (L * WIDE_BATCHES);
        uint32_t cur = 0xffffffffu;
        double a0 = 0.0, a1 = 0.0;
        for (int b = 0; b < WIDE_BATCHES; b++) {
            const uint64_t i = g0 + (uint64_t)b * L + sub;
            const bool ok = i < p.nnz;
            uint32_t rt = 0xffffffffu, ro[NO];
            double v = 0.0;
            {
                const uint64_t c = ok ? __ldg(p.coords + i) : 0;
                const uint64_t f = ok ? __ldg(p.field + i) : 0;
                v = ok ? __ldg(p.vals + i) : 0.0;
                if (ok) rt = (uint32_t)wide_row(p.L, p.mode, c, f);
#pragma unroll
                for (int k = 0; k < NO; k++) ro[k] = (uint32_t)wide_row(p.L, p.other[k], c, f);
            }
            // U nonzeros at a time: every gather of the U is issued before
            // the first product, so each lane has U x (NM-1) loads in flight
            constexpr int U = 4;
#pragma unroll 1
            for (int j0 = 0; j0 < L; j0 += U) {
                uint32_t r[U];
                double vv[U];
                double2 x[U][NO];
#pragma unroll
                for (int u = 0; u < U; u++) {
                    r[u] = __shfl_sync(0xffffffffu, rt, j0 + u, L);
                    vv[u] = __shfl_sync(0xffffffffu, v, j0 + u, L);
#pragma unroll
                    for (int k = 0; k < NO; k++) {
                        const uint32_t rr = __shfl_sync(0xffffffffu, ro[k], j0 + u, L);
                        const double2* src;
                        if (OFF32) src = reinterpret_cast<const double2*>(p.fo[k] + (rr * (uint32_t)R + (uint32_t)col));
                        else src = reinterpret_cast<const double2*>(p.fo[k] + ((uint64_t)rr * R + col));
                        // rows of nonzeros past the end decode to row 0: in bounds
                        x[u][k] = cok ? __ldg(src) : make_double2(0.0, 0.0);
                    }
                }
#pragma unroll
                for (int u = 0; u < U; u++) {
                    if (r[u] == 0xffffffffu) continue; // past the end of the stream
                    if (r[u] != cur) {
                        if (cur != 0xffffffffu && cok) {
                            double* o = p.out + (uint64_t)cur * R + col;
                            atomicAdd(o, a0);
                            atomicAdd(o + 1, a1);
                        }
                        a0 = a1 = 0.0;
                        cur = r[u];
                    }
                    double p0 = vv[u], p1 = vv[u];
#pragma unroll
                    for (int k = 0; k < NO; k++) {
                        p0 *= x[u][k].x;
                        p1 *= x[u][k].y;
                    }
                    a0 += p0;
                    a1 += p1;
                }
            }
        }
        if (cur != 0xffffffffu && cok) {
            double* o = p.out + (uint64_t)cur * R + col;
            atomicAdd(o, a0);
            atomicAdd(o + 1, a1);
        }
    }
}

template <int NM>
int launch_wide2(const WideParams2& p, int grid, int lanes, bool off32, cudaStream_t s)
{
#define WIDE2_CASE(LL)                                                                     \
    if (lanes == LL) {                                                                     \
        if (off32) k_mttkrp_wide2<NM, LL, true><<<grid, WIDE_THREADS, 0, s>>>(p);          \
        else k_mttkrp_wide2<NM, LL, false><<<grid, WIDE_THREADS, 0, s>>>(p);               \
        BLCO_CHECK_LAUNCH("k_mttkrp_wide2");                                               \
        return BLCO_OK;                                                                    \
    }
    WIDE2_CASE(4)
    WIDE2_CASE(8)
    WIDE2_CASE(16)
    WIDE2_CASE(32)
#undef WIDE2_CASE
    return fail(BLCO_ERR_INVALID, "wide MTTKRP: bad lane count");
}

// Mixed form: FP32 values and factors, four columns per lane (16-byte
// gathers), FP32 products summed in FP64 registers along a row's run and
// added to the FP32 output when the row changes.  L = lanes per nonzero
// (4 * L >= the columns of the slab, at most 128).
struct WideParams4 {
    const uint64_t* coords;
    const uint64_t* field;
    const float* vals;
    uint64_t nnz;
    Layout L;
    const float* fo[BLCO_MAX_MODES - 1];
    int other[BLCO_MAX_MODES - 1];
    void* out; // TO
    int mode;
    int rank;
    int col0;
};

template <int NM, int L, typename TO>
__global__ __launch_bounds__(WIDE_THREADS) void k_mttkrp_wide4(const WideParams4 p)
{
    constexpr int NO = NM - 1;
    const int lane = threadIdx.x & 31;
    const int sub = lane % L;
    const int grp = lane / L;
    constexpr uint64_t WARP_TASK = (uint64_t)32 * WIDE_BATCHES;
    const uint64_t nwarps = (uint64_t)gridDim.x * (WIDE_THREADS / 32);
    const uint64_t wid = (uint64_t)blockIdx.x * (WIDE_THREADS / 32) + (threadIdx.x >> 5);
    const int R = p.rank;
    const int col = p.col0 + 4 * sub;
    const bool cok = col < R; // col + 3 < R too: R is a multiple of 4
    const uint64_t ntasks = (p.nnz + WARP_TASK - 1) / WARP_TASK;
    for (uint64_t task = wid; task < ntasks; task += nwarps) {
        const uint64_t g0 = task * WARP_TASK + (uint64_t)grp * (L * WIDE_BATCHES);
        uint32_t cur = 0xffffffffu;
        double a[4] = {0.0, 0.0, 0.0, 0.0};
        auto flush = [&]() {
            if (cur != 0xffffffffu && cok) {
                TO* o = static_cast<TO*>(p.out) + (uint64_t)cur * R + col;
#pragma unroll
                for (int j = 0; j < 4; j++) atomicAdd(o + j, (TO)a[j]);
            }
        };
        for (int b = 0; b < WIDE_BATCHES; b++) {
            const uint64_t i = g0 + (uint64_t)b * L + sub;
            const bool ok = i < p.nnz;
            uint32_t rt = 0xffffffffu, ro[NO];
            float v = 0.f;
            {
                const uint64_t c = ok ? __ldg(p.coords + i) : 0;
                const uint64_t f = ok ? __ldg(p.field + i) : 0;
                v = ok ? __ldg(p.vals + i) : 0.f;
                if (ok) rt = (uint32_t)wide_row(p.L, p.mode, c, f);
#pragma unroll
                for (int k = 0; k < NO; k++) ro[k] = (uint32_t)wide_row(p.L, p.other[k], c, f);
            }
            constexpr int U = L >= 4 ? 4 : L;
#pragma unroll 1
            for (int j0 = 0; j0 < L; j0 += U) {
                uint32_t r[U];
                float vv[U];
                float4 x[U][NO];
#pragma unroll
                for (int u = 0; u < U; u++) {
                    r[u] = __shfl_sync(0xffffffffu, rt, j0 + u, L);
                    vv[u] = __shfl_sync(0xffffffffu, v, j0 + u, L);
#pragma unroll
                    for (int k = 0; k < NO; k++) {
                        const uint32_t rr = __shfl_sync(0xffffffffu, ro[k], j0 + u, L);
                        // rows of nonzeros past the end decode to row 0: in bounds
                        x[u][k] = cok ? __ldg(reinterpret_cast<const float4*>(p.fo[k] + ((uint64_t)rr * R + col)))
                                      : make_float4(0.f, 0.f, 0.f, 0.f);
                    }
                }
#pragma unroll
                for (int u = 0; u < U; u++) {
                    if (r[u] == 0xffffffffu) continue;
                    if (r[u] != cur) {
                        flush();
                        a[0] = a[1] = a[2] = a[3] = 0.0;
                        cur = r[u];
                    }
                    float q0 = vv[u], q1 = vv[u], q2 = vv[u], q3 = vv[u];
#pragma unroll
                    for (int k = 0; k < NO; k++) {
                        q0 *= x[u][k].x;
                        q1 *= x[u][k].y;
                        q2 *= x[u][k].z;
                        q3 *= x[u][k].w;
                    }
                    a[0] += (double)q0;
                    a[1] += (double)q1;
                    a[2] += (double)q2;
                    a[3] += (double)q3;
                }
            }
        }
        flush();
    }
}

template <int NM, typename TO>
int launch_wide4(const WideParams4& p, int grid, int lanes, cudaStream_t s)
{
    switch (lanes) {
    case 4: k_mttkrp_wide4<NM, 4, TO><<<grid, WIDE_THREADS, 0, s>>>(p); break;
    case 8: k_mttkrp_wide4<NM, 8, TO><<<grid, WIDE_THREADS, 0, s>>>(p); break;
    case 16: k_mttkrp_wide4<NM, 16, TO><<<grid, WIDE_THREADS, 0, s>>>(p); break;
    case 32: k_mttkrp_wide4<NM, 32, TO><<<grid, WIDE_THREADS, 0, s>>>(p); break;
    default: return fail(BLCO_ERR_INVALID, "wide MTTKRP: bad lane count");
    }
    BLCO_CHECK_LAUNCH("k_mttkrp_wide4");
    return BLCO_OK;
}

} // namespace

// FP32 copy of mode n's row-sorted values (wide keys, mixed form; made on
// first use).
static int wide_vals32(const blco_tensor* t, int n, cudaStream_t s, const float** out)
{
    blco_tensor::WideCopy& w = const_cast<blco_tensor::WideCopy&>(t->wide_copy[n]);
    if (!w.d_vals32) {
        BLCO_CUDA(cudaMalloc(&w.d_vals32, std::max<uint64_t>(1, t->nnz) * sizeof(float)));
        if (t->nnz) {
            k_to_f32<<<1024, 256, 0, s>>>(w.d_vals, w.d_vals32, t->nnz);
            BLCO_CHECK_LAUNCH("k_to_f32");
        }
    }
    *out = w.d_vals32;
    return BLCO_OK;
}

int mttkrp_wide_launch(const blco_tensor* t, const MttkrpArgs& a, cudaStream_t s)
{
    if (a.nnz == 0) return BLCO_OK;
    if (a.factor_dtype == BLCO_DTYPE_BF16)
        return fail(BLCO_ERR_UNSUPPORTED, "keys above 64 bits: FP64 or FP32 factors (no BF16 gathers)");
    const bool f32 = a.factor_dtype == BLCO_DTYPE_F32;
    const blco_tensor::WideCopy& w = t->wide_copy[a.mode];
    if (!t->resident || !w.d_coords) return fail(BLCO_ERR_STATE, "wide-key tensor without its per-mode copies");
    DeviceInfo di;
    BLCO_TRY(device_info(t->device, &di));
    WideParams p;
    memset(&p, 0, sizeof(p));
    p.coords = w.d_coords;
    p.field = w.d_field;
    if (f32) {
        const float* v32 = nullptr;
        BLCO_TRY(wide_vals32(t, a.mode, s, &v32));
        p.vals = v32;
    } else {
        p.vals = w.d_vals;
    }
    p.nnz = a.nnz;
    p.L = t->layout;
    for (int m = 0; m < t->layout.nmodes; m++) p.f[m] = a.factors[m];
    p.out = a.out;
    p.mode = a.mode;
    p.rank = a.rank;
    const uint64_t ntasks = (a.nnz + 32 * WIDE_BATCHES - 1) / (32 * WIDE_BATCHES);
    const int grid = (int)std::min<uint64_t>((ntasks + WIDE_THREADS / 32 - 1) / (WIDE_THREADS / 32),
                                             (uint64_t)di.sm_count * 8);
    if (f32) {
        bool quads = a.rank % 4 == 0 && ((uintptr_t)a.out & 15) == 0;
        for (int m = 0; m < t->layout.nmodes; m++)
            if (m != a.mode && ((uintptr_t)a.factors[m] & 15)) quads = false;
        const int nm = t->layout.nmodes;
        if (quads && nm >= 3) {
            WideParams4 q;
            memset(&q, 0, sizeof(q));
            q.coords = p.coords;
            q.field = p.field;
            q.vals = static_cast<const float*>(p.vals);
            q.nnz = p.nnz;
            q.L = p.L;
            q.out = a.out;
            q.mode = a.mode;
            q.rank = a.rank;
            for (int m = 0, k = 0; m < nm; m++)
                if (m != a.mode) {
                    q.fo[k] = static_cast<const float*>(a.factors[m]);
                    q.other[k++] = m;
                }
            for (int c0 = 0; c0 < a.rank; c0 += 128) {
                q.col0 = c0;
                const int cols = std::min(128, a.rank - c0);
                const int lanes = cols <= 16 ? 4 : cols <= 32 ? 8 : cols <= 64 ? 16 : 32;
                int st;
                if (a.out64) {
                    if (nm == 3) st = launch_wide4<3, double>(q, grid, lanes, s);
                    else if (nm == 4) st = launch_wide4<4, double>(q, grid, lanes, s);
                    else st = launch_wide4<5, double>(q, grid, lanes, s);
                } else {
                    if (nm == 3) st = launch_wide4<3, float>(q, grid, lanes, s);
                    else if (nm == 4) st = launch_wide4<4, float>(q, grid, lanes, s);
                    else st = launch_wide4<5, float>(q, grid, lanes, s);
                }
                if (st != BLCO_OK) return st;
            }
            return BLCO_OK;
        }
        for (int c0 = 0; c0 < a.rank; c0 += 128) {
            p.col0 = c0;
            const int cols = std::min(128, a.rank - c0);
            if (a.out64) {
                if (a.rank <= 8) k_mttkrp_wide<float, double, 8, 1><<<grid, WIDE_THREADS, 0, s>>>(p);
                else if (a.rank <= 16) k_mttkrp_wide<float, double, 16, 1><<<grid, WIDE_THREADS, 0, s>>>(p);
                else if (cols <= 32) k_mttkrp_wide<float, double, 32, 1><<<grid, WIDE_THREADS, 0, s>>>(p);
                else if (cols <= 64) k_mttkrp_wide<float, double, 32, 2><<<grid, WIDE_THREADS, 0, s>>>(p);
                else k_mttkrp_wide<float, double, 32, 4><<<grid, WIDE_THREADS, 0, s>>>(p);
            } else {
                if (a.rank <= 8) k_mttkrp_wide<float, float, 8, 1><<<grid, WIDE_THREADS, 0, s>>>(p);
                else if (a.rank <= 16) k_mttkrp_wide<float, float, 16, 1><<<grid, WIDE_THREADS, 0, s>>>(p);
                else if (cols <= 32) k_mttkrp_wide<float, float, 32, 1><<<grid, WIDE_THREADS, 0, s>>>(p);
                else if (cols <= 64) k_mttkrp_wide<float, float, 32, 2><<<grid, WIDE_THREADS, 0, s>>>(p);
                else k_mttkrp_wide<float, float, 32, 4><<<grid, WIDE_THREADS, 0, s>>>(p);
            }
            BLCO_CHECK_LAUNCH("k_mttkrp_wide");
        }
        return BLCO_OK;
    }
    // two columns per lane when every factor row starts on 16 bytes
    bool pairs = a.rank % 2 == 0 && ((uintptr_t)a.out & 15) == 0;
    uint64_t maxdim = 0;
    for (int m = 0; m < t->layout.nmodes; m++) {
        if (m != a.mode && ((uintptr_t)a.factors[m] & 15)) pairs = false;
        maxdim = std::max(maxdim, t->layout.dims[m]);
    }
    const int nm = t->layout.nmodes;
    if (pairs && nm >= 3) {
        WideParams2 q;
        memset(&q, 0, sizeof(q));
        q.coords = p.coords;
        q.field = p.field;
        q.vals = static_cast<const double*>(p.vals);
        q.nnz = p.nnz;
        q.L = p.L;
        q.out = static_cast<double*>(p.out);
        q.mode = p.mode;
        q.rank = p.rank;
        for (int m = 0, k = 0; m < nm; m++)
            if (m != a.mode) {
                q.fo[k] = static_cast<const double*>(p.f[m]);
                q.other[k++] = m;
            }
        const bool off32 = maxdim * (uint64_t)a.rank < (1ull << 32);
        for (int c0 = 0; c0 < a.rank; c0 += 64) {
            q.col0 = c0;
            const int cols = std::min(64, a.rank - c0);
            const int lanes = cols <= 8 ? 4 : cols <= 16 ? 8 : cols <= 32 ? 16 : 32;
            int st;
            if (nm == 3) st = launch_wide2<3>(q, grid, lanes, off32, s);
            else if (nm == 4) st = launch_wide2<4>(q, grid, lanes, off32, s);
            else st = launch_wide2<5>(q, grid, lanes, off32, s);
            if (st != BLCO_OK) return st;
        }
        return BLCO_OK;
    }
    for (int c0 = 0; c0 < a.rank; c0 += 128) {
        p.col0 = c0;
        const int cols = std::min(128, a.rank - c0);
        if (a.rank <= 8) k_mttkrp_wide<double, double, 8, 1><<<grid, WIDE_THREADS, 0, s>>>(p);
        else if (a.rank <= 16) k_mttkrp_wide<double, double, 16, 1><<<grid, WIDE_THREADS, 0, s>>>(p);
        else if (cols <= 32) k_mttkrp_wide<double, double, 32, 1><<<grid, WIDE_THREADS, 0, s>>>(p);
        else if (cols <= 64) k_mttkrp_wide<double, double, 32, 2><<<grid, WIDE_THREADS, 0, s>>>(p);
        else k_mttkrp_wide<double, double, 32, 4><<<grid, WIDE_THREADS, 0, s>>>(p);
        BLCO_CHECK_LAUNCH("k_mttkrp_wide");
    }
    return BLCO_OK;
}

int mttkrp_launch(const blco_tensor* t, const MttkrpArgs& a, cudaStream_t s)
{
    const Layout& L = t->layout;
    if (L.wide) {
        if (a.rank < 1 || a.rank > 256) return fail(BLCO_ERR_UNSUPPORTED, "rank must be 1..256");
        return mttkrp_wide_launch(t, a, s);
    }
    if (a.nnz == 0) return BLCO_OK;
    if (a.rank < 1 || a.rank > 256) return fail(BLCO_ERR_UNSUPPORTED, "rank must be 1..256");
    if (fibre_route(t, a)) return mttkrp_fibre_launch(const_cast<blco_tensor*>(t), a, s);
    if (a.factor_dtype != BLCO_DTYPE_F64 && a.factor_dtype != BLCO_DTYPE_F32 && a.factor_dtype != BLCO_DTYPE_BF16)
        return fail(BLCO_ERR_INVALID, "unknown factor dtype");
    DeviceInfo di;
    BLCO_TRY(device_info(t->device, &di));
    MtParams p;
    memset(&p, 0, sizeof(p));
    p.coords = a.coords;
    p.vals = a.vals;
    p.nnz = a.nnz;
    for (int m = 0; m < L.nmodes; m++) {
        p.f[m] = a.factors[m];
        p.mask[m] = L.mode_masks[m];
        p.pos[m] = L.mode_pos[m];
    }
    p.out = a.out;
    p.mode = a.mode;
    p.rank = a.rank;
    p.merge = 1;
    p.interleave = a.interleave;
    const size_t accb = acc_elem_bytes(a.factor_dtype);
    int kern = mttkrp_select_kernel(t, a.mode, a.rank, a.kernel, a.factor_dtype);
    if (kern == BLCO_KERNEL_FIBRE) // the fibre copy does not serve this call (alignment or a streamed block)
        kern = t->hot[a.mode].nhot > 0 && t->hot[a.mode].hot_nnz >= AUTO_HOT_MIN_NNZ ? BLCO_KERNEL_LVL2
                                                                                      : BLCO_KERNEL_LVL1;
    // the automatic rule deals the cold tiles round-robin when heavy rows
    // are split off (a few percent faster in sweeps)
    if (a.kernel == BLCO_KERNEL_AUTO && kern == BLCO_KERNEL_LVL2) p.interleave = 1;
    const size_t stage = stage_bytes(a.rank, policy_vec(a.factor_dtype));
    const HotTable& ht = t->hot[a.mode];
    // The vectorised kernels load 16 bytes at a time: every factor must start
    // on a 16-byte boundary (and the FP32 output on 16 bytes for the vector
    // atomics), otherwise take the scalar kernel.
    bool aligned16 = ((uintptr_t)a.out & 15u) == 0;
    for (int m = 0; m < L.nmodes; m++)
        if (m != a.mode && ((uintptr_t)a.factors[m] & 15u) != 0) aligned16 = false;
    size_t hash_bytes = 0;
    HotFn hot_fn = nullptr;
    if (kern == BLCO_KERNEL_LVL2 && ht.nhot > 0 && !ht.d_hcoords && aligned16 && a.coords == t->d_coords)
        BLCO_TRY(build_mode_copies(const_cast<blco_tensor*>(t), a.mode, s)); // first use
    if (kern == BLCO_KERNEL_LVL2 && ht.nhot > 0 && ht.d_hcoords && aligned16 && a.coords == t->d_coords) {
        switch (a.factor_dtype) {
        case BLCO_DTYPE_F64: hot_fn = pick_hot<PolicyF64>(L.nmodes, a.rank); break;
        case BLCO_DTYPE_F32: hot_fn = pick_hot<PolicyF32>(L.nmodes, a.rank); break;
        default: hot_fn = pick_hot<PolicyBF16>(L.nmodes, a.rank); break;
        }
    }
    if (kern == BLCO_KERNEL_LVL3) {
        p.direct = 1;
    } else if (hot_fn) {
        // Hot rows go to the CSR kernel; the tile kernel runs on the mode's
        // cold stream copy with global atomics only.
        HotTable& hm = const_cast<HotTable&>(ht);
        p.coords = ht.d_ccoords;
        p.nnz = ht.cold_nnz;
        if (a.factor_dtype == BLCO_DTYPE_F64) {
            p.vals = ht.d_cvals;
        } else {
            if (!hm.d_cvals32 && ht.cold_nnz) {
                BLCO_CUDA(cudaMalloc(&hm.d_cvals32, ht.cold_nnz * sizeof(float)));
                k_to_f32<<<1024, 256, 0, s>>>(ht.d_cvals, hm.d_cvals32, ht.cold_nnz);
                BLCO_CHECK_LAUNCH("k_to_f32");
            }
            p.vals = hm.d_cvals32;
        }
    } else if (kern == BLCO_KERNEL_LVL2 && ht.nhot > 0) {
        p.hot_keys = ht.d_keys;
        p.hot_slot = ht.d_slot;
        p.hot_rows = ht.d_rows;
        p.hash_size = ht.hash_size;
        hash_bytes = 2 * sizeof(uint32_t) * ht.hash_size;
        size_t avail = di.smem_optin - stage - hash_bytes - 1024;
        size_t fit = avail / (accb * a.rank);
        p.nhot = (int)std::min<size_t>(fit, (size_t)ht.nhot);
        if (p.nhot == 0) p.hash_size = 0, hash_bytes = 0;
    } else if (kern == BLCO_KERNEL_ATOMIC) {
        p.merge = 0;
    }
    const size_t nacc = p.direct ? (size_t)L.dims[a.mode] : (size_t)p.nhot;
    p.nacc = (int)nacc;
    const size_t smem = hash_bytes + nacc * a.rank * accb + stage + 16;
    if (smem > di.smem_optin) return fail(BLCO_ERR_UNSUPPORTED, "MTTKRP shared memory plan exceeds the device limit");
    if (hot_fn) {
        HotTable& hm = const_cast<HotTable&>(ht);
        HotParams h;
        h.coords = ht.d_hcoords;
        h.ptr = ht.d_ptr;
        h.rows = ht.d_rows;
        h.nhot = ht.nhot;
        h.total = (uint32_t)ht.hot_nnz;
        h.chunk = a.hot_chunk > 0 ? (uint32_t)a.hot_chunk : auto_hot_chunk(ht.hot_nnz);
        h.acc = nullptr;
        if (a.factor_dtype == BLCO_DTYPE_F64) {
            h.vals = ht.d_hvals;
        } else {
            // Mixed form: FP32 copy of the hot values, FP64 per-slot sums.
            if (!hm.d_hvals32) {
                BLCO_CUDA(cudaMalloc(&hm.d_hvals32, ht.hot_nnz * sizeof(float)));
                k_to_f32<<<1024, 256, 0, s>>>(ht.d_hvals, hm.d_hvals32, ht.hot_nnz);
                BLCO_CHECK_LAUNCH("k_to_f32");
            }
            if (hm.acc_rank < a.rank) {
                cudaFree(hm.d_acc);
                hm.d_acc = nullptr;
                BLCO_CUDA(cudaMalloc(&hm.d_acc, (size_t)ht.nhot * a.rank * sizeof(double)));
                hm.acc_rank = a.rank;
            }
            BLCO_CUDA(cudaMemsetAsync(hm.d_acc, 0, (size_t)ht.nhot * a.rank * sizeof(double), s));
            h.vals = hm.d_hvals32;
            h.acc = hm.d_acc;
        }
        const size_t hsmem = (size_t)(2 * ht.nhot + 1) * sizeof(uint32_t) + 16 + stage;
        BLCO_CUDA(cudaFuncSetAttribute((const void*)hot_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hsmem));
        const uint32_t nchunks = (h.total + h.chunk - 1) / h.chunk;
        const uint32_t hgrid = std::max<uint32_t>(1, std::min<uint32_t>(di.sm_count, nchunks));
        hot_fn<<<hgrid, MT_THREADS, hsmem, s>>>(p, h);
        BLCO_CHECK_LAUNCH("k_mttkrp_hot");
        if (h.acc) {
            k_merge_hot<<<std::max(1, std::min(1024, (ht.nhot * a.rank + 255) / 256)), 256, 0, s>>>(
                h.acc, ht.d_rows, ht.nhot, a.rank, reinterpret_cast<float*>(a.out));
            BLCO_CHECK_LAUNCH("k_merge_hot");
        }
    }
    if (p.nnz == 0) return BLCO_OK;
    KernelFn fn;
    switch (a.factor_dtype) {
    case BLCO_DTYPE_F64: fn = pick_kernel<PolicyF64>(L.nmodes, a.rank, aligned16); break;
    case BLCO_DTYPE_F32: fn = pick_kernel<PolicyF32>(L.nmodes, a.rank, aligned16); break;
    default: fn = pick_kernel<PolicyBF16>(L.nmodes, a.rank, aligned16); break;
    }
    BLCO_CUDA(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const uint64_t ntiles = (p.nnz + 31) / 32;
    uint64_t grid = std::min<uint64_t>((uint64_t)di.sm_count, (ntiles + MT_WARPS - 1) / MT_WARPS);
    if (grid < 1) grid = 1;
    p.tiles_per_cta = (ntiles + grid - 1) / grid;
    fn<<<(unsigned)grid, MT_THREADS, smem, s>>>(p);
    BLCO_CHECK_LAUNCH("k_mttkrp");
    return BLCO_OK;
}

// ------------------------------------------------------ streamed blocks --

struct StreamRing {
    int nbuf = 0;
    uint64_t B = 0;
    std::vector<uint64_t*> dc;
    std::vector<double*> dv;
    std::vector<cudaEvent_t> copied, consumed;
    cudaStream_t cs = nullptr;
};

uint64_t stream_ring_bytes(const StreamRing* r) { return r ? (uint64_t)r->nbuf * r->B * 16 : 0; }

int stream_ring_destroy(StreamRing* r)
{
    if (!r) return BLCO_OK;
    if (r->cs) cudaStreamSynchronize(r->cs);
    for (int i = 0; i < r->nbuf; i++) {
        if (r->consumed[i]) cudaEventSynchronize(r->consumed[i]);
        cudaFree(r->dc[i]);
        cudaFree(r->dv[i]);
        if (r->copied[i]) cudaEventDestroy(r->copied[i]);
        if (r->consumed[i]) cudaEventDestroy(r->consumed[i]);
    }
    if (r->cs) cudaStreamDestroy(r->cs);
    delete r;
    return BLCO_OK;
}

// A ring of device block buffers (at most residency_bytes of them, 8 GiB
// when 0; between 2 and 8 buffers) and a copy stream, for tensors whose
// blocks stay in pinned host memory.  Callers pass what the device budget
// leaves after their factors and workspace.
int stream_ring_create(const blco_tensor* t, uint64_t residency_bytes, StreamRing** out)
{
    *out = nullptr;
    StreamRing* r = new StreamRing();
    // Copies are block-sized, or smaller when two blocks would not fit the
    // budget: an MTTKRP over any contiguous range of a 64-bit stream is
    // valid (its block coordinates are zero), so the cap always holds.
    const uint64_t budget = residency_bytes ? residency_bytes : (8ull << 30);
    const uint64_t blk = t->max_block_size ? t->max_block_size : t->nnz;
    r->B = std::max<uint64_t>(1, std::min<uint64_t>(blk, budget / (2 * 16)));
    const uint64_t pieces = (t->nnz + r->B - 1) / r->B;
    int nbuf = (int)std::max<uint64_t>(2, std::min<uint64_t>(8, budget / (r->B * 16)));
    nbuf = (int)std::min<uint64_t>((uint64_t)nbuf, std::max<uint64_t>(1, pieces));
    r->nbuf = nbuf;
    r->dc.assign(nbuf, nullptr);
    r->dv.assign(nbuf, nullptr);
    r->copied.assign(nbuf, nullptr);
    r->consumed.assign(nbuf, nullptr);
    cudaError_t e = cudaStreamCreateWithFlags(&r->cs, cudaStreamNonBlocking);
    for (int i = 0; i < nbuf && e == cudaSuccess; i++) {
        e = cudaMalloc(&r->dc[i], std::max<uint64_t>(1, r->B) * 8);
        if (e == cudaSuccess) e = cudaMalloc(&r->dv[i], std::max<uint64_t>(1, r->B) * 8);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->copied[i], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->consumed[i], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        stream_ring_destroy(r);
        return cuda_fail(e, "streamed block ring", __FILE__, __LINE__);
    }
    *out = r;
    return BLCO_OK;
}

// One MTTKRP over every piece of the stream (a block, or a budget-sized
// part of one): piece b is copied into buffer b % nbuf on the copy stream
// (after the kernel that used that buffer before), and its MTTKRP runs on s
// after the copy.
int mttkrp_streamed_ring(const blco_tensor* t, const MttkrpArgs& base, StreamRing* r, cudaStream_t s)
{
    const bool f32 = base.factor_dtype != BLCO_DTYPE_F64;
    if (f32 && !t->h_values32) return fail(BLCO_ERR_STATE, "streamed mixed form without FP32 host values");
    // the copies must not overtake work already queued on s
    BLCO_CUDA(cudaEventRecord(r->consumed[0], s));
    BLCO_CUDA(cudaStreamWaitEvent(r->cs, r->consumed[0], 0));
    const uint64_t pieces = (t->nnz + r->B - 1) / r->B;
    for (uint64_t b = 0; b < pieces; b++) {
        const int k = (int)(b % r->nbuf);
        const uint64_t beg = b * r->B, n = std::min(r->B, t->nnz - beg);
        if (b >= (uint64_t)r->nbuf) BLCO_CUDA(cudaStreamWaitEvent(r->cs, r->consumed[k], 0));
        BLCO_CUDA(cudaMemcpyAsync(r->dc[k], t->h_coords + beg, n * 8, cudaMemcpyHostToDevice, r->cs));
        if (f32)  // the mixed forms stream 4-byte values
            BLCO_CUDA(cudaMemcpyAsync(r->dv[k], t->h_values32 + beg, n * 4, cudaMemcpyHostToDevice, r->cs));
        else
            BLCO_CUDA(cudaMemcpyAsync(r->dv[k], t->h_values + beg, n * 8, cudaMemcpyHostToDevice, r->cs));
        BLCO_CUDA(cudaEventRecord(r->copied[k], r->cs));
        BLCO_CUDA(cudaStreamWaitEvent(s, r->copied[k], 0));
        MttkrpArgs a = base;
        a.coords = r->dc[k];
        a.vals = r->dv[k];
        a.nnz = n;
        BLCO_TRY(mttkrp_launch(t, a, s));
        BLCO_CUDA(cudaEventRecord(r->consumed[k], s));
    }
    return BLCO_OK;
}

} // namespace blco
