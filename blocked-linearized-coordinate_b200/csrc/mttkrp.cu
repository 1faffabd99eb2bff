// mttkrp.cu -- sparse MTTKRP over the 64-bit BLCO stream (plain FP64 form).
//
//   out[r_t(i), :] += val_i * prod_{m != t} U_m[r_m(i), :]
//
// The reference computes this with one-warp CTAs over 32-nonzero tiles
// (mttkrp_lvl1/lvl2/lvl3/atomic, src/alto_dev.cu:31-1847).  This file keeps
// the tile-level conflict resolution idea but is laid out for B200:
//   * persistent CTAs, one per SM (grid = SM count), each owning one
//     contiguous slice of the ALTO-ordered stream, 24 warps per CTA;
//   * a warp takes 32 nonzeros, decodes rows with shifts and masks
//     (alt_pext, src/alto_dev.cu:13-16), groups equal output rows with
//     __match_any_sync and orders the tile by group (counting sort in
//     registers + a per-warp shared staging area);
//   * factor rows are gathered with 128-bit loads: R/2 lanes per nonzero,
//     two FP64 columns per lane, several nonzeros in flight per warp;
//   * runs of equal output rows are summed in registers and flushed once:
//     into a shared-memory accumulator when the row is one of the mode's
//     heaviest rows (a per-CTA privatised copy, written back once per CTA),
//     or into the whole output when the mode is short enough to fit
//     (the lvl3 role), otherwise with FP64 global atomics (red.global).
#include <algorithm>
#include <cstring>

#include "internal.cuh"

namespace blco {
namespace {

constexpr int MT_THREADS = 768; // 24 warps, one CTA per SM
constexpr int MT_WARPS = MT_THREADS / 32;
constexpr int MT_UNROLL = 4;

struct MtParams {
    const uint64_t* coords;
    const double* vals;
    uint64_t nnz;
    const double* f[BLCO_MAX_MODES];
    double* out;
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
    uint64_t tiles_per_cta;
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

// Shared memory: [hash keys | hash slots] [accumulator nhot x R doubles]
// [per-warp staging].
template <int NM>
struct Stage {
    uint32_t row[32];
    uint32_t oth[NM > 1 ? NM - 1 : 1][32];
    double val[32];
};

// Per-thread copy of the target/other mode fields, resolved once with
// compile-time indices so the hot loop keeps them in registers.
template <int NM>
struct ModeSel {
    static constexpr int NO = NM > 1 ? NM - 1 : 1;
    int tpos;
    uint64_t tmask;
    int opos[NO];
    uint64_t omask[NO];
    const double* of[NO];

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

// Sorts the warp's tile by output row into the staging area.  Returns the
// number of valid entries and the bitmask of positions that end a run.
template <int NM>
__device__ __forceinline__ int stage_tile(const MtParams& p, const ModeSel<NM>& ms, uint64_t i0, Stage<NM>* st,
                                          uint32_t& ends)
{
    const int lane = threadIdx.x & 31;
    const uint64_t i = i0 + lane;
    const bool valid = i < p.nnz;
    uint64_t c = valid ? __ldcs(p.coords + i) : 0;
    double v = valid ? __ldcs(p.vals + i) : 0.0;
    uint32_t rt = (uint32_t)((c >> ms.tpos) & ms.tmask);
    uint32_t ro[ModeSel<NM>::NO];
#pragma unroll
    for (int k = 0; k < NM - 1; k++) ro[k] = (uint32_t)((c >> ms.opos[k]) & ms.omask[k]);
    uint32_t key = valid ? rt : 0xffffffffu;
    uint32_t peers = __match_any_sync(0xffffffffu, key);
    const uint32_t lt = (1u << lane) - 1;
    int leader = __ffs(peers) - 1;
    uint32_t x = lane == leader ? (uint32_t)__popc(peers) : 0u;
    uint32_t inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    uint32_t start = __shfl_sync(0xffffffffu, inc - x, leader);
    int sp = (int)start + __popc(peers & lt);
    bool last = (peers >> lane) == 1u;
    ends = __reduce_or_sync(0xffffffffu, last ? (1u << sp) : 0u);
    st->row[sp] = rt;
#pragma unroll
    for (int k = 0; k < NM - 1; k++) st->oth[k][sp] = ro[k];
    st->val[sp] = v;
    __syncwarp();
    uint64_t rem = p.nnz - i0;
    return rem >= 32 ? 32 : (int)rem;
}

template <int R>
__device__ __forceinline__ void flush2(const MtParams& p, double* sacc, const uint32_t* skeys,
                                       const uint32_t* sslot, uint32_t row, int q, double2 a)
{
    int s = hot_lookup(p, skeys, sslot, row);
    if (s >= 0) {
        atomicAdd(sacc + (size_t)s * R + 2 * q, a.x);
        atomicAdd(sacc + (size_t)s * R + 2 * q + 1, a.y);
    } else {
        double* o = p.out + (size_t)row * R + 2 * q;
        atomicAdd(o, a.x);
        atomicAdd(o + 1, a.y);
    }
}

// Vectorised kernel: R in {2,4,...,64}; LPN = R/2 lanes per nonzero, each
// lane two columns.
template <int NM, int R>
__global__ void __launch_bounds__(MT_THREADS, 1) k_mttkrp_vec(MtParams p)
{
    constexpr int LPN = R / 2;
    constexpr int SLOTS = 32 / LPN;
    constexpr int PER = 32 / SLOTS;
    extern __shared__ __align__(16) unsigned char smem[];
    uint32_t* skeys = reinterpret_cast<uint32_t*>(smem);
    uint32_t* sslot = skeys + p.hash_size;
    double* sacc = reinterpret_cast<double*>(sslot + p.hash_size + ((2 * p.hash_size) & 1));
    const int nacc = p.nacc;
    Stage<NM>* stages = reinterpret_cast<Stage<NM>*>(sacc + (size_t)nacc * R);

    for (int i = threadIdx.x; i < p.hash_size; i += blockDim.x) {
        skeys[i] = p.hot_keys[i];
        sslot[i] = p.hot_slot[i];
    }
    for (size_t i = threadIdx.x; i < (size_t)nacc * R; i += blockDim.x) sacc[i] = 0.0;
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int slot = lane / LPN, q = lane % LPN;
    Stage<NM>* st = stages + warp;
    const uint64_t ntiles = (p.nnz + 31) / 32;
    const uint64_t t_beg = (uint64_t)blockIdx.x * p.tiles_per_cta;
    const uint64_t t_end = min(ntiles, t_beg + p.tiles_per_cta);
    const ModeSel<NM> ms(p);
    const double2* fv[ModeSel<NM>::NO];
#pragma unroll
    for (int k = 0; k < NM - 1; k++) fv[k] = reinterpret_cast<const double2*>(ms.of[k]);

    for (uint64_t tile = t_beg + warp; tile < t_end; tile += MT_WARPS) {
        uint32_t ends;
        const int count = stage_tile<NM>(p, ms, tile * 32, st, ends);
        if (!p.merge) ends = 0xffffffffu;
        const int pb = slot * PER, pe = min(pb + PER, count);
        double2 acc = make_double2(0.0, 0.0);
        for (int p0 = pb; p0 < pe; p0 += MT_UNROLL) {
            double2 g[MT_UNROLL][ModeSel<NM>::NO];
            double vv[MT_UNROLL];
#pragma unroll
            for (int u = 0; u < MT_UNROLL; u++) {
                int pp = p0 + u;
                if (pp < pe) {
                    vv[u] = st->val[pp];
#pragma unroll
                    for (int k = 0; k < NM - 1; k++)
                        g[u][k] = __ldg(fv[k] + (size_t)st->oth[k][pp] * LPN + q);
                }
            }
#pragma unroll
            for (int u = 0; u < MT_UNROLL; u++) {
                int pp = p0 + u;
                if (pp < pe) {
                    double2 prod = make_double2(vv[u], vv[u]);
#pragma unroll
                    for (int k = 0; k < NM - 1; k++) {
                        prod.x *= g[u][k].x;
                        prod.y *= g[u][k].y;
                    }
                    acc.x += prod.x;
                    acc.y += prod.y;
                    if (((ends >> pp) & 1u) || pp == pe - 1) {
                        flush2<R>(p, sacc, skeys, sslot, st->row[pp], q, acc);
                        acc = make_double2(0.0, 0.0);
                    }
                }
            }
        }
        __syncwarp();
    }
    __syncthreads();
    // Write the privatised rows back once.
    for (size_t i = threadIdx.x; i < (size_t)nacc * R; i += blockDim.x) {
        double v = sacc[i];
        if (v != 0.0) {
            size_t s = i / R;
            uint32_t row = p.direct ? (uint32_t)s : p.hot_rows[s];
            atomicAdd(p.out + (size_t)row * R + (i % R), v);
        }
    }
}

// Generic kernel: any R up to 256, a whole warp per nonzero, columns
// lane, lane+32, ...
constexpr int GEN_MAXC = 8;

template <int NM>
__global__ void __launch_bounds__(MT_THREADS, 1) k_mttkrp_gen(MtParams p)
{
    extern __shared__ __align__(16) unsigned char smem[];
    uint32_t* skeys = reinterpret_cast<uint32_t*>(smem);
    uint32_t* sslot = skeys + p.hash_size;
    double* sacc = reinterpret_cast<double*>(sslot + p.hash_size + ((2 * p.hash_size) & 1));
    const int R = p.rank;
    const int nacc = p.nacc;
    Stage<NM>* stages = reinterpret_cast<Stage<NM>*>(sacc + (size_t)nacc * R);
    for (int i = threadIdx.x; i < p.hash_size; i += blockDim.x) {
        skeys[i] = p.hot_keys[i];
        sslot[i] = p.hot_slot[i];
    }
    for (size_t i = threadIdx.x; i < (size_t)nacc * R; i += blockDim.x) sacc[i] = 0.0;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Stage<NM>* st = stages + warp;
    const uint64_t ntiles = (p.nnz + 31) / 32;
    const uint64_t t_beg = (uint64_t)blockIdx.x * p.tiles_per_cta;
    const uint64_t t_end = min(ntiles, t_beg + p.tiles_per_cta);
    const ModeSel<NM> ms(p);
    const int ncol = (R + 31) / 32;
    for (uint64_t tile = t_beg + warp; tile < t_end; tile += MT_WARPS) {
        uint32_t ends;
        const int count = stage_tile<NM>(p, ms, tile * 32, st, ends);
        if (!p.merge) ends = 0xffffffffu;
        double acc[GEN_MAXC];
#pragma unroll
        for (int j = 0; j < GEN_MAXC; j++) acc[j] = 0.0;
        for (int pp = 0; pp < count; pp++) {
            const double v = st->val[pp];
#pragma unroll
            for (int j = 0; j < GEN_MAXC; j++) {
                int c = lane + 32 * j;
                if (j < ncol && c < R) {
                    double prod = v;
#pragma unroll
                    for (int k = 0; k < NM - 1; k++) prod *= __ldg(ms.of[k] + (size_t)st->oth[k][pp] * R + c);
                    acc[j] += prod;
                }
            }
            if (((ends >> pp) & 1u) || pp == count - 1) {
                const uint32_t row = st->row[pp];
                int s = hot_lookup(p, skeys, sslot, row);
#pragma unroll
                for (int j = 0; j < GEN_MAXC; j++) {
                    int c = lane + 32 * j;
                    if (j < ncol && c < R) {
                        if (s >= 0) atomicAdd(sacc + (size_t)s * R + c, acc[j]);
                        else atomicAdd(p.out + (size_t)row * R + c, acc[j]);
                    }
                    acc[j] = 0.0;
                }
            }
        }
        __syncwarp();
    }
    __syncthreads();
    for (size_t i = threadIdx.x; i < (size_t)nacc * R; i += blockDim.x) {
        double v = sacc[i];
        if (v != 0.0) {
            size_t s = i / R;
            uint32_t row = p.direct ? (uint32_t)s : p.hot_rows[s];
            atomicAdd(p.out + (size_t)row * R + (i % R), v);
        }
    }
}

template <int NM>
size_t stage_bytes() { return sizeof(Stage<NM>) * MT_WARPS; }

size_t stage_bytes_rt(int nm)
{
    switch (nm) {
    case 1: return stage_bytes<1>();
    case 2: return stage_bytes<2>();
    case 3: return stage_bytes<3>();
    case 4: return stage_bytes<4>();
    default: return stage_bytes<5>();
    }
}

typedef void (*KernelFn)(MtParams);

template <int NM>
KernelFn pick_vec(int R)
{
    switch (R) {
    case 2: return k_mttkrp_vec<NM, 2>;
    case 4: return k_mttkrp_vec<NM, 4>;
    case 8: return k_mttkrp_vec<NM, 8>;
    case 16: return k_mttkrp_vec<NM, 16>;
    case 32: return k_mttkrp_vec<NM, 32>;
    case 64: return k_mttkrp_vec<NM, 64>;
    default: return nullptr;
    }
}

KernelFn pick_generic(int nm)
{
    switch (nm) {
    case 1: return k_mttkrp_gen<1>;
    case 2: return k_mttkrp_gen<2>;
    case 3: return k_mttkrp_gen<3>;
    case 4: return k_mttkrp_gen<4>;
    default: return k_mttkrp_gen<5>;
    }
}

KernelFn pick_kernel(int nm, int R)
{
    KernelFn f = nullptr;
    switch (nm) {
    case 1: f = pick_vec<1>(R); break;
    case 2: f = pick_vec<2>(R); break;
    case 3: f = pick_vec<3>(R); break;
    case 4: f = pick_vec<4>(R); break;
    case 5: f = pick_vec<5>(R); break;
    }
    return f ? f : pick_generic(nm);
}

} // namespace

int mttkrp_select_kernel(const blco_tensor* t, int mode, int rank, int requested)
{
    DeviceInfo di;
    if (device_info(t->device, &di) != BLCO_OK) return BLCO_KERNEL_LVL1;
    size_t budget = di.smem_optin - stage_bytes_rt(t->layout.nmodes) - 2 * sizeof(uint32_t) * 4096 - 1024;
    bool fits_direct = t->layout.dims[mode] * (uint64_t)rank * sizeof(double) <= budget;
    switch (requested) {
    case BLCO_KERNEL_LVL1:
    case BLCO_KERNEL_BATCHED:
    case BLCO_KERNEL_BATCHED_V2: return BLCO_KERNEL_LVL1;
    case BLCO_KERNEL_LVL2: return BLCO_KERNEL_LVL2;
    case BLCO_KERNEL_LVL3: return fits_direct ? BLCO_KERNEL_LVL3 : BLCO_KERNEL_LVL2;
    case BLCO_KERNEL_ATOMIC: return BLCO_KERNEL_ATOMIC;
    default:
        if (fits_direct) return BLCO_KERNEL_LVL3;
        return t->hot[mode].nhot > 0 ? BLCO_KERNEL_LVL2 : BLCO_KERNEL_LVL1;
    }
}

int mttkrp_launch(const blco_tensor* t, const MttkrpArgs& a, cudaStream_t s)
{
    const Layout& L = t->layout;
    if (a.nnz == 0) return BLCO_OK;
    if (a.rank < 1 || a.rank > 256) return fail(BLCO_ERR_UNSUPPORTED, "rank must be 1..256");
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
    const int kern = mttkrp_select_kernel(t, a.mode, a.rank, a.kernel);
    const size_t stage = stage_bytes_rt(L.nmodes);
    const HotTable& ht = t->hot[a.mode];
    size_t hash_bytes = 0;
    if (kern == BLCO_KERNEL_LVL3) {
        p.direct = 1;
    } else if (kern == BLCO_KERNEL_LVL2 && ht.nhot > 0) {
        p.hot_keys = ht.d_keys;
        p.hot_slot = ht.d_slot;
        p.hot_rows = ht.d_rows;
        p.hash_size = ht.hash_size;
        hash_bytes = 2 * sizeof(uint32_t) * ht.hash_size + 8;
        size_t avail = di.smem_optin - stage - hash_bytes - 1024;
        size_t fit = avail / (sizeof(double) * a.rank);
        p.nhot = (int)std::min<size_t>(fit, (size_t)ht.nhot);
        if (p.nhot == 0) p.hash_size = 0, hash_bytes = 0;
    } else if (kern == BLCO_KERNEL_ATOMIC) {
        p.merge = 0;
    }
    const size_t nacc = p.direct ? (size_t)L.dims[a.mode] : (size_t)p.nhot;
    p.nacc = (int)nacc;
    const size_t smem = hash_bytes + nacc * a.rank * sizeof(double) + stage + 16;
    if (smem > di.smem_optin) return fail(BLCO_ERR_UNSUPPORTED, "MTTKRP shared memory plan exceeds the device limit");
    // The vectorised kernels load two FP64 columns at a time: every factor
    // must start on a 16-byte boundary, otherwise take the scalar kernel.
    bool aligned16 = true;
    for (int m = 0; m < L.nmodes; m++)
        if (m != a.mode && ((uintptr_t)a.factors[m] & 15u) != 0) aligned16 = false;
    KernelFn fn = aligned16 ? pick_kernel(L.nmodes, a.rank) : pick_generic(L.nmodes);
    BLCO_CUDA(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const uint64_t ntiles = (a.nnz + 31) / 32;
    uint64_t grid = std::min<uint64_t>((uint64_t)di.sm_count, (ntiles + MT_WARPS - 1) / MT_WARPS);
    if (grid < 1) grid = 1;
    p.tiles_per_cta = (ntiles + grid - 1) / grid;
    fn<<<(unsigned)grid, MT_THREADS, smem, s>>>(p);
    BLCO_CHECK_LAUNCH("k_mttkrp");
    return BLCO_OK;
}

} // namespace blco
