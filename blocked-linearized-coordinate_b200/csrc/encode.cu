// encode.cu -- BLCO encoder on the GPU.
//
// Reproduces gen_blcotensor_host<uint64> (include/blco.hpp:196-331), which
// runs gen_alto (include/alto.hpp:107-186) and sort_alto
// (include/alto.hpp:704-754) on the host, as four device phases:
//   1. linearize: key_i = OR_n pdep(c_n,i, alto_mask_n)      (k_alto_keys)
//   2. sort (key, value) pairs by key: stable LSD radix sort, 8-bit digits,
//      one pass per 8 significant key bits                   (k_rs_*)
//   3. re-linearize: coord_i = OR_n pext(key_i, alto_mask_n) << mode_pos_n,
//      fused into the last sort pass                         (k_rs_scatter)
//   4. block split: consecutive max_block_size slices (host arithmetic; the
//      upper key half is always zero for 64-bit keys, so every nonzero is in
//      histogram bucket 0, include/blco.hpp:249-321)
// Then per-mode row statistics and heavy-row tables for the MTTKRP kernels.
// Further sections: keys of 65-128 bits (the reference's 128-bit build,
// blocks with block coordinates), the chunked encode of streamed tensors
// larger than their residency budget, and the allocation-free encoder.
#include <algorithm>
#include <cstring>
#include <atomic>
#include <memory>
#include <mutex>
#include <new>
#include <thread>

#include "internal.cuh"

namespace blco {

int make_layout(int nmodes, const uint64_t* dims, Layout* L)
{
    if (nmodes < 1 || nmodes > BLCO_MAX_MODES) return fail(BLCO_ERR_INVALID, "nmodes must be 1..5");
    memset(L, 0, sizeof(*L));
    L->nmodes = nmodes;
    int bits[BLCO_MAX_MODES], order[BLCO_MAX_MODES];
    int total = 0, maxbits = 0;
    for (int n = 0; n < nmodes; n++) {
        if (dims[n] == 0) return fail(BLCO_ERR_INVALID, "mode length 0");
        if (dims[n] > 0xffffffffull) return fail(BLCO_ERR_UNSUPPORTED, "mode length above 2^32-1");
        L->dims[n] = dims[n];
        // 64 - clz(dim - 1) (include/alto.hpp:613); dim == 1 -> 0 bits.
        bits[n] = dims[n] <= 1 ? 0 : 64 - __builtin_clzll(dims[n] - 1);
        total += bits[n];
        maxbits = std::max(maxbits, bits[n]);
        order[n] = n;
    }
    // 128 bits is the widest key of the reference (ALTO_MASK_LENGTH=128,
    // include/alto.hpp:634).
    if (total > 128) return fail(BLCO_ERR_UNSUPPORTED, "coordinates need more than 128 key bits");
    // Shortest mode first, ties in natural order; LSB-first round robin over
    // bit levels (include/alto.hpp:659-685), positions 64..127 in the upper
    // key word.
    std::stable_sort(order, order + nmodes, [&](int a, int b) { return bits[a] < bits[b]; });
    int shift = 0;
    for (int level = 0; level < maxbits; level++)
        for (int k = 0; k < nmodes; k++)
            if (level < bits[order[k]]) {
                if (shift < 64) L->alto_masks[order[k]] |= 1ull << shift;
                else L->alto_masks_hi[order[k]] |= 1ull << (shift - 64);
                shift++;
            }
    // Fields of the low-word bits, include/blco.hpp:222-233 (all bits when
    // the key fits 64 bits); block fields of the rest.
    for (int n = 0; n < nmodes; n++) {
        const int lb = __builtin_popcountll(L->alto_masks[n]);
        const int hb = bits[n] - lb;
        L->low_bits[n] = lb;
        L->mode_masks[n] = lb >= 64 ? ~0ull : ((1ull << lb) - 1);
        L->mode_pos[n] = n == 0 ? 0 : L->mode_pos[n - 1] + L->low_bits[n - 1];
        L->bmask[n] = hb >= 64 ? ~0ull : ((1ull << hb) - 1);
        L->bpos[n] = n == 0 ? 0 : L->bpos[n - 1] + (bits[n - 1] - L->low_bits[n - 1]);
    }
    L->alto_bits = total;
    L->wide = total > 64;
    return BLCO_OK;
}

namespace {

struct CooPtrs {
    const uint64_t* c[BLCO_MAX_MODES];
};

// Byte tables for the bit permutations of the encoder:
//   dep[n][b][v] = pdep(v << 8b, alto_mask_n)            (coordinate -> key)
//   rel[b][v]    = relinearized field bits of (v << 8b)   (key -> BLCO coord)
// so a key is the OR of one lookup per coordinate byte and a BLCO coordinate
// the OR of one lookup per key byte.
struct EncTables {
    uint64_t dep[BLCO_MAX_MODES][4][256];
    uint64_t rel[8][256];
};

EncTables make_tables(const Layout& L)
{
    EncTables T;
    memset(&T, 0, sizeof(T));
    int mode_of[64], bit_of[64];
    for (int p = 0; p < 64; p++) mode_of[p] = -1;
    for (int n = 0; n < L.nmodes; n++) {
        int j = 0;
        for (int p = 0; p < 64; p++)
            if (L.alto_masks[n] >> p & 1) {
                mode_of[p] = n;
                bit_of[p] = j++;
            }
    }
    for (int n = 0; n < L.nmodes; n++)
        for (int b = 0; b < 4; b++)
            for (int v = 0; v < 256; v++) {
                uint64_t key = 0;
                for (int p = 0; p < 64; p++)
                    if (mode_of[p] == n && bit_of[p] >= 8 * b && bit_of[p] < 8 * b + 8 && (v >> (bit_of[p] - 8 * b) & 1))
                        key |= 1ull << p;
                T.dep[n][b][v] = key;
            }
    for (int b = 0; b < 8; b++)
        for (int v = 0; v < 256; v++) {
            uint64_t c = 0;
            for (int j = 0; j < 8; j++) {
                int p = 8 * b + j;
                if ((v >> j & 1) && mode_of[p] >= 0) c |= 1ull << (L.mode_pos[mode_of[p]] + bit_of[p]);
            }
            T.rel[b][v] = c;
        }
    return T;
}

__device__ __forceinline__ uint64_t relin(const uint64_t (*rel)[256], uint64_t key, int nbytes)
{
    uint64_t c = 0;
#pragma unroll
    for (int b = 0; b < 8; b++)
        if (b < nbytes) c |= rel[b][(key >> (8 * b)) & 255];
    return c;
}

// Re-linearization on its own, for streams the sort leaves untouched (a
// single nonzero).
__global__ void k_relin(uint64_t* __restrict__ keys, uint64_t n, const EncTables* __restrict__ tabs, int nbytes)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        keys[i] = relin(tabs->rel, keys[i], nbytes);
}

__global__ void k_alto_keys(CooPtrs coo, const double* __restrict__ vals, uint64_t nnz, Layout L,
                            const EncTables* __restrict__ tabs, uint64_t* __restrict__ keys,
                            double* __restrict__ vout, int* __restrict__ bad)
{
    __shared__ uint64_t dep[BLCO_MAX_MODES][4][256];
    for (int i = threadIdx.x; i < BLCO_MAX_MODES * 4 * 256; i += blockDim.x)
        (&dep[0][0][0])[i] = (&tabs->dep[0][0][0])[i];
    __syncthreads();
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nnz;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t key = 0;
        bool ok = true;
#pragma unroll
        for (int n = 0; n < BLCO_MAX_MODES; n++) {
            if (n < L.nmodes) {
                uint64_t c = coo.c[n][i];
                ok &= c < L.dims[n];
#pragma unroll
                for (int b = 0; b < 4; b++) key |= dep[n][b][(c >> (8 * b)) & 255];
            }
        }
        if (!ok) atomicExch(bad, 1);
        keys[i] = key;
        vout[i] = vals[i];
    }
}

// ----------------------------------------------------------- radix sort --

constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ITEMS = 8;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS; // 2048 keys per tile
constexpr int RS_RADIX = 256;
constexpr size_t RS_SMEM = RS_TILE * 16 + (RS_WARPS + 2) * RS_RADIX * 4 + 8 * 256 * 8;

// Per-tile digit counts, digit-major: counts[d * ntiles + tile].
__global__ __launch_bounds__(RS_THREADS) void k_rs_hist(const uint64_t* __restrict__ keys, uint64_t n, int shift,
                                                        uint32_t* __restrict__ counts, uint32_t ntiles)
{
    __shared__ uint32_t h[RS_RADIX];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * RS_TILE;
#pragma unroll 4
    for (int j = 0; j < RS_ITEMS; j++) {
        uint64_t idx = base + (uint64_t)j * RS_THREADS + threadIdx.x;
        uint32_t d = idx < n ? (uint32_t)((keys[idx] >> shift) & 255) : 256u;
        uint32_t peers = __match_any_sync(0xffffffffu, d);
        if (d < 256 && (peers & ((1u << (threadIdx.x & 31)) - 1)) == 0) atomicAdd(&h[d], (uint32_t)__popc(peers));
    }
    __syncthreads();
    counts[(uint64_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of a uint32 array in three kernels.
constexpr int SC_THREADS = 256;
constexpr int SC_ITEMS = 16;
constexpr int SC_CHUNK = SC_THREADS * SC_ITEMS;

__device__ __forceinline__ uint32_t block_excl_scan_256(uint32_t x, uint32_t* wsum, uint32_t* total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t z = lane < SC_THREADS / 32 ? wsum[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, z, o);
            if (lane >= o) z += y;
        }
        if (lane < SC_THREADS / 32) wsum[lane] = z;
    }
    __syncthreads();
    uint32_t excl = inc - x + (warp > 0 ? wsum[warp - 1] : 0);
    if (total) *total = wsum[SC_THREADS / 32 - 1];
    __syncthreads();
    return excl;
}

__global__ __launch_bounds__(SC_THREADS) void k_scan_sums(const uint32_t* __restrict__ a, uint64_t n,
                                                          uint32_t* __restrict__ sums)
{
    __shared__ uint32_t wsum[SC_THREADS / 32];
    uint64_t base = (uint64_t)blockIdx.x * SC_CHUNK + (uint64_t)threadIdx.x * SC_ITEMS;
    uint32_t s = 0;
#pragma unroll
    for (int j = 0; j < SC_ITEMS; j++)
        if (base + j < n) s += a[base + j];
    uint32_t total;
    block_excl_scan_256(s, wsum, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ __launch_bounds__(SC_THREADS) void k_scan_top(uint32_t* __restrict__ sums, uint32_t nb)
{
    __shared__ uint32_t wsum[SC_THREADS / 32];
    uint32_t carry = 0;
    for (uint32_t base = 0; base < nb; base += SC_THREADS) {
        uint32_t i = base + threadIdx.x;
        uint32_t x = i < nb ? sums[i] : 0;
        uint32_t total;
        uint32_t e = block_excl_scan_256(x, wsum, &total);
        if (i < nb) sums[i] = e + carry;
        carry += total;
    }
}

__global__ __launch_bounds__(SC_THREADS) void k_scan_apply(uint32_t* __restrict__ a, uint64_t n,
                                                           const uint32_t* __restrict__ sums)
{
    __shared__ uint32_t wsum[SC_THREADS / 32];
    uint64_t base = (uint64_t)blockIdx.x * SC_CHUNK + (uint64_t)threadIdx.x * SC_ITEMS;
    uint32_t v[SC_ITEMS];
    uint32_t s = 0;
#pragma unroll
    for (int j = 0; j < SC_ITEMS; j++) {
        v[j] = base + j < n ? a[base + j] : 0;
        s += v[j];
    }
    uint32_t run = block_excl_scan_256(s, wsum, nullptr) + sums[blockIdx.x];
#pragma unroll
    for (int j = 0; j < SC_ITEMS; j++) {
        if (base + j < n) a[base + j] = run;
        run += v[j];
    }
}

// Stable scatter of one radix pass.  Warp w of a tile owns the 512
// consecutive keys [tile*4096 + w*512, +512), read as 16 rounds of 32; the
// rank of a key is (digit start in tile) + (keys of that digit in earlier
// warps) + (earlier rounds and lower lanes of its own warp), which keeps the
// input order of equal digits.  The tile is reordered in shared memory and
// written out with per-digit global offsets.
// With rel != nullptr (last pass of the encoder sort) the keys are written
// out re-linearized into BLCO coordinates.
__global__ __launch_bounds__(RS_THREADS) void k_rs_scatter(const uint64_t* __restrict__ kin,
                                                           const double* __restrict__ vin,
                                                           uint64_t* __restrict__ kout, double* __restrict__ vout,
                                                           uint64_t n, int shift, const uint32_t* __restrict__ offsets,
                                                           uint32_t ntiles, const EncTables* __restrict__ rel_tabs,
                                                           int rel_bytes)
{
    extern __shared__ __align__(16) unsigned char rs_smem[];
    uint64_t* skeys = reinterpret_cast<uint64_t*>(rs_smem);
    double* svals = reinterpret_cast<double*>(skeys + RS_TILE);
    uint64_t(*rel)[256] = reinterpret_cast<uint64_t(*)[256]>(svals + RS_TILE);
    uint32_t* whist = reinterpret_cast<uint32_t*>(svals + RS_TILE + 8 * 256);
    uint32_t* tstart = whist + RS_WARPS * RS_RADIX;
    uint32_t* gbase = tstart + RS_RADIX;
    __shared__ uint32_t wsum[SC_THREADS / 32];
    if (rel_tabs)
        for (int i = threadIdx.x; i < 8 * 256; i += RS_THREADS) (&rel[0][0])[i] = (&rel_tabs->rel[0][0])[i];

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1;
    for (int i = threadIdx.x; i < RS_WARPS * RS_RADIX; i += RS_THREADS) whist[i] = 0;
    __syncthreads();

    const uint64_t tile_base = (uint64_t)blockIdx.x * RS_TILE;
    const uint64_t base = tile_base + (uint64_t)warp * (32 * RS_ITEMS);
    uint64_t k[RS_ITEMS];
    double v[RS_ITEMS];
    uint32_t lp[RS_ITEMS];
    uint32_t* wh = whist + warp * RS_RADIX;
#pragma unroll
    for (int j = 0; j < RS_ITEMS; j++) {
        uint64_t idx = base + (uint64_t)j * 32 + lane;
        bool ok = idx < n;
        k[j] = ok ? kin[idx] : 0;
        v[j] = ok ? vin[idx] : 0.0;
    }
#pragma unroll
    for (int j = 0; j < RS_ITEMS; j++) {
        uint64_t idx = base + (uint64_t)j * 32 + lane;
        uint32_t d = idx < n ? (uint32_t)((k[j] >> shift) & 255) : 256u;
        uint32_t peers = __match_any_sync(0xffffffffu, d);
        uint32_t prev = d < 256 ? wh[d] : 0;
        lp[j] = prev + __popc(peers & lt);
        __syncwarp();
        if (d < 256 && (peers & lt) == 0) wh[d] = prev + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    {
        const int d = threadIdx.x; // RS_THREADS == RS_RADIX
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < RS_WARPS; w++) {
            uint32_t c = whist[w * RS_RADIX + d];
            whist[w * RS_RADIX + d] = run;
            run += c;
        }
        gbase[d] = offsets[(uint64_t)d * ntiles + blockIdx.x];
        uint32_t ex = block_excl_scan_256(run, wsum, nullptr);
        tstart[d] = ex;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < RS_ITEMS; j++) {
        uint64_t idx = base + (uint64_t)j * 32 + lane;
        if (idx < n) {
            uint32_t d = (uint32_t)((k[j] >> shift) & 255);
            uint32_t sp = tstart[d] + wh[d] + lp[j];
            skeys[sp] = k[j];
            svals[sp] = v[j];
        }
    }
    __syncthreads();
    const uint32_t tile_n = (uint32_t)min((uint64_t)RS_TILE, n - tile_base);
    for (uint32_t i = threadIdx.x; i < tile_n; i += RS_THREADS) {
        uint64_t kk = skeys[i];
        uint32_t d = (uint32_t)((kk >> shift) & 255);
        uint64_t o = (uint64_t)gbase[d] + (i - tstart[d]);
        kout[o] = rel_tabs ? relin(rel, kk, rel_bytes) : kk;
        vout[o] = svals[i];
    }
}

int scan_u32(uint32_t* a, uint64_t n, uint32_t* sums, cudaStream_t s)
{
    uint32_t nb = (uint32_t)((n + SC_CHUNK - 1) / SC_CHUNK);
    k_scan_sums<<<nb, SC_THREADS, 0, s>>>(a, n, sums);
    BLCO_CHECK_LAUNCH("k_scan_sums");
    k_scan_top<<<1, SC_THREADS, 0, s>>>(sums, nb);
    BLCO_CHECK_LAUNCH("k_scan_top");
    k_scan_apply<<<nb, SC_THREADS, 0, s>>>(a, n, sums);
    BLCO_CHECK_LAUNCH("k_scan_apply");
    return BLCO_OK;
}

// Sorts (k0, v0) stably by key bits [begin_bit, end_bit); ping-pongs with
// (k1, v1).  *in_alt is set when the result ends up in (k1, v1).
int radix_sort_pairs(uint64_t* k0, double* v0, uint64_t* k1, double* v1, uint64_t n, int begin_bit, int end_bit,
                     cudaStream_t s, bool* in_alt, const EncTables* rel_tabs = nullptr)
{
    *in_alt = false;
    const int bits = end_bit;
    if (n <= 1 || end_bit <= begin_bit) return BLCO_OK;
    uint32_t ntiles = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
    uint64_t L = (uint64_t)RS_RADIX * ntiles;
    uint32_t nsums = (uint32_t)((L + SC_CHUNK - 1) / SC_CHUNK);
    uint32_t *counts = nullptr, *sums = nullptr;
    BLCO_CUDA(cudaMallocAsync(&counts, L * sizeof(uint32_t), s));
    BLCO_CUDA(cudaMallocAsync(&sums, (nsums + 1) * sizeof(uint32_t), s));
    BLCO_CUDA(cudaFuncSetAttribute(k_rs_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RS_SMEM));
    uint64_t *ki = k0, *ko = k1;
    double *vi = v0, *vo = v1;
    int st = BLCO_OK;
    for (int shift = begin_bit; shift < bits; shift += 8) {
        k_rs_hist<<<ntiles, RS_THREADS, 0, s>>>(ki, n, shift, counts, ntiles);
        count_launch();
        if ((st = scan_u32(counts, L, sums, s)) != BLCO_OK) break;
        const bool last = shift + 8 >= bits;
        k_rs_scatter<<<ntiles, RS_THREADS, RS_SMEM, s>>>(ki, vi, ko, vo, n, shift, counts, ntiles,
                                                         last ? rel_tabs : nullptr, (bits + 7) / 8);
        count_launch();
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) { st = cuda_fail(e, "k_rs_scatter", __FILE__, __LINE__); break; }
        std::swap(ki, ko);
        std::swap(vi, vo);
        *in_alt = !*in_alt;
    }
    cudaFreeAsync(counts, s);
    cudaFreeAsync(sums, s);
    return st;
}

// ------------------------------------------------------ row statistics --

constexpr int RC_THREADS = 256;
constexpr int RC_HASH = 1024; // per mode, shared memory aggregation table

__device__ __forceinline__ uint32_t hash_row(uint32_t r) { return (r * 2654435761u) >> 7; }

struct CountPtrs {
    uint32_t* c[BLCO_MAX_MODES];
};

// Nonzeros per row of every mode.  Rows are aggregated inside the warp
// (match_any) and then in a per-block shared hash table before the global
// atomics, so rows holding a large share of the nonzeros do not serialise
// on one address.
__global__ __launch_bounds__(RC_THREADS) void k_row_counts(const uint64_t* __restrict__ coords, uint64_t nnz,
                                                           Layout L, CountPtrs counts)
{
    __shared__ uint32_t hkey[BLCO_MAX_MODES][RC_HASH];
    __shared__ uint32_t hcnt[BLCO_MAX_MODES][RC_HASH];
    for (int i = threadIdx.x; i < BLCO_MAX_MODES * RC_HASH; i += RC_THREADS) {
        (&hkey[0][0])[i] = 0;
        (&hcnt[0][0])[i] = 0;
    }
    __syncthreads();
    const uint64_t per = (nnz + gridDim.x - 1) / gridDim.x;
    const uint64_t beg = per * blockIdx.x, end = min(nnz, beg + per);
    const int lane = threadIdx.x & 31;
    for (uint64_t b0 = beg; b0 < end; b0 += RC_THREADS) {
        uint64_t i = b0 + threadIdx.x;
        bool ok = i < end;
        uint64_t c = ok ? coords[i] : 0;
        for (int n = 0; n < L.nmodes; n++) {
            uint32_t row = ok ? (uint32_t)((c >> L.mode_pos[n]) & L.mode_masks[n]) : 0xffffffffu;
            uint32_t peers = __match_any_sync(0xffffffffu, row);
            if (!ok || (peers & ((1u << lane) - 1)) != 0) continue;
            uint32_t cnt = __popc(peers);
            uint32_t h = hash_row(row) & (RC_HASH - 1);
            bool placed = false;
            for (int probe = 0; probe < 8 && !placed; probe++) {
                uint32_t slot = (h + probe) & (RC_HASH - 1);
                uint32_t prev = atomicCAS(&hkey[n][slot], 0u, row + 1);
                if (prev == 0u || prev == row + 1) {
                    atomicAdd(&hcnt[n][slot], cnt);
                    placed = true;
                }
            }
            if (!placed) atomicAdd(&counts.c[n][row], cnt);
        }
    }
    __syncthreads();
    for (int n = 0; n < L.nmodes; n++)
        for (int i = threadIdx.x; i < RC_HASH; i += RC_THREADS)
            if (hkey[n][i]) atomicAdd(&counts.c[n][hkey[n][i] - 1], hcnt[n][i]);
}

struct StatOut {
    unsigned long long hist[40];
    unsigned long long nonempty;
    unsigned long long maxc;
};

// Nonzeros per row of every mode, from COO arrays (the chunked encoder,
// whose stream never sits whole on the device); warp-aggregated atomics.
// Coordinates at or above the mode length are skipped here (k_alto_keys
// reports them; the encode then fails).
__global__ __launch_bounds__(RC_THREADS) void k_coo_counts(CooPtrs coo, uint64_t nnz, Layout L, CountPtrs counts)
{
    const int lane = threadIdx.x & 31;
    for (uint64_t b0 = blockIdx.x * (uint64_t)RC_THREADS; b0 < nnz; b0 += (uint64_t)gridDim.x * RC_THREADS) {
        const uint64_t i = b0 + threadIdx.x;
        for (int n = 0; n < L.nmodes; n++) {
            const uint64_t c = i < nnz ? coo.c[n][i] : ~0ull;
            const bool ok = c < L.dims[n];
            const uint32_t row = ok ? (uint32_t)c : 0xffffffffu;
            const uint32_t peers = __match_any_sync(0xffffffffu, row);
            if (ok && (peers & ((1u << lane) - 1)) == 0) atomicAdd(&counts.c[n][row], (uint32_t)__popc(peers));
        }
    }
}

__global__ void k_row_stats(const uint32_t* __restrict__ counts, uint64_t rows, StatOut* out)
{
    __shared__ unsigned long long h[40];
    __shared__ unsigned long long ne, mx;
    if (threadIdx.x < 40) h[threadIdx.x] = 0;
    if (threadIdx.x == 0) { ne = 0; mx = 0; }
    __syncthreads();
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < rows; r += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t c = counts[r];
        if (c) {
            atomicAdd(&h[31 - __clz(c)], 1ull);
            atomicAdd(&ne, 1ull);
            atomicMax(&mx, (unsigned long long)c);
        }
    }
    __syncthreads();
    if (threadIdx.x < 40 && h[threadIdx.x]) atomicAdd(&out->hist[threadIdx.x], h[threadIdx.x]);
    if (threadIdx.x == 0) {
        if (ne) atomicAdd(&out->nonempty, ne);
        if (mx) atomicMax(&out->maxc, mx);
    }
}

constexpr int HOT_CAND_MAX = 8192;
constexpr int HOT_MAX = 4096;     // rows kept per mode
constexpr int HOT_HASH = 8192;    // hash size (power of two, 2x HOT_MAX)
constexpr uint32_t HOT_MIN_COUNT = 256;

__global__ void k_collect_hot(const uint32_t* __restrict__ counts, uint64_t rows, uint32_t thresh,
                              uint32_t* __restrict__ cand_row, uint32_t* __restrict__ cand_cnt,
                              uint32_t* __restrict__ ncand)
{
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < rows; r += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t c = counts[r];
        if (c >= thresh) {
            uint32_t k = atomicAdd(ncand, 1u);
            if (k < HOT_CAND_MAX) {
                cand_row[k] = (uint32_t)r;
                cand_cnt[k] = c;
            }
        }
    }
}

// key_i = (mode-n row of nonzero i) << 32 | i: sorting by the row bits
// orders the stream by row, stream (ALTO) order inside a row.
__global__ void k_row_keys(const uint64_t* __restrict__ coords, uint64_t nnz, int pos, uint64_t mask,
                           uint64_t* __restrict__ keys)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nnz; i += (uint64_t)gridDim.x * blockDim.x)
        keys[i] = (((coords[i] >> pos) & mask) << 32) | i;
}

// From the row-sorted keys rk: key_j = (slot of the row, or 0xffff) << 32 |
// (stream position), so that a stable sort by slot puts the hot rows first,
// grouped by slot, and the cold nonzeros after them in row order.
__global__ void k_hot_keys(const uint64_t* __restrict__ rk, uint64_t nnz, const uint32_t* __restrict__ hkeys,
                            const uint32_t* __restrict__ hslot, int hsize, uint64_t* __restrict__ keys)
{
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < nnz; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t row = (uint32_t)(rk[j] >> 32), i = (uint32_t)rk[j];
        uint32_t h = hash_row(row) & (hsize - 1), slot = 0xffffu;
        for (int probe = 0; probe < hsize; probe++) {
            uint32_t k = hkeys[h];
            if (k == row + 1) {
                slot = hslot[h];
                break;
            }
            if (k == 0) break;
            h = (h + 1) & (hsize - 1);
        }
        keys[j] = ((uint64_t)slot << 32) | i;
    }
}

// hc[j] = coords[pos_j], hv[j] = vals[pos_j] with pos_j the low 32 bits of
// the sorted key j.
__global__ void k_gather_hot(const uint64_t* __restrict__ keys, uint64_t n, const uint64_t* __restrict__ coords,
                             const double* __restrict__ vals, uint64_t* __restrict__ hc, double* __restrict__ hv)
{
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t i = (uint32_t)keys[j];
        hc[j] = coords[i];
        hv[j] = vals[i];
    }
}

__global__ void k_sumsq(const double* __restrict__ v, uint64_t n, double* __restrict__ partial)
{
    __shared__ double ws[32];
    double s = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        s += v[i] * v[i];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < blockDim.x / 32 ? ws[threadIdx.x] : 0.0;
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) partial[blockIdx.x] = s;
    }
}

// ------------------------------------------------------------ wide keys --
//
// Keys of 65..128 bits (the reference's 128-bit build, gen_blcotensor_host
// <unsigned __int128>, include/blco.hpp:196-331).  The key is a low and an
// upper 64-bit word; the order is (upper, low), so two stable radix sorts
// of an index permutation run: by the low word, then by the upper word.
// The BLCO arrays are then gathered straight from the COO input: fields of
// the low-word bits, the values, and the block field (Layout).  Blocks are
// the runs of equal upper words (the reference's histogram buckets, in
// increasing order), split into max_block_size slices.

// lo[n][b][v] / hi[n][b][v]: the low / upper key word bits of coordinate
// byte b of mode n with value v.
struct WideTables {
    uint64_t lo[BLCO_MAX_MODES][4][256];
    uint64_t hi[BLCO_MAX_MODES][4][256];
};

WideTables make_wide_tables(const Layout& L)
{
    WideTables T;
    memset(&T, 0, sizeof(T));
    for (int n = 0; n < L.nmodes; n++) {
        // key position of coordinate bit j: the j-th set bit of the 128-bit mask
        int posn[64];
        int j = 0;
        for (int p = 0; p < 128; p++) {
            const uint64_t w = p < 64 ? L.alto_masks[n] : L.alto_masks_hi[n];
            if (w >> (p & 63) & 1) posn[j++] = p;
        }
        for (int b = 0; b < 4; b++)
            for (int v = 0; v < 256; v++)
                for (int k = 0; k < 8; k++) {
                    const int bit = 8 * b + k;
                    if (bit >= j || !(v >> k & 1)) continue;
                    if (posn[bit] < 64) T.lo[n][b][v] |= 1ull << posn[bit];
                    else T.hi[n][b][v] |= 1ull << (posn[bit] - 64);
                }
    }
    return T;
}

__global__ void k_wide_keys(CooPtrs coo, uint64_t nnz, Layout L, const WideTables* __restrict__ tabs,
                            uint64_t* __restrict__ lo, uint64_t* __restrict__ idx, uint64_t* __restrict__ hi,
                            int* __restrict__ bad)
{
    extern __shared__ __align__(16) unsigned char wk_smem[];
    WideTables* T = reinterpret_cast<WideTables*>(wk_smem);
    const uint4* src = reinterpret_cast<const uint4*>(tabs);
    uint4* dst = reinterpret_cast<uint4*>(wk_smem);
    for (int i = threadIdx.x; i < (int)(sizeof(WideTables) / 16); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nnz;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t kl = 0, kh = 0;
        bool ok = true;
#pragma unroll
        for (int n = 0; n < BLCO_MAX_MODES; n++) {
            if (n < L.nmodes) {
                const uint64_t c = coo.c[n][i];
                ok &= c < L.dims[n];
#pragma unroll
                for (int b = 0; b < 4; b++) {
                    const uint32_t v = (uint32_t)(c >> (8 * b)) & 255;
                    kl |= T->lo[n][b][v];
                    kh |= T->hi[n][b][v];
                }
            }
        }
        if (!ok) atomicExch(bad, 1);
        lo[i] = kl;
        idx[i] = i;
        hi[i] = kh;
    }
}

__global__ void k_gather_u64(const uint64_t* __restrict__ src, const uint64_t* __restrict__ idx, uint64_t n,
                             uint64_t* __restrict__ dst)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        dst[i] = src[idx[i]];
}

// BLCO arrays at sorted position i from the COO entry idx[i]; flags[i] = 1
// where a run of equal upper words starts.
__global__ void k_wide_finish(CooPtrs coo, const double* __restrict__ vals, const uint64_t* __restrict__ idx,
                              const uint64_t* __restrict__ hi, uint64_t nnz, Layout L, uint64_t* __restrict__ coords,
                              double* __restrict__ vout, uint64_t* __restrict__ field, uint32_t* __restrict__ flags)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nnz;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t src = idx[i];
        uint64_t c = 0, f = 0;
#pragma unroll
        for (int n = 0; n < BLCO_MAX_MODES; n++) {
            if (n < L.nmodes) {
                const uint64_t x = coo.c[n][src];
                c |= (x & L.mode_masks[n]) << L.mode_pos[n];
                f |= (x >> L.low_bits[n]) << L.bpos[n];
            }
        }
        coords[i] = c;
        vout[i] = vals[src];
        field[i] = f;
        flags[i] = (i == 0 || hi[i] != hi[i - 1]) ? 1u : 0u;
    }
}

__global__ void k_wide_runs(const uint32_t* __restrict__ rank, const uint64_t* __restrict__ hi,
                            const uint64_t* __restrict__ field, uint64_t nnz, uint64_t* __restrict__ run_start,
                            uint64_t* __restrict__ run_field)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nnz;
         i += (uint64_t)gridDim.x * blockDim.x) {
        if (i == 0 || hi[i] != hi[i - 1]) {
            run_start[rank[i]] = i;
            run_field[rank[i]] = field[i];
        }
    }
}

// key[i] = row of mode n of nonzero i, idx[i] = i.
__global__ void k_wide_row_keys(const uint64_t* __restrict__ coords, const uint64_t* __restrict__ field,
                                uint64_t nnz, Layout L, int n, uint64_t* __restrict__ key, uint64_t* __restrict__ idx)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nnz;
         i += (uint64_t)gridDim.x * blockDim.x) {
        key[i] = wide_row(L, n, coords[i], field[i]);
        idx[i] = i;
    }
}

__global__ void k_gather3(const uint64_t* __restrict__ idx, uint64_t n, const uint64_t* __restrict__ a,
                          const uint64_t* __restrict__ b, const double* __restrict__ c, uint64_t* __restrict__ oa,
                          uint64_t* __restrict__ ob, double* __restrict__ oc)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t j = idx[i];
        oa[i] = a[j];
        ob[i] = b[j];
        oc[i] = c[j];
    }
}

} // namespace

int radix_sort_pairs_u64(uint64_t* k0, uint64_t* v0, uint64_t* k1, uint64_t* v1, uint64_t n, int end_bit,
                         cudaStream_t s, bool* in_alt)
{
    // the sort moves the 8-byte payloads without reading them as numbers
    return radix_sort_pairs(k0, reinterpret_cast<double*>(v0), k1, reinterpret_cast<double*>(v1), n, 0, end_bit, s,
                            in_alt);
}

int scan_u32_ext(uint32_t* a, uint64_t n, uint32_t* sums, cudaStream_t s) { return scan_u32(a, n, sums, s); }

// Per-mode copies of a wide-key stream sorted by that mode's row (stable:
// key order inside a row), so that the MTTKRP of mode n sums each row's
// nonzeros in registers and writes it once per warp task.
static int build_wide_copies(blco_tensor* t, cudaStream_t s, const DeviceInfo& di)
{
    const uint64_t nnz = t->nnz;
    const Layout& L = t->layout;
    if (nnz == 0) return BLCO_OK;
    uint64_t* tmp[4] = {};
    auto release = [&]() {
        cudaStreamSynchronize(s);
        for (auto& b : tmp) { cudaFree(b); b = nullptr; }
    };
    for (auto& b : tmp) {
        cudaError_t e = cudaMalloc(&b, nnz * 8);
        if (e != cudaSuccess) { release(); return cuda_fail(e, "wide copy scratch", __FILE__, __LINE__); }
    }
    const int grid = (int)std::min<uint64_t>((nnz + 255) / 256, (uint64_t)di.sm_count * 8);
    for (int n = 0; n < L.nmodes; n++) {
        const int bits = L.low_bits[n] + __builtin_popcountll(L.alto_masks_hi[n]);
        k_wide_row_keys<<<grid, 256, 0, s>>>(t->d_coords, t->d_bfield, nnz, L, n, tmp[0], tmp[1]);
        count_launch();
        bool alt = false;
        int st = radix_sort_pairs(tmp[0], reinterpret_cast<double*>(tmp[1]), tmp[2], reinterpret_cast<double*>(tmp[3]),
                                  nnz, 0, bits, s, &alt);
        if (st != BLCO_OK) { release(); return st; }
        const uint64_t* idx = alt ? tmp[3] : tmp[1];
        blco_tensor::WideCopy& w = t->wide_copy[n];
        cudaError_t e = cudaMalloc(&w.d_coords, nnz * 8);
        if (e == cudaSuccess) e = cudaMalloc(&w.d_field, nnz * 8);
        if (e == cudaSuccess) e = cudaMalloc(&w.d_vals, nnz * 8);
        if (e != cudaSuccess) { release(); return cuda_fail(e, "wide copy", __FILE__, __LINE__); }
        k_gather3<<<grid, 256, 0, s>>>(idx, nnz, t->d_coords, t->d_bfield, t->d_values, w.d_coords, w.d_field,
                                       w.d_vals);
        count_launch();
        e = cudaGetLastError();
        if (e != cudaSuccess) { release(); return cuda_fail(e, "k_gather3", __FILE__, __LINE__); }
    }
    release();
    return BLCO_OK;
}

// Wide-key encode of the resident stream: fills t->d_coords, d_values,
// d_bfield, block_offsets, block_coords, block_count and norm_sq.
static int encode_wide(blco_tensor* t, const uint64_t* const* d_cidx, const double* d_vals, cudaStream_t s,
                       const DeviceInfo& di)
{
    const uint64_t nnz = t->nnz;
    const Layout& L = t->layout;
    if (nnz == 0) return BLCO_OK;
    uint64_t* buf[5] = {};      // k0, v0, k1, v1, hi
    uint32_t* flags = nullptr;  // nnz + 1
    int* d_bad = nullptr;
    WideTables* d_tabs = nullptr;
    uint64_t *run_start = nullptr, *run_field = nullptr;
    int st = BLCO_OK;
    auto release = [&]() {
        cudaStreamSynchronize(s);
        for (uint64_t*& b : buf) { cudaFree(b); b = nullptr; }
        cudaFree(flags);
        cudaFree(d_bad);
        cudaFree(d_tabs);
        cudaFree(run_start);
        cudaFree(run_field);
    };
#define WIDE_CUDA(call)                                                         \
    do {                                                                        \
        cudaError_t _e = (call);                                                \
        if (_e != cudaSuccess) {                                                \
            int _s = cuda_fail(_e, #call, __FILE__, __LINE__);                  \
            release();                                                          \
            return _s;                                                          \
        }                                                                       \
    } while (0)
    for (auto& b : buf) WIDE_CUDA(cudaMalloc(&b, nnz * 8));
    WIDE_CUDA(cudaMalloc(&flags, (nnz + 1) * sizeof(uint32_t)));
    WIDE_CUDA(cudaMalloc(&d_bad, sizeof(int)));
    WIDE_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(int), s));
    WIDE_CUDA(cudaMemsetAsync(flags + nnz, 0, sizeof(uint32_t), s));
    {
        WideTables* h = new WideTables(make_wide_tables(L));
        cudaError_t e = cudaMalloc(&d_tabs, sizeof(WideTables));
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_tabs, h, sizeof(WideTables), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        delete h;
        WIDE_CUDA(e);
    }
    CooPtrs coo;
    memset(&coo, 0, sizeof(coo));
    for (int n = 0; n < L.nmodes; n++) coo.c[n] = d_cidx[n];
    const int grid = (int)std::min<uint64_t>((nnz + 255) / 256, (uint64_t)di.sm_count * 8);
    WIDE_CUDA(cudaFuncSetAttribute(k_wide_keys, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(WideTables)));
    k_wide_keys<<<grid, 256, sizeof(WideTables), s>>>(coo, nnz, L, d_tabs, buf[0], buf[1], buf[4], d_bad);
    count_launch();
    WIDE_CUDA(cudaGetLastError());
    int bad = 0;
    WIDE_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    WIDE_CUDA(cudaStreamSynchronize(s));
    if (bad) {
        release();
        return fail(BLCO_ERR_INVALID, "a coordinate is not below its mode length");
    }
    // (low word, index) by the low word, then (upper word, index) by the
    // upper word: the index order of the 128-bit key, ties in input order.
    bool alt = false;
    double* v0 = reinterpret_cast<double*>(buf[1]);
    double* v1 = reinterpret_cast<double*>(buf[3]);
    if ((st = radix_sort_pairs(buf[0], v0, buf[2], v1, nnz, 0, 64, s, &alt)) != BLCO_OK) { release(); return st; }
    uint64_t* kA = alt ? buf[2] : buf[0];
    uint64_t* iA = alt ? buf[3] : buf[1];
    uint64_t* kB = alt ? buf[0] : buf[2];
    uint64_t* iB = alt ? buf[1] : buf[3];
    k_gather_u64<<<grid, 256, 0, s>>>(buf[4], iA, nnz, kA);
    count_launch();
    WIDE_CUDA(cudaGetLastError());
    if ((st = radix_sort_pairs(kA, reinterpret_cast<double*>(iA), kB, reinterpret_cast<double*>(iB), nnz, 0,
                               L.alto_bits - 64, s, &alt)) != BLCO_OK) {
        release();
        return st;
    }
    uint64_t* hiF = alt ? kB : kA;  // sorted upper words
    uint64_t* idxF = alt ? iB : iA; // sorted permutation
    uint64_t* outC = alt ? kA : kB; // free now
    uint64_t* outV = alt ? iA : iB;
    uint64_t* outF = buf[4];
    k_wide_finish<<<grid, 256, 0, s>>>(coo, d_vals, idxF, hiF, nnz, L, outC, reinterpret_cast<double*>(outV), outF,
                                       flags);
    count_launch();
    WIDE_CUDA(cudaGetLastError());
    uint32_t* sums = nullptr;
    {
        const uint64_t nsums = (nnz + 1 + SC_CHUNK - 1) / SC_CHUNK + 1;
        WIDE_CUDA(cudaMallocAsync(&sums, nsums * sizeof(uint32_t), s));
        st = scan_u32(flags, nnz + 1, sums, s);
        cudaFreeAsync(sums, s);
        if (st != BLCO_OK) { release(); return st; }
    }
    uint32_t nruns = 0;
    WIDE_CUDA(cudaMemcpyAsync(&nruns, flags + nnz, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    WIDE_CUDA(cudaStreamSynchronize(s));
    WIDE_CUDA(cudaMalloc(&run_start, (uint64_t)nruns * 8));
    WIDE_CUDA(cudaMalloc(&run_field, (uint64_t)nruns * 8));
    k_wide_runs<<<grid, 256, 0, s>>>(flags, hiF, outF, nnz, run_start, run_field);
    count_launch();
    WIDE_CUDA(cudaGetLastError());
    std::vector<uint64_t> hs(nruns), hf(nruns);
    WIDE_CUDA(cudaMemcpyAsync(hs.data(), run_start, (uint64_t)nruns * 8, cudaMemcpyDeviceToHost, s));
    WIDE_CUDA(cudaMemcpyAsync(hf.data(), run_field, (uint64_t)nruns * 8, cudaMemcpyDeviceToHost, s));
    // sum of squared values (the partial sums reuse the sorted-index buffer)
    const int g2 = std::min(grid, 1024);
    k_sumsq<<<g2, 256, 0, s>>>(reinterpret_cast<const double*>(outV), nnz, reinterpret_cast<double*>(idxF));
    count_launch();
    WIDE_CUDA(cudaGetLastError());
    std::vector<double> hp(g2);
    WIDE_CUDA(cudaMemcpyAsync(hp.data(), idxF, g2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    WIDE_CUDA(cudaStreamSynchronize(s));
#undef WIDE_CUDA
    double ss = 0.0;
    for (double x : hp) ss += x;
    t->norm_sq = ss;
    // Blocks: each run split into max_block_size slices, block_coords[n] =
    // (block field of mode n) << low_bits[n] (include/blco.hpp:290-321).
    const uint64_t B = t->max_block_size ? t->max_block_size : nnz;
    t->block_offsets.clear();
    t->block_coords.clear();
    for (uint32_t r = 0; r < nruns; r++) {
        const uint64_t b0 = hs[r], b1 = r + 1 < nruns ? hs[r + 1] : nnz;
        for (uint64_t o = b0; o < b1; o += B) {
            t->block_offsets.push_back(o);
            for (int n = 0; n < L.nmodes; n++)
                t->block_coords.push_back(((hf[r] >> L.bpos[n]) & L.bmask[n]) << L.low_bits[n]);
        }
    }
    t->block_count = t->block_offsets.size();
    t->block_offsets.push_back(nnz);
    // keep the three output arrays, release the rest
    t->d_coords = outC;
    t->d_values = reinterpret_cast<double*>(outV);
    t->d_bfield = outF;
    for (uint64_t*& b : buf)
        if (b == outC || b == outV || b == outF) b = nullptr;
    release();
    return build_wide_copies(t, s, di);
}

uint32_t host_hash_row(uint32_t r) { return (r * 2654435761u) >> 7; }

// Per-mode execution copies of the stream: a stable radix sort of
// (row << 32 | position) on the row bits, then of (slot << 32 | position) on
// the slot bits, gives the hot-row positions grouped by slot followed by the
// cold positions by row (ALTO order inside each row in both); coordinates
// and values are gathered into a hot stream and a cold stream.  Together
// they hold every nonzero once, so a mode's MTTKRP reads 16 bytes per
// nonzero as with the BLCO stream itself.  In the row-ordered cold stream a
// 32-nonzero tile spans few rows, so the tile kernel's segmented reduction
// leaves few atomics (FP64 MTTKRP about 30% faster than on ALTO order).
// Built for one mode on its first use by a schedule that reads them (the
// heavy-row kernel beside the tile kernel), or at plan creation for such a
// schedule; the compressed-fibre schedule never reads them.
int build_mode_copies(blco_tensor* t, int mode, cudaStream_t s)
{
    const Layout& L = t->layout;
    if (t->nnz == 0 || !t->resident || mode < 0 || mode >= L.nmodes) return BLCO_OK;
    if (t->hot[mode].nhot == 0 || t->hot[mode].hot_nnz == 0 || t->hot[mode].d_hcoords) return BLCO_OK;
    DeviceInfo di;
    BLCO_TRY(device_info(t->device, &di));
    uint64_t *k0 = nullptr, *k1 = nullptr;
    double *v0 = nullptr, *v1 = nullptr;
    int st = BLCO_OK;
    auto cleanup = [&]() {
        cudaStreamSynchronize(s);
        cudaFree(k0);
        cudaFree(k1);
        cudaFree(v0);
        cudaFree(v1);
    };
    cudaError_t e = cudaMalloc(&k0, t->nnz * 8);
    if (e == cudaSuccess) e = cudaMalloc(&k1, t->nnz * 8);
    if (e == cudaSuccess) e = cudaMalloc(&v0, t->nnz * 8);
    if (e == cudaSuccess) e = cudaMalloc(&v1, t->nnz * 8);
    if (e != cudaSuccess) {
        cleanup();
        return cuda_fail(e, "hot-row index scratch", __FILE__, __LINE__);
    }
    const int grid = (int)std::min<uint64_t>((t->nnz + 255) / 256, (uint64_t)di.sm_count * 16);
    for (int n = mode; n == mode && st == BLCO_OK; n++) {
        HotTable& ht = t->hot[n];
        k_row_keys<<<grid, 256, 0, s>>>(t->d_coords, t->nnz, L.mode_pos[n], L.mode_masks[n], k0);
        count_launch();
        bool alt0 = false;
        const int rbits = __builtin_popcountll(L.mode_masks[n]);
        if ((st = radix_sort_pairs(k0, v0, k1, v1, t->nnz, 32, 32 + rbits, s, &alt0)) != BLCO_OK) break;
        k_hot_keys<<<grid, 256, 0, s>>>(alt0 ? k1 : k0, t->nnz, ht.d_keys, ht.d_slot, ht.hash_size, alt0 ? k0 : k1);
        count_launch();
        if ((e = cudaGetLastError()) != cudaSuccess) { st = cuda_fail(e, "k_hot_keys", __FILE__, __LINE__); break; }
        bool alt = false;
        uint64_t *ka = alt0 ? k0 : k1, *kb = alt0 ? k1 : k0;
        if ((st = radix_sort_pairs(ka, v0, kb, v1, t->nnz, 32, 48, s, &alt)) != BLCO_OK) break;
        if (ka != k0) alt = !alt; // sk below picks from (k0, k1)
        // Sorted keys: the hot positions grouped by slot, then the cold
        // positions by row (stream order inside a row).
        ht.cold_nnz = t->nnz - ht.hot_nnz;
        e = cudaMalloc(&ht.d_hcoords, ht.hot_nnz * sizeof(uint64_t));
        if (e == cudaSuccess) e = cudaMalloc(&ht.d_hvals, ht.hot_nnz * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&ht.d_ccoords, std::max<uint64_t>(1, ht.cold_nnz) * sizeof(uint64_t));
        if (e == cudaSuccess) e = cudaMalloc(&ht.d_cvals, std::max<uint64_t>(1, ht.cold_nnz) * sizeof(double));
        if (e != cudaSuccess) { st = cuda_fail(e, "per-mode stream copies", __FILE__, __LINE__); break; }
        const uint64_t* sk = alt ? k1 : k0;
        k_gather_hot<<<grid, 256, 0, s>>>(sk, ht.hot_nnz, t->d_coords, t->d_values, ht.d_hcoords, ht.d_hvals);
        count_launch();
        if ((e = cudaGetLastError()) != cudaSuccess) { st = cuda_fail(e, "k_gather_hot", __FILE__, __LINE__); break; }
        if (ht.cold_nnz) {
            k_gather_hot<<<grid, 256, 0, s>>>(sk + ht.hot_nnz, ht.cold_nnz, t->d_coords, t->d_values, ht.d_ccoords,
                                              ht.d_cvals);
            count_launch();
            if ((e = cudaGetLastError()) != cudaSuccess) { st = cuda_fail(e, "k_gather_hot", __FILE__, __LINE__); break; }
        }
    }
    cleanup();
    return st;
}

// A copy of the tensor's stream sorted stably by the row index of `mode`
// (ALTO order inside each row), written to d_coords / d_vals (nnz entries
// each); tmp_k / tmp_v are nnz-entry scratch arrays.
int sort_stream_by_mode(const blco_tensor* t, int mode, uint64_t* d_coords, double* d_vals, uint64_t* tmp_k,
                        double* tmp_v, cudaStream_t s)
{
    const Layout& L = t->layout;
    if (t->nnz == 0) return BLCO_OK;
    BLCO_CUDA(cudaMemcpyAsync(d_coords, t->d_coords, t->nnz * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
    BLCO_CUDA(cudaMemcpyAsync(d_vals, t->d_values, t->nnz * sizeof(double), cudaMemcpyDeviceToDevice, s));
    const int bits = __builtin_popcountll(L.mode_masks[mode]);
    if (bits == 0) return BLCO_OK;
    bool alt = false;
    BLCO_TRY(radix_sort_pairs(d_coords, d_vals, tmp_k, tmp_v, t->nnz, L.mode_pos[mode], L.mode_pos[mode] + bits, s,
                              &alt));
    if (alt) {
        BLCO_CUDA(cudaMemcpyAsync(d_coords, tmp_k, t->nnz * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
        BLCO_CUDA(cudaMemcpyAsync(d_vals, tmp_v, t->nnz * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    return BLCO_OK;
}

// Heavy-row statistics and tables.  counts_in (device, the per-row
// nonzero counts of every mode concatenated) is used when given; otherwise
// the counts are taken from the resident stream.
static int build_hot_tables_impl(blco_tensor* t, cudaStream_t s, uint32_t* counts_in)
{
    const Layout& L = t->layout;
    DeviceInfo di;
    BLCO_TRY(device_info(t->device, &di));
    CountPtrs cp;
    memset(&cp, 0, sizeof(cp));
    uint64_t total_rows = 0;
    for (int n = 0; n < L.nmodes; n++) total_rows += L.dims[n];
    uint32_t* counts = counts_in;
    if (!counts) {
        BLCO_CUDA(cudaMallocAsync(&counts, total_rows * sizeof(uint32_t), s));
        BLCO_CUDA(cudaMemsetAsync(counts, 0, total_rows * sizeof(uint32_t), s));
    }
    uint64_t off = 0;
    for (int n = 0; n < L.nmodes; n++) {
        cp.c[n] = counts + off;
        off += L.dims[n];
    }
    if (t->nnz && !counts_in) {
        k_row_counts<<<di.sm_count * 4, RC_THREADS, 0, s>>>(t->d_coords, t->nnz, L, cp);
        BLCO_CHECK_LAUNCH("k_row_counts");
    }
    StatOut* d_stats = nullptr;
    uint32_t *cand = nullptr, *ncand = nullptr;
    BLCO_CUDA(cudaMallocAsync(&d_stats, sizeof(StatOut) * L.nmodes, s));
    BLCO_CUDA(cudaMemsetAsync(d_stats, 0, sizeof(StatOut) * L.nmodes, s));
    BLCO_CUDA(cudaMallocAsync(&cand, sizeof(uint32_t) * 2 * HOT_CAND_MAX * L.nmodes, s));
    BLCO_CUDA(cudaMallocAsync(&ncand, sizeof(uint32_t) * L.nmodes, s));
    BLCO_CUDA(cudaMemsetAsync(ncand, 0, sizeof(uint32_t) * L.nmodes, s));
    for (int n = 0; n < L.nmodes; n++) {
        int grid = (int)std::min<uint64_t>((L.dims[n] + 255) / 256, (uint64_t)di.sm_count * 8);
        k_row_stats<<<grid, 256, 0, s>>>(cp.c[n], L.dims[n], d_stats + n);
        BLCO_CHECK_LAUNCH("k_row_stats");
    }
    std::vector<StatOut> hs(L.nmodes);
    BLCO_CUDA(cudaMemcpyAsync(hs.data(), d_stats, sizeof(StatOut) * L.nmodes, cudaMemcpyDeviceToHost, s));
    BLCO_CUDA(cudaStreamSynchronize(s));
    std::vector<uint32_t> thresh(L.nmodes, 0);
    for (int n = 0; n < L.nmodes; n++) {
        ModeStats& ms = t->stats[n];
        ms.max_row_nnz = hs[n].maxc;
        ms.nonempty_rows = hs[n].nonempty;
        for (int b = 0; b < 40; b++) ms.log2_hist[b] = hs[n].hist[b];
        // Lowest power-of-two threshold with at most HOT_CAND_MAX rows above it.
        uint64_t above = 0;
        int bsel = 40;
        for (int b = 39; b >= 0; b--) {
            if (above + hs[n].hist[b] > (uint64_t)HOT_CAND_MAX) break;
            above += hs[n].hist[b];
            bsel = b;
        }
        uint64_t th = bsel >= 40 ? ~0u : (1ull << bsel);
        thresh[n] = (uint32_t)std::max<uint64_t>(th, HOT_MIN_COUNT);
    }
    for (int n = 0; n < L.nmodes; n++) {
        int grid = (int)std::min<uint64_t>((L.dims[n] + 255) / 256, (uint64_t)di.sm_count * 8);
        k_collect_hot<<<grid, 256, 0, s>>>(cp.c[n], L.dims[n], thresh[n], cand + 2 * HOT_CAND_MAX * n,
                                           cand + 2 * HOT_CAND_MAX * n + HOT_CAND_MAX, ncand + n);
        BLCO_CHECK_LAUNCH("k_collect_hot");
    }
    std::vector<uint32_t> hc(2 * HOT_CAND_MAX * L.nmodes), hn(L.nmodes);
    BLCO_CUDA(cudaMemcpyAsync(hc.data(), cand, hc.size() * 4, cudaMemcpyDeviceToHost, s));
    BLCO_CUDA(cudaMemcpyAsync(hn.data(), ncand, hn.size() * 4, cudaMemcpyDeviceToHost, s));
    BLCO_CUDA(cudaStreamSynchronize(s));
    if (!counts_in) cudaFreeAsync(counts, s);
    cudaFreeAsync(d_stats, s);
    cudaFreeAsync(cand, s);
    cudaFreeAsync(ncand, s);

    for (int n = 0; n < L.nmodes; n++) {
        HotTable& ht = t->hot[n];
        uint32_t nc = std::min<uint32_t>(hn[n], HOT_CAND_MAX);
        std::vector<std::pair<uint32_t, uint32_t>> rows; // (count, row)
        for (uint32_t k = 0; k < nc; k++)
            rows.push_back({hc[2 * HOT_CAND_MAX * n + HOT_CAND_MAX + k], hc[2 * HOT_CAND_MAX * n + k]});
        std::sort(rows.begin(), rows.end(), [](auto& a, auto& b) {
            return a.first != b.first ? a.first > b.first : a.second < b.second;
        });
        if (rows.size() > (size_t)HOT_MAX) rows.resize(HOT_MAX);
        ht.nhot = (int)rows.size();
        ht.hot_nnz = 0;
        if (ht.nhot == 0) continue;
        ht.hash_size = HOT_HASH;
        std::vector<uint32_t> keys(HOT_HASH, 0), slots(HOT_HASH, 0);
        for (int k = 0; k < ht.nhot; k++) {
            uint32_t r = rows[k].second;
            ht.hot_nnz += rows[k].first;
            uint32_t h = host_hash_row(r) & (HOT_HASH - 1);
            while (keys[h]) h = (h + 1) & (HOT_HASH - 1);
            keys[h] = r + 1;
            slots[h] = (uint32_t)k; // slots in descending heaviness
        }
        std::vector<uint32_t> rowlist(ht.nhot);
        for (int k = 0; k < ht.nhot; k++) rowlist[k] = rows[k].second;
        BLCO_CUDA(cudaMalloc(&ht.d_keys, HOT_HASH * sizeof(uint32_t)));
        BLCO_CUDA(cudaMalloc(&ht.d_slot, HOT_HASH * sizeof(uint32_t)));
        BLCO_CUDA(cudaMalloc(&ht.d_rows, ht.nhot * sizeof(uint32_t)));
        BLCO_CUDA(cudaMemcpyAsync(ht.d_keys, keys.data(), HOT_HASH * 4, cudaMemcpyHostToDevice, s));
        BLCO_CUDA(cudaMemcpyAsync(ht.d_slot, slots.data(), HOT_HASH * 4, cudaMemcpyHostToDevice, s));
        BLCO_CUDA(cudaMemcpyAsync(ht.d_rows, rowlist.data(), ht.nhot * 4, cudaMemcpyHostToDevice, s));
        std::vector<uint32_t> ptr(ht.nhot + 1, 0);
        for (int k = 0; k < ht.nhot; k++) ptr[k + 1] = ptr[k] + rows[k].first;
        BLCO_CUDA(cudaMalloc(&ht.d_ptr, (ht.nhot + 1) * sizeof(uint32_t)));
        BLCO_CUDA(cudaMemcpyAsync(ht.d_ptr, ptr.data(), (ht.nhot + 1) * 4, cudaMemcpyHostToDevice, s));
    }
    BLCO_CUDA(cudaStreamSynchronize(s));
    // The per-mode execution copies (build_mode_copies) are made on first
    // use, for resident streams only; a streamed tensor keeps just the
    // statistics and hash tables, so that its device footprint stays the
    // ring of block buffers.
    return BLCO_OK;
}

int build_hot_tables(blco_tensor* t, cudaStream_t s) { return build_hot_tables_impl(t, s, nullptr); }

// ------------------------------------------------- chunked streamed encode --
//
// A streamed tensor lives in pinned host memory, so it may be larger than
// the device.  Its encode then runs in chunks that fit the residency
// budget: per chunk, the COO slice is copied in (from host or device
// memory), keyed (k_alto_keys), counted per row (k_coo_counts), sorted by
// key (stable radix sort) and copied back as (key, value) runs.  The runs
// are then merged on the GPU, one budget-sized output segment at a time
// (each run's share of the segment found by a search on the host, ties in
// chunk order), so the result is the stable key order of the whole input,
// the same as the one-pass encoder's; the merge's last sort pass writes BLCO
// coordinates (key re-linearized through the byte table) and the segment
// goes to the pinned stream.

uint64_t stream_chunk_nnz(const blco_opts* opts, int nmodes)
{
    const uint64_t budget = (opts && opts->residency_bytes) ? opts->residency_bytes : (8ull << 30);
    // device bytes per nonzero of a chunk: COO slice, two key/value buffers
    const uint64_t per = (uint64_t)nmodes * 8 + 8 + 32;
    return std::max<uint64_t>(4096, budget / per);
}

static int encode_chunked(blco_tensor* t, const uint64_t* const* cidx, const double* vals, cudaStream_t s,
                          const DeviceInfo& di, uint64_t C)
{
    const Layout& L = t->layout;
    const uint64_t nnz = t->nnz;
    const int nm = L.nmodes;
    const uint64_t nchunks = (nnz + C - 1) / C;
    uint64_t* dc[BLCO_MAX_MODES] = {};
    double* dvin = nullptr;
    uint64_t *k0 = nullptr, *k1 = nullptr;
    double *v0 = nullptr, *v1 = nullptr, *dpart = nullptr;
    uint32_t* counts = nullptr;
    int* d_bad = nullptr;
    EncTables* d_tabs = nullptr;
    // sorted keys and values of every chunk: pageable host memory (pinning
    // 16 B per nonzero costs more than the slower copies into it save)
    std::unique_ptr<uint64_t[]> hk_own;
    std::unique_ptr<double[]> hv_own;
    uint64_t* hk = nullptr;
    double* hv = nullptr;
    // the pinned stream itself is allocated on two host threads while the
    // chunks are sorted (page-locking is the slowest step of this encode)
    std::thread pin_c, pin_v;
    cudaError_t pin_e[2] = {cudaSuccess, cudaSuccess};
    auto join_pins = [&]() {
        if (pin_c.joinable()) pin_c.join();
        if (pin_v.joinable()) pin_v.join();
    };
    auto release = [&]() {
        cudaStreamSynchronize(s);
        for (auto& p : dc) { cudaFree(p); p = nullptr; }
        cudaFree(dvin);
        cudaFree(k0);
        cudaFree(k1);
        cudaFree(v0);
        cudaFree(v1);
        cudaFree(dpart);
        cudaFree(counts);
        cudaFree(d_bad);
        cudaFree(d_tabs);
        join_pins();
    };
#define CH_CUDA(call)                                                           \
    do {                                                                        \
        cudaError_t _e = (call);                                                \
        if (_e != cudaSuccess) {                                                \
            int _s = cuda_fail(_e, #call, __FILE__, __LINE__);                  \
            release();                                                          \
            return _s;                                                          \
        }                                                                       \
    } while (0)
    uint64_t total_rows = 0;
    for (int n = 0; n < nm; n++) total_rows += L.dims[n];
    for (int n = 0; n < nm; n++) CH_CUDA(cudaMalloc(&dc[n], C * 8));
    CH_CUDA(cudaMalloc(&dvin, C * 8));
    CH_CUDA(cudaMalloc(&k0, C * 8));
    CH_CUDA(cudaMalloc(&k1, C * 8));
    CH_CUDA(cudaMalloc(&v0, C * 8));
    CH_CUDA(cudaMalloc(&v1, C * 8));
    const int grid = (int)std::min<uint64_t>((C + 255) / 256, (uint64_t)di.sm_count * 16);
    const int g2 = std::min(grid, 1024);
    CH_CUDA(cudaMalloc(&dpart, (size_t)g2 * sizeof(double)));
    CH_CUDA(cudaMalloc(&counts, total_rows * sizeof(uint32_t)));
    CH_CUDA(cudaMemsetAsync(counts, 0, total_rows * sizeof(uint32_t), s));
    CH_CUDA(cudaMalloc(&d_bad, sizeof(int)));
    CH_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(int), s));
    EncTables htabs = make_tables(L);
    CH_CUDA(cudaMalloc(&d_tabs, sizeof(EncTables)));
    CH_CUDA(cudaMemcpyAsync(d_tabs, &htabs, sizeof(EncTables), cudaMemcpyHostToDevice, s));
    hk_own.reset(new (std::nothrow) uint64_t[nnz]);
    hv_own.reset(new (std::nothrow) double[nnz]);
    hk = hk_own.get();
    hv = hv_own.get();
    if (!hk || !hv) {
        release();
        return fail(BLCO_ERR_NOMEM, "host memory for the sorted chunks");
    }
    {
        // first touch of the run buffers on many host threads, before any
        // copy lands there (page faults dominate a copy into fresh memory)
        const unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
        std::vector<std::thread> th;
        for (unsigned w = 0; w < nt; w++)
            th.emplace_back([&, w]() {
                const uint64_t a = nnz * w / nt, b = nnz * (w + 1) / nt;
                memset(hk + a, 0, (b - a) * 8);
                memset(hv + a, 0, (b - a) * 8);
            });
        for (auto& x : th) x.join();
    }
    {
        const int dev = t->device;
        pin_c = std::thread([&, dev]() {
            cudaSetDevice(dev);
            pin_e[0] = cudaMallocHost(&t->h_coords, nnz * 8);
        });
        pin_v = std::thread([&, dev]() {
            cudaSetDevice(dev);
            pin_e[1] = cudaMallocHost(&t->h_values, nnz * 8);
        });
    }
    CountPtrs cp;
    memset(&cp, 0, sizeof(cp));
    {
        uint64_t off = 0;
        for (int n = 0; n < nm; n++) {
            cp.c[n] = counts + off;
            off += L.dims[n];
        }
    }
    std::vector<double> part((size_t)nchunks * g2);
    for (uint64_t c = 0; c < nchunks; c++) {
        const uint64_t o = c * C, n = std::min(C, nnz - o);
        for (int m = 0; m < nm; m++)
            CH_CUDA(cudaMemcpyAsync(dc[m], cidx[m] + o, n * 8, cudaMemcpyDefault, s));
        CH_CUDA(cudaMemcpyAsync(dvin, vals + o, n * 8, cudaMemcpyDefault, s));
        CooPtrs coo;
        memset(&coo, 0, sizeof(coo));
        for (int m = 0; m < nm; m++) coo.c[m] = dc[m];
        const int gk = (int)std::min<uint64_t>((n + 255) / 256, (uint64_t)di.sm_count * 16);
        k_alto_keys<<<gk, 256, 0, s>>>(coo, dvin, n, L, d_tabs, k0, v0, d_bad);
        count_launch();
        CH_CUDA(cudaGetLastError());
        k_coo_counts<<<(int)std::min<uint64_t>((n + RC_THREADS - 1) / RC_THREADS, (uint64_t)di.sm_count * 8),
                       RC_THREADS, 0, s>>>(coo, n, L, cp);
        count_launch();
        CH_CUDA(cudaGetLastError());
        k_sumsq<<<g2, 256, 0, s>>>(v0, n, dpart);
        count_launch();
        CH_CUDA(cudaGetLastError());
        CH_CUDA(cudaMemcpyAsync(part.data() + c * g2, dpart, g2 * sizeof(double), cudaMemcpyDeviceToHost, s));
        bool alt = false;
        int st = radix_sort_pairs(k0, v0, k1, v1, n, 0, L.alto_bits, s, &alt);
        if (st != BLCO_OK) { release(); return st; }
        CH_CUDA(cudaMemcpyAsync(hk + o, alt ? k1 : k0, n * 8, cudaMemcpyDeviceToHost, s));
        CH_CUDA(cudaMemcpyAsync(hv + o, alt ? v1 : v0, n * 8, cudaMemcpyDeviceToHost, s));
        // the next chunk's uploads overwrite the buffers these copies read:
        // stream order keeps them apart
    }
    int bad = 0;
    CH_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    CH_CUDA(cudaStreamSynchronize(s));
    if (bad) {
        release();
        return fail(BLCO_ERR_INVALID, "a coordinate is not below its mode length");
    }
    double ss = 0.0;
    for (double x : part) ss += x; // fixed order: chunk by chunk
    t->norm_sq = ss;
    // Merge the sorted runs into the pinned stream.
    join_pins();
    if (pin_e[0] != cudaSuccess || pin_e[1] != cudaSuccess) {
        release();
        return fail(BLCO_ERR_NOMEM, "pinned host allocation for streamed blocks failed");
    }
    std::vector<uint64_t> rb(nchunks), re(nchunks);
    for (uint64_t c = 0; c < nchunks; c++) {
        rb[c] = c * C;
        re[c] = std::min(nnz, (c + 1) * C);
    }
    // The merge runs on the GPU, one output segment of at most C nonzeros at
    // a time: the segment's slice of every run (found below) is copied in,
    // in run order, and the stable radix sort of the concatenation is the
    // merged order (equal keys keep run order, i.e. input order); its last
    // pass writes BLCO coordinates through the byte table.
    // split(o): per run, how many of its nonzeros come before output rank o:
    // all keys below v, then keys equal to v in run order, v the smallest key
    // with at least o keys at or below it.
    auto split_at = [&](uint64_t o, std::vector<uint64_t>& cut) {
        cut.assign(nchunks, 0);
        if (o >= nnz) {
            for (uint64_t c = 0; c < nchunks; c++) cut[c] = re[c] - rb[c];
            return;
        }
        auto count_le = [&](uint64_t v) {
            uint64_t n = 0;
            for (uint64_t c = 0; c < nchunks; c++) n += (uint64_t)(std::upper_bound(hk + rb[c], hk + re[c], v) - (hk + rb[c]));
            return n;
        };
        uint64_t lo = 0, hi = ~0ull; // count_le(hi) = nnz >= o + 1 > o
        while (lo < hi) {
            const uint64_t mid = lo + (hi - lo) / 2;
            if (count_le(mid) >= o + 1) hi = mid;
            else lo = mid + 1;
        }
        // lo: the key of the nonzero at rank o; the first o nonzeros are the
        // keys below lo and the first ones equal to lo, in run order
        uint64_t rem = o;
        for (uint64_t c = 0; c < nchunks; c++) {
            cut[c] = (uint64_t)(std::lower_bound(hk + rb[c], hk + re[c], lo) - (hk + rb[c]));
            rem -= cut[c];
        }
        for (uint64_t c = 0; c < nchunks && rem; c++) {
            const uint64_t eq = (uint64_t)(std::upper_bound(hk + rb[c], hk + re[c], lo) - (hk + rb[c])) - cut[c];
            const uint64_t take = std::min(eq, rem);
            cut[c] += take;
            rem -= take;
        }
    };
    const uint64_t nseg = (nnz + C - 1) / C;
    std::vector<uint64_t> cut_lo, cut_hi;
    split_at(0, cut_lo);
    const int nbytes = (L.alto_bits + 7) / 8;
    for (uint64_t k = 0; k < nseg; k++) {
        const uint64_t o0 = k * C, o1 = std::min(nnz, o0 + C);
        split_at(o1, cut_hi);
        uint64_t n = 0;
        for (uint64_t c = 0; c < nchunks; c++) {
            const uint64_t len = cut_hi[c] - cut_lo[c];
            if (!len) continue;
            CH_CUDA(cudaMemcpyAsync(k0 + n, hk + rb[c] + cut_lo[c], len * 8, cudaMemcpyHostToDevice, s));
            CH_CUDA(cudaMemcpyAsync(v0 + n, hv + rb[c] + cut_lo[c], len * 8, cudaMemcpyHostToDevice, s));
            n += len;
        }
        if (n != o1 - o0) {
            release();
            return fail(BLCO_ERR_STATE, "streamed encode: merge segment sizes do not add up");
        }
        bool alt = false;
        int st = BLCO_OK;
        if (n > 1 && L.alto_bits > 0) st = radix_sort_pairs(k0, v0, k1, v1, n, 0, L.alto_bits, s, &alt, d_tabs);
        else if (n && L.alto_bits > 0) {
            k_relin<<<1, 32, 0, s>>>(k0, n, d_tabs, nbytes);
            count_launch();
            if (cudaGetLastError() != cudaSuccess) st = fail(BLCO_ERR_CUDA, "k_relin launch failed");
        }
        if (st != BLCO_OK) { release(); return st; }
        CH_CUDA(cudaMemcpyAsync(t->h_coords + o0, alt ? k1 : k0, n * 8, cudaMemcpyDeviceToHost, s));
        CH_CUDA(cudaMemcpyAsync(t->h_values + o0, alt ? v1 : v0, n * 8, cudaMemcpyDeviceToHost, s));
        cut_lo.swap(cut_hi);
    }
    CH_CUDA(cudaStreamSynchronize(s));
    // heavy-row statistics and tables from the row counts
    hk_own.reset();
    hv_own.reset();
    hk = nullptr;
    hv = nullptr;
    int st = build_hot_tables_impl(t, s, counts);
    release();
#undef CH_CUDA
    return st;
}

int encode_impl(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* const* d_cidx,
                const double* d_vals, uint64_t max_block_size, const blco_opts* opts, blco_tensor** out)
{
    *out = nullptr;
    if (!dims || !out || (nnz && (!d_cidx || !d_vals))) return fail(BLCO_ERR_INVALID, "null argument");
    if (nnz >= 0xffffffffull) return fail(BLCO_ERR_UNSUPPORTED, "nnz must be below 2^32-1 for the device encoder");
    blco_tensor* t = new blco_tensor();
    int st = make_layout(nmodes, dims, &t->layout);
    if (st != BLCO_OK) { delete t; return st; }
    for (int n = 0; n < nmodes; n++)
        if (nnz && !d_cidx[n]) { delete t; return fail(BLCO_ERR_INVALID, "null coordinate array"); }
    t->device = opts ? opts->device : 0;
    t->nnz = nnz;
    t->max_block_size = max_block_size;
    uint64_t B = max_block_size ? max_block_size : nnz;
    t->block_count = nnz == 0 ? 0 : (nnz + B - 1) / B;
    t->resident = !(opts && opts->stream_data);
    if (t->layout.wide && !t->resident) {
        delete t;
        return fail(BLCO_ERR_UNSUPPORTED, "keys above 64 bits are encoded resident only (no streamed blocks)");
    }

    auto cleanup_fail = [&](int s) { blco_tensor_free(t); return s; };
    cudaError_t e = cudaSetDevice(t->device);
    if (e != cudaSuccess) return cleanup_fail(cuda_fail(e, "cudaSetDevice", __FILE__, __LINE__));
    cudaStream_t s = pick_stream(t, opts);
    if (!t->resident && !t->layout.wide && nnz > stream_chunk_nnz(opts, nmodes)) {
        // streamed and larger than one chunk of the residency budget
        DeviceInfo cdi;
        if ((st = device_info(t->device, &cdi)) != BLCO_OK) return cleanup_fail(st);
        if ((st = encode_chunked(t, d_cidx, d_vals, s, cdi, stream_chunk_nnz(opts, nmodes))) != BLCO_OK)
            return cleanup_fail(st);
        *out = t;
        return BLCO_OK;
    }
    if (t->layout.wide) {
        DeviceInfo wdi;
        if ((st = device_info(t->device, &wdi)) != BLCO_OK) return cleanup_fail(st);
        if ((st = encode_wide(t, d_cidx, d_vals, s, wdi)) != BLCO_OK) return cleanup_fail(st);
        *out = t;
        return BLCO_OK;
    }

    uint64_t n_alloc = nnz ? nnz : 1;
    uint64_t *k0 = nullptr, *k1 = nullptr;
    double *v0 = nullptr, *v1 = nullptr;
    int* d_bad = nullptr;
    EncTables* d_tabs = nullptr;
    auto free_tmp = [&]() {
        cudaStreamSynchronize(s);
        cudaFree(k1);
        cudaFree(v1);
        cudaFree(d_bad);
        cudaFree(d_tabs);
        k1 = nullptr;
        v1 = nullptr;
        d_bad = nullptr;
        d_tabs = nullptr;
    };
#define ENC_CUDA(call)                                                          \
    do {                                                                        \
        cudaError_t _e = (call);                                                \
        if (_e != cudaSuccess) {                                                \
            int _s = cuda_fail(_e, #call, __FILE__, __LINE__);                  \
            free_tmp();                                                         \
            cudaFree(k0);                                                       \
            cudaFree(v0);                                                       \
            return cleanup_fail(_s);                                            \
        }                                                                       \
    } while (0)
    ENC_CUDA(cudaMalloc(&k0, n_alloc * 8));
    ENC_CUDA(cudaMalloc(&v0, n_alloc * 8));
    ENC_CUDA(cudaMalloc(&k1, n_alloc * 8));
    ENC_CUDA(cudaMalloc(&v1, n_alloc * 8));
    ENC_CUDA(cudaMalloc(&d_bad, sizeof(int)));
    ENC_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(int), s));

    DeviceInfo di;
    if ((st = device_info(t->device, &di)) != BLCO_OK) {
        free_tmp();
        cudaFree(k0);
        cudaFree(v0);
        return cleanup_fail(st);
    }
    bool in_alt = false;
    if (nnz) {
        CooPtrs coo;
        memset(&coo, 0, sizeof(coo));
        for (int n = 0; n < nmodes; n++) coo.c[n] = d_cidx[n];
        int grid = (int)std::min<uint64_t>((nnz + 255) / 256, (uint64_t)di.sm_count * 16);
        EncTables htabs = make_tables(t->layout);
        ENC_CUDA(cudaMalloc(&d_tabs, sizeof(EncTables)));
        ENC_CUDA(cudaMemcpyAsync(d_tabs, &htabs, sizeof(EncTables), cudaMemcpyHostToDevice, s));
        k_alto_keys<<<grid, 256, 0, s>>>(coo, d_vals, nnz, t->layout, d_tabs, k0, v0, d_bad);
        count_launch();
        ENC_CUDA(cudaGetLastError());
        int bad = 0;
        ENC_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, s));
        ENC_CUDA(cudaStreamSynchronize(s));
        if (bad) {
            free_tmp();
            cudaFree(k0);
            cudaFree(v0);
            return cleanup_fail(fail(BLCO_ERR_INVALID, "a coordinate is not below its mode length"));
        }
        // The last pass writes BLCO coordinates (re-linearized keys).  With
        // a key of 0 bits (every mode of length 1) no pass runs and the keys
        // are all 0, which is also the coordinate.
        st = radix_sort_pairs(k0, v0, k1, v1, nnz, 0, t->layout.alto_bits, s, &in_alt, d_tabs);
        if (st == BLCO_OK && nnz <= 1 && t->layout.alto_bits > 0) {
            k_relin<<<1, 32, 0, s>>>(k0, nnz, d_tabs, (t->layout.alto_bits + 7) / 8);
            count_launch();
            if (cudaGetLastError() != cudaSuccess) st = fail(BLCO_ERR_CUDA, "k_relin launch failed");
        }
        if (st != BLCO_OK) {
            free_tmp();
            cudaFree(k0);
            cudaFree(v0);
            return cleanup_fail(st);
        }
        if (in_alt) {
            std::swap(k0, k1);
            std::swap(v0, v1);
        }
        double* partial = reinterpret_cast<double*>(k1); // k1 is free now
        int g2 = std::min(grid, 1024);
        k_sumsq<<<g2, 256, 0, s>>>(v0, nnz, partial);
        count_launch();
        ENC_CUDA(cudaGetLastError());
        std::vector<double> hp(g2);
        ENC_CUDA(cudaMemcpyAsync(hp.data(), partial, g2 * sizeof(double), cudaMemcpyDeviceToHost, s));
        ENC_CUDA(cudaStreamSynchronize(s));
        double ss = 0.0;
        for (double x : hp) ss += x;
        t->norm_sq = ss;
    }
    free_tmp();
    t->d_coords = k0;
    t->d_values = v0;
    k0 = nullptr;
    v0 = nullptr;
    ENC_CUDA(cudaStreamSynchronize(s));
#undef ENC_CUDA
    if ((st = build_hot_tables(t, s)) != BLCO_OK) return cleanup_fail(st);
    if (!t->resident) {
        // Streamed form: the encoded stream moves to pinned host memory and
        // the device copy is released; blocks are copied back per use.
        cudaError_t e1 = cudaMallocHost(&t->h_coords, n_alloc * 8);
        cudaError_t e2 = cudaMallocHost(&t->h_values, n_alloc * 8);
        if (e1 != cudaSuccess || e2 != cudaSuccess)
            return cleanup_fail(fail(BLCO_ERR_NOMEM, "pinned host allocation for streamed blocks failed"));
        BLCO_CUDA(cudaMemcpyAsync(t->h_coords, t->d_coords, nnz * 8, cudaMemcpyDeviceToHost, s));
        BLCO_CUDA(cudaMemcpyAsync(t->h_values, t->d_values, nnz * 8, cudaMemcpyDeviceToHost, s));
        BLCO_CUDA(cudaStreamSynchronize(s));
        cudaFree(t->d_coords);
        cudaFree(t->d_values);
        t->d_coords = nullptr;
        t->d_values = nullptr;
    }
    *out = t;
    return BLCO_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free encoder.
//
// Some callers of this library cannot allocate device memory when they
// encode: a process whose device memory is owned by another allocator (a
// framework's pool, a budgeted service), or code that must not call
// cudaMalloc, which synchronises the device and can fail at a bad time.
// blco_encode_device_noalloc serves them: the caller passes the COO input and
// the two output arrays, and the sort's scratch lives in the file-scope array
// below, which every GPU that loads this library holds until exit.
//
// Limits and sharing: at most BLCO_NOALLOC_MAX_NNZ nonzeros; one array per
// device shared by every call, so calls that overlap on the GPU (other
// streams, other host threads) race and must be serialised by the caller.
// Every call looks up the array's device address (cudaGetSymbolAddress);
// the first call on a device also does the library's set-up there (loading
// its device code), so make that first call before any stream capture.
// Every call synchronises its stream twice: after the copy of the encoder's
// tables from pageable host memory, and to read back the range check.

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = 32ull << 20; // 32 MiB per device
constexpr uint64_t NOALLOC_TILES = (BLCO_NOALLOC_MAX_NNZ + RS_TILE - 1) / RS_TILE;
constexpr uint64_t NOALLOC_COUNTS = (uint64_t)RS_RADIX * NOALLOC_TILES;
constexpr uint64_t NOALLOC_SUMS = (NOALLOC_COUNTS + SC_CHUNK - 1) / SC_CHUNK + 1;
constexpr size_t na_align(size_t x) { return (x + 255) & ~(size_t)255; }
// Scratch layout: alternate keys | alternate values | digit counts | scan
// sums | encoder tables | invalid-coordinate flag.
constexpr size_t NA_K1 = 0;
constexpr size_t NA_V1 = NA_K1 + na_align(BLCO_NOALLOC_MAX_NNZ * 8);
constexpr size_t NA_COUNTS = NA_V1 + na_align(BLCO_NOALLOC_MAX_NNZ * 8);
constexpr size_t NA_SUMS = NA_COUNTS + na_align(NOALLOC_COUNTS * 4);
constexpr size_t NA_TABS = NA_SUMS + na_align(NOALLOC_SUMS * 4);
constexpr size_t NA_BAD = NA_TABS + na_align(sizeof(EncTables));
constexpr size_t NA_END = NA_BAD + 256;
static_assert(NA_END <= NOALLOC_SCRATCH_BYTES, "allocation-free encoder scratch layout exceeds the array");

__device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// The same passes as radix_sort_pairs, with the digit counts and scan sums
// in caller-provided memory.
int radix_sort_pairs_in(uint64_t* k0, double* v0, uint64_t* k1, double* v1, uint64_t n, int end_bit,
                        cudaStream_t s, bool* in_alt, const EncTables* rel_tabs, uint32_t* counts, uint32_t* sums)
{
    *in_alt = false;
    if (n <= 1 || end_bit <= 0) return BLCO_OK;
    const uint32_t ntiles = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
    const uint64_t L = (uint64_t)RS_RADIX * ntiles;
    BLCO_CUDA(cudaFuncSetAttribute(k_rs_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RS_SMEM));
    uint64_t *ki = k0, *ko = k1;
    double *vi = v0, *vo = v1;
    for (int shift = 0; shift < end_bit; shift += 8) {
        k_rs_hist<<<ntiles, RS_THREADS, 0, s>>>(ki, n, shift, counts, ntiles);
        BLCO_CHECK_LAUNCH("k_rs_hist");
        BLCO_TRY(scan_u32(counts, L, sums, s));
        const bool last = shift + 8 >= end_bit;
        k_rs_scatter<<<ntiles, RS_THREADS, RS_SMEM, s>>>(ki, vi, ko, vo, n, shift, counts, ntiles,
                                                         last ? rel_tabs : nullptr, (end_bit + 7) / 8);
        BLCO_CHECK_LAUNCH("k_rs_scatter");
        std::swap(ki, ko);
        std::swap(vi, vo);
        *in_alt = !*in_alt;
    }
    return BLCO_OK;
}

} // namespace

// Device address of g_noalloc_scratch in the current context, looked up on
// every call (a cached address would go stale after a device reset).
static int noalloc_scratch(unsigned char** out)
{
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
    *out = static_cast<unsigned char*>(p);
    return BLCO_OK;
}

int encode_noalloc_impl(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* const* d_cidx,
                        const double* d_vals, uint64_t* d_coords_out, double* d_vals_out, cudaStream_t s)
{
    if (!dims || (nnz && (!d_cidx || !d_vals || !d_coords_out || !d_vals_out)))
        return fail(BLCO_ERR_INVALID, "null argument");
    if (nnz > BLCO_NOALLOC_MAX_NNZ)
        return fail(BLCO_ERR_UNSUPPORTED, "nnz above BLCO_NOALLOC_MAX_NNZ, the limit of the allocation-free encoder");
    Layout L;
    BLCO_TRY(make_layout(nmodes, dims, &L));
    if (L.wide)
        return fail(BLCO_ERR_UNSUPPORTED, "the allocation-free encoder takes keys of at most 64 bits (no block "
                                          "coordinates in its output)");
    for (int n = 0; n < nmodes; n++)
        if (nnz && !d_cidx[n]) return fail(BLCO_ERR_INVALID, "null coordinate array");
    if (nnz == 0) return BLCO_OK;
    int device = 0;
    BLCO_CUDA(cudaGetDevice(&device));
    DeviceInfo di;
    BLCO_TRY(device_info(device, &di));
    unsigned char* base = nullptr;
    BLCO_TRY(noalloc_scratch(&base));
    uint64_t* k1 = reinterpret_cast<uint64_t*>(base + NA_K1);
    double* v1 = reinterpret_cast<double*>(base + NA_V1);
    uint32_t* counts = reinterpret_cast<uint32_t*>(base + NA_COUNTS);
    uint32_t* sums = reinterpret_cast<uint32_t*>(base + NA_SUMS);
    EncTables* tabs = reinterpret_cast<EncTables*>(base + NA_TABS);
    int* bad = reinterpret_cast<int*>(base + NA_BAD);

    // The flag keeps the previous call's value: clear it.
    BLCO_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), s));
    {
        EncTables htabs = make_tables(L);
        BLCO_CUDA(cudaMemcpyAsync(tabs, &htabs, sizeof(EncTables), cudaMemcpyHostToDevice, s));
        // htabs is pageable host memory: make sure the copy has read it.
        BLCO_CUDA(cudaStreamSynchronize(s));
    }
    CooPtrs coo;
    memset(&coo, 0, sizeof(coo));
    for (int n = 0; n < nmodes; n++) coo.c[n] = d_cidx[n];
    const int grid = (int)std::min<uint64_t>((nnz + 255) / 256, (uint64_t)di.sm_count * 16);
    k_alto_keys<<<grid, 256, 0, s>>>(coo, d_vals, nnz, L, tabs, d_coords_out, d_vals_out, bad);
    BLCO_CHECK_LAUNCH("k_alto_keys");
    bool in_alt = false;
    BLCO_TRY(radix_sort_pairs_in(d_coords_out, d_vals_out, k1, v1, nnz, L.alto_bits, s, &in_alt, tabs, counts, sums));
    if (nnz <= 1 && L.alto_bits > 0) {
        k_relin<<<1, 32, 0, s>>>(d_coords_out, nnz, tabs, (L.alto_bits + 7) / 8);
        BLCO_CHECK_LAUNCH("k_relin");
    }
    if (in_alt) {
        BLCO_CUDA(cudaMemcpyAsync(d_coords_out, k1, nnz * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
        BLCO_CUDA(cudaMemcpyAsync(d_vals_out, v1, nnz * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    int bad_h = 0;
    BLCO_CUDA(cudaMemcpyAsync(&bad_h, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    BLCO_CUDA(cudaStreamSynchronize(s));
    if (bad_h) return fail(BLCO_ERR_INVALID, "a coordinate is not below its mode length");
    return BLCO_OK;
}

} // namespace blco
