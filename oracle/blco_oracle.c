/*
 * blco_oracle.c -- CPU oracle (test infrastructure only; see blco_oracle.h).
 *
 * Plain C restatement of the reference's encoder, MTTKRP and GPU CP-ALS
 * arithmetic.  Each function cites the reference lines it follows.
 */
#include "blco_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

uint64_t orc_pdep(uint64_t x, uint64_t mask)
{
    /* include/bitops.hpp:18-29: walk the set bits of mask from the LSB,
     * depositing successive bits of x into them. */
    uint64_t res = 0;
    for (uint64_t b = 1; mask != 0; b += b) {
        if (x & b) res |= mask & (~mask + 1);
        mask &= mask - 1;
    }
    return res;
}

uint64_t orc_pext(uint64_t x, uint64_t mask)
{
    /* include/bitops.hpp:31-41 */
    uint64_t res = 0;
    for (uint64_t b = 1; mask != 0; b += b) {
        if (x & mask & (~mask + 1)) res |= b;
        mask &= mask - 1;
    }
    return res;
}

int orc_mode_bits(uint64_t dim)
{
    if (dim <= 1) return 0;
    return 64 - __builtin_clzll(dim - 1);
}

int orc_alto_masks(int nmodes, const uint64_t* dims, uint64_t* alto_masks)
{
    /* include/alto.hpp:597-695 with po = LSB_FIRST, mo = SHORT_FIRST.
     * The modes are ordered by ascending bit count; the reference sorts at
     * most MAX_NUM_MODES=5 entries with std::sort, which is insertion sort
     * at that size and therefore keeps ties in natural order. */
    int order[ORC_MAX_MODES], bits[ORC_MAX_MODES];
    int total = 0, maxbits = 0;
    if (nmodes < 1 || nmodes > ORC_MAX_MODES) return -1;
    for (int n = 0; n < nmodes; n++) {
        bits[n] = orc_mode_bits(dims[n]);
        order[n] = n;
        total += bits[n];
        if (bits[n] > maxbits) maxbits = bits[n];
        alto_masks[n] = 0;
    }
    if (total > 64) return -1;
    for (int i = 1; i < nmodes; i++) { /* stable insertion sort */
        int m = order[i], j = i - 1;
        while (j >= 0 && bits[order[j]] > bits[m]) { order[j + 1] = order[j]; j--; }
        order[j + 1] = m;
    }
    int shift = 0;
    for (int level = 0; level < maxbits; level++) {
        for (int k = 0; k < nmodes; k++) {
            int m = order[k];
            if (level < bits[m]) alto_masks[m] |= (uint64_t)1 << shift++;
        }
    }
    return total;
}

typedef struct {
    uint64_t key;
    uint64_t idx;
} orc_pair;

static int orc_pair_cmp(const void* a, const void* b)
{
    const orc_pair* x = (const orc_pair*)a;
    const orc_pair* y = (const orc_pair*)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    if (x->idx != y->idx) return x->idx < y->idx ? -1 : 1;
    return 0;
}

int orc_blco_encode(int nmodes, const uint64_t* dims, uint64_t nnz,
                    const uint64_t* cidx, const double* vals,
                    uint64_t max_block_size,
                    uint64_t* coords_out, double* vals_out,
                    uint64_t* mode_masks_out, int* mode_pos_out,
                    uint64_t* alto_masks_out,
                    uint64_t* nblocks_out, uint64_t* block_offsets_out)
{
    uint64_t amask[ORC_MAX_MODES];
    if (orc_alto_masks(nmodes, dims, amask) < 0) return -1;
    for (int n = 0; n < nmodes; n++) {
        if (dims[n] == 0) return -1;
        alto_masks_out[n] = amask[n];
    }

    /* BLCO per-mode masks and shifts, include/blco.hpp:221-233. */
    for (int n = 0; n < nmodes; n++) {
        int b = __builtin_popcountll(amask[n]);
        mode_masks_out[n] = (b >= 64) ? ~(uint64_t)0 : (((uint64_t)1 << b) - 1);
        mode_pos_out[n] = (n == 0) ? 0 : mode_pos_out[n - 1] + __builtin_popcountll(amask[n - 1]);
    }

    /* Linearize (include/alto.hpp:157-175) and sort by ALTO key
     * (include/alto.hpp:704-754). */
    orc_pair* pairs = (orc_pair*)malloc((nnz ? nnz : 1) * sizeof(orc_pair));
    if (!pairs) return -1;
    for (uint64_t i = 0; i < nnz; i++) {
        uint64_t key = 0;
        for (int n = 0; n < nmodes; n++) {
            uint64_t c = cidx[(uint64_t)n * nnz + i];
            if (c >= dims[n]) { free(pairs); return -1; }
            key |= orc_pdep(c, amask[n]);
        }
        pairs[i].key = key;
        pairs[i].idx = i;
    }
    qsort(pairs, nnz, sizeof(orc_pair), orc_pair_cmp);

    /* Re-linearize into concatenated fields, include/blco.hpp:274-286. */
    for (uint64_t i = 0; i < nnz; i++) {
        uint64_t key = pairs[i].key, c = 0;
        for (int n = 0; n < nmodes; n++)
            c |= (orc_pext(key, amask[n]) & mode_masks_out[n]) << mode_pos_out[n];
        coords_out[i] = c;
        vals_out[i] = vals[pairs[i].idx];
    }
    free(pairs);

    /* Blocks, include/blco.hpp:249-321.  With a 64-bit key the upper half is
     * always 0, so every entry is in histogram bucket 0 and the blocks are
     * consecutive max_block_size slices (max_block_size 0 means nnz). */
    uint64_t B = max_block_size ? max_block_size : nnz;
    uint64_t nb = (nnz == 0) ? 0 : (nnz + B - 1) / B;
    *nblocks_out = nb;
    for (uint64_t b = 0; b < nb; b++) block_offsets_out[b] = b * B;
    block_offsets_out[nb] = nnz;
    return 0;
}

/* ---- 128-bit ALTO keys (the cpd128 build, ALTO_MASK_LENGTH=128) ---- */

typedef unsigned __int128 orc_u128;

/* 128-bit deposit / extract, include/bitops.hpp:89-108: the low mask word
 * takes the first popcount(low word) bits of x, the high word the rest. */
static orc_u128 orc_pdep128(uint64_t x, orc_u128 mask)
{
    uint64_t lo = (uint64_t)mask, hi = (uint64_t)(mask >> 64);
    int shift = __builtin_popcountll(lo);
    orc_u128 r = orc_pdep(x, lo);
    if (shift < 64) r |= (orc_u128)orc_pdep(x >> shift, hi) << 64;
    return r;
}

static uint64_t orc_pext128(orc_u128 x, orc_u128 mask)
{
    uint64_t lo = (uint64_t)mask, hi = (uint64_t)(mask >> 64);
    int shift = __builtin_popcountll(lo);
    uint64_t r = orc_pext((uint64_t)x, lo);
    if (shift < 64) r |= orc_pext((uint64_t)(x >> 64), hi) << shift;
    return r;
}

int orc_alto_masks128(int nmodes, const uint64_t* dims, uint64_t* masks_lo, uint64_t* masks_hi)
{
    /* include/alto.hpp:597-695 with a 128-bit LIT: the same ordering and
     * LSB-first round robin as orc_alto_masks, over up to 128 positions. */
    int order[ORC_MAX_MODES], bits[ORC_MAX_MODES];
    int total = 0, maxbits = 0;
    if (nmodes < 1 || nmodes > ORC_MAX_MODES) return -1;
    for (int n = 0; n < nmodes; n++) {
        bits[n] = orc_mode_bits(dims[n]);
        order[n] = n;
        total += bits[n];
        if (bits[n] > maxbits) maxbits = bits[n];
        masks_lo[n] = masks_hi[n] = 0;
    }
    if (total > 128) return -1;
    for (int i = 1; i < nmodes; i++) {
        int m = order[i], j = i - 1;
        while (j >= 0 && bits[order[j]] > bits[m]) { order[j + 1] = order[j]; j--; }
        order[j + 1] = m;
    }
    int shift = 0;
    for (int level = 0; level < maxbits; level++)
        for (int k = 0; k < nmodes; k++) {
            int m = order[k];
            if (level < bits[m]) {
                if (shift < 64) masks_lo[m] |= (uint64_t)1 << shift;
                else masks_hi[m] |= (uint64_t)1 << (shift - 64);
                shift++;
            }
        }
    return total;
}

typedef struct {
    orc_u128 key;
    uint64_t idx;
} orc_pair128;

static int orc_pair128_cmp(const void* a, const void* b)
{
    const orc_pair128* x = (const orc_pair128*)a;
    const orc_pair128* y = (const orc_pair128*)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    if (x->idx != y->idx) return x->idx < y->idx ? -1 : 1;
    return 0;
}

int orc_blco_encode128(int nmodes, const uint64_t* dims, uint64_t nnz,
                       const uint64_t* cidx, const double* vals,
                       uint64_t max_block_size,
                       uint64_t* coords_out, double* vals_out,
                       uint64_t* mode_masks_out, int* mode_pos_out,
                       uint64_t* alto_lo_out, uint64_t* alto_hi_out,
                       uint64_t* nblocks_out, uint64_t* block_offsets_out,
                       uint64_t* block_coords_out)
{
    orc_u128 amask[ORC_MAX_MODES];
    int tbits[ORC_MAX_MODES];
    if (orc_alto_masks128(nmodes, dims, alto_lo_out, alto_hi_out) < 0) return -1;
    for (int n = 0; n < nmodes; n++) {
        if (dims[n] == 0) return -1;
        amask[n] = ((orc_u128)alto_hi_out[n] << 64) | alto_lo_out[n];
    }
    /* Fields hold the bits of each mode that lie in the low key word,
     * include/blco.hpp:222-233. */
    for (int n = 0; n < nmodes; n++) {
        tbits[n] = __builtin_popcountll(alto_lo_out[n]);
        mode_masks_out[n] = (tbits[n] >= 64) ? ~(uint64_t)0 : (((uint64_t)1 << tbits[n]) - 1);
        mode_pos_out[n] = (n == 0) ? 0 : mode_pos_out[n - 1] + tbits[n - 1];
    }
    orc_pair128* pairs = (orc_pair128*)malloc((nnz ? nnz : 1) * sizeof(orc_pair128));
    if (!pairs) return -1;
    for (uint64_t i = 0; i < nnz; i++) {
        orc_u128 key = 0;
        for (int n = 0; n < nmodes; n++) {
            uint64_t c = cidx[(uint64_t)n * nnz + i];
            if (c >= dims[n]) { free(pairs); return -1; }
            key |= orc_pdep128(c, amask[n]);
        }
        pairs[i].key = key;
        pairs[i].idx = i;
    }
    qsort(pairs, nnz, sizeof(orc_pair128), orc_pair128_cmp);
    /* Re-linearize the low-word bits, include/blco.hpp:274-286. */
    for (uint64_t i = 0; i < nnz; i++) {
        uint64_t c = 0;
        for (int n = 0; n < nmodes; n++)
            c |= (orc_pext128(pairs[i].key, amask[n]) & mode_masks_out[n]) << mode_pos_out[n];
        coords_out[i] = c;
        vals_out[i] = vals[pairs[i].idx];
    }
    /* Blocks, include/blco.hpp:244-321: one histogram bucket per value of
     * the upper key word, in increasing order (the sorted order), each split
     * into max_block_size slices; block_coords[n] = pext(upper word, upper
     * mask word of mode n) << (its low-word bit count). */
    uint64_t B = max_block_size ? max_block_size : nnz;
    uint64_t nb = 0;
    for (uint64_t s = 0; s < nnz;) {
        uint64_t up = (uint64_t)(pairs[s].key >> 64), e = s + 1;
        while (e < nnz && (uint64_t)(pairs[e].key >> 64) == up) e++;
        for (uint64_t o = s; o < e; o += B) {
            block_offsets_out[nb] = o;
            for (int n = 0; n < nmodes; n++) {
                uint64_t bc = orc_pext(up, alto_hi_out[n]);
                block_coords_out[nb * nmodes + n] = tbits[n] >= 64 ? 0 : bc << tbits[n];
            }
            nb++;
        }
        s = e;
    }
    block_offsets_out[nb] = nnz;
    *nblocks_out = nb;
    free(pairs);
    return 0;
}

void orc_mttkrp_blco128(int nmodes, const uint64_t* mode_masks, const int* mode_pos, uint64_t nblocks,
                        const uint64_t* block_offsets, const uint64_t* block_coords, const uint64_t* coords,
                        const double* vals, const double* const* factors, int rank, int mode, double* out)
{
    /* Per block, a row index is the field plus the block's coordinate,
     * alt_pext (src/alto_dev.cu:13-16). */
    for (uint64_t b = 0; b < nblocks; b++) {
        const uint64_t* bc = block_coords + b * nmodes;
        for (uint64_t i = block_offsets[b]; i < block_offsets[b + 1]; i++) {
            uint64_t c = coords[i];
            double* o = out + (((c >> mode_pos[mode]) & mode_masks[mode]) | bc[mode]) * (uint64_t)rank;
            for (int r = 0; r < rank; r++) {
                double p = vals[i];
                for (int m = 0; m < nmodes; m++) {
                    if (m == mode) continue;
                    uint64_t rid = ((c >> mode_pos[m]) & mode_masks[m]) | bc[m];
                    p *= factors[m][rid * (uint64_t)rank + r];
                }
                o[r] += p;
            }
        }
    }
}

void orc_mttkrp_coo(int nmodes, uint64_t nnz, const uint64_t* cidx,
                    const double* vals, int rank, const double* const* factors,
                    int mode, double* out)
{
    /* include/cpd.hpp:510-544 */
    double* row = (double*)malloc(sizeof(double) * (size_t)rank);
    for (uint64_t i = 0; i < nnz; i++) {
        for (int r = 0; r < rank; r++) row[r] = vals[i];
        for (int m = 0; m < nmodes; m++) {
            if (m == mode) continue;
            const double* u = factors[m] + cidx[(uint64_t)m * nnz + i] * (uint64_t)rank;
            for (int r = 0; r < rank; r++) row[r] *= u[r];
        }
        double* o = out + cidx[(uint64_t)mode * nnz + i] * (uint64_t)rank;
        for (int r = 0; r < rank; r++) o[r] += row[r];
    }
    free(row);
}

void orc_mttkrp_blco(int nmodes, const uint64_t* mode_masks,
                     const int* mode_pos, uint64_t nnz, const uint64_t* coords,
                     const double* vals, int rank,
                     const double* const* factors, int mode, double* out)
{
    double* row = (double*)malloc(sizeof(double) * (size_t)rank);
    for (uint64_t i = 0; i < nnz; i++) {
        uint64_t c = coords[i];
        for (int r = 0; r < rank; r++) row[r] = vals[i];
        for (int m = 0; m < nmodes; m++) {
            if (m == mode) continue;
            uint64_t rid = (c >> mode_pos[m]) & mode_masks[m];
            const double* u = factors[m] + rid * (uint64_t)rank;
            for (int r = 0; r < rank; r++) row[r] *= u[r];
        }
        uint64_t rid = (c >> mode_pos[mode]) & mode_masks[mode];
        double* o = out + rid * (uint64_t)rank;
        for (int r = 0; r < rank; r++) o[r] += row[r];
    }
    free(row);
}

int orc_pinv_sym(int n, const double* a_in, double* p)
{
    /* Eigen-decomposition A = Q diag(w) Q^T by cyclic Jacobi rotations,
     * then P = Q diag(f(w)) Q^T with f(w) = 1/w when |w| > n*ulp(max|w|),
     * else 0: the cut-off of src/cpd_gpu.cu:484-490 (an SVD of a symmetric
     * matrix has singular values |w|, and V S^-1 U^T = Q diag(1/w) Q^T). */
    size_t nn = (size_t)n * (size_t)n;
    double* a = (double*)malloc(nn * sizeof(double));
    double* q = (double*)malloc(nn * sizeof(double));
    if (!a || !q) { free(a); free(q); return -1; }
    memcpy(a, a_in, nn * sizeof(double));
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) q[i * n + j] = (i == j) ? 1.0 : 0.0;

    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0, tot = 0.0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                double v = a[i * n + j] * a[i * n + j];
                tot += v;
                if (i != j) off += v;
            }
        if (off <= 1e-30 * tot || off == 0.0) break;
        for (int pi = 0; pi < n - 1; pi++) {
            for (int qi = pi + 1; qi < n; qi++) {
                double apq = a[pi * n + qi];
                if (apq == 0.0) continue;
                double app = a[pi * n + pi], aqq = a[qi * n + qi];
                double theta = (aqq - app) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; k++) { /* A <- A J (columns p, q) */
                    double akp = a[k * n + pi], akq = a[k * n + qi];
                    a[k * n + pi] = c * akp - s * akq;
                    a[k * n + qi] = s * akp + c * akq;
                }
                for (int k = 0; k < n; k++) { /* A <- J^T A (rows p, q) */
                    double apk = a[pi * n + k], aqk = a[qi * n + k];
                    a[pi * n + k] = c * apk - s * aqk;
                    a[qi * n + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; k++) { /* Q <- Q J */
                    double qkp = q[k * n + pi], qkq = q[k * n + qi];
                    q[k * n + pi] = c * qkp - s * qkq;
                    q[k * n + qi] = s * qkp + c * qkq;
                }
            }
        }
    }
    double smax = 0.0;
    for (int i = 0; i < n; i++) if (fabs(a[i * n + i]) > smax) smax = fabs(a[i * n + i]);
    double tol = n * (nextafter(smax, smax + 1.0) - smax);
    double* f = (double*)malloc((size_t)n * sizeof(double));
    for (int i = 0; i < n; i++) {
        double w = a[i * n + i];
        f[i] = (fabs(w) > tol) ? 1.0 / w : 0.0;
    }
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            double s = 0.0;
            for (int k = 0; k < n; k++) s += q[i * n + k] * f[k] * q[j * n + k];
            p[i * n + j] = s;
        }
    free(f);
    free(a);
    free(q);
    return 0;
}

static void orc_gram(uint64_t rows, int R, const double* u, double* g)
{
    /* ata_gpu (src/cpd_gpu.cu:547-568): G = U^T U. */
    for (int a = 0; a < R; a++)
        for (int b = 0; b < R; b++) g[a * R + b] = 0.0;
    for (uint64_t i = 0; i < rows; i++) {
        const double* r = u + i * (uint64_t)R;
        for (int a = 0; a < R; a++)
            for (int b = 0; b < R; b++) g[a * R + b] += r[a] * r[b];
    }
}

/* The MTTKRP of one CP-ALS step, over whichever form the caller holds. */
typedef struct {
    int kind; /* 0: BLCO stream, 1: COO */
    const uint64_t* mode_masks;
    const int* mode_pos;
    const uint64_t* coords;
    const uint64_t* cidx;
} orc_mt_src;

static void orc_mt(const orc_mt_src* src, int N, uint64_t nnz, const double* vals, int R,
                   const double* const* factors, int n, double* M)
{
    if (src->kind == 0)
        orc_mttkrp_blco(N, src->mode_masks, src->mode_pos, nnz, src->coords, vals, R, factors, n, M);
    else
        orc_mttkrp_coo(N, nnz, src->cidx, vals, R, factors, n, M);
}

static int orc_cpals_src(int nmodes, const uint64_t* dims, const orc_mt_src* src, uint64_t nnz,
                         const double* vals, int rank, double* const* factors,
                         double* lambda, int maxiter, double tol, double* fits)
{
    const int R = rank, N = nmodes;
    uint64_t maxdim = 0;
    for (int n = 0; n < N; n++) if (dims[n] > maxdim) maxdim = dims[n];

    double* M = (double*)malloc(sizeof(double) * maxdim * (uint64_t)R);
    double* grams[ORC_MAX_MODES];
    double* V = (double*)malloc(sizeof(double) * (size_t)R * R);
    double* P = (double*)malloc(sizeof(double) * (size_t)R * R);
    double* W = (double*)malloc(sizeof(double) * (size_t)R * R);
    double* colsq = (double*)malloc(sizeof(double) * (size_t)R);
    double* mrow = (double*)malloc(sizeof(double) * (size_t)R);

    /* ||X||, src/cpd_gpu.cu:106-109 */
    double xn2 = 0.0;
    for (uint64_t i = 0; i < nnz; i++) xn2 += vals[i] * vals[i];
    double X_norm = sqrt(xn2);

    for (int n = 0; n < N; n++) {
        grams[n] = (double*)malloc(sizeof(double) * (size_t)R * R);
        orc_gram(dims[n], R, factors[n], grams[n]);
    }

    /* Modes by descending length, ties in natural order
     * (src/cpd_gpu.cu:137-139; std::sort of <= 5 entries is stable). */
    int order[ORC_MAX_MODES];
    for (int n = 0; n < N; n++) order[n] = n;
    for (int i = 1; i < N; i++) {
        int m = order[i], j = i - 1;
        while (j >= 0 && dims[order[j]] < dims[m]) { order[j + 1] = order[j]; j--; }
        order[j + 1] = m;
    }

    double fit = 0.0, fit_old = 0.0;
    int it;
    for (it = 0; it < maxiter; it++) {
        for (int k = 0; k < N; k++) {
            int n = order[k];
            uint64_t I = dims[n];
            memset(M, 0, sizeof(double) * I * (uint64_t)R);
            orc_mt(src, N, nnz, vals, R, (const double* const*)factors, n, M);
            /* V = hadamard of the other Grams (src/cpd_gpu.cu:160-163) */
            for (int e = 0; e < R * R; e++) V[e] = 1.0;
            for (int m = 0; m < N; m++)
                if (m != n)
                    for (int e = 0; e < R * R; e++) V[e] *= grams[m][e];
            orc_pinv_sym(R, V, P);
            /* U_n = M P^T (the cublasDgemm of src/cpd_gpu.cu:175). */
            double* U = factors[n];
            for (uint64_t i = 0; i < I; i++) {
                for (int c = 0; c < R; c++) mrow[c] = M[i * R + c];
                for (int c = 0; c < R; c++) {
                    double s = 0.0;
                    for (int kk = 0; kk < R; kk++) s += mrow[kk] * P[c * R + kk];
                    U[i * R + c] = s;
                }
            }
            /* columnwise_normscal (src/cpd_gpu.cu:244-291) */
            for (int c = 0; c < R; c++) colsq[c] = 0.0;
            for (uint64_t i = 0; i < I; i++)
                for (int c = 0; c < R; c++) colsq[c] += U[i * R + c] * U[i * R + c];
            for (int c = 0; c < R; c++) {
                lambda[c] = sqrt(lambda[c] + colsq[c]);
                colsq[c] = (lambda[c] == 0.0) ? 0.0 : 1.0 / lambda[c];
            }
            for (uint64_t i = 0; i < I; i++)
                for (int c = 0; c < R; c++) U[i * R + c] *= colsq[c];
            orc_gram(I, R, U, grams[n]);
        }
        /* kruskal_fit_gpu (src/cpd_gpu.cu:331-384); M holds the MTTKRP of
         * the last mode processed. */
        int lm = order[N - 1];
        double iprod = 0.0;
        for (int c = 0; c < R; c++) colsq[c] = 0.0;
        for (uint64_t i = 0; i < dims[lm]; i++)
            for (int c = 0; c < R; c++) colsq[c] += factors[lm][i * R + c] * M[i * R + c];
        for (int c = 0; c < R; c++) iprod += colsq[c] * lambda[c];
        for (int a = 0; a < R; a++)
            for (int b = 0; b < R; b++) W[a * R + b] = lambda[a] * lambda[b];
        for (int m = 0; m < N; m++)
            for (int e = 0; e < R * R; e++) W[e] *= grams[m][e];
        double na = 0.0;
        for (int e = 0; e < R * R; e++) na += W[e];
        na = sqrt(fabs(na));
        fit = na * na - 2.0 * iprod;
        if (X_norm != 0.0) {
            fit = sqrt(fabs(fit + X_norm * X_norm));
            fit = 1.0 - fit / X_norm;
        }
        if (fits) fits[it] = fit;
        if (fabs(fit - fit_old) < tol || isnan(fit)) { it++; break; }
        fit_old = fit;
    }

    for (int n = 0; n < N; n++) free(grams[n]);
    free(M); free(V); free(P); free(W); free(colsq); free(mrow);
    return it;
}

int orc_cpals(int nmodes, const uint64_t* dims, const uint64_t* mode_masks,
              const int* mode_pos, uint64_t nnz, const uint64_t* coords,
              const double* vals, int rank, double* const* factors,
              double* lambda, int maxiter, double tol, double* fits)
{
    orc_mt_src src = {0, mode_masks, mode_pos, coords, NULL};
    return orc_cpals_src(nmodes, dims, &src, nnz, vals, rank, factors, lambda, maxiter, tol, fits);
}

int orc_cpals_coo(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* cidx,
                  const double* vals, int rank, double* const* factors,
                  double* lambda, int maxiter, double tol, double* fits)
{
    orc_mt_src src = {1, NULL, NULL, NULL, cidx};
    return orc_cpals_src(nmodes, dims, &src, nnz, vals, rank, factors, lambda, maxiter, tol, fits);
}

void orc_kruskal_random_init(int nmodes, const uint64_t* dims, int rank,
                             unsigned int seed, int nthreads,
                             double* const* factors, double* lambda)
{
    /* src/kruskal_model.cpp:93-110 under libgomp's static schedule: with
     * q = n / T and r = n % T, thread t < r gets q+1 entries starting at
     * t*(q+1), thread t >= r gets q entries starting at t*q + r. */
    for (int r = 0; r < rank; r++) lambda[r] = 1.0;
    if (nthreads < 1) nthreads = 1;
    for (int n = 0; n < nmodes; n++) {
        uint64_t total = dims[n] * (uint64_t)rank;
        uint64_t q = total / (uint64_t)nthreads, rem = total % (uint64_t)nthreads;
        for (int t = 0; t < nthreads; t++) {
            uint64_t cnt = q + ((uint64_t)t < rem ? 1 : 0);
            uint64_t start = (uint64_t)t * q + ((uint64_t)t < rem ? (uint64_t)t : rem);
            unsigned int s = seed + (unsigned int)t;
            for (uint64_t i = 0; i < cnt; i++)
                factors[n][start + i] = (double)rand_r(&s) / RAND_MAX;
        }
    }
}
