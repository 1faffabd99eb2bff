// cpals.cu -- CP-ALS on the GPU: the plain FP64 form and the mixed forms
// (FP32 or BF16 gathers, FP64 solve, lambda and fit), resident or streamed
// tensors, one tensor per plan (optionally sharded over ranks: the plan hands
// each mode's MTTKRP to the caller's sum over the ranks), and the batched
// CP-ALS of many small tensors (second half of the file).
//
// Keeps the arithmetic of cpals_blco_dev (src/cpd_gpu.cu:21-242) but runs
// every step as this library's own kernels on one stream, with no host
// round trip inside a mode update (the reference synchronises the host
// about eight times per mode and calls cuBLAS/cuSOLVER):
//   per mode n (descending length order, src/cpd_gpu.cu:137-139)
//     M      = MTTKRP(n)                                  (mttkrp.cu)
//     P      = pinv( hadamard_{m != n} Gram_m )           (k_solve: Cholesky
//              inverse, falling back to a Jacobi eigen pseudoinverse with the
//              reference cut-off n*ulp(s_max), src/cpd_gpu.cu:452-532)
//     U_n    = M P^T, column sums of squares fused         (k_update)
//     lambda = sqrt(lambda + colsq); U_n /= lambda, Gram_n (k_lambda,
//              k_scale_gram; lambda is never reset, src/cpd_gpu.cu:244-291)
//   fit as kruskal_fit_gpu (src/cpd_gpu.cu:331-384)        (k_iprod, k_fit)
// Reductions over rows use per-block partials summed in a fixed order, so
// a given launch shape gives the same bits on every run (the MTTKRP's FP64
// atomics are the one non-deterministic step).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "internal.cuh"

namespace blco {
namespace {

constexpr int DN_THREADS = 256;
constexpr int MAX_SOLVE_R = 96; // k_solve keeps two R x R FP64 buffers in shared memory

// ---------------------------------------------------------------- Gram --
// Partial Gram of rows [beg, end) of a row-major I x R matrix, optionally
// scaling the rows by inv[c] first and writing the scaled rows back.
// Thread tile: TS x TS entries of the R x R result (TS = 4 up to R = 64,
// 8 up to R = 128, so that 256 threads cover the result).
constexpr int GR_CH = 128; // rows staged per step

__device__ __forceinline__ float round_bf16(float x, uint16_t* bits)
{
    uint32_t u = __float_as_uint(x);
    uint32_t r = (u + 0x7fffu + ((u >> 16) & 1u)) & 0xffff0000u;
    *bits = (uint16_t)(r >> 16);
    return __uint_as_float(r);
}

// With BF16OUT the (scaled) factor is rounded to BF16 precision, the rounded
// value is kept in U and its BF16 bits are written to bf16_out, so the Gram,
// the fit and the MTTKRP gathers all see the same factor.
template <typename T, bool SCALE, int TS, bool BF16OUT = false>
__global__ __launch_bounds__(DN_THREADS) void k_gram(T* __restrict__ U, uint64_t I, int R,
                                                     const double* __restrict__ inv, double* __restrict__ partials,
                                                     uint16_t* __restrict__ bf16_out = nullptr)
{
    // The Gram is symmetric: thread tiles cover the TS x TS blocks (i, j)
    // with i <= j only, and each is written to both halves at the end.  Rows
    // are staged in shared memory as FP64 (converted once), so the inner
    // loop is 2*TS shared loads per TS*TS FMAs.
    extern __shared__ __align__(16) double gs[];
    double* red = gs;                                 // R x R reduction buffer
    double* tile = gs + R * R;                        // GR_CH x R
    const int nb = (R + TS - 1) / TS;                 // blocks per side
    const int ntile = nb * (nb + 1) / 2;
    const int groups = max(1, DN_THREADS / ntile);
    const int tid = threadIdx.x;
    const int g = tid / ntile, e = tid % ntile;
    const bool active = g < groups && tid < groups * ntile;
    int bi = 0, rem = e;
    while (rem >= nb - bi) {
        rem -= nb - bi;
        bi++;
    }
    const int a0 = bi * TS, b0 = (bi + rem) * TS;
    double acc[TS][TS];
#pragma unroll
    for (int x = 0; x < TS; x++)
#pragma unroll
        for (int y = 0; y < TS; y++) acc[x][y] = 0.0;

    const uint64_t per = (I + gridDim.x - 1) / gridDim.x;
    const uint64_t beg = per * blockIdx.x, end = min(I, beg + per);
    for (uint64_t r0 = beg; r0 < end; r0 += GR_CH) {
        const int nr = (int)min((uint64_t)GR_CH, end - r0);
        __syncthreads();
        for (int k = tid; k < nr * R; k += DN_THREADS) {
            T v = U[r0 * R + k];
            if (SCALE) v = (T)((double)v * inv[k % R]);
            if constexpr (BF16OUT) {
                uint16_t b;
                v = (T)round_bf16((float)v, &b);
                bf16_out[r0 * R + k] = b;
            }
            if (SCALE || BF16OUT) U[r0 * R + k] = v;
            tile[k] = (double)v;
        }
        __syncthreads();
        if (active) {
            // Blocks that reach past R read columns clamped to R-1 and are
            // discarded at the end.
            for (int r = g; r < nr; r += groups) {
                const double* row = tile + r * R;
                double va[TS], vb[TS];
#pragma unroll
                for (int x = 0; x < TS; x++) {
                    va[x] = row[min(a0 + x, R - 1)];
                    vb[x] = row[min(b0 + x, R - 1)];
                }
#pragma unroll
                for (int x = 0; x < TS; x++)
#pragma unroll
                    for (int y = 0; y < TS; y++) acc[x][y] += va[x] * vb[y];
            }
        }
    }
    // Reduce the row groups in a fixed order; mirror the off-diagonal blocks.
    for (int k = tid; k < R * R; k += DN_THREADS) red[k] = 0.0;
    __syncthreads();
    for (int gg = 0; gg < groups; gg++) {
        if (active && g == gg) {
#pragma unroll
            for (int x = 0; x < TS; x++)
#pragma unroll
                for (int y = 0; y < TS; y++)
                    if (a0 + x < R && b0 + y < R) {
                        red[(a0 + x) * R + b0 + y] += acc[x][y];
                        if (a0 != b0) red[(b0 + y) * R + a0 + x] += acc[x][y];
                    }
        }
        __syncthreads();
    }
    for (int k = tid; k < R * R; k += DN_THREADS) partials[(size_t)blockIdx.x * R * R + k] = red[k];
}

// out[k] = sum_b partials[b][k], b ascending.
__global__ void k_sum_partials(const double* __restrict__ partials, int nblocks, int len, double* __restrict__ out)
{
    // a warp per entry: lane l sums partials l, l + 32, ... in order, then
    // the lanes combine in a fixed tree (the same bits on every run)
    const int lane = threadIdx.x & 31;
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (int k = w; k < len; k += nw) {
        double s = 0.0;
        for (int b = lane; b < nblocks; b += 32) s += partials[(size_t)b * len + k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) out[k] = s;
    }
}

// -------------------------------------------------------------- update --
// U[i][c] = sum_k M[i][k] * P[c][k] (the cublasDgemm of src/cpd_gpu.cu:175
// applied to the column-major pseudoinverse), plus per-block column sums of
// squares of U.  A warp computes a row; lane c owns columns c, c+32, ...
constexpr int UP_MAXC = 4; // R <= 128

template <typename TM, typename T>
__global__ __launch_bounds__(DN_THREADS) void k_update(const TM* __restrict__ M, const double* __restrict__ P,
                                                       T* __restrict__ U, uint64_t I, int R,
                                                       double* __restrict__ colsq_partials)
{
    extern __shared__ __align__(16) double us[];
    double* csq = us;                   // [warps][R]
    double* PT = us + (DN_THREADS / 32) * R; // PT[k][c] = P[c][k]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = DN_THREADS / 32;
    for (int k = tid; k < R * R; k += DN_THREADS) {
        int c = k / R, kk = k % R;
        PT[kk * R + c] = P[k];
    }
    __syncthreads();
    double sq[UP_MAXC];
#pragma unroll
    for (int j = 0; j < UP_MAXC; j++) sq[j] = 0.0;
    const uint64_t per = (I + gridDim.x - 1) / gridDim.x;
    const uint64_t beg = per * blockIdx.x, end = min(I, beg + per);
    for (uint64_t i = beg + warp; i < end; i += nw) {
        const TM* mrow = M + i * R;
        double mreg[UP_MAXC];
#pragma unroll
        for (int j = 0; j < UP_MAXC; j++) mreg[j] = (lane + 32 * j < R) ? (double)mrow[lane + 32 * j] : 0.0;
        double acc[UP_MAXC];
#pragma unroll
        for (int j = 0; j < UP_MAXC; j++) acc[j] = 0.0;
#pragma unroll
        for (int kb = 0; kb < UP_MAXC; kb++) {
            if (32 * kb >= R) break;
            const int kn = min(32, R - 32 * kb);
            for (int kk = 0; kk < kn; kk++) {
                const int k = 32 * kb + kk;
                double mk = __shfl_sync(0xffffffffu, mreg[kb], kk);
#pragma unroll
                for (int j = 0; j < UP_MAXC; j++) {
                    int c = lane + 32 * j;
                    if (c < R) acc[j] += mk * PT[k * R + c];
                }
            }
        }
#pragma unroll
        for (int j = 0; j < UP_MAXC; j++) {
            int c = lane + 32 * j;
            if (c < R) {
                const T u = (T)acc[j];
                U[i * R + c] = u;
                sq[j] += (double)u * (double)u;
            }
        }
    }
#pragma unroll
    for (int j = 0; j < UP_MAXC; j++) {
        int c = lane + 32 * j;
        if (c < R) csq[warp * R + c] = sq[j];
    }
    __syncthreads();
    for (int c = tid; c < R; c += DN_THREADS) {
        double s = 0.0;
        for (int w = 0; w < nw; w++) s += csq[w * R + c];
        colsq_partials[(size_t)blockIdx.x * R + c] = s;
    }
}

// Register-tiled form of k_update for R in {16, 32, 64} (U 16-byte
// aligned).  The product is formed in FP64 whatever the storage type T: the
// pseudoinverse of an ill-conditioned Hadamard product of Grams turns FP32
// rounding in this step into fit errors well above 1e-5.
template <int R>
struct UpdShape {
    static constexpr int CG = R / 4;            // column groups: 4 columns of U per thread
    static constexpr int RG = DN_THREADS / CG;  // row groups: 4 rows of U per thread
    static constexpr int TR = 4 * RG;           // rows of M per tile
    static constexpr int TRP = TR + 2;          // padded row stride of the transposed tile (even: 16-byte reads)
    static constexpr int NL = TR * R / DN_THREADS; // elements of M each thread loads per tile
    static constexpr size_t SMEM = ((size_t)R * R + (size_t)R * TRP + (size_t)RG * R) * sizeof(double);
};

template <typename TM, typename T, int R>
__global__ __launch_bounds__(DN_THREADS, 2) void k_update_tiled(const TM* __restrict__ M, const double* __restrict__ P,
                                                                T* __restrict__ U, uint64_t I,
                                                                double* __restrict__ colsq_partials)
{
    // U = M P^T in FP64, tile by tile: TR rows of M staged transposed in
    // shared memory (MsT[k][row]), each thread a 4 x 4 block of U, so every
    // k step is four 16-byte shared loads (4 rows of M, 4 columns of P^T) for
    // 16 FMAs; the next tile's M is loaded into registers while this one is
    // multiplied.  Column sums of squares of the stored U ride along.
    using S = UpdShape<R>;
    extern __shared__ __align__(16) double us[];
    double* PT = us;                  // [R][R], PT[k][c] = P[c][k]
    double* MsT = PT + R * R;         // [R][TRP]
    double* csq = MsT + R * S::TRP;   // [RG][R]
    const int tid = threadIdx.x, rg = tid / S::CG, cg = tid % S::CG;
    for (int k = tid; k < R * R; k += DN_THREADS) {
        const int c = k / R, kk = k % R;
        PT[kk * R + c] = P[k];
    }
    double sq[4] = {0.0, 0.0, 0.0, 0.0};
    const uint64_t ntile = (I + S::TR - 1) / S::TR;
    const uint64_t per = (ntile + gridDim.x - 1) / gridDim.x;
    const uint64_t t_beg = per * blockIdx.x, t_end = min(ntile, t_beg + per);
    double nxt[S::NL];
    auto load = [&](uint64_t t) {
        const uint64_t base = t * S::TR * (uint64_t)R, lim = I * (uint64_t)R;
#pragma unroll
        for (int i = 0; i < S::NL; i++) {
            const uint64_t e = base + tid + (uint64_t)i * DN_THREADS;
            nxt[i] = e < lim ? (double)M[e] : 0.0;
        }
    };
    if (t_beg < t_end) load(t_beg);
    for (uint64_t t = t_beg; t < t_end; t++) {
        __syncthreads(); // the previous tile's MsT reads are done
#pragma unroll
        for (int i = 0; i < S::NL; i++) {
            const int e = tid + i * DN_THREADS;
            MsT[(e % R) * S::TRP + e / R] = nxt[i];
        }
        __syncthreads();
        if (t + 1 < t_end) load(t + 1);
        double acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) acc[i][j] = 0.0;
#pragma unroll 8
        for (int k = 0; k < R; k++) {
            const double2 m01 = *reinterpret_cast<const double2*>(MsT + k * S::TRP + 4 * rg);
            const double2 m23 = *reinterpret_cast<const double2*>(MsT + k * S::TRP + 4 * rg + 2);
            const double2 p01 = *reinterpret_cast<const double2*>(PT + k * R + 4 * cg);
            const double2 p23 = *reinterpret_cast<const double2*>(PT + k * R + 4 * cg + 2);
            const double m[4] = {m01.x, m01.y, m23.x, m23.y};
            const double pv[4] = {p01.x, p01.y, p23.x, p23.y};
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fma(m[i], pv[j], acc[i][j]);
        }
        const uint64_t r0 = t * S::TR + 4 * rg;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            if (r0 + i < I) {
                T u[4];
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    u[j] = (T)acc[i][j];
                    sq[j] += (double)u[j] * (double)u[j];
                }
                T* dst = U + (r0 + i) * R + 4 * cg;
                if constexpr (sizeof(T) == 4) {
                    *reinterpret_cast<float4*>(dst) = make_float4(u[0], u[1], u[2], u[3]);
                } else {
                    reinterpret_cast<double2*>(dst)[0] = make_double2(u[0], u[1]);
                    reinterpret_cast<double2*>(dst)[1] = make_double2(u[2], u[3]);
                }
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 4; j++) csq[rg * R + 4 * cg + j] = sq[j];
    __syncthreads();
    for (int c = tid; c < R; c += DN_THREADS) {
        double x = 0.0;
        for (int g = 0; g < S::RG; g++) x += csq[g * R + c];
        colsq_partials[(size_t)blockIdx.x * R + c] = x;
    }
}

// lambda_c = sqrt(lambda_c + sum_b colsq[b][c]); inv_c = 1/lambda_c (0 if 0).
__global__ void k_lambda(const double* __restrict__ colsq_partials, int nblocks, int R, double* __restrict__ lambda,
                         double* __restrict__ inv)
{
    for (int c = threadIdx.x; c < R; c += blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nblocks; b++) s += colsq_partials[(size_t)b * R + c];
        double l = sqrt(lambda[c] + s);
        lambda[c] = l;
        inv[c] = l == 0.0 ? 0.0 : 1.0 / l;
    }
}

// --------------------------------------------------------------- solve --
struct GramPtrs {
    const double* g[BLCO_MAX_MODES];
};

// P = pinv(V), V = hadamard of the Grams of every mode except `skip`.
// One CTA.  Cholesky V = L L^T; P = L^-T L^-1.  If a pivot is not clearly
// positive, the pseudoinverse is taken from a cyclic Jacobi
// eigen-decomposition V = Q diag(w) Q^T instead, dropping |w| <= R*ulp(max|w|)
// as the reference does for its SVD.
//
// cond (may be null) receives an estimate of V's condition number: the
// squared ratio of the largest to the smallest Cholesky pivot (a lower
// bound), or, on the eigen path, max|w| over the smallest |w| (infinity
// when an eigenvalue is exactly zero).  With
// pinv, the eigen path is taken whatever the pivots (the reference's
// pseudoinverse, src/cpd_gpu.cu:452-532, in every case).
__device__ void solve_body(GramPtrs gp, int nmodes, int skip, int R, double* __restrict__ Pout,
                           int* __restrict__ used_eigen, double* __restrict__ cond, bool pinv)
{
    extern __shared__ __align__(16) double ss[];
    double* A = ss;          // R x R
    double* W = ss + R * R;  // R x R
    __shared__ double fw[MAX_SOLVE_R];
    __shared__ int bad;
    __shared__ double maxdiag;
    const int tid = threadIdx.x, RR = R * R;
    for (int k = tid; k < RR; k += DN_THREADS) {
        double v = 1.0;
        for (int m = 0; m < nmodes; m++)
            if (m != skip) v *= gp.g[m][k];
        A[k] = v;
    }
    if (tid == 0) bad = pinv ? 1 : 0;
    __syncthreads();
    if (tid == 0) {
        double md = 0.0;
        for (int i = 0; i < R; i++) md = fmax(md, fabs(A[i * R + i]));
        maxdiag = md;
    }
    __syncthreads();
    const double piv_tol = 64.0 * R * 2.220446049250313e-16 * maxdiag;
    for (int k = 0; k < R && !bad; k++) {
        if (tid == 0) {
            double d = A[k * R + k];
            if (!(d > piv_tol)) bad = 1;
            A[k * R + k] = sqrt(fmax(d, 0.0));
        }
        __syncthreads();
        if (bad) break;
        const double dk = A[k * R + k];
        for (int i = k + 1 + tid; i < R; i += DN_THREADS) A[i * R + k] /= dk;
        __syncthreads();
        const int n = R - k - 1;
        for (int e = tid; e < n * n; e += DN_THREADS) {
            int i = k + 1 + e / n, j = k + 1 + e % n;
            if (j <= i) A[i * R + j] -= A[i * R + k] * A[j * R + k];
        }
        __syncthreads();
    }
    if (!bad) {
        if (cond && tid == 0) {
            double lo = A[0], hi = A[0];
            for (int i = 1; i < R; i++) lo = fmin(lo, A[i * R + i]), hi = fmax(hi, A[i * R + i]);
            *cond = (hi / lo) * (hi / lo);
        }
        // W = L^-1 (lower), column j by forward substitution.
        for (int j = tid; j < R; j += DN_THREADS) {
            for (int i = 0; i < j; i++) W[i * R + j] = 0.0;
            for (int i = j; i < R; i++) {
                double s = (i == j) ? 1.0 : 0.0;
                for (int k = j; k < i; k++) s -= A[i * R + k] * W[k * R + j];
                W[i * R + j] = s / A[i * R + i];
            }
        }
        __syncthreads();
        for (int e = tid; e < RR; e += DN_THREADS) {
            int a = e / R, b = e % R, k0 = max(a, b);
            double s = 0.0;
            for (int k = k0; k < R; k++) s += W[k * R + a] * W[k * R + b];
            Pout[e] = s;
        }
        if (tid == 0) *used_eigen = 0;
        return;
    }
    // ---- Jacobi eigen fallback: A <- V (recomputed), W <- I.
    __syncthreads();
    for (int e = tid; e < RR; e += DN_THREADS) {
        double v = 1.0;
        for (int m = 0; m < nmodes; m++)
            if (m != skip) v *= gp.g[m][e];
        A[e] = v;
        W[e] = (e / R == e % R) ? 1.0 : 0.0;
    }
    __syncthreads();
    __shared__ double off_s, tot_s;
    for (int sweep = 0; sweep < 60; sweep++) {
        if (tid == 0) {
            double off = 0.0, tot = 0.0;
            for (int e = 0; e < RR; e++) {
                double v = A[e] * A[e];
                tot += v;
                if (e / R != e % R) off += v;
            }
            off_s = off;
            tot_s = tot;
        }
        __syncthreads();
        if (off_s <= 1e-30 * tot_s || off_s == 0.0) break;
        for (int pi = 0; pi < R - 1; pi++) {
            for (int qi = pi + 1; qi < R; qi++) {
                const double apq = A[pi * R + qi];
                if (apq == 0.0) continue; // uniform across threads (read before any write)
                const double app = A[pi * R + pi], aqq = A[qi * R + qi];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                __syncthreads();
                for (int k = tid; k < R; k += DN_THREADS) {
                    double akp = A[k * R + pi], akq = A[k * R + qi];
                    A[k * R + pi] = c * akp - s * akq;
                    A[k * R + qi] = s * akp + c * akq;
                    double qkp = W[k * R + pi], qkq = W[k * R + qi];
                    W[k * R + pi] = c * qkp - s * qkq;
                    W[k * R + qi] = s * qkp + c * qkq;
                }
                __syncthreads();
                for (int k = tid; k < R; k += DN_THREADS) {
                    double apk = A[pi * R + k], aqk = A[qi * R + k];
                    A[pi * R + k] = c * apk - s * aqk;
                    A[qi * R + k] = s * apk + c * aqk;
                }
                __syncthreads();
            }
        }
        __syncthreads(); // every thread has read off_s before thread 0 rewrites it
    }
    __shared__ double smax;
    if (tid == 0) {
        double m = 0.0;
        for (int i = 0; i < R; i++) m = fmax(m, fabs(A[i * R + i]));
        smax = m;
    }
    __syncthreads();
    const double tol = R * (nextafter(smax, smax + 1.0) - smax);
    for (int i = tid; i < R; i += DN_THREADS) {
        double w = A[i * R + i];
        fw[i] = fabs(w) > tol ? 1.0 / w : 0.0;
    }
    __syncthreads();
    if (cond && tid == 0) {
        // every eigenvalue counts, the dropped ones too: a numerically
        // singular V reports (near) infinity, not the kept part's ratio
        double lo = smax;
        for (int i = 0; i < R; i++) lo = fmin(lo, fabs(A[i * R + i]));
        *cond = smax == 0.0 ? 0.0 : lo > 0.0 ? smax / lo : HUGE_VAL;
    }
    for (int e = tid; e < RR; e += DN_THREADS) {
        int a = e / R, b = e % R;
        double s = 0.0;
        for (int k = 0; k < R; k++) s += W[a * R + k] * fw[k] * W[b * R + k];
        Pout[e] = s;
    }
    if (tid == 0) *used_eigen = 1;
}

__global__ __launch_bounds__(DN_THREADS) void k_solve(GramPtrs gp, int nmodes, int skip, int R,
                                                      double* __restrict__ Pout, int* __restrict__ used_eigen,
                                                      double* __restrict__ cond, int pinv)
{
    solve_body(gp, nmodes, skip, R, Pout, used_eigen, cond, pinv != 0);
}

// ----------------------------------------------------------------- fit --
// Per-block column sums of U[i][c] * M[i][c] (columnwise_inner_product,
// src/cpd_gpu.cu:307-330).
template <typename T, typename TM>
__global__ __launch_bounds__(DN_THREADS) void k_iprod(const T* __restrict__ U, const TM* __restrict__ M,
                                                      uint64_t I, int R, double* __restrict__ partials)
{
    extern __shared__ __align__(16) double ip[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = DN_THREADS / 32;
    double s[UP_MAXC];
#pragma unroll
    for (int j = 0; j < UP_MAXC; j++) s[j] = 0.0;
    const uint64_t per = (I + gridDim.x - 1) / gridDim.x;
    const uint64_t beg = per * blockIdx.x, end = min(I, beg + per);
    for (uint64_t i = beg + warp; i < end; i += nw) {
#pragma unroll
        for (int j = 0; j < UP_MAXC; j++) {
            int c = lane + 32 * j;
            if (c < R) s[j] += (double)U[i * R + c] * (double)M[i * R + c];
        }
    }
#pragma unroll
    for (int j = 0; j < UP_MAXC; j++) {
        int c = lane + 32 * j;
        if (c < R) ip[warp * R + c] = s[j];
    }
    __syncthreads();
    for (int c = tid; c < R; c += DN_THREADS) {
        double t = 0.0;
        for (int w = 0; w < nw; w++) t += ip[w * R + c];
        partials[(size_t)blockIdx.x * R + c] = t;
    }
}

// fit = 1 - sqrt(| ||A||^2 - 2 <X,A> + ||X||^2 |) / ||X|| (src/cpd_gpu.cu:331-384)
// Block-wide sum of one value per thread (blockDim.x == DN_THREADS).
__device__ double block_sum(double v, double* red)
{
    const int tid = threadIdx.x;
    red[tid] = v;
    __syncthreads();
    for (int o = DN_THREADS / 2; o; o >>= 1) {
        if (tid < o) red[tid] += red[tid + o];
        __syncthreads();
    }
    const double r = red[0];
    __syncthreads();
    return r;
}

// fit from <X, A> (iprod), the Grams and lambda; every thread returns it.
__device__ double fit_body(double iprod, GramPtrs gp, int nmodes, int R, const double* __restrict__ lambda,
                           double xnorm, double* red)
{
    double na = 0.0;
    for (int e = threadIdx.x; e < R * R; e += DN_THREADS) {
        double v = lambda[e / R] * lambda[e % R];
        for (int m = 0; m < nmodes; m++) v *= gp.g[m][e];
        na += v;
    }
    na = block_sum(na, red);
    double norm_a = sqrt(fabs(na));
    double fit = norm_a * norm_a - 2.0 * iprod;
    if (xnorm != 0.0) {
        fit = sqrt(fabs(fit + xnorm * xnorm));
        fit = 1.0 - fit / xnorm;
    }
    return fit;
}

__global__ void k_fit(const double* __restrict__ ipart, int nblocks, GramPtrs gp, int nmodes, int R,
                      const double* __restrict__ lambda, double xnorm, double* __restrict__ fit_out)
{
    __shared__ double red[DN_THREADS];
    const int tid = threadIdx.x;
    // iprod
    double ip = 0.0;
    for (int c = tid; c < R; c += blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nblocks; b++) s += ipart[(size_t)b * R + c];
        ip += s * lambda[c];
    }
    const double iprod = block_sum(ip, red);
    const double fit = fit_body(iprod, gp, nmodes, R, lambda, xnorm, red);
    if (tid == 0) fit_out[0] = fit;
}

int grid_rows(uint64_t I, int sm)
{
    uint64_t g = (I + 63) / 64;
    return (int)std::max<uint64_t>(1, std::min<uint64_t>(g, (uint64_t)sm * 2));
}

} // namespace
} // namespace blco

struct blco_cpals_plan {
    blco_tensor* t = nullptr;
    int R = 0, N = 0;
    blco_reduce_fn reduce = nullptr; // sharded CP-ALS: sum of the MTTKRP over the ranks
    void* reduce_ctx = nullptr;
    double* U[BLCO_MAX_MODES] = {};   // caller's FP64 factors
    double* lambda = nullptr;         // caller's FP64 lambda
    double* M = nullptr;              // MTTKRP result (FP64, plain form)
    // mixed form working set
    bool mixed = false;
    int gather_dtype = BLCO_DTYPE_F64;
    float* Uf[BLCO_MAX_MODES] = {};   // FP32 working factors
    void* Ub[BLCO_MAX_MODES] = {};    // BF16 gather copies (BF16 gathers only)
    float* Mf = nullptr;              // MTTKRP result (FP32)
    bool m64[BLCO_MAX_MODES] = {};    // mixed form: this mode's MTTKRP result is in M (FP64), not Mf
    const float* vals32 = nullptr;
    blco::MttkrpArgs sched[BLCO_MAX_MODES] = {}; // per-mode schedule (kernel, hot_chunk, interleave)
    blco::StreamRing* ring = nullptr; // streamed tensors: device block buffers
    bool gram_tc = false;             // mixed form: Grams on the tensor cores
    double* tc_partials = nullptr;    // gram_tc_max_ctas x R x R
    int* d_err = nullptr;             // set by a timed-out tensor-core wait
    double* grams[BLCO_MAX_MODES] = {};
    double* P = nullptr;
    double* partials = nullptr; // max(grid) * R * R
    double* inv = nullptr;      // R
    double* fit = nullptr;      // 1
    int* used_eigen = nullptr;
    int order[BLCO_MAX_MODES] = {};
    double cond[BLCO_MAX_MODES] = {}; // condition estimate of each mode's last solve
    bool promoted = false;            // a mixed plan that continues in FP64
    bool mixed_updated = false;       // a factor has been updated in the mixed form
    uint64_t dev_bytes = 0;           // device bytes: caller's factors and lambda, workspace, ring
    double xnorm = 0.0;
    double fit_old = 0.0;
    int iters_run = 0;
    blco_opts opts;
    cudaStream_t s = nullptr;
    int sm = 148;
    cudaEvent_t ev[2 * BLCO_MAX_MODES] = {};
    double mttkrp_ms[BLCO_MAX_MODES] = {};
    int mttkrp_calls = 0;
};

namespace blco {
namespace {

__global__ void k_f64_to_f32(const double* __restrict__ in, float* __restrict__ out, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

__global__ void k_f32_to_f64(const float* __restrict__ in, double* __restrict__ out, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = (double)in[i];
}

int plan_free(blco_cpals_plan* p)
{
    if (!p) return BLCO_OK;
    if (p->s) cudaStreamSynchronize(p->s);
    cudaFree(p->M);
    cudaFree(p->Mf);
    for (int n = 0; n < BLCO_MAX_MODES; n++) {
        cudaFree(p->grams[n]);
        cudaFree(p->Uf[n]);
        cudaFree(p->Ub[n]);
    }
    cudaFree(p->P);
    cudaFree(p->partials);
    cudaFree(p->inv);
    cudaFree(p->fit);
    cudaFree(p->used_eigen);
    cudaFree(p->tc_partials);
    cudaFree(p->d_err);
    stream_ring_destroy(p->ring);
    for (auto& e : p->ev)
        if (e) cudaEventDestroy(e);
    delete p;
    return BLCO_OK;
}

template <typename T>
int gram_launch(blco_cpals_plan* p, T* U, uint64_t I, const double* inv, double* G, uint16_t* bf16_out = nullptr)
{
    const int R = p->R;
    int grid = grid_rows(I, p->sm);
    size_t smem = (size_t)R * R * sizeof(double) + (size_t)GR_CH * R * sizeof(double);
    void (*fn)(T*, uint64_t, int, const double*, double*, uint16_t*);
    if (bf16_out) {
        if (R <= 64) fn = inv ? k_gram<T, true, 4, true> : k_gram<T, false, 4, true>;
        else fn = inv ? k_gram<T, true, 8, true> : k_gram<T, false, 8, true>;
    } else {
        if (R <= 64) fn = inv ? k_gram<T, true, 4> : k_gram<T, false, 4>;
        else fn = inv ? k_gram<T, true, 8> : k_gram<T, false, 8>;
    }
    BLCO_CUDA(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    fn<<<grid, DN_THREADS, smem, p->s>>>(U, I, R, inv, p->partials, bf16_out);
    BLCO_CHECK_LAUNCH("k_gram");
    k_sum_partials<<<(R * R * 32 + 255) / 256, 256, 0, p->s>>>(p->partials, grid, R * R, G);
    BLCO_CHECK_LAUNCH("k_sum_partials");
    return BLCO_OK;
}

// Standalone Gram G = U^T U (FP64 result) of a device FP32 matrix.
int gram_f32_impl(float* U, uint64_t I, int R, double* G, bool tensor_cores, int sm, cudaStream_t s)
{
    double* parts = nullptr;
    int* d_err = nullptr;
    const int maxp = std::max(gram_tc_max_ctas(sm), grid_rows(I, sm));
    cudaError_t e = cudaMalloc(&parts, (size_t)maxp * R * R * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemsetAsync(d_err, 0, sizeof(int), s);
    int st = e == cudaSuccess ? BLCO_OK : cuda_fail(e, "Gram buffers", __FILE__, __LINE__);
    int np = 0;
    if (st == BLCO_OK) {
        if (tensor_cores) {
            st = gram_tc_launch(U, I, R, nullptr, nullptr, parts, sm, d_err, s, &np);
        } else {
            np = grid_rows(I, sm);
            const size_t smem = (size_t)R * R * sizeof(double) + (size_t)GR_CH * R * sizeof(double);
            auto fn = R <= 64 ? k_gram<float, false, 4> : k_gram<float, false, 8>;
            e = cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e == cudaSuccess) {
                fn<<<np, DN_THREADS, smem, s>>>(U, I, R, nullptr, parts, nullptr);
                count_launch();
                e = cudaGetLastError();
            }
            if (e != cudaSuccess) st = cuda_fail(e, "k_gram", __FILE__, __LINE__);
        }
    }
    if (st == BLCO_OK) {
        k_sum_partials<<<(R * R * 32 + 255) / 256, 256, 0, s>>>(parts, np, R * R, G);
        count_launch();
        int herr = 0;
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_fail(e, "Gram", __FILE__, __LINE__);
        else if (herr) st = fail(BLCO_ERR_TIMEOUT, "tensor-core Gram: an MMA completion wait timed out");
    }
    cudaStreamSynchronize(s);
    cudaFree(parts);
    cudaFree(d_err);
    return st;
}

// The mixed form's Gram on the tensor cores (gram_tc.cu).
int gram_launch_tc(blco_cpals_plan* p, float* U, uint64_t I, const double* inv, double* G, uint16_t* bf16_out)
{
    const int R = p->R;
    int np = 0;
    BLCO_TRY(gram_tc_launch(U, I, R, inv, bf16_out, p->tc_partials, p->sm, p->d_err, p->s, &np));
    k_sum_partials<<<(R * R * 32 + 255) / 256, 256, 0, p->s>>>(p->tc_partials, np, R * R, G);
    BLCO_CHECK_LAUNCH("k_sum_partials");
    return BLCO_OK;
}

template <typename TM, typename T>
int update_launch(blco_cpals_plan* p, const TM* M, T* U, uint64_t I, int grid)
{
    const int R = p->R;
    if ((R == 16 || R == 32 || R == 64) && reinterpret_cast<uintptr_t>(U) % 16 == 0) {
        const size_t smem = R == 16 ? UpdShape<16>::SMEM : R == 32 ? UpdShape<32>::SMEM : UpdShape<64>::SMEM;
        void (*fn)(const TM*, const double*, T*, uint64_t, double*) =
            R == 16 ? k_update_tiled<TM, T, 16> : R == 32 ? k_update_tiled<TM, T, 32> : k_update_tiled<TM, T, 64>;
        BLCO_CUDA(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        fn<<<grid, DN_THREADS, smem, p->s>>>(M, p->P, U, I, p->partials);
    } else {
        size_t smem = (size_t)(R * R + (DN_THREADS / 32) * R) * sizeof(double);
        BLCO_CUDA(cudaFuncSetAttribute(k_update<TM, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_update<TM, T><<<grid, DN_THREADS, smem, p->s>>>(M, p->P, U, I, R, p->partials);
    }
    BLCO_CHECK_LAUNCH("k_update");
    return BLCO_OK;
}

int conv_grid(uint64_t n, int sm) { return (int)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)sm * 8)); }

int promote_fp64(blco_cpals_plan* p, bool from_f32 = true);
double guard_of(const blco_cpals_plan* p);

int mode_update(blco_cpals_plan* p, int n)
{
    blco_tensor* t = p->t;
    const int R = p->R, N = p->N;
    const uint64_t I = t->layout.dims[n];
    MttkrpArgs a;
    memset(&a, 0, sizeof(a));
    a.coords = t->d_coords;
    a.nnz = t->nnz;
    a.mode = n;
    a.rank = R;
    a.kernel = p->sched[n].kernel;
    a.hot_chunk = p->sched[n].hot_chunk;
    a.interleave = p->sched[n].interleave;
    a.thread_cf = p->opts.thread_cf;
    if (p->mixed) {
        a.vals = p->vals32;
        for (int m = 0; m < N; m++)
            a.factors[m] = p->gather_dtype == BLCO_DTYPE_BF16 ? (const void*)p->Ub[m] : (const void*)p->Uf[m];
        a.factor_dtype = p->gather_dtype;
        a.out = p->M;
        a.out64 = 1;
        // The fibre schedule sums rows in FP64 and keeps the result in FP64
        // for the update; wide keys do the same and round once below.
        p->m64[n] = !t->layout.wide && t->resident && fibre_route(t, a);
        if (t->layout.wide || p->m64[n]) {
            BLCO_CUDA(cudaMemsetAsync(p->M, 0, I * R * sizeof(double), p->s));
        } else {
            BLCO_CUDA(cudaMemsetAsync(p->Mf, 0, I * R * sizeof(float), p->s));
            a.out = p->Mf;
            a.out64 = 0;
        }
    } else {
        BLCO_CUDA(cudaMemsetAsync(p->M, 0, I * R * sizeof(double), p->s));
        a.vals = t->d_values;
        for (int m = 0; m < N; m++) a.factors[m] = p->U[m];
        a.out = p->M;
        a.factor_dtype = BLCO_DTYPE_F64;
    }
    BLCO_CUDA(cudaEventRecord(p->ev[2 * n], p->s));
    if (t->resident) BLCO_TRY(mttkrp_launch(t, a, p->s));
    else BLCO_TRY(mttkrp_streamed_ring(t, a, p->ring, p->s)); // blocks copied through the plan's ring
    if (p->reduce) {
        // sharded tensor: sum this mode's MTTKRP over the ranks (the one exchange)
        const bool f64 = !p->mixed || a.out64;
        if (p->reduce(p->reduce_ctx, f64 ? (void*)p->M : (void*)p->Mf, I * (uint64_t)R,
                      f64 ? BLCO_DTYPE_F64 : BLCO_DTYPE_F32, (void*)p->s) != 0)
            return fail(BLCO_ERR_CUDA, "the MTTKRP sum over the ranks failed");
    }
    if (p->mixed && t->layout.wide) {
        k_f64_to_f32<<<conv_grid(I * R, p->sm), 256, 0, p->s>>>(p->M, p->Mf, I * R);
        BLCO_CHECK_LAUNCH("k_f64_to_f32");
    }
    BLCO_CUDA(cudaEventRecord(p->ev[2 * n + 1], p->s));

    GramPtrs gp;
    memset(&gp, 0, sizeof(gp));
    for (int m = 0; m < N; m++) gp.g[m] = p->grams[m];
    size_t ssmem = 2 * (size_t)R * R * sizeof(double);
    BLCO_CUDA(cudaFuncSetAttribute(k_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ssmem));
    k_solve<<<1, DN_THREADS, ssmem, p->s>>>(gp, N, n, R, p->P, p->used_eigen, p->fit + 1 + n,
                                            p->opts.solve == BLCO_SOLVE_PINV);
    BLCO_CHECK_LAUNCH("k_solve");
    if (p->mixed && guard_of(p) > 0.0) {
        // The guard reads this mode's estimate before any factor is updated
        // with it: above the guard, the plan continues in FP64 and this mode
        // starts again (MTTKRP and solve in FP64).
        double c = 0.0;
        BLCO_CUDA(cudaMemcpyAsync(&c, p->fit + 1 + n, sizeof(double), cudaMemcpyDeviceToHost, p->s));
        BLCO_CUDA(cudaStreamSynchronize(p->s));
        if (!(c <= guard_of(p))) {
            // before the first mixed update the caller's FP64 factors are still current
            BLCO_TRY(promote_fp64(p, p->mixed_updated));
            return mode_update(p, n);
        }
    }

    int grid = grid_rows(I, p->sm);
    int ust;
    if (p->mixed) p->mixed_updated = true;
    if (p->mixed && p->m64[n]) ust = update_launch<double, float>(p, p->M, p->Uf[n], I, grid);
    else if (p->mixed) ust = update_launch<float, float>(p, p->Mf, p->Uf[n], I, grid);
    else ust = update_launch<double, double>(p, p->M, p->U[n], I, grid);
    BLCO_TRY(ust);
    k_lambda<<<1, 128, 0, p->s>>>(p->partials, grid, R, p->lambda, p->inv);
    BLCO_CHECK_LAUNCH("k_lambda");
    if (p->mixed) {
        uint16_t* b = p->gather_dtype == BLCO_DTYPE_BF16 ? (uint16_t*)p->Ub[n] : nullptr;
        if (p->gram_tc) BLCO_TRY(gram_launch_tc(p, p->Uf[n], I, p->inv, p->grams[n], b));
        else BLCO_TRY(gram_launch<float>(p, p->Uf[n], I, p->inv, p->grams[n], b));
    } else {
        BLCO_TRY(gram_launch<double>(p, p->U[n], I, p->inv, p->grams[n]));
    }
    return BLCO_OK;
}

int fit_launch(blco_cpals_plan* p)
{
    const int R = p->R, N = p->N;
    const int lm = p->order[N - 1];
    const uint64_t I = p->t->layout.dims[lm];
    int grid = grid_rows(I, p->sm);
    size_t smem = (size_t)(DN_THREADS / 32) * R * sizeof(double);
    if (p->mixed && p->m64[lm])
        k_iprod<float, double><<<grid, DN_THREADS, smem, p->s>>>(p->Uf[lm], p->M, I, R, p->partials);
    else if (p->mixed)
        k_iprod<float, float><<<grid, DN_THREADS, smem, p->s>>>(p->Uf[lm], p->Mf, I, R, p->partials);
    else k_iprod<double, double><<<grid, DN_THREADS, smem, p->s>>>(p->U[lm], p->M, I, R, p->partials);
    BLCO_CHECK_LAUNCH("k_iprod");
    GramPtrs gp;
    memset(&gp, 0, sizeof(gp));
    for (int m = 0; m < N; m++) gp.g[m] = p->grams[m];
    k_fit<<<1, DN_THREADS, 0, p->s>>>(p->partials, grid, gp, N, R, p->lambda, p->xnorm, p->fit);
    BLCO_CHECK_LAUNCH("k_fit");
    return BLCO_OK;
}

// A mixed plan continues in FP64: the FP32 working factors are copied into
// the caller's FP64 arrays, which the plain form works on from here, and
// every Gram is formed again from them.  Taken when the R x R system is too
// ill-conditioned for the FP32 working set: the rounding of the factors and
// of the MTTKRP grows with the condition number through the solve.
// (At plan creation the caller's arrays still hold the FP64 initial
// factors: from_f32 = false keeps them.)
int promote_fp64(blco_cpals_plan* p, bool from_f32)
{
    for (int n = 0; n < p->N && from_f32; n++) {
        const uint64_t I = p->t->layout.dims[n];
        k_f32_to_f64<<<conv_grid(I * p->R, p->sm), 256, 0, p->s>>>(p->Uf[n], p->U[n], I * p->R);
        BLCO_CHECK_LAUNCH("k_f32_to_f64");
    }
    p->mixed = false;
    p->gather_dtype = BLCO_DTYPE_F64;
    p->promoted = true;
    for (int n = 0; n < p->N; n++)
        BLCO_TRY(gram_launch<double>(p, p->U[n], p->t->layout.dims[n], nullptr, p->grams[n]));
    return BLCO_OK;
}

double guard_of(const blco_cpals_plan* p) { return p->opts.guard_cond == 0.0 ? BLCO_GUARD_COND : p->opts.guard_cond; }

// Condition estimates of every mode's R x R system from the current Grams
// into p->cond (the solves' P is discarded).
int initial_condition(blco_cpals_plan* p)
{
    const int R = p->R, N = p->N;
    GramPtrs gp;
    memset(&gp, 0, sizeof(gp));
    for (int m = 0; m < N; m++) gp.g[m] = p->grams[m];
    size_t ssmem = 2 * (size_t)R * R * sizeof(double);
    BLCO_CUDA(cudaFuncSetAttribute(k_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ssmem));
    for (int n = 0; n < N; n++) {
        k_solve<<<1, DN_THREADS, ssmem, p->s>>>(gp, N, n, R, p->P, p->used_eigen, p->fit + 1 + n,
                                                p->opts.solve == BLCO_SOLVE_PINV);
        BLCO_CHECK_LAUNCH("k_solve");
    }
    double c[BLCO_MAX_MODES];
    BLCO_CUDA(cudaMemcpyAsync(c, p->fit + 1, N * sizeof(double), cudaMemcpyDeviceToHost, p->s));
    BLCO_CUDA(cudaStreamSynchronize(p->s));
    for (int n = 0; n < N; n++) p->cond[n] = c[n];
    return BLCO_OK;
}

// Mixed form: FP32 working factors back into the caller's FP64 arrays.
int export_factors(blco_cpals_plan* p)
{
    if (!p->mixed) return BLCO_OK;
    for (int n = 0; n < p->N; n++) {
        const uint64_t len = p->t->layout.dims[n] * (uint64_t)p->R;
        k_f32_to_f64<<<conv_grid(len, p->sm), 256, 0, p->s>>>(p->Uf[n], p->U[n], len);
        BLCO_CHECK_LAUNCH("k_f32_to_f64");
    }
    return BLCO_OK;
}

} // namespace

// Self-check of the tensor-core Gram's bounded wait: one launch on a small
// matrix that issues no MMA and no commit (so its wait on the completion
// barrier runs out after 64 polls), then an ordinary launch on the same
// device.  *timeout_status: what the first reported (BLCO_ERR_TIMEOUT
// expected); *after_status: the second's status, BLCO_OK when it ran and its
// Gram is exact (the first freed its TMEM and left the context usable).
int gram_tc_timeout_check(int device, int* timeout_status, int* after_status)
{
    BLCO_CUDA(cudaSetDevice(device));
    int sm = 0;
    BLCO_CUDA(cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, device));
    const int R = 8;
    const uint64_t I = 200;
    float* U = nullptr;
    double* parts = nullptr;
    double* G = nullptr;
    int* d_err = nullptr;
    cudaStream_t s = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&U, I * R * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&parts, (size_t)gram_tc_max_ctas(sm) * R * R * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&G, (size_t)R * R * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_err, sizeof(int));
    std::vector<float> h(I * R);
    for (uint64_t k = 0; k < I * R; k++) h[k] = (float)((int)(k % 7) - 3); // small integers: an exact Gram
    if (e == cudaSuccess) e = cudaMemcpy(U, h.data(), I * R * sizeof(float), cudaMemcpyHostToDevice);
    int st = e == cudaSuccess ? BLCO_OK : cuda_fail(e, "Gram self-check buffers", __FILE__, __LINE__);
    for (int pass = 0; pass < 2 && st == BLCO_OK; pass++) {
        int herr = 0, np = 0;
        e = cudaMemsetAsync(d_err, 0, sizeof(int), s);
        if (e != cudaSuccess) { st = cuda_fail(e, "memset", __FILE__, __LINE__); break; }
        st = gram_tc_launch(U, I, R, nullptr, nullptr, parts, sm, d_err, s, &np, pass == 0 ? 64u : 0u,
                            pass == 0 ? 1 : 0);
        if (st != BLCO_OK) break;
        k_sum_partials<<<(R * R * 32 + 255) / 256, 256, 0, s>>>(parts, np, R * R, G);
        count_launch();
        e = cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) { st = cuda_fail(e, "Gram self-check", __FILE__, __LINE__); break; }
        int res = herr ? BLCO_ERR_TIMEOUT : BLCO_OK;
        if (pass == 1 && res == BLCO_OK) {
            std::vector<double> g(R * R);
            e = cudaMemcpy(g.data(), G, g.size() * sizeof(double), cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) { st = cuda_fail(e, "Gram self-check", __FILE__, __LINE__); break; }
            for (int a = 0; a < R && res == BLCO_OK; a++)
                for (int c = 0; c < R; c++) {
                    double want = 0.0;
                    for (uint64_t k = 0; k < I; k++) want += (double)h[k * R + a] * h[k * R + c];
                    if (g[a * R + c] != want) {
                        res = fail(BLCO_ERR_CUDA, "tensor-core Gram self-check: the Gram after the timeout is wrong");
                        break;
                    }
                }
        }
        *(pass == 0 ? timeout_status : after_status) = res;
    }
    if (s) cudaStreamSynchronize(s);
    cudaFree(U);
    cudaFree(parts);
    cudaFree(G);
    cudaFree(d_err);
    if (s) cudaStreamDestroy(s);
    return st;
}

int gram_f32(float* U, uint64_t I, int R, double* G, bool tensor_cores, int sm, cudaStream_t s)
{
    return gram_f32_impl(U, I, R, G, tensor_cores, sm, s);
}

int plan_create(blco_tensor* t, int rank, double* const* d_factors, double* d_lambda, const blco_opts* opts,
                blco_cpals_plan** out)
{
    *out = nullptr;
    if (!t || !d_factors || !d_lambda) return fail(BLCO_ERR_INVALID, "null argument");
    if (rank < 1 || rank > MAX_SOLVE_R) return fail(BLCO_ERR_UNSUPPORTED, "CP-ALS rank must be 1..96");
    if (t->layout.wide && opts && opts->precision == BLCO_PRECISION_MIXED_BF16)
        return fail(BLCO_ERR_UNSUPPORTED, "CP-ALS with keys above 64 bits: FP64 or mixed FP32 (no BF16 gathers)");
    blco_cpals_plan* p = new blco_cpals_plan();
    p->t = t;
    p->R = rank;
    p->N = t->layout.nmodes;
    p->lambda = d_lambda;
    if (opts) p->opts = *opts;
    else blco_opts_init(&p->opts);
    DeviceInfo di;
    int st = device_info(t->device, &di);
    if (st != BLCO_OK) { plan_free(p); return st; }
    p->sm = di.sm_count;
    p->s = pick_stream(t, opts);
    uint64_t maxdim = 0;
    for (int n = 0; n < p->N; n++) {
        p->U[n] = d_factors[n];
        maxdim = std::max(maxdim, t->layout.dims[n]);
    }
    const int R = rank;
    int gmax = std::max(grid_rows(maxdim, p->sm), 1);
#define PC(call)                                                               \
    do {                                                                       \
        cudaError_t _e = (call);                                               \
        if (_e != cudaSuccess) {                                               \
            int _s = cuda_fail(_e, #call, __FILE__, __LINE__);                 \
            plan_free(p);                                                      \
            return _s;                                                         \
        }                                                                      \
    } while (0)
    // device bytes of the plan: the caller's FP64 factors and lambda, then
    // every buffer below (a streamed tensor's ring gets what the residency
    // budget leaves)
    for (int n = 0; n < p->N; n++) p->dev_bytes += t->layout.dims[n] * (uint64_t)R * sizeof(double);
    p->dev_bytes += (uint64_t)R * sizeof(double);
#define PCA(ptr, bytes)                                                        \
    do {                                                                       \
        PC(cudaMalloc((ptr), (bytes)));                                        \
        p->dev_bytes += (uint64_t)(bytes);                                     \
    } while (0)
    p->mixed = p->opts.precision != BLCO_PRECISION_FP64;
    p->gather_dtype = p->opts.precision == BLCO_PRECISION_MIXED_BF16 ? BLCO_DTYPE_BF16
                      : p->mixed                                     ? BLCO_DTYPE_F32
                                                                     : BLCO_DTYPE_F64;
    if (p->mixed) {
        // tensor-core Grams up to rank 64 (the kernel's limit) unless the
        // caller asks for the CUDA cores
        p->gram_tc = p->opts.gram_tensor_cores >= 0 && R <= 64;
        if (p->gram_tc) {
            PCA(&p->tc_partials, (size_t)gram_tc_max_ctas(p->sm) * R * R * sizeof(double));
            PCA(&p->d_err, sizeof(int));
            PC(cudaMemsetAsync(p->d_err, 0, sizeof(int), p->s));
        }
        PCA(&p->Mf, std::max<uint64_t>(maxdim, 1) * R * sizeof(float));
        // FP64 result of the wide-key and fibre schedules
        PCA(&p->M, std::max<uint64_t>(maxdim, 1) * R * sizeof(double));
        for (int n = 0; n < p->N; n++) {
            const uint64_t len = t->layout.dims[n] * (uint64_t)R;
            PCA(&p->Uf[n], len * sizeof(float));
            if (p->gather_dtype == BLCO_DTYPE_BF16) PCA(&p->Ub[n], len * 2);
        }
    } else {
        PCA(&p->M, std::max<uint64_t>(maxdim, 1) * R * sizeof(double));
    }
    for (int n = 0; n < p->N; n++) PCA(&p->grams[n], (size_t)R * R * sizeof(double));
    PCA(&p->P, (size_t)R * R * sizeof(double));
    PCA(&p->partials, (size_t)gmax * R * R * sizeof(double));
    PCA(&p->inv, (size_t)R * sizeof(double));
    // fit, then the condition estimate of every mode's solve: read together
    PCA(&p->fit, (1 + BLCO_MAX_MODES) * sizeof(double));
    PC(cudaMemsetAsync(p->fit, 0, (1 + BLCO_MAX_MODES) * sizeof(double), p->s));
    PCA(&p->used_eigen, sizeof(int));
    for (auto& e : p->ev) PC(cudaEventCreate(&e));
#undef PCA
#undef PC
    if (!t->resident) {
        // the ring of block buffers holds what the budget leaves
        const uint64_t budget = p->opts.residency_bytes ? p->opts.residency_bytes : (8ull << 30);
        // two pieces of at least 4096 nonzeros (smaller pieces are valid
        // but leave each copy and kernel launch-bound)
        const uint64_t min_ring = 2 * 16 * std::min<uint64_t>(t->nnz, 4096);
        if (budget < p->dev_bytes + min_ring) {
            plan_free(p);
            return fail(BLCO_ERR_NOMEM, "the residency budget does not cover the plan's factors and workspace "
                                        "and two block buffers");
        }
        st = stream_ring_create(t, budget - p->dev_bytes, &p->ring);
        if (st != BLCO_OK) { plan_free(p); return st; }
        p->dev_bytes += stream_ring_bytes(p->ring);
    }
    p->xnorm = std::sqrt(t->norm_sq);
    if (p->mixed) {
        // streamed: 4-byte values copied per block from a pinned FP32 copy
        st = t->resident ? values_f32(t, p->s, &p->vals32) : host_values_f32(t);
        if (st != BLCO_OK) { plan_free(p); return st; }
    }
    for (int n = 0; n < p->N; n++) {
        const uint64_t len = t->layout.dims[n] * (uint64_t)R;
        if (p->mixed) {
            k_f64_to_f32<<<conv_grid(len, p->sm), 256, 0, p->s>>>(p->U[n], p->Uf[n], len);
            count_launch();
            uint16_t* b = p->gather_dtype == BLCO_DTYPE_BF16 ? (uint16_t*)p->Ub[n] : nullptr;
            st = p->gram_tc ? gram_launch_tc(p, p->Uf[n], t->layout.dims[n], nullptr, p->grams[n], b)
                            : gram_launch<float>(p, p->Uf[n], t->layout.dims[n], nullptr, p->grams[n], b);
        } else {
            st = gram_launch<double>(p, p->U[n], t->layout.dims[n], nullptr, p->grams[n]);
        }
        if (st != BLCO_OK) { plan_free(p); return st; }
    }
    // A mixed plan whose initial R x R systems are already too ill-conditioned
    // for its FP32 working set runs in FP64 from the start.
    if (p->mixed && guard_of(p) > 0.0) {
        st = initial_condition(p);
        double worst = 0.0;
        for (int n = 0; n < p->N; n++) worst = std::max(worst, p->cond[n]);
        if (st == BLCO_OK && !(worst <= guard_of(p))) st = promote_fp64(p, false);
        if (st != BLCO_OK) { plan_free(p); return st; }
    }
    // Per-mode MTTKRP schedules, resolved once (kernels 20 and 21 may time
    // the autotuner's sweep here).
    for (int n = 0; n < p->N && st == BLCO_OK; n++)
        st = resolve_schedule(t, n, R, p->gather_dtype, p->opts.kernel, p->s, &p->sched[n]);
    if (st != BLCO_OK) { plan_free(p); return st; }
    // the stream copies the modes' schedules read (compressed fibres, or
    // heavy rows and cold stream), built now rather than inside the first
    // iteration; the modes' fibre builds share one scratch
    FibScratch fsc;
    for (int n = 0; n < p->N && st == BLCO_OK; n++) {
        if (!t->resident) continue;
        const int k = mttkrp_select_kernel(t, n, R, p->sched[n].kernel, p->gather_dtype);
        if (k == BLCO_KERNEL_FIBRE &&
            (p->sched[n].kernel == BLCO_KERNEL_FIBRE || p->sched[n].kernel == BLCO_KERNEL_AUTO))
            st = build_fibre_copy(t, n, p->s, &fsc);
        else if (k == BLCO_KERNEL_LVL2) // the heavy-row schedule's stream copies, likewise
            st = build_mode_copies(t, n, p->s);
    }
    fib_scratch_free(fsc);
    if (st != BLCO_OK) { plan_free(p); return st; }
    // Descending mode length, ties in natural order (src/cpd_gpu.cu:137-139).
    for (int n = 0; n < p->N; n++) p->order[n] = n;
    std::stable_sort(p->order, p->order + p->N,
                     [&](int a, int b) { return t->layout.dims[a] > t->layout.dims[b]; });
    cudaError_t e = cudaStreamSynchronize(p->s);
    if (e != cudaSuccess) {
        int s2 = cuda_fail(e, "plan setup", __FILE__, __LINE__);
        plan_free(p);
        return s2;
    }
    *out = p;
    return BLCO_OK;
}

int plan_iterate(blco_cpals_plan* p, int iters, double tol, double* fits, int* iters_done, bool verbose)
{
    if (iters_done) *iters_done = 0;
    int done = 0;
    cudaEvent_t it0, it1;
    BLCO_CUDA(cudaEventCreate(&it0));
    BLCO_CUDA(cudaEventCreate(&it1));
    int st = BLCO_OK;
    for (int it = 0; it < iters; it++) {
        cudaEventRecord(it0, p->s);
        for (int k = 0; k < p->N && st == BLCO_OK; k++) st = mode_update(p, p->order[k]);
        if (st == BLCO_OK) st = fit_launch(p);
        if (st != BLCO_OK) break;
        cudaEventRecord(it1, p->s);
        double fc[1 + BLCO_MAX_MODES];
        cudaError_t e = cudaMemcpyAsync(fc, p->fit, (1 + p->N) * sizeof(double), cudaMemcpyDeviceToHost, p->s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(p->s);
        if (e != cudaSuccess) { st = cuda_fail(e, "CP-ALS iteration", __FILE__, __LINE__); break; }
        const double fit = fc[0];
        double worst = 0.0;
        for (int n = 0; n < p->N; n++) {
            p->cond[n] = fc[1 + n];
            worst = std::max(worst, fc[1 + n]);
        }
        const double guard = guard_of(p);
        if (p->mixed && guard > 0.0 && !(worst <= guard) && (st = promote_fp64(p, p->mixed_updated)) != BLCO_OK) break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, it0, it1);
        for (int n = 0; n < p->N; n++) {
            float m = 0.f;
            cudaEventElapsedTime(&m, p->ev[2 * n], p->ev[2 * n + 1]);
            p->mttkrp_ms[n] += m;
        }
        p->mttkrp_calls++;
        if (fits) fits[it] = fit;
        done++;
        if (verbose)
            printf("--> Iter %3d: f = %0.6f f-delta = %0.6f time = %0.6f, (s)\n", p->iters_run, fit, fit - p->fit_old,
                   ms / 1000.0f);
        p->iters_run++;
        bool stop = std::fabs(fit - p->fit_old) < tol || std::isnan(fit);
        p->fit_old = fit;
        if (stop) break;
    }
    cudaEventDestroy(it0);
    cudaEventDestroy(it1);
    if (st == BLCO_OK && p->gram_tc) {
        int herr = 0;
        cudaError_t e = cudaMemcpyAsync(&herr, p->d_err, sizeof(int), cudaMemcpyDeviceToHost, p->s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(p->s);
        if (e != cudaSuccess) st = cuda_fail(e, "tensor-core Gram status", __FILE__, __LINE__);
        else if (herr) st = fail(BLCO_ERR_TIMEOUT, "tensor-core Gram: an MMA completion wait timed out");
    }
    if (st == BLCO_OK) st = export_factors(p);
    if (iters_done) *iters_done = done;
    return st;
}

int plan_destroy(blco_cpals_plan* p) { return plan_free(p); }

int cpals_host(blco_tensor* t, int rank, double* const* factors, double* lambda, int maxiter, double tol,
               const blco_opts* opts, double* fit_out, double* fits, int* iters_out)
{
    if (!t || !factors || !lambda) return fail(BLCO_ERR_INVALID, "null argument");
    // forms the plan rejects are rejected before any factor is copied
    if (opts && opts->precision == BLCO_PRECISION_MIXED_BF16 && t->layout.wide)
        return fail(BLCO_ERR_UNSUPPORTED, "CP-ALS with keys above 64 bits: FP64 or mixed FP32 (no BF16 gathers)");
    const int N = t->layout.nmodes;
    cudaStream_t s = pick_stream(t, opts);
    double* dU[BLCO_MAX_MODES] = {};
    double* dl = nullptr;
    int st = BLCO_OK;
    auto cleanup = [&]() {
        cudaStreamSynchronize(s);
        for (int n = 0; n < N; n++) cudaFree(dU[n]);
        cudaFree(dl);
    };
    for (int n = 0; n < N && st == BLCO_OK; n++) {
        size_t b = t->layout.dims[n] * (size_t)rank * sizeof(double);
        cudaError_t e = cudaMalloc(&dU[n], b);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dU[n], factors[n], b, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) st = cuda_fail(e, "factor upload", __FILE__, __LINE__);
    }
    if (st == BLCO_OK) {
        cudaError_t e = cudaMalloc(&dl, rank * sizeof(double));
        if (e == cudaSuccess) e = cudaMemcpyAsync(dl, lambda, rank * sizeof(double), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) st = cuda_fail(e, "lambda upload", __FILE__, __LINE__);
    }
    blco_cpals_plan* p = nullptr;
    if (st == BLCO_OK) st = plan_create(t, rank, dU, dl, opts, &p);
    const bool verbose = opts && opts->verbose;
    if (st == BLCO_OK && verbose)
        printf("Begin CP-ALS decomposition, rank=%d maxiter=%d tolerance=%f\n", rank, maxiter, tol);
    int done = 0;
    if (st == BLCO_OK) st = plan_iterate(p, maxiter, tol, fits, &done, verbose);
    if (st == BLCO_OK) {
        if (fit_out) *fit_out = p->fit_old;
        if (verbose) printf("Final fit: %0.9f\n", p->fit_old);
        for (int n = 0; n < N && st == BLCO_OK; n++) {
            cudaError_t e = cudaMemcpyAsync(factors[n], dU[n], t->layout.dims[n] * (size_t)rank * sizeof(double),
                                            cudaMemcpyDeviceToHost, s);
            if (e != cudaSuccess) st = cuda_fail(e, "factor download", __FILE__, __LINE__);
        }
        cudaError_t e = cudaMemcpyAsync(lambda, dl, rank * sizeof(double), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess && st == BLCO_OK) st = cuda_fail(e, "lambda download", __FILE__, __LINE__);
    }
    if (iters_out) *iters_out = done;
    plan_free(p);
    cleanup();
    return st;
}

int plan_set_reduce(blco_cpals_plan* p, blco_reduce_fn fn, void* ctx)
{
    if (!p) return fail(BLCO_ERR_INVALID, "null plan");
    p->reduce = fn;
    p->reduce_ctx = ctx;
    return BLCO_OK;
}

int plan_set_norm_sq(blco_cpals_plan* p, double norm_sq)
{
    if (!p) return fail(BLCO_ERR_INVALID, "null plan");
    if (!(norm_sq >= 0.0)) return fail(BLCO_ERR_INVALID, "norm_sq must be non-negative");
    p->xnorm = std::sqrt(norm_sq);
    return BLCO_OK;
}

int plan_device_bytes(const blco_cpals_plan* p, uint64_t* bytes)
{
    if (!p || !bytes) return fail(BLCO_ERR_INVALID, "null argument");
    *bytes = p->dev_bytes;
    return BLCO_OK;
}

int plan_condition(const blco_cpals_plan* p, double* cond, int* promoted)
{
    if (!p) return fail(BLCO_ERR_INVALID, "null plan");
    if (cond)
        for (int n = 0; n < p->N; n++) cond[n] = p->cond[n];
    if (promoted) *promoted = p->promoted ? 1 : 0;
    return BLCO_OK;
}

int plan_mttkrp_ms(const blco_cpals_plan* p, double* ms, int* calls)
{
    if (!p) return fail(BLCO_ERR_INVALID, "null plan");
    if (ms)
        for (int n = 0; n < p->N; n++) ms[n] = p->mttkrp_ms[n];
    if (calls) *calls = p->mttkrp_calls;
    return BLCO_OK;
}

} // namespace blco

// ==================================================================== batch
// Batched CP-ALS: many independent tensors of uneven nnz, order (1..5 modes)
// and rank (1..64), decomposed together.  Every step of a sweep is one launch
// over all tensors: the MTTKRP is one persistent launch over the chunks of
// every tensor's row-sorted stream copy (a chunk-offset table maps a global
// chunk to its tensor), and the dense steps
// use one CTA per tensor (solve, lambda, Gram reduction, fit) or per row
// chunk (update, Gram).  Tensor t takes its k-th mode (by descending length)
// in mode slot k.  Convergence is decided on the device per tensor (a tensor
// whose |fit - fit_old| < tol stops taking part), so the whole sweep is
// captured once as a CUDA graph and replayed once per iteration.

namespace blco {
namespace {

constexpr int BATCH_MAX_R = 64;
constexpr int BATCH_MAX_T = 4096;
constexpr int BATCH_CHUNK = 2048;      // rows per update / Gram CTA
constexpr int BATCH_FIT_RING = 4096;   // iterations of fits kept on the device

struct BDesc {
    const uint64_t* coords;
    const double* vals;
    uint64_t nnz;
    const uint64_t* sc[BLCO_MAX_MODES]; // stream copy sorted by the row of mode n
    const double* sv[BLCO_MAX_MODES];
    int nmodes, rank;
    int vec2;                          // rank even and 16-byte aligned rows: 2-double gathers
    int order[BLCO_MAX_MODES];         // modes by descending length
    uint64_t dims[BLCO_MAX_MODES];
    uint64_t mask[BLCO_MAX_MODES];
    int pos[BLCO_MAX_MODES];
    double* U[BLCO_MAX_MODES];
    double* lambda;
    double* M;                         // MTTKRP result, max dim x rank
    double* G[BLCO_MAX_MODES];         // Grams, rank x rank
    double* P;                         // pseudoinverse, rank x rank
    double* inv;                       // 1 / lambda
    double xnorm;
    double fit_old;
    int active;
    int iters;
};

__global__ void k_b_zero(BDesc* __restrict__ d, int T, int slot)
{
    const int t = blockIdx.x / 8, part = blockIdx.x % 8;
    if (t >= T) return;
    const BDesc& b = d[t];
    if (!b.active || slot >= b.nmodes) return;
    const uint64_t len = b.dims[b.order[slot]] * (uint64_t)b.rank;
    for (uint64_t i = (uint64_t)part * blockDim.x + threadIdx.x; i < len; i += 8ull * blockDim.x) b.M[i] = 0.0;
}

// One persistent launch over the chunks of all tensors.  For mode slot k,
// tensor t contributes ceil(nnz / BM_CHUNK) chunks of its stream copy sorted
// by the row of its k-th mode; a warp takes a chunk and splits it into one
// contiguous segment per lane group (LPN lanes, each owning VEC adjacent
// columns, W column blocks).  Each step the group loads LPN nonzeros (one per
// lane, coalesced), then walks them in order with the row, value and other
// indices broadcast by shuffles; the factor rows of U positions are gathered
// before they are multiplied.  Because the segment is row-sorted, the FP64
// partial sum stays in registers until the row changes and is then added to
// M with one atomic per column, so atomics scale with rows, not nonzeros.
// Chunks are dealt round-robin to the warps of the whole grid, which keeps
// the warps on neighbouring chunks (a few tensors at a time) and their
// factor rows in L2.
constexpr int BM_CHUNK = 256;
constexpr int BM_THREADS = 512;
constexpr int BM_WARPS = BM_THREADS / 32;
constexpr int BM_MINB = 1; // resident CTAs per SM

// VEC: 2 gathers two adjacent FP64 columns per lane (even rank, 16-byte
// aligned rows), 1 one column in each of two 32-column blocks.  NMO: the
// number of other modes (2 for third-order tensors, specialised) or -1 for
// any count up to 4 (runtime, fewer positions in flight).  lpn: lanes per
// nonzero (a power of two, 4..32).
template <int VEC, int NMO>
__device__ __forceinline__ void b_chunk(const BDesc& b, int n, uint64_t j0, uint64_t j1, int lane, int lpn)
{
    constexpr int KMAX = NMO > 0 ? NMO : 4;
    constexpr int U = NMO == 2 ? 4 : 2; // positions per gather batch; must not exceed the smallest lpn (4)
    constexpr int W = VEC == 2 ? 1 : 2;
    constexpr int NC = W * VEC;
    const int nmo = NMO >= 0 ? NMO : b.nmodes - 1;
    const int groups = 32 / lpn;
    const int grp = lane / lpn, q = lane % lpn;
    const int R = b.rank;
    const uint64_t* __restrict__ sc = b.sc[n];
    const double* __restrict__ sv = b.sv[n];
    const int rpos = b.pos[n];
    const uint64_t rmask = b.mask[n];
    const double* f[KMAX];
    int opos[KMAX];
    uint64_t omask[KMAX];
#pragma unroll
    for (int k = 0; k < KMAX; k++) {
        const int m = k + (k >= n ? 1 : 0); // the k-th mode other than n
        f[k] = k < nmo ? b.U[m] : nullptr;
        opos[k] = k < nmo ? b.pos[m] : 0;
        omask[k] = k < nmo ? b.mask[m] : 0;
    }
    const uint64_t len = j1 - j0;
    const uint64_t seg = ((len + groups - 1) / groups + lpn - 1) / lpn * lpn;
    const uint64_t gb = j0 + grp * seg, ge = min(j1, gb + seg);
    const int nsteps = (int)(seg / lpn);
    double acc[NC];
#pragma unroll
    for (int j = 0; j < NC; j++) acc[j] = 0.0;
    uint32_t acc_row = 0xffffffffu;
    auto col = [&](int w) { return VEC == 2 ? q * 2 : w * 32 + q; };
    auto flush = [&]() {
        double* o = b.M + (size_t)acc_row * R;
#pragma unroll
        for (int w = 0; w < W; w++) {
            const int c = col(w);
#pragma unroll
            for (int j = 0; j < VEC; j++)
                if (c + j < R) atomicAdd(o + c + j, acc[w * VEC + j]);
        }
    };
    // the next step's coordinate and value are loaded one step ahead
    uint64_t c_next = 0;
    double v_next = 0.0;
    if (gb + q < ge) {
        c_next = __ldcs(sc + gb + q);
        v_next = __ldcs(sv + gb + q);
    }
    for (int st = 0; st < nsteps; st++) {
        const uint64_t jj = gb + (uint64_t)st * lpn + q;
        const bool valid = jj < ge;
        const uint64_t c = c_next;
        const double v = v_next;
        c_next = 0;
        v_next = 0.0;
        if (st + 1 < nsteps && jj + lpn < ge) {
            c_next = __ldcs(sc + jj + lpn);
            v_next = __ldcs(sv + jj + lpn);
        }
        const uint32_t row = valid ? (uint32_t)((c >> rpos) & rmask) : 0xffffffffu;
        uint32_t oth[KMAX];
#pragma unroll
        for (int k = 0; k < KMAX; k++) oth[k] = (uint32_t)((c >> opos[k]) & omask[k]);
        for (int p0 = 0; p0 < lpn; p0 += U) {
            uint32_t rp[U];
            double vp[U];
            double g[U][KMAX][NC];
#pragma unroll
            for (int u = 0; u < U; u++) {
                rp[u] = __shfl_sync(0xffffffffu, row, p0 + u, lpn);
                vp[u] = __shfl_sync(0xffffffffu, v, p0 + u, lpn);
#pragma unroll
                for (int k = 0; k < KMAX; k++) {
                    const uint32_t o = __shfl_sync(0xffffffffu, oth[k], p0 + u, lpn);
#pragma unroll
                    for (int w = 0; w < W; w++) {
                        const int cc = col(w);
                        if (k < nmo && rp[u] != 0xffffffffu && cc < R) {
                            const double* a = f[k] + (size_t)o * R + cc;
                            if constexpr (VEC == 2) {
                                const double2 x = __ldg(reinterpret_cast<const double2*>(a));
                                g[u][k][w * 2] = x.x;
                                g[u][k][w * 2 + 1] = x.y;
                            } else {
                                g[u][k][w] = __ldg(a);
                            }
                        } else {
#pragma unroll
                            for (int j = 0; j < VEC; j++) g[u][k][w * VEC + j] = 1.0;
                        }
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                if (rp[u] != 0xffffffffu) {
                    if (rp[u] != acc_row) {
                        if (acc_row != 0xffffffffu) flush();
                        acc_row = rp[u];
#pragma unroll
                        for (int j = 0; j < NC; j++) acc[j] = 0.0;
                    }
#pragma unroll
                    for (int j = 0; j < NC; j++) {
                        double x = vp[u];
#pragma unroll
                        for (int k = 0; k < KMAX; k++)
                            if (NMO > 0 || k < nmo) x *= g[u][k][j];
                        acc[j] += x;
                    }
                }
            }
        }
    }
    if (acc_row != 0xffffffffu) flush();
}

__global__ void __launch_bounds__(BM_THREADS, BM_MINB) k_b_mttkrp(const BDesc* __restrict__ d, int T,
                                                           const uint32_t* __restrict__ choff, int slot)
{
    __shared__ uint32_t toff[BATCH_MAX_T + 1];
    for (int i = threadIdx.x; i <= T; i += blockDim.x) toff[i] = choff[i];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t nchunks = toff[T];
    for (uint32_t c = blockIdx.x * BM_WARPS + warp; c < nchunks; c += gridDim.x * BM_WARPS) {
        int lo = 0, hi = T - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (toff[mid] <= c) lo = mid;
            else hi = mid - 1;
        }
        const BDesc& b = d[lo];
        if (!b.active) continue; // warp-uniform
        const int n = b.order[slot];
        const uint64_t j0 = (uint64_t)(c - toff[lo]) * BM_CHUNK;
        const uint64_t j1 = min(b.nnz, j0 + BM_CHUNK);
        const int R = b.rank;
        if (b.vec2) {
            const int lpn = R <= 8 ? 4 : R <= 16 ? 8 : R <= 32 ? 16 : 32;
            if (b.nmodes == 3) b_chunk<2, 2>(b, n, j0, j1, lane, lpn);
            else b_chunk<2, -1>(b, n, j0, j1, lane, lpn);
        } else {
            if (b.nmodes == 3) b_chunk<1, 2>(b, n, j0, j1, lane, 32);
            else b_chunk<1, -1>(b, n, j0, j1, lane, 32);
        }
    }
}

__global__ __launch_bounds__(DN_THREADS) void k_b_solve(BDesc* __restrict__ d, int slot, int* __restrict__ dummy)
{
    const BDesc& b = d[blockIdx.x];
    if (!b.active || slot >= b.nmodes) return; // block-uniform
    GramPtrs gp;
    for (int m = 0; m < BLCO_MAX_MODES; m++) gp.g[m] = b.G[m];
    solve_body(gp, b.nmodes, b.order[slot], b.rank, b.P, dummy, nullptr, false);
}

// Register tiling shared by the batched update and Gram kernels: columns
// go in groups of 4 (cg = ceil(R / 4) groups, at most 16), and the 256
// threads of a CTA form (256 / cg) x cg; a block of rows staged in shared
// memory holds BT_ELEMS doubles.
constexpr int BT_ELEMS = 4096;
constexpr size_t BU_SMEM = (BATCH_MAX_R * BATCH_MAX_R + BT_ELEMS) * sizeof(double);

// One CTA per row chunk: U = M P^T in FP64, thread (rg, cg) computing rows
// 4*rg .. 4*rg+3 of each staged block and columns 4*cg .. 4*cg+3 (the sum
// over k runs in order, as in the single-tensor update).  Also the chunk's
// column sums of U^2 (for lambda) and of U .* M (for <X, model> when this is
// the tensor's last mode).
__global__ __launch_bounds__(DN_THREADS) void k_b_update(BDesc* __restrict__ d, const uint32_t* __restrict__ ct,
                                                         const uint32_t* __restrict__ cr0,
                                                         const uint32_t* __restrict__ cr1, int slot,
                                                         double* __restrict__ colsq, double* __restrict__ ippart)
{
    extern __shared__ __align__(16) double bus[];
    double* PT = bus;                          // R x R, transposed
    double* Ms = bus + BATCH_MAX_R * BATCH_MAX_R; // staged rows of M
    double* red = Ms;                          // [2][threads * 4], after the row loop
    const int chunk = blockIdx.x, t = ct[chunk];
    const BDesc& b = d[t];
    if (!b.active || slot >= b.nmodes) return; // block-uniform
    const int R = b.rank, n = b.order[slot], tid = threadIdx.x;
    const int cgs = (R + 3) / 4, rgs = DN_THREADS / cgs;
    const int cg = tid % cgs, rg = tid / cgs;
    const int c0 = cg * 4;
    const int rows_blk = (BT_ELEMS / R) / 4 * 4 < rgs * 4 ? (BT_ELEMS / R) / 4 * 4 : rgs * 4;
    for (int k = tid; k < R * R; k += DN_THREADS) PT[(k % R) * R + k / R] = b.P[k];
    double sq[4] = {0.0, 0.0, 0.0, 0.0}, ip[4] = {0.0, 0.0, 0.0, 0.0};
    const double* __restrict__ M = b.M;
    double* __restrict__ Un = b.U[n];
    for (uint32_t r0 = cr0[chunk]; r0 < cr1[chunk]; r0 += rows_blk) {
        const int nr = (int)min((uint32_t)rows_blk, cr1[chunk] - r0);
        __syncthreads();
        for (int k = tid; k < nr * R; k += DN_THREADS) Ms[k] = M[(size_t)r0 * R + k];
        __syncthreads();
        if (rg < rows_blk / 4 && cg < cgs) {
#pragma unroll 1
            for (int rr = 4 * rg; rr < nr; rr += 4 * rgs) {
                double acc[4][4];
#pragma unroll
                for (int i = 0; i < 4; i++)
#pragma unroll
                    for (int j = 0; j < 4; j++) acc[i][j] = 0.0;
                for (int k = 0; k < R; k++) {
                    double m[4], p[4];
#pragma unroll
                    for (int i = 0; i < 4; i++) m[i] = rr + i < nr ? Ms[(rr + i) * R + k] : 0.0;
#pragma unroll
                    for (int j = 0; j < 4; j++) p[j] = c0 + j < R ? PT[k * R + c0 + j] : 0.0;
#pragma unroll
                    for (int i = 0; i < 4; i++)
#pragma unroll
                        for (int j = 0; j < 4; j++) acc[i][j] += m[i] * p[j];
                }
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    if (rr + i >= nr) break;
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        const int c = c0 + j;
                        if (c < R) {
                            const double u = acc[i][j];
                            Un[(size_t)(r0 + rr + i) * R + c] = u;
                            sq[j] += u * u;
                            ip[j] += u * Ms[(rr + i) * R + c];
                        }
                    }
                }
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 4; j++) {
        red[tid * 4 + j] = sq[j];
        red[DN_THREADS * 4 + tid * 4 + j] = ip[j];
    }
    __syncthreads();
    for (int c = tid; c < R; c += DN_THREADS) {
        double s0 = 0.0, s1 = 0.0;
        const int g = c / 4, j = c % 4;
        for (int r = 0; r < rgs; r++) {
            s0 += red[(r * cgs + g) * 4 + j];
            s1 += red[DN_THREADS * 4 + (r * cgs + g) * 4 + j];
        }
        colsq[(size_t)chunk * BATCH_MAX_R + c] = s0;
        ippart[(size_t)chunk * BATCH_MAX_R + c] = s1;
    }
}

__global__ void k_b_lambda(BDesc* __restrict__ d, const uint32_t* __restrict__ cbeg, const uint32_t* __restrict__ cend,
                           int slot, const double* __restrict__ colsq)
{
    BDesc& b = d[blockIdx.x];
    if (!b.active || slot >= b.nmodes) return;
    for (int c = threadIdx.x; c < b.rank; c += blockDim.x) {
        double s = 0.0;
        for (uint32_t k = cbeg[blockIdx.x]; k < cend[blockIdx.x]; k++) s += colsq[(size_t)k * BATCH_MAX_R + c];
        const double l = sqrt(b.lambda[c] + s);
        b.lambda[c] = l;
        b.inv[c] = l == 0.0 ? 0.0 : 1.0 / l;
    }
}

// One CTA per row chunk: optionally scale the rows by inv (written back),
// then the chunk's Gram partial.  Thread (ag, cg) of the 4 x 4 blocks of
// the R x R Gram takes every `splits`-th row of each staged block; the
// splits are summed in shared memory at the end.
__global__ __launch_bounds__(DN_THREADS) void k_b_gram(BDesc* __restrict__ d, const uint32_t* __restrict__ ct,
                                                       const uint32_t* __restrict__ cr0,
                                                       const uint32_t* __restrict__ cr1, int slot, int scale,
                                                       double* __restrict__ gpart)
{
    __shared__ double tile[BT_ELEMS];
    double* red = tile; // [threads * 16], after the row loop
    const int chunk = blockIdx.x, t = ct[chunk];
    const BDesc& b = d[t];
    if ((scale && !b.active) || slot >= b.nmodes) return; // block-uniform
    const int R = b.rank, n = b.order[slot], tid = threadIdx.x;
    const int cgs = (R + 3) / 4, nblk = cgs * cgs, splits = DN_THREADS / nblk;
    const int blk = tid % nblk, sp = tid / nblk;
    const int a0 = (blk / cgs) * 4, c0 = (blk % cgs) * 4;
    const int rows_blk = BT_ELEMS / R;
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0.0;
    double* __restrict__ Un = b.U[n];
    for (uint32_t r0 = cr0[chunk]; r0 < cr1[chunk]; r0 += rows_blk) {
        const int nr = (int)min((uint32_t)rows_blk, cr1[chunk] - r0);
        __syncthreads();
        for (int k = tid; k < nr * R; k += DN_THREADS) {
            double v = Un[(size_t)r0 * R + k];
            if (scale) {
                v *= b.inv[k % R];
                Un[(size_t)r0 * R + k] = v;
            }
            tile[k] = v;
        }
        __syncthreads();
        if (sp < splits) {
            for (int r = sp; r < nr; r += splits) {
                double x[4], y[4];
#pragma unroll
                for (int i = 0; i < 4; i++) x[i] = a0 + i < R ? tile[r * R + a0 + i] : 0.0;
#pragma unroll
                for (int j = 0; j < 4; j++) y[j] = c0 + j < R ? tile[r * R + c0 + j] : 0.0;
#pragma unroll
                for (int i = 0; i < 4; i++)
#pragma unroll
                    for (int j = 0; j < 4; j++) acc[i][j] += x[i] * y[j];
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) red[tid * 16 + i * 4 + j] = acc[i][j];
    __syncthreads();
    for (int e = tid; e < R * R; e += DN_THREADS) {
        const int a = e / R, c = e % R;
        const int bk = (a / 4) * cgs + c / 4, ij = (a % 4) * 4 + c % 4;
        double s = 0.0;
        for (int q = 0; q < splits; q++) s += red[(q * nblk + bk) * 16 + ij];
        gpart[(size_t)chunk * BATCH_MAX_R * BATCH_MAX_R + e] = s;
    }
}

__global__ void k_b_gram_reduce(BDesc* __restrict__ d, const uint32_t* __restrict__ cbeg,
                                const uint32_t* __restrict__ cend, int slot, int need_active,
                                const double* __restrict__ gpart)
{
    BDesc& b = d[blockIdx.x];
    if ((need_active && !b.active) || slot >= b.nmodes) return;
    const int R = b.rank, n = b.order[slot];
    for (int e = threadIdx.x; e < R * R; e += blockDim.x) {
        double s = 0.0;
        for (uint32_t k = cbeg[blockIdx.x]; k < cend[blockIdx.x]; k++)
            s += gpart[(size_t)k * BATCH_MAX_R * BATCH_MAX_R + e];
        b.G[n][e] = s;
    }
}

struct SlotChunks {
    const uint32_t* beg[BLCO_MAX_MODES];
    const uint32_t* end[BLCO_MAX_MODES];
    const double* ip[BLCO_MAX_MODES];
};

// Per tensor: <X, model> from the last mode's chunk sums of U .* M (taken
// before U was scaled, so each column sum is multiplied by inv * lambda),
// the fit (kruskal_fit_gpu, src/cpd_gpu.cu:331-384) and the convergence
// test.
__global__ __launch_bounds__(DN_THREADS) void k_b_fit(BDesc* __restrict__ d, int T, const int* __restrict__ iter,
                                                      double tol, SlotChunks sc, double* __restrict__ fits)
{
    __shared__ double red[DN_THREADS];
    BDesc& b = d[blockIdx.x];
    if (!b.active) {
        if (threadIdx.x == 0) fits[(size_t)(*iter % BATCH_FIT_RING) * T + blockIdx.x] = b.fit_old;
        return;
    }
    const int R = b.rank, last = b.nmodes - 1;
    double ip = 0.0;
    for (int c = threadIdx.x; c < R; c += DN_THREADS) {
        double s = 0.0;
        for (uint32_t k = sc.beg[last][blockIdx.x]; k < sc.end[last][blockIdx.x]; k++)
            s += sc.ip[last][(size_t)k * BATCH_MAX_R + c];
        ip += s * (b.inv[c] * b.lambda[c]);
    }
    const double iprod = block_sum(ip, red);
    GramPtrs gp;
    for (int m = 0; m < BLCO_MAX_MODES; m++) gp.g[m] = b.G[m];
    const double fit = fit_body(iprod, gp, b.nmodes, R, b.lambda, b.xnorm, red);
    if (threadIdx.x == 0) {
        fits[(size_t)(*iter % BATCH_FIT_RING) * T + blockIdx.x] = fit;
        b.iters++;
        if (fabs(fit - b.fit_old) < tol || isnan(fit)) b.active = 0;
        b.fit_old = fit;
    }
}

__global__ void k_b_next(int* iter) { *iter += 1; }

} // namespace
} // namespace blco

struct blco_batch {
    int T = 0, maxN = 0, maxR = 0;
    blco::BDesc* d_desc = nullptr;
    std::vector<blco::BDesc> h_desc;
    uint32_t* d_choff = nullptr;       // per mode slot: T + 1 MTTKRP chunk offsets
    uint32_t mt_chunks[BLCO_MAX_MODES] = {};
    void* streams = nullptr;           // row-sorted stream copies of every mode
    // per mode slot: chunk -> tensor, row range; per tensor chunk range
    uint32_t* d_ct[BLCO_MAX_MODES] = {};
    uint32_t* d_cr0[BLCO_MAX_MODES] = {};
    uint32_t* d_cr1[BLCO_MAX_MODES] = {};
    uint32_t* d_cbeg[BLCO_MAX_MODES] = {};
    uint32_t* d_cend[BLCO_MAX_MODES] = {};
    int nchunks[BLCO_MAX_MODES] = {};
    double* d_colsq = nullptr;
    double* d_ippart = nullptr;        // per mode slot: maxchunks x 64
    size_t maxchunks = 1;
    double* d_gpart = nullptr;
    double* d_fits = nullptr;
    int* d_iter = nullptr;
    int* d_dummy = nullptr;
    void* pool = nullptr;
    int sm = 148;
    cudaStream_t s = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    long long graph_kernels = 0;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    double last_ms = 0.0;              // device time of the last iterate call
    double tol = 0.0;
    int iters_run = 0;
};

namespace blco {
namespace {

int batch_free(blco_batch* b)
{
    if (!b) return BLCO_OK;
    if (b->s) cudaStreamSynchronize(b->s);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (int k = 0; k < BLCO_MAX_MODES; k++) {
        cudaFree(b->d_ct[k]);
        cudaFree(b->d_cr0[k]);
        cudaFree(b->d_cr1[k]);
        cudaFree(b->d_cbeg[k]);
        cudaFree(b->d_cend[k]);
    }
    cudaFree(b->d_desc);
    cudaFree(b->d_choff);
    cudaFree(b->streams);
    cudaFree(b->d_colsq);
    cudaFree(b->d_ippart);
    cudaFree(b->d_gpart);
    cudaFree(b->d_fits);
    cudaFree(b->d_iter);
    cudaFree(b->d_dummy);
    cudaFree(b->pool);
    for (cudaEvent_t e : b->ev)
        if (e) cudaEventDestroy(e);
    if (b->s) cudaStreamDestroy(b->s);
    delete b;
    return BLCO_OK;
}

// One sweep over all mode slots plus the fit, enqueued on b->s.
int batch_enqueue_sweep(blco_batch* b)
{
    const size_t ssmem = 2 * (size_t)b->maxR * b->maxR * sizeof(double);
    for (int k = 0; k < b->maxN; k++) {
        k_b_zero<<<b->T * 8, 256, 0, b->s>>>(b->d_desc, b->T, k);
        BLCO_CHECK_LAUNCH("k_b_zero");
        if (b->mt_chunks[k]) {
            const unsigned grid =
                (unsigned)std::min<uint64_t>((uint64_t)b->sm * BM_MINB, (b->mt_chunks[k] + BM_WARPS - 1) / BM_WARPS);
            k_b_mttkrp<<<grid, BM_THREADS, 0, b->s>>>(b->d_desc, b->T, b->d_choff + (size_t)k * (b->T + 1), k);
            BLCO_CHECK_LAUNCH("k_b_mttkrp");
        }
        k_b_solve<<<b->T, DN_THREADS, ssmem, b->s>>>(b->d_desc, k, b->d_dummy);
        BLCO_CHECK_LAUNCH("k_b_solve");
        if (b->nchunks[k]) {
            k_b_update<<<b->nchunks[k], DN_THREADS, BU_SMEM, b->s>>>(b->d_desc, b->d_ct[k], b->d_cr0[k], b->d_cr1[k], k,
                                                                b->d_colsq,
                                                                b->d_ippart + (size_t)k * b->maxchunks * BATCH_MAX_R);
            BLCO_CHECK_LAUNCH("k_b_update");
        }
        k_b_lambda<<<b->T, 64, 0, b->s>>>(b->d_desc, b->d_cbeg[k], b->d_cend[k], k, b->d_colsq);
        BLCO_CHECK_LAUNCH("k_b_lambda");
        if (b->nchunks[k]) {
            k_b_gram<<<b->nchunks[k], DN_THREADS, 0, b->s>>>(b->d_desc, b->d_ct[k], b->d_cr0[k], b->d_cr1[k], k, 1,
                                                              b->d_gpart);
            BLCO_CHECK_LAUNCH("k_b_gram");
        }
        k_b_gram_reduce<<<b->T, 256, 0, b->s>>>(b->d_desc, b->d_cbeg[k], b->d_cend[k], k, 1, b->d_gpart);
        BLCO_CHECK_LAUNCH("k_b_gram_reduce");
    }
    SlotChunks sc;
    memset(&sc, 0, sizeof(sc));
    for (int k = 0; k < b->maxN; k++) {
        sc.beg[k] = b->d_cbeg[k];
        sc.end[k] = b->d_cend[k];
        sc.ip[k] = b->d_ippart + (size_t)k * b->maxchunks * BATCH_MAX_R;
    }
    k_b_fit<<<b->T, DN_THREADS, 0, b->s>>>(b->d_desc, b->T, b->d_iter, b->tol, sc, b->d_fits);
    BLCO_CHECK_LAUNCH("k_b_fit");
    k_b_next<<<1, 1, 0, b->s>>>(b->d_iter);
    BLCO_CHECK_LAUNCH("k_b_next");
    return BLCO_OK;
}

} // namespace

int batch_create(int T, blco_tensor* const* tensors, const int* ranks, double* const* const* d_factors,
                 double* const* d_lambdas, double tol, const blco_opts* opts, blco_batch** out)
{
    *out = nullptr;
    if (T < 1 || T > BATCH_MAX_T) return fail(BLCO_ERR_INVALID, "batch size must be 1..4096");
    if (!tensors || !ranks || !d_factors || !d_lambdas) return fail(BLCO_ERR_INVALID, "null argument");
    const int device = tensors[0] ? tensors[0]->device : 0;
    for (int t = 0; t < T; t++) {
        if (!tensors[t] || !d_factors[t] || !d_lambdas[t]) return fail(BLCO_ERR_INVALID, "null tensor or factors");
        if (!tensors[t]->resident) return fail(BLCO_ERR_UNSUPPORTED, "batched CP-ALS needs resident tensors");
        if (tensors[t]->layout.wide)
            return fail(BLCO_ERR_UNSUPPORTED, "batched CP-ALS takes keys of at most 64 bits");
        if (tensors[t]->device != device) return fail(BLCO_ERR_INVALID, "all tensors must be on one device");
        if (ranks[t] < 1 || ranks[t] > BATCH_MAX_R) return fail(BLCO_ERR_UNSUPPORTED, "batched rank must be 1..64");
        for (int n = 0; n < tensors[t]->layout.nmodes; n++)
            if (!d_factors[t][n]) return fail(BLCO_ERR_INVALID, "null factor matrix");
    }
    BLCO_CUDA(cudaSetDevice(device));
    DeviceInfo di;
    BLCO_TRY(device_info(device, &di));
    blco_batch* b = new blco_batch();
    b->T = T;
    b->sm = di.sm_count;
    b->tol = tol;
    b->h_desc.resize(T);
    // workspace sizes
    size_t pool_doubles = 0;
    for (int t = 0; t < T; t++) {
        const Layout& L = tensors[t]->layout;
        uint64_t maxdim = 0;
        for (int n = 0; n < L.nmodes; n++) maxdim = std::max(maxdim, L.dims[n]);
        const size_t R = ranks[t];
        auto al = [](size_t x) { return (x + 3) & ~(size_t)3; };
        pool_doubles += al(maxdim * R) + (size_t)L.nmodes * al(R * R) + al(R * R) + al(R);
        b->maxN = std::max(b->maxN, L.nmodes);
        b->maxR = std::max(b->maxR, ranks[t]);
    }
    auto bail = [&](int st) {
        batch_free(b);
        return st;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&b->s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev[0]);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev[1]);
    if (e == cudaSuccess) e = cudaMalloc(&b->pool, pool_doubles * sizeof(double));
    if (e != cudaSuccess) return bail(cuda_fail(e, "batch workspace", __FILE__, __LINE__));
    double* cur = static_cast<double*>(b->pool);
    auto take = [&](size_t nd) {
        double* r = cur;
        cur += (nd + 3) & ~(size_t)3; // 32-byte aligned pieces
        return r;
    };
    for (int t = 0; t < T; t++) {
        blco_tensor* x = tensors[t];
        const Layout& L = x->layout;
        BDesc& d = b->h_desc[t];
        memset(&d, 0, sizeof(d));
        d.coords = x->d_coords;
        d.vals = x->d_values;
        d.nnz = x->nnz;
        d.nmodes = L.nmodes;
        d.rank = ranks[t];
        d.vec2 = ranks[t] % 2 == 0;
        for (int n = 0; n < L.nmodes; n++) d.vec2 &= ((uintptr_t)d_factors[t][n] & 15) == 0;
        for (int n = 0; n < L.nmodes; n++) {
            d.dims[n] = L.dims[n];
            d.mask[n] = L.mode_masks[n];
            d.pos[n] = L.mode_pos[n];
            d.U[n] = d_factors[t][n];
            d.order[n] = n;
        }
        std::stable_sort(d.order, d.order + L.nmodes, [&](int a2, int b2) { return L.dims[a2] > L.dims[b2]; });
        d.lambda = d_lambdas[t];
        uint64_t maxdim = 0;
        for (int n = 0; n < L.nmodes; n++) maxdim = std::max(maxdim, L.dims[n]);
        const size_t R = ranks[t];
        d.M = take(maxdim * R);
        for (int n = 0; n < L.nmodes; n++) d.G[n] = take(R * R);
        d.P = take(R * R);
        d.inv = take(R);
        d.xnorm = std::sqrt(x->norm_sq);
        d.fit_old = 0.0;
        d.active = 1;
    }
    // Row-sorted stream copies of every mode of every tensor (16 bytes per
    // nonzero per mode) and the MTTKRP chunk offsets of every mode slot.
    {
        uint64_t total = 0, maxnnz = 0;
        for (int t = 0; t < T; t++) {
            total += tensors[t]->nnz * (uint64_t)tensors[t]->layout.nmodes;
            maxnnz = std::max(maxnnz, tensors[t]->nnz);
        }
        uint64_t *tk = nullptr;
        double* tv = nullptr;
        e = cudaMalloc(&b->streams, std::max<uint64_t>(1, total) * 16);
        if (e == cudaSuccess) e = cudaMalloc(&tk, std::max<uint64_t>(1, maxnnz) * 8);
        if (e == cudaSuccess) e = cudaMalloc(&tv, std::max<uint64_t>(1, maxnnz) * 8);
        if (e != cudaSuccess) {
            cudaFree(tk);
            cudaFree(tv);
            return bail(cuda_fail(e, "batch stream copies", __FILE__, __LINE__));
        }
        uint64_t* sc = static_cast<uint64_t*>(b->streams);
        double* sv = reinterpret_cast<double*>(sc + total);
        int st = BLCO_OK;
        for (int t = 0; t < T && st == BLCO_OK; t++) {
            BDesc& d = b->h_desc[t];
            for (int n = 0; n < d.nmodes && st == BLCO_OK; n++) {
                st = sort_stream_by_mode(tensors[t], n, sc, sv, tk, tv, b->s);
                d.sc[n] = sc;
                d.sv[n] = sv;
                sc += d.nnz;
                sv += d.nnz;
            }
        }
        cudaStreamSynchronize(b->s);
        cudaFree(tk);
        cudaFree(tv);
        if (st != BLCO_OK) return bail(st);
        std::vector<uint32_t> choff((size_t)b->maxN * (T + 1));
        for (int k = 0; k < b->maxN; k++) {
            uint64_t c = 0;
            for (int t = 0; t < T; t++) {
                choff[(size_t)k * (T + 1) + t] = (uint32_t)c;
                if (k < b->h_desc[t].nmodes) c += (b->h_desc[t].nnz + BM_CHUNK - 1) / BM_CHUNK;
            }
            if (c >= (1ull << 32)) return bail(fail(BLCO_ERR_UNSUPPORTED, "batch holds too many nonzeros"));
            choff[(size_t)k * (T + 1) + T] = (uint32_t)c;
            b->mt_chunks[k] = (uint32_t)c;
        }
        e = cudaMalloc(&b->d_choff, choff.size() * 4);
        if (e == cudaSuccess)
            e = cudaMemcpy(b->d_choff, choff.data(), choff.size() * 4, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return bail(cuda_fail(e, "batch chunk offsets", __FILE__, __LINE__));
    }
    // chunk tables per slot
    int maxchunks = 0;
    for (int k = 0; k < b->maxN; k++) {
        std::vector<uint32_t> ct, cr0, cr1, cbeg(T, 0), cend(T, 0);
        for (int t = 0; t < T; t++) {
            const BDesc& d = b->h_desc[t];
            cbeg[t] = (uint32_t)ct.size();
            if (k < d.nmodes) {
                const uint64_t I = d.dims[d.order[k]];
                for (uint64_t r = 0; r < I; r += BATCH_CHUNK) {
                    ct.push_back((uint32_t)t);
                    cr0.push_back((uint32_t)r);
                    cr1.push_back((uint32_t)std::min<uint64_t>(I, r + BATCH_CHUNK));
                }
            }
            cend[t] = (uint32_t)ct.size();
        }
        b->nchunks[k] = (int)ct.size();
        maxchunks = std::max(maxchunks, b->nchunks[k]);
        const size_t nc = std::max<size_t>(1, ct.size());
        e = cudaMalloc(&b->d_ct[k], nc * 4);
        if (e == cudaSuccess) e = cudaMalloc(&b->d_cr0[k], nc * 4);
        if (e == cudaSuccess) e = cudaMalloc(&b->d_cr1[k], nc * 4);
        if (e == cudaSuccess) e = cudaMalloc(&b->d_cbeg[k], T * 4);
        if (e == cudaSuccess) e = cudaMalloc(&b->d_cend[k], T * 4);
        if (e == cudaSuccess && !ct.empty()) {
            e = cudaMemcpyAsync(b->d_ct[k], ct.data(), ct.size() * 4, cudaMemcpyHostToDevice, b->s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_cr0[k], cr0.data(), ct.size() * 4, cudaMemcpyHostToDevice, b->s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_cr1[k], cr1.data(), ct.size() * 4, cudaMemcpyHostToDevice, b->s);
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_cbeg[k], cbeg.data(), T * 4, cudaMemcpyHostToDevice, b->s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_cend[k], cend.data(), T * 4, cudaMemcpyHostToDevice, b->s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->s);
        if (e != cudaSuccess) return bail(cuda_fail(e, "batch chunk tables", __FILE__, __LINE__));
    }
    const size_t mc = std::max(1, maxchunks);
    b->maxchunks = mc;
    e = cudaMalloc(&b->d_colsq, mc * BATCH_MAX_R * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_ippart, (size_t)b->maxN * mc * BATCH_MAX_R * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_gpart, mc * BATCH_MAX_R * BATCH_MAX_R * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_fits, (size_t)BATCH_FIT_RING * T * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_iter, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_dummy, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_desc, T * sizeof(BDesc));
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_iter, 0, sizeof(int), b->s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_desc, b->h_desc.data(), T * sizeof(BDesc), cudaMemcpyHostToDevice, b->s);
    if (e != cudaSuccess) return bail(cuda_fail(e, "batch buffers", __FILE__, __LINE__));
    e = cudaFuncSetAttribute(k_b_solve, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(2 * (size_t)b->maxR * b->maxR * sizeof(double)));
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_b_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)BU_SMEM);
    if (e != cudaSuccess) return bail(cuda_fail(e, "k_b_solve shared memory", __FILE__, __LINE__));
    // initial Grams of every mode (unscaled)
    for (int k = 0; k < b->maxN; k++) {
        if (b->nchunks[k]) {
            k_b_gram<<<b->nchunks[k], DN_THREADS, 0, b->s>>>(b->d_desc, b->d_ct[k], b->d_cr0[k], b->d_cr1[k], k, 0,
                                                              b->d_gpart);
            count_launch();
        }
        k_b_gram_reduce<<<T, 256, 0, b->s>>>(b->d_desc, b->d_cbeg[k], b->d_cend[k], k, 0, b->d_gpart);
        count_launch();
    }
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->s);
    if (e != cudaSuccess) return bail(cuda_fail(e, "batch initial Grams", __FILE__, __LINE__));
    // capture one sweep as a graph
    const bool use_graph = !(opts && opts->verbose < 0);
    if (use_graph) {
        e = cudaStreamBeginCapture(b->s, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return bail(cuda_fail(e, "cudaStreamBeginCapture", __FILE__, __LINE__));
        const unsigned long long before = launches_so_far();
        int st = batch_enqueue_sweep(b);
        // captured launches run only when the graph is replayed
        b->graph_kernels = (long long)(launches_so_far() - before);
        add_launches(-b->graph_kernels);
        cudaGraph_t g = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(b->s, &g);
        if (st != BLCO_OK) {
            if (g) cudaGraphDestroy(g);
            return bail(st);
        }
        if (e2 != cudaSuccess) return bail(cuda_fail(e2, "cudaStreamEndCapture", __FILE__, __LINE__));
        b->graph = g;
        e = cudaGraphInstantiate(&b->exec, g, 0);
        if (e != cudaSuccess) return bail(cuda_fail(e, "cudaGraphInstantiate", __FILE__, __LINE__));
    }
    *out = b;
    return BLCO_OK;
}

int batch_iterate(blco_batch* b, int iters, double* fits, int* iters_done)
{
    if (iters < 0 || iters > BATCH_FIT_RING) return fail(BLCO_ERR_INVALID, "iterations per call must be 0..4096");
    BLCO_CUDA(cudaEventRecord(b->ev[0], b->s));
    for (int i = 0; i < iters; i++) {
        if (b->exec) {
            BLCO_CUDA(cudaGraphLaunch(b->exec, b->s));
            add_launches(b->graph_kernels);
        } else {
            BLCO_TRY(batch_enqueue_sweep(b));
        }
    }
    BLCO_CUDA(cudaEventRecord(b->ev[1], b->s));
    BLCO_CUDA(cudaStreamSynchronize(b->s));
    float ms = 0.f;
    BLCO_CUDA(cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]));
    b->last_ms = ms;
    const int first = b->iters_run;
    b->iters_run += iters;
    BLCO_CUDA(cudaMemcpy(b->h_desc.data(), b->d_desc, b->T * sizeof(BDesc), cudaMemcpyDeviceToHost));
    if (fits && iters) {
        // ring rows first..first+iters-1 (mod the ring), in at most two pieces
        const int r0 = first % BATCH_FIT_RING;
        const int n1 = std::min(iters, BATCH_FIT_RING - r0);
        const size_t row = (size_t)b->T * sizeof(double);
        BLCO_CUDA(cudaMemcpy(fits, b->d_fits + (size_t)r0 * b->T, n1 * row, cudaMemcpyDeviceToHost));
        if (iters > n1)
            BLCO_CUDA(cudaMemcpy(fits + (size_t)n1 * b->T, b->d_fits, (iters - n1) * row, cudaMemcpyDeviceToHost));
    }
    if (iters_done)
        for (int t = 0; t < b->T; t++) iters_done[t] = b->h_desc[t].iters;
    return BLCO_OK;
}

int batch_destroy(blco_batch* b) { return batch_free(b); }

double batch_last_ms(const blco_batch* b) { return b->last_ms; }

// Device time of one sweep's MTTKRP launches alone (k_b_mttkrp of every mode
// slot, each after its k_b_zero), outside the graph.  The MTTKRP results are
// workspace that every sweep recomputes before use, so the iteration state
// is unchanged.
int batch_mttkrp_ms(blco_batch* b, double* ms)
{
    cudaEvent_t e[2 * BLCO_MAX_MODES] = {};
    cudaError_t err = cudaSuccess;
    for (int i = 0; i < 2 * BLCO_MAX_MODES && err == cudaSuccess; i++) err = cudaEventCreate(&e[i]);
    int st = err == cudaSuccess ? BLCO_OK : cuda_fail(err, "cudaEventCreate", __FILE__, __LINE__);
    int timed = 0;
    for (int k = 0; k < b->maxN && st == BLCO_OK; k++) {
        if (!b->mt_chunks[k]) continue;
        k_b_zero<<<b->T * 8, 256, 0, b->s>>>(b->d_desc, b->T, k);
        count_launch();
        const unsigned grid =
            (unsigned)std::min<uint64_t>((uint64_t)b->sm * BM_MINB, (b->mt_chunks[k] + BM_WARPS - 1) / BM_WARPS);
        cudaEventRecord(e[2 * k], b->s);
        k_b_mttkrp<<<grid, BM_THREADS, 0, b->s>>>(b->d_desc, b->T, b->d_choff + (size_t)k * (b->T + 1), k);
        count_launch();
        cudaEventRecord(e[2 * k + 1], b->s);
        err = cudaGetLastError();
        if (err != cudaSuccess) st = cuda_fail(err, "k_b_mttkrp", __FILE__, __LINE__);
        timed |= 1 << k;
    }
    if (st == BLCO_OK) {
        err = cudaStreamSynchronize(b->s);
        if (err != cudaSuccess) st = cuda_fail(err, "batch MTTKRP timing", __FILE__, __LINE__);
    }
    double total = 0.0;
    for (int k = 0; k < b->maxN && st == BLCO_OK; k++) {
        if (!(timed & (1 << k))) continue;
        float x = 0.f;
        err = cudaEventElapsedTime(&x, e[2 * k], e[2 * k + 1]);
        if (err != cudaSuccess) st = cuda_fail(err, "cudaEventElapsedTime", __FILE__, __LINE__);
        total += x;
    }
    for (cudaEvent_t x : e)
        if (x) cudaEventDestroy(x);
    if (st == BLCO_OK) *ms = total;
    return st;
}

} // namespace blco
