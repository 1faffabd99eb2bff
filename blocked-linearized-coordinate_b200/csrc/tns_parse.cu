// tns_parse.cu -- the FROSTT .tns text loader on the GPU, feeding the encoder
// without a host COO copy.
//
// Semantics follow the reference loader (src/sptensor.cpp:74-160) as this
// library's host loader (host/tns_io.cpp) states them: a data line has at
// least one character besides the newline and does not start with '#' (a
// lone "\r" is not data); the mode count is the number of fields of the first
// data line minus one; each data line holds nmodes 1-based indices
// (strtoull) and a value (strtod); each mode's length is its largest index.
//
// Pipeline: the file is read into pinned host chunks and copied to HBM;
// newlines are counted per 64 KiB block and their positions written in order
// (line starts); data lines are counted per 256-line block and given output
// slots by a block scan over the host-scanned block counts; one thread per
// line parses it.  Values are converted to double on the device with
// correct rounding: the Clinger fast path (significand < 2^53, |q| <= 22) or
// the exact 192-bit product of the normalised significand and a 128-bit
// approximation of 5^q (pow5_table.h), rounded only when the approximation's
// one-unit error cannot change the result.  Lines the device cannot decide
// (more than 19 significant digits, halfway cases, subnormal or overflowing
// results, hex / inf / nan forms, signed indices) are re-parsed on the host
// with strtoull / strtod, so every value equals the host loader's.
#include <fcntl.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "internal.cuh"
#include "pow5_table.h"

namespace blco {
namespace {

#define P10_INIT {1e0, 1e1, 1e2, 1e3, 1e4, 1e5, 1e6, 1e7, 1e8, 1e9, 1e10, 1e11, \
                  1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22}
__constant__ uint64_t c_pow5_t[POW5_COUNT][2] = POW5_T_INIT;
__constant__ int16_t c_pow5_e[POW5_COUNT] = POW5_E_INIT;
__constant__ double c_p10[23] = P10_INIT;
#ifndef __CUDA_ARCH__
const uint64_t h_pow5_t[POW5_COUNT][2] = POW5_T_INIT;
const int16_t h_pow5_e[POW5_COUNT] = POW5_E_INIT;
const double h_p10[23] = P10_INIT;
#endif

enum { PD_OK = 0, PD_HOST = 1, PD_ERROR = 2 };

__host__ __device__ inline bool ws(char c)
{
    return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
}
__host__ __device__ inline bool dig(char c) { return c >= '0' && c <= '9'; }

__host__ __device__ inline void mul_64x64(uint64_t a, uint64_t b, uint64_t* hi, uint64_t* lo)
{
#ifdef __CUDA_ARCH__
    *lo = a * b;
    *hi = __umul64hi(a, b);
#else
    const unsigned __int128 p = (unsigned __int128)a * b;
    *lo = (uint64_t)p;
    *hi = (uint64_t)(p >> 64);
#endif
}

__host__ __device__ inline int clz64(uint64_t x)
{
#ifdef __CUDA_ARCH__
    return __clzll((long long)x);
#else
    return __builtin_clzll(x);
#endif
}

// strtoull's syntax for an unsigned decimal (leading white space, optional
// '+', digits).  '-' (strtoull negates) goes to the host; no digits or a
// value above 2^64 - 1 is an error, as in the host loader.
__host__ __device__ inline int parse_u64(const char*& s, const char* e, uint64_t* out)
{
    while (s < e && ws(*s)) s++;
    if (s < e && *s == '-') return PD_HOST;
    if (s < e && *s == '+') s++;
    if (s >= e || !dig(*s)) return PD_ERROR;
    uint64_t v = 0;
    while (s < e && dig(*s)) {
        const uint64_t d = (uint64_t)(*s - '0');
        if (v > (0xffffffffffffffffull - d) / 10) return PD_ERROR;
        v = v * 10 + d;
        s++;
    }
    *out = v;
    return PD_OK;
}

// w 10^q (w > 0) rounded to the nearest double; `exact` allows the Clinger
// fast path (w is the whole significand).  PD_HOST when undecided.
__host__ __device__ inline int dec_to_double(uint64_t w, int q, bool neg, bool exact, double* out)
{
    if (exact && w < (1ull << 53) && q >= -22 && q <= 22) {
#ifdef __CUDA_ARCH__
        const double* p10 = c_p10;
#else
        const double* p10 = h_p10;
#endif
        double v = (double)w;
        v = q >= 0 ? v * p10[q] : v / p10[-q];
        *out = neg ? -v : v;
        return PD_OK;
    }
    if (q < POW5_QMIN || q > POW5_QMAX) return PD_HOST;
#ifdef __CUDA_ARCH__
    const uint64_t th = c_pow5_t[q - POW5_QMIN][0], tl = c_pow5_t[q - POW5_QMIN][1];
    const int e5 = c_pow5_e[q - POW5_QMIN];
#else
    const uint64_t th = h_pow5_t[q - POW5_QMIN][0], tl = h_pow5_t[q - POW5_QMIN][1];
    const int e5 = h_pow5_e[q - POW5_QMIN];
#endif
    // value = w 10^q = (wn 2^-l)(T 2^e5) 2^q, P = wn T exact in 192 bits
    const int l = clz64(w);
    const uint64_t wn = w << l;
    uint64_t a1, a0, b1, b0;
    mul_64x64(wn, tl, &a1, &a0);
    mul_64x64(wn, th, &b1, &b0);
    const uint64_t p1 = a1 + b0;
    const uint64_t p2 = b1 + (p1 < a1 ? 1u : 0u);
    const int top = (int)(p2 >> 63);
    const int sh = top ? 11 : 10;            // 53 mantissa bits from p2
    uint64_t m = p2 >> sh;
    // remainder below the mantissa, in units of 2^64: (rh : p1), half = 2^(sh-1) : 0
    const uint64_t rh = p2 & ((1ull << sh) - 1), hh = 1ull << (sh - 1);
    // P is within wn < 2^64 of the exact product (T within one unit of 5^q 2^-e5)
    const bool down = rh < hh - 1 || (rh == hh - 1 && p1 <= 0xfffffffffffffffeull);
    const bool up = rh > hh || (rh == hh && p1 >= 1);
    if (!down && !up) return PD_HOST;
    // value ~= m 2^(128 + sh + e5 + q - l), m in [2^52, 2^53)
    int X = e5 + q - l + sh + 128;
    if (up) {
        m++;
        if (m == (1ull << 53)) {
            m = 1ull << 52;
            X++;
        }
    }
    const int B = X + 52 + 1023;
    if (B <= 0 || B >= 2047) return PD_HOST;
    const uint64_t bits = ((uint64_t)neg << 63) | ((uint64_t)B << 52) | (m & ((1ull << 52) - 1));
    double v;
    memcpy(&v, &bits, 8);
    *out = v;
    return PD_OK;
}

// strtod's decimal syntax: white space, sign, digits with an optional '.',
// an optional exponent.  Returns PD_OK with the correctly rounded double,
// PD_HOST when the device does not decide it, PD_ERROR when there is no
// number at all.
__host__ __device__ inline int parse_f64(const char*& s, const char* e, double* out)
{
    while (s < e && ws(*s)) s++;
    bool neg = false;
    if (s < e && (*s == '+' || *s == '-')) {
        neg = *s == '-';
        s++;
    }
    if (s < e && !dig(*s) && *s != '.') return (*s == 'i' || *s == 'I' || *s == 'n' || *s == 'N') ? PD_HOST : PD_ERROR;
    if (s + 1 < e && s[0] == '0' && (s[1] == 'x' || s[1] == 'X')) return PD_HOST;
    uint64_t w = 0;
    int nd = 0, q = 0;
    bool any = false, trunc = false;
    while (s < e && dig(*s)) {
        any = true;
        const int d = *s - '0';
        if (nd == 0 && d == 0) {
        } else if (nd < 19) {
            w = w * 10 + (uint64_t)d;
            nd++;
        } else {
            q++;
            if (d) trunc = true;
        }
        s++;
    }
    if (s < e && *s == '.') {
        const char* dot = s++;
        bool frac = false;
        while (s < e && dig(*s)) {
            frac = true;
            const int d = *s - '0';
            if (nd == 0 && d == 0) {
                q--;
            } else if (nd < 19) {
                w = w * 10 + (uint64_t)d;
                nd++;
                q--;
            } else if (d) {
                trunc = true;
            }
            s++;
        }
        any = any || frac;
        if (!any) {
            s = dot;
            return PD_ERROR;
        }
    }
    if (!any) return PD_ERROR;
    if (s < e && (*s == 'e' || *s == 'E')) {
        const char* t = s + 1;
        bool eneg = false;
        if (t < e && (*t == '+' || *t == '-')) {
            eneg = *t == '-';
            t++;
        }
        if (t < e && dig(*t)) {
            int x = 0;
            while (t < e && dig(*t)) {
                if (x < 100000) x = x * 10 + (*t - '0');
                t++;
            }
            q += eneg ? -x : x;
            s = t;
        }
    }
    if (w == 0) {
        *out = neg ? -0.0 : 0.0;
        return PD_OK;
    }
    if (trunc) {
        // digits beyond the 19th were dropped: the value lies strictly
        // between w 10^q and (w + 1) 10^q; decided when both round alike
        double lo_v, hi_v;
        if (dec_to_double(w, q, neg, false, &lo_v) != PD_OK || dec_to_double(w + 1, q, neg, false, &hi_v) != PD_OK)
            return PD_HOST;
        uint64_t lb, hb;
        memcpy(&lb, &lo_v, 8);
        memcpy(&hb, &hi_v, 8);
        if (lb != hb) return PD_HOST;
        *out = lo_v;
        return PD_OK;
    }
    return dec_to_double(w, q, neg, true, out);
}

constexpr uint64_t TP_BLOCK_BYTES = 1u << 16; // newline counting block
constexpr int TP_THREADS = 256;
constexpr uint32_t TP_HOST_CAP = 1u << 20;    // lines re-parsed on the host, at most

__device__ inline uint32_t block_exclusive_scan(uint32_t v, uint32_t* total)
{
    __shared__ uint32_t wsum[TP_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t x = lane < TP_THREADS / 32 ? wsum[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane < TP_THREADS / 32) wsum[lane] = x;
    }
    __syncthreads();
    const uint32_t base = warp ? wsum[warp - 1] : 0u;
    *total = wsum[TP_THREADS / 32 - 1];
    __syncthreads();
    return base + inc - v;
}

// Newlines that start a line (all but one in the file's last byte), per block.
__global__ __launch_bounds__(TP_THREADS) void k_nl_count(const char* __restrict__ text, uint64_t N,
                                                         uint32_t* __restrict__ counts)
{
    __shared__ uint32_t red[TP_THREADS];
    const uint64_t b0 = (uint64_t)blockIdx.x * TP_BLOCK_BYTES, b1 = min(N, b0 + TP_BLOCK_BYTES);
    uint32_t c = 0;
    for (uint64_t i = b0 + threadIdx.x; i < b1; i += TP_THREADS) c += (text[i] == '\n' && i + 1 < N) ? 1u : 0u;
    red[threadIdx.x] = c;
    __syncthreads();
    for (int s = TP_THREADS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) counts[blockIdx.x] = red[0];
}

// Line starts in file order: block b writes its starts from index base[b].
__global__ __launch_bounds__(TP_THREADS) void k_nl_write(const char* __restrict__ text, uint64_t N,
                                                         const uint64_t* __restrict__ base,
                                                         uint64_t* __restrict__ starts)
{
    const uint64_t b0 = (uint64_t)blockIdx.x * TP_BLOCK_BYTES, b1 = min(N, b0 + TP_BLOCK_BYTES);
    uint64_t run = base[blockIdx.x];
    for (uint64_t r = b0; r < b1; r += TP_THREADS * 16) {
        const uint64_t i0 = r + (uint64_t)threadIdx.x * 16;
        uint32_t c = 0;
        for (int k = 0; k < 16; k++) c += (i0 + k < b1 && text[i0 + k] == '\n' && i0 + k + 1 < N) ? 1u : 0u;
        uint32_t tot;
        uint32_t off = block_exclusive_scan(c, &tot);
        for (int k = 0; k < 16; k++)
            if (i0 + k < b1 && text[i0 + k] == '\n' && i0 + k + 1 < N) starts[run + off++] = i0 + k + 1;
        run += tot;
    }
}

__device__ inline void line_span(const char* text, uint64_t N, const uint64_t* starts, uint64_t L, uint64_t k,
                                 uint64_t* b, uint64_t* e)
{
    *b = starts[k];
    if (k + 1 < L) *e = starts[k + 1] - 1;
    else *e = (N > 0 && text[N - 1] == '\n') ? N - 1 : N;
}

__device__ inline bool data_line(const char* text, uint64_t b, uint64_t e)
{
    const uint64_t len = e - b;
    return len >= 1 && text[b] != '#' && !(len == 1 && text[b] == '\r');
}

__global__ __launch_bounds__(TP_THREADS) void k_data_count(const char* __restrict__ text, uint64_t N,
                                                           const uint64_t* __restrict__ starts, uint64_t L,
                                                           uint32_t* __restrict__ counts)
{
    const uint64_t k = (uint64_t)blockIdx.x * TP_THREADS + threadIdx.x;
    uint32_t d = 0;
    if (k < L) {
        uint64_t b, e;
        line_span(text, N, starts, L, k, &b, &e);
        d = data_line(text, b, e) ? 1u : 0u;
    }
    const uint32_t any = __syncthreads_count(d);
    if (threadIdx.x == 0) counts[blockIdx.x] = any;
}

struct ParseOut {
    uint64_t* cidx[BLCO_MAX_MODES]; // 0-based indices
    double* vals;
    unsigned long long* dims;       // per-mode largest 1-based index
    uint32_t* host_count;           // lines left to the host
    uint64_t* host_line;            // their line numbers (0-based)
    uint64_t* host_slot;            // output slots
    uint64_t* host_span;            // and byte ranges [b, e), two per line
    unsigned long long* err;        // min over error lines of (line << 2 | code), ULLONG_MAX: none;
                                    // code 1 malformed, 2 index 0, 3 too many host lines
};

__global__ __launch_bounds__(TP_THREADS) void k_parse(const char* __restrict__ text, uint64_t N,
                                                      const uint64_t* __restrict__ starts, uint64_t L,
                                                      const uint64_t* __restrict__ slot_base, int nmodes,
                                                      ParseOut o)
{
    const uint64_t k = (uint64_t)blockIdx.x * TP_THREADS + threadIdx.x;
    uint64_t b = 0, e = 0;
    bool d = false;
    if (k < L) {
        line_span(text, N, starts, L, k, &b, &e);
        d = data_line(text, b, e);
    }
    uint32_t tot;
    const uint32_t off = block_exclusive_scan(d ? 1u : 0u, &tot);
    uint64_t mx[BLCO_MAX_MODES] = {0, 0, 0, 0, 0};
    if (d) {
        const uint64_t slot = slot_base[blockIdx.x] + off;
        const char* s = text + b;
        const char* end = text + e;
        uint64_t c[BLCO_MAX_MODES] = {0, 0, 0, 0, 0};
        int st = PD_OK;
        for (int n = 0; n < nmodes && st == PD_OK; n++) st = parse_u64(s, end, &c[n]);
        double v = 0.0;
        if (st == PD_OK) st = parse_f64(s, end, &v);
        if (st == PD_OK) {
            for (int n = 0; n < nmodes; n++)
                if (c[n] == 0) st = -1;
        }
        if (st == PD_OK) {
            for (int n = 0; n < nmodes; n++) {
                o.cidx[n][slot] = c[n] - 1;
                mx[n] = c[n];
            }
            o.vals[slot] = v;
        } else if (st == PD_HOST) {
            const uint32_t h = atomicAdd(o.host_count, 1u);
            if (h < TP_HOST_CAP) {
                o.host_line[h] = k;
                o.host_slot[h] = slot;
                o.host_span[2 * h] = b;
                o.host_span[2 * h + 1] = e;
            } else {
                atomicMin(o.err, (unsigned long long)((k << 2) | 3));
            }
        } else {
            atomicMin(o.err, (unsigned long long)((k << 2) | (st == -1 ? 2u : 1u)));
        }
    }
    for (int n = 0; n < nmodes; n++) {
        unsigned long long m = mx[n];
#pragma unroll
        for (int s2 = 16; s2 > 0; s2 >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, s2));
        if ((threadIdx.x & 31) == 0 && m) atomicMax(o.dims + n, m);
    }
}

__global__ void k_scatter_host(const uint64_t* __restrict__ slots, const uint64_t* __restrict__ hc,
                               const double* __restrict__ hv, uint32_t n, int nmodes, ParseOut o)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint64_t s = slots[i];
        for (int m = 0; m < nmodes; m++) {
            o.cidx[m][s] = hc[(size_t)i * BLCO_MAX_MODES + m] - 1;
            atomicMax(o.dims + m, (unsigned long long)hc[(size_t)i * BLCO_MAX_MODES + m]);
        }
        o.vals[s] = hv[i];
    }
}

// The host loader's line rule and parse (strtoull / strtod), for the lines
// the device leaves to the host.
bool host_data_line(const char* b, const char* e)
{
    const size_t len = (size_t)(e - b);
    return len >= 1 && b[0] != '#' && !(len == 1 && b[0] == '\r');
}

int host_parse_line(const std::string& line, int nmodes, uint64_t* c, double* v)
{
    const char* p = line.c_str();
    for (int n = 0; n < nmodes; n++) {
        char* q;
        errno = 0;
        const unsigned long long x = strtoull(p, &q, 10);
        if (q == p || errno) return 1;
        c[n] = x;
        p = q;
    }
    char* q;
    *v = strtod(p, &q);
    if (q == p) return 1;
    for (int n = 0; n < nmodes; n++)
        if (c[n] == 0) return 2;
    return 0;
}

struct FileReader {
    int fd = -1;
    uint64_t size = 0;
    ~FileReader()
    {
        if (fd >= 0) close(fd);
    }
    bool read_at(uint64_t off, void* dst, uint64_t n) const
    {
        char* d = static_cast<char*>(dst);
        while (n) {
            const ssize_t r = pread(fd, d, n, (off_t)off);
            if (r <= 0) return false;
            d += r;
            off += (uint64_t)r;
            n -= (uint64_t)r;
        }
        return true;
    }
};

// Field count of the first data line minus one (the mode count).
int detect_modes(const FileReader& f)
{
    std::string buf;
    const uint64_t step = 1u << 16;
    uint64_t pos = 0;
    std::string carry;
    while (pos < f.size) {
        const uint64_t n = std::min(step, f.size - pos);
        buf.resize(n);
        if (!f.read_at(pos, &buf[0], n)) return -1;
        carry += buf;
        pos += n;
        size_t b = 0;
        for (;;) {
            const size_t nl = carry.find('\n', b);
            if (nl == std::string::npos && pos < f.size) break;
            const size_t e = nl == std::string::npos ? carry.size() : nl;
            if (host_data_line(carry.data() + b, carry.data() + e)) {
                int tok = 0;
                bool in = false;
                for (size_t p = b; p < e; p++) {
                    const char ch = carry[p];
                    const bool w = ch == ' ' || ch == '\t' || ch == '\r';
                    if (!w && !in) tok++;
                    in = !w;
                }
                return tok - 1;
            }
            if (nl == std::string::npos) return -1;
            b = nl + 1;
        }
        carry.erase(0, b);
    }
    return -1;
}

} // namespace

int parse_decimal_host(const char* s, int len, double* out, int* consumed)
{
    const char* p = s;
    const int st = parse_f64(p, s + len, out);
    if (consumed) *consumed = (int)(p - s);
    return st;
}

int encode_tns_impl(const char* path, uint64_t max_block_size, const blco_opts* opts, blco_tensor** out,
                    blco_tns_info* info)
{
    *out = nullptr;
    FileReader f;
    f.fd = open(path, O_RDONLY);
    if (f.fd < 0) return fail(BLCO_ERR_IO, std::string("cannot open ") + path);
    const off_t sz = lseek(f.fd, 0, SEEK_END);
    if (sz < 0) return fail(BLCO_ERR_IO, std::string("cannot read ") + path);
    f.size = (uint64_t)sz;
    const int nmodes = detect_modes(f);
    if (nmodes < 1 || nmodes > BLCO_MAX_MODES)
        return fail(BLCO_ERR_INVALID, std::string("no data line with 2..6 fields in ") + path);
    const int device = opts ? opts->device : 0;
    BLCO_CUDA(cudaSetDevice(device));
    DeviceInfo di;
    BLCO_TRY(device_info(device, &di));
    cudaStream_t s = opts && opts->stream ? (cudaStream_t)opts->stream : nullptr;
    const uint64_t N = f.size;

    char* d_text = nullptr;
    uint64_t *d_starts = nullptr, *d_base = nullptr, *d_cidx[BLCO_MAX_MODES] = {}, *d_hline = nullptr,
             *d_hslot = nullptr, *d_hspan = nullptr;
    uint32_t *d_counts = nullptr, *d_hcount = nullptr;
    double* d_vals = nullptr;
    unsigned long long *d_dims = nullptr, *d_err = nullptr;
    char* pinned[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    int st = BLCO_OK;
    auto cleanup = [&]() {
        if (s) cudaStreamSynchronize(s);
        else cudaDeviceSynchronize();
        cudaFree(d_text);
        cudaFree(d_starts);
        cudaFree(d_base);
        for (auto p : d_cidx) cudaFree(p);
        cudaFree(d_hline);
        cudaFree(d_hslot);
        cudaFree(d_hspan);
        cudaFree(d_counts);
        cudaFree(d_hcount);
        cudaFree(d_vals);
        cudaFree(d_dims);
        cudaFree(d_err);
        for (auto p : pinned) cudaFreeHost(p);
        for (auto e2 : ev)
            if (e2) cudaEventDestroy(e2);
    };
#define TC(call)                                                               \
    do {                                                                       \
        cudaError_t _e = (call);                                               \
        if (_e != cudaSuccess) {                                               \
            st = cuda_fail(_e, #call, __FILE__, __LINE__);                     \
            cleanup();                                                         \
            return st;                                                         \
        }                                                                      \
    } while (0)
    // 1. the file into HBM through two pinned chunks
    const uint64_t CH = 64ull << 20;
    TC(cudaMalloc(&d_text, std::max<uint64_t>(N, 1)));
    TC(cudaMallocHost(&pinned[0], CH));
    TC(cudaMallocHost(&pinned[1], CH));
    TC(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
    TC(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
    for (uint64_t off = 0, i = 0; off < N; off += CH, i++) {
        const int k = (int)(i & 1);
        const uint64_t n = std::min(CH, N - off);
        if (i >= 2) TC(cudaEventSynchronize(ev[k]));
        if (!f.read_at(off, pinned[k], n)) {
            cleanup();
            return fail(BLCO_ERR_IO, std::string("read error in ") + path);
        }
        TC(cudaMemcpyAsync(d_text + off, pinned[k], n, cudaMemcpyHostToDevice, s));
        TC(cudaEventRecord(ev[k], s));
    }
    // 2. line starts
    const uint64_t nb = (N + TP_BLOCK_BYTES - 1) / TP_BLOCK_BYTES;
    TC(cudaMalloc(&d_counts, std::max<uint64_t>(nb, 1) * sizeof(uint32_t)));
    if (nb) {
        k_nl_count<<<(unsigned)nb, TP_THREADS, 0, s>>>(d_text, N, d_counts);
        count_launch();
        TC(cudaGetLastError());
    }
    std::vector<uint32_t> hc(nb);
    std::vector<uint64_t> hb(std::max<uint64_t>(nb, 1));
    if (nb) TC(cudaMemcpyAsync(hc.data(), d_counts, nb * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    TC(s ? cudaStreamSynchronize(s) : cudaDeviceSynchronize());
    uint64_t L = N ? 1 : 0;
    for (uint64_t b = 0; b < nb; b++) {
        hb[b] = L;
        L += hc[b];
    }
    TC(cudaMalloc(&d_starts, std::max<uint64_t>(L, 1) * sizeof(uint64_t)));
    TC(cudaMalloc(&d_base, std::max<uint64_t>(nb, 1) * sizeof(uint64_t)));
    TC(cudaMemsetAsync(d_starts, 0, sizeof(uint64_t), s));
    if (nb) {
        TC(cudaMemcpyAsync(d_base, hb.data(), nb * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
        k_nl_write<<<(unsigned)nb, TP_THREADS, 0, s>>>(d_text, N, d_base, d_starts);
        count_launch();
        TC(cudaGetLastError());
    }
    // 3. data lines and their output slots
    const uint64_t lb = (L + TP_THREADS - 1) / TP_THREADS;
    cudaFree(d_counts);
    d_counts = nullptr;
    cudaFree(d_base);
    d_base = nullptr;
    TC(cudaMalloc(&d_counts, std::max<uint64_t>(lb, 1) * sizeof(uint32_t)));
    TC(cudaMalloc(&d_base, std::max<uint64_t>(lb, 1) * sizeof(uint64_t)));
    if (lb) {
        k_data_count<<<(unsigned)lb, TP_THREADS, 0, s>>>(d_text, N, d_starts, L, d_counts);
        count_launch();
        TC(cudaGetLastError());
    }
    hc.assign(lb, 0);
    hb.assign(std::max<uint64_t>(lb, 1), 0);
    if (lb) TC(cudaMemcpyAsync(hc.data(), d_counts, lb * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    TC(s ? cudaStreamSynchronize(s) : cudaDeviceSynchronize());
    uint64_t nnz = 0;
    for (uint64_t b = 0; b < lb; b++) {
        hb[b] = nnz;
        nnz += hc[b];
    }
    if (nnz == 0) {
        cleanup();
        return fail(BLCO_ERR_INVALID, std::string("no data lines in ") + path);
    }
    if (lb) TC(cudaMemcpyAsync(d_base, hb.data(), lb * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
    // 4. parse
    ParseOut o;
    memset(&o, 0, sizeof(o));
    for (int n = 0; n < nmodes; n++) {
        TC(cudaMalloc(&d_cidx[n], nnz * sizeof(uint64_t)));
        o.cidx[n] = d_cidx[n];
    }
    TC(cudaMalloc(&d_vals, nnz * sizeof(double)));
    TC(cudaMalloc(&d_dims, BLCO_MAX_MODES * sizeof(unsigned long long)));
    TC(cudaMalloc(&d_hcount, sizeof(uint32_t)));
    TC(cudaMalloc(&d_hline, TP_HOST_CAP * sizeof(uint64_t)));
    TC(cudaMalloc(&d_hslot, TP_HOST_CAP * sizeof(uint64_t)));
    TC(cudaMalloc(&d_hspan, 2 * TP_HOST_CAP * sizeof(uint64_t)));
    TC(cudaMalloc(&d_err, sizeof(unsigned long long)));
    TC(cudaMemsetAsync(d_dims, 0, BLCO_MAX_MODES * sizeof(unsigned long long), s));
    TC(cudaMemsetAsync(d_hcount, 0, sizeof(uint32_t), s));
    TC(cudaMemsetAsync(d_err, 0xff, sizeof(unsigned long long), s));
    o.vals = d_vals;
    o.dims = d_dims;
    o.host_count = d_hcount;
    o.host_line = d_hline;
    o.host_slot = d_hslot;
    o.host_span = d_hspan;
    o.err = d_err;
    k_parse<<<(unsigned)lb, TP_THREADS, 0, s>>>(d_text, N, d_starts, L, d_base, nmodes, o);
    count_launch();
    TC(cudaGetLastError());
    unsigned long long herr = 0;
    uint32_t nhost = 0;
    TC(cudaMemcpyAsync(&herr, d_err, sizeof(herr), cudaMemcpyDeviceToHost, s));
    TC(cudaMemcpyAsync(&nhost, d_hcount, sizeof(nhost), cudaMemcpyDeviceToHost, s));
    TC(s ? cudaStreamSynchronize(s) : cudaDeviceSynchronize());
    nhost = std::min(nhost, TP_HOST_CAP);
    // 5. the lines left to the host (an error among them counts as well)
    std::vector<uint64_t> hl(nhost), hs(nhost), hsp(2 * (size_t)nhost), hcx((size_t)nhost * BLCO_MAX_MODES, 0);
    std::vector<double> hv(nhost);
    if (nhost) {
        TC(cudaMemcpyAsync(hl.data(), d_hline, nhost * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        TC(cudaMemcpyAsync(hs.data(), d_hslot, nhost * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        TC(cudaMemcpyAsync(hsp.data(), d_hspan, 2 * nhost * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        TC(s ? cudaStreamSynchronize(s) : cudaDeviceSynchronize());
        for (uint32_t i = 0; i < nhost; i++) {
            const uint64_t b = hsp[2 * i], e = hsp[2 * i + 1];
            std::string line(e - b, '\0');
            if (e > b && !f.read_at(b, &line[0], e - b)) {
                cleanup();
                return fail(BLCO_ERR_IO, std::string("read error in ") + path);
            }
            const int r = host_parse_line(line, nmodes, &hcx[(size_t)i * BLCO_MAX_MODES], &hv[i]);
            if (r) herr = std::min<unsigned long long>(herr, (hl[i] << 2) | (unsigned)r);
        }
    }
    if (herr != 0xffffffffffffffffull) {
        cleanup();
        const int hcode = (int)(herr & 3);
        const std::string where = " on line " + std::to_string((herr >> 2) + 1) + " of " + path;
        if (hcode == 2) return fail(BLCO_ERR_INVALID, "index 0" + where + " (indices are 1-based)");
        if (hcode == 3) return fail(BLCO_ERR_UNSUPPORTED, "more than 2^20 values need the host parser" + where);
        return fail(BLCO_ERR_INVALID, "malformed line" + where);
    }
    if (nhost) {
        uint64_t *d_s = nullptr, *d_c = nullptr;
        double* d_v = nullptr;
        cudaError_t e = cudaMalloc(&d_s, nhost * sizeof(uint64_t));
        if (e == cudaSuccess) e = cudaMalloc(&d_c, hcx.size() * sizeof(uint64_t));
        if (e == cudaSuccess) e = cudaMalloc(&d_v, nhost * sizeof(double));
        if (e == cudaSuccess) e = cudaMemcpy(d_s, hs.data(), nhost * sizeof(uint64_t), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(d_c, hcx.data(), hcx.size() * sizeof(uint64_t), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(d_v, hv.data(), nhost * sizeof(double), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) {
            k_scatter_host<<<std::max(1u, std::min(1024u, (nhost + 255) / 256)), 256, 0, s>>>(d_s, d_c, d_v, nhost,
                                                                                               nmodes, o);
            count_launch();
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = s ? cudaStreamSynchronize(s) : cudaDeviceSynchronize();
        cudaFree(d_s);
        cudaFree(d_c);
        cudaFree(d_v);
        if (e != cudaSuccess) {
            st = cuda_fail(e, "host-parsed lines", __FILE__, __LINE__);
            cleanup();
            return st;
        }
    }
    uint64_t dims[BLCO_MAX_MODES] = {};
    TC(cudaMemcpy(dims, d_dims, BLCO_MAX_MODES * sizeof(uint64_t), cudaMemcpyDeviceToHost));
    // the text and line tables are no longer needed before the encoder runs
    cudaFree(d_text);
    d_text = nullptr;
    cudaFree(d_starts);
    d_starts = nullptr;
    // 6. encode from the device COO
    st = encode_impl(nmodes, dims, nnz, d_cidx, d_vals, max_block_size, opts, out);
#undef TC
    cleanup();
    if (st != BLCO_OK) return st;
    if (info) {
        memset(info, 0, sizeof(*info));
        info->nmodes = nmodes;
        for (int n = 0; n < nmodes; n++) info->dims[n] = dims[n];
        info->nnz = nnz;
        info->lines = L;
        info->host_parsed = nhost;
    }
    return BLCO_OK;
}

} // namespace blco
