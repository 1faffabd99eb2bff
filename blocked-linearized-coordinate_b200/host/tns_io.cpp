// tns_io.cpp -- sparse tensor files and Kruskal models (host side of cpd64).
#include "tns_io.h"

#include <errno.h>
#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <thread>

namespace blco_host {

namespace {

struct Mapped {
    const char* p = nullptr;
    size_t n = 0;
    int fd = -1;
    ~Mapped()
    {
        if (p && n) munmap((void*)p, n);
        if (fd >= 0) close(fd);
    }
};

bool map_file(const std::string& path, Mapped* m, std::string* err)
{
    m->fd = open(path.c_str(), O_RDONLY);
    if (m->fd < 0) {
        *err = "cannot open " + path + ": " + strerror(errno);
        return false;
    }
    struct stat st;
    if (fstat(m->fd, &st) != 0) {
        *err = "cannot stat " + path;
        return false;
    }
    m->n = (size_t)st.st_size;
    if (m->n == 0) return true;
    void* p = mmap(nullptr, m->n, PROT_READ, MAP_PRIVATE, m->fd, 0);
    if (p == MAP_FAILED) {
        *err = "cannot map " + path;
        return false;
    }
    m->p = (const char*)p;
    return true;
}

bool is_data_line(const char* b, const char* e)
{
    // A line with at least one character besides the newline that does not
    // start with '#' (src/sptensor.cpp:89, 116).
    size_t len = (size_t)(e - b);
    return len >= 1 && b[0] != '#' && !(len == 1 && b[0] == '\r');
}

// Parses one data line into coords (1-based) and value.
bool parse_line(const char* b, const char* e, int nmodes, uint64_t* c, double* v)
{
    char buf[1024];
    size_t len = std::min((size_t)(e - b), sizeof(buf) - 1);
    memcpy(buf, b, len);
    buf[len] = 0;
    char* p = buf;
    for (int n = 0; n < nmodes; n++) {
        char* q;
        errno = 0;
        unsigned long long x = strtoull(p, &q, 10);
        if (q == p || errno) return false;
        c[n] = x;
        p = q;
    }
    char* q;
    *v = strtod(p, &q);
    return q != p;
}

} // namespace

bool read_tns(const std::string& path, Coo* out, std::string* err, int threads)
{
    Mapped m;
    if (!map_file(path, &m, err)) return false;
    const char* s = m.p;
    const char* end = m.p + m.n;
    // mode count from the first data line
    int nmodes = -1;
    for (const char* b = s; b < end;) {
        const char* e = (const char*)memchr(b, '\n', end - b);
        if (!e) e = end;
        if (is_data_line(b, e)) {
            int tok = 0;
            bool in = false;
            for (const char* p = b; p < e; p++) {
                bool ws = *p == ' ' || *p == '\t' || *p == '\r';
                if (!ws && !in) tok++;
                in = !ws;
            }
            nmodes = tok - 1;
            break;
        }
        b = e + 1;
    }
    if (nmodes < 1 || nmodes > 5) {
        *err = "no data line with 2..6 fields in " + path;
        return false;
    }
    // split the file into chunks on line boundaries
    int T = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
    T = (int)std::min<size_t>((size_t)T, std::max<size_t>(1, m.n / (1 << 20)));
    std::vector<const char*> cut(T + 1);
    cut[0] = s;
    cut[T] = end;
    for (int t = 1; t < T; t++) {
        const char* p = s + (m.n * t) / T;
        const char* nl = (const char*)memchr(p, '\n', end - p);
        cut[t] = nl ? nl + 1 : end;
        if (cut[t] < cut[t - 1]) cut[t] = cut[t - 1];
    }
    std::vector<std::vector<uint64_t>> pc(T);
    std::vector<std::vector<double>> pv(T);
    std::vector<std::string> perr(T);
    std::vector<std::thread> th;
    for (int t = 0; t < T; t++) {
        th.emplace_back([&, t]() {
            uint64_t c[5];
            double v;
            for (const char* b = cut[t]; b < cut[t + 1];) {
                const char* e = (const char*)memchr(b, '\n', cut[t + 1] - b);
                if (!e) e = cut[t + 1];
                if (is_data_line(b, e)) {
                    if (!parse_line(b, e, nmodes, c, &v)) {
                        perr[t] = "malformed line in " + path;
                        return;
                    }
                    for (int n = 0; n < nmodes; n++) {
                        if (c[n] == 0) {
                            perr[t] = "index 0 in " + path + " (indices are 1-based)";
                            return;
                        }
                        pc[t].push_back(c[n] - 1);
                    }
                    pv[t].push_back(v);
                }
                b = e + 1;
            }
        });
    }
    for (auto& x : th) x.join();
    for (int t = 0; t < T; t++)
        if (!perr[t].empty()) {
            *err = perr[t];
            return false;
        }
    uint64_t nnz = 0;
    for (auto& v : pv) nnz += v.size();
    out->nmodes = nmodes;
    out->dims.assign(nmodes, 0);
    out->cidx.assign(nmodes, std::vector<uint64_t>(nnz));
    out->vals.resize(nnz);
    uint64_t o = 0;
    for (int t = 0; t < T; t++) {
        for (size_t i = 0; i < pv[t].size(); i++) {
            for (int n = 0; n < nmodes; n++) {
                uint64_t x = pc[t][i * nmodes + n];
                out->cidx[n][o + i] = x;
                out->dims[n] = std::max(out->dims[n], x + 1);
            }
            out->vals[o + i] = pv[t][i];
        }
        o += pv[t].size();
    }
    return true;
}

bool write_tns(const std::string& path, const Coo& x, std::string* err)
{
    FILE* f = fopen(path.c_str(), "w");
    if (!f) {
        *err = "cannot write " + path;
        return false;
    }
    for (uint64_t i = 0; i < x.nnz(); i++) {
        for (int n = 0; n < x.nmodes; n++) fprintf(f, "%llu ", (unsigned long long)(x.cidx[n][i] + 1));
        fprintf(f, "%g\n", x.vals[i]);
    }
    fclose(f);
    return true;
}

bool read_bin(const std::string& path, Coo* out, std::string* err)
{
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) {
        *err = "cannot open " + path;
        return false;
    }
    uint64_t nm = 0, nnz = 0;
    bool ok = fread(&nm, 8, 1, f) == 1 && nm >= 1 && nm <= 5;
    std::vector<uint64_t> dims(ok ? nm : 0);
    ok = ok && fread(dims.data(), 8, nm, f) == nm && fread(&nnz, 8, 1, f) == 1;
    if (ok) {
        out->nmodes = (int)nm;
        out->dims = dims;
        out->cidx.assign(nm, std::vector<uint64_t>(nnz));
        out->vals.resize(nnz);
        for (uint64_t n = 0; n < nm && ok; n++) ok = fread(out->cidx[n].data(), 8, nnz, f) == nnz;
        ok = ok && fread(out->vals.data(), 8, nnz, f) == nnz;
    }
    fclose(f);
    if (!ok) *err = "truncated or malformed binary tensor " + path;
    return ok;
}

bool write_bin(const std::string& path, const Coo& x, std::string* err)
{
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) {
        *err = "cannot write " + path;
        return false;
    }
    uint64_t nm = x.nmodes, nnz = x.nnz();
    fwrite(&nm, 8, 1, f);
    fwrite(x.dims.data(), 8, nm, f);
    fwrite(&nnz, 8, 1, f);
    for (int n = 0; n < x.nmodes; n++) fwrite(x.cidx[n].data(), 8, nnz, f);
    fwrite(x.vals.data(), 8, nnz, f);
    fclose(f);
    return true;
}

void kruskal_random_init(Kruskal* k, unsigned int seed, int nthreads)
{
    if (nthreads < 1) nthreads = 1;
    k->lambda.assign(k->rank, 1.0);
    k->U.resize(k->nmodes);
    for (int n = 0; n < k->nmodes; n++) {
        const uint64_t total = k->dims[n] * (uint64_t)k->rank;
        k->U[n].assign(total, 0.0);
        const uint64_t q = total / nthreads, r = total % nthreads;
        for (int t = 0; t < nthreads; t++) {
            const uint64_t cnt = q + ((uint64_t)t < r ? 1 : 0);
            const uint64_t beg = (uint64_t)t * q + std::min<uint64_t>((uint64_t)t, r);
            unsigned int s = seed + (unsigned int)t;
            for (uint64_t i = 0; i < cnt; i++) k->U[n][beg + i] = (double)rand_r(&s) / RAND_MAX;
        }
    }
}

bool export_kruskal(const Kruskal& k, const std::string& path, std::string* err)
{
    for (int n = 0; n < k.nmodes; n++) {
        std::string p = path + "." + std::to_string(n) + ".out";
        FILE* f = fopen(p.c_str(), "w");
        if (!f) {
            *err = "cannot write " + p;
            return false;
        }
        fprintf(f, "matrix\n2\n%llu %llu\n", (unsigned long long)k.dims[n], (unsigned long long)k.rank);
        for (int r = 0; r < k.rank; r++)
            for (uint64_t i = 0; i < k.dims[n]; i++) fprintf(f, "%.20lf\n", k.U[n][i * k.rank + r]);
        fclose(f);
    }
    std::string p = path + ".lambda.out";
    FILE* f = fopen(p.c_str(), "w");
    if (!f) {
        *err = "cannot write " + p;
        return false;
    }
    fprintf(f, "vector\n1\n%llu\n", (unsigned long long)k.rank);
    for (int r = 0; r < k.rank; r++) fprintf(f, "%.20lf\n", k.lambda[r]);
    fclose(f);
    return true;
}

} // namespace blco_host
