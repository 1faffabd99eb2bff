// tns_io.h -- sparse tensor files and Kruskal models for the cpd64 tool.
#pragma once

#include <stdint.h>

#include <string>
#include <vector>

namespace blco_host {

struct Coo {
    int nmodes = 0;
    std::vector<uint64_t> dims;               // mode lengths
    std::vector<std::vector<uint64_t>> cidx;  // [mode][nnz], 0-based
    std::vector<double> vals;
    uint64_t nnz() const { return vals.size(); }
};

// FROSTT text format, as ImportSparseTensor(TEXT_FORMAT)
// (src/sptensor.cpp:74-160): blank lines and lines starting with '#' are
// skipped, the mode count is the token count of the first data line minus
// one, indices are 1-based, and each mode length is the largest index seen.
// Returns false with a message on malformed input.
bool read_tns(const std::string& path, Coo* out, std::string* err, int threads = 0);
bool write_tns(const std::string& path, const Coo& x, std::string* err);

// Binary format of src/sptensor.cpp:56-68, 207-242: uint64 nmodes,
// uint64 dims[nmodes], uint64 nnz, uint64 cidx[nmodes][nnz] (0-based),
// double vals[nnz].
bool read_bin(const std::string& path, Coo* out, std::string* err);
bool write_bin(const std::string& path, const Coo& x, std::string* err);

struct Kruskal {
    int nmodes = 0;
    int rank = 0;
    std::vector<uint64_t> dims;
    std::vector<std::vector<double>> U; // row-major dims[n] x rank
    std::vector<double> lambda;
};

// KruskalModelRandomInit (src/kruskal_model.cpp:93-110): lambda = 1 and
// U_n[i] = rand_r(&s) / RAND_MAX where each of `nthreads` threads owns a
// contiguous static chunk of dims[n]*rank entries and starts from
// s = seed + thread id, for every mode.  With the same thread count this
// reproduces the reference's initial factors.
void kruskal_random_init(Kruskal* k, unsigned int seed, int nthreads);

// ExportKruskalModel (src/kruskal_model.cpp:11-42): <path>.<n>.out holds
// "matrix\n2\n<dim> <rank>\n" then the matrix column by column with
// "%.20lf"; <path>.lambda.out holds "vector\n1\n<rank>\n" and lambda.
bool export_kruskal(const Kruskal& k, const std::string& path, std::string* err);

} // namespace blco_host
