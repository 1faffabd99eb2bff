// ref_harness.cpp -- builds the reference's own CPU code into oracle/_ref.
//
// TEST INFRASTRUCTURE ONLY.  This file is compiled together with the
// reference's headers and src/{sptensor,kruskal_model,common}.cpp, read in
// place from the reference checkout (oracle/Makefile, target `ref`).  It
// exposes a small extern "C" surface so tests and bench.py's CPU-baseline
// leg can run:
//   * the reference BLCO encoder gen_blcotensor_host<uint64> and, for the
//     cpd128 build's 128-bit keys, <unsigned __int128>
//     (include/blco.hpp:196-331),
//   * the reference sequential COO MTTKRP, the -c check oracle
//     (include/cpd.hpp:510-544),
//   * the reference OpenMP ALTO CPU MTTKRP mttkrp_alto_par
//     (include/alto.hpp:544-550) on a create_alto tensor,
//   * the reference KruskalModelRandomInit (src/kruskal_model.cpp:93-110),
//   * the reference's CPU CP-ALS cpd_alto (include/cpd.hpp:44-187), the CPU
//     baseline: its BLAS/LAPACK calls (cblas_dsyrk, dpotrf_, dpotrs_,
//     dgelsy_) are forwarded to the OpenBLAS that scipy bundles (exported as
//     scipy_cblas_dsyrk, scipy_dpotrf_, ...; linked by oracle/Makefile).
//
// Stand-ins needed to run the reference host code without a GPU driver:
//   * cudaHostAlloc/cudaMallocHost/cudaFreeHost map to malloc/free;
//   * AlignedMalloc zero-fills, because gen_alto leaves prtn_ptr,
//     prtn_intervals and cr_masks uninitialised and destroy_alto frees them
//     (include/alto.hpp:118, 248-250).
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#include <stdio.h>
#include <string>

static int refh_zero_memalign(void** p, size_t a, size_t n)
{
    int r = posix_memalign(p, a, n ? n : 1);
    if (r == 0) memset(*p, 0, n);
    return r;
}
#define posix_memalign refh_zero_memalign
#include "common.hpp"
#undef posix_memalign

#include "sptensor.hpp"
#include "kruskal_model.hpp"
#include "alto.hpp"
#include "blco.hpp"
#include "cpd.hpp"

extern "C" cudaError_t cudaHostAlloc(void** p, size_t n, unsigned int)
{
    *p = malloc(n ? n : 1);
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
extern "C" cudaError_t cudaMallocHost(void** p, size_t n) { return cudaHostAlloc(p, n, 0); }
extern "C" cudaError_t cudaFreeHost(void* p) { free(p); return cudaSuccess; }
extern "C" const char* cudaGetErrorString(cudaError_t) { return "host stand-in error"; }

void check_cuda(cudaError_t status, std::string message)
{
    if (status != cudaSuccess) {
        fprintf(stderr, "ref_harness: %s failed\n", message.c_str());
        abort();
    }
}

// scipy's OpenBLAS (32-bit integers) under its prefixed names
extern "C" void scipy_cblas_dsyrk(int, int, int, int, int, double, const double*, int, double, double*, int);
extern "C" void scipy_dpotrf_(char*, lapack_int*, double*, lapack_int*, lapack_int*);
extern "C" void scipy_dpotrs_(char*, lapack_int*, lapack_int*, double*, lapack_int*, double*, lapack_int*,
                              lapack_int*);
extern "C" void scipy_dgelsy_(lapack_int*, lapack_int*, lapack_int*, double*, lapack_int*, double*, lapack_int*,
                              lapack_int*, double*, lapack_int*, double*, lapack_int*, lapack_int*);

extern "C" void cblas_dsyrk(CBLAS_ORDER o, CBLAS_UPLO u, CBLAS_TRANSPOSE t, int n, int k, double alpha,
                            const double* a, int lda, double beta, double* c, int ldc)
{
    scipy_cblas_dsyrk((int)o, (int)u, (int)t, n, k, alpha, a, lda, beta, c, ldc);
}
extern "C" void dpotrf_(char* uplo, lapack_int* n, double* a, lapack_int* lda, lapack_int* info)
{
    scipy_dpotrf_(uplo, n, a, lda, info);
}
extern "C" void dpotrs_(char* uplo, lapack_int* n, lapack_int* nrhs, double* a, lapack_int* lda, double* b,
                        lapack_int* ldb, lapack_int* info)
{
    scipy_dpotrs_(uplo, n, nrhs, a, lda, b, ldb, info);
}
extern "C" void dgelsy_(lapack_int* m, lapack_int* n, lapack_int* nrhs, double* a, lapack_int* lda, double* b,
                        lapack_int* ldb, lapack_int* jpvt, double* rcond, lapack_int* rank, double* work,
                        lapack_int* lwork, lapack_int* info)
{
    scipy_dgelsy_(m, n, nrhs, a, lda, b, ldb, jpvt, rcond, rank, work, lwork, info);
}

static SparseTensor* refh_make_tensor(int nmodes, const uint64_t* dims, uint64_t nnz,
                                      const uint64_t* cidx, const double* vals)
{
    SparseTensor* X = (SparseTensor*)AlignedMalloc(sizeof(SparseTensor));
    X->nmodes = nmodes;
    X->nnz = nnz;
    X->dims = (IType*)AlignedMalloc(sizeof(IType) * nmodes);
    X->cidx = (IType**)AlignedMalloc(sizeof(IType*) * nmodes);
    for (int n = 0; n < nmodes; n++) {
        X->dims[n] = dims[n];
        X->cidx[n] = (IType*)AlignedMalloc(sizeof(IType) * (nnz ? nnz : 1));
        memcpy(X->cidx[n], cidx + (size_t)n * nnz, sizeof(IType) * nnz);
    }
    X->vals = (FType*)AlignedMalloc(sizeof(FType) * (nnz ? nnz : 1));
    memcpy(X->vals, vals, sizeof(FType) * nnz);
    return X;
}

template <typename LIT>
static int refh_blco_encode(int nmodes, const uint64_t* dims, uint64_t nnz,
                            const uint64_t* cidx, const double* vals,
                            uint64_t max_block_size, uint64_t* coords_out,
                            double* vals_out, uint64_t* mode_masks_out,
                            int* mode_pos_out, uint64_t* nblocks_out,
                            uint64_t* block_offsets_out, uint64_t* block_coords_out)
{
    SparseTensor* X = refh_make_tensor(nmodes, dims, nnz, cidx, vals);
    blcotensor* T = gen_blcotensor_host<LIT>(X, max_block_size);
    memcpy(coords_out, T->coords, sizeof(uint64_t) * nnz);
    memcpy(vals_out, T->values, sizeof(double) * nnz);
    for (int n = 0; n < nmodes; n++) {
        mode_masks_out[n] = T->mode_masks[n];
        mode_pos_out[n] = T->mode_pos[n];
    }
    *nblocks_out = T->block_count;
    for (IType b = 0; b < T->block_count; b++) {
        block_offsets_out[b] = (uint64_t)(T->blocks[b]->idx - T->coords);
        for (int n = 0; n < nmodes; n++)
            block_coords_out[b * nmodes + n] = T->blocks[b]->block_coords[n];
        free(T->blocks[b]->block_coords);
        delete T->blocks[b];
    }
    block_offsets_out[T->block_count] = nnz;
    delete[] T->blocks;
    free(T->coords);
    free(T->values);
    delete[] T->modes;
    delete[] T->mode_pos;
    delete[] T->mode_masks;
    delete T;
    DestroySparseTensor(X);
    return 0;
}

extern "C" int ref_blco_encode(int nmodes, const uint64_t* dims, uint64_t nnz,
                               const uint64_t* cidx, const double* vals,
                               uint64_t max_block_size, uint64_t* coords_out,
                               double* vals_out, uint64_t* mode_masks_out,
                               int* mode_pos_out, uint64_t* nblocks_out,
                               uint64_t* block_offsets_out, uint64_t* block_coords_out)
{
    return refh_blco_encode<unsigned long long>(nmodes, dims, nnz, cidx, vals, max_block_size, coords_out,
                                                vals_out, mode_masks_out, mode_pos_out, nblocks_out,
                                                block_offsets_out, block_coords_out);
}

// The cpd128 build's encoder (ALTO_MASK_LENGTH=128): gen_blcotensor_host
// with 128-bit ALTO keys.  block_offsets_out needs nnz + 1 entries and
// block_coords_out nnz * nmodes (one block per distinct upper key word and
// max_block_size slice).
extern "C" int ref_blco_encode128(int nmodes, const uint64_t* dims, uint64_t nnz,
                                  const uint64_t* cidx, const double* vals,
                                  uint64_t max_block_size, uint64_t* coords_out,
                                  double* vals_out, uint64_t* mode_masks_out,
                                  int* mode_pos_out, uint64_t* nblocks_out,
                                  uint64_t* block_offsets_out, uint64_t* block_coords_out)
{
    return refh_blco_encode<unsigned __int128>(nmodes, dims, nnz, cidx, vals, max_block_size, coords_out,
                                               vals_out, mode_masks_out, mode_pos_out, nblocks_out,
                                               block_offsets_out, block_coords_out);
}

extern "C" void ref_mttkrp_coo(int nmodes, const uint64_t* dims, uint64_t nnz,
                               const uint64_t* cidx, const double* vals, int rank,
                               double* const* factors, int mode)
{
    // The reference accumulates into U[mode] in place.
    SparseTensor* X = refh_make_tensor(nmodes, dims, nnz, cidx, vals);
    KruskalModel M;
    M.mode = nmodes;
    M.dims = X->dims;
    M.rank = rank;
    M.U = (FType**)factors;
    M.lambda = nullptr;
    M.U_dev = nullptr;
    mttkrp(X, &M, (IType)mode);
    DestroySparseTensor(X);
}

extern "C" void ref_kruskal_random_init(int nmodes, const uint64_t* dims, int rank,
                                        unsigned int seed, double* const* factors,
                                        double* lambda)
{
    KruskalModel* M;
    CreateKruskalModel(nmodes, (IType*)dims, rank, &M);
    KruskalModelRandomInit(M, seed);
    for (int n = 0; n < nmodes; n++)
        memcpy(factors[n], M->U[n], sizeof(double) * dims[n] * rank);
    memcpy(lambda, M->lambda, sizeof(double) * rank);
    DestroyKruskalModel(M);
}

template <typename LIT>
struct refh_alto {
    AltoTensor<LIT>* at;
    FType** ofibs;
    int target;
};

template <typename LIT>
static void* refh_alto_create(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* cidx,
                              const double* vals, int nprtn)
{
    SparseTensor* X = refh_make_tensor(nmodes, dims, nnz, cidx, vals);
    refh_alto<LIT>* h = new refh_alto<LIT>;
    create_alto(X, &h->at, nprtn);
    h->ofibs = nullptr;
    h->target = -2;
    DestroySparseTensor(X);
    return h;
}

template <typename LIT>
static void refh_alto_mttkrp(void* hv, int mode, int rank, double* const* factors)
{
    refh_alto<LIT>* h = (refh_alto<LIT>*)hv;
    if (h->ofibs == nullptr) {
        create_da_mem(-1, rank, h->at, &h->ofibs);
        h->target = -1;
    }
    mttkrp_alto_par(mode, (FType**)factors, (IType)rank, h->at, nullptr, h->ofibs);
}

template <typename LIT>
static void refh_alto_destroy(void* hv, int rank)
{
    refh_alto<LIT>* h = (refh_alto<LIT>*)hv;
    if (h->ofibs) destroy_da_mem(h->at, h->ofibs, rank, -1);
    destroy_alto(h->at);
    delete h;
}

extern "C" void* ref_alto_create(int nmodes, const uint64_t* dims, uint64_t nnz,
                                 const uint64_t* cidx, const double* vals, int nprtn)
{
    return refh_alto_create<unsigned long long>(nmodes, dims, nnz, cidx, vals, nprtn);
}
extern "C" void ref_alto_mttkrp(void* hv, int mode, int rank, double* const* factors)
{
    refh_alto_mttkrp<unsigned long long>(hv, mode, rank, factors);
}
extern "C" void ref_alto_destroy(void* hv, int rank) { refh_alto_destroy<unsigned long long>(hv, rank); }

// The 128-bit build's CPU ALTO MTTKRP (AltoTensor<unsigned __int128>), for
// keys above 64 bits.
extern "C" void* ref_alto_create128(int nmodes, const uint64_t* dims, uint64_t nnz,
                                    const uint64_t* cidx, const double* vals, int nprtn)
{
    return refh_alto_create<unsigned __int128>(nmodes, dims, nnz, cidx, vals, nprtn);
}
extern "C" void ref_alto_mttkrp128(void* hv, int mode, int rank, double* const* factors)
{
    refh_alto_mttkrp<unsigned __int128>(hv, mode, rank, factors);
}
extern "C" void ref_alto_destroy128(void* hv, int rank) { refh_alto_destroy<unsigned __int128>(hv, rank); }

// The reference's CPU CP-ALS (cpd_alto, include/cpd.hpp:44-187) on a COO
// tensor with the given initial factors and lambda (overwritten with the
// result), nthreads OpenMP threads.  cpd_alto reports on stdout; its output
// is captured and parsed: *ms_per_iter and *mttkrp_ms_per_iter from its
// "Per iteration" line (columns Total and MTTKRP, include/cpd.hpp:174-176),
// *fit from its last iteration line.  Returns the iterations run, or -1.
#include <omp.h>
#include <unistd.h>
extern "C" int ref_cpd_alto(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* cidx,
                            const double* vals, int rank, double* const* factors, double* lambda,
                            int max_iters, double epsilon, int nthreads, double* ms_per_iter,
                            double* mttkrp_ms_per_iter, double* fit)
{
    omp_set_num_threads(nthreads);
    SparseTensor* X = refh_make_tensor(nmodes, dims, nnz, cidx, vals);
    AltoTensor<unsigned long long>* AT = nullptr;
    create_alto(X, &AT, nthreads);
    KruskalModel* M;
    CreateKruskalModel(nmodes, (IType*)dims, rank, &M);
    for (int n = 0; n < nmodes; n++) memcpy(M->U[n], factors[n], sizeof(double) * dims[n] * rank);
    memcpy(M->lambda, lambda, sizeof(double) * rank);
    fflush(stdout);
    FILE* cap = tmpfile();
    const int saved = dup(1);
    if (!cap || saved < 0) return -1;
    dup2(fileno(cap), 1);
    cpd_alto(AT, M, max_iters, epsilon);
    fflush(stdout);
    dup2(saved, 1);
    close(saved);
    for (int n = 0; n < nmodes; n++) memcpy(factors[n], M->U[n], sizeof(double) * dims[n] * rank);
    memcpy(lambda, M->lambda, sizeof(double) * rank);
    DestroyKruskalModel(M);
    destroy_alto(AT);
    DestroySparseTensor(X);
    // parse the captured report
    fseek(cap, 0, SEEK_SET);
    char line[512];
    int iters = 0, per = 0;
    while (fgets(line, sizeof(line), cap)) {
        int it;
        double f;
        if (sscanf(line, "it: %d fit: %lf", &it, &f) == 2) {
            *fit = f;
            iters = it + 1;
        } else if (per == 1) {
            double tot = 0, mt = 0;
            if (sscanf(line, "%lf %lf", &tot, &mt) == 2) {
                *ms_per_iter = tot * 1e3;
                *mttkrp_ms_per_iter = mt * 1e3;
            }
            per = 2;
        } else if (strncmp(line, "Per iteration", 13) == 0) {
            per = 1;
        }
    }
    fclose(cap);
    return per == 2 ? iters : -1;
}

// The reference's .tns text reader, ImportSparseTensor with TEXT_FORMAT
// (src/sptensor.cpp:74-207): returns its SparseTensor with the mode count,
// lengths (largest 1-based index per mode) and nonzero count; ref_tns_copy
// copies the 0-based coordinates (nmodes x nnz) and the values out, and
// ref_tns_free frees the tensor.
extern "C" void* ref_tns_import(const char* path, int* nmodes, uint64_t* dims, uint64_t* nnz)
{
    SparseTensor* X = nullptr;
    ImportSparseTensor(path, TEXT_FORMAT, &X);
    fflush(stdout);
    *nmodes = X->nmodes;
    for (int n = 0; n < X->nmodes; n++) dims[n] = X->dims[n];
    *nnz = X->nnz;
    return X;
}

extern "C" void ref_tns_copy(void* h, uint64_t* cidx, double* vals)
{
    const SparseTensor* X = static_cast<const SparseTensor*>(h);
    for (int n = 0; n < X->nmodes; n++) memcpy(cidx + (size_t)n * X->nnz, X->cidx[n], sizeof(uint64_t) * X->nnz);
    memcpy(vals, X->vals, sizeof(double) * X->nnz);
}

extern "C" void ref_tns_free(void* h) { DestroySparseTensor(static_cast<SparseTensor*>(h)); }
