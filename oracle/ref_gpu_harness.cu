// ref_gpu_harness.cu -- builds the reference's own GPU CP-ALS into oracle/_ref.
//
// TEST INFRASTRUCTURE ONLY.  Compiled together with the reference's
// src/{alto_dev,blco,cpd_gpu,utils,kruskal_model}.cu and
// src/{kruskal_model,sptensor,common}.cpp, read in place from the reference
// checkout (oracle/Makefile, target `ref-gpu`), for sm_100a.  It exposes:
//   * refgpu_cpals: cpals_blco_dev (src/cpd_gpu.cu:21-242) on a tensor
//     encoded by gen_blcotensor_host<uint64> with one block, with factors
//     and lambda passed in explicitly (the reference's random init depends on
//     the host thread count), returning the final fit and the updated model;
//   * refgpu_mttkrp: mttkrp_alto_dev (src/alto_dev.cu:1857-1952), which adds
//     `iters` MTTKRPs into the target factor;
//   * refgpu_cpals128 / refgpu_mttkrp128: the same on the 128-bit build's
//     encoding (gen_blcotensor_host<unsigned __int128>), for keys above 64
//     bits.
// Only the in-memory path is exposed (no --stream-data, no --batch): there
// the swapped arguments of gen_blcotensor_device at src/cpd_gpu.cu:39 pass 0
// and false either way.
//
// gen_alto leaves prtn_ptr, prtn_intervals and cr_masks uninitialised and
// destroy_alto frees them (include/alto.hpp:118, 248-250); posix_memalign is
// therefore replaced inside this library by a zero-filling version (the
// library is linked with -Bsymbolic so only its own calls bind to it).
#include <malloc.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "alto_dev.hpp"
#include "blco.hpp"
#include "cpd_gpu.hpp"
#include "kruskal_model.hpp"
#include "sptensor.hpp"

extern "C" int posix_memalign(void** p, size_t a, size_t n)
{
    void* q = memalign(a, n ? n : 1);
    if (!q) return 12; // ENOMEM
    memset(q, 0, n);
    *p = q;
    return 0;
}

static SparseTensor* refg_make_tensor(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* cidx,
                                      const double* vals)
{
    SparseTensor* X = (SparseTensor*)AlignedMalloc(sizeof(SparseTensor));
    X->nmodes = nmodes;
    X->nnz = nnz;
    X->dims = (IType*)AlignedMalloc(sizeof(IType) * nmodes);
    X->cidx = (IType**)AlignedMalloc(sizeof(IType*) * nmodes);
    for (int n = 0; n < nmodes; n++) {
        X->dims[n] = dims[n];
        X->cidx[n] = (IType*)AlignedMalloc(sizeof(IType) * nnz);
        memcpy(X->cidx[n], cidx + (size_t)n * nnz, sizeof(IType) * nnz);
    }
    X->vals = (FType*)AlignedMalloc(sizeof(FType) * nnz);
    memcpy(X->vals, vals, sizeof(FType) * nnz);
    return X;
}

static KruskalModel* refg_make_model(int nmodes, const uint64_t* dims, int rank, double* const* factors,
                                     const double* lambda)
{
    KruskalModel* M;
    CreateKruskalModel(nmodes, (IType*)dims, rank, &M);
    for (int n = 0; n < nmodes; n++) memcpy(M->U[n], factors[n], sizeof(double) * dims[n] * rank);
    memcpy(M->lambda, lambda, sizeof(double) * rank);
    return M;
}

template <typename LIT>
static double refg_cpals(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* cidx,
                         const double* vals, int rank, double* const* factors, double* lambda, int maxiter,
                         double tol, int kernel, int nprtn, int thread_cf)
{
    SparseTensor* X = refg_make_tensor(nmodes, dims, nnz, cidx, vals);
    blcotensor* T = gen_blcotensor_host<LIT>(X, nnz);
    KruskalModel* M = refg_make_model(nmodes, dims, rank, factors, lambda);
    double fit = cpals_blco_dev(T, M, maxiter, tol, kernel, false, false, thread_cf, nprtn);
    for (int n = 0; n < nmodes; n++) memcpy(factors[n], M->U[n], sizeof(double) * dims[n] * rank);
    memcpy(lambda, M->lambda, sizeof(double) * rank);
    DestroyKruskalModel(M);
    delete_blcotensor_host(T);
    DestroySparseTensor(X);
    return fit;
}

template <typename LIT>
static void refg_mttkrp(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* cidx,
                        const double* vals, int rank, double* const* factors, int mode, int kernel,
                        int iters, int nprtn, int thread_cf)
{
    SparseTensor* X = refg_make_tensor(nmodes, dims, nnz, cidx, vals);
    blcotensor* T = gen_blcotensor_host<LIT>(X, nnz);
    std::vector<double> ones(rank, 1.0);
    KruskalModel* M = refg_make_model(nmodes, dims, rank, factors, ones.data());
    mttkrp_alto_dev<IType>(T, M, kernel, iters, mode, (IType)thread_cf, false, false, nprtn);
    memcpy(factors[mode], M->U[mode], sizeof(double) * dims[mode] * rank);
    DestroyKruskalModel(M);
    delete_blcotensor_host(T);
    DestroySparseTensor(X);
}

extern "C" double refgpu_cpals(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* cidx,
                               const double* vals, int rank, double* const* factors, double* lambda, int maxiter,
                               double tol, int kernel, int nprtn, int thread_cf)
{
    return refg_cpals<unsigned long long>(nmodes, dims, nnz, cidx, vals, rank, factors, lambda, maxiter, tol,
                                          kernel, nprtn, thread_cf);
}

extern "C" void refgpu_mttkrp(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* cidx,
                              const double* vals, int rank, double* const* factors, int mode, int kernel,
                              int iters, int nprtn, int thread_cf)
{
    refg_mttkrp<unsigned long long>(nmodes, dims, nnz, cidx, vals, rank, factors, mode, kernel, iters, nprtn,
                                    thread_cf);
}

// The 128-bit build (cpd128): the tensor encoded by
// gen_blcotensor_host<unsigned __int128>, one block per distinct upper key
// word (max_block_size = nnz), and the same GPU drivers.
extern "C" double refgpu_cpals128(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* cidx,
                                  const double* vals, int rank, double* const* factors, double* lambda,
                                  int maxiter, double tol, int kernel, int nprtn, int thread_cf)
{
    return refg_cpals<unsigned __int128>(nmodes, dims, nnz, cidx, vals, rank, factors, lambda, maxiter, tol,
                                         kernel, nprtn, thread_cf);
}

extern "C" void refgpu_mttkrp128(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* cidx,
                                 const double* vals, int rank, double* const* factors, int mode, int kernel,
                                 int iters, int nprtn, int thread_cf)
{
    refg_mttkrp<unsigned __int128>(nmodes, dims, nnz, cidx, vals, rank, factors, mode, kernel, iters, nprtn,
                                   thread_cf);
}
