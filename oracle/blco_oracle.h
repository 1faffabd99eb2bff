/*
 * blco_oracle.h -- CPU oracle for the BLCO encoder, MTTKRP and GPU CP-ALS.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithms (jeewhanchoi/blocked-linearized-coordinate), used by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker.
 * No product code path links, loads or calls it.
 *
 * Parity pin: the encoder restatement is checked bit-exactly against the
 * known-answer vectors in tests/golden/ (produced by the reference encoder
 * compiled from its own sources, oracle/ref_harness.cpp) and, where
 * oracle/_ref is built, against that reference build on random inputs.
 * The MTTKRP restatement follows the reference's sequential COO MTTKRP
 * (include/cpd.hpp:510-544), which is the reference's own -c check oracle.
 * The CP-ALS restatement follows src/cpd_gpu.cu:21-242; no reference test
 * pins CP-ALS numbers, so that part is pinned only through the MTTKRP and
 * encoder pins plus the algebraic identities tested in tests/.
 */
#ifndef BLCO_ORACLE_H_
#define BLCO_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_MODES 5

/* Software bit deposit / extract, the ALT_PEXT variants of
 * include/bitops.hpp:18-41. */
uint64_t orc_pdep(uint64_t x, uint64_t mask);
uint64_t orc_pext(uint64_t x, uint64_t mask);

/* Bits needed for a mode of length dim: 64 - clz(dim - 1)
 * (include/alto.hpp:613).  dim == 1 is undefined in the reference
 * (clz(0)); here it is 0 bits. */
int orc_mode_bits(uint64_t dim);

/* ALTO interleaved masks, setup_packed_alto(LSB_FIRST, SHORT_FIRST)
 * (include/alto.hpp:597-695).  Returns the total bit count, or -1 if it
 * exceeds 64 bits or nmodes is out of range. */
int orc_alto_masks(int nmodes, const uint64_t* dims, uint64_t* alto_masks);

/* BLCO encoding of a COO tensor, gen_blcotensor_host<uint64>
 * (include/blco.hpp:196-331) via gen_alto + sort_alto
 * (include/alto.hpp:107-186, 704-754).
 *   cidx:       nmodes arrays of nnz 0-based coordinates, mode-major
 *               (cidx[n*nnz + i]).
 *   coords_out, vals_out: nnz entries, ALTO order.
 *   mode_masks_out[n] = (1 << bits_n) - 1, mode_pos_out[n] = prefix of bits.
 *   alto_masks_out[n]: the interleaved masks.
 *   nblocks_out: number of blocks; block_offsets_out (nnz/B + 2 entries)
 *               gets the block start offsets plus the end offset.
 * Ties between equal keys keep input order (the reference's std::sort
 * leaves them unspecified).  Returns 0, or -1 on invalid input. */
int orc_blco_encode(int nmodes, const uint64_t* dims, uint64_t nnz,
                    const uint64_t* cidx, const double* vals,
                    uint64_t max_block_size,
                    uint64_t* coords_out, double* vals_out,
                    uint64_t* mode_masks_out, int* mode_pos_out,
                    uint64_t* alto_masks_out,
                    uint64_t* nblocks_out, uint64_t* block_offsets_out);

/* 128-bit ALTO masks (ALTO_MASK_LENGTH=128, include/alto.hpp:597-695):
 * low and high mask words per mode.  Returns the total bit count, or -1
 * above 128 bits. */
int orc_alto_masks128(int nmodes, const uint64_t* dims, uint64_t* masks_lo, uint64_t* masks_hi);

/* BLCO encoding with 128-bit ALTO keys, gen_blcotensor_host<__uint128_t>
 * (include/blco.hpp:196-331).  Fields hold each mode's low-key-word bits
 * (mode_masks_out[n] = (1 << t_n) - 1, t_n = popcount(low mask word));
 * blocks are the runs of equal upper key words in sorted order, each split
 * into max_block_size slices, with block_coords_out[b*nmodes + n] =
 * pext(upper word, upper mask word n) << t_n.  block_offsets_out needs
 * room for nnz + 1 entries, block_coords_out for nnz * nmodes.  With at
 * most 64 key bits the result equals orc_blco_encode's. */
int orc_blco_encode128(int nmodes, const uint64_t* dims, uint64_t nnz,
                       const uint64_t* cidx, const double* vals,
                       uint64_t max_block_size,
                       uint64_t* coords_out, double* vals_out,
                       uint64_t* mode_masks_out, int* mode_pos_out,
                       uint64_t* alto_lo_out, uint64_t* alto_hi_out,
                       uint64_t* nblocks_out, uint64_t* block_offsets_out,
                       uint64_t* block_coords_out);

/* MTTKRP over a blocked encoding: row = field | block coordinate
 * (src/alto_dev.cu:13-16); out += (dims[mode] x rank, zeroed by caller). */
void orc_mttkrp_blco128(int nmodes, const uint64_t* mode_masks, const int* mode_pos, uint64_t nblocks,
                        const uint64_t* block_offsets, const uint64_t* block_coords, const uint64_t* coords,
                        const double* vals, const double* const* factors, int rank, int mode, double* out);

/* Sequential COO MTTKRP, include/cpd.hpp:510-544:
 *   out[c_mode(i), :] += val_i * prod_{m != mode} U_m[c_m(i), :]
 * factors[m] row-major dims[m] x rank.  out accumulates (not zeroed). */
void orc_mttkrp_coo(int nmodes, uint64_t nnz, const uint64_t* cidx,
                    const double* vals, int rank, const double* const* factors,
                    int mode, double* out);

/* The same product over a BLCO stream: the row of mode n of entry i is
 * (coords[i] >> pos_n) & mask_n, as alt_pext in src/alto_dev.cu:13-16. */
void orc_mttkrp_blco(int nmodes, const uint64_t* mode_masks,
                     const int* mode_pos, uint64_t nnz, const uint64_t* coords,
                     const double* vals, int rank,
                     const double* const* factors, int mode, double* out);

/* Symmetric pseudoinverse with the reference's cut-off
 * (src/cpd_gpu.cu:452-532): eigenvalues with |s| <= n*ulp(max|s|) are
 * dropped.  a is n x n (symmetric), p receives the pseudoinverse.
 * Cyclic Jacobi eigen-decomposition (Golub & Van Loan, Alg. 8.5.3). */
int orc_pinv_sym(int n, const double* a, double* p);

/* CP-ALS exactly as cpals_blco_dev (src/cpd_gpu.cu:21-242), in FP64 on the
 * CPU:
 *   modes in descending length order (ties keep natural order);
 *   per mode: MTTKRP, V = hadamard of the other Grams, P = pinv(V),
 *   U_n = M P^T, lambda_c <- sqrt(lambda_c + sum_i U_n[i,c]^2) (lambda is
 *   never reset, src/cpd_gpu.cu:244-291), U_n[:,c] /= lambda_c, Gram_n;
 *   fit as kruskal_fit_gpu (src/cpd_gpu.cu:331-384), stop when
 *   |fit - fit_old| < tol or fit is NaN, fit_old starting at 0.
 * factors (row-major dims[n] x rank) and lambda are updated in place.
 * fits receives one fit per executed iteration.  Returns the number of
 * iterations executed. */
int orc_cpals(int nmodes, const uint64_t* dims, const uint64_t* mode_masks,
              const int* mode_pos, uint64_t nnz, const uint64_t* coords,
              const double* vals, int rank, double* const* factors,
              double* lambda, int maxiter, double tol, double* fits);

/* The same CP-ALS with the MTTKRP taken from the COO tensor (cidx as in
 * orc_blco_encode), for encodings with block coordinates. */
int orc_cpals_coo(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* cidx,
                  const double* vals, int rank, double* const* factors,
                  double* lambda, int maxiter, double tol, double* fits);

/* KruskalModelRandomInit (src/kruskal_model.cpp:93-110): lambda = 1 and
 * U_n[i] = rand_r(&s_t) / RAND_MAX where thread t of nthreads owns a static
 * contiguous chunk of dims[n]*rank entries and s_t = seed + t, reset for
 * every mode. */
void orc_kruskal_random_init(int nmodes, const uint64_t* dims, int rank,
                             unsigned int seed, int nthreads,
                             double* const* factors, double* lambda);

#ifdef __cplusplus
}
#endif

#endif
