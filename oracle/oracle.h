/* Oracle for the talsh-b200 hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference TAL-SH CPU path (CP-TAL,
 * tensor_algebra_cpu.F90, and the C<->Fortran glue in talshf.F90), used by the
 * test-suite as the checker, by __graft_entry__.smoke() as the checker, and by
 * bench.py as the timed CPU baseline.  Nothing in the product library links,
 * loads or calls this code.
 *
 * Conventions match the reference: dense column-major bodies, permutations are
 * 1-based, "O2N" maps an old (input) dimension to its new (output) position.
 * Data kinds are the TAL-SH codes R4=4, R8=8, C4=14, C8=18.
 */
#ifndef TALSH_ORACLE_H_
#define TALSH_ORACLE_H_
#include <stddef.h>

#define ORC_MAX_RANK 56

/* Pattern string -> digital pattern (talshf.F90:619-667 + tensor_algebra_cpu.F90:5307-5531).
 * Returns 0 or the reference's error code. */
int orc_str2dig(const char *s, int *dig, int *drank, int *lrank, int *rrank, int *conj_bits);

/* Digital pattern -> symbolic pattern (tensor_algebra_cpu.F90:5533-5611); out
 * holds at least 16 + 4 * (lrank + rrank) characters.  Returns ierr. */
int orc_pattern_sym(int lrank, int rrank, int conj_bits, const int *dig, char *out, int *cpl);

/* Matricization permutations for GEMM(T,N); CPU variant with hyper-indices
 * (tensor_algebra_cpu.F90:5757-5956). Returns ierr. */
int orc_contraction_permutations(int gemm_tl, int gemm_tr, int lrank, int rrank, const int *cptrn,
                                 int conj_bits, int *dprm, int *lprm, int *rprm, int *ncd,
                                 int *nlu, int *nru, int *nhu);
/* GPU variant without hyper-indices (tensor_algebra_cpu.F90:5613-5755). Returns ierr. */
int orc_contr_permutations(int gemm_tl, int gemm_tr, int lrank, int rrank, const int *cptrn,
                           int conj_bits, int *dprm, int *lprm, int *rprm, int *ncd, int *nlu,
                           int *nru);

/* out[O2N(idx)] = in[idx] (scatter definition of tensor_block_copy_dlf,
 * tensor_algebra_cpu.F90:3151-3310); conj negates imaginary parts of C4/C8. */
int orc_permute(int kind, int rank, const int *dims_in, const int *o2n, const void *in, void *out,
                int conj);
/* Same result through the reference's cache-blocked OpenMP scheme
 * (tensor_algebra_cpu.F90:7699-7940); used as the timed CPU baseline. */
int orc_permute_blocked(int kind, int rank, const int *dims_in, const int *o2n, const void *in,
                        void *out, int nthreads);

/* cpu_tensor_block_copy (talshf.F90:1817-1855). */
int orc_tensor_copy(int kind, const int *cptrn, int rank, const int *ldims, const void *L, void *D,
                    int conj_bits);
/* cpu_tensor_block_add (talshf.F90:1857-1904) -> tensor_block_add (:3312-3673). */
int orc_tensor_add(int kind, const int *cptrn, int rank, const int *ldims, const void *L, void *D,
                   double sr, double si, int conj_bits);
/* The same add as the reference runs it on the host cores: permute into a
 * temporary block with the cache-blocked OpenMP transpose, then one OpenMP add
 * loop (talshf.F90:1857-1904, tensor_algebra_cpu.F90:3312-3673); used as the
 * timed CPU baseline and for fast checks.  Bit-identical to orc_tensor_add. */
int orc_tensor_add_blocked(int kind, int rank, const int *dims_in, const int *o2n, const void *L,
                           void *D, double sr, double si, int nthreads);
/* tensor_block_scale (tensor_algebra_cpu.F90:1821-1890) via cpu_tensor_block_scale. */
int orc_tensor_scale(int kind, size_t vol, void *D, double sr, double si, int conj_bits);
/* tensor_block_init with a value (cpu_tensor_block_init, talshf.F90:1720-1749). */
int orc_tensor_init(int kind, size_t vol, void *D, double sr, double si, int conj_bits);
/* talshTensorImageNorm1_cpu (talshc.cpp:6207-6250): sum of moduli in double. */
double orc_norm1(int kind, size_t vol, const void *D);
/* tensor_block_contract (tensor_algebra_cpu.F90:3675-4358): TTGT with the CPU permutations,
 * a straightforward GEMM accumulated in double, and the back-transpose.
 * Rank-0 operands are single elements of their data kind. */
int orc_tensor_contract(int kind, const int *cptrn, int drank, const int *ddims, int lrank,
                        const int *ldims, int rrank, const int *rdims, void *D, const void *L,
                        const void *R, double sr, double si, int conj_bits, int accumulative);
/* cmplx8_to_real8 (tensor_algebra_cpu.F90:430-445). */
double orc_cmplx8_to_real8(double re, double im);

/* Slicing / insertion (tensor_block_slice_dlf_* tensor_algebra_cpu.F90:6900-6974,
 * tensor_block_insert_dlf_* :7216-7290): dst = dst*beta + src*alpha with alpha = 1,
 * beta = 1 when accumulative else 0, over the sub-block at 0-based offsets. */
int orc_tensor_slice(int kind, int rank, const int *full_dims, const int *slice_dims, const int *offsets,
                     const void *full, void *slice, int accumulative);
int orc_tensor_insert(int kind, int rank, const int *full_dims, const int *slice_dims, const int *offsets,
                      const void *slice, void *full, int accumulative);

/* Seeded generator: mt19937_64 stream, uniform[-1,1] = 2*(x>>11)*2^-53 - 1. */
void orc_fill_uniform(int kind, size_t vol, void *out, unsigned long long seed);

#endif
