/* talsh-b200: low-level constants and interoperable types of the TAL-SH C ABI.
 *
 * Every macro value and struct layout in this header is part of the binary
 * interface that existing TAL-SH callers were compiled against, so they keep
 * the values and field order of the reference header `tensor_algebra.h`
 * (constants :58-203, types :205-256).  The text is written for this core.
 *
 * Layout conventions used across the library:
 *  - dense tensor bodies are column-major ("dimension-led"): index 0 is the
 *    fastest-varying one;
 *  - complex kinds C4/C8 store interleaved (re, im) pairs;
 *  - flat device ids: 0 = Host, 1..8 = NVIDIA GPU 0..7 (then MIC, AMD ranges).
 */
#ifndef TALSH_B200_TENSOR_ALGEBRA_H_
#define TALSH_B200_TENSOR_ALGEBRA_H_

#include <stddef.h>
#include <stdint.h>

/* Global limits */
#define MAX_TENSOR_RANK 56              /* max tensor rank (multiple of 4) */
#define MAX_TENSOR_OPERANDS 4           /* max tensor operands of one operation */
#define MAX_CONTRACTION_PATTERN_LEN 1024 /* max length of a symbolic pattern */
#define MAX_MLNDS_PER_TENS 4

/* Data kinds */
#define NO_TYPE 0
#define R4 4   /* float */
#define R8 8   /* double */
#define C4 14  /* float complex (re, im) */
#define C8 18  /* double complex (re, im) */

/* Device kinds and flat id ranges */
#define MAX_GPUS_PER_NODE 8
#define MAX_MICS_PER_NODE 8
#define MAX_AMDS_PER_NODE 8
#define DEV_NULL -1
#define DEV_DEFAULT DEV_NULL
#define DEV_HOST 0
#define DEV_NVIDIA_GPU 1
#define DEV_INTEL_MIC 2
#define DEV_AMD_GPU 3
#define DEV_MAX (1 + MAX_GPUS_PER_NODE + MAX_MICS_PER_NODE + MAX_AMDS_PER_NODE)

/* Host memory allocation policy */
#define MEM_ALLOC_REGULAR 0
#define MEM_ALLOC_TMP_BUF 1
#define MEM_ALLOC_ALL_BUF 2

/* Aliases and non-error statuses */
#define NOPE 0
#define YEP 1
#define BLAS_ON 0
#define BLAS_OFF 1
#define EFF_TRN_OFF 0
#define EFF_TRN_ON 1
#define EFF_TRN_ON_CUTT 2
#define DEVICE_UNABLE -546372819   /* the device cannot run this request: not an error */
#define TRY_LATER -918273645       /* temporary resource shortage: not an error */
#define NOT_CLEAN -192837465       /* resources released with a warning */
#define NUM_INSTABILITY -374628195

#define EVERYTHING 0
#define SOURCE 1
#define DESTINATION 2
#define TEMPORARY 3

#define DEV_OFF 0
#define DEV_ON 1
#define DEV_ON_BLAS 2
#define GPU_OFF 0
#define GPU_MINE 1
#define GPU_MINE_CUBLAS 2
#define NO_COPY_BACK 0
#define COPY_BACK 1

/* Coherence (copy) control.  Each tensor argument gets two bits
 * (D=discard, M=move, T=temporary, K=keep); the destination tensor owns the
 * senior bits: COPY_XYZ = 16*X + 4*Y + Z with D=0, M=1, T=2, K=3. */
#define COPY_D 0
#define COPY_M 1
#define COPY_T 2
#define COPY_K 3
#define COPY_DD 0
#define COPY_DM 1
#define COPY_DT 2
#define COPY_DK 3
#define COPY_MD 4
#define COPY_MM 5
#define COPY_MT 6
#define COPY_MK 7
#define COPY_TD 8
#define COPY_TM 9
#define COPY_TT 10
#define COPY_TK 11
#define COPY_KD 12
#define COPY_KM 13
#define COPY_KT 14
#define COPY_KK 15
#define COPY_DDD 0
#define COPY_DDM 1
#define COPY_DDT 2
#define COPY_DDK 3
#define COPY_DMD 4
#define COPY_DMM 5
#define COPY_DMT 6
#define COPY_DMK 7
#define COPY_DTD 8
#define COPY_DTM 9
#define COPY_DTT 10
#define COPY_DTK 11
#define COPY_DKD 12
#define COPY_DKM 13
#define COPY_DKT 14
#define COPY_DKK 15
#define COPY_MDD 16
#define COPY_MDM 17
#define COPY_MDT 18
#define COPY_MDK 19
#define COPY_MMD 20
#define COPY_MMM 21
#define COPY_MMT 22
#define COPY_MMK 23
#define COPY_MTD 24
#define COPY_MTM 25
#define COPY_MTT 26
#define COPY_MTK 27
#define COPY_MKD 28
#define COPY_MKM 29
#define COPY_MKT 30
#define COPY_MKK 31
#define COPY_TDD 32
#define COPY_TDM 33
#define COPY_TDT 34
#define COPY_TDK 35
#define COPY_TMD 36
#define COPY_TMM 37
#define COPY_TMT 38
#define COPY_TMK 39
#define COPY_TTD 40
#define COPY_TTM 41
#define COPY_TTT 42
#define COPY_TTK 43
#define COPY_TKD 44
#define COPY_TKM 45
#define COPY_TKT 46
#define COPY_TKK 47
#define COPY_KDD 48
#define COPY_KDM 49
#define COPY_KDT 50
#define COPY_KDK 51
#define COPY_KMD 52
#define COPY_KMM 53
#define COPY_KMT 54
#define COPY_KMK 55
#define COPY_KTD 56
#define COPY_KTM 57
#define COPY_KTT 58
#define COPY_KTK 59
#define COPY_KKD 60
#define COPY_KKM 61
#define COPY_KKT 62
#define COPY_KKK 63

/* Interoperable types (field order is ABI). */
typedef struct {
  int num_dim;      /* rank, -1 = empty */
  size_t *offsets;  /* base offsets of each dimension */
} talsh_tens_signature_t;

typedef struct {
  int num_dim;  /* rank, -1 = empty */
  int *dims;    /* extents */
  int *divs;    /* dimension dividers */
  int *grps;    /* dimension groups */
} talsh_tens_shape_t;

typedef struct {
  void *base;
  size_t volume;
  int data_kind;
} talsh_tens_data_t;

typedef struct {
  int num_dim;
  int data_kind;
  void *body;
  size_t bases[MAX_TENSOR_RANK];
  size_t dims[MAX_TENSOR_RANK];
} talsh_tens_dense_t;

/* One body image of a tensor on one device. */
typedef struct {
  int dev_id;        /* flat device id, -1 = none */
  void *gmem_p;      /* body pointer in that device's memory */
  int buf_entry;     /* allocator handle (>=0) or -1 */
  int mem_attached;  /* 1 = caller-owned memory, never freed by the library */
} talsh_dev_rsc_t;

/* User-defined initializer for a freshly allocated Host body. */
typedef int (*talsh_tens_init_i)(const talsh_tens_data_t *tens_data,
                                 const talsh_tens_shape_t *tens_shape,
                                 const talsh_tens_signature_t *tens_signature);

/* C++ default arguments, as in the reference headers (none in C). */
#ifndef TALSH_DEFAULT
#ifdef __cplusplus
#define TALSH_DEFAULT(x) = x
#else
#define TALSH_DEFAULT(x)
#endif
#endif

#ifdef __cplusplus
extern "C" {
#endif
/* Initializer that leaves the body untouched. */
int talsh_tens_no_init(const talsh_tens_data_t *, const talsh_tens_shape_t *,
                       const talsh_tens_signature_t *);
/* YEP if datk is a valid data kind (NO_TYPE included); its byte size in *datk_size. */
int tens_valid_data_kind(int datk, int *datk_size TALSH_DEFAULT(NULL));
int tens_valid_data_kind_(int datk, int *datk_size);
/* YEP if perm[base..base+perm_len-1] is the identity (values 1-based). */
int permutation_trivial(const int perm_len, const int *perm, const int base TALSH_DEFAULT(0));
/* Two-bit coherence component of argument arg_num out of tot_args. */
unsigned int argument_coherence_get_value(unsigned int coh_ctrl, unsigned int tot_args,
                                          unsigned int arg_num);
int argument_coherence_set_value(unsigned int *coh_ctrl, unsigned int tot_args,
                                 unsigned int arg_num, unsigned int coh_val);
/* Flat device id codec. */
int valid_device_kind(int dev_kind);
int encode_device_id(int dev_kind, int dev_num);
int decode_device_id(int dev_id, int *dev_kind);
/* Digital contraction pattern -> matricization permutations (GEMM 'T','N').
 * dprm is N2O, lprm/rprm are O2N, all with element 0 = sign, 1-based values. */
void get_contr_permutations(int gemm_tl, int gemm_tr, int lrank, int rrank, const int *cptrn,
                            int conj_bits, int *dprm, int *lprm, int *rprm, int *ncd, int *nlu,
                            int *nru, int *ierr);
void get_contraction_permutations(int gemm_tl, int gemm_tr, int lrank, int rrank,
                                  const int *cptrn, int conj_bits, int *dprm, int *lprm,
                                  int *rprm, int *ncd, int *nlu, int *nru, int *nhu, int *ierr);
/* Digital pattern -> symbolic pattern string (reference tensor_algebra.h:265,
 * tensor_algebra_cpu.F90:5533-5611); *cpl = its length, *ierr = 0 on success. */
void get_contr_pattern_sym(const int *rank_left, const int *rank_right, const int *conj_bits,
                           const int *cptrn_dig, char *cptrn_sym, int *cpl, int *ierr);
/* Symbolic pattern string -> digital pattern (0 = success). */
int talsh_get_contr_ptrn_str2dig(const char *c_str, int *dig_ptrn, int *drank, int *lrank,
                                 int *rrank, int *conj_bits);
/* Shape helpers. */
int tensShape_create(talsh_tens_shape_t **tshape);
int tensShape_clean(talsh_tens_shape_t *tshape);
int tensShape_construct(talsh_tens_shape_t *tshape, int pinned, int rank, const int *dims,
                        const int *divs, const int *grps);
int tensShape_destruct(talsh_tens_shape_t *tshape);
int tensShape_destroy(talsh_tens_shape_t *tshape);
size_t tensShape_volume(const talsh_tens_shape_t *tshape);
int tensShape_rank(const talsh_tens_shape_t *tshape);
/* New extents of the same volume: 0, or -2 when the volume changed (the new
 * shape stays), -3 / -4 for a shape without extents / extents for rank 0. */
int tensShape_reshape(talsh_tens_shape_t *tshape, int rank, const int *dims TALSH_DEFAULT(NULL),
                      const int *divs TALSH_DEFAULT(NULL), const int *grps TALSH_DEFAULT(NULL));
/* Prints the extents as "[d1,d2,...]". */
void tensShape_print(const talsh_tens_shape_t *tshape);
/* Tensor signatures (reference tensor_algebra.h:298-304). */
int tensSignature_create(talsh_tens_signature_t **tsigna);
int tensSignature_clean(talsh_tens_signature_t *tsigna);
int tensSignature_construct(talsh_tens_signature_t *tsigna, int rank, const size_t *offsets TALSH_DEFAULT(NULL));
int tensSignature_destruct(talsh_tens_signature_t *tsigna);
int tensSignature_destroy(talsh_tens_signature_t *tsigna);
/* A C pointer as an integer, for Fortran callers. */
size_t fortran_cptr_int(void *cptr);
/* Column-major element offset <-> zero-based multi-index (reference
 * tensor_algebra.h:274-275). */
size_t tens_elem_offset_f(unsigned int num_dim, const unsigned int *dims, const unsigned int *mlndx);
void tens_elem_mlndx_f(size_t offset, unsigned int num_dim, const unsigned int *dims, unsigned int *mlndx);
/* Device resource helpers. */
int tensDevRsc_clean(talsh_dev_rsc_t *drsc);
int tensDevRsc_is_empty(talsh_dev_rsc_t *drsc);
int tensDevRsc_device_id(talsh_dev_rsc_t *drsc);
/* Device-resource descriptors (reference tensor_algebra.h:283-295,
 * tensor_algebra_gpu.cpp:278-555), with the reference's return codes.  Allocated
 * memory comes from the library's allocators (Host: pinned when a GPU is in use;
 * GPU: the stream-ordered pool under its budget, TRY_LATER above it); there is
 * no argument buffer, so in_arg_buf is ignored. */
int tensDevRsc_create(talsh_dev_rsc_t **drsc);
int tensDevRsc_same(const talsh_dev_rsc_t *drsc0, const talsh_dev_rsc_t *drsc1);
int tensDevRsc_clone(const talsh_dev_rsc_t *drsc_in, talsh_dev_rsc_t *drsc_out);
int tensDevRsc_attach_mem(talsh_dev_rsc_t *drsc, int dev_id, void *mem_p, int buf_entry TALSH_DEFAULT(-1));
int tensDevRsc_detach_mem(talsh_dev_rsc_t *drsc);
int tensDevRsc_allocate_mem(talsh_dev_rsc_t *drsc, int dev_id, size_t mem_size, int in_arg_buf TALSH_DEFAULT(NOPE));
int tensDevRsc_free_mem(talsh_dev_rsc_t *drsc);
int tensDevRsc_get_gmem_ptr(talsh_dev_rsc_t *drsc, void **gmem_p);
int tensDevRsc_release_all(talsh_dev_rsc_t *drsc);
int tensDevRsc_destroy(talsh_dev_rsc_t *drsc);
#ifdef __cplusplus
}
#endif

#endif /* TALSH_B200_TENSOR_ALGEBRA_H_ */
