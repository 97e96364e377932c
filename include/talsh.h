/* talsh-b200: the TAL-SH device-unified C API, served by a B200-native core.
 *
 * This header is the drop-in boundary.  Names, argument order and meaning,
 * return codes and struct layouts follow the reference `talsh.h` (types
 * :84-136, prototypes :143-596) so that callers compiled against TAL-SH
 * rebuild unchanged.  Default arguments exist only for C++ callers, as in the
 * reference; every defaulted entry point also has a `_`-suffixed twin without
 * defaults.
 *
 * Execution model of this implementation:
 *  - Every tensor operation executes on an NVIDIA GPU (sm_100a kernels written
 *    for this library).  Requests that name DEV_HOST as the execution device
 *    return TALSH_NOT_AVAILABLE: there is no CPU compute path.  Host images of
 *    tensors remain fully supported as data (construction, import, transfer).
 *  - A call with talsh_task == NULL blocks until the operation completed; with
 *    a clean task it returns after scheduling on a CUDA stream and the task is
 *    completed by talshTaskComplete / talshTaskWait.
 *  - Scheduling is single-threaded: one host thread issues TAL-SH calls.
 *  - Entry points of the reference that this core does not provide (SVD,
 *    orthogonalization, tensor-operation objects) return
 *    TALSH_NOT_IMPLEMENTED; talshTensorSlice / talshTensorInsert run on the
 *    GPU, and slice descriptor objects are host-side views.
 */
#ifndef TALSH_B200_TALSH_H_
#define TALSH_B200_TALSH_H_

#include "tensor_algebra.h"

#ifndef TALSH_DEFAULT
#ifdef __cplusplus
#define TALSH_DEFAULT(x) = x
#else
#define TALSH_DEFAULT(x)
#endif
#endif

/* Parameters */
#define TALSH_MAX_DEV_PRESENT 16         /* max body images per tensor */
#define TALSH_MEM_ALLOC_POLICY_HOST MEM_ALLOC_TMP_BUF
#define TALSH_MEM_ALLOC_FALLBACK_HOST 1
#define TALSH_CPTAL_MIN_BUF_SIZE 1073741824
#define TALSH_NO_HOST_BUFFER 16777216
#define TALSH_GFLOP_THRESH_GPU 4

/* Error codes */
#define TALSH_SUCCESS 0
#define TALSH_FAILURE -666
#define TALSH_NOT_AVAILABLE -888
#define TALSH_NOT_IMPLEMENTED -999
#define TALSH_NOT_INITIALIZED 1000000
#define TALSH_ALREADY_INITIALIZED 1000001
#define TALSH_INVALID_ARGS 1000002
#define TALSH_INTEGER_OVERFLOW 1000003
#define TALSH_OBJECT_NOT_EMPTY 1000004
#define TALSH_OBJECT_IS_EMPTY 1000005
#define TALSH_IN_PROGRESS 1000006
#define TALSH_NOT_ALLOWED 1000007
#define TALSH_LIMIT_EXCEEDED 1000008
#define TALSH_NOT_FOUND 1000009
#define TALSH_OBJECT_BROKEN 1000010
#define TALSH_INVALID_REQUEST 1000011

/* Task status */
#define TALSH_TASK_ERROR 1999999
#define TALSH_TASK_EMPTY 2000000
#define TALSH_TASK_SCHEDULED 2000001
#define TALSH_TASK_STARTED 2000002
#define TALSH_TASK_INPUT_READY 2000003
#define TALSH_TASK_OUTPUT_READY 2000004
#define TALSH_TASK_COMPLETED 2000005

/* Tensor operation kinds */
#define TALSH_TENSOR_NOOP -1
#define TALSH_TENSOR_INIT 68
#define TALSH_TENSOR_NORM1 69
#define TALSH_TENSOR_NORM2 70
#define TALSH_TENSOR_MIN 71
#define TALSH_TENSOR_MAX 72
#define TALSH_TENSOR_FOLD 73
#define TALSH_TENSOR_UNFOLD 74
#define TALSH_TENSOR_SLICE 75
#define TALSH_TENSOR_INSERT 76
#define TALSH_TENSOR_COPY 77
#define TALSH_TENSOR_PERMUTE 78
#define TALSH_TENSOR_SCALE 79
#define TALSH_TENSOR_ADD 80
#define TALSH_TENSOR_TRACE 81
#define TALSH_TENSOR_CONTRACT 82
#define TALSH_TENSOR_HADAMARD 83
#define TALSH_TENSOR_KHATRIRAO 84

/* Tensor operation stages */
#define TALSH_OP_UNDEFINED -1
#define TALSH_OP_EMPTY 0
#define TALSH_OP_PARTIAL 1
#define TALSH_OP_DEFINED 2
#define TALSH_OP_RESOURCED 3
#define TALSH_OP_LOADED 4
#define TALSH_OP_SCHEDULED 5
#define TALSH_OP_COMPLETED 6
#define TALSH_OP_STORED 7
#define TALSH_OP_RETIRED 8

/* Dense tensor with up to TALSH_MAX_DEV_PRESENT body images. */
typedef struct {
  talsh_tens_shape_t *shape_p;  /* shape */
  talsh_dev_rsc_t *dev_rsc;     /* body image per device */
  int *data_kind;               /* data kind of each image */
  int *avail;                   /* YEP if the image may be used */
  int dev_rsc_len;              /* capacity of the three arrays */
  int ndev;                     /* images present */
} talsh_tens_t;

typedef struct {
  talsh_tens_t *tensor;
  talsh_tens_signature_t bases;
  talsh_tens_shape_t shape;
} talsh_tens_slice_t;

typedef struct {
  talsh_tens_t *tens_p;
  int source_image;
} talshTensArg_t;

/* Task handle: task_p points to this library's device task record. */
typedef struct {
  void *task_p;
  int task_error;   /* -1 pending/empty, 0 success, >0 error */
  int dev_kind;
  int data_kind;
  int coherence;
  int num_args;
  talshTensArg_t tens_args[MAX_TENSOR_OPERANDS];
  double data_vol;
  double flops;
  double exec_time;
} talsh_task_t;

typedef struct {
  int opkind;
  int data_kind;
  unsigned int num_args;
  talsh_tens_slice_t tens_slice[MAX_TENSOR_OPERANDS];
  const char *symb_pattern;
  double alpha_real;
  double alpha_imag;
  talsh_tens_t tens_arg[MAX_TENSOR_OPERANDS];
  talsh_task_t task_handle;
  int exec_dev_id;
  int stage;
  double time_started;
  double time_scheduled;
  double time_completed;
  double time_finished;
} talsh_tens_op_t;

#ifdef __cplusplus
extern "C" {
#endif
/* Timers */
double time_sys_sec(void);
double time_high_sec(void);

/* Helpers and control */
int talshValidDataKind(int datk, int *datk_size);
int talshInit(size_t *host_buf_size, int *host_arg_max, int ngpus, int gpu_list[], int nmics,
              int mic_list[], int namds, int amd_list[]);
int talshShutdown(void);
void talshSetMemAllocPolicyHost(int mem_policy, int fallback, int *ierr);
int talshEnableFastMath(int dev_kind, int dev_id TALSH_DEFAULT(DEV_DEFAULT));
int talshDisableFastMath(int dev_kind, int dev_id TALSH_DEFAULT(DEV_DEFAULT));
int talshQueryFastMath(int dev_kind, int dev_id);
int talshDeviceCount(int dev_kind, int *dev_count);
int talshFlatDevId(int dev_kind, int dev_num);
int talshKindDevId(int dev_id, int *dev_kind);
int talshDeviceState(int dev_num, int dev_kind TALSH_DEFAULT(DEV_NULL));
int talshDeviceState_(int dev_num, int dev_kind);
int talshDeviceBusyLeast(int dev_kind TALSH_DEFAULT(DEV_NULL));
int talshDeviceBusyLeast_(int dev_kind);
int talshDetermineOptimalDevice(const talsh_tens_t *tens0,
                                const talsh_tens_t *tens1 TALSH_DEFAULT(NULL),
                                const talsh_tens_t *tens2 TALSH_DEFAULT(NULL));
size_t talshDeviceMemorySize(int dev_num, int dev_kind TALSH_DEFAULT(DEV_NULL));
size_t talshDeviceMemorySize_(int dev_num, int dev_kind);
size_t talshDeviceBufferSize(int dev_num, int dev_kind TALSH_DEFAULT(DEV_NULL));
size_t talshDeviceBufferSize_(int dev_num, int dev_kind);
size_t talshDeviceTensorSize(int dev_num, int dev_kind TALSH_DEFAULT(DEV_NULL));
size_t talshDeviceTensorSize_(int dev_num, int dev_kind);
size_t talshDeviceBufferFreeSize(int dev_num, int dev_kind TALSH_DEFAULT(DEV_NULL));
size_t talshDeviceBufferFreeSize_(int dev_num, int dev_kind);
void *talshDeviceBufferBasePtr(int dev_num, int dev_kind TALSH_DEFAULT(DEV_NULL));
void *talshDeviceBufferBasePtr_(int dev_num, int dev_kind);
double talshDeviceGetFlops(int dev_kind TALSH_DEFAULT(DEV_DEFAULT),
                           int dev_id TALSH_DEFAULT(DEV_DEFAULT));
void talshMemManagerLogStart(void);
void talshMemManagerLogFinish(void);
void talshTensorOpLogStart(void);
void talshTensorOpLogFinish(void);
int talshStats(int dev_id TALSH_DEFAULT(-1), int dev_kind TALSH_DEFAULT(DEV_NULL));
int talshStats_(int dev_id, int dev_kind);

/* Tensor block API */
int talshTensorCreate(talsh_tens_t **tens_block);
int talshTensorClean(talsh_tens_t *tens_block);
int talshTensorIsEmpty(const talsh_tens_t *tens_block);
int talshTensorConstruct(talsh_tens_t *tens_block, int data_kind, int tens_rank,
                         const int tens_dims[], int dev_id TALSH_DEFAULT(0),
                         void *ext_mem TALSH_DEFAULT(NULL), int in_hab TALSH_DEFAULT(-1),
                         talsh_tens_init_i init_method TALSH_DEFAULT(NULL),
                         double init_val_real TALSH_DEFAULT(0.0),
                         double init_val_imag TALSH_DEFAULT(0.0));
int talshTensorConstruct_(talsh_tens_t *tens_block, int data_kind, int tens_rank,
                          const int tens_dims[], int dev_id, void *ext_mem, int in_hab,
                          talsh_tens_init_i init_method, double init_val_real,
                          double init_val_imag);
int talshTensorImportData(talsh_tens_t *tens_block, int data_kind, const void *ext_data);
int talshTensorDestruct(talsh_tens_t *tens_block);
int talshTensorDestroy(talsh_tens_t *tens_block);
int talshTensorRank(const talsh_tens_t *tens_block);
size_t talshTensorVolume(const talsh_tens_t *tens_block);
size_t talshTensorSizeAllImages(const talsh_tens_t *tens_block, int *num_images);
const int *talshTensorDimExtents(const talsh_tens_t *tens_block, int *rank);
int talshTensorShape(const talsh_tens_t *tens_block, talsh_tens_shape_t *tens_shape);
int talshTensorDataKind(const talsh_tens_t *tens_block, int *num_images, int *data_kinds);
int talshTensorReshape(talsh_tens_t *tens_block, int tens_rank, const int tens_dims[]);
int talshTensorInUse(const talsh_tens_t *tens_block);
int talshTensorPresence(const talsh_tens_t *tens_block, int *ncopies, int copies[],
                        int data_kinds[], int dev_kind TALSH_DEFAULT(DEV_NULL),
                        int dev_id TALSH_DEFAULT(-1));
int talshTensorPresence_(const talsh_tens_t *tens_block, int *ncopies, int copies[],
                         int data_kinds[], int dev_kind, int dev_id);
int talshTensorGetBodyAccess(talsh_tens_t *tens_block, void **body_p, int data_kind, int dev_id,
                             int dev_kind TALSH_DEFAULT(DEV_NULL));
int talshTensorGetBodyAccess_(talsh_tens_t *tens_block, void **body_p, int data_kind, int dev_id,
                              int dev_kind);
int talshTensorGetBodyAccessConst(const talsh_tens_t *tens_block, const void **body_p,
                                  int data_kind, int dev_id, int dev_kind TALSH_DEFAULT(DEV_NULL));
int talshTensorGetScalar(talsh_tens_t *tens_block, double *scalar_real, double *scalar_imag);
void talshTensorPrint(const talsh_tens_t *tens_block);
void talshTensorPrintInfo(const talsh_tens_t *tens_block);
void talshTensorPrintBody(const talsh_tens_t *tens_block, double thresh);

/* Tensor slice descriptor objects: a non-owning pointer to a tensor, the base
 * offsets of a window inside it and the window's extents (reference
 * talshc.cpp:1857-1932; host-side only).  Construct refuses a window that leaves
 * the tensor (TALSH_INVALID_ARGS) and releases a previous window's extents. */
int talshTensorSliceCreate(talsh_tens_slice_t **slice);
int talshTensorSliceClean(talsh_tens_slice_t *slice);
int talshTensorSliceConstruct(talsh_tens_slice_t *slice, const talsh_tens_t *tensor,
                              const size_t *offsets, const int *dims,
                              const int *divs TALSH_DEFAULT(NULL),
                              const int *grps TALSH_DEFAULT(NULL));
size_t talshTensorSliceVolume(const talsh_tens_slice_t *slice);
int talshTensorSliceDestruct(talsh_tens_slice_t *slice);
int talshTensorSliceDestroy(talsh_tens_slice_t *slice);

/* Task API */
int talshTaskCreate(talsh_task_t **talsh_task);
int talshTaskClean(talsh_task_t *talsh_task);
int talshTaskIsEmpty(const talsh_task_t *talsh_task);
int talshTaskDestruct(talsh_task_t *talsh_task);
int talshTaskDestroy(talsh_task_t *talsh_task);
int talshTaskDevId(talsh_task_t *talsh_task, int *dev_kind TALSH_DEFAULT(NULL));
int talshTaskDevId_(talsh_task_t *talsh_task, int *dev_kind);
int talshTaskArgCoherence(const talsh_task_t *talsh_task);
const talshTensArg_t *talshTaskTensArgs(const talsh_task_t *talsh_task, int *num_args);
int talshTaskStatus(talsh_task_t *talsh_task);
int talshTaskComplete(talsh_task_t *talsh_task, int *stats, int *ierr);
int talshTaskWait(talsh_task_t *talsh_task, int *stats);
int talshTasksWait(int ntasks, talsh_task_t talsh_tasks[], int stats[]);
int talshTaskTime(talsh_task_t *talsh_task, double *total, double *comput TALSH_DEFAULT(NULL),
                  double *input TALSH_DEFAULT(NULL), double *output TALSH_DEFAULT(NULL),
                  double *mmul TALSH_DEFAULT(NULL));
int talshTaskTime_(talsh_task_t *talsh_task, double *total, double *comput, double *input,
                   double *output, double *mmul);
void talshTaskPrint(const talsh_task_t *talsh_task);

/* Tensor-operation objects (not provided by this core: TALSH_NOT_IMPLEMENTED) */
int talshTensorOpCreate(talsh_tens_op_t **tens_op);
int talshTensorOpClean(talsh_tens_op_t *tens_op);
int talshTensorOpSetArgument(talsh_tens_op_t *tens_op, const talsh_tens_t *tensor,
                             const size_t *offsets, const int *dims);
int talshTensorOpSpecify(talsh_tens_op_t *tens_op, int operation_kind, int data_kind,
                         const char *symbolic_pattern TALSH_DEFAULT(NULL),
                         double prefactor_real TALSH_DEFAULT(1.0),
                         double prefactor_imag TALSH_DEFAULT(0.0));
int talshTensorOpSetExecDevice(talsh_tens_op_t *tens_op, int dev_id,
                               int dev_kind TALSH_DEFAULT(DEV_DEFAULT));
int talshTensorOpActivate(talsh_tens_op_t *tens_op);
int talshTensorOpLoadInput(talsh_tens_op_t *tens_op);
int talshTensorOpExecute(talsh_tens_op_t *tens_op, int dev_id TALSH_DEFAULT(DEV_DEFAULT),
                         int dev_kind TALSH_DEFAULT(DEV_DEFAULT));
int talshTensorOpTest(talsh_tens_op_t *tens_op, int *completed, int wait TALSH_DEFAULT(NOPE));
int talshTensorOpStoreOutput(talsh_tens_op_t *tens_op);
int talshTensorOpDeactivate(talsh_tens_op_t *tens_op);
int talshTensorOpDestruct(talsh_tens_op_t *tens_op);
int talshTensorOpDestroy(talsh_tens_op_t *tens_op);
int talshTensorOpProgress(talsh_tens_op_t *tens_op, int *done);
size_t talshTensorOpGetArgVolume(const talsh_tens_op_t *tens_op, unsigned int arg_num);
size_t talshTensorOpGetArgSize(const talsh_tens_op_t *tens_op, unsigned int arg_num);
double talshTensorOpGetByteCount(const talsh_tens_op_t *tens_op,
                                 unsigned int element_size TALSH_DEFAULT(1));
double talshTensorOpGetFlopCount(const talsh_tens_op_t *tens_op);
double talshTensorOpGetIntensity(const talsh_tens_op_t *tens_op);
int talshTensorOpDecompose2(const talsh_tens_op_t *tens_op, talsh_tens_op_t *child_op1,
                            talsh_tens_op_t *child_op2);
void talshTensorOpPrint(const talsh_tens_op_t *tens_op);

/* Data placement and tensor operations */
int talshTensorPlace(talsh_tens_t *tens, int dev_id, int dev_kind TALSH_DEFAULT(DEV_NULL),
                     void *dev_mem TALSH_DEFAULT(NULL), int copy_ctrl TALSH_DEFAULT(COPY_M),
                     talsh_task_t *talsh_task TALSH_DEFAULT(NULL));
int talshTensorPlace_(talsh_tens_t *tens, int dev_id, int dev_kind, void *dev_mem, int copy_ctrl,
                      talsh_task_t *talsh_task);
int talshTensorDiscard(talsh_tens_t *tens, int dev_id, int dev_kind TALSH_DEFAULT(DEV_NULL));
int talshTensorDiscard_(talsh_tens_t *tens, int dev_id, int dev_kind);
int talshTensorDiscardOther(talsh_tens_t *tens, int dev_id, int dev_kind TALSH_DEFAULT(DEV_NULL));
int talshTensorDiscardOther_(talsh_tens_t *tens, int dev_id, int dev_kind);
int talshTensorInit(talsh_tens_t *dtens, double val_real, double val_imag,
                    int dev_id TALSH_DEFAULT(DEV_DEFAULT), int dev_kind TALSH_DEFAULT(DEV_DEFAULT),
                    int copy_ctrl TALSH_DEFAULT(COPY_M),
                    talsh_task_t *talsh_task TALSH_DEFAULT(NULL));
int talshTensorInit_(talsh_tens_t *dtens, double val_real, double val_imag, int dev_id,
                     int dev_kind, int copy_ctrl, talsh_task_t *talsh_task);
int talshTensorScale(talsh_tens_t *dtens, double val_real, double val_imag,
                     int dev_id TALSH_DEFAULT(DEV_DEFAULT), int dev_kind TALSH_DEFAULT(DEV_DEFAULT),
                     int copy_ctrl TALSH_DEFAULT(COPY_M),
                     talsh_task_t *talsh_task TALSH_DEFAULT(NULL));
int talshTensorScale_(talsh_tens_t *dtens, double val_real, double val_imag, int dev_id,
                      int dev_kind, int copy_ctrl, talsh_task_t *talsh_task);
int talshTensorSlice(talsh_tens_t *dtens, talsh_tens_t *ltens, const int *offsets,
                     int dev_id TALSH_DEFAULT(DEV_DEFAULT), int dev_kind TALSH_DEFAULT(DEV_DEFAULT),
                     int copy_ctrl TALSH_DEFAULT(COPY_MT), int accumulative TALSH_DEFAULT(NOPE),
                     talsh_task_t *talsh_task TALSH_DEFAULT(NULL));
int talshTensorSlice_(talsh_tens_t *dtens, talsh_tens_t *ltens, const int *offsets, int dev_id,
                      int dev_kind, int copy_ctrl, int accumulative, talsh_task_t *talsh_task);
int talshTensorInsert(talsh_tens_t *dtens, talsh_tens_t *ltens, const int *offsets,
                      int dev_id TALSH_DEFAULT(DEV_DEFAULT), int dev_kind TALSH_DEFAULT(DEV_DEFAULT),
                      int copy_ctrl TALSH_DEFAULT(COPY_MT), int accumulative TALSH_DEFAULT(NOPE),
                      talsh_task_t *talsh_task TALSH_DEFAULT(NULL));
int talshTensorInsert_(talsh_tens_t *dtens, talsh_tens_t *ltens, const int *offsets, int dev_id,
                       int dev_kind, int copy_ctrl, int accumulative, talsh_task_t *talsh_task);
int talshTensorCopy(const char *cptrn, talsh_tens_t *dtens, talsh_tens_t *ltens,
                    int dev_id TALSH_DEFAULT(DEV_DEFAULT), int dev_kind TALSH_DEFAULT(DEV_DEFAULT),
                    int copy_ctrl TALSH_DEFAULT(COPY_MT),
                    talsh_task_t *talsh_task TALSH_DEFAULT(NULL));
int talshTensorCopy_(const char *cptrn, talsh_tens_t *dtens, talsh_tens_t *ltens, int dev_id,
                     int dev_kind, int copy_ctrl, talsh_task_t *talsh_task);
int talshTensorAdd(const char *cptrn, talsh_tens_t *dtens, talsh_tens_t *ltens,
                   double scale_real TALSH_DEFAULT(1.0), double scale_imag TALSH_DEFAULT(0.0),
                   int dev_id TALSH_DEFAULT(DEV_DEFAULT), int dev_kind TALSH_DEFAULT(DEV_DEFAULT),
                   int copy_ctrl TALSH_DEFAULT(COPY_MT),
                   talsh_task_t *talsh_task TALSH_DEFAULT(NULL));
int talshTensorAdd_(const char *cptrn, talsh_tens_t *dtens, talsh_tens_t *ltens,
                    double scale_real, double scale_imag, int dev_id, int dev_kind,
                    int copy_ctrl, talsh_task_t *talsh_task);
int talshTensorContract(const char *cptrn, talsh_tens_t *dtens, talsh_tens_t *ltens,
                        talsh_tens_t *rtens, double scale_real TALSH_DEFAULT(1.0),
                        double scale_imag TALSH_DEFAULT(0.0),
                        int dev_id TALSH_DEFAULT(DEV_DEFAULT),
                        int dev_kind TALSH_DEFAULT(DEV_DEFAULT),
                        int copy_ctrl TALSH_DEFAULT(COPY_MTT),
                        int accumulative TALSH_DEFAULT(YEP),
                        talsh_task_t *talsh_task TALSH_DEFAULT(NULL));
int talshTensorContract_(const char *cptrn, talsh_tens_t *dtens, talsh_tens_t *ltens,
                         talsh_tens_t *rtens, double scale_real, double scale_imag, int dev_id,
                         int dev_kind, int copy_ctrl, int accumulative, talsh_task_t *talsh_task);
int talshTensorContractXL(const char *cptrn, talsh_tens_t *dtens, talsh_tens_t *ltens,
                          talsh_tens_t *rtens, double scale_real TALSH_DEFAULT(1.0),
                          double scale_imag TALSH_DEFAULT(0.0),
                          int dev_id TALSH_DEFAULT(DEV_DEFAULT),
                          int dev_kind TALSH_DEFAULT(DEV_DEFAULT),
                          int accumulative TALSH_DEFAULT(YEP));
int talshTensorContractXL_(const char *cptrn, talsh_tens_t *dtens, talsh_tens_t *ltens,
                           talsh_tens_t *rtens, double scale_real, double scale_imag, int dev_id,
                           int dev_kind, int accumulative);
int talshTensorDecomposeSVD(const char *cptrn, talsh_tens_t *dtens, talsh_tens_t *ltens,
                            talsh_tens_t *rtens, talsh_tens_t *stens,
                            const char absorb TALSH_DEFAULT('N'),
                            int dev_id TALSH_DEFAULT(DEV_DEFAULT),
                            int dev_kind TALSH_DEFAULT(DEV_DEFAULT));
int talshTensorDecomposeSVDL(const char *cptrn, talsh_tens_t *dtens, talsh_tens_t *ltens,
                             talsh_tens_t *rtens, int dev_id TALSH_DEFAULT(DEV_DEFAULT),
                             int dev_kind TALSH_DEFAULT(DEV_DEFAULT));
int talshTensorDecomposeSVDR(const char *cptrn, talsh_tens_t *dtens, talsh_tens_t *ltens,
                             talsh_tens_t *rtens, int dev_id TALSH_DEFAULT(DEV_DEFAULT),
                             int dev_kind TALSH_DEFAULT(DEV_DEFAULT));
int talshTensorDecomposeSVDLR(const char *cptrn, talsh_tens_t *dtens, talsh_tens_t *ltens,
                              talsh_tens_t *rtens, int dev_id TALSH_DEFAULT(DEV_DEFAULT),
                              int dev_kind TALSH_DEFAULT(DEV_DEFAULT));
int talshTensorOrthogonalizeSVD(const char *cptrn, talsh_tens_t *dtens,
                                int dev_id TALSH_DEFAULT(DEV_DEFAULT),
                                int dev_kind TALSH_DEFAULT(DEV_DEFAULT));
int talshTensorOrthogonalizeMGS(talsh_tens_t *dtens, int num_iso_dims, int *iso_dims,
                                int dev_id TALSH_DEFAULT(DEV_DEFAULT),
                                int dev_kind TALSH_DEFAULT(DEV_DEFAULT));

/* 1-norm (sum of moduli) of the tensor's Host image; -1.0 on failure. */
double talshTensorImageNorm1_cpu(const talsh_tens_t *talsh_tens);

/* Extension of this core (no counterpart in the reference C API, which only
 * has the Host-image norm above): 1-norm computed on a GPU by a deterministic
 * two-pass reduction, accumulated in double for every data kind.  Blocking.
 * Returns -1.0 on failure, like talshTensorImageNorm1_cpu. */
double talshTensorNorm1(talsh_tens_t *tens, int dev_id TALSH_DEFAULT(DEV_DEFAULT),
                        int dev_kind TALSH_DEFAULT(DEV_DEFAULT));
double talshTensorNorm1_(talsh_tens_t *tens, int dev_id, int dev_kind);

/* Entry points of the reference's C side that its Fortran module (talshf.F90:528-547)
 * binds.  Body image information (reference talshc.cpp:245-267): TALSH_NOT_ALLOWED
 * when the image is no longer available; *buf_entry is -1 for bodies the library
 * allocates (no carved buffer here), the caller's value for external memory. */
int talsh_tensor_image_info(const talsh_tens_t *talsh_tens, int image_id, int *dev_id, int *data_kind,
                            void **gmem_p, int *buf_entry);
/* GPU count (reference tensor_algebra_gpu_nvidia.cu:2728-2739): 0, or 1 with
 * *dev_count = -1 when the CUDA runtime cannot tell. */
int gpu_get_device_count(int *dev_count);

/* Extension of this core (no counterpart in the reference): the form R8 and
 * C8 contractions of talshTensorContract run in.  0 (default) = plain FP64,
 * the drop-in behaviour; 2..7 = split precision on the tensor cores with that
 * many int8 slices (see tcTensorContractSplit in talsh_b200.h; 6 keeps the
 * relative error below 1e-10; C8 runs as one real contraction of twice the
 * extents).  Also set by the environment variable TALSH_B200_R8_SLICES at
 * talshInit.  Contractions the split form cannot take (hyper-indices, rank-0
 * operands, R8 with conjugation flags) run plain, and talshTensorContractXL
 * uses the split form for R8 only.  Returns TALSH_INVALID_ARGS for other values. */
int talshContractSlicesSet(int slices);
int talshContractSlicesGet(void);
/* Extension of this core (no counterpart in the reference): the split form and
 * slice count talshTensorContract uses for R8/C8 (the forms TC_SPLIT_INT8,
 * TC_SPLIT_BF16, TC_SPLIT_TF32, TC_SPLIT_FP8 of tcTensorContractSplitForm in
 * talsh_b200.h; slices 0 = the form's default, else 2..7).
 * talshContractSlicesSet(0) returns to plain FP64.  TALSH_INVALID_ARGS for
 * other values. */
int talshContractSplitFormSet(int form, int slices);
int talshContractSplitFormGet(int *form, int *slices);
#ifdef __cplusplus
}
#endif

#endif /* TALSH_B200_TALSH_H_ */
