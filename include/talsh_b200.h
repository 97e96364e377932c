/* talsh-b200: device-level C ABI of the sm_100a kernels.
 *
 * These entry points sit below the TAL-SH API (talsh.h).  They take device
 * pointers and a CUDA stream (cudaStream_t passed as void*, NULL = legacy
 * default stream), launch asynchronously and return 0 on success or a TAL-SH
 * error code.  They replace the NV-TAL internal interface
 * (`gpu_tensor_block_{copy,add,contract_dlf,init,scale}`,
 * reference device_algebra.h:259-274); only talsh.h is a compatibility
 * promise, this layer is specific to this core.
 *
 * Conventions: column-major bodies (dimension 0 fastest); permutations are
 * 1-based O2N arrays (o2n[i] = output position of input dimension i, as in
 * the reference's `transp(1:n)` of tensor_block_copy); data kinds R4, R8, C4,
 * C8 from tensor_algebra.h.  Scale factors follow the reference CPU rules
 * (real kinds use cmplx8_to_real8(alpha) for add/scale, real(alpha) for
 * contraction).
 */
#ifndef TALSH_B200_CORE_H_
#define TALSH_B200_CORE_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* dst = permute(src): dst[O2N(idx)] = src[idx]; conj != 0 negates imaginary
 * parts (C4/C8).  Pure data movement, bit-exact.
 * Replaces gpu_tensor_block_copy (reference tensor_algebra_gpu_nvidia.cu:4806). */
int tcTensorPermute(int data_kind, int rank, const int *dims_in, const int *o2n, const void *src,
                    void *dst, int conj, void *stream);

/* dst += permute(src) * alpha, evaluated per element as d + l*s without FMA
 * contraction (bit-exact with the reference CPU add).  conj applies to src.
 * Replaces gpu_tensor_block_add (reference tensor_algebra_gpu_nvidia.cu:5203). */
int tcTensorPermuteAdd(int data_kind, int rank, const int *dims_in, const int *o2n,
                       const void *src, void *dst, double alpha_re, double alpha_im, int conj,
                       void *stream);

/* Transpose autotuner.  Cases fall in classes by data kind, operation (copy,
 * or add when accumulate != 0), the rank and permutation after fusing the
 * dimensions that stay adjacent, the volume bucket (floor log2), the log2
 * buckets of the input- and output-minor extents and whether those extents
 * fill whole 16-byte units.  tcTensorPermuteTune runs this case with each
 * candidate plan choice, choice = b + 3 s + 6 f + 12 g + 36 r (b: 0 the
 * planner's read path, 1 bulk reads forced on, 2 off; s = 1: tiles of at most 4
 * elements per thread; f = 1: the other tile walk order; g: 0 the planner's
 * tile growth (the shorter run first), 1 input runs first, 2 output runs
 * first; r = 1 / 2: initial runs of 2 / 4 times the planner's minimum length;
 * add 108 to keep the full tile budget for small tensors, which the planner
 * otherwise shrinks so that every SM gets tiles; 0 is the planner's
 * heuristics throughout), 1 + reps times each on `stream` (the first run is a warm-up),
 * times them with CUDA events, and records the fastest for the class; every
 * later tcTensorPermute / tcTensorPermuteAdd call of the class (and the tiled
 * tasks of a permutation batch) uses it.  Results are identical under every
 * choice; only the speed changes.  src and dst are device buffers of the case's
 * volume; dst is overwritten (adds accumulate into it 216 x (1 + reps) times
 * at most).  *choice receives the recorded choice (0 when the case has a single
 * plan).  Synchronises the stream.  The reference has no autotuner: its
 * gpu_tensor_block_copy_dlf (tensor_algebra_gpu_nvidia.cu:4806) picks a kernel
 * by fixed rules. */
int tcTensorPermuteTune(int data_kind, int rank, const int *dims_in, const int *o2n, int accumulate,
                        const void *src, void *dst, void *stream, int reps, int *choice);
/* The recorded choice of the case's class, or -1 in *choice when none. */
int tcTensorPermuteTuned(int data_kind, int rank, const int *dims_in, const int *o2n, int accumulate,
                         int *choice);
/* Records `choice` (0-215) for the case's class without timing -- a saved tuning
 * table can be restored this way -- or forgets the class's entry (choice -1).
 * TALSH_INVALID_ARGS when the choice has no plan for this case. */
int tcTensorPermuteTuneSet(int data_kind, int rank, const int *dims_in, const int *o2n, int accumulate,
                           int choice);
/* Forgets every recorded choice (the heuristics apply again). */
void tcTensorPermuteTuneReset(void);

/* dst[0..vol) = value.  Replaces gpu_tensor_block_init (:4467). */
int tcTensorInit(int data_kind, size_t vol, void *dst, double val_re, double val_im, void *stream);

/* dst[0..vol) *= alpha.  Replaces gpu_tensor_block_scale (:4525). */
int tcTensorScale(int data_kind, size_t vol, void *dst, double alpha_re, double alpha_im,
                  void *stream);

/* Bytes of device scratch tcTensorNorm1 needs for a tensor of vol elements. */
size_t tcTensorNorm1Scratch(size_t vol);

/* *result_dev (device double) = sum of |x| over src[0..vol), accumulated in
 * double with a fixed two-pass reduction (run-to-run deterministic).
 * scratch: device buffer of at least tcTensorNorm1Scratch(vol) bytes.
 * No reference GPU counterpart: the reference norm is host-only
 * (talshTensorImageNorm1_cpu, talshc.cpp:6207). */
int tcTensorNorm1(int data_kind, size_t vol, const void *src, double *result_dev, void *scratch,
                  size_t scratch_bytes, void *stream);

/* Bytes of device scratch tcTensorContract needs for this shape (offset
 * tables of the gather-GEMM, plus the partial sums of a full contraction). */
size_t tcTensorContractScratch(int data_kind, const int *cptrn, int drank, const int *ddims,
                               int lrank, const int *ldims, int rrank, const int *rdims);

/* D = beta*D + alpha * contraction(L, R) for a digital pattern cptrn[lrank+rrank]
 * (reference format: >0 position in D, <0 minus the position in the other
 * operand).  Indices present in D, L and R at once (hyper-indices) run as one
 * GEMM per combination of their values, all in the same launch.  beta = 1 if
 * accumulative else D is overwritten.
 * conj_bits: bit0 D, bit1 L, bit2 R (complex kinds only).  Rank-0 operands are
 * single elements of the data kind, resident in device memory.  scratch:
 * device buffer of tcTensorContractScratch(...) bytes (may be NULL when that is 0).
 * Replaces gpu_tensor_block_contract_dlf (reference :5847). */
int tcTensorContract(int data_kind, const int *cptrn, int drank, const int *ddims, int lrank,
                     const int *ldims, int rrank, const int *rdims, void *D, const void *L,
                     const void *R, double alpha_re, double alpha_im, int conj_bits,
                     int accumulative, void *scratch, size_t scratch_bytes, void *stream);

/* Bytes of device scratch tcTensorContractSplit needs (0 when the form does
 * not apply: not R8 or C8, an operand of rank 0, hyper-indices, or an invalid
 * pattern). */
size_t tcTensorContractSplitScratch(int data_kind, const int *cptrn, int drank, const int *ddims,
                                    int lrank, const int *ldims, int rrank, const int *rdims,
                                    int slices);

/* Split-precision R8 contraction on the tensor cores (tcgen05 kind::i8): the
 * operands are permuted to matrices, cut into `slices` int8 slices of 7 bits
 * per row with power-of-two row scales, all slice pairs (s, t) with
 * s + t <= slices + 1 are multiplied exactly in int32 and recombined in FP64
 * (the Ozaki scheme).  Same pattern, alpha/accumulative and D layout rules as
 * tcTensorContract; slices 2..7, 0 = 6 (relative error about sqrt(K)*2^-46 on
 * random data, below 1e-10 for contracted volumes up to ~10^8).  Indices
 * present in D, L and R at once return TALSH_NOT_IMPLEMENTED.  Inputs must be
 * finite.  C8: conj_bits and a complex alpha as in tcTensorContract; the
 * contraction runs as one real contraction (L and D read as real tensors with
 * a leading (re, im) index, R's conjugated and i-rotated copies, alpha folded
 * in, stacked in the scratch), so the error bound is that of the real form with
 * twice the contracted extent.  A split-precision form of
 * gpu_tensor_block_contract_dlf (reference :5847); no reference counterpart. */
int tcTensorContractSplit(int data_kind, const int *cptrn, int drank, const int *ddims, int lrank,
                          const int *ldims, int rrank, const int *rdims, void *D, const void *L,
                          const void *R, double alpha_re, double alpha_im, int conj_bits,
                          int accumulative, int slices, void *scratch, size_t scratch_bytes,
                          void *stream);

/* Split forms of the tensor-core contraction (tcTensorContractSplitForm). */
#define TC_SPLIT_INT8 0 /* int8 digits, exact int32 sums (tcTensorContractSplit) */
#define TC_SPLIT_BF16 1 /* bf16 slices, fp32 sums per diagonal (kind::f16) */
#define TC_SPLIT_TF32 2 /* tf32 slices, fp32 sums per diagonal (kind::tf32) */
#define TC_SPLIT_FP8 3  /* e4m3 slices with per-row power-of-two scales (kind::f8f6f4) */

/* Bytes of device scratch tcTensorContractSplitForm needs (0 when the form
 * does not apply, as for tcTensorContractSplitScratch, or for an invalid form
 * or slice count). */
size_t tcTensorContractSplitFormScratch(int data_kind, const int *cptrn, int drank, const int *ddims,
                                        int lrank, const int *ldims, int rrank, const int *rdims,
                                        int form, int slices);

/* tcTensorContractSplit in a chosen form: TC_SPLIT_INT8 is that function;
 * the floating-point forms cut each row-scaled operand into `slices` slices of
 * bf16 (8 significant bits each), tf32 (11) or e4m3 (4), y_s = round(r_s 2^(b s)),
 * r_{s+1} = r_s - y_s 2^(-b s) (exact in FP64), multiply the slice pairs
 * s + t <= slices - 1 on the tensor cores with one fp32 accumulator per
 * diagonal s + t in tensor memory (each product exact in fp32, the sums
 * rounded to fp32) and recombine the diagonals in FP64 into D.  slices: 0 =
 * the form's default (6 for int8, 3 otherwise), else 2..7.  The error is
 * dominated by the fp32 sums for bf16 and tf32 (they grow with the number of
 * tensor-core K steps: about 1e-6 relative at a contracted volume of 1024,
 * 1e-5 to 1e-4 at 10^4 to 4x10^4) and by the dropped pairs, about
 * 2^(-4 slices), for e4m3; callers state it per result.  The BF16x3 / TF32x3 / FP8 forms of a
 * split-precision gpu_tensor_block_contract_dlf (reference :5847); no
 * reference counterpart. */
int tcTensorContractSplitForm(int data_kind, const int *cptrn, int drank, const int *ddims, int lrank,
                              const int *ldims, int rrank, const int *rdims, void *D, const void *L,
                              const void *R, double alpha_re, double alpha_im, int conj_bits,
                              int accumulative, int form, int slices, void *scratch, size_t scratch_bytes,
                              void *stream);

/* Slicing: slice (+)= full[offsets : offsets + slice_dims] (0-based offsets, both
 * tensors dense column-major of the same rank and kind).  Replaces
 * gpu_tensor_block_slice (tensor_algebra_gpu_nvidia.cu:4788, a stub there) with
 * the semantics of the CPU path tensor_block_slice_dlf_* (tensor_algebra_cpu.F90:6900);
 * accumulative = 0 overwrites the slice. */
int tcTensorSlice(int data_kind, int rank, const int *full_dims, const int *slice_dims, const int *offsets,
                  const void *full, void *slice, int accumulative, void *stream);
/* Insertion: full[offsets : offsets + slice_dims] (+)= slice.  Replaces
 * gpu_tensor_block_insert (tensor_algebra_gpu_nvidia.cu:4798, a stub there);
 * semantics of tensor_block_insert_dlf_* (tensor_algebra_cpu.F90:7216). */
int tcTensorInsert(int data_kind, int rank, const int *full_dims, const int *slice_dims, const int *offsets,
                   const void *slice, void *full, int accumulative, void *stream);

#define TC_BATCH_MAX_RANK 8

/* Batched transposes: many independent transposes / transpose-adds recorded
 * once into a CUDA graph whose `branches` (1..32) run concurrently, then
 * replayed with one launch per tcPermuteBatchLaunch.  Each task keeps the tile
 * plan a single tcTensorPermute(Add) call would use.  The graph holds the
 * tasks' pointers: replays read and write the same buffers.  Tasks must not
 * write overlapping destinations.  No reference counterpart (the reference
 * issues one gpu_tensor_block_copy / _add per call). */
typedef struct {
  int data_kind, rank;
  int dims[TC_BATCH_MAX_RANK];        /* input extents */
  int o2n[TC_BATCH_MAX_RANK];         /* 1-based output position of each input index */
  const void *src;
  void *dst;
  int add;                            /* 0: dst = permute(src); 1: dst += alpha * permute(src) */
  double alpha_re, alpha_im;
  int conj;                           /* complex kinds: conjugate the source */
} tcPermuteTask;
typedef struct tcPermuteBatch tcPermuteBatch;
int tcPermuteBatchCreate(int ntasks, const tcPermuteTask *tasks, int branches, tcPermuteBatch **batch);
int tcPermuteBatchLaunch(tcPermuteBatch *batch, void *stream);
int tcPermuteBatchDestroy(tcPermuteBatch *batch);

/* Batched contractions (many small tasks, one launch per tile configuration). */
typedef struct {
  int data_kind;                      /* R4, R8, C4, C8 */
  int drank, lrank, rrank;            /* each at most TC_BATCH_MAX_RANK */
  int cptrn[2 * TC_BATCH_MAX_RANK];   /* digital pattern, lrank + rrank entries */
  int ddims[TC_BATCH_MAX_RANK], ldims[TC_BATCH_MAX_RANK], rdims[TC_BATCH_MAX_RANK];
  void *D;                            /* device pointers */
  const void *L, *R;
  double alpha_re, alpha_im;
  int conj_bits, accumulative;
} tcContractTask;

/* Bytes of device scratch tcTensorContractBatch needs for these tasks (0 when
 * a task is invalid). */
size_t tcTensorContractBatchScratch(int ntasks, const tcContractTask *tasks);

/* Runs every task with tcTensorContract's semantics.  The tasks' offset
 * tables are built by one launch and the GEMM tiles of all tasks run in one
 * persistent launch per tile configuration (FP64 tensor-pipe 64x64 or 32x32
 * tiles for R8 and C8, SIMT for R4/C4), each CTA finding its task from a tile
 * prefix sum (a full
 * contraction is a 1 x 1 tile: its sum order differs from tcTensorContract's
 * two-pass dot product); scalar operands and hyper-indices take the
 * single-task path.
 * Tasks must not write overlapping D regions (they run concurrently).  A
 * batched form of gpu_tensor_block_contract_dlf; no reference
 * counterpart (the reference schedules one task per call). */
int tcTensorContractBatch(int ntasks, const tcContractTask *tasks, void *scratch, size_t scratch_bytes,
                          void *stream);

/* A batch recorded once and replayed: tcContractBatchGraphCreate plans the
 * tasks, uploads their descriptors into `scratch` (at least
 * tcTensorContractBatchScratch bytes, owned by the caller and kept for the
 * graph's life), builds their offset tables (synchronously on `stream`) and
 * captures the GEMM work in one CUDA graph: the persistent kernels of the tile
 * configurations (and the single-task fallbacks) run as concurrent branches.
 * tcContractBatchGraphLaunch replays it on a stream -- the same tasks on the
 * same operand buffers, whose contents may change between replays.  Results
 * equal tcTensorContractBatch's bit for bit.  No reference counterpart. */
typedef struct tcContractBatchGraph tcContractBatchGraph;
int tcContractBatchGraphCreate(int ntasks, const tcContractTask *tasks, void *scratch, size_t scratch_bytes,
                               void *stream, tcContractBatchGraph **graph);
int tcContractBatchGraphLaunch(tcContractBatchGraph *graph, void *stream);
int tcContractBatchGraphDestroy(tcContractBatchGraph *graph);

/* ---------------------------------------------------------------- serving
 * A contraction server on the current GPU: tasks arrive one by one
 * (tcServerSubmit), wait for admission under a device-memory budget, and run
 * as soon as their inputs are ready.  Small tasks are gathered into
 * continuous batches (one tcTensorContractBatch-style launch set per batch,
 * a new batch whenever a batch slot is free); tasks at or above a flop
 * threshold run alone on a second stream, R8 ones in split precision when
 * r8_slices > 0.  A task may take an operand from an earlier task's output
 * (l_from / r_from), which the server allocates and keeps on the device
 * until its declared consumers have completed.  Results do not depend on what
 * else is in flight: every tile is computed by the same code in the same order
 * whichever batch carries it.  Single scheduling thread (as the reference's
 * task scheduler, tensor_algebra_gpu_nvidia.cu:205).  The reference has no
 * serving layer; its per-call scheduling is talshTensorContract +
 * talshTaskComplete (talshc.cpp:5073, :2336-2561). */
typedef struct tcServer tcServer;
typedef struct {
  size_t budget_bytes;  /* device bytes for server-held outputs and scratch (0: 90% of free memory);
                           the server's memory pool keeps up to this much mapped between tasks */
  int r8_slices;        /* 0: plain FP64 for large R8 tasks, 2..7: split precision with that many slices */
  int max_batch;        /* tasks per batch launch (0: 4096) */
  int max_inflight;     /* batches in flight at once (0: 2) */
  double large_flop;    /* tasks with at least this many flops run alone (0: 1e10) */
  size_t prealloc_bytes;/* device memory mapped into the server's pool at creation, so that
                           admissions up to that much never map pages on the scheduling thread */
} tcServeConfig;
typedef struct {
  tcContractTask op;    /* op.D == NULL: the server allocates the output and overwrites it */
  uint64_t l_from;      /* nonzero: L is the output of that earlier submission (op.L ignored) */
  uint64_t r_from;      /* nonzero: R is the output of that earlier submission (op.R ignored) */
  int consumers;        /* later submissions that will read this task's output */
  int keep_output;      /* 1: a server-allocated output stays until tcServerRelease */
} tcServeTask;
typedef struct {
  unsigned long long submitted, completed, failed, batches, batched_tasks, large_tasks, admission_waits;
  size_t bytes_in_use, bytes_peak, budget_bytes;
  double sched_s;       /* host seconds spent in scheduling steps */
  double max_step_s;    /* longest single scheduling step */
} tcServeStats;

int tcServerCreate(const tcServeConfig *cfg, tcServer **srv);
int tcServerDestroy(tcServer *srv);  /* waits for work in flight, frees everything */
/* Queues one task; *id (nonzero) names it from then on. */
int tcServerSubmit(tcServer *srv, const tcServeTask *task, uint64_t *id);
/* One scheduling step: retires finished batches, admits queued tasks,
 * launches ready ones.  Returns the number of tasks not yet completed. */
int tcServerProgress(tcServer *srv);
/* Pops up to max completed tasks: ids, submit-to-completion seconds, status
 * (TALSH_SUCCESS or an error code).  Returns how many were written. */
int tcServerPoll(tcServer *srv, int max, uint64_t *ids, double *latency_s, int *status);
/* Runs tcServerProgress until every submitted task has completed. */
int tcServerDrain(tcServer *srv);
/* Device address of a completed task's server-held output. */
int tcServerOutput(tcServer *srv, uint64_t id, void **ptr);
/* Gives up a kept output (freed once its consumers have completed). */
int tcServerRelease(tcServer *srv, uint64_t id);
int tcServerGetStats(tcServer *srv, tcServeStats *stats);
/* Zeroes the counters; the peak restarts from the bytes in use. */
int tcServerResetStats(tcServer *srv);
/* Replays n tasks arriving at arrival_s[i] seconds after the call (ascending):
 * submits each on time, runs the scheduling loop in between, returns when all
 * have completed.  l_from / r_from in these tasks are 1-based indices into the
 * array.  ids[i] and latency_s[i] (either may be NULL) receive each task's id
 * and submit-to-completion time.  Returns TALSH_SUCCESS or the first error. */
int tcServerReplay(tcServer *srv, int n, const tcServeTask *tasks, const double *arrival_s, uint64_t *ids,
                   double *latency_s);

/* Autotuner of the batched form: tasks fall in classes by kind (R8, C8) and
 * the buckets of their GEMM sizes M and N (< 16, < 48, < 128, >= 128).  For
 * each class present among `tasks`, runs that class's tasks as one batch with
 * 32x32 and with 64x64 tiles (`reps` timed runs each after one warm-up, CUDA
 * events on `stream`) and keeps the faster tile for the class; later batches
 * (tcTensorContractBatch, the contraction server) use it, so query
 * tcTensorContractBatchScratch again afterwards (the scratch size depends on
 * the tiles).  The tasks are executed several times, so their D contents are
 * unspecified afterwards.
 * scratch: at least tcTensorContractBatchScratch(ntasks, tasks) bytes.  Not to
 * run concurrently with other batch launches. */
int tcTensorContractBatchTune(int ntasks, const tcContractTask *tasks, void *scratch, size_t scratch_bytes,
                              void *stream, int reps);
/* Tile edge chosen for a class (0: not tuned, the shape rule applies; -1: bad class). */
int tcTensorContractBatchTuned(int data_kind, int m_bucket, int n_bucket);
/* Forgets every tuned choice. */
void tcTensorContractBatchTuneReset(void);

/* Size of the fixed scratch array behind tcTensorContractNoAlloc: 8 MiB per GPU. */
#define TC_CONTRACT_NOALLOC_SCRATCH_BYTES ((size_t)8 << 20)

/* tcTensorContract without caller scratch and without any allocation, for
 * callers that cannot allocate device memory (code running inside an
 * allocator or memory-pool callback, a host whose device budget belongs to
 * another runtime, a loop where the implicit synchronisation of cudaMalloc is
 * not allowed).  Same arguments and results as tcTensorContract minus the
 * scratch pair.  Its scratch is one array of TC_CONTRACT_NOALLOC_SCRATCH_BYTES
 * compiled into the library, held on every GPU that loads the library until
 * exit.  Shapes whose tcTensorContractScratch(...) exceeds that size are
 * rejected with TALSH_LIMIT_EXCEEDED (tcLastErrorString says why).  The first
 * call on a device looks up the array's device address, so make that first
 * call before any stream capture; the address is kept for the life of the
 * process, so a device reset (cudaDeviceReset) after that first call is not
 * supported.  All calls share the one array: calls that
 * may overlap on the GPU (other streams, other host threads) race and must be
 * serialised by the caller.  No counterpart in the reference. */
int tcTensorContractNoAlloc(int data_kind, const int *cptrn, int drank, const int *ddims,
                            int lrank, const int *ldims, int rrank, const int *rdims, void *D,
                            const void *L, const void *R, double alpha_re, double alpha_im,
                            int conj_bits, int accumulative, void *stream);
/* TC_CONTRACT_NOALLOC_SCRATCH_BYTES as compiled into the loaded library. */
size_t tcTensorContractNoAllocMaxScratch(void);

/* Host view of the transpose tile plan (diagnostics): info[0] fused rank,
 * [1] identity flag, [2] tile volume, [3] input run, [4] output run,
 * [5] input runs, [6] output runs, [7] input vector width, [8] output vector
 * width, [9] shared bytes, [10] tile count, [11] per-element tables in use. */
int tcPermutePlanInfo(int data_kind, int rank, const int *dims_in, const int *o2n, int *info);

/* Sub-contractions the last talshTensorContractXL call ran (diagnostics). */
size_t tcContractXLLastOps(void);
/* The sub-contractions talshTensorContractXL forms for this shape when
 * budget_bytes of device memory are free (host-side planning only, no GPU
 * needed): the contraction is halved with the choice rule of the reference's
 * talshTensorOpDecompose2 (talshc.cpp:3150-3294) until the D, L and R blocks of
 * every piece take at most a quarter of the budget.  Writes, per piece, the
 * block offsets and extents of D, L and R in that order (drank + lrank + rrank
 * ints each; either array may be NULL) for up to max_ops pieces and returns the
 * number of pieces, TALSH_LIMIT_EXCEEDED if there would be more than max_ops,
 * or TALSH_INVALID_ARGS. */
int tcContractXLPlan(int data_kind, const int *cptrn, int drank, const int *ddims, int lrank, const int *ldims,
                     int rrank, const int *rdims, size_t budget_bytes, int max_ops, int *offsets, int *extents);
/* Number of CTAs on the current GPU that gave up one of the split-precision
 * GEMM's bounded waits since the library was loaded, or -1 when it cannot be
 * read (reference gpu_get_error_count, device_algebra.h:200).  A CTA that gives
 * up waits (bounded) for its own copies in flight, frees its tensor memory and
 * returns; the context stays usable.  talshTensorContract tasks in split
 * precision that see the count rise finish with TALSH_TASK_ERROR. */
int gpu_get_error_count(void);
/* Test hook for the failure path above: while enabled, split-precision GEMM
 * launches issue no operand copies and give up their first wait after 4096
 * polls.  Off by default. */
int tcTestSplitStall(int enable);
/* Number of kernels this library launched since load (diagnostics). */
unsigned long long tcKernelLaunchCount(void);
/* Last CUDA error text seen by the library (diagnostics). */
const char *tcLastErrorString(void);

#ifdef __cplusplus
}
#endif

#endif /* TALSH_B200_CORE_H_ */
