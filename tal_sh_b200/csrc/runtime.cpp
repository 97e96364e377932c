// The TAL-SH runtime of talsh-b200: implements talsh.h on top of the sm_100a
// kernels (talsh_b200.h).
//
// Behaviour follows the reference runtime talshc.cpp (talshInit :546,
// talshTensorConstruct :1167, talshTaskFinalize :2064, talshTaskStatus :2336,
// talshTensorPlace :3318, talshTensorCopy :4530, talshTensorAdd :4795,
// talshTensorContract :5073): tensors own up to TALSH_MAX_DEV_PRESENT body
// images, every operation picks a source image per argument, stages images
// that live elsewhere onto the executing GPU, and applies the two-bit
// coherence code of each argument when its task completes (D discard, M move,
// T temporary, K keep).
//
// B200-specific design:
//  * one in-order compute stream per GPU carries every task's kernels, so
//    device-side dependencies between asynchronous tasks need no tracking;
//    staging copies in and copies back out run on two more streams, chained
//    to the compute stream by the task's events, so consecutive tasks overlap
//    their transfers; Host ranges still being copied back are tracked and
//    waited for before they are staged again;
//  * each task records four events (start, inputs ready, compute done,
//    finished) that give the TAL-SH task status ladder and timings;
//  * device memory comes from the stream-ordered CUDA allocator with a byte
//    budget per GPU (90% of free memory at init by default, environment
//    variable TALSH_B200_GPU_BUDGET_BYTES overrides it); exceeding the budget
//    returns TRY_LATER and the operation leaves no trace;
//  * Host bodies allocated by the library are pinned, so staging copies are
//    asynchronous DMA transfers.
// There is no CPU compute path: operations requested on DEV_HOST return
// TALSH_NOT_AVAILABLE.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "common.h"

namespace tb {
int norm1_launch(int data_kind, size_t vol, const void *src, double *result_dev, double *partial,
                 cudaStream_t st);
size_t contract_scratch_bytes(int kind, const int *cptrn, int drank, const int *ddims, int lrank,
                              const int *ldims, int rrank, const int *rdims);
size_t contract_split_scratch(int kind, const int *cptrn, int drank, const int *ddims, int lrank,
                              const int *ldims, int rrank, const int *rdims, int slices);
int contract_split_launch(int kind, const int *cptrn, int drank, const int *ddims, int lrank,
                          const int *ldims, int rrank, const int *rdims, void *D, const void *L,
                          const void *R, double alpha_re, int accumulative, int slices, void *scratch,
                          size_t scratch_bytes, void *stream);
int contract_launch(int kind, const int *cptrn, int drank, const int *ddims, int lrank,
                    const int *ldims, int rrank, const int *rdims, void *D, const void *L,
                    const void *R, double alpha_re, double alpha_im, int conj_bits,
                    int accumulative, void *scratch, size_t scratch_bytes, void *stream);

namespace {

constexpr unsigned kTwoBits = 3u;

struct AllocRec {
  int gpu;       // -1: host
  size_t bytes;
  bool pinned;   // host only
};

// A copy back into memory outside the executing GPU (a Host image, or another
// GPU's) still in flight: later reads of an overlapping range wait for it.
struct PendingWrite {
  const char *p;
  size_t n;
  cudaEvent_t ev;
};

struct GpuCtx {
  bool in_use = false;
  cudaStream_t stream = nullptr;  // compute (and all work of operations without staging)
  cudaStream_t h2d = nullptr;     // staging copies into the GPU (even tasks)
  cudaStream_t h2d_b = nullptr;   // staging copies of odd tasks: one task's wait for a copy back
                                  // does not hold up the next task's uploads
  unsigned staged = 0;            // tasks staged so far (picks the staging stream)
  cudaStream_t d2h = nullptr;     // copies back out of the GPU
  std::vector<PendingWrite> pending;
  size_t budget = 0, used = 0, peak = 0;
  double flops = 0.0, bytes = 0.0;
  unsigned long long tasks_ok = 0, tasks_failed = 0, try_later = 0;
  std::vector<cudaEvent_t> event_pool;
  int device_errors = 0;  // gpu_get_error_count() as last seen
};

struct Runtime {
  bool on = false;
  GpuCtx gpu[MAX_GPUS_PER_NODE];
  std::unordered_map<void *, AllocRec> allocs;
  bool log_ops = false;
  size_t host_bytes = 0;
  int mem_policy = MEM_ALLOC_TMP_BUF, mem_fallback = 1;
};
Runtime R;
std::recursive_mutex g_mu;
// R8 contraction form: 0 = plain FP64 (the drop-in default), 2..7 = split
// precision with that many int8 slices (TALSH_B200_R8_SLICES or
// talshContractSlicesSet).
std::atomic<int> g_r8_slices{0};
// Sub-contractions of the last talshTensorContractXL call (diagnostics).
size_t g_xl_last_ops = 0;
constexpr size_t kXLMaxOps = 1 << 16;  // cap on the sub-contractions of one call

int node_gpu_count() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

// ---------------------------------------------------------------- memory
void *host_alloc(size_t bytes, bool try_pinned) {
  void *p = nullptr;
  bool pinned = false;
  if (try_pinned && cudaHostAlloc(&p, bytes, cudaHostAllocPortable) == cudaSuccess) {
    pinned = true;
  } else {
    cudaGetLastError();
    p = std::malloc(bytes);
  }
  if (p) {
    R.allocs[p] = AllocRec{-1, bytes, pinned};
    R.host_bytes += bytes;
  }
  return p;
}

bool any_gpu_in_use() {
  for (auto &g : R.gpu) if (g.in_use) return true;
  return false;
}

int dev_alloc(int gpu, size_t bytes, void **p) {
  GpuCtx &G = R.gpu[gpu];
  if (bytes == 0) bytes = 16;
  bytes = (bytes + 255) & ~size_t(255);
  if (G.used + bytes > G.budget) { G.try_later++; return TRY_LATER; }
  cudaSetDevice(gpu);
  if (cudaMallocAsync(p, bytes, G.stream) != cudaSuccess) {
    cudaGetLastError();
    G.try_later++;
    return TRY_LATER;
  }
  G.used += bytes;
  if (G.used > G.peak) G.peak = G.used;
  R.allocs[*p] = AllocRec{gpu, bytes, false};
  return TALSH_SUCCESS;
}

// Frees library-owned memory (host or device); unknown pointers are ignored.
int mem_free(void *p) {
  if (p == nullptr) return TALSH_SUCCESS;
  auto it = R.allocs.find(p);
  if (it == R.allocs.end()) return NOT_CLEAN;
  const AllocRec a = it->second;
  R.allocs.erase(it);
  if (a.gpu < 0) {
    if (a.pinned) cudaFreeHost(p); else std::free(p);
    R.host_bytes -= a.bytes;
  } else {
    GpuCtx &G = R.gpu[a.gpu];
    cudaSetDevice(a.gpu);
    cudaFreeAsync(p, G.stream);
    G.used -= a.bytes;
  }
  return TALSH_SUCCESS;
}

cudaEvent_t event_get(int gpu) {
  GpuCtx &G = R.gpu[gpu];
  if (!G.event_pool.empty()) {
    cudaEvent_t e = G.event_pool.back();
    G.event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaSetDevice(gpu);
  cudaEventCreate(&e);
  return e;
}
void event_put(int gpu, cudaEvent_t e) {
  if (e) R.gpu[gpu].event_pool.push_back(e);
}

// Drops the records of copies back that have completed.
void prune_pending(int gpu) {
  GpuCtx &G = R.gpu[gpu];
  for (size_t i = 0; i < G.pending.size();) {
    if (cudaEventQuery(G.pending[i].ev) == cudaSuccess) {
      event_put(gpu, G.pending[i].ev);
      G.pending[i] = G.pending.back();
      G.pending.pop_back();
    } else {
      ++i;
    }
  }
  cudaGetLastError();  // a not-ready query is not an error
}

// Makes stream s wait for every copy back in flight into [p, p + n).
void wait_pending(int gpu, cudaStream_t s, const void *p, size_t n) {
  prune_pending(gpu);
  const char *a = (const char *)p;
  for (const PendingWrite &w : R.gpu[gpu].pending)
    if (a < w.p + w.n && w.p < a + n) cudaStreamWaitEvent(s, w.ev, 0);
}

// Blocks the host until every copy back into [p, p + n) on any GPU is done.
void sync_pending(const void *p, size_t n) {
  const char *a = (const char *)p;
  for (int g = 0; g < MAX_GPUS_PER_NODE; ++g) {
    if (!R.gpu[g].in_use) continue;
    for (const PendingWrite &w : R.gpu[g].pending)
      if (a < w.p + w.n && w.p < a + n) cudaEventSynchronize(w.ev);
  }
}

// Waits for everything queued on the GPU's streams.
void sync_gpu_streams(int gpu) {
  GpuCtx &G = R.gpu[gpu];
  cudaStreamSynchronize(G.h2d);
  cudaStreamSynchronize(G.h2d_b);
  cudaStreamSynchronize(G.stream);
  cudaStreamSynchronize(G.d2h);
}

// Records a copy back into [p, p + n) just issued on stream s.
void note_pending(int gpu, const void *p, size_t n, cudaStream_t s) {
  if (R.gpu[gpu].pending.size() >= 64) prune_pending(gpu);  // keep the list short without staging reads
  cudaEvent_t e = event_get(gpu);
  cudaEventRecord(e, s);
  R.gpu[gpu].pending.push_back(PendingWrite{(const char *)p, n, e});
}

// ---------------------------------------------------------------- tensors
size_t shape_volume(const talsh_tens_shape_t *s) {
  size_t v = 1;
  for (int i = 0; i < s->num_dim; ++i) v *= (size_t)s->dims[i];
  return v;
}

bool healthy(const talsh_tens_t *t) {
  return t->shape_p != nullptr && t->dev_rsc != nullptr && t->data_kind != nullptr &&
         t->avail != nullptr && t->ndev >= 0 && t->ndev <= t->dev_rsc_len;
}

// Releases the memory behind an image descriptor (attached memory is only detached).
int rsc_release(talsh_dev_rsc_t *r) {
  int rc = TALSH_SUCCESS;
  if (r->gmem_p != nullptr && r->mem_attached == 0) rc = mem_free(r->gmem_p);
  tensDevRsc_clean(r);
  return rc;
}

// Discards image i (not allowed when no other available image exists).
int image_discard(talsh_tens_t *t, int i) {
  if (i < 0 || i >= t->ndev) return TALSH_INVALID_ARGS;
  int others = 0;
  for (int j = 0; j < t->ndev; ++j) if (j != i && t->avail[j] == YEP) ++others;
  if (others == 0) return TALSH_NOT_ALLOWED;
  const int rc = rsc_release(&t->dev_rsc[i]);
  const int last = t->ndev - 1;
  if (i < last) {
    t->dev_rsc[i] = t->dev_rsc[last];
    t->data_kind[i] = t->data_kind[last];
    t->avail[i] = t->avail[last];
  }
  tensDevRsc_clean(&t->dev_rsc[last]);
  t->data_kind[last] = NO_TYPE;
  t->avail[last] = NOPE;
  t->ndev--;
  return rc;
}

// Keeps only image i, moved to slot 0.
int image_discard_other(talsh_tens_t *t, int i) {
  if (i < 0 || i >= t->ndev || t->avail[i] != YEP) return TALSH_NOT_ALLOWED;
  int rc = TALSH_SUCCESS;
  for (int j = 0; j < t->ndev; ++j) {
    if (j == i) continue;
    if (rsc_release(&t->dev_rsc[j]) != TALSH_SUCCESS) rc = NOT_CLEAN;
  }
  if (i > 0) {
    t->dev_rsc[0] = t->dev_rsc[i];
    t->data_kind[0] = t->data_kind[i];
    t->avail[0] = t->avail[i];
  }
  for (int j = 1; j < t->dev_rsc_len; ++j) {
    tensDevRsc_clean(&t->dev_rsc[j]);
    t->data_kind[j] = NO_TYPE;
    t->avail[j] = NOPE;
  }
  t->ndev = 1;
  return rc;
}

int find_image(const talsh_tens_t *t, int dev_id, const void *p) {
  for (int i = 0; i < t->ndev; ++i)
    if (t->dev_rsc[i].dev_id == dev_id && t->dev_rsc[i].gmem_p == p) return i;
  return -1;
}

// The image a task made unavailable, or -1 when a later task has dropped it
// already (an output's other images are discarded when the next operation on
// it is scheduled); the same body may meanwhile be a second, available image
// (a placement back into the same Host buffer), which is not this task's.
int find_held_image(const talsh_tens_t *t, int dev_id, const void *p) {
  for (int i = 0; i < t->ndev; ++i)
    if (t->dev_rsc[i].dev_id == dev_id && t->dev_rsc[i].gmem_p == p && t->avail[i] != YEP) return i;
  return -1;
}

// Preferred image for execution on [dvk, dvn]: that device, then that kind, then Host.
// GPU bodies that became images of their tensors when the task writing them
// was scheduled (a moved output, a kept or moved staged input, an output kept
// in place), mapped to their GPU until that task completes.  Work on the same
// GPU's compute stream is ordered after the writer and may use them at once;
// work that would read them from anywhere else waits for the task.
struct TaskRec;
std::unordered_map<const void *, const TaskRec *> g_early;  // body -> the task writing it

bool early_image(const talsh_tens_t *t, int i) { return g_early.count(t->dev_rsc[i].gmem_p) != 0; }

int choose_image(const talsh_tens_t *t, int dvk, int dvn) {
  int same_kind = -1, host = -1;
  for (int i = 0; i < t->ndev; ++i) {
    if (t->avail[i] != YEP) continue;
    int dk = DEV_NULL;
    const int dn = decode_device_id(t->dev_rsc[i].dev_id, &dk);
    if (dn < 0) continue;
    if (dk == DEV_NVIDIA_GPU && early_image(t, i) && !(dvk == DEV_NVIDIA_GPU && dn == dvn)) continue;
    if (dk == dvk) {
      if (dn == dvn) return i;
      if (same_kind < 0) same_kind = i;
    }
    if (dk == DEV_HOST && host < 0) host = i;
  }
  return same_kind >= 0 ? same_kind : host;
}

// ---------------------------------------------------------------- tasks
struct ArgRec {
  talsh_tens_t *t = nullptr;
  int src_dev = -1;        // flat id of the source image
  void *src_ptr = nullptr;
  void *dptr = nullptr;    // body used on the executing GPU
  bool dalloc = false;     // staged copy owned by the task
  unsigned coh = COPY_T;
  bool output = false;
  bool need_input = true;
  bool copy_back = false;  // output copied back into the source image
  bool early = false;      // the GPU body became an image of the tensor at submission
  bool held = false;       // the source image was made unavailable at submission
  size_t bytes = 0;
};

struct TaskRec {
  int gpu = -1;
  cudaStream_t st = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // start, comput, output, finish
  int nargs = 0;
  ArgRec a[MAX_TENSOR_OPERANDS];
  void *scratch = nullptr;
  int split_slices = 0;  // > 0: the contraction runs in the split-precision form
  int failed = 0;
  bool finalized = false;
  double times[4] = {0, 0, 0, 0};  // total, comput, input, output (seconds)
};

TaskRec *rec_of(const talsh_task_t *t) { return (TaskRec *)t->task_p; }

void release_task_events(TaskRec *tr) {
  for (auto &e : tr->ev) { event_put(tr->gpu, e); e = nullptr; }
}

// Applies coherence control and frees task resources (reference talshTaskFinalize :2064).
int task_finalize(talsh_task_t *task, bool success) {
  TaskRec *tr = rec_of(task);
  if (tr == nullptr || tr->finalized) return TALSH_SUCCESS;
  int rc = TALSH_SUCCESS;
  if (success) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, tr->ev[0], tr->ev[3]) == cudaSuccess) tr->times[0] = ms * 1e-3;
    if (cudaEventElapsedTime(&ms, tr->ev[1], tr->ev[2]) == cudaSuccess) tr->times[1] = ms * 1e-3;
    if (cudaEventElapsedTime(&ms, tr->ev[0], tr->ev[1]) == cudaSuccess) tr->times[2] = ms * 1e-3;
    if (cudaEventElapsedTime(&ms, tr->ev[2], tr->ev[3]) == cudaSuccess) tr->times[3] = ms * 1e-3;
    cudaGetLastError();
    task->exec_time = tr->times[0];
  }
  for (int i = tr->nargs - 1; i >= 0; --i) {
    ArgRec &a = tr->a[i];
    talsh_tens_t *t = a.t;
    if (t == nullptr || !healthy(t)) { rc = TALSH_FAILURE; continue; }
    int img = a.held ? find_held_image(t, a.src_dev, a.src_ptr) : find_image(t, a.src_dev, a.src_ptr);
    void *early_body = a.early ? (a.dalloc ? a.dptr : a.src_ptr) : nullptr;
    if (early_body) {
      const auto it = g_early.find(early_body);
      if (it != g_early.end() && it->second == tr) g_early.erase(it);
    }
    if (a.dalloc && a.early) {
      a.dptr = nullptr;  // an image of the tensor since the task was scheduled
    } else if (a.dalloc) {
      if (success && (a.coh == COPY_M || a.coh == COPY_K) && t->ndev < t->dev_rsc_len) {
        const int k = t->ndev++;
        t->dev_rsc[k].dev_id = encode_device_id(DEV_NVIDIA_GPU, tr->gpu);
        t->dev_rsc[k].gmem_p = a.dptr;
        t->dev_rsc[k].buf_entry = -1;
        t->dev_rsc[k].mem_attached = 0;
        t->data_kind[k] = task->data_kind;
        t->avail[k] = YEP;
      } else {
        mem_free(a.dptr);
      }
      a.dptr = nullptr;
    }
    // Only a source image this task made unavailable is released or dropped
    // here: later tasks may already have taken over the others.
    if (img >= 0 && a.held) {
      if (success && (a.coh == COPY_D || a.coh == COPY_M) && t->ndev > 1) {
        if (image_discard(t, img) != TALSH_SUCCESS) rc = NOT_CLEAN;
      } else {
        t->avail[img] = YEP;
      }
    }
    // A failed task's staged body holds no result: it stops being an image.
    if (!success && a.dalloc && early_body) {
      for (int j = 0; j < t->ndev; ++j)
        if (t->dev_rsc[j].gmem_p == early_body) {
          if (image_discard(t, j) != TALSH_SUCCESS) rc = NOT_CLEAN;
          break;
        }
    }
  }
  if (tr->scratch) { mem_free(tr->scratch); tr->scratch = nullptr; }
  GpuCtx &G = R.gpu[tr->gpu];
  if (success) {
    G.tasks_ok++;
    G.flops += task->flops;
    G.bytes += task->data_vol;
  } else {
    G.tasks_failed++;
  }
  tr->finalized = true;
  task->task_error = success ? (rc == TALSH_SUCCESS ? 0 : 13) : (tr->failed > 0 ? tr->failed : 13);
  return rc;
}

// Polls (wait=false) or waits for the task's last event; finalizes when done.
int task_progress(talsh_task_t *task, bool wait) {
  TaskRec *tr = rec_of(task);
  if (tr == nullptr) return TALSH_INVALID_ARGS;
  if (tr->finalized) return task->task_error == 0 ? TALSH_TASK_COMPLETED : TALSH_TASK_ERROR;
  cudaSetDevice(tr->gpu);
  cudaError_t e = wait ? cudaEventSynchronize(tr->ev[3]) : cudaEventQuery(tr->ev[3]);
  if (e == cudaSuccess && tr->split_slices > 0 && !tr->finalized) {
    // The split GEMM's bounded waits count the CTAs that gave up in a device
    // counter: a rise since the last look fails the task.
    const int n = gpu_get_error_count();
    GpuCtx &G = R.gpu[tr->gpu];
    if (n > G.device_errors) {
      G.device_errors = n;
      note_error_text("split-precision contraction: a bounded wait ran out on the device");
      tr->failed = 15;
      task_finalize(task, false);
      return TALSH_TASK_ERROR;
    }
  }
  if (e == cudaSuccess) {
    task_finalize(task, true);
    return task->task_error == 0 ? TALSH_TASK_COMPLETED : TALSH_TASK_ERROR;
  }
  if (e != cudaErrorNotReady) {
    note_cuda_error("task", (int)e);
    tr->failed = 14;
    task_finalize(task, false);
    return TALSH_TASK_ERROR;
  }
  cudaGetLastError();
  if (cudaEventQuery(tr->ev[2]) == cudaSuccess) return TALSH_TASK_OUTPUT_READY;
  if (cudaEventQuery(tr->ev[1]) == cudaSuccess) return TALSH_TASK_INPUT_READY;
  if (cudaEventQuery(tr->ev[0]) == cudaSuccess) return TALSH_TASK_STARTED;
  cudaGetLastError();
  return TALSH_TASK_SCHEDULED;
}

// ------------------------------------------------------- operation driver
enum OpKind { kOpInit, kOpScale, kOpCopy, kOpAdd, kOpContract, kOpNorm1, kOpPlace, kOpSlice, kOpInsert };

struct OpSpec {
  OpKind kind;
  int nt = 0;                        // tensors: D, L, R
  talsh_tens_t *t[3] = {nullptr, nullptr, nullptr};
  unsigned coh_ctrl = 0;
  int dig[2 * MAX_TENSOR_RANK];
  int drank = 0, lrank = 0, rrank = 0, conj = 0;
  double sr = 0.0, si = 0.0;
  int accumulative = YEP;
  double *norm_out = nullptr;        // host result of kOpNorm1
  int offsets[MAX_TENSOR_RANK];      // kOpSlice / kOpInsert base offsets (0-based)
};

// Resolves the execution GPU: returns its ordinal or a negative TAL-SH error.
int resolve_gpu(int dev_id, int dev_kind, talsh_tens_t *const *ts, int nt, int &err) {
  int dvk = DEV_NULL, dvn = -1;
  if (dev_kind == DEV_DEFAULT) {
    if (dev_id == DEV_DEFAULT) {
      dvk = DEV_NVIDIA_GPU;  // every operation of this core runs on a GPU
      dvn = -1;
    } else {
      dvn = decode_device_id(dev_id, &dvk);
      if (dvn < 0) { err = TALSH_INVALID_ARGS; return -1; }
    }
  } else {
    if (valid_device_kind(dev_kind) != YEP) { err = TALSH_INVALID_ARGS; return -1; }
    dvk = dev_kind;
    dvn = (dev_id == DEV_DEFAULT) ? -1 : dev_id;
    if (dvn >= 0 && encode_device_id(dvk, dvn) >= DEV_MAX) { err = TALSH_INVALID_ARGS; return -1; }
  }
  if (dvk != DEV_NVIDIA_GPU) { err = TALSH_NOT_AVAILABLE; return -1; }
  if (dvn < 0) {
    // a GPU already holding the first tensor, else the first GPU in use
    for (int k = 0; k < nt && dvn < 0; ++k) {
      const talsh_tens_t *t = ts[k];
      for (int i = 0; t && i < t->ndev; ++i) {
        int dk = DEV_NULL;
        const int dn = decode_device_id(t->dev_rsc[i].dev_id, &dk);
        if (dk == DEV_NVIDIA_GPU && dn >= 0 && dn < MAX_GPUS_PER_NODE && R.gpu[dn].in_use) { dvn = dn; break; }
      }
    }
    for (int g = 0; g < MAX_GPUS_PER_NODE && dvn < 0; ++g) if (R.gpu[g].in_use) dvn = g;
    if (dvn < 0) { err = TALSH_NOT_AVAILABLE; return -1; }
  }
  if (dvn >= MAX_GPUS_PER_NODE || !R.gpu[dvn].in_use) { err = TALSH_INVALID_ARGS; return -1; }
  return dvn;
}

int kind_size_checked(int kind) { return kind_size(kind); }

int copy_between(void *dst, int dst_dev, const void *src, int src_dev, size_t bytes, cudaStream_t st) {
  int sk = DEV_NULL, dk = DEV_NULL;
  const int sn = decode_device_id(src_dev, &sk), dn = decode_device_id(dst_dev, &dk);
  cudaError_t e;
  if (sk == DEV_NVIDIA_GPU && dk == DEV_NVIDIA_GPU && sn != dn)
    e = cudaMemcpyPeerAsync(dst, dn, src, sn, bytes, st);
  else
    e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, st);
  if (e != cudaSuccess) { note_cuda_error("cudaMemcpyAsync", (int)e); return TALSH_FAILURE; }
  return TALSH_SUCCESS;
}

// Schedules one operation (the shared body of the reference dispatchers).
int schedule(OpSpec &op, int dev_id, int dev_kind, talsh_task_t *user_task) {
  if (!R.on) return TALSH_NOT_INITIALIZED;
  for (int k = 0; k < op.nt; ++k) {
    if (op.t[k] == nullptr) return TALSH_INVALID_ARGS;
    if (talshTensorIsEmpty(op.t[k]) != NOPE) return TALSH_OBJECT_IS_EMPTY;
    if (!healthy(op.t[k])) return TALSH_FAILURE;
  }
  if (user_task != nullptr && talshTaskStatus(user_task) != TALSH_TASK_EMPTY) return TALSH_OBJECT_NOT_EMPTY;
  int err = 0;
  const int gpu = resolve_gpu(dev_id, dev_kind, op.t, op.nt, err);
  if (gpu < 0) return err;
  const int exec_dev = encode_device_id(DEV_NVIDIA_GPU, gpu);
  GpuCtx &G = R.gpu[gpu];

  // Images and data kinds.
  int img[3] = {-1, -1, -1};
  for (int k = 0; k < op.nt; ++k) {
    img[k] = choose_image(op.t[k], DEV_NVIDIA_GPU, gpu);
    if (img[k] < 0) {
      // Every image held by a task still in flight (its output, or a moved
      // input): the operation can run once that task has completed.
      bool held = false;
      for (int i = 0; i < op.t[k]->ndev; ++i) held = held || op.t[k]->avail[i] != YEP || early_image(op.t[k], i);
      return held ? TRY_LATER : TALSH_FAILURE;
    }
  }
  const int dkind = op.t[0]->data_kind[img[0]];
  for (int k = 1; k < op.nt; ++k)
    if (op.t[k]->data_kind[img[k]] != dkind) return TALSH_INVALID_ARGS;
  const int esz = kind_size_checked(dkind);
  if (esz == 0) return TALSH_INVALID_ARGS;

  TaskRec *tr = new TaskRec();
  tr->gpu = gpu;
  tr->st = G.stream;
  tr->nargs = op.nt;
  for (int k = 0; k < op.nt; ++k) {
    ArgRec &a = tr->a[k];
    talsh_tens_t *t = op.t[k];
    a.t = t;
    a.src_dev = t->dev_rsc[img[k]].dev_id;
    a.src_ptr = t->dev_rsc[img[k]].gmem_p;
    a.coh = argument_coherence_get_value(op.coh_ctrl, op.nt, k);
    a.bytes = shape_volume(t->shape_p) * esz;
    a.output = (k == 0) && op.kind != kOpNorm1 && op.kind != kOpPlace;
    a.need_input = !(k == 0 && (op.kind == kOpInit || op.kind == kOpCopy ||
                               ((op.kind == kOpContract || op.kind == kOpSlice) && op.accumulative == NOPE)));
    if (a.src_dev == exec_dev) {
      a.dptr = a.src_ptr;
    } else {
      const int rc = dev_alloc(gpu, a.bytes, &a.dptr);
      if (rc != TALSH_SUCCESS) {
        for (int j = 0; j < k; ++j) if (tr->a[j].dalloc) mem_free(tr->a[j].dptr);
        delete tr;
        return rc;
      }
      a.dalloc = true;
      a.copy_back = a.output && (a.coh == COPY_T || a.coh == COPY_K);
    }
  }
  size_t scratch = 0;
  if (op.kind == kOpContract) {
    int dd[MAX_TENSOR_RANK], ld[MAX_TENSOR_RANK], rd[MAX_TENSOR_RANK];
    for (int i = 0; i < op.drank; ++i) dd[i] = op.t[0]->shape_p->dims[i];
    for (int i = 0; i < op.lrank; ++i) ld[i] = op.t[1]->shape_p->dims[i];
    for (int i = 0; i < op.rrank; ++i) rd[i] = op.t[2]->shape_p->dims[i];
    const int sl = g_r8_slices.load();
    // Split precision: R8 without conjugation flags, C8 with any (rewritten as
    // one real contraction); 0 scratch where the form does not apply.
    const bool split_kind = (dkind == R8 && op.conj == 0) || dkind == C8;
    const size_t split =
        (sl > 0 && split_kind)
            ? tcTensorContractSplitFormScratch(dkind, op.dig, op.drank, dd, op.lrank, ld, op.rrank, rd, sl >> 4,
                                               sl & 15)
            : 0;
    bool hyper = false;
    for (int i = 0; i < op.lrank && !hyper; ++i)
      for (int j = 0; j < op.rrank; ++j)
        if (op.dig[i] > 0 && op.dig[i] == op.dig[op.lrank + j]) { hyper = true; break; }
    if (split > 0 && !hyper) {
      scratch = split;
      tr->split_slices = sl;
    } else {
      scratch = contract_scratch_bytes(dkind, op.dig, op.drank, dd, op.lrank, ld, op.rrank, rd);
    }
  } else if (op.kind == kOpNorm1) {
    scratch = tcTensorNorm1Scratch(shape_volume(op.t[0]->shape_p)) + 256;
  }
  if (scratch > 0) {
    const int rc = dev_alloc(gpu, scratch, &tr->scratch);
    if (rc != TALSH_SUCCESS) {
      for (int j = 0; j < op.nt; ++j) if (tr->a[j].dalloc) mem_free(tr->a[j].dptr);
      delete tr;
      return rc;
    }
  }
  // Resources acquired: commit image bookkeeping (reference: discard other
  // output images, mark moved/discarded sources unavailable).  GPU bodies that
  // outlive the task (a moved output, an output kept in place, a kept or
  // moved staged input) become images right away, usable by later work on
  // this GPU's compute stream (g_early); the rest wait for the task.
  auto register_early = [&](talsh_tens_t *t, ArgRec &a) {
    if (t->ndev >= t->dev_rsc_len) return;
    const int k = t->ndev++;
    t->dev_rsc[k].dev_id = exec_dev;
    t->dev_rsc[k].gmem_p = a.dptr;
    t->dev_rsc[k].buf_entry = -1;
    t->dev_rsc[k].mem_attached = 0;
    t->data_kind[k] = dkind;
    t->avail[k] = YEP;
    g_early[a.dptr] = tr;
    a.early = true;
  };
  if (op.kind != kOpNorm1 && op.kind != kOpPlace) {
    talsh_tens_t *D = op.t[0];
    ArgRec &a0 = tr->a[0];
    const int di = find_image(D, a0.src_dev, a0.src_ptr);
    image_discard_other(D, di);
    if (!a0.dalloc && (a0.coh == COPY_K || a0.coh == COPY_M)) {
      g_early[a0.src_ptr] = tr;  // written in place on this GPU and kept
      a0.early = true;
    } else {
      D->avail[0] = NOPE;
      a0.held = true;
      if (a0.dalloc && a0.coh == COPY_M) register_early(D, a0);
    }
  }
  for (int k = (op.kind == kOpNorm1 || op.kind == kOpPlace) ? 0 : 1; k < op.nt; ++k) {
    ArgRec &a = tr->a[k];
    const int i = find_image(a.t, a.src_dev, a.src_ptr);
    if (a.coh == COPY_D || (a.coh == COPY_M && a.src_dev != exec_dev)) {
      a.t->avail[i] = NOPE;
      a.held = true;
    }
    if (op.kind != kOpNorm1 && op.kind != kOpPlace && a.dalloc && (a.coh == COPY_K || a.coh == COPY_M))
      register_early(a.t, a);
  }

  talsh_task_t *task = user_task;
  if (task == nullptr) {
    if (talshTaskCreate(&task) != TALSH_SUCCESS || task == nullptr) return TALSH_FAILURE;
  }
  task->task_p = tr;
  task->task_error = -1;
  task->dev_kind = DEV_NVIDIA_GPU;
  task->data_kind = dkind;
  task->coherence = (int)op.coh_ctrl;
  task->num_args = op.nt;
  task->data_vol = 0.0;
  for (int k = 0; k < op.nt; ++k) {
    task->tens_args[k].tens_p = op.t[k];
    task->tens_args[k].source_image = find_image(op.t[k], tr->a[k].src_dev, tr->a[k].src_ptr);
    task->data_vol += (double)tr->a[k].bytes;
  }
  task->flops = 0.0;

  // Enqueue: inputs on the staging stream, compute on the GPU's stream,
  // outputs on the copy-back stream, chained by the task's events, so the
  // copies of consecutive asynchronous tasks overlap each other and the
  // compute.  A staging read waits for copies back still in flight into the
  // same Host (or peer) range.
  cudaSetDevice(gpu);
  cudaStream_t st = G.stream;
  for (auto &e : tr->ev) e = event_get(gpu);
  int rc = TALSH_SUCCESS;
  cudaEventRecord(tr->ev[0], st);  // after the staging buffers' stream-ordered allocation
  bool any_in = false, any_out = false;
  for (int k = 0; k < op.nt; ++k) {
    any_in = any_in || (tr->a[k].dalloc && tr->a[k].need_input);
    any_out = any_out || tr->a[k].copy_back;
  }
  if (any_in) {
    // Consecutive tasks stage on alternating streams.  Ordering stays safe: a
    // staging read waits for copies back into its Host range (wait_pending),
    // and a later copy back into a range an earlier task reads follows that
    // task's compute on the single compute stream.
    cudaStream_t hs = (G.staged++ & 1u) ? G.h2d_b : G.h2d;
    cudaStreamWaitEvent(hs, tr->ev[0], 0);
    // inputs first, the destination (most likely to wait for a copy back) last
    for (int k = op.nt - 1; k >= 0 && rc == TALSH_SUCCESS; --k) {
      ArgRec &a = tr->a[k];
      if (!(a.dalloc && a.need_input)) continue;
      wait_pending(gpu, hs, a.src_ptr, a.bytes);
      rc = copy_between(a.dptr, exec_dev, a.src_ptr, a.src_dev, a.bytes, hs);
    }
    cudaEventRecord(tr->ev[1], hs);
    cudaStreamWaitEvent(st, tr->ev[1], 0);
  } else {
    cudaEventRecord(tr->ev[1], st);
  }
  if (rc == TALSH_SUCCESS) {
    const size_t vol = shape_volume(op.t[0]->shape_p);
    switch (op.kind) {
      case kOpInit:
        rc = tcTensorInit(dkind, vol, tr->a[0].dptr, op.sr, op.si, st);
        break;
      case kOpScale:
        rc = tcTensorScale(dkind, vol, tr->a[0].dptr, op.sr, op.si, st);
        task->flops = (kind_is_complex(dkind) ? 6.0 : 1.0) * (double)vol;
        break;
      case kOpCopy: {
        const int lconj = ((op.conj >> 1) ^ op.conj) & 1;
        rc = tcTensorPermute(dkind, op.lrank, op.t[1]->shape_p->dims, op.dig, tr->a[1].dptr,
                             tr->a[0].dptr, lconj, st);
        break;
      }
      case kOpAdd: {
        const int lconj = ((op.conj >> 1) ^ op.conj) & 1;
        rc = tcTensorPermuteAdd(dkind, op.lrank, op.t[1]->shape_p->dims, op.dig, tr->a[1].dptr,
                                tr->a[0].dptr, op.sr, op.si, lconj, st);
        task->flops = (kind_is_complex(dkind) ? 8.0 : 2.0) * (double)vol;
        break;
      }
      case kOpContract: {
        const int *dd = op.t[0]->shape_p->dims, *ld = op.t[1]->shape_p->dims, *rd = op.t[2]->shape_p->dims;
        if (tr->split_slices > 0)
          rc = tcTensorContractSplitForm(dkind, op.dig, op.drank, dd, op.lrank, ld, op.rrank, rd, tr->a[0].dptr,
                                         tr->a[1].dptr, tr->a[2].dptr, op.sr, op.si, op.conj, op.accumulative,
                                         tr->split_slices >> 4, tr->split_slices & 15, tr->scratch, scratch, st);
        else
          rc = contract_launch(dkind, op.dig, op.drank, dd, op.lrank, ld, op.rrank, rd, tr->a[0].dptr,
                               tr->a[1].dptr, tr->a[2].dptr, op.sr, op.si, op.conj, op.accumulative,
                               tr->scratch, scratch, st);
        task->flops = contract_flops(dkind, op.dig, op.lrank, ld, op.rrank, rd);
        break;
      }
      case kOpNorm1: {
        double *res = (double *)((char *)tr->scratch + scratch - 256);
        rc = norm1_launch(dkind, vol, tr->a[0].dptr, res, (double *)tr->scratch, st);
        if (rc == TALSH_SUCCESS && op.norm_out) {
          const cudaError_t e = cudaMemcpyAsync(op.norm_out, res, sizeof(double), cudaMemcpyDeviceToHost, st);
          if (e != cudaSuccess) { note_cuda_error("norm1 readback", (int)e); rc = TALSH_FAILURE; }
        }
        break;
      }
      case kOpPlace:
        break;
      case kOpSlice:   // D = slice of L
        rc = tcTensorSlice(dkind, op.drank, op.t[1]->shape_p->dims, op.t[0]->shape_p->dims, op.offsets,
                           tr->a[1].dptr, tr->a[0].dptr, op.accumulative == YEP ? 1 : 0, st);
        break;
      case kOpInsert:  // L inserted into D
        rc = tcTensorInsert(dkind, op.drank, op.t[0]->shape_p->dims, op.t[1]->shape_p->dims, op.offsets,
                            tr->a[1].dptr, tr->a[0].dptr, op.accumulative == YEP ? 1 : 0, st);
        break;
    }
  }
  cudaEventRecord(tr->ev[2], st);
  if (any_out) {
    cudaStreamWaitEvent(G.d2h, tr->ev[2], 0);
    for (int k = 0; k < op.nt && rc == TALSH_SUCCESS; ++k) {
      ArgRec &a = tr->a[k];
      if (!a.copy_back) continue;
      rc = copy_between(a.src_ptr, a.src_dev, a.dptr, exec_dev, a.bytes, G.d2h);
      if (rc == TALSH_SUCCESS) note_pending(gpu, a.src_ptr, a.bytes, G.d2h);
    }
    cudaEventRecord(tr->ev[3], G.d2h);
  } else {
    cudaEventRecord(tr->ev[3], st);
  }
  if (rc != TALSH_SUCCESS) {
    // Scheduling failed after the task was recorded: the work already queued
    // must drain before its buffers can be released.
    cudaStreamSynchronize(G.h2d);
    cudaStreamSynchronize(G.h2d_b);
    cudaStreamSynchronize(G.d2h);
    cudaStreamSynchronize(st);
    cudaGetLastError();
    tr->failed = 20;
    task_finalize(task, false);
    if (user_task == nullptr) talshTaskDestroy(task);
    return TALSH_FAILURE;
  }
  if (R.log_ops) std::printf("#TALSH-B200: op %d scheduled on GPU %d\n", (int)op.kind, gpu);
  if (user_task == nullptr) {
    int stats = 0;
    int e = talshTaskWait(task, &stats);
    if (e == TALSH_SUCCESS && stats != TALSH_TASK_COMPLETED) e = TALSH_TASK_ERROR;
    const int d = talshTaskDestroy(task);
    if (e == TALSH_SUCCESS && d != TALSH_SUCCESS) e = d;
    return e;
  }
  return TALSH_SUCCESS;
}

int parse_and_check(const char *cptrn, OpSpec &op, int want_inputs) {
  if (cptrn == nullptr) return TALSH_INVALID_ARGS;
  int dr, lr, rr, cj;
  if (talsh_get_contr_ptrn_str2dig(cptrn, op.dig, &dr, &lr, &rr, &cj) != 0) return TALSH_INVALID_ARGS;
  op.drank = dr; op.lrank = lr; op.rrank = rr; op.conj = cj;
  if (op.t[0] && talshTensorRank(op.t[0]) != dr) return TALSH_INVALID_ARGS;
  if (op.t[1] && talshTensorRank(op.t[1]) != lr) return TALSH_INVALID_ARGS;
  if (want_inputs == 2) {
    if (op.t[2] && talshTensorRank(op.t[2]) != rr) return TALSH_INVALID_ARGS;
  } else if (rr != 0) {
    return TALSH_INVALID_ARGS;
  }
  if (want_inputs == 1) {  // copy/add: a permutation of D's indices with matching extents
    if (dr != lr) return TALSH_INVALID_ARGS;
    for (int i = 0; i < lr; ++i) {
      const int p = op.dig[i];
      if (p < 1 || p > dr || op.t[0]->shape_p->dims[p - 1] != op.t[1]->shape_p->dims[i]) return TALSH_INVALID_ARGS;
    }
  }
  return TALSH_SUCCESS;
}

}  // namespace
}  // namespace tb

using namespace tb;

// ===================================================================== C ABI
extern "C" {

double time_sys_sec(void) {
  return std::chrono::duration<double>(std::chrono::system_clock::now().time_since_epoch()).count();
}
double time_high_sec(void) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int talsh_tens_no_init(const talsh_tens_data_t *, const talsh_tens_shape_t *, const talsh_tens_signature_t *) {
  return TALSH_SUCCESS;
}

int tens_valid_data_kind(int datk, int *datk_size) {
  int sz = -1;
  switch (datk) {
    case NO_TYPE: sz = 0; break;
    case R4: sz = 4; break;
    case R8: sz = 8; break;
    case C4: sz = 8; break;
    case C8: sz = 16; break;
    default: break;
  }
  if (datk_size) *datk_size = sz;
  return sz >= 0 ? YEP : NOPE;
}
int tens_valid_data_kind_(int datk, int *datk_size) { return tens_valid_data_kind(datk, datk_size); }
int talshValidDataKind(int datk, int *datk_size) { return tens_valid_data_kind(datk, datk_size); }

int permutation_trivial(const int perm_len, const int *perm, const int base) {
  for (int i = 0; i < perm_len; ++i) if (perm[base + i] != i + 1) return NOPE;
  return YEP;
}

unsigned int argument_coherence_get_value(unsigned int coh_ctrl, unsigned int tot_args, unsigned int arg_num) {
  return (coh_ctrl >> ((tot_args - (arg_num + 1)) * 2)) & kTwoBits;
}

int argument_coherence_set_value(unsigned int *coh_ctrl, unsigned int tot_args, unsigned int arg_num,
                                 unsigned int coh_val) {
  if (arg_num >= tot_args) return 1;
  if (coh_val & ~kTwoBits) return 2;
  const unsigned sh = (tot_args - (arg_num + 1)) * 2;
  *coh_ctrl = (*coh_ctrl & ~(kTwoBits << sh)) | (coh_val << sh);
  return 0;
}

int valid_device_kind(int dev_kind) {
  return (dev_kind == DEV_NULL || dev_kind == DEV_HOST || dev_kind == DEV_NVIDIA_GPU ||
          dev_kind == DEV_INTEL_MIC || dev_kind == DEV_AMD_GPU) ? YEP : NOPE;
}

int encode_device_id(int dev_kind, int dev_num) {
  switch (dev_kind) {
    case DEV_HOST: return dev_num == 0 ? 0 : DEV_MAX;
    case DEV_NVIDIA_GPU: return (dev_num >= 0 && dev_num < MAX_GPUS_PER_NODE) ? 1 + dev_num : DEV_MAX;
    case DEV_INTEL_MIC: return (dev_num >= 0 && dev_num < MAX_MICS_PER_NODE) ? 1 + MAX_GPUS_PER_NODE + dev_num : DEV_MAX;
    case DEV_AMD_GPU:
      return (dev_num >= 0 && dev_num < MAX_AMDS_PER_NODE) ? 1 + MAX_GPUS_PER_NODE + MAX_MICS_PER_NODE + dev_num : DEV_MAX;
    default: return DEV_MAX;
  }
}

int decode_device_id(int dev_id, int *dev_kind) {
  const int id = dev_id < 0 ? -dev_id : dev_id;
  int dk = DEV_NULL, dn = DEV_NULL;
  if (id == 0) { dk = DEV_HOST; dn = 0; }
  else if (id <= MAX_GPUS_PER_NODE) { dk = DEV_NVIDIA_GPU; dn = id - 1; }
  else if (id <= MAX_GPUS_PER_NODE + MAX_MICS_PER_NODE) { dk = DEV_INTEL_MIC; dn = id - 1 - MAX_GPUS_PER_NODE; }
  else if (id <= MAX_GPUS_PER_NODE + MAX_MICS_PER_NODE + MAX_AMDS_PER_NODE) {
    dk = DEV_AMD_GPU; dn = id - 1 - MAX_GPUS_PER_NODE - MAX_MICS_PER_NODE;
  }
  if (dev_kind) *dev_kind = dk;
  return dn;
}

int tensDevRsc_clean(talsh_dev_rsc_t *drsc) {
  if (drsc == nullptr) return -1;
  drsc->dev_id = DEV_NULL;
  drsc->gmem_p = nullptr;
  drsc->buf_entry = -1;
  drsc->mem_attached = 0;
  return 0;
}
int tensDevRsc_is_empty(talsh_dev_rsc_t *drsc) {
  if (drsc == nullptr) return TALSH_INVALID_ARGS;
  return (drsc->dev_id < 0 || drsc->gmem_p == nullptr) ? YEP : NOPE;
}
int tensDevRsc_device_id(talsh_dev_rsc_t *drsc) { return drsc ? drsc->dev_id : DEV_NULL; }

// The rest of the device-resource API (reference tensor_algebra_gpu.cpp:278-555),
// with the reference's return codes.  Memory a descriptor allocates comes from
// the same allocators as tensor bodies: Host memory pinned when a GPU is in use
// (there is no Host argument buffer, so in_arg_buf is ignored), GPU memory from
// that GPU's stream-ordered pool under its byte budget (TRY_LATER above it).
int tensDevRsc_create(talsh_dev_rsc_t **drsc) {
  if (drsc == nullptr) return TALSH_INVALID_ARGS;
  *drsc = (talsh_dev_rsc_t *)std::malloc(sizeof(talsh_dev_rsc_t));
  if (*drsc == nullptr) return TRY_LATER;
  return tensDevRsc_clean(*drsc);
}

int tensDevRsc_same(const talsh_dev_rsc_t *drsc0, const talsh_dev_rsc_t *drsc1) {
  if (drsc0 == nullptr) return -1;
  if (drsc1 == nullptr) return -2;
  return (drsc0->dev_id == drsc1->dev_id && drsc0->gmem_p == drsc1->gmem_p) ? YEP : NOPE;
}

int tensDevRsc_clone(const talsh_dev_rsc_t *drsc_in, talsh_dev_rsc_t *drsc_out) {
  if (drsc_in == nullptr) return -1;
  if (drsc_out == nullptr) return -2;
  *drsc_out = *drsc_in;
  return 0;
}

int tensDevRsc_attach_mem(talsh_dev_rsc_t *drsc, int dev_id, void *mem_p, int buf_entry) {
  if (drsc == nullptr) return -1;
  if (dev_id < 0 || dev_id >= DEV_MAX) return -2;
  if (mem_p == nullptr) return -3;
  if (drsc->dev_id >= 0 && drsc->dev_id != dev_id) return 1;  // bound to another device
  if (drsc->gmem_p != nullptr || drsc->buf_entry >= 0) return 2;  // memory present already
  drsc->dev_id = dev_id;
  drsc->gmem_p = mem_p;
  drsc->buf_entry = buf_entry;
  drsc->mem_attached = 1;
  return 0;
}

int tensDevRsc_detach_mem(talsh_dev_rsc_t *drsc) {
  if (drsc == nullptr) return -1;
  if (drsc->dev_id < 0 || drsc->dev_id >= DEV_MAX) return -2;
  if (drsc->gmem_p == nullptr || drsc->mem_attached == 0) return 1;  // nothing attached
  return tensDevRsc_clean(drsc);  // the memory itself is the caller's
}

int tensDevRsc_allocate_mem(talsh_dev_rsc_t *drsc, int dev_id, size_t mem_size, int in_arg_buf) {
  (void)in_arg_buf;
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (drsc == nullptr) return -1;
  if (dev_id < 0 || dev_id >= DEV_MAX) return -2;
  if (mem_size == 0) return -3;
  int kind = DEV_NULL;
  const int num = decode_device_id(dev_id, &kind);
  if (num < 0) return -4;
  if (drsc->dev_id >= 0 && drsc->dev_id != dev_id) return 1;
  if (drsc->gmem_p != nullptr || drsc->buf_entry >= 0) return 2;
  void *p = nullptr;
  if (kind == DEV_HOST) {
    p = host_alloc(mem_size, any_gpu_in_use());
    if (p == nullptr) return 3;
  } else if (kind == DEV_NVIDIA_GPU) {
    if (!R.on || num >= MAX_GPUS_PER_NODE || !R.gpu[num].in_use) return 5;
    const int rc = dev_alloc(num, mem_size, &p);
    if (rc != TALSH_SUCCESS) return rc;  // TRY_LATER: over the budget, not an error
    // The block comes from the library's stream-ordered pool; the caller may use
    // it on any stream (the reference's gpu_mem_alloc is synchronous), so the
    // allocation is complete before the pointer is handed out.
    if (cudaStreamSynchronize(R.gpu[num].stream) != cudaSuccess) {
      note_cuda_error("tensDevRsc_allocate_mem", (int)cudaGetLastError());
      mem_free(p);
      return TALSH_FAILURE;
    }
  } else {
    return kind == DEV_INTEL_MIC ? -6 : kind == DEV_AMD_GPU ? -7 : -8;
  }
  drsc->dev_id = dev_id;
  drsc->gmem_p = p;
  drsc->buf_entry = -1;
  drsc->mem_attached = 0;
  return 0;
}

int tensDevRsc_free_mem(talsh_dev_rsc_t *drsc) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (drsc == nullptr) return -1;
  if (drsc->dev_id < 0 || drsc->dev_id >= DEV_MAX) return -2;
  if (drsc->gmem_p == nullptr) return -3;
  int kind = DEV_NULL;
  if (decode_device_id(drsc->dev_id, &kind) < 0) return -4;
  if (drsc->mem_attached != 0) return 1;  // attached, not allocated: detach it instead
  if (kind == DEV_NVIDIA_GPU) {
    // The caller's own work on the block may run on any of its streams; like the
    // reference's synchronous gpu_mem_free, wait for the device before the block
    // goes back to the pool, and for the release itself.
    const int num = decode_device_id(drsc->dev_id, &kind);
    cudaSetDevice(num);
    cudaDeviceSynchronize();
    cudaGetLastError();
    const int rc = mem_free(drsc->gmem_p) == TALSH_SUCCESS ? 0 : NOT_CLEAN;
    if (num < MAX_GPUS_PER_NODE) cudaStreamSynchronize(R.gpu[num].stream);
    cudaGetLastError();
    tensDevRsc_clean(drsc);
    return rc;
  }
  const int rc = mem_free(drsc->gmem_p) == TALSH_SUCCESS ? 0 : NOT_CLEAN;
  tensDevRsc_clean(drsc);
  return rc;
}

int tensDevRsc_get_gmem_ptr(talsh_dev_rsc_t *drsc, void **gmem_p) {
  if (drsc == nullptr || gmem_p == nullptr) return -1;
  if (tensDevRsc_is_empty(drsc) == YEP) return 1;
  *gmem_p = drsc->gmem_p;
  return 0;
}

int tensDevRsc_release_all(talsh_dev_rsc_t *drsc) {
  if (drsc == nullptr) return -1;
  int rc = 0;
  if (drsc->dev_id >= 0 && drsc->dev_id < DEV_MAX && drsc->gmem_p != nullptr) {
    const int e = drsc->mem_attached ? tensDevRsc_detach_mem(drsc) : tensDevRsc_free_mem(drsc);
    if (e != 0) rc = NOT_CLEAN;
  }
  tensDevRsc_clean(drsc);
  return rc;
}

int tensDevRsc_destroy(talsh_dev_rsc_t *drsc) {
  if (drsc == nullptr) return -1;
  const int rc = tensDevRsc_release_all(drsc) != 0 ? NOT_CLEAN : 0;
  std::free(drsc);
  return rc;
}

int tensShape_create(talsh_tens_shape_t **tshape) {
  if (tshape == nullptr) return TALSH_INVALID_ARGS;
  *tshape = (talsh_tens_shape_t *)std::malloc(sizeof(talsh_tens_shape_t));
  if (*tshape == nullptr) return TRY_LATER;
  return tensShape_clean(*tshape);
}
int tensShape_clean(talsh_tens_shape_t *s) {
  if (s == nullptr) return TALSH_INVALID_ARGS;
  s->num_dim = -1; s->dims = nullptr; s->divs = nullptr; s->grps = nullptr;
  return TALSH_SUCCESS;
}
int tensShape_construct(talsh_tens_shape_t *s, int, int rank, const int *dims, const int *divs, const int *grps) {
  if (s == nullptr || rank < 0 || rank > MAX_TENSOR_RANK) return TALSH_INVALID_ARGS;
  if (s->num_dim >= 0) return TALSH_OBJECT_NOT_EMPTY;
  if (rank > 0 && dims == nullptr) return TALSH_INVALID_ARGS;
  for (int i = 0; i < rank; ++i) if (dims[i] <= 0) return TALSH_INVALID_ARGS;
  if (rank > 0) {
    s->dims = (int *)std::malloc(sizeof(int) * rank);
    s->divs = (int *)std::malloc(sizeof(int) * rank);
    s->grps = (int *)std::malloc(sizeof(int) * rank);
    if (!s->dims || !s->divs || !s->grps) { tensShape_destruct(s); return TRY_LATER; }
    for (int i = 0; i < rank; ++i) {
      s->dims[i] = dims[i];
      s->divs[i] = divs ? divs[i] : dims[i];
      s->grps[i] = grps ? grps[i] : 0;
    }
  }
  s->num_dim = rank;
  return TALSH_SUCCESS;
}
int tensShape_destruct(talsh_tens_shape_t *s) {
  if (s == nullptr) return TALSH_INVALID_ARGS;
  std::free(s->dims); std::free(s->divs); std::free(s->grps);
  return tensShape_clean(s);
}
int tensShape_destroy(talsh_tens_shape_t *s) {
  if (s == nullptr) return TALSH_INVALID_ARGS;
  tensShape_destruct(s);
  std::free(s);
  return TALSH_SUCCESS;
}
size_t tensShape_volume(const talsh_tens_shape_t *s) {
  if (s == nullptr || s->num_dim < 0) return 0;
  return shape_volume(s);
}
int tensShape_rank(const talsh_tens_shape_t *s) { return s ? s->num_dim : -1; }

// New extents of the same volume (reference tensor_algebra_gpu.cpp): -2 when the
// volume changed (the new shape stays), -3 for a ranked shape without extents,
// -4 for extents given to a rank-0 or empty shape.
int tensShape_reshape(talsh_tens_shape_t *tshape, int rank, const int *dims, const int *divs, const int *grps) {
  if (tshape == nullptr) return -1;
  if (tensShape_rank(tshape) <= 0) return (dims != nullptr || divs != nullptr || grps != nullptr) ? -4 : 0;
  if (tshape->dims == nullptr) return -3;
  const size_t vol = tensShape_volume(tshape);
  int rc = tensShape_destruct(tshape);
  if (rc == 0) rc = tensShape_construct(tshape, NOPE, rank, dims, divs, grps);
  if (rc == 0 && tensShape_volume(tshape) != vol) rc = -2;
  return rc;
}

// Prints the extents as "[d1,d2,...]" (reference tensShape_print).
void tensShape_print(const talsh_tens_shape_t *tshape) {
  if (tshape == nullptr) return;
  std::printf("[");
  for (int i = 0; i < tshape->num_dim; ++i) std::printf(i + 1 < tshape->num_dim ? "%d," : "%d", tshape->dims[i]);
  std::printf("]");
}

// Tensor signatures: a rank and one offset per dimension (reference
// tensor_algebra_gpu.cpp tensSignature_*), with its return codes.
int tensSignature_create(talsh_tens_signature_t **tsigna) {
  if (tsigna == nullptr) return -1;
  *tsigna = (talsh_tens_signature_t *)std::malloc(sizeof(talsh_tens_signature_t));
  if (*tsigna == nullptr) return TRY_LATER;
  return tensSignature_clean(*tsigna);
}

int tensSignature_clean(talsh_tens_signature_t *tsigna) {
  if (tsigna == nullptr) return -1;
  tsigna->num_dim = -1;
  tsigna->offsets = nullptr;
  return 0;
}

int tensSignature_construct(talsh_tens_signature_t *tsigna, int rank, const size_t *offsets) {
  if (tsigna == nullptr) return -1;
  if (tsigna->num_dim >= 0) {
    const int rc = tensSignature_destruct(tsigna);
    if (rc != 0) return rc;
  }
  if (rank < 0) return -2;
  if (rank > 0) {
    if (offsets == nullptr) return -3;
    tsigna->offsets = (size_t *)std::malloc(sizeof(size_t) * (size_t)rank);
    if (tsigna->offsets == nullptr) return TRY_LATER;
    std::memcpy(tsigna->offsets, offsets, sizeof(size_t) * (size_t)rank);
  }
  tsigna->num_dim = rank;
  return 0;
}

int tensSignature_destruct(talsh_tens_signature_t *tsigna) {
  if (tsigna == nullptr) return -1;
  std::free(tsigna->offsets);
  return tensSignature_clean(tsigna);
}

int tensSignature_destroy(talsh_tens_signature_t *tsigna) {
  if (tsigna == nullptr) return -1;
  const int rc = tensSignature_destruct(tsigna);
  std::free(tsigna);
  return rc;
}

// A C pointer as an integer, for Fortran callers (reference tensor_algebra.h:261).
size_t fortran_cptr_int(void *cptr) { return (size_t)(uintptr_t)cptr; }

// Column-major element offset <-> zero-based multi-index (reference
// tensor_algebra_gpu.cpp:172-193; rank 0 is the single element at offset 0).
size_t tens_elem_offset_f(unsigned int num_dim, const unsigned int *dims, const unsigned int *mlndx) {
  size_t offset = 0;
  for (unsigned int i = num_dim; i-- > 0;) offset = offset * dims[i] + mlndx[i];
  return offset;
}

void tens_elem_mlndx_f(size_t offset, unsigned int num_dim, const unsigned int *dims, unsigned int *mlndx) {
  for (unsigned int i = 0; i < num_dim; ++i) {
    mlndx[i] = (unsigned int)(offset % dims[i]);
    offset /= dims[i];
  }
}

// ------------------------------------------------------------ control API
int talshInit(size_t *host_buf_size, int *host_arg_max, int ngpus, int gpu_list[], int nmics,
              int mic_list[], int namds, int amd_list[]) {
  (void)mic_list; (void)amd_list;
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (R.on) return TALSH_ALREADY_INITIALIZED;
  if (ngpus < 0 || ngpus > MAX_GPUS_PER_NODE || nmics < 0 || namds < 0) return TALSH_INVALID_ARGS;
  if (nmics > 0 || namds > 0) return TALSH_NOT_AVAILABLE;
  const int avail = ngpus > 0 ? node_gpu_count() : 0;
  for (int i = 0; i < ngpus; ++i) {
    if (gpu_list == nullptr || gpu_list[i] < 0 || gpu_list[i] >= avail) return TALSH_INVALID_ARGS;
    if (i > 0 && gpu_list[i] != gpu_list[i - 1] + 1) return TALSH_INVALID_ARGS;  // consecutive range
  }
  const char *env = std::getenv("TALSH_B200_GPU_BUDGET_BYTES");
  if (const char *sl = std::getenv("TALSH_B200_R8_SLICES")) {
    const int v = std::atoi(sl);
    if (v == 0 || (v >= 2 && v <= 7)) g_r8_slices = v;
  }
  for (int i = 0; i < ngpus; ++i) {
    const int g = gpu_list[i];
    GpuCtx &G = R.gpu[g];
    if (cudaSetDevice(g) != cudaSuccess) { cudaGetLastError(); return TALSH_FAILURE; }
    if (cudaStreamCreateWithFlags(&G.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&G.h2d, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&G.h2d_b, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&G.d2h, cudaStreamNonBlocking) != cudaSuccess)
      return TALSH_FAILURE;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, g) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    G.budget = env ? (size_t)std::strtoull(env, nullptr, 10) : (fr / 10) * 9;
    G.used = G.peak = 0;
    G.device_errors = std::max(0, gpu_get_error_count());
    G.in_use = true;
  }
  cudaGetLastError();
  if (host_arg_max) *host_arg_max = 1 << 20;
  (void)host_buf_size;  // Host bodies are pinned per tensor; the requested size is reported unchanged
  R.on = true;
  return TALSH_SUCCESS;
}

int talshShutdown(void) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!R.on) return TALSH_NOT_INITIALIZED;
  for (int g = 0; g < MAX_GPUS_PER_NODE; ++g) {
    GpuCtx &G = R.gpu[g];
    if (!G.in_use) continue;
    cudaSetDevice(g);
    sync_gpu_streams(g);
  }
  for (auto &kv : R.allocs) {
    if (kv.second.gpu < 0) { if (kv.second.pinned) cudaFreeHost(kv.first); else std::free(kv.first); }
    else { cudaSetDevice(kv.second.gpu); cudaFree(kv.first); }
  }
  R.allocs.clear();
  R.host_bytes = 0;
  for (int g = 0; g < MAX_GPUS_PER_NODE; ++g) {
    GpuCtx &G = R.gpu[g];
    if (!G.in_use) continue;
    cudaSetDevice(g);
    for (const PendingWrite &w : G.pending) cudaEventDestroy(w.ev);
    G.pending.clear();
    for (cudaEvent_t e : G.event_pool) cudaEventDestroy(e);
    G.event_pool.clear();
    cudaStreamDestroy(G.stream);
    cudaStreamDestroy(G.h2d);
    cudaStreamDestroy(G.h2d_b);
    cudaStreamDestroy(G.d2h);
    G = GpuCtx();
  }
  cudaGetLastError();
  R.on = false;
  return TALSH_SUCCESS;
}

void talshSetMemAllocPolicyHost(int mem_policy, int fallback, int *ierr) {
  R.mem_policy = mem_policy;
  R.mem_fallback = fallback;
  if (ierr) *ierr = TALSH_SUCCESS;
}
int talshEnableFastMath(int, int) { return TALSH_NOT_AVAILABLE; }
int talshDisableFastMath(int, int) { return TALSH_SUCCESS; }
int talshQueryFastMath(int, int) { return NOPE; }

int talshDeviceCount(int dev_kind, int *dev_count) {
  if (dev_count == nullptr) return TALSH_INVALID_ARGS;
  switch (dev_kind) {
    case DEV_HOST: *dev_count = 1; return TALSH_SUCCESS;
    case DEV_NVIDIA_GPU: *dev_count = node_gpu_count(); return TALSH_SUCCESS;
    case DEV_INTEL_MIC:
    case DEV_AMD_GPU: *dev_count = 0; return TALSH_SUCCESS;
    default: return TALSH_INVALID_ARGS;
  }
}
int talshFlatDevId(int dev_kind, int dev_num) { return encode_device_id(dev_kind, dev_num); }
int talshKindDevId(int dev_id, int *dev_kind) { return decode_device_id(dev_id, dev_kind); }

int talshDeviceState(int dev_num, int dev_kind) {
  int dk = dev_kind, dn = dev_num;
  if (dev_kind == DEV_NULL) dn = decode_device_id(dev_num, &dk);
  if (dk == DEV_HOST) return R.on ? DEV_ON : DEV_OFF;
  if (dk == DEV_NVIDIA_GPU && dn >= 0 && dn < MAX_GPUS_PER_NODE) return R.gpu[dn].in_use ? DEV_ON : DEV_OFF;
  return DEV_OFF;
}
int talshDeviceState_(int dev_num, int dev_kind) { return talshDeviceState(dev_num, dev_kind); }

int talshDeviceBusyLeast(int dev_kind) {
  if (dev_kind == DEV_NVIDIA_GPU || dev_kind == DEV_NULL) {
    int best = -1;
    size_t best_used = (size_t)-1;
    for (int g = 0; g < MAX_GPUS_PER_NODE; ++g)
      if (R.gpu[g].in_use && R.gpu[g].used < best_used) { best = g; best_used = R.gpu[g].used; }
    if (best >= 0) return dev_kind == DEV_NULL ? encode_device_id(DEV_NVIDIA_GPU, best) : best;
  }
  if (dev_kind == DEV_HOST || dev_kind == DEV_NULL) return 0;
  return TALSH_NOT_AVAILABLE;
}
int talshDeviceBusyLeast_(int dev_kind) { return talshDeviceBusyLeast(dev_kind); }

int talshDetermineOptimalDevice(const talsh_tens_t *tens0, const talsh_tens_t *tens1, const talsh_tens_t *tens2) {
  const talsh_tens_t *ts[3] = {tens0, tens1, tens2};
  for (const talsh_tens_t *t : ts) {
    if (t == nullptr || t->dev_rsc == nullptr) continue;
    for (int i = 0; i < t->ndev; ++i) {
      int dk = DEV_NULL;
      const int dn = decode_device_id(t->dev_rsc[i].dev_id, &dk);
      if (dk == DEV_NVIDIA_GPU && dn >= 0 && R.gpu[dn].in_use) return t->dev_rsc[i].dev_id;
    }
  }
  for (int g = 0; g < MAX_GPUS_PER_NODE; ++g) if (R.gpu[g].in_use) return encode_device_id(DEV_NVIDIA_GPU, g);
  return DEV_NULL;
}

static int gpu_of(int dev_num, int dev_kind) {
  int dk = dev_kind, dn = dev_num;
  if (dev_kind == DEV_NULL) dn = decode_device_id(dev_num, &dk);
  if (dk != DEV_NVIDIA_GPU || dn < 0 || dn >= MAX_GPUS_PER_NODE) return -1;
  return dn;
}
size_t talshDeviceMemorySize(int dev_num, int dev_kind) {
  const int g = gpu_of(dev_num, dev_kind);
  if (g < 0) return 0;
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, g) != cudaSuccess) { cudaGetLastError(); return 0; }
  return p.totalGlobalMem;
}
size_t talshDeviceMemorySize_(int dev_num, int dev_kind) { return talshDeviceMemorySize(dev_num, dev_kind); }
size_t talshDeviceBufferSize(int dev_num, int dev_kind) {
  const int g = gpu_of(dev_num, dev_kind);
  return (g >= 0 && R.gpu[g].in_use) ? R.gpu[g].budget : 0;
}
size_t talshDeviceBufferSize_(int dev_num, int dev_kind) { return talshDeviceBufferSize(dev_num, dev_kind); }
size_t talshDeviceTensorSize(int dev_num, int dev_kind) { return talshDeviceBufferSize(dev_num, dev_kind); }
size_t talshDeviceTensorSize_(int dev_num, int dev_kind) { return talshDeviceTensorSize(dev_num, dev_kind); }
size_t talshDeviceBufferFreeSize(int dev_num, int dev_kind) {
  const int g = gpu_of(dev_num, dev_kind);
  return (g >= 0 && R.gpu[g].in_use) ? R.gpu[g].budget - R.gpu[g].used : 0;
}
size_t talshDeviceBufferFreeSize_(int dev_num, int dev_kind) { return talshDeviceBufferFreeSize(dev_num, dev_kind); }
void *talshDeviceBufferBasePtr(int, int) { return nullptr; }
void *talshDeviceBufferBasePtr_(int a, int b) { return talshDeviceBufferBasePtr(a, b); }
double talshDeviceGetFlops(int dev_kind, int dev_id) {
  double f = 0.0;
  for (int g = 0; g < MAX_GPUS_PER_NODE; ++g) {
    if (!R.gpu[g].in_use) continue;
    if (dev_kind == DEV_NVIDIA_GPU && dev_id != DEV_DEFAULT && dev_id != g) continue;
    if (dev_kind == DEV_HOST) continue;
    f += R.gpu[g].flops;
  }
  return f;
}
void talshMemManagerLogStart(void) {}
void talshMemManagerLogFinish(void) {}
void talshTensorOpLogStart(void) { R.log_ops = true; }
void talshTensorOpLogFinish(void) { R.log_ops = false; }

int talshStats(int dev_id, int dev_kind) {
  for (int g = 0; g < MAX_GPUS_PER_NODE; ++g) {
    const GpuCtx &G = R.gpu[g];
    if (!G.in_use) continue;
    if (dev_id >= 0 && gpu_of(dev_id, dev_kind) != g) continue;
    std::printf("#TALSH-B200 GPU %d: tasks ok %llu failed %llu deferred %llu; flops %.6e; bytes %.6e; "
                "pool used %zu peak %zu budget %zu\n",
                g, G.tasks_ok, G.tasks_failed, G.try_later, G.flops, G.bytes, G.used, G.peak, G.budget);
  }
  std::printf("#TALSH-B200 Host: library-owned bytes %zu\n", R.host_bytes);
  return TALSH_SUCCESS;
}
int talshStats_(int dev_id, int dev_kind) { return talshStats(dev_id, dev_kind); }

// ------------------------------------------------------------- tensors
int talshTensorCreate(talsh_tens_t **tens_block) {
  if (tens_block == nullptr) return TALSH_INVALID_ARGS;
  *tens_block = (talsh_tens_t *)std::malloc(sizeof(talsh_tens_t));
  if (*tens_block == nullptr) return TRY_LATER;
  return talshTensorClean(*tens_block);
}

int talshTensorClean(talsh_tens_t *t) {
  if (t == nullptr) return TALSH_INVALID_ARGS;
  t->shape_p = nullptr; t->dev_rsc = nullptr; t->data_kind = nullptr; t->avail = nullptr;
  t->dev_rsc_len = 0; t->ndev = 0;
  return TALSH_SUCCESS;
}

int talshTensorIsEmpty(const talsh_tens_t *t) {
  if (t == nullptr) return TALSH_INVALID_ARGS;
  return t->shape_p == nullptr ? YEP : NOPE;
}

int talshTensorConstruct(talsh_tens_t *t, int data_kind, int tens_rank, const int tens_dims[], int dev_id,
                         void *ext_mem, int in_hab, talsh_tens_init_i init_method, double init_val_real,
                         double init_val_imag) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!R.on) return TALSH_NOT_INITIALIZED;
  if (t == nullptr) return TALSH_INVALID_ARGS;
  if (talshTensorIsEmpty(t) != YEP) return TALSH_OBJECT_NOT_EMPTY;
  int dksize = 0;
  if (tens_valid_data_kind(data_kind, &dksize) != YEP) return TALSH_INVALID_ARGS;
  int dev_kind = DEV_NULL;
  const int dev_num = decode_device_id(dev_id, &dev_kind);
  if (dev_num < 0) return TALSH_INVALID_ARGS;
  if (dev_kind != DEV_HOST && dev_kind != DEV_NVIDIA_GPU) return TALSH_NOT_AVAILABLE;
  if (dev_kind == DEV_NVIDIA_GPU && (dev_num >= MAX_GPUS_PER_NODE || !R.gpu[dev_num].in_use))
    return TALSH_INVALID_ARGS;
  int rc = tensShape_create(&t->shape_p);
  if (rc) return rc;
  rc = tensShape_construct(t->shape_p, NOPE, tens_rank, tens_dims, nullptr, nullptr);
  if (rc) { std::free(t->shape_p); t->shape_p = nullptr; return rc == TALSH_OBJECT_NOT_EMPTY ? TALSH_FAILURE : rc; }
  t->dev_rsc = (talsh_dev_rsc_t *)std::malloc(TALSH_MAX_DEV_PRESENT * sizeof(talsh_dev_rsc_t));
  t->data_kind = (int *)std::malloc(TALSH_MAX_DEV_PRESENT * sizeof(int));
  t->avail = (int *)std::malloc(TALSH_MAX_DEV_PRESENT * sizeof(int));
  if (!t->dev_rsc || !t->data_kind || !t->avail) { talshTensorDestruct(t); return TRY_LATER; }
  t->dev_rsc_len = TALSH_MAX_DEV_PRESENT;
  t->ndev = 0;
  for (int j = 0; j < TALSH_MAX_DEV_PRESENT; ++j) {
    tensDevRsc_clean(&t->dev_rsc[j]);
    t->data_kind[j] = NO_TYPE;
    t->avail[j] = NOPE;
  }
  if (ext_mem != nullptr) {
    t->dev_rsc[0].dev_id = dev_id;
    t->dev_rsc[0].gmem_p = ext_mem;
    t->dev_rsc[0].buf_entry = in_hab >= 0 ? in_hab : -1;
    t->dev_rsc[0].mem_attached = 1;
    t->data_kind[0] = data_kind;
    t->avail[0] = YEP;
    t->ndev = 1;
    return TALSH_SUCCESS;
  }
  if (data_kind == NO_TYPE) return TALSH_SUCCESS;
  const size_t vol = shape_volume(t->shape_p);
  const size_t bytes = vol * (size_t)dksize;
  void *p = nullptr;
  if (dev_kind == DEV_HOST) {
    p = host_alloc(bytes, any_gpu_in_use());
    if (p == nullptr) { talshTensorDestruct(t); return TRY_LATER; }
  } else {
    rc = dev_alloc(dev_num, bytes, &p);
    if (rc) { talshTensorDestruct(t); return rc; }
  }
  t->dev_rsc[0].dev_id = dev_id;
  t->dev_rsc[0].gmem_p = p;
  t->dev_rsc[0].buf_entry = -1;
  t->dev_rsc[0].mem_attached = 0;
  t->data_kind[0] = data_kind;
  t->avail[0] = YEP;
  t->ndev = 1;
  // Initialization (reference :1257-1298): Host bodies are filled here, GPU
  // bodies by a blocking talshTensorInit.
  int erc = TALSH_SUCCESS;
  if (dev_kind == DEV_HOST) {
    if (init_method != nullptr) {
      talsh_tens_data_t tdd{p, vol, data_kind};
      if (init_method(&tdd, t->shape_p, nullptr) != 0) erc = NOT_CLEAN;
    } else {
      switch (data_kind) {
        case R4: { float v = (float)init_val_real; float *q = (float *)p; for (size_t i = 0; i < vol; ++i) q[i] = v; break; }
        case R8: { double *q = (double *)p; for (size_t i = 0; i < vol; ++i) q[i] = init_val_real; break; }
        case C4: { float *q = (float *)p; for (size_t i = 0; i < vol; ++i) { q[2 * i] = (float)init_val_real; q[2 * i + 1] = (float)init_val_imag; } break; }
        case C8: { double *q = (double *)p; for (size_t i = 0; i < vol; ++i) { q[2 * i] = init_val_real; q[2 * i + 1] = init_val_imag; } break; }
      }
    }
  } else {
    if (talshTensorInit(t, init_val_real, init_val_imag, dev_id, DEV_DEFAULT, COPY_M, nullptr) != TALSH_SUCCESS)
      erc = NOT_CLEAN;
  }
  return erc;
}

int talshTensorConstruct_(talsh_tens_t *t, int data_kind, int tens_rank, const int tens_dims[], int dev_id,
                          void *ext_mem, int in_hab, talsh_tens_init_i init_method, double vr, double vi) {
  return talshTensorConstruct(t, data_kind, tens_rank, tens_dims, dev_id, ext_mem, in_hab, init_method, vr, vi);
}

int talshTensorImportData(talsh_tens_t *t, int data_kind, const void *ext_data) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!R.on) return TALSH_NOT_INITIALIZED;
  if (t == nullptr || ext_data == nullptr) return TALSH_INVALID_ARGS;
  if (talshTensorIsEmpty(t) != NOPE) return TALSH_OBJECT_IS_EMPTY;
  int es = 0;
  if (tens_valid_data_kind(data_kind, &es) != YEP || es <= 0) return TALSH_INVALID_ARGS;
  const size_t bytes = shape_volume(t->shape_p) * (size_t)es;
  int found = -1;
  for (int i = 0; i < t->ndev; ++i) {
    if (t->data_kind[i] != data_kind || t->avail[i] != YEP) continue;
    found = i;
    int dk = DEV_NULL;
    const int dn = decode_device_id(t->dev_rsc[i].dev_id, &dk);
    if (dk == DEV_HOST) {
      std::memcpy(t->dev_rsc[i].gmem_p, ext_data, bytes);
    } else if (dk == DEV_NVIDIA_GPU) {
      cudaSetDevice(dn);
      if (R.gpu[dn].in_use) sync_gpu_streams(dn);
      if (cudaMemcpy(t->dev_rsc[i].gmem_p, ext_data, bytes, cudaMemcpyDefault) != cudaSuccess) {
        cudaGetLastError();
        return TALSH_FAILURE;
      }
    }
  }
  // Other images (other data kinds) are no longer coherent.
  if (found >= 0)
    for (int i = t->ndev - 1; i >= 0; --i) if (t->data_kind[i] != data_kind) image_discard(t, i);
  return found >= 0 ? TALSH_SUCCESS : TALSH_NOT_FOUND;
}

int talshTensorDestruct(talsh_tens_t *t) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (t == nullptr) return TALSH_INVALID_ARGS;
  int rc = TALSH_SUCCESS;
  if (t->dev_rsc != nullptr) {
    for (int i = 0; i < t->ndev; ++i) {
      int dk = DEV_NULL;
      const int dn = decode_device_id(t->dev_rsc[i].dev_id, &dk);
      if (dk == DEV_NVIDIA_GPU && dn >= 0 && dn < MAX_GPUS_PER_NODE && R.gpu[dn].in_use) {
        cudaSetDevice(dn);
        sync_gpu_streams(dn);  // no queued task may still use the body
      }
      if (rsc_release(&t->dev_rsc[i]) != TALSH_SUCCESS) rc = NOT_CLEAN;
    }
  }
  std::free(t->dev_rsc); std::free(t->data_kind); std::free(t->avail);
  if (t->shape_p) tensShape_destroy(t->shape_p);
  talshTensorClean(t);
  return rc;
}

int talshTensorDestroy(talsh_tens_t *t) {
  if (t == nullptr) return TALSH_INVALID_ARGS;
  const int rc = talshTensorDestruct(t);
  std::free(t);
  return rc;
}

int talshTensorRank(const talsh_tens_t *t) {
  if (t == nullptr) return -1;
  if (t->shape_p == nullptr) return -1;
  return t->shape_p->num_dim;
}

size_t talshTensorVolume(const talsh_tens_t *t) {
  if (t == nullptr || t->shape_p == nullptr) return 0;
  return shape_volume(t->shape_p);
}

size_t talshTensorSizeAllImages(const talsh_tens_t *t, int *num_images) {
  if (num_images) *num_images = 0;
  if (t == nullptr || t->shape_p == nullptr) return 0;
  size_t total = 0;
  const size_t vol = shape_volume(t->shape_p);
  for (int i = 0; i < t->ndev; ++i) { int es = 0; tens_valid_data_kind(t->data_kind[i], &es); total += vol * (size_t)es; }
  if (num_images) *num_images = t->ndev;
  return total;
}

const int *talshTensorDimExtents(const talsh_tens_t *t, int *rank) {
  if (t == nullptr || t->shape_p == nullptr) { if (rank) *rank = -1; return nullptr; }
  if (rank) *rank = t->shape_p->num_dim;
  return t->shape_p->dims;
}

int talshTensorShape(const talsh_tens_t *t, talsh_tens_shape_t *s) {
  if (t == nullptr || s == nullptr) return TALSH_INVALID_ARGS;
  if (t->shape_p == nullptr) return TALSH_OBJECT_IS_EMPTY;
  if (s->num_dim >= 0) tensShape_destruct(s);
  return tensShape_construct(s, NOPE, t->shape_p->num_dim, t->shape_p->dims, t->shape_p->divs, t->shape_p->grps);
}

int talshTensorDataKind(const talsh_tens_t *t, int *num_images, int *data_kinds) {
  if (t == nullptr || num_images == nullptr || data_kinds == nullptr) return TALSH_INVALID_ARGS;
  if (t->shape_p == nullptr) return TALSH_OBJECT_IS_EMPTY;
  *num_images = t->ndev;
  for (int i = 0; i < t->ndev; ++i) data_kinds[i] = t->data_kind[i];
  return TALSH_SUCCESS;
}

int talshTensorReshape(talsh_tens_t *t, int tens_rank, const int tens_dims[]) {
  if (t == nullptr || t->shape_p == nullptr) return TALSH_INVALID_ARGS;
  talsh_tens_shape_t s;
  tensShape_clean(&s);
  const int rc = tensShape_construct(&s, NOPE, tens_rank, tens_dims, nullptr, nullptr);
  if (rc) return rc;
  if (shape_volume(&s) != shape_volume(t->shape_p)) { tensShape_destruct(&s); return TALSH_INVALID_ARGS; }
  tensShape_destruct(t->shape_p);
  *t->shape_p = s;
  return TALSH_SUCCESS;
}

int talshTensorInUse(const talsh_tens_t *t) {
  if (t == nullptr || t->shape_p == nullptr) return TALSH_INVALID_ARGS;
  for (int i = 0; i < t->ndev; ++i) if (t->avail[i] != YEP) return YEP;
  return NOPE;
}

int talshTensorPresence(const talsh_tens_t *t, int *ncopies, int copies[], int data_kinds[], int dev_kind, int dev_id) {
  if (t == nullptr || ncopies == nullptr || copies == nullptr || data_kinds == nullptr) return TALSH_INVALID_ARGS;
  if (t->shape_p == nullptr) return TALSH_OBJECT_IS_EMPTY;
  *ncopies = 0;
  for (int i = 0; i < t->ndev; ++i) {
    int dk = DEV_NULL;
    const int dn = decode_device_id(t->dev_rsc[i].dev_id, &dk);
    if (dev_kind != DEV_NULL && dk != dev_kind) continue;
    if (dev_kind != DEV_NULL && dev_id >= 0 && dn != dev_id) continue;
    copies[*ncopies] = t->dev_rsc[i].dev_id;
    data_kinds[*ncopies] = t->data_kind[i];
    (*ncopies)++;
  }
  return TALSH_SUCCESS;
}
int talshTensorPresence_(const talsh_tens_t *t, int *n, int c[], int d[], int k, int i) { return talshTensorPresence(t, n, c, d, k, i); }

int talshTensorGetBodyAccess(talsh_tens_t *t, void **body_p, int data_kind, int dev_id, int dev_kind) {
  if (t == nullptr || body_p == nullptr) return TALSH_INVALID_ARGS;
  if (t->shape_p == nullptr) return TALSH_OBJECT_IS_EMPTY;
  const int flat = (dev_kind == DEV_NULL) ? dev_id : encode_device_id(dev_kind, dev_id);
  *body_p = nullptr;
  for (int i = 0; i < t->ndev; ++i) {
    if (t->dev_rsc[i].dev_id == flat && t->data_kind[i] == data_kind) {
      if (t->avail[i] != YEP) return TALSH_NOT_ALLOWED;
      int dk = DEV_NULL;
      const int dn = decode_device_id(flat, &dk);
      if (dk == DEV_NVIDIA_GPU && R.gpu[dn].in_use) { cudaSetDevice(dn); sync_gpu_streams(dn); }
      *body_p = t->dev_rsc[i].gmem_p;
      return TALSH_SUCCESS;
    }
  }
  return TALSH_NOT_FOUND;
}
int talshTensorGetBodyAccess_(talsh_tens_t *t, void **b, int k, int i, int dk) { return talshTensorGetBodyAccess(t, b, k, i, dk); }
int talshTensorGetBodyAccessConst(const talsh_tens_t *t, const void **body_p, int data_kind, int dev_id, int dev_kind) {
  void *p = nullptr;
  const int rc = talshTensorGetBodyAccess(const_cast<talsh_tens_t *>(t), &p, data_kind, dev_id, dev_kind);
  if (body_p) *body_p = p;
  return rc;
}

int talshTensorGetScalar(talsh_tens_t *t, double *sr, double *si) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (t == nullptr || sr == nullptr || si == nullptr) return TALSH_INVALID_ARGS;
  if (t->shape_p == nullptr) return TALSH_OBJECT_IS_EMPTY;
  if (t->shape_p->num_dim != 0) return TALSH_INVALID_ARGS;
  for (int i = 0; i < t->ndev; ++i) {
    if (t->avail[i] != YEP) continue;
    unsigned char buf[16];
    int es = 0;
    tens_valid_data_kind(t->data_kind[i], &es);
    int dk = DEV_NULL;
    const int dn = decode_device_id(t->dev_rsc[i].dev_id, &dk);
    if (dk == DEV_HOST) {
      std::memcpy(buf, t->dev_rsc[i].gmem_p, es);
    } else if (dk == DEV_NVIDIA_GPU && R.gpu[dn].in_use) {
      cudaSetDevice(dn);
      sync_gpu_streams(dn);
      if (cudaMemcpy(buf, t->dev_rsc[i].gmem_p, es, cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaGetLastError();
        return TALSH_FAILURE;
      }
    } else {
      continue;
    }
    switch (t->data_kind[i]) {
      case R4: { float v; std::memcpy(&v, buf, 4); *sr = v; *si = 0.0; break; }
      case R8: { double v; std::memcpy(&v, buf, 8); *sr = v; *si = 0.0; break; }
      case C4: { float v[2]; std::memcpy(v, buf, 8); *sr = v[0]; *si = v[1]; break; }
      case C8: { double v[2]; std::memcpy(v, buf, 16); *sr = v[0]; *si = v[1]; break; }
      default: return TALSH_FAILURE;
    }
    return TALSH_SUCCESS;
  }
  return TALSH_NOT_FOUND;
}

void talshTensorPrint(const talsh_tens_t *t) {
  if (t == nullptr || t->shape_p == nullptr) { std::printf("#TENSOR: empty\n"); return; }
  std::printf("#TENSOR: rank %d: dims (", t->shape_p->num_dim);
  for (int i = 0; i < t->shape_p->num_dim; ++i) std::printf(i ? ",%d" : "%d", t->shape_p->dims[i]);
  std::printf(")\n");
}
void talshTensorPrintInfo(const talsh_tens_t *t) {
  talshTensorPrint(t);
  if (t == nullptr || t->shape_p == nullptr) return;
  for (int i = 0; i < t->ndev; ++i)
    std::printf("#  image %d: device %d kind %d avail %d ptr %p attached %d\n", i, t->dev_rsc[i].dev_id,
                t->data_kind[i], t->avail[i], t->dev_rsc[i].gmem_p, t->dev_rsc[i].mem_attached);
}
void talshTensorPrintBody(const talsh_tens_t *t, double thresh) {
  if (t == nullptr || t->shape_p == nullptr) return;
  for (int i = 0; i < t->ndev; ++i) {
    if (t->dev_rsc[i].dev_id != 0) continue;
    const size_t vol = shape_volume(t->shape_p);
    for (size_t l = 0; l < vol; ++l) {
      double re = 0, im = 0;
      switch (t->data_kind[i]) {
        case R4: re = ((float *)t->dev_rsc[i].gmem_p)[l]; break;
        case R8: re = ((double *)t->dev_rsc[i].gmem_p)[l]; break;
        case C4: re = ((float *)t->dev_rsc[i].gmem_p)[2 * l]; im = ((float *)t->dev_rsc[i].gmem_p)[2 * l + 1]; break;
        case C8: re = ((double *)t->dev_rsc[i].gmem_p)[2 * l]; im = ((double *)t->dev_rsc[i].gmem_p)[2 * l + 1]; break;
      }
      if (std::hypot(re, im) > thresh) std::printf("%zu: %.15e %.15e\n", l, re, im);
    }
    return;
  }
}

// ------------------------------------------------------------- slices
// Slice views: a non-owning pointer to a tensor, the base offsets of the slice
// inside it and the slice's extents (reference talshc.cpp:1857-1932), with the
// reference's return codes.  Constructing an already constructed view releases
// its previous extents first.
int talshTensorSliceCreate(talsh_tens_slice_t **slice) {
  if (slice == nullptr) return TALSH_INVALID_ARGS;
  *slice = (talsh_tens_slice_t *)std::malloc(sizeof(talsh_tens_slice_t));
  if (*slice == nullptr) return TRY_LATER;
  return talshTensorSliceClean(*slice);
}

int talshTensorSliceClean(talsh_tens_slice_t *slice) {
  if (slice == nullptr) return TALSH_INVALID_ARGS;
  slice->tensor = nullptr;
  int rc = tensSignature_clean(&slice->bases);
  if (rc == 0) rc = tensShape_clean(&slice->shape);
  return rc;
}

int talshTensorSliceConstruct(talsh_tens_slice_t *slice, const talsh_tens_t *tensor, const size_t *offsets,
                              const int *dims, const int *divs, const int *grps) {
  if (slice == nullptr || tensor == nullptr) return TALSH_INVALID_ARGS;
  int rank = -1;
  const int *ext = talshTensorDimExtents(tensor, &rank);
  if (rank < 0 || (rank > 0 && (offsets == nullptr || dims == nullptr || ext == nullptr))) return TALSH_INVALID_ARGS;
  for (int i = 0; i < rank; ++i)
    if (dims[i] <= 0 || offsets[i] + (size_t)dims[i] > (size_t)ext[i]) return TALSH_INVALID_ARGS;
  if (slice->shape.num_dim >= 0) tensShape_destruct(&slice->shape);
  int rc = tensSignature_construct(&slice->bases, rank, offsets);
  if (rc == 0) rc = tensShape_construct(&slice->shape, NOPE, rank, dims, divs, grps);
  if (rc != 0) {
    talshTensorSliceDestruct(slice);
    return rc;
  }
  slice->tensor = const_cast<talsh_tens_t *>(tensor);
  return TALSH_SUCCESS;
}

size_t talshTensorSliceVolume(const talsh_tens_slice_t *slice) {
  return slice != nullptr ? tensShape_volume(&slice->shape) : 0;
}

int talshTensorSliceDestruct(talsh_tens_slice_t *slice) {
  if (slice == nullptr) return TALSH_INVALID_ARGS;
  int rc = tensShape_destruct(&slice->shape);
  if (rc == 0) rc = tensSignature_destruct(&slice->bases);
  const int rc2 = talshTensorSliceClean(slice);
  return rc != 0 ? rc : rc2;
}

int talshTensorSliceDestroy(talsh_tens_slice_t *slice) {
  if (slice == nullptr) return TALSH_INVALID_ARGS;
  const int rc = talshTensorSliceDestruct(slice);
  std::free(slice);
  return rc;
}

// ------------------------------------------------------------- tasks
int talshTaskCreate(talsh_task_t **task) {
  if (task == nullptr) return TALSH_INVALID_ARGS;
  *task = (talsh_task_t *)std::malloc(sizeof(talsh_task_t));
  if (*task == nullptr) return TRY_LATER;
  return talshTaskClean(*task);
}

int talshTaskClean(talsh_task_t *t) {
  if (t == nullptr) return TALSH_INVALID_ARGS;
  t->task_p = nullptr;
  t->task_error = -1;
  t->dev_kind = DEV_NULL;
  t->data_kind = NO_TYPE;
  t->coherence = -1;
  t->num_args = 0;
  for (int i = 0; i < MAX_TENSOR_OPERANDS; ++i) { t->tens_args[i].tens_p = nullptr; t->tens_args[i].source_image = -1; }
  t->data_vol = 0.0;
  t->flops = 0.0;
  t->exec_time = 0.0;
  return TALSH_SUCCESS;
}

int talshTaskIsEmpty(const talsh_task_t *t) {
  if (t == nullptr) return TALSH_INVALID_ARGS;
  return t->dev_kind == DEV_NULL ? YEP : NOPE;
}

int talshTaskDestruct(talsh_task_t *t) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (t == nullptr) return TALSH_INVALID_ARGS;
  if (t->dev_kind == DEV_NULL) return talshTaskClean(t);
  const int s = talshTaskStatus(t);
  if (s != TALSH_TASK_COMPLETED && s != TALSH_TASK_ERROR) return TALSH_IN_PROGRESS;
  TaskRec *tr = rec_of(t);
  if (tr) { release_task_events(tr); delete tr; }
  return talshTaskClean(t);
}

int talshTaskDestroy(talsh_task_t *t) {
  if (t == nullptr) return TALSH_INVALID_ARGS;
  const int rc = talshTaskDestruct(t);
  if (rc == TALSH_IN_PROGRESS) return rc;
  std::free(t);
  return rc;
}

int talshTaskDevId(talsh_task_t *t, int *dev_kind) {
  if (t == nullptr || t->dev_kind == DEV_NULL || t->task_p == nullptr) return DEV_NULL;
  if (dev_kind) { *dev_kind = t->dev_kind; return rec_of(t)->gpu; }
  return encode_device_id(t->dev_kind, rec_of(t)->gpu);
}
int talshTaskDevId_(talsh_task_t *t, int *dev_kind) { return talshTaskDevId(t, dev_kind); }
int talshTaskArgCoherence(const talsh_task_t *t) { return t ? t->coherence : -1; }
const talshTensArg_t *talshTaskTensArgs(const talsh_task_t *t, int *num_args) {
  if (t == nullptr) { if (num_args) *num_args = 0; return nullptr; }
  if (num_args) *num_args = t->num_args;
  return t->tens_args;
}

int talshTaskStatus(talsh_task_t *t) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!R.on) return TALSH_NOT_INITIALIZED;
  if (t == nullptr) return TALSH_INVALID_ARGS;
  if (t->dev_kind == DEV_NULL) return TALSH_TASK_EMPTY;
  if (t->task_error >= 0) return t->task_error > 0 ? TALSH_TASK_ERROR : TALSH_TASK_COMPLETED;
  if (t->task_p == nullptr) return TALSH_INVALID_ARGS;
  return task_progress(t, false);
}

int talshTaskComplete(talsh_task_t *t, int *stats, int *ierr) {
  if (ierr == nullptr) return TALSH_INVALID_ARGS;
  if (!R.on) { *ierr = TALSH_NOT_INITIALIZED; return NOPE; }
  if (t == nullptr || stats == nullptr) { *ierr = TALSH_INVALID_ARGS; return NOPE; }
  *ierr = TALSH_SUCCESS;
  const int s = talshTaskStatus(t);
  if (s == TALSH_TASK_EMPTY) { *stats = s; *ierr = TALSH_OBJECT_IS_EMPTY; return NOPE; }
  if (s != TALSH_TASK_COMPLETED && s != TALSH_TASK_ERROR && s < TALSH_TASK_EMPTY) { *ierr = s; return NOPE; }
  *stats = s;
  return (s == TALSH_TASK_COMPLETED || s == TALSH_TASK_ERROR) ? YEP : NOPE;
}

int talshTaskWait(talsh_task_t *t, int *stats) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!R.on) return TALSH_NOT_INITIALIZED;
  if (t == nullptr || stats == nullptr) return TALSH_INVALID_ARGS;
  if (t->dev_kind == DEV_NULL) { *stats = TALSH_TASK_EMPTY; return TALSH_OBJECT_IS_EMPTY; }
  if (t->task_error >= 0) { *stats = t->task_error > 0 ? TALSH_TASK_ERROR : TALSH_TASK_COMPLETED; return TALSH_SUCCESS; }
  *stats = task_progress(t, true);
  return TALSH_SUCCESS;
}

int talshTasksWait(int ntasks, talsh_task_t tasks[], int stats[]) {
  if (ntasks < 0 || (ntasks > 0 && (tasks == nullptr || stats == nullptr))) return TALSH_INVALID_ARGS;
  int rc = TALSH_SUCCESS;
  for (int i = 0; i < ntasks; ++i) {
    const int e = talshTaskWait(&tasks[i], &stats[i]);
    if (e != TALSH_SUCCESS && rc == TALSH_SUCCESS) rc = e;
  }
  return rc;
}

int talshTaskTime(talsh_task_t *t, double *total, double *comput, double *input, double *output, double *mmul) {
  if (t == nullptr || total == nullptr) return TALSH_INVALID_ARGS;
  int s = talshTaskStatus(t);
  if (s != TALSH_TASK_COMPLETED) return (s == TALSH_TASK_ERROR) ? TALSH_TASK_ERROR : TALSH_IN_PROGRESS;
  TaskRec *tr = rec_of(t);
  if (tr == nullptr) return TALSH_INVALID_ARGS;
  *total = tr->times[0];
  if (comput) *comput = tr->times[1];
  if (input) *input = tr->times[2];
  if (output) *output = tr->times[3];
  if (mmul) *mmul = tr->times[1];
  return TALSH_SUCCESS;
}
int talshTaskTime_(talsh_task_t *t, double *a, double *b, double *c, double *d, double *e) { return talshTaskTime(t, a, b, c, d, e); }

void talshTaskPrint(const talsh_task_t *t) {
  if (t == nullptr) return;
  std::printf("#TASK: dev_kind %d data_kind %d coherence %d args %d error %d flops %.3e bytes %.3e time %.6f\n",
              t->dev_kind, t->data_kind, t->coherence, t->num_args, t->task_error, t->flops, t->data_vol, t->exec_time);
}

// ------------------------------------------------- tensor-operation objects
int talshTensorOpCreate(talsh_tens_op_t **) { return TALSH_NOT_IMPLEMENTED; }
int talshTensorOpClean(talsh_tens_op_t *) { return TALSH_NOT_IMPLEMENTED; }
int talshTensorOpSetArgument(talsh_tens_op_t *, const talsh_tens_t *, const size_t *, const int *) { return TALSH_NOT_IMPLEMENTED; }
int talshTensorOpSpecify(talsh_tens_op_t *, int, int, const char *, double, double) { return TALSH_NOT_IMPLEMENTED; }
int talshTensorOpSetExecDevice(talsh_tens_op_t *, int, int) { return TALSH_NOT_IMPLEMENTED; }
int talshTensorOpActivate(talsh_tens_op_t *) { return TALSH_NOT_IMPLEMENTED; }
int talshTensorOpLoadInput(talsh_tens_op_t *) { return TALSH_NOT_IMPLEMENTED; }
int talshTensorOpExecute(talsh_tens_op_t *, int, int) { return TALSH_NOT_IMPLEMENTED; }
int talshTensorOpTest(talsh_tens_op_t *, int *, int) { return TALSH_NOT_IMPLEMENTED; }
int talshTensorOpStoreOutput(talsh_tens_op_t *) { return TALSH_NOT_IMPLEMENTED; }
int talshTensorOpDeactivate(talsh_tens_op_t *) { return TALSH_NOT_IMPLEMENTED; }
int talshTensorOpDestruct(talsh_tens_op_t *) { return TALSH_NOT_IMPLEMENTED; }
int talshTensorOpDestroy(talsh_tens_op_t *) { return TALSH_NOT_IMPLEMENTED; }
int talshTensorOpProgress(talsh_tens_op_t *, int *) { return TALSH_NOT_IMPLEMENTED; }
size_t talshTensorOpGetArgVolume(const talsh_tens_op_t *, unsigned int) { return 0; }
size_t talshTensorOpGetArgSize(const talsh_tens_op_t *, unsigned int) { return 0; }
double talshTensorOpGetByteCount(const talsh_tens_op_t *, unsigned int) { return 0.0; }
double talshTensorOpGetFlopCount(const talsh_tens_op_t *) { return 0.0; }
double talshTensorOpGetIntensity(const talsh_tens_op_t *) { return 0.0; }
int talshTensorOpDecompose2(const talsh_tens_op_t *, talsh_tens_op_t *, talsh_tens_op_t *) { return TALSH_NOT_IMPLEMENTED; }
void talshTensorOpPrint(const talsh_tens_op_t *) {}

// ------------------------------------------------------ data placement
int talshTensorPlace(talsh_tens_t *t, int dev_id, int dev_kind, void *dev_mem, int copy_ctrl, talsh_task_t *task) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!R.on) return TALSH_NOT_INITIALIZED;
  if (t == nullptr) return TALSH_INVALID_ARGS;
  if (talshTensorIsEmpty(t) != NOPE) return TALSH_OBJECT_IS_EMPTY;
  if (!healthy(t)) return TALSH_FAILURE;
  const int flat = (dev_kind == DEV_DEFAULT) ? dev_id : encode_device_id(dev_kind, dev_id);
  int dvk = DEV_NULL;
  const int dvn = decode_device_id(flat, &dvk);
  if (dvn < 0) return TALSH_INVALID_ARGS;
  if (copy_ctrl != COPY_M && copy_ctrl != COPY_K) return TALSH_INVALID_ARGS;
  if (dvk != DEV_HOST && dvk != DEV_NVIDIA_GPU) return TALSH_NOT_AVAILABLE;
  if (dvk == DEV_NVIDIA_GPU && (dvn >= MAX_GPUS_PER_NODE || !R.gpu[dvn].in_use)) return TALSH_INVALID_ARGS;
  // Source image: one on the destination device means nothing to do.
  int src = -1;
  bool held = false;
  for (int i = 0; i < t->ndev; ++i) {
    if (t->avail[i] != YEP) { held = true; continue; }
    if (t->dev_rsc[i].dev_id == flat) {
      if (task) { talshTaskClean(task); task->task_error = 0; }
      return TALSH_SUCCESS;
    }
    int dk = DEV_NULL;
    decode_device_id(t->dev_rsc[i].dev_id, &dk);
    // a GPU image still being written is copied to the Host on its own GPU's
    // streams (ordered after the writer), but not to another GPU
    if (dk == DEV_NVIDIA_GPU && dvk == DEV_NVIDIA_GPU && early_image(t, i)) { held = true; continue; }
    if (src < 0 || dk == DEV_HOST) src = i;
  }
  if (src < 0) {
    // Every image held by a task still in flight: the placement can run once
    // that task has completed (as for the operations).
    return held ? TRY_LATER : TALSH_NOT_FOUND;
  }
  int es = 0;
  tens_valid_data_kind(t->data_kind[src], &es);
  const size_t bytes = shape_volume(t->shape_p) * (size_t)es;
  int sk = DEV_NULL;
  const int sn = decode_device_id(t->dev_rsc[src].dev_id, &sk);
  const int gpu = (dvk == DEV_NVIDIA_GPU) ? dvn : sn;  // the GPU whose stream moves the data
  if (sk != DEV_NVIDIA_GPU && dvk != DEV_NVIDIA_GPU) return TALSH_FAILURE;
  if (gpu < 0 || gpu >= MAX_GPUS_PER_NODE || !R.gpu[gpu].in_use) return TALSH_INVALID_ARGS;
  // Destination body.
  void *dst = dev_mem;
  bool owned = false;
  if (dst == nullptr) {
    if (dvk == DEV_HOST) {
      dst = host_alloc(bytes, true);
      if (dst == nullptr) return TRY_LATER;
    } else {
      const int rc = dev_alloc(dvn, bytes, &dst);
      if (rc) return rc;
    }
    owned = true;
  }
  GpuCtx &G = R.gpu[gpu];
  cudaSetDevice(gpu);
  talsh_task_t *tk = task;
  if (tk == nullptr) { if (talshTaskCreate(&tk) != TALSH_SUCCESS) { if (owned) mem_free(dst); return TALSH_FAILURE; } }
  else if (talshTaskStatus(tk) != TALSH_TASK_EMPTY) { if (owned) mem_free(dst); return TALSH_OBJECT_NOT_EMPTY; }
  TaskRec *tr = new TaskRec();
  tr->gpu = gpu;
  tr->st = G.stream;
  tr->nargs = 0;  // set below for a move: the source is discarded when the task completes
  // A copy of a GPU image to the Host runs on the copy-back stream after the
  // work queued on the compute stream (which may still be producing the
  // image), so it overlaps later tasks' compute and staging; other
  // placements run on the compute stream.
  const bool to_host = (dvk == DEV_HOST);
  cudaStream_t cs = to_host ? G.d2h : G.stream;
  for (auto &e : tr->ev) e = event_get(gpu);
  cudaEventRecord(tr->ev[0], G.stream);
  if (to_host) cudaStreamWaitEvent(cs, tr->ev[0], 0);
  cudaEventRecord(tr->ev[1], cs);
  wait_pending(gpu, cs, t->dev_rsc[src].gmem_p, bytes);
  int rc = copy_between(dst, flat, t->dev_rsc[src].gmem_p, t->dev_rsc[src].dev_id, bytes, cs);
  if (to_host && rc == TALSH_SUCCESS) note_pending(gpu, dst, bytes, cs);
  cudaEventRecord(tr->ev[2], cs);
  cudaEventRecord(tr->ev[3], cs);
  // A kept source may be written by later work on the compute stream: that
  // work waits for the copy.
  if (to_host && copy_ctrl == COPY_K) cudaStreamWaitEvent(G.stream, tr->ev[3], 0);
  tk->task_p = tr;
  tk->task_error = -1;
  tk->dev_kind = DEV_NVIDIA_GPU;
  tk->data_kind = t->data_kind[src];
  tk->coherence = copy_ctrl;
  tk->num_args = 1;
  tk->tens_args[0].tens_p = t;
  tk->tens_args[0].source_image = src;
  tk->data_vol = (double)bytes;
  if (rc != TALSH_SUCCESS) {
    sync_gpu_streams(gpu);
    if (owned) mem_free(dst);
    tr->failed = 20;
    task_finalize(tk, false);
    if (task == nullptr) talshTaskDestroy(tk);
    return TALSH_FAILURE;
  }
  // The new image becomes visible right away (reads of a GPU image are ordered
  // on the compute stream; staging reads of a Host image wait for the copy,
  // which is recorded as pending); a moved source becomes unavailable now and
  // is discarded when the task completes (task_finalize applies COPY_M).
  if (t->ndev >= t->dev_rsc_len) { sync_gpu_streams(gpu); if (owned) mem_free(dst); return TALSH_LIMIT_EXCEEDED; }
  const int k = t->ndev++;
  t->dev_rsc[k].dev_id = flat;
  t->dev_rsc[k].gmem_p = dst;
  t->dev_rsc[k].buf_entry = -1;
  t->dev_rsc[k].mem_attached = owned ? 0 : 1;
  t->data_kind[k] = t->data_kind[src];
  t->avail[k] = YEP;
  if (copy_ctrl == COPY_M) {
    ArgRec &a = tr->a[0];
    a.t = t;
    a.src_dev = t->dev_rsc[src].dev_id;
    a.src_ptr = t->dev_rsc[src].gmem_p;
    a.coh = COPY_M;
    a.bytes = bytes;
    a.held = true;
    tr->nargs = 1;
    t->avail[src] = NOPE;
  }
  if (task == nullptr) {
    int stats = 0;
    int e = talshTaskWait(tk, &stats);
    if (e == TALSH_SUCCESS && stats != TALSH_TASK_COMPLETED) e = TALSH_TASK_ERROR;
    talshTaskDestroy(tk);
    return e;
  }
  return TALSH_SUCCESS;
}
int talshTensorPlace_(talsh_tens_t *t, int a, int b, void *c, int d, talsh_task_t *e) { return talshTensorPlace(t, a, b, c, d, e); }

int talshTensorDiscard(talsh_tens_t *t, int dev_id, int dev_kind) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!R.on) return TALSH_NOT_INITIALIZED;
  if (t == nullptr) return TALSH_INVALID_ARGS;
  if (talshTensorIsEmpty(t) != NOPE) return TALSH_OBJECT_IS_EMPTY;
  const int flat = (dev_kind == DEV_NULL) ? dev_id : encode_device_id(dev_kind, dev_id);
  for (int i = t->ndev - 1; i >= 0; --i) {
    if (t->dev_rsc[i].dev_id != flat) continue;
    int dk = DEV_NULL;
    const int dn = decode_device_id(flat, &dk);
    if (dk == DEV_NVIDIA_GPU && R.gpu[dn].in_use) { cudaSetDevice(dn); sync_gpu_streams(dn); }
    return image_discard(t, i);
  }
  return TALSH_SUCCESS;
}
int talshTensorDiscard_(talsh_tens_t *t, int a, int b) { return talshTensorDiscard(t, a, b); }

int talshTensorDiscardOther(talsh_tens_t *t, int dev_id, int dev_kind) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!R.on) return TALSH_NOT_INITIALIZED;
  if (t == nullptr) return TALSH_INVALID_ARGS;
  if (talshTensorIsEmpty(t) != NOPE) return TALSH_OBJECT_IS_EMPTY;
  const int flat = (dev_kind == DEV_NULL) ? dev_id : encode_device_id(dev_kind, dev_id);
  for (int i = 0; i < t->ndev; ++i) {
    if (t->dev_rsc[i].dev_id != flat) continue;
    for (int g = 0; g < MAX_GPUS_PER_NODE; ++g)
      if (R.gpu[g].in_use) { cudaSetDevice(g); sync_gpu_streams(g); }
    return image_discard_other(t, i);
  }
  return TALSH_NOT_FOUND;
}
int talshTensorDiscardOther_(talsh_tens_t *t, int a, int b) { return talshTensorDiscardOther(t, a, b); }

// ------------------------------------------------------ tensor operations
int talshTensorInit(talsh_tens_t *d, double vr, double vi, int dev_id, int dev_kind, int copy_ctrl, talsh_task_t *task) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  OpSpec op;
  op.kind = kOpInit;
  op.nt = 1;
  op.t[0] = d;
  op.coh_ctrl = (unsigned)copy_ctrl;
  op.sr = vr;
  op.si = vi;
  if (copy_ctrl < 0 || copy_ctrl > 3) return TALSH_INVALID_ARGS;
  return schedule(op, dev_id, dev_kind, task);
}
int talshTensorInit_(talsh_tens_t *d, double a, double b, int c, int e, int f, talsh_task_t *g) { return talshTensorInit(d, a, b, c, e, f, g); }

int talshTensorScale(talsh_tens_t *d, double vr, double vi, int dev_id, int dev_kind, int copy_ctrl, talsh_task_t *task) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  OpSpec op;
  op.kind = kOpScale;
  op.nt = 1;
  op.t[0] = d;
  op.coh_ctrl = (unsigned)copy_ctrl;
  op.sr = vr;
  op.si = vi;
  if (copy_ctrl < 0 || copy_ctrl > 3) return TALSH_INVALID_ARGS;
  return schedule(op, dev_id, dev_kind, task);
}
int talshTensorScale_(talsh_tens_t *d, double a, double b, int c, int e, int f, talsh_task_t *g) { return talshTensorScale(d, a, b, c, e, f, g); }

// Slicing and insertion (reference talshc.cpp:4008-4268, :4269-4528): the
// slice's extents plus the offsets must lie inside the full tensor; the
// reference runs them on the CPU only (its GPU entry points are stubs).
static int slice_or_insert(OpKind kind, talsh_tens_t *d, talsh_tens_t *l, const int *offsets, int dev_id,
                           int dev_kind, int copy_ctrl, int accumulative, talsh_task_t *task) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!R.on) return TALSH_NOT_INITIALIZED;
  if (d == nullptr || l == nullptr || offsets == nullptr) return TALSH_INVALID_ARGS;
  if (talshTensorIsEmpty(d) != NOPE || talshTensorIsEmpty(l) != NOPE) return TALSH_OBJECT_IS_EMPTY;
  if (copy_ctrl < 0 || copy_ctrl > 15) return TALSH_INVALID_ARGS;
  const int rank = d->shape_p->num_dim;
  if (rank < 1 || l->shape_p->num_dim != rank) return TALSH_INVALID_ARGS;
  const talsh_tens_shape_t *full = (kind == kOpSlice) ? l->shape_p : d->shape_p;
  const talsh_tens_shape_t *part = (kind == kOpSlice) ? d->shape_p : l->shape_p;
  OpSpec op;
  op.kind = kind;
  op.nt = 2;
  op.t[0] = d;
  op.t[1] = l;
  op.coh_ctrl = (unsigned)copy_ctrl;
  op.accumulative = accumulative == YEP ? YEP : NOPE;
  op.drank = op.lrank = rank;
  for (int i = 0; i < rank; ++i) {
    if (offsets[i] < 0 || (int64_t)offsets[i] + part->dims[i] > full->dims[i]) return TALSH_INVALID_ARGS;
    op.offsets[i] = offsets[i];
  }
  return schedule(op, dev_id, dev_kind, task);
}

int talshTensorSlice(talsh_tens_t *d, talsh_tens_t *l, const int *offsets, int dev_id, int dev_kind, int copy_ctrl,
                     int accumulative, talsh_task_t *task) {
  return slice_or_insert(kOpSlice, d, l, offsets, dev_id, dev_kind, copy_ctrl, accumulative, task);
}
int talshTensorSlice_(talsh_tens_t *a, talsh_tens_t *b, const int *c, int d, int e, int f, int g, talsh_task_t *h) {
  return talshTensorSlice(a, b, c, d, e, f, g, h);
}
int talshTensorInsert(talsh_tens_t *d, talsh_tens_t *l, const int *offsets, int dev_id, int dev_kind, int copy_ctrl,
                      int accumulative, talsh_task_t *task) {
  return slice_or_insert(kOpInsert, d, l, offsets, dev_id, dev_kind, copy_ctrl, accumulative, task);
}
int talshTensorInsert_(talsh_tens_t *a, talsh_tens_t *b, const int *c, int d, int e, int f, int g, talsh_task_t *h) {
  return talshTensorInsert(a, b, c, d, e, f, g, h);
}

int talshTensorCopy(const char *cptrn, talsh_tens_t *d, talsh_tens_t *l, int dev_id, int dev_kind, int copy_ctrl,
                    talsh_task_t *task) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!R.on) return TALSH_NOT_INITIALIZED;
  if (d == nullptr || l == nullptr) return TALSH_INVALID_ARGS;
  if (talshTensorIsEmpty(d) != NOPE || talshTensorIsEmpty(l) != NOPE) return TALSH_OBJECT_IS_EMPTY;
  if (copy_ctrl < 0 || copy_ctrl > 15) return TALSH_INVALID_ARGS;
  OpSpec op;
  op.kind = kOpCopy;
  op.nt = 2;
  op.t[0] = d;
  op.t[1] = l;
  op.coh_ctrl = (unsigned)copy_ctrl;
  const int rc = parse_and_check(cptrn, op, 1);
  if (rc) return rc;
  return schedule(op, dev_id, dev_kind, task);
}
int talshTensorCopy_(const char *p, talsh_tens_t *d, talsh_tens_t *l, int a, int b, int c, talsh_task_t *t) {
  return talshTensorCopy(p, d, l, a, b, c, t);
}

int talshTensorAdd(const char *cptrn, talsh_tens_t *d, talsh_tens_t *l, double sr, double si, int dev_id, int dev_kind,
                   int copy_ctrl, talsh_task_t *task) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!R.on) return TALSH_NOT_INITIALIZED;
  if (d == nullptr || l == nullptr) return TALSH_INVALID_ARGS;
  if (talshTensorIsEmpty(d) != NOPE || talshTensorIsEmpty(l) != NOPE) return TALSH_OBJECT_IS_EMPTY;
  if (copy_ctrl < 0 || copy_ctrl > 15) return TALSH_INVALID_ARGS;
  OpSpec op;
  op.kind = kOpAdd;
  op.nt = 2;
  op.t[0] = d;
  op.t[1] = l;
  op.coh_ctrl = (unsigned)copy_ctrl;
  op.sr = sr;
  op.si = si;
  const int rc = parse_and_check(cptrn, op, 1);
  if (rc) return rc;
  return schedule(op, dev_id, dev_kind, task);
}
int talshTensorAdd_(const char *p, talsh_tens_t *d, talsh_tens_t *l, double a, double b, int c, int e, int f, talsh_task_t *t) {
  return talshTensorAdd(p, d, l, a, b, c, e, f, t);
}

int talshTensorContract(const char *cptrn, talsh_tens_t *d, talsh_tens_t *l, talsh_tens_t *r, double sr, double si,
                        int dev_id, int dev_kind, int copy_ctrl, int accumulative, talsh_task_t *task) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!R.on) return TALSH_NOT_INITIALIZED;
  if (d == nullptr || l == nullptr || r == nullptr) return TALSH_INVALID_ARGS;
  if (talshTensorIsEmpty(d) != NOPE || talshTensorIsEmpty(l) != NOPE || talshTensorIsEmpty(r) != NOPE)
    return TALSH_OBJECT_IS_EMPTY;
  if (copy_ctrl < 0 || copy_ctrl > 63) return TALSH_INVALID_ARGS;
  OpSpec op;
  op.kind = kOpContract;
  op.nt = 3;
  op.t[0] = d;
  op.t[1] = l;
  op.t[2] = r;
  op.coh_ctrl = (unsigned)copy_ctrl;
  op.sr = sr;
  op.si = si;
  op.accumulative = accumulative == NOPE ? NOPE : YEP;
  const int rc = parse_and_check(cptrn, op, 2);
  if (rc) return rc;
  return schedule(op, dev_id, dev_kind, task);
}
int talshTensorContract_(const char *p, talsh_tens_t *d, talsh_tens_t *l, talsh_tens_t *r, double a, double b, int c,
                         int e, int f, int g, talsh_task_t *t) {
  return talshTensorContract(p, d, l, r, a, b, c, e, f, g, t);
}

// ------------------------------------------------- out-of-core contraction
namespace tb {
namespace {

// A sub-contraction: offsets and extents of its D, L and R blocks.
struct XLBlock {
  int off[3][MAX_TENSOR_RANK];
  int dims[3][MAX_TENSOR_RANK];
};

size_t xl_bytes(const XLBlock &b, int a, int rank, int es) {
  size_t v = (size_t)es;
  for (int i = 0; i < rank; ++i) v *= (size_t)b.dims[a][i];
  return v;
}

// One index group of a sub-contraction: its volume and its largest extent
// (the later position on ties), as an operand position.
struct XLGroup {
  size_t vol = 1, top = 0;
  int where = -1;
  void note(size_t ext, int pos) {
    vol *= ext;
    if (ext >= top) { top = ext; where = pos; }
  }
};

// Halves one dimension of a sub-contraction.  The choice follows the rule of
// the reference's talshTensorOpDecompose2 (talshc.cpp:3150-3294), which fixes
// the order in which partial results are summed: an index present in D, L and
// R (a batch index) if there is one, the largest; otherwise the largest index
// of the biggest group, comparing the indices free in R, then free in L, then
// contracted (ties go to that order).  A batch index is halved in all three
// blocks, a free index in D and its operand, a contracted index in L and R.
// Returns false when nothing can be split.
bool xl_split(const XLBlock &p, const int *dig, int drank, int lrank, int rrank, XLBlock &c1, XLBlock &c2) {
  (void)drank;
  XLGroup con, left, right, batch;
  int l_of_d[MAX_TENSOR_RANK] = {0};  // 1 + the L position of each D index that L carries
  for (int i = 0; i < lrank; ++i) {
    const size_t ext = (size_t)p.dims[1][i];
    if (dig[i] < 0) {
      con.note(ext, i);
    } else if (dig[i] > 0) {
      l_of_d[dig[i] - 1] = i + 1;
      left.note(ext, i);
    }
  }
  for (int j = 0; j < rrank; ++j) {
    const int dpos = dig[lrank + j];
    if (dpos <= 0) continue;
    const size_t ext = (size_t)p.dims[2][j];
    if (l_of_d[dpos - 1] == 0) {
      right.note(ext, lrank + j);
    } else {  // in L as well: a batch index, no longer counted as free in L
      left.vol /= ext;
      batch.note(ext, lrank + j);
    }
  }
  if (batch.vol <= 1 && right.vol <= 1 && left.vol <= 1 && con.vol <= 1) return false;
  int cut[3] = {-1, -1, -1};  // the halved dimension's position in D, L and R (-1: untouched)
  if (batch.vol > 1) {
    cut[0] = dig[batch.where] - 1;
    cut[1] = l_of_d[cut[0]] - 1;
    cut[2] = batch.where - lrank;
  } else if (right.vol >= left.vol && right.vol >= con.vol) {
    cut[0] = dig[right.where] - 1;
    cut[2] = right.where - lrank;
  } else if (left.vol >= right.vol && left.vol >= con.vol) {
    cut[0] = dig[left.where] - 1;
    cut[1] = left.where;
  } else {
    cut[1] = con.where;
    cut[2] = -dig[con.where] - 1;
  }
  c1 = p;
  c2 = p;
  for (int a = 0; a < 3; ++a) {
    const int x = cut[a];
    if (x < 0) continue;
    const int first = (p.dims[a][x] + 1) / 2, second = p.dims[a][x] - first;
    if (second <= 0) return false;
    c1.dims[a][x] = first;
    c2.dims[a][x] = second;
    c2.off[a][x] += first;
  }
  return true;
}

// Halves sub-contractions until the D, L and R blocks of each take at most a
// quarter of `avail` bytes (or nothing is left to split).  Children replace
// their parent in place, in order.
int xl_decompose(const int *dig, const int rank[3], const int *const full[3], int es, size_t avail,
                 size_t max_ops, std::vector<XLBlock> &ops) {
  std::vector<XLBlock> next;
  ops.assign(1, XLBlock());
  std::memset(&ops[0], 0, sizeof(XLBlock));
  for (int a = 0; a < 3; ++a)
    for (int i = 0; i < rank[a]; ++i) ops[0].dims[a][i] = full[a][i];
  for (bool again = true; again;) {
    again = false;
    next.clear();
    for (const XLBlock &b : ops) {
      const size_t need = xl_bytes(b, 0, rank[0], es) + xl_bytes(b, 1, rank[1], es) + xl_bytes(b, 2, rank[2], es);
      XLBlock c1, c2;
      if (need * 4 > avail && xl_split(b, dig, rank[0], rank[1], rank[2], c1, c2)) {
        next.push_back(c1);
        next.push_back(c2);
        again = true;
      } else {
        next.push_back(b);
      }
    }
    ops.swap(next);
    if (ops.size() > max_ops) return TALSH_LIMIT_EXCEEDED;
  }
  return TALSH_SUCCESS;
}

// Device address of a Host body: pinned bodies are mapped already; other
// (caller) memory is registered for the duration of the call.
void *xl_map(void *host, size_t bytes, bool &registered) {
  registered = false;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, host) == cudaSuccess && at.type == cudaMemoryTypeHost && at.devicePointer)
    return at.devicePointer;
  cudaGetLastError();
  const cudaError_t e = cudaHostRegister(host, bytes, cudaHostRegisterMapped | cudaHostRegisterPortable);
  if (e == cudaErrorHostMemoryAlreadyRegistered) {
    cudaGetLastError();  // registered by someone else: just map it
  } else if (e != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  } else {
    registered = true;
  }
  void *dp = nullptr;
  if (cudaHostGetDevicePointer(&dp, host, 0) != cudaSuccess) {
    cudaGetLastError();
    cudaHostUnregister(host);
    registered = false;
    return nullptr;
  }
  return dp;
}

}  // namespace
}  // namespace tb

// Out-of-core contraction (reference talshTensorContractXL, talshc.cpp:5394-5648):
// the operands are placed on the Host, the contraction is halved along its
// largest dimension until the three blocks of every sub-contraction fit a
// quarter of the GPU's free budget, and the sub-contractions run one after
// another on the GPU's stream: gather the L, R and D blocks straight from
// mapped Host memory (tcTensorSlice), contract into the D block, write it back
// (tcTensorInsert).  Sub-contractions that split a contracted dimension add
// into the same D block in stream order.  Blocking, like the reference.
int talshTensorContractXL(const char *cptrn, talsh_tens_t *d, talsh_tens_t *l, talsh_tens_t *r, double sr, double si,
                          int dev_id, int dev_kind, int accumulative) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!R.on) return TALSH_NOT_INITIALIZED;
  if (cptrn == nullptr || d == nullptr || l == nullptr || r == nullptr) return TALSH_INVALID_ARGS;
  if (talshTensorIsEmpty(d) != NOPE || talshTensorIsEmpty(l) != NOPE || talshTensorIsEmpty(r) != NOPE)
    return TALSH_OBJECT_IS_EMPTY;
  if (!healthy(d) || !healthy(l) || !healthy(r)) return TALSH_OBJECT_BROKEN;
  OpSpec op;
  op.kind = kOpContract;
  op.nt = 3;
  op.t[0] = d; op.t[1] = l; op.t[2] = r;
  int rc = parse_and_check(cptrn, op, 2);
  if (rc) return rc;
  int err = 0;
  talsh_tens_t *ts[3] = {d, l, r};
  const int gpu = resolve_gpu(dev_id, dev_kind, ts, 3, err);
  if (gpu < 0) return err;
  // Operands on the Host; D keeps only its Host image.
  for (talsh_tens_t *t : {r, l, d})
    if ((rc = talshTensorPlace(t, 0, DEV_HOST, nullptr, COPY_K, nullptr)) != TALSH_SUCCESS) return rc;
  if ((rc = talshTensorDiscardOther(d, 0, DEV_HOST)) != TALSH_SUCCESS) return rc;
  // Earlier asynchronous tasks may still stage from or copy back into these
  // Host bodies; the blocks below are read and written directly.
  sync_gpu_streams(gpu);
  void *hp[3];
  int kind = NO_TYPE;
  for (int a = 0; a < 3; ++a) {
    const int i = choose_image(ts[a], DEV_HOST, 0);
    if (i < 0) return TALSH_FAILURE;
    hp[a] = ts[a]->dev_rsc[i].gmem_p;
    if (a == 0) kind = ts[a]->data_kind[i];
    else if (ts[a]->data_kind[i] != kind) return TALSH_INVALID_ARGS;
  }
  const int es = kind_size(kind);
  if (es == 0) return TALSH_INVALID_ARGS;
  // Copies back into these bodies may also be in flight from tasks on other GPUs.
  for (int a = 0; a < 3; ++a) sync_pending(hp[a], shape_volume(ts[a]->shape_p) * (size_t)es);
  const int rank[3] = {op.drank, op.lrank, op.rrank};
  const int *full[3] = {d->shape_p->dims, l->shape_p->dims, r->shape_p->dims};
  // Decomposition.
  GpuCtx &G = R.gpu[gpu];
  const size_t avail = G.budget > G.used ? G.budget - G.used : 0;
  std::vector<XLBlock> ops;
  if ((rc = xl_decompose(op.dig, rank, full, es, avail, kXLMaxOps, ops)) != TALSH_SUCCESS) return rc;
  // Device buffers sized for the largest block of each argument, and scratch.
  size_t bb[3] = {0, 0, 0}, scratch_bytes = 0;
  const int sl = g_r8_slices.load();
  bool hyper = false;
  for (int i = 0; i < op.lrank && !hyper; ++i)
    for (int j = 0; j < op.rrank; ++j)
      if (op.dig[i] > 0 && op.dig[i] == op.dig[op.lrank + j]) { hyper = true; break; }
  const bool split = sl > 0 && kind == R8 && op.conj == 0 && !hyper && op.drank > 0 && op.lrank > 0 && op.rrank > 0;
  for (const XLBlock &b : ops) {
    for (int a = 0; a < 3; ++a) bb[a] = std::max(bb[a], xl_bytes(b, a, rank[a], es));
    const size_t sc = split ? contract_split_scratch(kind, op.dig, op.drank, b.dims[0], op.lrank, b.dims[1], op.rrank,
                                                     b.dims[2], sl)
                            : contract_scratch_bytes(kind, op.dig, op.drank, b.dims[0], op.lrank, b.dims[1],
                                                     op.rrank, b.dims[2]);
    scratch_bytes = std::max(scratch_bytes, sc);
  }
  void *db[3] = {nullptr, nullptr, nullptr}, *scr = nullptr;
  bool reg[3] = {false, false, false};
  void *mp[3] = {nullptr, nullptr, nullptr};
  auto cleanup = [&]() {
    cudaStreamSynchronize(G.stream);
    cudaGetLastError();
    for (int a = 0; a < 3; ++a) {
      if (db[a]) mem_free(db[a]);
      if (reg[a]) cudaHostUnregister(hp[a]);
    }
    if (scr) mem_free(scr);
  };
  cudaSetDevice(gpu);
  for (int a = 0; a < 3 && rc == TALSH_SUCCESS; ++a) rc = dev_alloc(gpu, bb[a], &db[a]);
  if (rc == TALSH_SUCCESS && scratch_bytes) rc = dev_alloc(gpu, scratch_bytes, &scr);
  for (int a = 0; a < 3 && rc == TALSH_SUCCESS; ++a) {
    const size_t whole = shape_volume(ts[a]->shape_p) * (size_t)es;
    mp[a] = xl_map(hp[a], whole, reg[a]);
    if (mp[a] == nullptr) rc = TALSH_FAILURE;
  }
  if (rc != TALSH_SUCCESS) {
    cleanup();
    return rc;
  }
  if (accumulative == NOPE) std::memset(hp[0], 0, shape_volume(d->shape_p) * (size_t)es);
  cudaStream_t st = G.stream;
  double flops = 0.0;
  for (const XLBlock &b : ops) {
    // gather the blocks (rank-0 arguments are single elements)
    for (int a = 0; a < 3 && rc == TALSH_SUCCESS; ++a) {
      if (rank[a] == 0) {
        const cudaError_t e = cudaMemcpyAsync(db[a], mp[a], (size_t)es, cudaMemcpyDefault, st);
        if (e != cudaSuccess) { note_cuda_error("XL scalar gather", (int)e); rc = TALSH_FAILURE; }
      } else {
        rc = tcTensorSlice(kind, rank[a], full[a], b.dims[a], b.off[a], mp[a], db[a], 0, st);
      }
    }
    if (rc != TALSH_SUCCESS) break;
    if (split)
      rc = contract_split_launch(kind, op.dig, op.drank, b.dims[0], op.lrank, b.dims[1], op.rrank, b.dims[2], db[0],
                                 db[1], db[2], sr, YEP, sl, scr, scratch_bytes, st);
    else
      rc = contract_launch(kind, op.dig, op.drank, b.dims[0], op.lrank, b.dims[1], op.rrank, b.dims[2], db[0], db[1],
                           db[2], sr, si, op.conj, 1, scr, scratch_bytes, st);
    if (rc != TALSH_SUCCESS) break;
    if (rank[0] == 0) {
      const cudaError_t e = cudaMemcpyAsync(mp[0], db[0], (size_t)es, cudaMemcpyDefault, st);
      if (e != cudaSuccess) { note_cuda_error("XL scalar store", (int)e); rc = TALSH_FAILURE; }
    } else {
      rc = tcTensorInsert(kind, rank[0], full[0], b.dims[0], b.off[0], db[0], mp[0], 0, st);
    }
    if (rc != TALSH_SUCCESS) break;
    flops += contract_flops(kind, op.dig, op.lrank, b.dims[1], op.rrank, b.dims[2]);
  }
  const cudaError_t se = cudaStreamSynchronize(st);
  if (rc == TALSH_SUCCESS && se != cudaSuccess) {
    note_cuda_error("XL contraction", (int)se);
    rc = TALSH_FAILURE;
  }
  cleanup();
  if (rc == TALSH_SUCCESS) {
    G.flops += flops;
    G.tasks_ok++;
    g_xl_last_ops = ops.size();
  } else {
    G.tasks_failed++;
  }
  return rc;
}
size_t tcContractXLLastOps(void) { return g_xl_last_ops; }

int tcContractXLPlan(int data_kind, const int *cptrn, int drank, const int *ddims, int lrank, const int *ldims,
                     int rrank, const int *rdims, size_t budget_bytes, int max_ops, int *offsets, int *extents) {
  const int es = kind_size(data_kind);
  if (es == 0 || drank < 0 || lrank < 0 || rrank < 0 || drank > MAX_TENSOR_RANK || lrank > MAX_TENSOR_RANK ||
      rrank > MAX_TENSOR_RANK || lrank + rrank == 0 || cptrn == nullptr || max_ops < 1 ||
      (drank > 0 && ddims == nullptr) || (lrank > 0 && ldims == nullptr) || (rrank > 0 && rdims == nullptr))
    return TALSH_INVALID_ARGS;
  const int rank[3] = {drank, lrank, rrank};
  const int *full[3] = {ddims, ldims, rdims};
  for (int a = 0; a < 3; ++a)
    for (int i = 0; i < rank[a]; ++i)
      if (full[a][i] <= 0) return TALSH_INVALID_ARGS;
  std::vector<XLBlock> ops;
  const int rc = xl_decompose(cptrn, rank, full, es, budget_bytes, (size_t)max_ops, ops);
  if (rc != TALSH_SUCCESS) return rc;
  const int w = drank + lrank + rrank;
  for (size_t o = 0; o < ops.size(); ++o) {
    int j = 0;
    for (int a = 0; a < 3; ++a)
      for (int i = 0; i < rank[a]; ++i, ++j) {
        if (offsets) offsets[o * w + j] = ops[o].off[a][i];
        if (extents) extents[o * w + j] = ops[o].dims[a][i];
      }
  }
  return (int)ops.size();
}

int talshTensorContractXL_(const char *p, talsh_tens_t *d, talsh_tens_t *l, talsh_tens_t *r, double a, double b, int c,
                           int e, int f) {
  return talshTensorContractXL(p, d, l, r, a, b, c, e, f);
}

int talshTensorDecomposeSVD(const char *, talsh_tens_t *, talsh_tens_t *, talsh_tens_t *, talsh_tens_t *, const char, int, int) {
  return TALSH_NOT_IMPLEMENTED;
}
int talshTensorDecomposeSVDL(const char *, talsh_tens_t *, talsh_tens_t *, talsh_tens_t *, int, int) { return TALSH_NOT_IMPLEMENTED; }
int talshTensorDecomposeSVDR(const char *, talsh_tens_t *, talsh_tens_t *, talsh_tens_t *, int, int) { return TALSH_NOT_IMPLEMENTED; }
int talshTensorDecomposeSVDLR(const char *, talsh_tens_t *, talsh_tens_t *, talsh_tens_t *, int, int) { return TALSH_NOT_IMPLEMENTED; }
int talshTensorOrthogonalizeSVD(const char *, talsh_tens_t *, int, int) { return TALSH_NOT_IMPLEMENTED; }
int talshTensorOrthogonalizeMGS(talsh_tens_t *, int, int *, int, int) { return TALSH_NOT_IMPLEMENTED; }

double talshTensorImageNorm1_cpu(const talsh_tens_t *t) {
  if (t == nullptr || t->shape_p == nullptr) return -1.0;
  for (int i = 0; i < t->ndev; ++i) {
    if (t->dev_rsc[i].dev_id != 0) continue;
    const size_t n = shape_volume(t->shape_p);
    const void *p = t->dev_rsc[i].gmem_p;
    {
      int es = 0;
      tens_valid_data_kind(t->data_kind[i], &es);
      std::lock_guard<std::recursive_mutex> lk(g_mu);
      if (R.on) sync_pending(p, n * (size_t)es);  // copies back into this image still in flight
    }
    double s = 0.0;
    switch (t->data_kind[i]) {
      case R4: for (size_t j = 0; j < n; ++j) s += (double)std::fabs(((const float *)p)[j]); break;
      case R8: for (size_t j = 0; j < n; ++j) s += std::fabs(((const double *)p)[j]); break;
      case C4: for (size_t j = 0; j < n; ++j) s += (double)std::hypot(((const float *)p)[2 * j], ((const float *)p)[2 * j + 1]); break;
      case C8: for (size_t j = 0; j < n; ++j) s += std::hypot(((const double *)p)[2 * j], ((const double *)p)[2 * j + 1]); break;
      default: return -1.0;
    }
    return s;
  }
  return -1.0;
}

double talshTensorNorm1(talsh_tens_t *t, int dev_id, int dev_kind) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!R.on || t == nullptr || talshTensorIsEmpty(t) != NOPE) return -1.0;
  // One pinned result slot for the process, allocated on first use (the call
  // is blocking and serialised by the library lock).
  static double *out = nullptr;
  if (out == nullptr) {
    if (cudaMallocHost((void **)&out, sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      out = nullptr;
      return -1.0;
    }
  }
  *out = -1.0;
  OpSpec op;
  op.kind = kOpNorm1;
  op.nt = 1;
  op.t[0] = t;
  op.coh_ctrl = COPY_T;  // a staged copy of a Host image is temporary
  op.norm_out = out;
  const int rc = schedule(op, dev_id, dev_kind, nullptr);
  return (rc == TALSH_SUCCESS) ? *out : -1.0;
}
double talshTensorNorm1_(talsh_tens_t *t, int dev_id, int dev_kind) { return talshTensorNorm1(t, dev_id, dev_kind); }

int talshContractSlicesSet(int slices) {
  if (slices != 0 && (slices < 2 || slices > 7)) return TALSH_INVALID_ARGS;
  g_r8_slices = slices;
  return TALSH_SUCCESS;
}

int talshContractSlicesGet(void) { return g_r8_slices.load() & 15; }

int talshContractSplitFormSet(int form, int slices) {
  if (form < 0 || form > 3) return TALSH_INVALID_ARGS;
  if (slices != 0 && (slices < 2 || slices > 7)) return TALSH_INVALID_ARGS;
  if (form == 0 && slices == 0) {  // int8 digits at their default count
    g_r8_slices = 6;
    return TALSH_SUCCESS;
  }
  g_r8_slices = (form << 4) | slices;
  return TALSH_SUCCESS;
}

int talshContractSplitFormGet(int *form, int *slices) {
  if (form == nullptr || slices == nullptr) return TALSH_INVALID_ARGS;
  const int v = g_r8_slices.load();
  *form = (v >> 4) & 15;
  *slices = v & 15;
  return TALSH_SUCCESS;
}

}  // extern "C"

// Pinning of caller memory (include/mem_manager.h), for the reference's C++
// layer.  Portable: the pinned range serves every GPU of the process.
#include "mem_manager.h"

int host_mem_register(void *host_ptr, size_t tsize) {
  const cudaError_t e = cudaHostRegister(host_ptr, tsize, cudaHostRegisterPortable);
  if (e != cudaSuccess) {
    cudaGetLastError();
    tb::note_cuda_error("host_mem_register", (int)e);
    return 1;
  }
  return 0;
}

int host_mem_unregister(void *host_ptr) {
  const cudaError_t e = cudaHostUnregister(host_ptr);
  if (e != cudaSuccess) {
    cudaGetLastError();
    tb::note_cuda_error("host_mem_unregister", (int)e);
    return 1;
  }
  return 0;
}

// Entry points of the reference's C side that its Fortran module binds
// (talshf.F90:528-547).

// One body image of a tensor (reference talshc.cpp:245-267): its flat device
// id, data kind, address and argument-buffer entry (-1 for bodies the library
// allocates, which are not in a carved buffer; the caller's value for external
// memory); TALSH_NOT_ALLOWED when the image is no longer available.
int talsh_tensor_image_info(const talsh_tens_t *talsh_tens, int image_id, int *dev_id, int *data_kind,
                            void **gmem_p, int *buf_entry) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (talsh_tens == nullptr || dev_id == nullptr || data_kind == nullptr || gmem_p == nullptr ||
      buf_entry == nullptr)
    return TALSH_INVALID_ARGS;
  if (talshTensorIsEmpty(talsh_tens) != NOPE) return TALSH_OBJECT_IS_EMPTY;
  if (!healthy(talsh_tens)) return TALSH_FAILURE;
  if (image_id < 0 || image_id >= talsh_tens->ndev) return TALSH_INVALID_ARGS;
  talsh_dev_rsc_t *r = &talsh_tens->dev_rsc[image_id];
  if (tensDevRsc_is_empty(r) != NOPE) return TALSH_FAILURE;
  if (talsh_tens->avail[image_id] != YEP) return TALSH_NOT_ALLOWED;
  *dev_id = r->dev_id;
  *data_kind = talsh_tens->data_kind[image_id];
  *gmem_p = r->gmem_p;
  *buf_entry = r->buf_entry;
  return TALSH_SUCCESS;
}

// Number of NVIDIA GPUs on the node (reference tensor_algebra_gpu_nvidia.cu:2728-2739):
// 0, or 1 with *dev_count = -1 when the CUDA runtime cannot tell.
int gpu_get_device_count(int *dev_count) {
  if (dev_count == nullptr) return 1;
  const cudaError_t e = cudaGetDeviceCount(dev_count);
  if (e != cudaSuccess) {
    cudaGetLastError();
    tb::note_cuda_error("gpu_get_device_count", (int)e);
    *dev_count = -1;
    return 1;
  }
  return 0;
}
