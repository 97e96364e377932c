// Contraction server (tcServer*, declared in talsh_b200.h).
//
// A single scheduling thread drives three queues:
//  * admission: submitted tasks in arrival order, one queue for small and one
//    for large tasks (a large task waiting for memory never holds up small
//    ones); a head is admitted when its server-held output (and, for a large
//    task, its scratch) fits the device-memory budget, and large tasks only
//    while fewer than max_inflight + 1 of them are admitted and unfinished; a
//    task that alone exceeds the budget fails with TALSH_LIMIT_EXCEEDED;
//  * waiting: admitted tasks whose producers have not been launched yet;
//  * in flight: launched batches, each with one event.
// Small tasks are gathered into continuous batches on stream 0 (one
// batch_launch_with call per batch: one table launch and one persistent
// gather-GEMM launch per tile configuration).  Tasks at or above the flop
// threshold run alone on stream 1 (split precision for R8 when configured).
// A consumer on the producer's stream only needs the producer launched
// (stream order); a large consumer of a small producer waits on the
// producer's batch event; a small consumer of a large producer waits until
// the producer has completed, so a long task never stalls the batch stream.
// Server-held outputs are freed once their declared consumers have completed
// (and, when kept, after tcServerRelease).
//
// The reference schedules one operation per talshTensorContract call and
// tracks it with a talsh_task_t (talshc.cpp:5073-5392, :2336-2561); there is
// no admission control or batching there.  Latency is measured from the
// submission (or, in tcServerReplay, the scheduled arrival) to the host
// observing the batch's completion event.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <unordered_map>
#include <vector>

#include "common.h"

namespace tb {
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
int contract_validate(int kind, const int *cptrn, int drank, const int *ddims, int lrank, const int *ldims,
                      int rrank, const int *rdims);
}  // namespace tb

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

size_t round_bytes(size_t b) { return (std::max<size_t>(b, 16) + 255) & ~size_t(255); }

enum State { kQueued = 0, kAdmitted = 1, kLaunched = 2, kDone = 3 };

struct STask {
  tcServeTask spec;
  int state = kQueued;
  bool large = false;
  bool own_out = false;
  bool waited = false;     // held at admission at least once
  bool released = false;   // tcServerRelease called
  bool split = false;      // large R8 task in split precision
  bool counted = false;    // large task counted in large_active
  void *out = nullptr;     // D used by the launch
  size_t out_bytes = 0;    // server-held output bytes (0: caller's D)
  void *scratch = nullptr; // large tasks: scratch allocated at admission
  size_t scratch_bytes = 0;
  size_t reserve = 0;      // small tasks: budget held for their share of a batch's scratch
  int consumers_left = 0;  // declared consumers that have not completed
  int readers = 0;         // submitted consumers that have not completed
  int stream = 0;          // 0: batch stream, 1: large-task stream
  cudaEvent_t launch_ev = nullptr;  // event of the batch that carries it (while in flight)
  double t_submit = 0.0;
  int status = TALSH_SUCCESS;
};

struct Inflight {
  int stream = 0;
  cudaEvent_t ev = nullptr;
  std::vector<uint64_t> ids;
  void *scratch = nullptr;
  size_t scratch_bytes = 0;
  void *stage = nullptr;
  size_t stage_bytes = 0;
};

struct DoneRec {
  uint64_t id;
  double latency;
  int status;
};

int64_t vol(const int *d, int n) {
  int64_t v = 1;
  for (int i = 0; i < n; ++i) v *= d[i];
  return v;
}

double task_flops(const tcContractTask &t) {
  return tb::contract_flops(t.data_kind, t.cptrn, t.lrank, t.ldims, t.rrank, t.rdims);
}

}  // namespace

struct tcServer {
  int dev = 0;
  cudaStream_t st[2] = {nullptr, nullptr};
  cudaMemPool_t pool = nullptr;  // the server's own stream-ordered pool; it keeps freed memory
  tcServeConfig cfg{};
  size_t used = 0, peak = 0;
  size_t reserved = 0;  // batch scratch promised to admitted, unlaunched small tasks
  uint64_t next_id = 1;
  size_t pending = 0;  // submitted, not completed
  std::unordered_map<uint64_t, STask> tasks;
  std::deque<uint64_t> admit_q[2];  // per stream: small, large
  int large_active = 0;              // large tasks admitted and not completed
  std::vector<uint64_t> waiting;
  std::deque<Inflight> inflight;
  std::deque<DoneRec> done;
  std::vector<std::pair<void *, size_t>> stages;  // free pinned staging blocks
  std::vector<cudaEvent_t> events;
  tcServeStats stats{};
};

namespace {

int dalloc(tcServer *s, size_t bytes, int stream, void **p) {
  bytes = round_bytes(bytes);
  if (s->used + s->reserved + bytes > s->cfg.budget_bytes) return TRY_LATER;
  if (cudaMallocFromPoolAsync(p, bytes, s->pool, s->st[stream]) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return TRY_LATER;
  }
  s->used += bytes;
  s->peak = std::max(s->peak, s->used);
  return TALSH_SUCCESS;
}

void dfree(tcServer *s, void *p, size_t bytes, int stream) {
  if (p == nullptr) return;
  cudaFreeAsync(p, s->st[stream]);
  s->used -= round_bytes(bytes);
}

cudaEvent_t event_get(tcServer *s) {
  if (!s->events.empty()) {
    cudaEvent_t e = s->events.back();
    s->events.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return e;
}

void *stage_get(tcServer *s, size_t bytes, size_t *got) {
  for (size_t i = 0; i < s->stages.size(); ++i) {
    if (s->stages[i].second >= bytes) {
      void *p = s->stages[i].first;
      *got = s->stages[i].second;
      s->stages.erase(s->stages.begin() + (long)i);
      return p;
    }
  }
  const size_t b = std::max<size_t>(bytes, 64 << 10);
  void *p = nullptr;
  if (cudaHostAlloc(&p, b, cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  *got = b;
  return p;
}

void maybe_free_output(tcServer *s, STask &t) {
  if (!t.own_out || t.out == nullptr || t.state != kDone || t.readers > 0 || t.consumers_left > 0) return;
  if (t.spec.keep_output && !t.released) return;
  dfree(s, t.out, t.out_bytes, t.stream);
  t.out = nullptr;
}

void complete(tcServer *s, uint64_t id, int status, double t_now) {
  STask &t = s->tasks[id];
  t.state = kDone;
  t.status = status;
  t.launch_ev = nullptr;
  s->done.push_back(DoneRec{id, t_now - t.t_submit, status});
  s->reserved -= t.reserve;
  t.reserve = 0;
  if (t.counted) s->large_active--;
  t.counted = false;
  s->pending--;
  if (status == TALSH_SUCCESS) s->stats.completed++; else s->stats.failed++;
  for (uint64_t p : {t.spec.l_from, t.spec.r_from}) {
    if (p == 0) continue;
    auto it = s->tasks.find(p);
    if (it == s->tasks.end()) continue;
    it->second.readers--;
    it->second.consumers_left--;
    maybe_free_output(s, it->second);
  }
  if (t.scratch) {
    dfree(s, t.scratch, t.scratch_bytes, t.stream);
    t.scratch = nullptr;
  }
  if (status != TALSH_SUCCESS && t.own_out && t.out) {  // a failed output is never read
    dfree(s, t.out, t.out_bytes, t.stream);
    t.out = nullptr;
  }
  maybe_free_output(s, t);
}

void retire(tcServer *s) {
  for (auto it = s->inflight.begin(); it != s->inflight.end();) {
    const cudaError_t q = cudaEventQuery(it->ev);
    if (q == cudaErrorNotReady) {
      ++it;
      continue;
    }
    int status = TALSH_SUCCESS;
    if (q != cudaSuccess) {
      tb::note_cuda_error("served batch", (int)q);
      cudaGetLastError();
      status = TALSH_FAILURE;
    }
    const double t = now_s();
    for (uint64_t id : it->ids) complete(s, id, status, t);
    if (it->scratch) dfree(s, it->scratch, it->scratch_bytes, it->stream);
    if (it->stage) s->stages.emplace_back(it->stage, it->stage_bytes);
    s->events.push_back(it->ev);
    it = s->inflight.erase(it);
  }
}

// Scratch bytes a large task reserves at admission.
size_t large_scratch(const STask &t, int slices) {
  const tcContractTask &x = t.spec.op;
  if (t.split)
    return tb::contract_split_scratch(x.data_kind, x.cptrn, x.drank, x.ddims, x.lrank, x.ldims, x.rrank, x.rdims,
                                      slices);
  return tb::contract_scratch_bytes(x.data_kind, x.cptrn, x.drank, x.ddims, x.lrank, x.ldims, x.rrank, x.rdims);
}

void admit(tcServer *s, int cls) {
  std::deque<uint64_t> &q = s->admit_q[cls];
  while (!q.empty()) {
    if (cls == 1 && s->large_active >= s->cfg.max_inflight + 1) return;
    const uint64_t id = q.front();
    STask &t = s->tasks[id];
    if (t.large) {
      t.split = t.spec.op.data_kind == R8 && s->cfg.r8_slices > 0 && t.spec.op.drank > 0;
      if (t.split && large_scratch(t, s->cfg.r8_slices) == 0) t.split = false;
      t.scratch_bytes = large_scratch(t, s->cfg.r8_slices);
    }
    // Admitted tasks always leave room for the batch scratch of every admitted,
    // unlaunched small task plus one batch's fixed part, so a launch never
    // waits for memory that only a later launch could free.
    const size_t resv = t.large ? 0 : round_bytes(tb::batch_task_scratch_bound(t.spec.op));
    const size_t need = (t.own_out ? round_bytes(t.out_bytes) : 0) +
                        (t.scratch_bytes ? round_bytes(t.scratch_bytes) : 0) + resv + tb::batch_fixed_scratch();
    if (need > s->cfg.budget_bytes) {
      q.pop_front();
      tb::note_error_text("served task needs more device memory than the server budget");
      complete(s, id, TALSH_LIMIT_EXCEEDED, now_s());
      continue;
    }
    if (s->used + s->reserved + need > s->cfg.budget_bytes) {
      if (!t.waited) s->stats.admission_waits++;
      t.waited = true;
      return;
    }
    if (t.own_out && dalloc(s, t.out_bytes, t.stream, &t.out) != TALSH_SUCCESS) {
      if (!t.waited) s->stats.admission_waits++;
      t.waited = true;
      return;
    }
    if (t.scratch_bytes && dalloc(s, t.scratch_bytes, t.stream, &t.scratch) != TALSH_SUCCESS) {
      if (t.own_out) {
        dfree(s, t.out, t.out_bytes, t.stream);
        t.out = nullptr;
      }
      if (!t.waited) s->stats.admission_waits++;
      t.waited = true;
      return;
    }
    if (!t.own_out) t.out = t.spec.op.D;
    t.reserve = resv;
    s->reserved += resv;
    t.state = kAdmitted;
    if (t.large) {
      t.counted = true;
      s->large_active++;
    }
    q.pop_front();
    s->waiting.push_back(id);
  }
}

// 1: launchable on `stream`, 0: not yet, -1: a producer failed.
int deps_ready(tcServer *s, const STask &t, int stream) {
  for (uint64_t p : {t.spec.l_from, t.spec.r_from}) {
    if (p == 0) continue;
    const STask &P = s->tasks[p];
    if (P.state == kDone) {
      if (P.status != TALSH_SUCCESS) return -1;
      continue;
    }
    if (P.state != kLaunched) return 0;
    if (P.stream == stream) continue;
    if (stream == 1) continue;  // the large stream waits on the producer's batch event
    return 0;
  }
  return 1;
}

tcContractTask resolve(tcServer *s, const STask &t) {
  tcContractTask x = t.spec.op;
  x.D = t.out;
  if (t.spec.l_from) x.L = s->tasks[t.spec.l_from].out;
  if (t.spec.r_from) x.R = s->tasks[t.spec.r_from].out;
  if (t.own_out) x.accumulative = 0;
  return x;
}

struct ScratchCtx {
  tcServer *s;
  void *scratch = nullptr;
  size_t scratch_bytes = 0;
  void *stage = nullptr;
  size_t stage_bytes = 0;
};

void *batch_scratch(void *ctx, size_t scratch_bytes, size_t stage_bytes, void **stage) {
  ScratchCtx &c = *(ScratchCtx *)ctx;
  void *p = nullptr;
  if (dalloc(c.s, scratch_bytes, 0, &p) != TALSH_SUCCESS) return nullptr;
  size_t got = 0;
  void *h = stage_get(c.s, std::max<size_t>(stage_bytes, 1), &got);
  if (h == nullptr) {
    dfree(c.s, p, scratch_bytes, 0);
    return nullptr;
  }
  c.scratch = p;
  c.scratch_bytes = scratch_bytes;
  c.stage = h;
  c.stage_bytes = got;
  *stage = h;
  return p;
}

int count_inflight(const tcServer *s, int stream) {
  int n = 0;
  for (const auto &b : s->inflight) n += b.stream == stream;
  return n;
}

void fail_now(tcServer *s, uint64_t id, int status) {
  s->waiting.erase(std::find(s->waiting.begin(), s->waiting.end(), id));
  complete(s, id, status, now_s());
}

void launch_batches(tcServer *s) {
  while (count_inflight(s, 0) < s->cfg.max_inflight) {
    std::vector<uint64_t> sel;
    std::vector<uint64_t> failed;
    for (uint64_t id : s->waiting) {
      const STask &t = s->tasks[id];
      if (t.large) continue;
      const int r = deps_ready(s, t, 0);
      if (r < 0) failed.push_back(id);
      if (r > 0) sel.push_back(id);
      if ((int)sel.size() >= s->cfg.max_batch) break;
    }
    for (uint64_t id : failed) fail_now(s, id, TALSH_FAILURE);
    if (sel.empty()) return;
    size_t n = sel.size();
    int rc = TRY_LATER;
    ScratchCtx ctx{s};
    std::vector<tcContractTask> ops;
    while (n > 0) {
      ops.clear();
      size_t resv = 0;
      for (size_t i = 0; i < n; ++i) {
        ops.push_back(resolve(s, s->tasks[sel[i]]));
        resv += s->tasks[sel[i]].reserve;
      }
      s->reserved -= resv;  // the reservations become this batch's scratch
      rc = tb::batch_launch_with((int)n, ops.data(), batch_scratch, &ctx, s->st[0]);
      if (rc != TRY_LATER) {
        for (size_t i = 0; i < n; ++i) s->tasks[sel[i]].reserve = 0;
        break;
      }
      s->reserved += resv;
      if (!s->inflight.empty()) break;
      n /= 2;  // nothing in flight will free memory: try a smaller batch
    }
    if (rc == TRY_LATER) {
      if (n == 0) {
        tb::note_error_text("served task's batch scratch does not fit the server budget");
        fail_now(s, sel[0], TALSH_LIMIT_EXCEEDED);
        continue;
      }
      return;
    }
    sel.resize(n);
    Inflight b;
    b.stream = 0;
    b.scratch = ctx.scratch;
    b.scratch_bytes = ctx.scratch_bytes;
    b.stage = ctx.stage;
    b.stage_bytes = ctx.stage_bytes;
    b.ev = event_get(s);
    if (rc == TALSH_SUCCESS && (b.ev == nullptr || cudaEventRecord(b.ev, s->st[0]) != cudaSuccess)) {
      cudaGetLastError();
      rc = TALSH_FAILURE;
    }
    for (uint64_t id : sel) s->waiting.erase(std::find(s->waiting.begin(), s->waiting.end(), id));
    if (rc != TALSH_SUCCESS) {
      // nothing of this batch is known to have run: release it after the stream drains
      cudaStreamSynchronize(s->st[0]);
      cudaGetLastError();
      const double t = now_s();
      for (uint64_t id : sel) complete(s, id, rc, t);
      if (b.scratch) dfree(s, b.scratch, b.scratch_bytes, 0);
      if (b.stage) s->stages.emplace_back(b.stage, b.stage_bytes);
      if (b.ev) s->events.push_back(b.ev);
      continue;
    }
    for (uint64_t id : sel) {
      STask &t = s->tasks[id];
      t.state = kLaunched;
      t.launch_ev = b.ev;
    }
    b.ids = std::move(sel);
    s->stats.batches++;
    s->stats.batched_tasks += b.ids.size();
    s->inflight.push_back(std::move(b));
  }
}

void launch_large(tcServer *s) {
  while (count_inflight(s, 1) < s->cfg.max_inflight) {
    uint64_t pick = 0;
    std::vector<uint64_t> failed;
    for (uint64_t id : s->waiting) {
      const STask &t = s->tasks[id];
      if (!t.large) continue;
      const int r = deps_ready(s, t, 1);
      if (r < 0) failed.push_back(id);
      if (r > 0) {
        pick = id;
        break;
      }
    }
    for (uint64_t id : failed) fail_now(s, id, TALSH_FAILURE);
    if (pick == 0) return;
    STask &t = s->tasks[pick];
    for (uint64_t p : {t.spec.l_from, t.spec.r_from}) {
      if (p == 0) continue;
      const STask &P = s->tasks[p];
      if (P.state == kLaunched && P.stream != 1 && P.launch_ev) cudaStreamWaitEvent(s->st[1], P.launch_ev, 0);
    }
    const tcContractTask x = resolve(s, t);
    int rc;
    if (t.split)
      rc = tb::contract_split_launch(x.data_kind, x.cptrn, x.drank, x.ddims, x.lrank, x.ldims, x.rrank, x.rdims,
                                     x.D, x.L, x.R, x.alpha_re, x.accumulative, s->cfg.r8_slices, t.scratch,
                                     t.scratch_bytes, s->st[1]);
    else
      rc = tb::contract_launch(x.data_kind, x.cptrn, x.drank, x.ddims, x.lrank, x.ldims, x.rrank, x.rdims, x.D,
                               x.L, x.R, x.alpha_re, x.alpha_im, x.conj_bits, x.accumulative, t.scratch,
                               t.scratch_bytes, s->st[1]);
    Inflight b;
    b.stream = 1;
    b.ev = event_get(s);
    if (rc == TALSH_SUCCESS && (b.ev == nullptr || cudaEventRecord(b.ev, s->st[1]) != cudaSuccess)) {
      cudaGetLastError();
      rc = TALSH_FAILURE;
    }
    s->waiting.erase(std::find(s->waiting.begin(), s->waiting.end(), pick));
    if (rc != TALSH_SUCCESS) {
      cudaStreamSynchronize(s->st[1]);
      cudaGetLastError();
      complete(s, pick, rc, now_s());
      if (b.ev) s->events.push_back(b.ev);
      continue;
    }
    t.state = kLaunched;
    t.launch_ev = b.ev;
    b.ids.push_back(pick);
    s->stats.large_tasks++;
    s->inflight.push_back(std::move(b));
  }
}

int progress_step(tcServer *s);

int progress(tcServer *s) {
  const double t0 = now_s();
  const int r = progress_step(s);
  const double dt = now_s() - t0;
  s->stats.sched_s += dt;
  s->stats.max_step_s = std::max(s->stats.max_step_s, dt);
  return r;
}

int progress_step(tcServer *s) {
  retire(s);
  admit(s, 1);
  admit(s, 0);
  launch_large(s);
  launch_batches(s);
  if (s->inflight.empty()) {
    // Nothing could be launched and nothing running can free memory for the
    // heads of the queues: the budget is held by kept outputs.
    for (auto &q : s->admit_q) {
      if (q.empty()) continue;
      const uint64_t id = q.front();
      q.pop_front();
      tb::note_error_text("served task cannot be admitted: the budget is held by kept outputs");
      complete(s, id, TALSH_LIMIT_EXCEEDED, now_s());
    }
  }
  return (int)std::min<size_t>(s->pending, 0x7fffffff);
}

int submit_at(tcServer *s, const tcServeTask *task, double t_submit, uint64_t *id) {
  const tcContractTask &x = task->op;
  const int es = tb::kind_size(x.data_kind);
  if (es == 0 || x.drank < 0 || x.lrank < 0 || x.rrank < 0 || x.drank > TC_BATCH_MAX_RANK ||
      x.lrank > TC_BATCH_MAX_RANK || x.rrank > TC_BATCH_MAX_RANK || task->consumers < 0)
    return TALSH_INVALID_ARGS;
  for (int i = 0; i < x.drank; ++i) if (x.ddims[i] <= 0) return TALSH_INVALID_ARGS;
  for (int i = 0; i < x.lrank; ++i) if (x.ldims[i] <= 0) return TALSH_INVALID_ARGS;
  for (int i = 0; i < x.rrank; ++i) if (x.rdims[i] <= 0) return TALSH_INVALID_ARGS;
  int rc = tb::contract_validate(x.data_kind, x.cptrn, x.drank, x.ddims, x.lrank, x.ldims, x.rrank, x.rdims);
  if (rc) return rc;
  // Operands taken from earlier outputs: same kind, same shape, still held.
  const int *odims[2] = {x.ldims, x.rdims};
  const int orank[2] = {x.lrank, x.rrank};
  const uint64_t from[2] = {task->l_from, task->r_from};
  for (int o = 0; o < 2; ++o) {
    if (from[o] == 0) {
      if ((o == 0 ? x.L : x.R) == nullptr) return TALSH_INVALID_ARGS;
      continue;
    }
    auto it = s->tasks.find(from[o]);
    if (it == s->tasks.end()) return TALSH_INVALID_ARGS;
    const STask &P = it->second;
    if (!P.own_out || P.spec.op.data_kind != x.data_kind || P.spec.op.drank != orank[o]) return TALSH_INVALID_ARGS;
    if (P.state == kDone && (P.out == nullptr || P.status != TALSH_SUCCESS)) return TALSH_INVALID_ARGS;
    for (int i = 0; i < orank[o]; ++i) if (P.spec.op.ddims[i] != odims[o][i]) return TALSH_INVALID_ARGS;
  }
  STask t;
  t.spec = *task;
  t.own_out = x.D == nullptr;
  t.out_bytes = t.own_out ? (size_t)vol(x.ddims, x.drank) * (size_t)es : 0;
  t.consumers_left = task->consumers;
  t.large = task_flops(x) >= s->cfg.large_flop;
  t.stream = t.large ? 1 : 0;
  t.t_submit = t_submit;
  const uint64_t nid = s->next_id++;
  for (int o = 0; o < 2; ++o)
    if (from[o]) s->tasks[from[o]].readers++;
  s->tasks.emplace(nid, t);
  s->admit_q[t.stream].push_back(nid);
  s->pending++;
  s->stats.submitted++;
  *id = nid;
  return TALSH_SUCCESS;
}

}  // namespace

extern "C" int tcServerCreate(const tcServeConfig *cfg, tcServer **srv) {
  if (srv == nullptr) return TALSH_INVALID_ARGS;
  *srv = nullptr;
  tcServeConfig c{};
  if (cfg) c = *cfg;
  if (c.r8_slices != 0 && (c.r8_slices < 2 || c.r8_slices > 7)) return TALSH_INVALID_ARGS;
  if (c.max_batch < 0 || c.max_inflight < 0 || c.large_flop < 0) return TALSH_INVALID_ARGS;
  if (c.max_batch == 0) c.max_batch = 4096;
  c.max_batch = std::min(c.max_batch, 65535);
  if (c.max_inflight == 0) c.max_inflight = 2;
  if (c.large_flop == 0) c.large_flop = 1e10;
  tcServer *s = new tcServer();
  if (cudaGetDevice(&s->dev) != cudaSuccess) {
    cudaGetLastError();
    delete s;
    return TALSH_FAILURE;
  }
  if (c.budget_bytes == 0) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      cudaGetLastError();
      delete s;
      return TALSH_FAILURE;
    }
    c.budget_bytes = (size_t)(0.9 * (double)fr);
  }
  s->cfg = c;
  // A pool of its own whose freed blocks stay mapped (release threshold =
  // budget): admissions after a burst reuse memory instead of mapping new
  // pages on the scheduling thread.
  cudaMemPoolProps props;
  std::memset(&props, 0, sizeof(props));
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = s->dev;
  uint64_t keep = (uint64_t)c.budget_bytes;
  if (cudaMemPoolCreate(&s->pool, &props) != cudaSuccess ||
      cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) {
    cudaGetLastError();
    if (s->pool) cudaMemPoolDestroy(s->pool);
    delete s;
    return TALSH_FAILURE;
  }
  // The batch stream outranks the large-task stream: CTAs of a small batch are
  // dispatched ahead of the remaining CTAs of a long contraction.
  int prio_low = 0, prio_high = 0;
  if (cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high) != cudaSuccess) {
    cudaGetLastError();
    prio_low = prio_high = 0;
  }
  for (int i = 0; i < 2; ++i) {
    if (cudaStreamCreateWithPriority(&s->st[i], cudaStreamNonBlocking, i == 0 ? prio_high : prio_low) !=
        cudaSuccess) {
      cudaGetLastError();
      if (s->st[0]) cudaStreamDestroy(s->st[0]);
      cudaMemPoolDestroy(s->pool);
      delete s;
      return TALSH_FAILURE;
    }
  }
  if (c.prealloc_bytes > 0) {
    // Map the pool's first pages now: one allocation, freed at once, stays in
    // the pool (release threshold = budget).
    void *p = nullptr;
    const size_t b = std::min(c.prealloc_bytes, c.budget_bytes);
    if (cudaMallocFromPoolAsync(&p, b, s->pool, s->st[0]) == cudaSuccess) {
      cudaFreeAsync(p, s->st[0]);
      cudaStreamSynchronize(s->st[0]);
    }
    cudaGetLastError();
  }
  *srv = s;
  return TALSH_SUCCESS;
}

extern "C" int tcServerSubmit(tcServer *srv, const tcServeTask *task, uint64_t *id) {
  if (srv == nullptr || task == nullptr || id == nullptr) return TALSH_INVALID_ARGS;
  cudaSetDevice(srv->dev);
  return submit_at(srv, task, now_s(), id);
}

extern "C" int tcServerProgress(tcServer *srv) {
  if (srv == nullptr) return TALSH_INVALID_ARGS;
  cudaSetDevice(srv->dev);
  return progress(srv);
}

extern "C" int tcServerPoll(tcServer *srv, int max, uint64_t *ids, double *latency_s, int *status) {
  if (srv == nullptr || max < 0) return TALSH_INVALID_ARGS;
  int n = 0;
  while (n < max && !srv->done.empty()) {
    const DoneRec d = srv->done.front();
    srv->done.pop_front();
    if (ids) ids[n] = d.id;
    if (latency_s) latency_s[n] = d.latency;
    if (status) status[n] = d.status;
    ++n;
    // Forget a task nothing can refer to any more: no pending or declared
    // consumer and no output held for the caller.
    auto it = srv->tasks.find(d.id);
    if (it != srv->tasks.end()) {
      const STask &t = it->second;
      if (t.readers <= 0 && t.consumers_left <= 0 && (!t.own_out || t.out == nullptr)) srv->tasks.erase(it);
    }
  }
  return n;
}

extern "C" int tcServerDrain(tcServer *srv) {
  if (srv == nullptr) return TALSH_INVALID_ARGS;
  cudaSetDevice(srv->dev);
  while (progress(srv) > 0) {
  }
  return TALSH_SUCCESS;
}

extern "C" int tcServerOutput(tcServer *srv, uint64_t id, void **ptr) {
  if (srv == nullptr || ptr == nullptr) return TALSH_INVALID_ARGS;
  auto it = srv->tasks.find(id);
  if (it == srv->tasks.end() || it->second.state != kDone) return TALSH_INVALID_ARGS;
  if (it->second.status != TALSH_SUCCESS) return it->second.status;
  if (it->second.out == nullptr) return TALSH_INVALID_ARGS;
  *ptr = it->second.out;
  return TALSH_SUCCESS;
}

extern "C" int tcServerRelease(tcServer *srv, uint64_t id) {
  if (srv == nullptr) return TALSH_INVALID_ARGS;
  auto it = srv->tasks.find(id);
  if (it == srv->tasks.end()) return TALSH_INVALID_ARGS;
  cudaSetDevice(srv->dev);
  it->second.released = true;
  maybe_free_output(srv, it->second);
  return TALSH_SUCCESS;
}

extern "C" int tcServerGetStats(tcServer *srv, tcServeStats *stats) {
  if (srv == nullptr || stats == nullptr) return TALSH_INVALID_ARGS;
  *stats = srv->stats;
  stats->bytes_in_use = srv->used;
  stats->bytes_peak = srv->peak;
  stats->budget_bytes = srv->cfg.budget_bytes;
  return TALSH_SUCCESS;
}

extern "C" int tcServerResetStats(tcServer *srv) {
  if (srv == nullptr) return TALSH_INVALID_ARGS;
  srv->stats = tcServeStats{};
  srv->peak = srv->used;
  return TALSH_SUCCESS;
}

extern "C" int tcServerReplay(tcServer *srv, int n, const tcServeTask *tasks, const double *arrival_s,
                              uint64_t *ids, double *latency_s) {
  if (srv == nullptr || n < 0 || (n > 0 && (tasks == nullptr || arrival_s == nullptr))) return TALSH_INVALID_ARGS;
  for (int i = 1; i < n; ++i)
    if (arrival_s[i] < arrival_s[i - 1]) return TALSH_INVALID_ARGS;
  cudaSetDevice(srv->dev);
  std::vector<uint64_t> id_of(n, 0);
  std::unordered_map<uint64_t, int> index_of;
  int first_err = TALSH_SUCCESS;
  std::vector<DoneRec> keep;  // completions of tasks submitted before this call
  const double t0 = now_s();
  int i = 0, left = n;
  std::vector<uint64_t> pid(256);
  std::vector<double> plat(256);
  std::vector<int> pst(256);
  while (i < n || left > 0) {
    const double t = now_s() - t0;
    while (i < n && arrival_s[i] <= t) {
      tcServeTask x = tasks[i];
      int rc = TALSH_SUCCESS;
      for (uint64_t *f : {&x.l_from, &x.r_from}) {
        if (*f == 0) continue;
        if (*f > (uint64_t)i || id_of[*f - 1] == 0) rc = TALSH_INVALID_ARGS; else *f = id_of[*f - 1];
      }
      uint64_t id = 0;
      if (rc == TALSH_SUCCESS) rc = submit_at(srv, &x, t0 + arrival_s[i], &id);
      if (rc != TALSH_SUCCESS) {
        if (first_err == TALSH_SUCCESS) first_err = rc;
        if (latency_s) latency_s[i] = -1.0;
        --left;
      } else {
        id_of[i] = id;
        index_of[id] = i;
      }
      if (ids) ids[i] = id;
      ++i;
    }
    progress(srv);
    int got;
    while ((got = tcServerPoll(srv, 256, pid.data(), plat.data(), pst.data())) > 0) {
      for (int j = 0; j < got; ++j) {
        auto it = index_of.find(pid[j]);
        if (it == index_of.end()) {
          keep.push_back(DoneRec{pid[j], plat[j], pst[j]});
          continue;
        }
        if (latency_s) latency_s[it->second] = plat[j];
        if (pst[j] != TALSH_SUCCESS && first_err == TALSH_SUCCESS) first_err = pst[j];
        --left;
      }
    }
  }
  for (auto it = keep.rbegin(); it != keep.rend(); ++it) srv->done.push_front(*it);
  return first_err;
}

extern "C" int tcServerDestroy(tcServer *srv) {
  if (srv == nullptr) return TALSH_INVALID_ARGS;
  cudaSetDevice(srv->dev);
  for (int i = 0; i < 2; ++i) cudaStreamSynchronize(srv->st[i]);
  cudaGetLastError();
  for (auto &b : srv->inflight) {
    if (b.scratch) cudaFreeAsync(b.scratch, srv->st[b.stream]);
    if (b.stage) cudaFreeHost(b.stage);
    if (b.ev) cudaEventDestroy(b.ev);
  }
  for (auto &kv : srv->tasks) {
    STask &t = kv.second;
    if (t.own_out && t.out) cudaFreeAsync(t.out, srv->st[t.stream]);
    if (t.scratch) cudaFreeAsync(t.scratch, srv->st[t.stream]);
  }
  for (int i = 0; i < 2; ++i) cudaStreamSynchronize(srv->st[i]);
  for (auto &p : srv->stages) cudaFreeHost(p.first);
  for (auto e : srv->events) cudaEventDestroy(e);
  for (int i = 0; i < 2; ++i) cudaStreamDestroy(srv->st[i]);
  cudaMemPoolDestroy(srv->pool);
  cudaGetLastError();
  delete srv;
  return TALSH_SUCCESS;
}
