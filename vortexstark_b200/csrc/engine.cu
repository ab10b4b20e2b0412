// Batched and served execution: a pool of slots (host worker thread + CUDA
// streams) over an engine-wide pool of cached device workspaces (batched and
// graph-captured Fibonacci provers, column-commitment buffers).
//
// Jobs wait in one FIFO. A free slot takes the head job (under the size-priority
// policy a quarter of the slots take only small jobs, oldest first) together with
// the queued Fibonacci jobs of the same trace size, up to the batch capacity of
// that size, and runs them as one batched proof (one graph launch, one kernel per
// stage for all of them). It needs a workspace of the job's shape (for a batch,
// one that holds at least its proofs): an idle cached one, or a new one (a batch's
// sized to the batch) when the device memory the engine holds stays within the HBM
// budget. The held memory is every cached workspace, idle or in use, plus the
// library's twiddle tables on the device (and the tables the new shape would
// build). When a new workspace does not fit, idle workspaces of other shapes are
// freed, least recently used first; when it still does not fit the job waits for
// running jobs, and a job that cannot fit even on an idle engine fails with
// VS_ERR_BUDGET. So jobs that arrive while others run are admitted as slots and
// memory free up, their work overlaps on the device, and the engine never holds
// more device memory than the budget. Each job's result depends only on the job
// (never on its batch or on what ran beside it).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "batch_prover.h"
#include "merkle.h"
#include "ntt.h"
#include "prover.h"
#include "prover_graph.h"
#include "twiddles.h"
#include "vs_common.cuh"

namespace vs {

namespace {

using Clock = std::chrono::steady_clock;

// Commitment workspaces hold at least kCommitCols columns (wider jobs get their own).
constexpr uint32_t kCommitCols = 34;

uint64_t align256(uint64_t b) { return (b + 255) & ~255ull; }
uint64_t round2m(uint64_t b) { return (b + (2ull << 20) - 1) & ~((2ull << 20) - 1); }

// One device allocation: columns, LDE, root and Merkle scratch.
struct CommitWs {
  uint8_t* mem = nullptr;
  uint32_t *cols = nullptr, *lde = nullptr, *root = nullptr, *scratch = nullptr, *h_root = nullptr;
  ~CommitWs() {
    if (mem) cudaFree(mem);
    if (h_root) cudaFreeHost(h_root);
  }
};
uint64_t commit_layout(uint32_t log_n, uint32_t capacity, CommitWs* w) {
  const uint64_t n = 1ull << log_n, N = n << 2;
  uint64_t off = 0;
  auto take = [&](uint64_t bytes) -> uint32_t* {
    uint32_t* p = w && w->mem ? (uint32_t*)(w->mem + off) : nullptr;
    off += align256(bytes);
    return p;
  };
  uint32_t* cols = take((uint64_t)capacity * n * 4);
  uint32_t* lde = take((uint64_t)capacity * N * 4);
  uint32_t* root = take(32);
  uint32_t* scratch = take(std::max<uint64_t>(merkle_scratch_words_any(N), 8) * 4);
  if (w) { w->cols = cols; w->lde = lde; w->root = root; w->scratch = scratch; }
  return off;
}

// Workspace shapes.
enum { WS_BATCH = 0, WS_GRAPH = 1, WS_COMMIT = 2 };
uint64_t ws_key(uint32_t kind, uint32_t log_n, uint32_t capacity) {
  return ((uint64_t)kind << 48) | ((uint64_t)log_n << 32) | capacity;
}

struct Ws {
  uint64_t key = 0, bytes = 0, last_use = 0;
  std::unique_ptr<BatchProver> batch;
  std::unique_ptr<GraphProver> graph;
  std::unique_ptr<CommitWs> commit;
};

// Per-job working set, used only to pick a job's stream priority and whether a
// small-only slot may take it (unchanged by batching).
uint64_t class_bytes(const vs_job& j) {
  const uint64_t n = 1ull << j.log_n, N = n << 2;
  if (j.kind == VS_JOB_COMMIT) return (uint64_t)j.n_cols * (n + N) * 4 + merkle_scratch_words_any(N) * 4 + 64;
  return n * 4 + N * 4 * 3 + N * 16 + (16u << 20) +
         merkle_tile_scratch_bytes(N, N >= (1ull << 20) ? MK_TILE_SPLIT_MAX : 0u);
}

// Jobs run at one of three stream priorities by working-set size (small jobs
// first), so a small proof admitted beside large ones is not stuck behind their
// queued kernels. Priority changes only scheduling, never a result.
constexpr int kPrioLevels = 3;
int prio_level(uint64_t job_bytes) {
  return job_bytes <= (64ull << 20) ? 0 : (job_bytes <= (512ull << 20) ? 1 : 2);
}

struct Slot {
  int device = 0;
  bool small_only = false;  // takes only jobs of priority level 0
  cudaStream_t st[kPrioLevels] = {};
  std::thread th;
};

struct Result {
  vs_job job{};
  int status = VS_OK;
  std::vector<uint8_t> bytes;
  double t_submit = 0, t_start = 0, t_end = 0;
  bool done = false, running = false;
  std::string error;
};

// What a slot will run next: the tickets of one job or batch and how it gets its workspace.
struct Plan {
  std::vector<std::deque<uint64_t>::iterator> picks;  // queue positions, oldest first
  uint64_t key = 0, need = 0;
  size_t idle_at = SIZE_MAX;  // index of an idle workspace of this shape
  bool reject = false;        // cannot fit the budget even on an idle engine
};

}  // namespace

struct Engine {
  int device = 0;
  int prio_greatest = 0, prio_least = 0;  // CUDA stream priority range (greatest is numerically lowest)
  bool by_size = true;                     // false: every job at the least priority
  uint64_t budget = 0, next_ticket = 1;
  uint32_t batch_limit = 0;  // 0: BatchProver::default_capacity; 1: no batching
  Clock::time_point t0 = Clock::now();
  std::vector<std::unique_ptr<Slot>> slots;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<uint64_t> queue;
  std::map<uint64_t, Result> results;
  bool stop = false;
  uint64_t in_flight = 0;
  // workspace pool (all under mu)
  std::vector<std::unique_ptr<Ws>> idle;
  uint64_t resident = 0, peak_held = 0, evictions = 0, use_clock = 0, created = 0;
  uint32_t busy = 0, running_jobs = 0, inject_oom = 0;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
  int priority(int level) const {  // level 0 -> greatest priority, last level -> least
    return prio_greatest + (prio_least - prio_greatest) * level / (kPrioLevels - 1);
  }
  int level_of(const vs_job& j) const { return by_size ? prio_level(class_bytes(j)) : kPrioLevels - 1; }

  // Jobs per batch at a trace size: the default capacity (or the set limit), halved
  // until the workspace fits the budget, so a small budget gets smaller batches
  // instead of refused jobs.
  uint32_t batch_capacity(uint32_t log_n) const {
    uint32_t c = BatchProver::default_capacity(log_n);
    if (batch_limit) c = std::min(c, batch_limit);
    while (c > 1 && round2m(BatchProver::bytes_for(log_n, c)) > budget) c = (c + 1) / 2;
    return c;
  }
  bool batched(const vs_job& j) const { return j.kind == VS_JOB_FIB && j.log_n >= 4 && j.log_n <= BATCH_MAX_LOG_N; }

  // Workspace shape of a job and its device bytes.
  uint64_t key_of(const vs_job& j) const {
    if (j.kind == VS_JOB_COMMIT) return ws_key(WS_COMMIT, j.log_n, std::max(kCommitCols, j.n_cols));
    if (batched(j)) return ws_key(WS_BATCH, j.log_n, batch_capacity(j.log_n));
    return ws_key(WS_GRAPH, j.log_n, 1);
  }
  static uint64_t bytes_of(uint64_t key) {
    const uint32_t kind = (uint32_t)(key >> 48), log_n = (uint32_t)(key >> 32) & 0xFFFF, cap = (uint32_t)key;
    if (kind == WS_COMMIT) return round2m(commit_layout(log_n, cap, nullptr));
    if (kind == WS_BATCH) return round2m(BatchProver::bytes_for(log_n, cap));
    return GraphProver::bytes_estimate(log_n);
  }
  // Twiddle tables a new workspace of this shape would build on the device.
  uint64_t twiddles_needed(uint64_t key) const {
    const uint32_t kind = (uint32_t)(key >> 48), log_n = (uint32_t)(key >> 32) & 0xFFFF;
    if (kind == WS_COMMIT)
      return twiddle_bytes_if_missing(device, TW_STWO, log_n) + twiddle_bytes_if_missing(device, TW_STWO, log_n + 2);
    const uint32_t le = log_n + BLOWUP_BITS;
    uint64_t b = twiddle_bytes_if_missing(device, TW_NATIVE, log_n) + twiddle_bytes_if_missing(device, TW_NATIVE, le);
    for (uint32_t l = 0; l + LOG_LAST_LAYER < le; l++)
      b += twiddle_bytes_if_missing(device, 16 + (l == 0 ? COSET_HALF_COSET : COSET_HALF_ODDS), le - l);
    return b;
  }
  uint64_t held_with(uint64_t extra) const { return resident + twiddle_cache_bytes(device) + extra; }

  // Picks the next job (and its batch) this slot may run, and how it gets its workspace.
  bool choose(const Slot& s, Plan& p) {
    auto head = queue.end();
    if (s.small_only) {  // the oldest small job, wherever it is in the queue
      for (auto it = queue.begin(); it != queue.end(); ++it)
        if (prio_level(class_bytes(results[*it].job)) == 0) { head = it; break; }
    } else if (!queue.empty()) {
      head = queue.begin();
    }
    if (head == queue.end()) return false;
    const vs_job& j = results[*head].job;
    p = Plan{};
    p.key = key_of(j);
    p.picks.push_back(head);
    if (batched(j)) {
      // queued jobs of this size are shared among the slots that are free now
      // (concurrent batches keep the GPU busier than one large batch and a wait)
      uint32_t same = 0;
      for (auto it = head; it != queue.end(); ++it) {
        const vs_job& o = results[*it].job;
        same += o.kind == j.kind && o.log_n == j.log_n;
      }
      const uint32_t free_slots = std::max<uint32_t>(1, (uint32_t)slots.size() - busy);
      const uint32_t cap = std::min(batch_capacity(j.log_n), (same + free_slots - 1) / free_slots);
      for (auto it = std::next(head); it != queue.end() && p.picks.size() < cap; ++it) {
        const vs_job& o = results[*it].job;
        if (o.kind == j.kind && o.log_n == j.log_n &&
            (!s.small_only || prio_level(class_bytes(o)) == 0))
          p.picks.push_back(it);
      }
      // The batch runs in the smallest idle workspace of its size that holds it,
      // else in a new one sized to the batch (the next power of two, up to the
      // capacity), so slots that share a burst of small proofs do not each hold a
      // full-capacity workspace: 16 slots running batches of 4 log_n 16 proofs hold
      // 16 x 53 MB instead of 16 x 0.85 GB (throughput the same within run-to-run
      // noise, 8.9-9.4 k proofs/s). Prepared workspaces (full capacity) serve
      // every batch size.
      const uint32_t n_picks = (uint32_t)p.picks.size();
      size_t best = SIZE_MAX;
      for (size_t i = 0; i < idle.size(); i++) {
        const uint64_t k = idle[i]->key;
        if ((k >> 32) != (p.key >> 32) || (uint32_t)k < n_picks) continue;
        if (best == SIZE_MAX || (uint32_t)k < (uint32_t)idle[best]->key) best = i;
      }
      if (best != SIZE_MAX) {
        p.key = idle[best]->key;
        p.idle_at = best;
        return true;
      }
      uint32_t want = 1;
      while (want < n_picks) want <<= 1;
      p.key = ws_key(WS_BATCH, j.log_n, std::min(batch_capacity(j.log_n), want));
    }
    for (size_t i = 0; i < idle.size(); i++)
      if (idle[i]->key == p.key) { p.idle_at = i; return true; }
    p.need = bytes_of(p.key) + twiddles_needed(p.key);
    if (held_with(p.need) <= budget) return true;
    uint64_t evictable = 0;
    for (auto& w : idle) evictable += w->bytes;
    if (held_with(p.need) - evictable <= budget) return true;
    if (busy == 0) { p.reject = true; return true; }
    return false;  // wait for running jobs to release memory
  }

  // Frees idle workspaces, least recently used first, until `need` more bytes fit.
  void evict_for(uint64_t need) {
    while (held_with(need) > budget && !idle.empty()) {
      auto lru = std::min_element(idle.begin(), idle.end(),
                                  [](const std::unique_ptr<Ws>& a, const std::unique_ptr<Ws>& b) {
                                    return a->last_use < b->last_use;
                                  });
      resident -= (*lru)->bytes;
      idle.erase(lru);  // frees its device memory (synchronises its own work first)
      evictions++;
    }
  }

  int create(uint64_t key, int level, cudaStream_t st, std::unique_ptr<Ws>& out) {
    const uint32_t kind = (uint32_t)(key >> 48), log_n = (uint32_t)(key >> 32) & 0xFFFF, cap = (uint32_t)key;
    auto w = std::make_unique<Ws>();
    w->key = key;
    w->bytes = bytes_of(key);
    if (kind == WS_BATCH) {
      w->batch = std::make_unique<BatchProver>();
      VS_TRY(w->batch->init(log_n, cap));
    } else if (kind == WS_GRAPH) {
      w->graph = std::make_unique<GraphProver>();
      VS_TRY(w->graph->init(log_n, priority(level)));
    } else {
      auto c = std::make_unique<CommitWs>();
      cudaError_t e = cudaMalloc((void**)&c->mem, commit_layout(log_n, cap, nullptr));
      if (e != cudaSuccess) {
        c->mem = nullptr;
        return set_error(VS_ERR_OOM, "commit workspace: %s", cudaGetErrorString(e));
      }
      commit_layout(log_n, cap, c.get());
      VS_CUDA(cudaMallocHost((void**)&c->h_root, 32));
      const TwiddleSet* t = nullptr;
      VS_TRY(get_twiddles(TW_STWO, log_n, &t, st));
      VS_TRY(get_twiddles(TW_STWO, log_n + 2, &t, st));
      w->commit = std::move(c);
    }
    out = std::move(w);
    return VS_OK;
  }

  int run(Slot& s, Ws& w, const std::vector<vs_job>& jobs, std::vector<std::vector<uint8_t>>& outs) {
    const vs_job& j = jobs[0];
    cudaStream_t st = s.st[level_of(j)];
    outs.resize(jobs.size());
    if (w.batch) {
      std::vector<uint32_t> ab;
      for (const vs_job& x : jobs) { ab.push_back(x.a); ab.push_back(x.b); }
      VS_TRY(w.batch->launch(ab.data(), (uint32_t)jobs.size(), st));
      return w.batch->finish(outs);
    }
    if (w.graph) {
      VS_TRY(w.graph->launch(j.a, j.b, st));
      return w.graph->finish(j.a, j.b, outs[0]);
    }
    CommitWs& c = *w.commit;
    const uint64_t n = 1ull << j.log_n, N = n << 2;
    VS_TRY(vs_fill_uniform_m31(c.cols, (uint64_t)j.n_cols * n, j.seed, 0, (vs_stream_t)st));
    VS_TRY(lde_cached(TW_STWO, c.cols, n, c.lde, N, j.n_cols, j.log_n, 2, st));
    VS_TRY(merkle_root(LeafRowPacked{c.lde, N, j.n_cols}, N, c.root, st, c.scratch, merkle_split()));
    VS_CUDA(cudaMemcpyAsync(c.h_root, c.root, 32, cudaMemcpyDeviceToHost, st));
    VS_CUDA(cudaStreamSynchronize(st));
    outs[0].assign((uint8_t*)c.h_root, (uint8_t*)c.h_root + 32);
    return VS_OK;
  }

  static bool valid(const vs_job& j) {
    if (j.kind == VS_JOB_FIB) return j.log_n >= 4 && j.log_n + BLOWUP_BITS <= 30;
    return j.kind == VS_JOB_COMMIT && j.n_cols > 0 && j.log_n >= 2 && j.log_n + 2 <= 30;
  }

  void finish_ticket(uint64_t t, int rc, const std::string& err, std::vector<uint8_t>&& bytes) {
    Result& r = results[t];
    r.status = rc;
    r.error = err;
    r.bytes = std::move(bytes);
    r.t_end = now();
    r.done = true;
    r.running = false;
    in_flight--;
  }

  void worker(Slot* s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
      if (stop) return;
      Plan p;
      if (!choose(*s, p)) {
        cv_work.wait(lk);
        continue;
      }
      std::vector<uint64_t> tickets;
      std::vector<vs_job> jobs;
      for (auto it : p.picks) { tickets.push_back(*it); jobs.push_back(results[*it].job); }
      queue.erase(std::remove_if(queue.begin(), queue.end(),
                                 [&](uint64_t t) { return std::find(tickets.begin(), tickets.end(), t) != tickets.end(); }),
                  queue.end());
      if (p.reject) {
        for (uint64_t t : tickets)
          finish_ticket(t, VS_ERR_BUDGET, "job workspace does not fit the HBM budget", {});
        cv_done.notify_all();
        continue;
      }
      const double t_start = now();
      for (uint64_t t : tickets) { results[t].t_start = t_start; results[t].running = true; }
      std::unique_ptr<Ws> ws;
      bool fresh = false, inject = false;
      if (p.idle_at != SIZE_MAX) {
        ws = std::move(idle[p.idle_at]);
        idle.erase(idle.begin() + p.idle_at);
      } else {
        evict_for(p.need);
        const uint64_t bytes = bytes_of(p.key);
        resident += bytes;
        peak_held = std::max(peak_held, held_with(p.need - bytes));
        fresh = true;
        if (inject_oom) { inject_oom--; inject = true; }
      }
      busy++;
      running_jobs += (uint32_t)jobs.size();
      lk.unlock();

      clear_error();
      const int level = level_of(jobs[0]);
      int rc = VS_OK;
      for (const vs_job& j : jobs)
        if (rc == VS_OK && !valid(j)) rc = set_error(VS_ERR_INVALID, "bad job");
      if (rc == VS_OK && fresh) rc = inject ? set_error(VS_ERR_OOM, "injected workspace allocation failure")
                                            : create(p.key, level, s->st[level], ws);
      std::vector<std::vector<uint8_t>> outs;
      if (rc == VS_OK) rc = run(*s, *ws, jobs, outs);
      const std::string err = rc == VS_OK ? "" : vs_last_error();
      if (rc != VS_OK) ws.reset();  // a workspace that failed is not reused

      lk.lock();
      busy--;
      running_jobs -= (uint32_t)jobs.size();
      if (ws) {
        ws->last_use = ++use_clock;
        if (fresh) created++;
        idle.push_back(std::move(ws));
      } else if (fresh || p.idle_at != SIZE_MAX) {
        resident -= bytes_of(p.key);
      }
      for (size_t i = 0; i < tickets.size(); i++)
        finish_ticket(tickets[i], rc, err, rc == VS_OK ? std::move(outs[i]) : std::vector<uint8_t>());
      cv_done.notify_all();
      cv_work.notify_all();
    }
  }

  // Builds up to `count` idle workspaces of a job's shape that fit the budget
  // without evicting anything (workers must be idle).
  int prepare(const vs_job& shape, uint32_t count) {
    const uint64_t key = key_of(shape);
    uint32_t have = 0;
    for (auto& w : idle) have += w->key == key;
    for (; have < count; have++) {
      const uint64_t need = bytes_of(key) + twiddles_needed(key);
      if (held_with(need) > budget) break;
      std::unique_ptr<Ws> w;
      VS_TRY(create(key, level_of(shape), slots[0]->st[level_of(shape)], w));
      resident += w->bytes;
      peak_held = std::max(peak_held, held_with(0));
      w->last_use = ++use_clock;
      created++;
      idle.push_back(std::move(w));
    }
    return VS_OK;
  }
};

}  // namespace vs

using namespace vs;

extern "C" {

int vs_engine_create(uint32_t n_slots, uint64_t hbm_budget_bytes, void** out) {
  return vs_engine_create_ex(n_slots, hbm_budget_bytes, 0, out);
}

int vs_engine_create_ex(uint32_t n_slots, uint64_t hbm_budget_bytes, uint32_t flags, void** out) {
  clear_error();
  if (!out || n_slots == 0 || n_slots > 64) return set_error(VS_ERR_INVALID, "vs_engine_create: 1..64 slots");
  if (flags & ~VS_ENGINE_FIFO_PRIORITY) return set_error(VS_ERR_INVALID, "vs_engine_create_ex: unknown flags %#x", flags);
  auto* e = new Engine();
  e->by_size = !(flags & VS_ENGINE_FIFO_PRIORITY);
  VS_CUDA(cudaGetDevice(&e->device));
  VS_CUDA(cudaDeviceGetStreamPriorityRange(&e->prio_least, &e->prio_greatest));
  e->budget = hbm_budget_bytes ? hbm_budget_bytes : ~0ull;
  for (uint32_t i = 0; i < n_slots; i++) {
    auto s = std::make_unique<Slot>();
    s->device = e->device;
    for (int l = 0; l < kPrioLevels; l++) {
      if (cudaStreamCreateWithPriority(&s->st[l], cudaStreamNonBlocking, e->priority(l)) != cudaSuccess) {
        for (auto& o : e->slots)
          for (cudaStream_t x : o->st) if (x) cudaStreamDestroy(x);
        for (cudaStream_t x : s->st) if (x) cudaStreamDestroy(x);
        delete e;
        return set_error(VS_ERR_CUDA, "vs_engine_create: stream");
      }
    }
    e->slots.push_back(std::move(s));
  }
  // With size priorities, a quarter of the slots (from 4 slots up) take only
  // small jobs, so a small job never queues behind large ones for a slot.
  if (e->by_size)
    for (uint32_t i = n_slots - n_slots / 4; i < n_slots; i++) e->slots[i]->small_only = true;
  for (auto& s : e->slots) s->th = std::thread(&Engine::worker, e, s.get());
  *out = e;
  return VS_OK;
}

int vs_engine_destroy(void* h) {
  auto* e = static_cast<Engine*>(h);
  if (!e) return VS_OK;
  {
    std::lock_guard<std::mutex> lk(e->mu);
    e->stop = true;
  }
  e->cv_work.notify_all();
  for (auto& s : e->slots) {
    if (s->th.joinable()) s->th.join();
  }
  e->idle.clear();
  for (auto& s : e->slots)
    for (cudaStream_t x : s->st)
      if (x) cudaStreamDestroy(x);
  delete e;
  return VS_OK;
}

int vs_engine_prepare(void* h, const vs_job* shape) {
  clear_error();
  auto* e = static_cast<Engine*>(h);
  if (!e || !shape) return set_error(VS_ERR_INVALID, "vs_engine_prepare: null");
  if (!Engine::valid(*shape)) return set_error(VS_ERR_INVALID, "vs_engine_prepare: bad job shape");
  std::lock_guard<std::mutex> lk(e->mu);  // workers idle on the queue; preparation is not concurrent with jobs
  uint32_t eligible = 0;
  for (auto& s : e->slots) eligible += !(s->small_only && prio_level(class_bytes(*shape)) != 0);
  VS_TRY(e->prepare(*shape, eligible));
  VS_CUDA(cudaDeviceSynchronize());
  return VS_OK;
}

int vs_engine_submit(void* h, const vs_job* job, uint64_t* ticket) {
  clear_error();
  auto* e = static_cast<Engine*>(h);
  if (!e || !job || !ticket) return set_error(VS_ERR_INVALID, "vs_engine_submit: null");
  if (job->kind != VS_JOB_FIB && job->kind != VS_JOB_COMMIT) return set_error(VS_ERR_INVALID, "unknown job kind");
  {
    std::lock_guard<std::mutex> lk(e->mu);
    const uint64_t t = e->next_ticket++;
    Result& r = e->results[t];
    r.job = *job;
    r.t_submit = e->now();
    e->queue.push_back(t);
    e->in_flight++;
    *ticket = t;
  }
  e->cv_work.notify_all();  // slots differ in what they may take: wake them all
  return VS_OK;
}

int vs_engine_submit_many(void* h, const vs_job* jobs, uint32_t n, uint64_t* tickets) {
  clear_error();
  auto* e = static_cast<Engine*>(h);
  if (!e || (n && (!jobs || !tickets))) return set_error(VS_ERR_INVALID, "vs_engine_submit_many: null");
  for (uint32_t i = 0; i < n; i++)
    if (jobs[i].kind != VS_JOB_FIB && jobs[i].kind != VS_JOB_COMMIT)
      return set_error(VS_ERR_INVALID, "unknown job kind (job %u); nothing submitted", i);
  {
    std::lock_guard<std::mutex> lk(e->mu);
    const double t = e->now();
    for (uint32_t i = 0; i < n; i++) {
      const uint64_t tk = e->next_ticket++;
      Result& r = e->results[tk];
      r.job = jobs[i];
      r.t_submit = t;
      e->queue.push_back(tk);
      e->in_flight++;
      tickets[i] = tk;
    }
  }
  e->cv_work.notify_all();
  return VS_OK;
}

int vs_engine_wait_for(void* h, uint64_t ticket, double timeout_s, vs_job_result* res, uint8_t* out, uint64_t cap) {
  clear_error();
  auto* e = static_cast<Engine*>(h);
  if (!e || !res) return set_error(VS_ERR_INVALID, "vs_engine_wait: null");
  std::unique_lock<std::mutex> lk(e->mu);
  auto it = e->results.find(ticket);
  if (it == e->results.end()) return set_error(VS_ERR_INVALID, "unknown ticket %llu", (unsigned long long)ticket);
  if (timeout_s < 0 || timeout_s > 1e6) {  // no limit (longer limits would overflow the clock's range)
    e->cv_done.wait(lk, [&] { return it->second.done; });
  } else if (!e->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] { return it->second.done; })) {
    return set_error(VS_ERR_TIMEOUT, "job %llu not finished after %.3f s", (unsigned long long)ticket, timeout_s);
  }
  Result& r = it->second;
  res->status = r.status;
  res->out_len = r.bytes.size();
  res->t_submit = r.t_submit;
  res->t_start = r.t_start;
  res->t_end = r.t_end;
  if (r.status != VS_OK) {
    const int st = r.status;
    const std::string msg = r.error;
    if (out) e->results.erase(it);  // a failed ticket is retired like a finished one
    return set_error(st, "job %llu failed: %s", (unsigned long long)ticket, msg.c_str());
  }
  if (!out) return VS_OK;  // length query; the result stays available
  if (cap < r.bytes.size()) return set_error(VS_ERR_INVALID, "result needs %zu bytes", r.bytes.size());
  std::copy(r.bytes.begin(), r.bytes.end(), out);
  e->results.erase(it);
  return VS_OK;
}

int vs_engine_wait(void* h, uint64_t ticket, vs_job_result* res, uint8_t* out, uint64_t cap) {
  return vs_engine_wait_for(h, ticket, -1.0, res, out, cap);
}

int vs_engine_cancel(void* h, uint64_t ticket) {
  clear_error();
  auto* e = static_cast<Engine*>(h);
  if (!e) return set_error(VS_ERR_INVALID, "vs_engine_cancel: null");
  {
    std::lock_guard<std::mutex> lk(e->mu);
    auto it = e->results.find(ticket);
    if (it == e->results.end()) return set_error(VS_ERR_INVALID, "unknown ticket %llu", (unsigned long long)ticket);
    if (it->second.done) return set_error(VS_ERR_BUSY, "job %llu already finished", (unsigned long long)ticket);
    auto q = std::find(e->queue.begin(), e->queue.end(), ticket);
    if (q == e->queue.end()) return set_error(VS_ERR_BUSY, "job %llu is running", (unsigned long long)ticket);
    e->queue.erase(q);
    e->finish_ticket(ticket, VS_ERR_CANCELLED, "cancelled before it started", {});
  }
  e->cv_done.notify_all();
  e->cv_work.notify_all();
  return VS_OK;
}

int vs_engine_drain(void* h) {
  auto* e = static_cast<Engine*>(h);
  if (!e) return VS_OK;
  std::unique_lock<std::mutex> lk(e->mu);
  e->cv_done.wait(lk, [&] { return e->in_flight == 0; });
  return VS_OK;
}

double vs_engine_now(void* h) {
  auto* e = static_cast<Engine*>(h);
  return e ? e->now() : 0.0;
}

int vs_engine_set_batch_limit(void* h, uint32_t max_jobs) {
  clear_error();
  auto* e = static_cast<Engine*>(h);
  if (!e) return set_error(VS_ERR_INVALID, "vs_engine_set_batch_limit: null");
  std::lock_guard<std::mutex> lk(e->mu);
  e->batch_limit = max_jobs;
  return VS_OK;
}

int vs_engine_inject_alloc_failures(void* h, uint32_t count) {
  clear_error();
  auto* e = static_cast<Engine*>(h);
  if (!e) return set_error(VS_ERR_INVALID, "vs_engine_inject_alloc_failures: null");
  std::lock_guard<std::mutex> lk(e->mu);
  e->inject_oom = count;
  return VS_OK;
}

int vs_engine_workspace_bytes(void* h, const vs_job* shape, uint64_t* bytes) {
  clear_error();
  auto* e = static_cast<Engine*>(h);
  if (!e || !shape || !bytes) return set_error(VS_ERR_INVALID, "vs_engine_workspace_bytes: null");
  if (!Engine::valid(*shape)) return set_error(VS_ERR_INVALID, "vs_engine_workspace_bytes: bad job shape");
  std::lock_guard<std::mutex> lk(e->mu);
  *bytes = Engine::bytes_of(e->key_of(*shape));
  return VS_OK;
}

int vs_engine_get_stats(void* h, vs_engine_stats* out) {
  clear_error();
  auto* e = static_cast<Engine*>(h);
  if (!e || !out) return set_error(VS_ERR_INVALID, "vs_engine_get_stats: null");
  std::lock_guard<std::mutex> lk(e->mu);
  *out = vs_engine_stats{};
  out->budget_bytes = e->budget == ~0ull ? 0 : e->budget;
  out->resident_bytes = e->resident;
  out->twiddle_bytes = twiddle_cache_bytes(e->device);
  out->peak_held_bytes = e->peak_held;
  out->evictions = e->evictions;
  out->workspaces_created = e->created;
  out->idle_workspaces = (uint32_t)e->idle.size();
  out->busy_workspaces = e->busy;
  out->queued = (uint32_t)e->queue.size();
  out->running = e->running_jobs;
  return VS_OK;
}

}  // extern "C"
