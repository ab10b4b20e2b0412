// Batched and served execution: a pool of slots, each a host worker thread with
// its own CUDA stream and cached per-shape workspaces (graph-captured Fibonacci
// provers, column-commitment buffers). Jobs wait in one FIFO; a free slot takes
// the head job only when the bytes reserved by running jobs plus the head job's
// working set fit the HBM budget, so jobs that arrive while others run are
// admitted as slots and memory free up, and their work overlaps on the device.
// Under the default size-priority policy small jobs also run on higher-priority
// streams, and a quarter of the slots take only small jobs (oldest first).
// Each job's result depends only on the job (never on what ran beside it).
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "merkle.h"
#include "ntt.h"
#include "prover_graph.h"
#include "twiddles.h"
#include "vs_common.cuh"

namespace vs {

namespace {

using Clock = std::chrono::steady_clock;

// Workspaces are cached per (kind, log_n); commitment buffers hold at least
// kCommitCols columns and grow for wider jobs.
constexpr uint32_t kCommitCols = 34;
uint64_t shape_key(const vs_job& j) { return ((uint64_t)j.kind << 32) | j.log_n; }

struct CommitWs {
  uint32_t *cols = nullptr, *lde = nullptr, *root = nullptr, *scratch = nullptr, *h_root = nullptr;
  uint64_t bytes = 0;
  uint32_t capacity = 0;  // columns
  ~CommitWs() {
    if (cols) cudaFree(cols);
    if (lde) cudaFree(lde);
    if (root) cudaFree(root);
    if (scratch) cudaFree(scratch);
    if (h_root) cudaFreeHost(h_root);
  }
};

uint64_t commit_bytes(uint32_t log_n, uint32_t n_cols) {
  const uint64_t n = 1ull << log_n, N = n << 2;
  return (uint64_t)n_cols * (n + N) * 4 + merkle_scratch_words_any(N) * 4 + 64;
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
  std::unordered_map<uint64_t, std::unique_ptr<GraphProver>> provers;
  std::unordered_map<uint64_t, std::unique_ptr<CommitWs>> commits;
  std::thread th;
};

struct Result {
  vs_job job{};
  int status = VS_OK;
  std::vector<uint8_t> bytes;
  double t_submit = 0, t_start = 0, t_end = 0;
  bool done = false;
  std::string error;
};

}  // namespace

struct Engine {
  int device = 0;
  int prio_greatest = 0, prio_least = 0;  // CUDA stream priority range (greatest is numerically lowest)
  bool by_size = true;                     // false: every job at the least priority
  uint64_t budget = 0, reserved = 0, next_ticket = 1;
  Clock::time_point t0 = Clock::now();
  std::vector<std::unique_ptr<Slot>> slots;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<uint64_t> queue;
  std::map<uint64_t, Result> results;
  bool stop = false;
  uint64_t in_flight = 0;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
  int priority(int level) const {  // level 0 -> greatest priority, last level -> least
    return prio_greatest + (prio_least - prio_greatest) * level / (kPrioLevels - 1);
  }
  int level_of(uint64_t bytes) const { return by_size ? prio_level(bytes) : kPrioLevels - 1; }

  int prover_for(Slot& s, uint32_t log_n, GraphProver** out) {
    vs_job j{};
    j.kind = VS_JOB_FIB;
    j.log_n = log_n;
    auto& p = s.provers[shape_key(j)];
    if (!p) {
      auto np = std::make_unique<GraphProver>();
      VS_TRY(np->init(log_n, priority(level_of(job_bytes(j)))));
      p = std::move(np);
    }
    *out = p.get();
    return VS_OK;
  }
  int commit_for(Slot& s, const vs_job& j, CommitWs** out) {
    auto& c = s.commits[shape_key(j)];
    if (!c || c->capacity < j.n_cols) {
      c.reset();
      auto w = std::make_unique<CommitWs>();
      const uint64_t n = 1ull << j.log_n, N = n << 2;
      w->capacity = std::max(kCommitCols, j.n_cols);
      VS_CUDA(cudaMalloc(&w->cols, (uint64_t)w->capacity * n * 4));
      VS_CUDA(cudaMalloc(&w->lde, (uint64_t)w->capacity * N * 4));
      VS_CUDA(cudaMalloc(&w->root, 32));
      VS_CUDA(cudaMalloc(&w->scratch, std::max<uint64_t>(merkle_scratch_words_any(N), 8) * 4));
      VS_CUDA(cudaMallocHost(&w->h_root, 32));
      w->bytes = commit_bytes(j.log_n, w->capacity);
      const TwiddleSet* t = nullptr;
      cudaStream_t st = s.st[level_of(commit_bytes(j.log_n, j.n_cols))];
      VS_TRY(get_twiddles(TW_STWO, j.log_n, &t, st));
      VS_TRY(get_twiddles(TW_STWO, j.log_n + 2, &t, st));
      c = std::move(w);
    }
    *out = c.get();
    return VS_OK;
  }

  uint64_t job_bytes(const vs_job& j) {
    if (j.kind == VS_JOB_COMMIT) return commit_bytes(j.log_n, j.n_cols);
    const uint64_t N = 1ull << (j.log_n + 2);
    return (1ull << j.log_n) * 4 + N * 4 * 3 + N * 16 + (16u << 20) +
           merkle_tile_scratch_bytes(N, N >= (1ull << 20) ? MK_TILE_SPLIT_MAX : 0u);
  }

  int run_job(Slot& s, const vs_job& j, std::vector<uint8_t>& out) {
    if (j.kind == VS_JOB_FIB) {
      GraphProver* p = nullptr;
      VS_TRY(prover_for(s, j.log_n, &p));
      VS_TRY(p->launch(j.a, j.b, s.st[level_of(job_bytes(j))]));
      return p->finish(j.a, j.b, out);
    }
    if (j.kind != VS_JOB_COMMIT || j.n_cols == 0 || j.log_n < 2 || j.log_n + 2 > 30)
      return set_error(VS_ERR_INVALID, "bad job");
    CommitWs* w = nullptr;
    VS_TRY(commit_for(s, j, &w));
    const uint64_t n = 1ull << j.log_n, N = n << 2;
    cudaStream_t st = s.st[level_of(commit_bytes(j.log_n, j.n_cols))];
    VS_TRY(vs_fill_uniform_m31(w->cols, (uint64_t)j.n_cols * n, j.seed, 0, (vs_stream_t)st));
    VS_TRY(lde_cached(TW_STWO, w->cols, n, w->lde, N, j.n_cols, j.log_n, 2, st));
    VS_TRY(merkle_root(LeafRowPacked{w->lde, N, j.n_cols}, N, w->root, st, w->scratch, merkle_split()));
    VS_CUDA(cudaMemcpyAsync(w->h_root, w->root, 32, cudaMemcpyDeviceToHost, st));
    VS_CUDA(cudaStreamSynchronize(st));
    out.assign((uint8_t*)w->h_root, (uint8_t*)w->h_root + 32);
    return VS_OK;
  }

  void worker(Slot* s) {
    cudaSetDevice(s->device);
    for (;;) {
      uint64_t ticket = 0;
      vs_job job{};
      uint64_t bytes = 0;
      {
        std::unique_lock<std::mutex> lk(mu);
        auto pick = queue.end();
        cv_work.wait(lk, [&] {
          if (stop) return true;
          auto fits = [&](const vs_job& j) { return reserved + job_bytes(j) <= budget || reserved == 0; };
          pick = queue.end();
          if (s->small_only) {  // the oldest small job, wherever it is in the queue
            for (auto it = queue.begin(); it != queue.end(); ++it) {
              const vs_job& j = results[*it].job;
              if (prio_level(job_bytes(j)) == 0) {
                if (fits(j)) pick = it;
                break;
              }
            }
          } else if (!queue.empty() && fits(results[queue.front()].job)) {  // FIFO; an oversized job runs alone
            pick = queue.begin();
          }
          return pick != queue.end();
        });
        if (stop) return;
        ticket = *pick;
        queue.erase(pick);
        job = results[ticket].job;
        bytes = job_bytes(job);
        reserved += bytes;
        results[ticket].t_start = now();
      }
      std::vector<uint8_t> out;
      clear_error();
      const int rc = run_job(*s, job, out);
      const std::string err = rc == VS_OK ? "" : vs_last_error();
      {
        std::lock_guard<std::mutex> lk(mu);
        Result& r = results[ticket];
        r.status = rc;
        r.error = err;
        r.bytes = std::move(out);
        r.t_end = now();
        r.done = true;
        reserved -= bytes;
        in_flight--;
      }
      cv_done.notify_all();
      cv_work.notify_all();
    }
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
  for (auto& s : e->slots) {
    s->provers.clear();
    s->commits.clear();
    for (cudaStream_t x : s->st)
      if (x) cudaStreamDestroy(x);
  }
  delete e;
  return VS_OK;
}

int vs_engine_prepare(void* h, const vs_job* shape) {
  clear_error();
  auto* e = static_cast<Engine*>(h);
  if (!e || !shape) return set_error(VS_ERR_INVALID, "vs_engine_prepare: null");
  std::lock_guard<std::mutex> lk(e->mu);  // workers idle on the queue; preparation is not concurrent with jobs
  for (auto& s : e->slots) {
    if (s->small_only && prio_level(e->job_bytes(*shape)) != 0) continue;  // never runs there
    if (shape->kind == VS_JOB_FIB) {
      GraphProver* p = nullptr;
      VS_TRY(e->prover_for(*s, shape->log_n, &p));
    } else {
      CommitWs* w = nullptr;
      VS_TRY(e->commit_for(*s, *shape, &w));
    }
  }
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

int vs_engine_wait(void* h, uint64_t ticket, vs_job_result* res, uint8_t* out, uint64_t cap) {
  clear_error();
  auto* e = static_cast<Engine*>(h);
  if (!e || !res) return set_error(VS_ERR_INVALID, "vs_engine_wait: null");
  std::unique_lock<std::mutex> lk(e->mu);
  auto it = e->results.find(ticket);
  if (it == e->results.end()) return set_error(VS_ERR_INVALID, "unknown ticket %llu", (unsigned long long)ticket);
  e->cv_done.wait(lk, [&] { return it->second.done; });
  Result& r = it->second;
  res->status = r.status;
  res->out_len = r.bytes.size();
  res->t_submit = r.t_submit;
  res->t_start = r.t_start;
  res->t_end = r.t_end;
  if (r.status != VS_OK) return set_error(r.status, "job %llu failed: %s", (unsigned long long)ticket, r.error.c_str());
  if (!out) return VS_OK;  // length query; the result stays available
  if (cap < r.bytes.size()) return set_error(VS_ERR_INVALID, "result needs %zu bytes", r.bytes.size());
  std::copy(r.bytes.begin(), r.bytes.end(), out);
  e->results.erase(it);
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

}  // extern "C"
