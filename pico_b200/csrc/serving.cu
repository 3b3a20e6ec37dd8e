// Serving path.  The reference proves chunks concurrently from a rayon pool
// (vm/src/instances/machine/riscv.rs:218-330), each chunk calling pcs.commit;
// here those commits arrive as requests.
//
// Policy:
//   - submit copies host inputs (or keeps device pointers), plans the commit
//     and queues it; nothing touches the device on the caller's thread;
//   - a dispatcher thread admits queued requests first-fit against the HBM
//     budget (LDEs + digest layers + scratch) while a stream slot is free and
//     fewer than pico_config.max_inflight requests are on the device; a
//     request that has waited longer than kStarveMs blocks later ones from
//     overtaking it, so large requests are not starved;
//   - each admitted request is enqueued whole on its own stream, so requests
//     that arrive while others run overlap with them on the device; a host
//     callback marks completion and returns the scratch budget at once;
//   - with pico_config.max_group > 1, queued batched requests of device
//     inputs and the same field join the request just admitted, up to
//     max_group members and kGroupCells trace cells, each within the budget:
//     the group runs on one stream with its LDE and row-hashing launches
//     shared (enqueue_commit_group) and its members finish together;
//   - LDEs and digest layers stay resident (and budgeted) until the caller
//     releases the commit handed over by pico_gpu_wait.
#include <chrono>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <list>

#include "serving.h"

using Clock = std::chrono::steady_clock;

struct pico_request {
  pico_ctx* ctx = nullptr;
  pico::CommitPlan plan;
  std::vector<std::vector<uint32_t>> host_copies;  // owned inputs
  enum State { QUEUED, RUNNING, DONE, FAILED, CANCELLED, TAKEN } state = QUEUED;
  pico_status status = PICO_OK;
  std::string error;
  pico_commit* commit = nullptr;
  std::vector<void*> scratch;
  uint32_t root_pinned_idx = 0;
  uint32_t* root_pinned = nullptr;  // 8 words of the slot's pinned root buffers
  uint32_t root[8] = {0};
  int slot = -1;
  uint32_t group_size = 1;  // members of the group it was admitted in
  Clock::time_point t_submit, t_admit, t_done;
};

namespace pico {

constexpr int kStarveMs = 200;
// A group takes no more members once it holds this many trace cells: a
// commit of 2^28 cells already fills the device, and a larger group would
// only delay its first member's completion.
constexpr uint64_t kGroupCells = 1ull << 28;

// Requests admitted together into one stream slot.
struct Group {
  std::vector<pico_request*> members;
  int slot = -1;
};

struct Server {
  pico_ctx* ctx;
  std::mutex mu;
  std::condition_variable cv;      // dispatcher wakeups
  std::condition_variable done_cv; // waiters
  std::list<pico_request*> queue;
  std::vector<bool> slot_busy;
  uint32_t* pinned_roots = nullptr;  // kMaxGroup 8-word roots per stream slot
  bool stop = false;
  std::thread thr;

  void run();
  bool admit(pico_request* r);
  void fill_group(Group* g, Clock::time_point now);
  bool groupable(const pico_request* r) const {
    return ctx->max_group > 1 && r->plan.input_device && r->plan.extend && !r->plan.plain && !r->plan.wide_groups;
  }
};

static void CUDART_CB on_request_done(void* arg) {
  pico_request* r = (pico_request*)arg;
  Server* sv = r->ctx->server;
  unreserve(r->ctx, r->plan.bytes_scratch);
  std::lock_guard<std::mutex> g(sv->mu);
  memcpy(r->root, r->root_pinned, 32);
  memcpy(r->commit->root, r->root_pinned, 32);
  // bounds guards (host memory only here: no CUDA calls in a stream callback;
  // the device records stay set until a synchronous call reports and clears them)
  const GuardRecord* gr = r->ctx->guard_host + 2 * r->slot;
  if (gr[0].count || gr[1].count) {
    char buf[160];
    snprintf(buf, sizeof buf, "internal bounds guard: %s kernel skipped an access (tag %llu)",
             gr[0].count ? "LDE" : "row hashing", gr[0].count ? gr[0].tag : gr[1].tag);
    r->status = PICO_ERR_CUDA;
    r->error = buf;
  }
  r->t_done = Clock::now();
  r->state = pico_request::DONE;
  sv->slot_busy[r->slot] = false;
  sv->cv.notify_all();
  sv->done_cv.notify_all();
}

// Caller holds mu.  Claims a stream slot and the request's budget; returns
// false (claiming nothing) if either is unavailable.
bool Server::admit(pico_request* r) {
  int slot = -1, busy = 0;
  for (int i = 0; i < (int)slot_busy.size(); i++) {
    if (slot_busy[i])
      busy++;
    else if (slot < 0)
      slot = i;
  }
  if (slot < 0 || busy >= (int)ctx->max_inflight) return false;
  const uint64_t need = r->plan.bytes_resident + r->plan.bytes_scratch;
  if (!try_reserve(ctx, need)) return false;
  slot_busy[slot] = true;
  r->slot = slot;
  r->state = pico_request::RUNNING;
  r->t_admit = Clock::now();
  r->root_pinned = pinned_roots + 8 * kMaxGroup * slot;
  return true;
}

// Caller holds mu.  Moves queued requests that can share the launches of
// g's first member into g, each claiming its budget; a request that has
// waited more than kStarveMs and cannot join stops the scan, so that none
// overtakes it.
void Server::fill_group(Group* g, Clock::time_point now) {
  const pico_request* first = g->members[0];
  if (!groupable(first)) return;
  uint64_t cells = first->plan.cells;
  for (auto it = queue.begin(); it != queue.end() && g->members.size() < ctx->max_group;) {
    pico_request* r = *it;
    if (groupable(r) && r->plan.field == first->plan.field && cells + r->plan.cells <= kGroupCells &&
        try_reserve(ctx, r->plan.bytes_resident + r->plan.bytes_scratch)) {
      r->slot = g->slot;
      r->state = pico_request::RUNNING;
      r->t_admit = Clock::now();
      r->root_pinned = pinned_roots + 8 * (kMaxGroup * g->slot + g->members.size());
      cells += r->plan.cells;
      g->members.push_back(r);
      it = queue.erase(it);
      continue;
    }
    const auto waited = std::chrono::duration_cast<std::chrono::milliseconds>(now - r->t_submit).count();
    if (waited > kStarveMs) break;
    ++it;
  }
}

// Completion of a group: every member done at once (host memory only, as in
// on_request_done).
static void CUDART_CB on_group_done(void* arg) {
  Group* grp = (Group*)arg;
  Server* sv = grp->members[0]->ctx->server;
  for (pico_request* r : grp->members) unreserve(r->ctx, r->plan.bytes_scratch);
  std::lock_guard<std::mutex> g(sv->mu);
  const GuardRecord* gr = sv->ctx->guard_host + 2 * grp->slot;
  const auto done = Clock::now();
  for (pico_request* r : grp->members) {
    r->group_size = (uint32_t)grp->members.size();
    memcpy(r->root, r->root_pinned, 32);
    memcpy(r->commit->root, r->root_pinned, 32);
    if (gr[0].count || gr[1].count) {
      char buf[160];
      snprintf(buf, sizeof buf, "internal bounds guard: %s kernel skipped an access (tag %llu)",
               gr[0].count ? "LDE" : "row hashing", gr[0].count ? gr[0].tag : gr[1].tag);
      r->status = PICO_ERR_CUDA;
      r->error = buf;
    }
    r->t_done = done;
    r->state = pico_request::DONE;
  }
  sv->slot_busy[grp->slot] = false;
  delete grp;
  sv->cv.notify_all();
  sv->done_cv.notify_all();
}

// Enqueue an admitted group of two or more requests on its slot's stream
// (without mu held, as launch_request).
static void launch_group(Server* sv, Group* grp) {
  pico_ctx* ctx = sv->ctx;
  cudaStream_t st = ctx->streams[grp->slot];
  std::vector<const CommitPlan*> plans;
  std::vector<pico_commit*> commits;
  std::vector<uint32_t*> roots;
  for (pico_request* r : grp->members) {
    r->commit = new pico_commit();
    plans.push_back(&r->plan);
    commits.push_back(r->commit);
    roots.push_back(r->root_pinned);
  }
  std::vector<void*> scratch;
  pico_status s = enqueue_commit_group(ctx, plans, st, commits, scratch, roots);
  for (void* p : scratch) cudaFreeAsync(p, st);
  if (s == PICO_OK) s = guard_enqueue(ctx, grp->slot, st);
  if (s == PICO_OK) s = cuda_status(cudaLaunchHostFunc(st, on_group_done, grp), "completion callback");
  if (s != PICO_OK) {
    const std::string msg = pico_gpu_last_error();
    cudaStreamSynchronize(st);
    for (pico_request* r : grp->members) free_commit_buffers(r->commit, st);
    cudaStreamSynchronize(st);
    for (pico_request* r : grp->members) {
      delete r->commit;
      r->commit = nullptr;
      unreserve(ctx, r->plan.bytes_resident + r->plan.bytes_scratch);
    }
    std::lock_guard<std::mutex> g(sv->mu);
    for (pico_request* r : grp->members) {
      r->status = s;
      r->error = msg;
      r->state = pico_request::FAILED;
    }
    sv->slot_busy[grp->slot] = false;
    delete grp;
    sv->done_cv.notify_all();
  }
}

// Enqueue an admitted request on its stream.  Called without mu held: the
// completion callback takes mu, and CUDA calls must not wait on it.
static void launch_request(Server* sv, pico_request* r) {
  pico_ctx* ctx = sv->ctx;
  cudaStream_t st = ctx->streams[r->slot];
  r->commit = new pico_commit();
  pico_status s = enqueue_commit(ctx, r->plan, st, ctx->copy_streams[r->slot], r->commit, r->scratch,
                                 r->root_pinned);
  if (s) cudaStreamSynchronize(ctx->copy_streams[r->slot]);  // copies may still target scratch
  for (void* p : r->scratch) cudaFreeAsync(p, st);
  r->scratch.clear();
  if (s == PICO_OK) s = guard_enqueue(ctx, r->slot, st);
  if (s == PICO_OK) s = cuda_status(cudaLaunchHostFunc(st, on_request_done, r), "completion callback");
  if (s != PICO_OK) {
    const std::string msg = pico_gpu_last_error();
    cudaStreamSynchronize(st);
    free_commit_buffers(r->commit, st);
    cudaStreamSynchronize(st);
    delete r->commit;
    r->commit = nullptr;
    unreserve(ctx, r->plan.bytes_resident + r->plan.bytes_scratch);
    std::lock_guard<std::mutex> g(sv->mu);
    r->status = s;
    r->error = msg;
    r->state = pico_request::FAILED;
    sv->slot_busy[r->slot] = false;
    sv->done_cv.notify_all();
  }
}

void Server::run() {
  cudaSetDevice(ctx->device);
  std::unique_lock<std::mutex> lk(mu);
  while (!stop) {
    pico_request* picked = nullptr;
    const auto now = Clock::now();
    for (auto it = queue.begin(); it != queue.end(); ++it) {
      pico_request* r = *it;
      if (admit(r)) {
        picked = r;
        queue.erase(it);
        break;
      }
      // a request that has waited long enough stops later ones overtaking it
      const auto waited = std::chrono::duration_cast<std::chrono::milliseconds>(now - r->t_submit).count();
      if (waited > kStarveMs) break;
    }
    if (picked) {
      Group* grp = new Group();
      grp->members.push_back(picked);
      grp->slot = picked->slot;
      fill_group(grp, now);
      lk.unlock();
      if (grp->members.size() == 1) {
        delete grp;
        launch_request(this, picked);
      } else {
        launch_group(this, grp);
      }
      lk.lock();
      continue;
    }
    // Wake on new requests or finished ones; the timeout also picks up budget
    // returned by released commits.
    cv.wait_for(lk, std::chrono::milliseconds(2));
  }
}

pico_status serving_start(pico_ctx* ctx) {
  auto* sv = new Server();
  sv->ctx = ctx;
  sv->slot_busy.assign(ctx->streams.size(), false);
  if (cudaMallocHost(&sv->pinned_roots, 32 * kMaxGroup * ctx->streams.size()) != cudaSuccess) {
    delete sv;
    return cuda_status(cudaGetLastError(), "pinned root buffers");
  }
  ctx->server = sv;
  sv->thr = std::thread([sv] { sv->run(); });
  return PICO_OK;
}

void serving_stop(pico_ctx* ctx) {
  Server* sv = ctx->server;
  if (!sv) return;
  {
    std::lock_guard<std::mutex> g(sv->mu);
    sv->stop = true;
    sv->cv.notify_all();
  }
  sv->thr.join();
  for (auto st : ctx->streams) cudaStreamSynchronize(st);
  for (pico_request* r : sv->queue) {
    r->state = pico_request::CANCELLED;
  }
  sv->queue.clear();
  cudaFreeHost(sv->pinned_roots);
  delete sv;
  ctx->server = nullptr;
}

}  // namespace pico

using namespace pico;

extern "C" pico_status pico_gpu_submit_commit(pico_ctx* ctx, pico_field field, const pico_matrix* mats,
                                              uint32_t n_mats, uint32_t log_blowup, uint32_t flags,
                                              pico_request** out) {
  if (!ctx || !out || !ctx->server) {
    set_error("submit_commit: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  *out = nullptr;
  auto r = std::make_unique<pico_request>();
  r->ctx = ctx;
  pico_status s = plan_commit(field, mats, n_mats, log_blowup, flags, true, r->plan);
  if (s) return s;
  if (r->plan.bytes_resident + r->plan.bytes_scratch > ctx->budget) {
    set_error("submit_commit: request needs %llu bytes, more than the whole budget %llu",
              (unsigned long long)(r->plan.bytes_resident + r->plan.bytes_scratch),
              (unsigned long long)ctx->budget);
    return PICO_ERR_OUT_OF_MEMORY;
  }
  if (!(flags & PICO_INPUT_DEVICE)) {
    r->host_copies.resize(r->plan.mats.size());
    for (size_t k = 0; k < r->plan.mats.size(); k++) {
      PlannedMat& m = r->plan.mats[k];
      const size_t cells = (size_t)m.w << m.log_n;
      r->host_copies[k].assign(m.src, m.src + cells);
      m.src = r->host_copies[k].data();
    }
  }
  r->t_submit = Clock::now();
  Server* sv = ctx->server;
  {
    std::lock_guard<std::mutex> g(sv->mu);
    sv->queue.push_back(r.get());
    sv->cv.notify_all();
  }
  *out = r.release();
  return PICO_OK;
}

extern "C" pico_status pico_gpu_poll(pico_ctx* ctx, pico_request* req) {
  if (!ctx || !req) {
    set_error("poll: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  std::lock_guard<std::mutex> g(ctx->server->mu);
  switch (req->state) {
    case pico_request::DONE:
    case pico_request::TAKEN:
      return PICO_OK;
    case pico_request::FAILED:
      set_error("%s", req->error.c_str());
      return req->status;
    case pico_request::CANCELLED:
      return PICO_ERR_CANCELLED;
    default:
      return PICO_ERR_NOT_READY;
  }
}

extern "C" pico_status pico_gpu_wait(pico_ctx* ctx, pico_request* req, int64_t timeout_ms, pico_commit** out,
                                     uint32_t root[8]) {
  if (!ctx || !req) {
    set_error("wait: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  Server* sv = ctx->server;
  std::unique_lock<std::mutex> lk(sv->mu);
  auto ready = [&] {
    return req->state == pico_request::DONE || req->state == pico_request::FAILED ||
           req->state == pico_request::CANCELLED || req->state == pico_request::TAKEN;
  };
  if (timeout_ms < 0)
    sv->done_cv.wait(lk, ready);
  else if (!sv->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
    return PICO_ERR_TIMEOUT;
  if (req->state == pico_request::FAILED) {
    set_error("%s", req->error.c_str());
    return req->status;
  }
  if (req->state == pico_request::CANCELLED) return PICO_ERR_CANCELLED;
  if (req->state == pico_request::TAKEN) {
    set_error("wait: result already taken");
    return PICO_ERR_INVALID_ARG;
  }
  if (root) memcpy(root, req->root, 32);
  pico_commit* c = req->commit;
  req->commit = nullptr;
  req->state = pico_request::TAKEN;
  lk.unlock();
  if (c && getenv("PICO_METRICS_LOG")) {
    finish_stats(c);
    const uint32_t fl = (req->plan.input_device ? PICO_INPUT_DEVICE : 0u) | (req->plan.plain ? PICO_COMMIT_PLAIN : 0u);
    metrics_record("request", req->plan.field, (uint32_t)req->plan.mats.size(), req->plan.log_b, fl, c->stats,
                   std::chrono::duration<double, std::micro>(req->t_admit - req->t_submit).count(),
                   std::chrono::duration<double, std::micro>(req->t_done - req->t_admit).count(), req->group_size);
  }
  if (out) {
    *out = c;
  } else if (c) {
    pico_gpu_release(ctx, c);
  }
  return PICO_OK;
}

extern "C" pico_status pico_gpu_cancel(pico_ctx* ctx, pico_request* req) {
  if (!ctx || !req) {
    set_error("cancel: bad arguments");
    return PICO_ERR_INVALID_ARG;
  }
  Server* sv = ctx->server;
  std::lock_guard<std::mutex> g(sv->mu);
  if (req->state != pico_request::QUEUED) {
    set_error("cancel: request already admitted");
    return PICO_ERR_NOT_READY;
  }
  sv->queue.remove(req);
  req->state = pico_request::CANCELLED;
  sv->done_cv.notify_all();
  return PICO_OK;
}

extern "C" pico_status pico_gpu_request_times(const pico_request* req, double* queued_us, double* run_us) {
  if (!req) {
    set_error("request_times: null request");
    return PICO_ERR_INVALID_ARG;
  }
  if (req->state != pico_request::DONE && req->state != pico_request::TAKEN) return PICO_ERR_NOT_READY;
  if (queued_us) *queued_us = std::chrono::duration<double, std::micro>(req->t_admit - req->t_submit).count();
  if (run_us) *run_us = std::chrono::duration<double, std::micro>(req->t_done - req->t_admit).count();
  return PICO_OK;
}

extern "C" pico_status pico_gpu_request_free(pico_ctx* ctx, pico_request* req) {
  if (!req) return PICO_OK;
  if (!ctx) {
    set_error("request_free: null context");
    return PICO_ERR_INVALID_ARG;
  }
  {
    std::unique_lock<std::mutex> lk(ctx->server->mu);
    if (req->state == pico_request::QUEUED) {
      ctx->server->queue.remove(req);
      req->state = pico_request::CANCELLED;
    }
    // A running request must finish before its bookkeeping can go.
    ctx->server->done_cv.wait(lk, [&] { return req->state != pico_request::RUNNING; });
  }
  if (req->commit) pico_gpu_release(ctx, req->commit);
  delete req;
  return PICO_OK;
}
