// Registration server: continuous batching of independent registrations.
//
// A pool is one Solver with S problem slots for one (grid, nt, solver-wide
// options) key, its own CUDA stream and its own host worker thread.  Requests
// are queued on submit; a pool's worker admits queued requests of its key
// into free slots at every GN-iteration boundary (Solver::begin), advances all
// running slots by one GN iteration per Solver::step, and retires the slots
// whose stopping test fired (Solver::finish), copying the velocity out and
// freeing the slot for the next request.  Host copies go through page-locked
// blocks that each pool allocates when it starts and that are recycled:
// submit puts the images into a free one, so the worker's upload is a DMA,
// and the worker writes each velocity into one that result() copies out, so
// the worker never copies a velocity on the CPU; without a free block the
// pageable path is used.  Pools of different keys run
// concurrently on their own streams, so the work of requests of different
// sizes overlaps on the device.  Pools are created while their footprint
// (Solver::estimate_bytes) fits the HBM budget and release their memory after
// idling, which lets queued requests of another key get a pool.
//
// The reference has no serving layer: each registration there is one
// CLAIREInterface::Run call (src/CLAIREInterface.cpp:709-885); the results of
// a request here are those of that call on the same inputs (the slots of a
// pool never mix data: every kernel and every reduction is per problem).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "solver.cuh"

namespace cb {
namespace srv {

using Clock = std::chrono::steady_clock;

struct Request {
  long long id = 0;
  claire_b200_opts opts{};
  std::vector<float> mR, mT;  // host copies of the inputs (pageable path)
  float* in_pin = nullptr;    // or page-locked: mR then mT
  std::vector<float> v;       // result velocity (pageable path)
  float* v_pin = nullptr;     // or page-locked
  bool staging = false;       // the stager is copying the inputs into a page-locked block
  claire_b200_stats stats{};
  int status = CB_REQ_QUEUED;
  int error = CB_OK;
  bool cancel = false;        // cancellation asked for while running
  Clock::time_point t_submit{}, t_done{};
};

// Options that must agree for problems to share a pool (everything but the
// per-slot regularisation norm and weights).
static bool same_pool(const claire_b200_opts& a, const claire_b200_opts& b) {
  return a.nx[0] == b.nx[0] && a.nx[1] == b.nx[1] && a.nx[2] == b.nx[2] && a.nt == b.nt && a.model == b.model &&
         a.maxit == b.maxit && a.opttol == b.opttol && a.gatol == b.gatol && a.krylovmaxit == b.krylovmaxit &&
         a.krylovtol[0] == b.krylovtol[0] && a.krylovtol[1] == b.krylovtol[1] &&
         a.krylovtol[2] == b.krylovtol[2] && a.krylovfseq == b.krylovfseq && a.precond == b.precond &&
         a.iporder == b.iporder && a.bf16_images == b.bf16_images && a.distance == b.distance;
}

struct Pool;

}  // namespace srv
}  // namespace cb

struct claire_b200_server {
  claire_b200_server_opts opts{};
  std::mutex mu;
  std::condition_variable cv;          // request state changes, new work
  std::deque<long long> queue;         // queued request ids, FIFO
  std::map<long long, cb::srv::Request> reqs;
  std::vector<std::unique_ptr<cb::srv::Pool>> pools;
  long long budget = 0, used = 0;
  long long next_id = 1;
  bool stop = false;
  // page-locked host blocks per direction (0 inputs, 1 results): free lists
  // and blocks allocated, by float count
  std::map<long long, std::vector<float*>> pinned_free[2];
  std::map<long long, int> pinned_count[2];
  std::thread stager;  // copies queued pageable inputs into free page-locked blocks
};

namespace cb {
namespace srv {

struct Pool {
  claire_b200_opts key{};
  std::unique_ptr<Solver> solver;
  std::vector<long long> slot_req;  // request id per slot, 0 = free
  long long bytes = 0;
  bool dead = false;    // worker is leaving: takes no more requests
  bool exited = false;  // worker has released the memory and returns: the thread can be joined
  std::thread worker;
  // Result copies run on their own stream: the worker queues a finished
  // slot's velocity copy and goes on; the publisher thread waits for the copy
  // and publishes the request.  The slot's next request waits (on the device)
  // for the copy out of the slot before its velocity is reset.
  cudaStream_t copy = nullptr;
  float* stage_out = nullptr;            // device, 3n floats per slot: finished velocities being copied out
  std::vector<cudaEvent_t> slot_ready;   // per slot: its velocity is in stage_out
  std::vector<cudaEvent_t> slot_copied;  // per slot: its last copy to the host is done
  std::vector<bool> slot_copy_issued;
  struct Pending {
    long long rid;
    float* pin;
    long long count;
    cudaEvent_t ev;
  };
  std::mutex pmu;  // guards pending, ev_free, pstop
  std::condition_variable pcv;
  std::deque<Pending> pending;
  std::vector<cudaEvent_t> ev_free;
  bool pstop = false;
  std::thread publisher;
};

// Join and drop the pools whose workers have exited.  Called with s->mu held,
// from client threads only (a worker never joins itself or another worker).
static void reap_locked(claire_b200_server* s) {
  for (auto it = s->pools.begin(); it != s->pools.end();) {
    if ((*it)->exited) {
      if ((*it)->worker.joinable()) (*it)->worker.join();
      it = s->pools.erase(it);
    } else {
      ++it;
    }
  }
}

// Page-locked blocks of `count` floats for direction dir (0: request inputs,
// 1: results).  A pool's worker allocates them when it starts (the pool's
// slot count twice over, at most kPinnedPerSize bytes of one size and
// direction); take_pinned only recycles, so no request waits on a
// page-locked allocation, and returns nullptr when none is free (the caller
// uses pageable memory).
constexpr long long kPinnedPerSize = 512LL << 20;

static float* take_pinned(claire_b200_server* s, int dir, long long count) {
  std::lock_guard<std::mutex> lk(s->mu);
  auto& fl = s->pinned_free[dir][count];
  if (fl.empty()) return nullptr;
  float* p = fl.back();
  fl.pop_back();
  return p;
}

// Return a block to its free list (caller holds s->mu).
static void give_pinned_locked(claire_b200_server* s, int dir, long long count, float* p) {
  if (p) s->pinned_free[dir][count].push_back(p);
}

// Bring the blocks of one size and direction up to `want` (bounded by
// kPinnedPerSize); called by a worker without s->mu held.
static void prealloc_pinned(claire_b200_server* s, int dir, long long count, int want) {
  const long long bytes = count * (long long)sizeof(float);
  want = (int)std::max(1LL, std::min<long long>(want, kPinnedPerSize / std::max(1LL, bytes)));
  while (true) {
    {
      std::lock_guard<std::mutex> lk(s->mu);
      if (s->pinned_count[dir][count] >= want) return;
      ++s->pinned_count[dir][count];
    }
    void* p = nullptr;
    if (cudaHostAlloc(&p, (size_t)bytes, cudaHostAllocPortable) != cudaSuccess) {
      cudaGetLastError();
      std::lock_guard<std::mutex> lk(s->mu);
      --s->pinned_count[dir][count];
      return;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->pinned_free[dir][count].push_back(static_cast<float*>(p));
  }
}

static long long pending_for(const claire_b200_server* s, const claire_b200_opts& key) {
  long long k = 0;
  for (long long id : s->queue)
    if (same_pool(s->reqs.at(id).opts, key)) ++k;
  return k;
}

static Pool* find_pool(claire_b200_server* s, const claire_b200_opts& key) {
  for (auto& p : s->pools)
    if (!p->dead && same_pool(p->key, key)) return p.get();
  return nullptr;
}

static void fail_request(claire_b200_server* s, long long id, int err) {
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return;
  it->second.status = CB_REQ_FAILED;
  it->second.error = err;
  it->second.t_done = Clock::now();
}

static void worker_main(claire_b200_server* s, Pool* p);

// Create pools for queued keys that have none while the budget allows.
// Caller holds s->mu.
static void create_pools_locked(claire_b200_server* s) {
  for (long long id : std::vector<long long>(s->queue.begin(), s->queue.end())) {
    Request& r = s->reqs.at(id);
    if (find_pool(s, r.opts)) continue;
    const int slots = std::max(1, s->opts.slots_per_pool);
    const long long nv = 3LL * r.opts.nx[0] * r.opts.nx[1] * r.opts.nx[2];
    const long long need = Solver::estimate_bytes(r.opts, slots) + slots * nv * (long long)sizeof(float);
    if (s->used + need > s->budget) continue;  // stays queued until memory frees up
    auto pool = std::make_unique<Pool>();
    pool->key = r.opts;
    pool->key.verbosity = 0;
    pool->solver = std::make_unique<Solver>();
    int caller_dev = 0;
    cudaGetDevice(&caller_dev);
    cudaSetDevice(s->opts.device);
    const int e = pool->solver->init(pool->key, slots);
    cudaSetDevice(caller_dev);
    if (e) {
      // this key cannot be served at all (unsupported grid, allocation failure)
      for (long long q : std::vector<long long>(s->queue.begin(), s->queue.end()))
        if (same_pool(s->reqs.at(q).opts, r.opts)) {
          fail_request(s, q, e < 0 ? e : CB_ERR_CUDA);
          s->queue.erase(std::find(s->queue.begin(), s->queue.end(), q));
        }
      s->cv.notify_all();
      continue;
    }
    pool->bytes = pool->solver->footprint() + slots * nv * (long long)sizeof(float);  // + stage_out
    pool->slot_req.assign(slots, 0);
    s->used += pool->bytes;
    Pool* raw = pool.get();
    s->pools.push_back(std::move(pool));
    raw->worker = std::thread(worker_main, s, raw);
  }
}

// Admit queued requests of the pool's key into free slots (caller holds mu).
static std::vector<std::pair<int, long long>> admit_locked(claire_b200_server* s, Pool* p) {
  std::vector<std::pair<int, long long>> out;
  for (auto it = s->queue.begin(); it != s->queue.end();) {
    const Request& r = s->reqs.at(*it);
    if (!same_pool(r.opts, p->key) || r.staging) {
      ++it;
      continue;
    }
    int slot = -1;
    for (int b = 0; b < (int)p->slot_req.size(); ++b)
      if (p->slot_req[b] == 0) {
        bool taken = false;
        for (auto& a : out) taken |= a.first == b;
        if (!taken) {
          slot = b;
          break;
        }
      }
    if (slot < 0) break;
    out.push_back({slot, *it});
    it = s->queue.erase(it);
  }
  for (auto& a : out) {
    p->slot_req[a.first] = a.second;
    s->reqs.at(a.second).status = CB_REQ_RUNNING;
  }
  return out;
}

// Inputs of request r into slot b, queued on the pool's stream; the caller
// synchronises (Solver::upload_problems, once for all admitted requests) before
// the request's input block is recycled.
static int load_slot(Solver& sv, int b, const Request& r) {
  const long long n = sv.n;
  const float* hR = r.in_pin ? r.in_pin : r.mR.data();
  const float* hT = r.in_pin ? r.in_pin + n : r.mT.data();
  if (sv.img16) {
    // stage through the free slot's PCG work vector, then round to bf16
    float* st = sv.x + b * 3 * n;
    if (cudaMemcpyAsync(st, hR, sizeof(float) * n, cudaMemcpyHostToDevice, sv.stream) != cudaSuccess ||
        cudaMemcpyAsync(st + n, hT, sizeof(float) * n, cudaMemcpyHostToDevice, sv.stream) != cudaSuccess)
      return CB_ERR_CUDA;
    if (int e = sv.load_images(b, st, st + n)) return e;
    if (cudaMemsetAsync(sv.v + b * 3 * n, 0, sizeof(float) * 3 * n, sv.stream) != cudaSuccess) return CB_ERR_CUDA;
  } else if (cudaMemcpyAsync(sv.mR + b * n, hR, sizeof(float) * n, cudaMemcpyHostToDevice, sv.stream) !=
                 cudaSuccess ||
             cudaMemcpyAsync(sv.mT + b * n, hT, sizeof(float) * n, cudaMemcpyHostToDevice, sv.stream) !=
                 cudaSuccess ||
             cudaMemsetAsync(sv.v + b * 3 * n, 0, sizeof(float) * 3 * n, sv.stream) != cudaSuccess) {
    return CB_ERR_CUDA;
  }
  sv.images_changed(b);
  return sv.set_problem(b, r.opts, false);  // per-slot norm and weights, uploaded by the caller
}

// Publisher thread of a pool: waits (without holding the server's lock) for
// each queued velocity copy and then publishes its request.  It leaves when
// the pool's worker asks it to and the queue is empty.
static void publisher_main(claire_b200_server* s, Pool* p) {
  cudaSetDevice(s->opts.device);
  while (true) {
    Pool::Pending x{};
    {
      std::unique_lock<std::mutex> lk(p->pmu);
      p->pcv.wait(lk, [&] { return p->pstop || !p->pending.empty(); });
      if (p->pending.empty()) break;
      x = p->pending.front();
      p->pending.pop_front();
    }
    const bool ok = cudaEventSynchronize(x.ev) == cudaSuccess;
    {
      std::lock_guard<std::mutex> lk(p->pmu);
      p->ev_free.push_back(x.ev);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(x.rid);
    if (it != s->reqs.end() && ok) {
      it->second.v_pin = x.pin;
      it->second.status = CB_REQ_DONE;
      it->second.t_done = Clock::now();
    } else {
      give_pinned_locked(s, 1, x.count, x.pin);
      if (it != s->reqs.end()) {
        it->second.status = CB_REQ_FAILED;
        it->second.error = CB_ERR_CUDA;
        it->second.t_done = Clock::now();
      }
    }
    s->cv.notify_all();
  }
}

// Queue the copy of slot b's velocity into the page-locked block pin on the
// pool's copy stream (after the slot's last kernel) and hand it to the
// publisher.  Called by the worker.
static int queue_result_copy(Pool* p, Solver& sv, int b, long long rid, float* pin) {
  const long long nv = 3 * sv.n;
  cudaEvent_t ev = nullptr;
  {
    std::lock_guard<std::mutex> lk(p->pmu);
    if (!p->ev_free.empty()) {
      ev = p->ev_free.back();
      p->ev_free.pop_back();
    }
  }
  if (!ev && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return CB_ERR_CUDA;
  // with stage_out the slot's velocity is first copied on the device (the slot
  // is then free at once); the host copy runs beside the next requests' work
  const float* src = sv.v + b * nv;
  bool ok = true;
  if (p->stage_out) {
    float* st = p->stage_out + b * nv;
    ok = (!p->slot_copy_issued[b] || cudaStreamWaitEvent(sv.stream, p->slot_copied[b], 0) == cudaSuccess) &&
         cudaMemcpyAsync(st, src, sizeof(float) * nv, cudaMemcpyDeviceToDevice, sv.stream) == cudaSuccess;
    src = st;
  }
  ok = ok && cudaEventRecord(p->slot_ready[b], sv.stream) == cudaSuccess &&
       cudaStreamWaitEvent(p->copy, p->slot_ready[b], 0) == cudaSuccess &&
       cudaMemcpyAsync(pin, src, sizeof(float) * nv, cudaMemcpyDeviceToHost, p->copy) == cudaSuccess &&
       cudaEventRecord(p->slot_copied[b], p->copy) == cudaSuccess && cudaEventRecord(ev, p->copy) == cudaSuccess;
  if (!ok) {
    cudaEventDestroy(ev);
    return CB_ERR_CUDA;
  }
  p->slot_copy_issued[b] = true;
  {
    std::lock_guard<std::mutex> lk(p->pmu);
    p->pending.push_back(Pool::Pending{rid, pin, nv, ev});
  }
  p->pcv.notify_all();
  return CB_OK;
}

// Stager thread: while a queued request still holds pageable inputs and a
// page-locked input block of its size is free, move the inputs into the block
// (the CPU copy runs here, beside the pools' GPU work, so the worker's upload
// of that request is a DMA).  A request is not admitted while it is staged.
static void stager_main(claire_b200_server* s) {
  std::unique_lock<std::mutex> lk(s->mu);
  while (!s->stop) {
    long long pick = 0, n = 0;
    float* blk = nullptr;
    for (long long id : s->queue) {
      Request& r = s->reqs.at(id);
      if (r.in_pin || r.staging || r.mR.empty()) continue;
      const long long nn = (long long)r.opts.nx[0] * r.opts.nx[1] * r.opts.nx[2];
      auto fl = s->pinned_free[0].find(2 * nn);
      if (fl == s->pinned_free[0].end() || fl->second.empty()) continue;
      blk = fl->second.back();
      fl->second.pop_back();
      pick = id;
      n = nn;
      break;
    }
    if (!pick) {
      s->cv.wait(lk);
      continue;
    }
    Request& r = s->reqs.at(pick);
    r.staging = true;
    std::vector<float> a = std::move(r.mR), b = std::move(r.mT);
    lk.unlock();
    std::memcpy(blk, a.data(), sizeof(float) * n);
    std::memcpy(blk + n, b.data(), sizeof(float) * n);
    lk.lock();
    auto it = s->reqs.find(pick);
    if (it != s->reqs.end() && it->second.status == CB_REQ_QUEUED) {
      it->second.in_pin = blk;
      it->second.staging = false;
    } else {
      // cancelled or failed meanwhile: its inputs are no longer needed
      if (it != s->reqs.end()) it->second.staging = false;
      give_pinned_locked(s, 0, 2 * n, blk);
    }
    s->cv.notify_all();
  }
}

static void fill_stats(const ProbState& ps, claire_b200_stats* st) {
  std::memset(st, 0, sizeof(*st));
  st->gn_iterations = ps.iter;
  st->pcg_iterations = ps.pcg_total;
  st->obj_evals = ps.obj_evals;
  st->grad_evals = ps.grad_evals;
  st->hess_matvecs = ps.hess_matvecs;
  st->pc_matvecs = ps.pc_matvecs;
  st->pde_solves = ps.pde_solves;
  st->converged_reason = ps.reason;
  st->J = ps.J;
  st->J0 = ps.J0;
  st->D = ps.D;
  st->D0 = ps.D0;
  st->R = ps.R;
  st->gnorm = ps.gnorm;
  st->gnorm0 = ps.gnorm0;
  st->rel_mismatch = ps.rel_mismatch;
  st->seconds = ps.seconds;
  st->beta = ps.beta0;
}

static void worker_main(claire_b200_server* s, Pool* p) {
  cudaSetDevice(s->opts.device);
  Solver& sv = *p->solver;
  const int S = sv.B;
  prealloc_pinned(s, 0, 2 * sv.n, 2 * S);
  prealloc_pinned(s, 1, 3 * sv.n, 2 * S);
  int err = CB_OK;
  p->slot_ready.assign(S, nullptr);
  p->slot_copied.assign(S, nullptr);
  p->slot_copy_issued.assign(S, false);
  if (cudaStreamCreateWithFlags(&p->copy, cudaStreamNonBlocking) != cudaSuccess) err = CB_ERR_CUDA;
  for (int b = 0; b < S && !err; ++b)
    if (cudaEventCreateWithFlags(&p->slot_ready[b], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&p->slot_copied[b], cudaEventDisableTiming) != cudaSuccess)
      err = CB_ERR_CUDA;
  if (!err && cudaMalloc((void**)&p->stage_out, sizeof(float) * 3 * sv.n * S) != cudaSuccess) {
    cudaGetLastError();
    p->stage_out = nullptr;  // copies go straight from the slots' velocities
  }
  p->publisher = std::thread(publisher_main, s, p);
  while (!err) {
    std::vector<std::pair<int, long long>> admits;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      if (s->stop) break;
      // cancelled requests leave their slots at this GN-iteration boundary
      bool cancelled = false;
      for (int b = 0; b < S; ++b) {
        if (!p->slot_req[b]) continue;
        Request& r = s->reqs.at(p->slot_req[b]);
        if (!r.cancel) continue;
        r.status = CB_REQ_CANCELLED;
        r.error = CB_ERR_CANCELLED;
        r.t_done = Clock::now();
        p->slot_req[b] = 0;
        sv.ps[b].running = false;
        sv.ps[b].done = true;
        cancelled = true;
      }
      if (cancelled) s->cv.notify_all();
      bool running = false;
      for (int b = 0; b < S; ++b) running |= p->slot_req[b] != 0;
      if (!running && s->opts.batch_window_us > 0) {
        // an idle pool with work: requests submitted together (a client's
        // batch) get a short window to arrive, so their GN loops start in the
        // same step instead of one GN iteration apart
        const long long pend = pending_for(s, p->key);
        if (pend > 0 && pend < S) {
          s->cv.wait_until(lk, Clock::now() + std::chrono::microseconds(s->opts.batch_window_us),
                           [&] { return s->stop || pending_for(s, p->key) >= S; });
          if (s->stop) break;
        }
      }
      admits = admit_locked(s, p);
      bool busy = !admits.empty();
      for (int b = 0; b < S; ++b) busy |= p->slot_req[b] != 0;
      if (!busy) {
        const bool got = s->cv.wait_for(lk, std::chrono::milliseconds(std::max(1, s->opts.idle_ms)), [&] {
          return s->stop || pending_for(s, p->key) > 0;
        });
        if (s->stop) break;
        if (!got) break;  // idle: release the pool
        continue;
      }
    }
    // admission: inputs into the slots (one synchronisation for all), then
    // InitializeOptimization for them
    std::vector<int> sel_new(S, 0);
    std::vector<Request*> loaded;
    for (auto& a : admits) {
      Request* r;
      {
        std::lock_guard<std::mutex> lk(s->mu);
        r = &s->reqs.at(a.second);
      }
      loaded.push_back(r);
      // without stage_out the slot's previous velocity is copied straight
      // from the slot, and must be out before the slot is reset
      if (!p->stage_out && p->slot_copy_issued[a.first] &&
          cudaStreamWaitEvent(sv.stream, p->slot_copied[a.first], 0) != cudaSuccess)
        err = CB_ERR_CUDA;
      if (!err) err = load_slot(sv, a.first, *r);
      if (err) break;
      sel_new[a.first] = 1;
    }
    if (!admits.empty()) {
      const int e = sv.upload_problems();  // synchronises: the uploads are done
      if (!err) err = e;
      std::lock_guard<std::mutex> lk(s->mu);
      for (Request* r : loaded)
        if (r->in_pin) {
          if (e) continue;  // an upload may still be in flight: keep the block with the request
          give_pinned_locked(s, 0, 2 * sv.n, r->in_pin);
          r->in_pin = nullptr;
        }
      s->cv.notify_all();  // the stager may fill the returned blocks for queued requests
    }
    if (!err && !admits.empty()) err = sv.begin(sel_new);
    std::vector<int> fin(S, 0);
    if (!err) err = sv.step(fin);
    // retire every slot whose GN loop has stopped
    std::vector<int> done(S, 0);
    bool anydone = false;
    if (!err)
      for (int b = 0; b < S; ++b)
        if (p->slot_req[b] && sv.ps[b].running && sv.ps[b].done) {
          done[b] = 1;
          anydone = true;
        }
    if (!err && anydone) err = sv.finish(done);
    if (err) break;
    if (anydone) {
      // velocities into page-locked blocks on the copy stream (published by the
      // publisher thread when they land), or, past the blocks, synchronously
      // into pageable vectors
      const long long nv = 3 * sv.n;
      std::vector<std::pair<int, std::vector<float>>> outv;
      std::vector<int> queued;
      for (int b = 0; b < S && !err; ++b) {
        if (!done[b]) continue;
        float* pin = take_pinned(s, 1, nv);
        long long rid;
        {
          // statistics first: the publisher may publish the request as soon as
          // its copy is queued
          std::lock_guard<std::mutex> lk(s->mu);
          rid = p->slot_req[b];
          fill_stats(sv.ps[b], &s->reqs.at(rid).stats);
        }
        if (pin) {
          err = queue_result_copy(p, sv, b, rid, pin);
          if (err) {
            std::lock_guard<std::mutex> lk(s->mu);
            give_pinned_locked(s, 1, nv, pin);
          } else {
            queued.push_back(b);
          }
          continue;
        }
        std::vector<float> vh((size_t)nv);
        if (cudaMemcpyAsync(vh.data(), sv.v + b * nv, sizeof(float) * nv, cudaMemcpyDeviceToHost, sv.stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(sv.stream) != cudaSuccess)
          err = CB_ERR_CUDA;
        else
          outv.push_back({b, std::move(vh)});
      }
      std::lock_guard<std::mutex> lk(s->mu);
      for (int b : queued) p->slot_req[b] = 0;  // published when their copies land
      for (auto& o : outv) {
        const int b = o.first;
        Request& r = s->reqs.at(p->slot_req[b]);
        r.v = std::move(o.second);
        r.status = CB_REQ_DONE;
        r.t_done = Clock::now();
        p->slot_req[b] = 0;
      }
      s->cv.notify_all();
      if (err) break;
    }
  }
  // exit: let the publisher finish the queued copies (it takes the server's
  // lock, so it is joined before this thread takes it), fail what this pool
  // still holds, release the memory, let queued requests of other keys get a
  // pool
  {
    std::lock_guard<std::mutex> lk(p->pmu);
    p->pstop = true;
  }
  p->pcv.notify_all();
  if (p->publisher.joinable()) p->publisher.join();
  if (p->copy) cudaStreamSynchronize(p->copy);
  for (cudaEvent_t e : p->ev_free) cudaEventDestroy(e);
  p->ev_free.clear();
  for (cudaEvent_t e : p->slot_ready)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : p->slot_copied)
    if (e) cudaEventDestroy(e);
  if (p->copy) cudaStreamDestroy(p->copy);
  p->copy = nullptr;
  if (p->stage_out) cudaFree(p->stage_out);
  p->stage_out = nullptr;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (int b = 0; b < S; ++b)
      if (p->slot_req[b]) fail_request(s, p->slot_req[b], err ? err : CB_ERR_STATE);
    p->dead = true;
  }
  p->solver.reset();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->used -= p->bytes;
    p->bytes = 0;
    if (!s->stop) create_pools_locked(s);
    p->exited = true;
    s->cv.notify_all();
  }
}

}  // namespace srv
}  // namespace cb

using cb::srv::Clock;

extern "C" {

void claire_b200_server_default_opts(claire_b200_server_opts* o) {
  if (!o) return;
  o->hbm_budget_bytes = 0;
  o->slots_per_pool = 4;
  o->idle_ms = 2000;
  o->device = 0;
  o->batch_window_us = 0;
}

int claire_b200_server_create(const claire_b200_server_opts* o, claire_b200_server** out) {
  if (!o || !out || o->slots_per_pool < 1 || o->slots_per_pool > 1024) return CB_ERR_ARG;
  *out = nullptr;
  auto* s = new (std::nothrow) claire_b200_server();
  if (!s) return CB_ERR_ALLOC;
  s->opts = *o;
  if (cudaSetDevice(o->device) != cudaSuccess) {
    delete s;
    return CB_ERR_CUDA;
  }
  size_t freeb = 0, total = 0;
  if (cudaMemGetInfo(&freeb, &total) != cudaSuccess) {
    delete s;
    return CB_ERR_CUDA;
  }
  s->budget = o->hbm_budget_bytes > 0 ? o->hbm_budget_bytes : (long long)(0.9 * (double)freeb);
  try {
    s->stager = std::thread(cb::srv::stager_main, s);
  } catch (...) {
    delete s;
    return CB_ERR_ALLOC;
  }
  *out = s;
  return CB_OK;
}

int claire_b200_server_submit(claire_b200_server* s, const claire_b200_opts* o, const float* mR, const float* mT,
                              long long* id) {
  if (!s || !o || !mR || !mT || !id) return CB_ERR_ARG;
  // a pool advances its slots one GN iteration at a time: the continuation
  // drivers (several solves per request) and the two-level preconditioner
  // (a nested coarse solve per Krylov iteration) run through claire_b200_run
  if (o->betacont > 0.0 || o->scalecont || o->gridcont || o->train || o->monitordefgrad ||
      o->precond == CB_PC_TWOLEVEL)
    return CB_ERR_UNSUPPORTED;
  if (o->nx[0] <= 0 || o->nx[1] <= 0 || o->nx[2] <= 0 || o->nt < 1) return CB_ERR_ARG;
  const long long n = (long long)o->nx[0] * o->nx[1] * o->nx[2];
  cb::srv::Request r;
  r.opts = *o;
  r.in_pin = cb::srv::take_pinned(s, 0, 2 * n);
  if (r.in_pin) {
    std::memcpy(r.in_pin, mR, sizeof(float) * n);
    std::memcpy(r.in_pin + n, mT, sizeof(float) * n);
  } else {
    try {
      r.mR.assign(mR, mR + n);
      r.mT.assign(mT, mT + n);
    } catch (...) {
      return CB_ERR_ALLOC;
    }
  }
  r.t_submit = Clock::now();
  std::lock_guard<std::mutex> lk(s->mu);
  const bool too_large = cb::Solver::estimate_bytes(*o, std::max(1, s->opts.slots_per_pool)) > s->budget;
  if (s->stop || too_large) {
    cb::srv::give_pinned_locked(s, 0, 2 * n, r.in_pin);
    return s->stop ? CB_ERR_STATE : CB_ERR_TOO_LARGE;
  }
  cb::srv::reap_locked(s);
  r.id = s->next_id++;
  *id = r.id;
  s->reqs.emplace(r.id, std::move(r));
  s->queue.push_back(*id);
  cb::srv::create_pools_locked(s);
  s->cv.notify_all();
  return CB_OK;
}

int claire_b200_server_poll(claire_b200_server* s, long long id, int* status) {
  if (!s || !status) return CB_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return CB_ERR_ARG;
  *status = it->second.status;
  return CB_OK;
}

int claire_b200_server_wait(claire_b200_server* s, long long id, int timeout_ms, int* status) {
  if (!s) return CB_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto finished = [&] {
    auto it = s->reqs.find(id);
    return it == s->reqs.end() || it->second.status == CB_REQ_DONE || it->second.status == CB_REQ_FAILED ||
           it->second.status == CB_REQ_CANCELLED;
  };
  if (timeout_ms < 0) s->cv.wait(lk, finished);
  else s->cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), finished);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return CB_ERR_ARG;
  if (status) *status = it->second.status;
  return CB_OK;
}

int claire_b200_server_result(claire_b200_server* s, long long id, float* v, claire_b200_stats* st,
                              double* latency_ms) {
  if (!s) return CB_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return CB_ERR_ARG;
  cb::srv::Request& r = it->second;
  const long long n = (long long)r.opts.nx[0] * r.opts.nx[1] * r.opts.nx[2];
  if (r.status == CB_REQ_FAILED || r.status == CB_REQ_CANCELLED) {
    const int e = r.error ? r.error : CB_ERR_STATE;
    cb::srv::give_pinned_locked(s, 0, 2 * n, r.in_pin);
    s->reqs.erase(it);
    return e;
  }
  if (r.status != CB_REQ_DONE) return CB_ERR_STATE;
  if (v) {
    if (r.v_pin) std::memcpy(v, r.v_pin, sizeof(float) * 3 * n);
    else std::memcpy(v, r.v.data(), sizeof(float) * r.v.size());
  }
  cb::srv::give_pinned_locked(s, 1, 3 * n, r.v_pin);
  if (st) *st = r.stats;
  if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r.t_done - r.t_submit).count();
  s->reqs.erase(it);
  return CB_OK;
}

int claire_b200_server_info(claire_b200_server* s, int* pools, long long* bytes_used, int* queued) {
  if (!s) return CB_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  cb::srv::reap_locked(s);
  int live = 0;
  for (auto& p : s->pools) live += p->dead ? 0 : 1;
  if (pools) *pools = live;
  if (bytes_used) *bytes_used = s->used;
  if (queued) *queued = (int)s->queue.size();
  return CB_OK;
}

int claire_b200_server_cancel(claire_b200_server* s, long long id) {
  if (!s) return CB_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  cb::srv::reap_locked(s);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return CB_ERR_ARG;
  cb::srv::Request& r = it->second;
  if (r.status == CB_REQ_QUEUED) {
    auto q = std::find(s->queue.begin(), s->queue.end(), id);
    if (q != s->queue.end()) s->queue.erase(q);
    r.status = CB_REQ_CANCELLED;
    r.error = CB_ERR_CANCELLED;
    r.t_done = Clock::now();
    s->cv.notify_all();
    return CB_OK;
  }
  if (r.status == CB_REQ_RUNNING) {
    r.cancel = true;  // its pool retires it at the next GN-iteration boundary
    return CB_OK;
  }
  return CB_ERR_STATE;  // already done, failed or cancelled
}

int claire_b200_server_destroy(claire_b200_server* s) {
  if (!s) return CB_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    for (long long id : s->queue) cb::srv::fail_request(s, id, CB_ERR_STATE);
    s->queue.clear();
    s->cv.notify_all();
  }
  if (s->stager.joinable()) s->stager.join();
  for (auto& p : s->pools)
    if (p->worker.joinable()) p->worker.join();
  for (auto& kv : s->reqs) {
    if (kv.second.in_pin) cudaFreeHost(kv.second.in_pin);
    if (kv.second.v_pin) cudaFreeHost(kv.second.v_pin);
  }
  for (auto& fl : s->pinned_free)
    for (auto& kv : fl)
      for (float* p : kv.second) cudaFreeHost(p);
  delete s;
  return CB_OK;
}

}  // extern "C"
