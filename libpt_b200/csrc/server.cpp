// Serving loop (pt_serve.h): admission of solves by device footprint into a
// pool, continuous batching of the resident solves' triples into shared
// rounds, completion of each solve's energy as soon as its last round ends.
//
// Threads:
//   admitter  takes queued solves in arrival order; when a block of the
//             solve's footprint is free in the pool (and fewer than
//             max_active solves are resident) it creates the solve's plan
//             inside that block (operands uploaded and prepared on the
//             preparation stream, overlapping the rounds on the run stream)
//             and hands it to the runner.
//   runner    builds a round from the resident solves (least remaining work
//             first, up to a flop budget, at most one round in flight per
//             solve since a solve's round workspace is reused), launches it
//             on the run stream by replaying the CUDA graph captured for
//             the round's set of kernel variants (the first round of a set
//             launches directly, then captures) -- and
//             retires finished rounds; a solve whose triples have all run
//             has its energy read back (queue-order compensated sum) and
//             its block returned to the pool.
// No call of the loop allocates device memory after creation.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "exec.h"
#include "plan.h"
#include "pt.h"
#include "pt_serve.h"

#define LIBPT_API extern "C" __attribute__((visibility("default")))

namespace ptb {
namespace {

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

constexpr size_t ALIGN = 256;
size_t up256(size_t x) { return (x + ALIGN - 1) & ~(ALIGN - 1); }

// First-fit allocator over [0, cap) with coalescing of freed blocks.
class Pool {
 public:
  void init(size_t cap) {
    free_.clear();
    if (cap) free_[0] = cap;
  }
  bool alloc(size_t n, size_t *off) {
    n = up256(n);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < n) continue;
      *off = it->first;
      const size_t rest = it->second - n, o2 = it->first + n;
      free_.erase(it);
      if (rest) free_[o2] = rest;
      return true;
    }
    return false;
  }
  void release(size_t off, size_t n) {
    n = up256(n);
    auto it = free_.emplace(off, n).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }

 private:
  std::map<size_t, size_t> free_;
};

struct Solve {
  uint64_t id = 0;
  int kind = 0, dtype = 0, precision = 0;
  size_t oa = 0, va = 0, ob = 0, vb = 0;
  bool host = true;
  std::vector<const void *> args;
  double t_submit = 0.0, t_done = 0.0;
  size_t bytes = 0, nb = 0, off = 0;
  libpt_plan *plan = nullptr;
  size_t total = 0, next = 0;    // queue entries, next to schedule
  int inflight = 0;              // rounds holding its triples, not retired
  int halves = 1;                // 2: its round resources are split so two
  int half = 0;                  // rounds can be in flight (next half)
  double remaining = 0.0;        // reference flops left to schedule
  bool done = false;
  bool cancelled = false;        // libpt_server_cancel: stop and report so
  bool consumed = false;         // inputs copied (or the solve ended)
  // phase marks (now_s): block granted, plan created (resident), first
  // round launched
  double t_admit = 0.0, t_ready = 0.0, t_first = 0.0;
  int status = LIBPT_OK;
  std::string error;             // message of a failure
  double energy = 0.0;
};

struct RoundRec {
  cudaEvent_t ev = nullptr;
  std::vector<std::shared_ptr<Solve>> solves;
};

// Round sizing: the flops of one round (about 50 ms of FP64 work) and the
// round workspace a solve gets.  Every round replays a captured graph: the
// kernels read their tensor maps from device memory there, which measured
// as fast as the kernel-parameter maps of direct launches (FP64 DMMA and
// every INT8 tile variant within 1 %, 477 x 65536 x 477 jobs), so the
// graphs cost large rounds nothing and save small rounds their launches.
constexpr double ROUND_FLOPS = 1.5e12;
constexpr size_t ROUND_TRIPLES = 8192;
constexpr size_t JOBS_PER_TRIPLE = 6;
constexpr size_t WS_TARGET = (size_t)4 << 30;   // per round, per solve

}  // namespace
}  // namespace ptb

using ptb::Solve;

struct libpt_server {
  std::mutex mu;
  std::condition_variable cv_admit, cv_run, cv_done;
  bool stop = false;
  char *pool_base = nullptr;
  size_t pool_bytes = 0, in_use = 0, peak = 0;
  ptb::Pool pool;
  int max_active = 64;
  cudaStream_t prep_st = nullptr, run_st = nullptr, read_st = nullptr;
  std::deque<std::shared_ptr<Solve>> pending;
  int admitting = 0;   // taken from pending, plan being created
  std::vector<std::shared_ptr<Solve>> resident;
  std::map<uint64_t, std::shared_ptr<Solve>> by_id;
  uint64_t next_id = 1;
  ptb::Executor exec;
  char *d_desc = nullptr;
  unsigned *d_err = nullptr;
  unsigned *h_err = nullptr;   // pinned mirror, refreshed after each round
  std::deque<ptb::RoundRec> inflight;
  std::thread admitter, runner;
  libpt_server_stats st{};
};

namespace ptb {
namespace {

void finish(libpt_server *S, const std::shared_ptr<Solve> &s, int status) {
  // caller holds S->mu; the message is this thread's last error
  s->done = true;
  s->consumed = true;
  s->status = status;
  if (status != LIBPT_OK) s->error = last_error();
  s->t_done = now_s();
  if (status == LIBPT_OK)
    ++S->st.completed;
  else
    ++S->st.failed;
  S->cv_done.notify_all();
}

// Triples in the queue of a solve (src/pt.c:208-221, 331-344): i<j<k per
// same-spin space, i<j (x) k per mixed-spin pair of spaces.
size_t queue_length(int kind, size_t oa, size_t va, size_t ob, size_t vb) {
  const bool unr = kind == 1 || kind == 3;
  if (!unr) {
    ob = oa;
    vb = va;
  }
  auto c3 = [](size_t o, size_t v) { return v ? o * (o - 1) * (o - 2) / 6 : 0; };
  auto c2k = [](size_t o1, size_t v1, size_t o2, size_t v2) {
    return (v1 && v2 && o2) ? o1 * (o1 - 1) / 2 * o2 : 0;
  };
  if (oa < 2 && ob < 2) return 0;
  size_t n = (oa >= 3 ? c3(oa, va) : 0) + (oa >= 2 ? c2k(oa, va, ob, vb) : 0);
  if (unr)
    n += (ob >= 3 ? c3(ob, vb) : 0) + (ob >= 2 ? c2k(ob, vb, oa, va) : 0);
  return n;
}

// Round triples a solve may hold: its whole queue when that fits the
// workspace target, else what the target holds (at least one), twice when
// its queue needs more than one round (two rounds in flight).
int size_solve(Solve &s) {
  const size_t f1 = plan_footprint(s.kind, s.oa, s.va, s.ob, s.vb, s.dtype,
                                   s.precision, s.host, 1);
  const size_t f2 = plan_footprint(s.kind, s.oa, s.va, s.ob, s.vb, s.dtype,
                                   s.precision, s.host, 2);
  if (!f1 || !f2) return LIBPT_ERR_ARG;
  const size_t per = f2 > f1 ? f2 - f1 : 1;
  size_t nb = std::max<size_t>(1, WS_TARGET / per);
  nb = std::min(nb, ROUND_TRIPLES);
  const size_t nq = queue_length(s.kind, s.oa, s.va, s.ob, s.vb);
  s.halves = nq > nb ? 2 : 1;
  s.nb = std::min(nb * s.halves, std::max<size_t>(nq, 1));
  s.bytes = plan_footprint(s.kind, s.oa, s.va, s.ob, s.vb, s.dtype,
                           s.precision, s.host, s.nb);
  return s.bytes ? LIBPT_OK : LIBPT_ERR_ARG;
}

void admit_loop(libpt_server *S) {
  for (;;) {
    std::shared_ptr<Solve> s;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_admit.wait(lk, [&] { return S->stop || !S->pending.empty(); });
      if (S->pending.empty()) return;   // stop requested and drained
      s = S->pending.front();
    }
    if (!s->bytes) {
      int r = size_solve(*s);
      if (!r && s->bytes > S->pool_bytes) r = LIBPT_ERR_NOMEM;
      if (r) {
        std::lock_guard<std::mutex> lk(S->mu);
        S->pending.pop_front();
        set_error("libpt_server: solve does not fit the device pool");
        finish(S, s, r);
        continue;
      }
    }
    {
      // wait for room: a free block and a resident slot (or a cancel)
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_admit.wait(lk, [&] {
        return s->cancelled || ((int)S->resident.size() < S->max_active &&
                                S->pool.alloc(s->bytes, &s->off));
      });
      S->pending.pop_front();
      if (s->cancelled) {
        set_error("libpt_server: solve cancelled");
        finish(S, s, LIBPT_ERR_CANCELLED);
        continue;
      }
      s->t_admit = now_s();
      ++S->admitting;
      S->in_use += up256(s->bytes);
      S->peak = std::max(S->peak, S->in_use);
    }
    libpt_plan *p = nullptr;
    const int r = plan_create(s->kind, s->oa, s->va, s->ob, s->vb,
                              s->args.data(), s->dtype, s->precision, s->host,
                              S->prep_st, &p, S->pool_base + s->off, s->bytes,
                              s->nb);
    std::lock_guard<std::mutex> lk(S->mu);
    if (r) {
      S->pool.release(s->off, s->bytes);
      S->in_use -= up256(s->bytes);
      --S->admitting;
      finish(S, s, r);
      S->cv_admit.notify_all();
      continue;
    }
    s->plan = p;
    s->consumed = true;   // plan_create synchronized its uploads
    s->total = p->queue.size();
    s->remaining = plan_flops(p, 0, (int64_t)s->total);
    s->t_ready = now_s();
    --S->admitting;
    if (s->cancelled) {   // cancelled while its plan was being created
      plan_destroy(p);
      s->plan = nullptr;
      S->pool.release(s->off, s->bytes);
      S->in_use -= up256(s->bytes);
      set_error("libpt_server: solve cancelled");
      finish(S, s, LIBPT_ERR_CANCELLED);
      S->cv_admit.notify_all();
      continue;
    }
    if (s->total == 0) {   // empty spaces: zero energy, nothing to run
      plan_destroy(p);
      s->plan = nullptr;
      S->pool.release(s->off, s->bytes);
      S->in_use -= up256(s->bytes);
      s->energy = 0.0;
      finish(S, s, LIBPT_OK);
      S->cv_admit.notify_all();
      continue;
    }
    S->resident.push_back(s);
    S->st.max_resident = std::max<uint64_t>(S->st.max_resident,
                                            S->resident.size());
    S->cv_run.notify_all();
  }
}

// Reads a finished solve's energy and returns its block (runner thread;
// S->mu not held).
void complete(libpt_server *S, const std::shared_ptr<Solve> &s, bool err) {
  double e = 0.0;
  int r = err ? LIBPT_ERR_TIMEOUT : LIBPT_OK;
  bool cancelled;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    cancelled = s->cancelled;
  }
  if (err) set_error("libpt_server: a device-side wait of the solve's round "
                     "exceeded its time limit, or the round failed to launch");
  if (!r && cancelled) {
    set_error("libpt_server: solve cancelled");
    r = LIBPT_ERR_CANCELLED;
  }
  if (!r) r = plan_energy(s->plan, nullptr, 0, &e, S->read_st);
  plan_destroy(s->plan);
  std::lock_guard<std::mutex> lk(S->mu);
  s->plan = nullptr;
  s->energy = e;
  S->pool.release(s->off, s->bytes);
  S->in_use -= up256(s->bytes);
  S->resident.erase(std::find(S->resident.begin(), S->resident.end(), s));
  finish(S, s, r);
  S->cv_admit.notify_all();
}

// Retires finished rounds (in order); block: wait for the oldest.
void retire(libpt_server *S, bool block) {
  while (!S->inflight.empty()) {
    RoundRec &rr = S->inflight.front();
    if (block) {
      cudaEventSynchronize(rr.ev);
      block = false;
    } else if (cudaEventQuery(rr.ev) != cudaSuccess) {
      break;
    }
    const bool err = *S->h_err != 0;
    if (err) {   // a wait in this round's kernels timed out: reset the flag
      *S->h_err = 0;
      cudaMemsetAsync(S->d_err, 0, sizeof(unsigned), S->run_st);
    }
    std::vector<std::shared_ptr<Solve>> fin;
    {
      std::lock_guard<std::mutex> lk(S->mu);
      for (auto &s : rr.solves)
        if (--s->inflight == 0 && (s->next == s->total || s->cancelled))
          fin.push_back(s);
    }
    cudaEventDestroy(rr.ev);
    S->inflight.pop_front();
    for (auto &s : fin) complete(S, s, err);
  }
}

void run_loop(libpt_server *S) {
  Round round;
  for (;;) {
    retire(S, false);
    // candidates: resident solves with triples to schedule and no round in
    // flight, least remaining work first
    std::vector<std::shared_ptr<Solve>> cand, drop;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      for (auto &s : S->resident) {
        if (s->cancelled) {   // no more rounds; ends once none is in flight
          if (s->inflight == 0) drop.push_back(s);
          continue;
        }
        if (s->next < s->total && s->inflight < s->halves) cand.push_back(s);
      }
      if (!drop.empty()) {
        lk.unlock();
        for (auto &s : drop) complete(S, s, false);
        continue;
      }
      if (cand.empty() && S->inflight.empty()) {
        if (S->stop && S->pending.empty() && S->admitting == 0 &&
            S->resident.empty())
          return;
        S->cv_run.wait_for(lk, std::chrono::milliseconds(2));
        continue;
      }
    }
    if (cand.empty()) {
      retire(S, true);
      continue;
    }
    std::sort(cand.begin(), cand.end(),
              [](const std::shared_ptr<Solve> &a,
                 const std::shared_ptr<Solve> &b) {
                return a->remaining < b->remaining;
              });
    round.clear();
    RoundRec rr;
    std::vector<int64_t> ents;
    for (auto &s : cand) {
      if (round.gemm_flops >= ROUND_FLOPS || round.triples >= ROUND_TRIPLES)
        break;
      libpt_plan *p = s->plan;
      // its kernel variants must fit the round's launch slots
      std::map<GemmGroup, int> groups;
      for (auto &kv : round.gemm) groups[kv.first] = 1;
      for (const SpinCase &c : p->cases)
        if (c.count) groups[plan_group(p, c)] = 1;
      if ((int)groups.size() > EXEC_MAX_GROUPS) continue;
      // its next triples, as many as its workspace and the budget allow
      const size_t room = std::min(ROUND_TRIPLES - round.triples,
                                   s->total - s->next);
      ents.clear();
      double f = 0.0;
      for (size_t x = 0; x < room; ++x) {
        const int64_t q = (int64_t)(s->next + x);
        ents.push_back(q);
        f += plan_flops(p, q, 1);
        if (round.gemm_flops + f >= ROUND_FLOPS) break;
      }
      PlanCursor cur;
      if (s->halves == 2) {   // alternate halves of its round resources
        const int h = s->half;
        cur.ws = h ? p->ws_cap / 2 : 0;
        cur.ws_end = h ? p->ws_cap : p->ws_cap / 2;
        cur.part = h ? p->part_cap / 2 : 0;
        cur.part_end = h ? p->part_cap : p->part_cap / 2;
        cur.triples = h ? p->tri_cap / 2 : 0;
        cur.tri_end = h ? p->tri_cap : p->tri_cap / 2;
      }
      size_t taken = 0;
      if (plan_append(p, ents.data(), ents.size(), cur, round, &taken) ||
          taken == 0)
        continue;
      s->remaining -= plan_flops(p, (int64_t)s->next, (int64_t)taken);
      s->next += taken;
      if (s->t_first == 0.0) s->t_first = now_s();
      s->half ^= 1;
      rr.solves.push_back(s);
    }
    if (rr.solves.empty()) {
      retire(S, true);
      continue;
    }
    {
      std::lock_guard<std::mutex> lk(S->mu);
      for (auto &s : rr.solves) ++s->inflight;
    }
    const bool replay = true;
    const int64_t replays0 = S->exec.graph_replays();
    int64_t launches = 0;
    int r = S->exec.run(round, S->d_err, nullptr, &launches, replay);
    if (!r) r = cudaMemcpyAsync(S->h_err, S->d_err, sizeof(unsigned),
                                cudaMemcpyDeviceToHost, S->run_st) == cudaSuccess
                    ? LIBPT_OK : LIBPT_ERR_CUDA;
    if (!r)
      r = cudaEventCreateWithFlags(&rr.ev, cudaEventDisableTiming) == cudaSuccess &&
                  cudaEventRecord(rr.ev, S->run_st) == cudaSuccess
              ? LIBPT_OK : LIBPT_ERR_CUDA;
    {
      std::lock_guard<std::mutex> lk(S->mu);
      ++S->st.rounds;
      S->st.graph_rounds += S->exec.graph_replays() > replays0;
      S->st.triples += round.triples;
      S->st.launches += (uint64_t)launches;
      S->st.flops += round.gemm_flops;
    }
    if (r) {
      // the round could not be issued: its solves fail
      cudaStreamSynchronize(S->run_st);
      if (rr.ev) cudaEventDestroy(rr.ev);
      for (auto &s : rr.solves) {
        {
          std::lock_guard<std::mutex> lk(S->mu);
          --s->inflight;
          s->next = s->total;
        }
        if (s->inflight == 0) complete(S, s, true);
      }
      continue;
    }
    S->inflight.push_back(rr);
  }
}

}  // namespace
}  // namespace ptb

using namespace ptb;

LIBPT_API size_t libpt_footprint(int kind, size_t oa, size_t va, size_t ob,
                                 size_t vb, int dtype, int precision,
                                 int host_inputs, size_t round_triples) {
  if (kind < 0 || kind > 3) return 0;
  Solve s;
  s.kind = kind;
  s.oa = oa;
  s.va = va;
  s.ob = ob;
  s.vb = vb;
  s.dtype = dtype;
  s.precision = precision;
  s.host = host_inputs != 0;
  if (round_triples)
    return plan_footprint(kind, oa, va, ob, vb, dtype, precision, s.host,
                          round_triples);
  return size_solve(s) ? 0 : s.bytes;
}

LIBPT_API int libpt_server_create(size_t mem_budget, int max_active,
                                  libpt_server **out) {
  if (!out) {
    set_error("libpt_server_create: NULL out");
    return LIBPT_ERR_ARG;
  }
  *out = nullptr;
  auto *S = new libpt_server();
  S->max_active = max_active > 0 ? max_active : 64;
  int r = LIBPT_OK;
  do {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      set_error("libpt_server_create: no CUDA device");
      r = LIBPT_ERR_CUDA;
      break;
    }
    // descriptors of the largest round (fixed graph layout)
    const size_t desc = Executor::bytes_for(ROUND_TRIPLES, JOBS_PER_TRIPLE, true);
    size_t budget = mem_budget ? mem_budget : (size_t)(0.9 * (double)fr);
    budget = up256(std::min(budget, fr > desc + ((size_t)1 << 30)
                                        ? fr - desc - ((size_t)1 << 30)
                                        : (size_t)0));
    if (budget == 0 || cudaMalloc((void **)&S->pool_base, budget) != cudaSuccess) {
      set_error("libpt_server_create: cannot reserve the device pool");
      cudaGetLastError();
      r = LIBPT_ERR_NOMEM;
      break;
    }
    S->pool_bytes = budget;
    S->pool.init(budget);
    if (cudaMalloc((void **)&S->d_desc, desc) != cudaSuccess ||
        cudaMalloc((void **)&S->d_err, sizeof(unsigned)) != cudaSuccess ||
        cudaHostAlloc((void **)&S->h_err, sizeof(unsigned),
                      cudaHostAllocDefault) != cudaSuccess) {
      set_error("libpt_server_create: allocation failed");
      r = LIBPT_ERR_NOMEM;
      break;
    }
    *S->h_err = 0;
    cudaMemset(S->d_err, 0, sizeof(unsigned));
    if (cudaStreamCreateWithFlags(&S->prep_st, cudaStreamNonBlocking) ||
        cudaStreamCreateWithFlags(&S->run_st, cudaStreamNonBlocking) ||
        cudaStreamCreateWithFlags(&S->read_st, cudaStreamNonBlocking)) {
      r = LIBPT_ERR_CUDA;
      break;
    }
    if ((r = S->exec.init(S->run_st, S->d_desc, desc, true, ROUND_TRIPLES,
                          JOBS_PER_TRIPLE)))
      break;
    S->st.pool_bytes = budget;
    S->admitter = std::thread(admit_loop, S);
    S->runner = std::thread(run_loop, S);
  } while (0);
  if (r) {
    libpt_server_destroy(S);
    return r;
  }
  *out = S;
  return LIBPT_OK;
}

LIBPT_API int libpt_server_submit(libpt_server *S, int kind, size_t oa,
                                  size_t va, size_t ob, size_t vb,
                                  const void *const *args, int dtype,
                                  int precision, int host_inputs,
                                  uint64_t *ticket) {
  if (!S || !args || !ticket || kind < 0 || kind > 3 || dtype < 0 ||
      dtype > 1) {
    set_error("libpt_server_submit: bad arguments");
    return LIBPT_ERR_ARG;
  }
  const bool unr = kind == 1 || kind == 3, ft = kind >= 2;
  auto s = std::make_shared<Solve>();
  s->kind = kind;
  s->oa = oa;
  s->va = va;
  s->ob = unr ? ob : oa;
  s->vb = unr ? vb : va;
  s->dtype = dtype;
  s->precision = precision;
  s->host = host_inputs != 0;
  s->args.assign(args, args + (ft ? 10 : 7));
  for (const void *a : s->args)
    if (!a) {
      set_error("libpt_server_submit: NULL tensor argument");
      return LIBPT_ERR_ARG;
    }
  s->t_submit = now_s();
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->stop) {
    set_error("libpt_server_submit: server is stopping");
    return LIBPT_ERR_ARG;
  }
  s->id = S->next_id++;
  S->by_id[s->id] = s;
  S->pending.push_back(s);
  ++S->st.submitted;
  *ticket = s->id;
  S->cv_admit.notify_all();
  return LIBPT_OK;
}

LIBPT_API int libpt_server_wait(libpt_server *S, uint64_t ticket,
                                double timeout_s, double *energy,
                                double *latency_s) {
  if (!S) return LIBPT_ERR_ARG;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->by_id.find(ticket);
  if (it == S->by_id.end()) {
    set_error("libpt_server_wait: unknown ticket");
    return LIBPT_ERR_ARG;
  }
  std::shared_ptr<Solve> s = it->second;
  auto ready = [&] { return s->done; };
  if (timeout_s < 0)
    S->cv_done.wait(lk, ready);
  else if (!S->cv_done.wait_for(
               lk, std::chrono::duration<double>(timeout_s), ready))
    return LIBPT_ERR_TIMEOUT;
  if (energy) *energy = s->energy;
  if (latency_s) *latency_s = s->t_done - s->t_submit;
  if (s->status != LIBPT_OK) set_error(s->error);
  return s->status;
}

LIBPT_API int libpt_server_cancel(libpt_server *S, uint64_t ticket) {
  if (!S) return LIBPT_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->by_id.find(ticket);
  if (it == S->by_id.end()) {
    set_error("libpt_server_cancel: unknown ticket");
    return LIBPT_ERR_ARG;
  }
  std::shared_ptr<Solve> s = it->second;
  if (s->done || s->cancelled) return LIBPT_OK;
  s->cancelled = true;
  // queued behind the solve the admitter holds: leave the queue now (the
  // admitter itself ends the one at the front of the queue)
  auto q = std::find(S->pending.begin(), S->pending.end(), s);
  if (q != S->pending.end() && q != S->pending.begin()) {
    S->pending.erase(q);
    set_error("libpt_server: solve cancelled");
    finish(S, s, LIBPT_ERR_CANCELLED);
  }
  S->cv_admit.notify_all();
  S->cv_run.notify_all();
  return LIBPT_OK;
}

LIBPT_API int libpt_server_solve_times(libpt_server *S, uint64_t ticket,
                                       double *times) {
  if (!S || !times) return LIBPT_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->by_id.find(ticket);
  if (it == S->by_id.end()) {
    set_error("libpt_server_solve_times: unknown ticket");
    return LIBPT_ERR_ARG;
  }
  const Solve &s = *it->second;
  if (!s.done) {
    set_error("libpt_server_solve_times: the solve has not ended");
    return LIBPT_ERR_TIMEOUT;
  }
  // phases that did not happen (a solve refused or cancelled early) take
  // the time of the next one that did
  const double admit = s.t_admit ? s.t_admit : s.t_done;
  const double ready = s.t_ready ? s.t_ready : s.t_done;
  const double first = s.t_first ? s.t_first : s.t_done;
  times[0] = admit - s.t_submit;
  times[1] = ready - admit;
  times[2] = first - ready;
  times[3] = s.t_done - first;
  return LIBPT_OK;
}

LIBPT_API int libpt_server_inputs_released(libpt_server *S, uint64_t ticket,
                                           int *released) {
  if (!S || !released) return LIBPT_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->by_id.find(ticket);
  if (it == S->by_id.end()) {
    set_error("libpt_server_inputs_released: unknown ticket");
    return LIBPT_ERR_ARG;
  }
  *released = it->second->consumed ? 1 : 0;
  return LIBPT_OK;
}

LIBPT_API int libpt_server_stats_get(libpt_server *S, libpt_server_stats *out) {
  if (!S || !out) return LIBPT_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  *out = S->st;
  out->pool_bytes = S->pool_bytes;
  out->bytes_in_use = S->in_use;
  out->peak_bytes_in_use = S->peak;
  return LIBPT_OK;
}

LIBPT_API int libpt_server_destroy(libpt_server *S) {
  if (!S) return LIBPT_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
    S->cv_admit.notify_all();
    S->cv_run.notify_all();
  }
  if (S->admitter.joinable()) S->admitter.join();
  if (S->runner.joinable()) S->runner.join();
  S->exec.destroy();
  for (auto &rr : S->inflight)
    if (rr.ev) cudaEventDestroy(rr.ev);
  if (S->prep_st) cudaStreamDestroy(S->prep_st);
  if (S->run_st) cudaStreamDestroy(S->run_st);
  if (S->read_st) cudaStreamDestroy(S->read_st);
  if (S->pool_base) cudaFree(S->pool_base);
  if (S->d_desc) cudaFree(S->d_desc);
  if (S->d_err) cudaFree(S->d_err);
  if (S->h_err) cudaFreeHost(S->h_err);
  delete S;
  return LIBPT_OK;
}
