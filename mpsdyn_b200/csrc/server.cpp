// Solve server: continuous batching of independent ground-state requests
// over the C ABI.  Worker threads (one context / CUDA stream each) take
// requests in arrival order; the head request is admitted when a worker is
// free and its estimated device footprint fits in the budget left by the
// running requests.  Every request keeps its MPO, MPS, environments and
// Lanczos basis on the device until it finishes; the work of different
// requests overlaps on the GPU through their streams.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "mpsgpu.h"

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Job {
  uint64_t id;
  mpsgpu_request req;
  long long footprint;
  double t_submit;
  volatile int cancel = 0;
};

// Bond schedule D_k = min(d^k, d^(L-k), D) as the initial states use it.
std::vector<long long> bonds(int L, int d, int D) {
  std::vector<long long> b(L + 1);
  for (int k = 0; k <= L; k++) {
    long long x = 1;
    const int e = std::min(k, L - k);
    for (int i = 0; i < e && x < D; i++) x *= d;
    b[k] = std::min<long long>(x, D);
  }
  return b;
}

}  // namespace

extern "C" long long mpsgpu_request_footprint(const mpsgpu_request* r) {
  if (!r || r->L < 2 || r->D < 1) return 0;
  const int d = 2;
  const int w = r->model == MPSGPU_MODEL_SCHWINGER ? 5 : 3;
  const std::vector<long long> b = bonds(r->L, d, r->D);
  long long mps = 0, env = 0, maxsite = 0;
  for (int k = 0; k < r->L; k++) {
    mps += (long long)d * b[k] * b[k + 1];
    env += 2LL * b[k] * b[k] * w;
    maxsite = std::max(maxsite, (long long)d * b[k] * b[k + 1]);
  }
  const long long D = r->D;
  const long long lanczos = maxsite * 66;            // basis (m = 64) + work vector
  const long long temps = 4 * D * D * w * d + 4 * d * D * D;  // contraction and QR workspaces
  const long long mpo = (long long)r->L * d * d * w * w * 5;  // tensor + leg matrices
  return 16 * (2 * mps + env + lanczos + temps + mpo) + (8 << 20);  // + scratch slack
}

struct mpsgpu_server {
  int device = 0;
  long long budget = 0;
  long long in_use = 0;
  double t0 = 0;
  uint64_t next_id = 1;
  bool stop = false;
  int running = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_idle;
  std::deque<std::shared_ptr<Job>> queue;
  std::map<uint64_t, std::shared_ptr<Job>> active;
  std::vector<mpsgpu_result> done;
  std::vector<std::thread> workers;
  std::vector<mpsgpu_context*> ctxs;

  void worker(int wi) {
    mpsgpu_context* ctx = ctxs[wi];
    for (;;) {
      std::shared_ptr<Job> job;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] {
          return stop || (!queue.empty() && in_use + queue.front()->footprint <= budget);
        });
        if (stop) return;
        job = queue.front();
        queue.pop_front();
        in_use += job->footprint;
        running++;
        active[job->id] = job;
      }
      mpsgpu_result res{};
      res.id = job->id;
      res.t_submit = job->t_submit - t0;
      res.t_start = now_s() - t0;
      res.footprint_bytes = job->footprint;
      res.status = run(ctx, *job, res);
      res.t_end = now_s() - t0;
      {
        std::lock_guard<std::mutex> lk(mu);
        in_use -= job->footprint;
        running--;
        active.erase(job->id);
        done.push_back(res);
      }
      cv_work.notify_all();
      cv_idle.notify_all();
    }
  }

  int run(mpsgpu_context* ctx, Job& job, mpsgpu_result& res) {
    const mpsgpu_request& r = job.req;
    if (job.cancel) return MPSGPU_CANCELLED;
    mpsgpu_mpo* mpo = nullptr;
    mpsgpu_mps* mps = nullptr;
    mpsgpu_status st;
    if (r.model == MPSGPU_MODEL_ISING) st = mpsgpu_mpo_ising(ctx, r.L, r.p0, r.p1, r.p2, &mpo);
    else if (r.model == MPSGPU_MODEL_SCHWINGER) st = mpsgpu_mpo_schwinger(ctx, r.L, r.p0, r.p1, 0.0, r.p2, &mpo);
    else st = MPSGPU_INVALID;
    if (st == MPSGPU_OK) st = mpsgpu_mps_random_state(ctx, r.L, 2, r.D, r.seed, &mps);
    if (st == MPSGPU_OK) {
      mpsgpu_options opt;
      mpsgpu_default_options(&opt);
      opt.convtol = r.convtol > 0 ? r.convtol : 1e-10;
      opt.precision = r.precision == 1 ? 1 : 0;
      opt.cancel_flag = &job.cancel;
      mpsgpu_stats stats{};
      double e = 0.0;
      st = mpsgpu_find_ground_state(ctx, mpo, r.D, 0.0, &opt, mps, &e, &stats);
      res.energy = e;
      res.rounds = stats.rounds;
      res.matvecs = stats.matvecs;
      res.flops = stats.flops;
    }
    if (mps) mpsgpu_mps_free(ctx, mps);
    if (mpo) mpsgpu_mpo_free(ctx, mpo);
    return st;
  }
};

extern "C" {

mpsgpu_status mpsgpu_server_create(int device, int slots, long long hbm_budget_bytes, mpsgpu_server** out) {
  if (!out || slots < 1 || slots > 256 || hbm_budget_bytes <= 0) return MPSGPU_INVALID;
  *out = nullptr;
  auto* s = new (std::nothrow) mpsgpu_server();
  if (!s) return MPSGPU_OOM;
  s->device = device;
  s->budget = hbm_budget_bytes;
  s->t0 = now_s();
  for (int i = 0; i < slots; i++) {
    mpsgpu_context* c = nullptr;
    mpsgpu_status st = mpsgpu_create(device, &c);
    if (st != MPSGPU_OK) {
      for (auto* x : s->ctxs) mpsgpu_destroy(x);
      delete s;
      return st;
    }
    s->ctxs.push_back(c);
  }
  for (int i = 0; i < slots; i++) s->workers.emplace_back(&mpsgpu_server::worker, s, i);
  *out = s;
  return MPSGPU_OK;
}

mpsgpu_status mpsgpu_server_submit(mpsgpu_server* s, const mpsgpu_request* req, uint64_t* id) {
  if (!s || !req) return MPSGPU_INVALID;
  const long long fp = mpsgpu_request_footprint(req);
  if (fp <= 0) return MPSGPU_BAD_SHAPE;
  if (fp > s->budget) return MPSGPU_OOM;  // can never be admitted
  auto job = std::make_shared<Job>();
  job->req = *req;
  job->footprint = fp;
  job->t_submit = now_s();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    job->id = s->next_id++;
    s->queue.push_back(job);
  }
  if (id) *id = job->id;
  s->cv_work.notify_all();
  return MPSGPU_OK;
}

mpsgpu_status mpsgpu_server_poll(mpsgpu_server* s, mpsgpu_result* out, int cap, int* n) {
  if (!s || !n || (cap > 0 && !out)) return MPSGPU_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  const int k = std::min<int>(cap, (int)s->done.size());
  for (int i = 0; i < k; i++) out[i] = s->done[i];
  s->done.erase(s->done.begin(), s->done.begin() + k);
  *n = k;
  return MPSGPU_OK;
}

mpsgpu_status mpsgpu_server_cancel(mpsgpu_server* s, uint64_t id) {
  if (!s) return MPSGPU_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  for (auto it = s->queue.begin(); it != s->queue.end(); ++it) {
    if ((*it)->id == id) {
      mpsgpu_result res{};
      res.id = id;
      res.status = MPSGPU_CANCELLED;
      res.t_submit = (*it)->t_submit - s->t0;
      res.t_start = res.t_end = now_s() - s->t0;
      res.footprint_bytes = (*it)->footprint;
      s->done.push_back(res);
      s->queue.erase(it);
      s->cv_idle.notify_all();
      return MPSGPU_OK;
    }
  }
  auto a = s->active.find(id);
  if (a == s->active.end()) return MPSGPU_INVALID;
  a->second->cancel = 1;
  return MPSGPU_OK;
}

mpsgpu_status mpsgpu_server_drain(mpsgpu_server* s, double timeout_s) {
  if (!s) return MPSGPU_INVALID;
  std::unique_lock<std::mutex> lk(s->mu);
  auto idle = [&] { return s->queue.empty() && s->running == 0; };
  if (timeout_s <= 0) {
    s->cv_idle.wait(lk, idle);
    return MPSGPU_OK;
  }
  return s->cv_idle.wait_for(lk, std::chrono::duration<double>(timeout_s), idle) ? MPSGPU_OK : MPSGPU_TIMEOUT;
}

mpsgpu_status mpsgpu_server_destroy(mpsgpu_server* s) {
  if (!s) return MPSGPU_INVALID;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (auto& kv : s->active) kv.second->cancel = 1;
    s->queue.clear();
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto& t : s->workers) t.join();
  for (auto* c : s->ctxs) mpsgpu_destroy(c);
  delete s;
  return MPSGPU_OK;
}

}  // extern "C"
