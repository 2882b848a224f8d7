// Solve server: continuous batching of independent ground-state and
// time-evolution requests over the C ABI.  Worker threads (one context /
// CUDA stream each) take requests first-fit in arrival order: the oldest
// queued request whose estimated device footprint fits in the budget left
// by the running requests starts when a worker is free; a request passed
// over kMaxBypass times blocks later ones until it fits.  Every request
// keeps its MPO, MPS, environments and Lanczos basis on the device until it
// finishes; the work of different requests overlaps on the GPU through
// their streams.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "mpsgpu.h"

namespace {

constexpr int kMaxBypass = 32;

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Job {
  uint64_t id;
  mpsgpu_request req;
  std::string result_file;
  long long footprint;
  double t_submit;
  int bypassed = 0;
  // read by the engine between two site steps through the const volatile
  // int* of mpsgpu_options; written and read with atomic builtins
  volatile int cancel = 0;
};

void raise_cancel(Job& j) { __atomic_store_n(&j.cancel, 1, __ATOMIC_RELEASE); }
bool is_cancelled(Job& j) { return __atomic_load_n(&j.cancel, __ATOMIC_ACQUIRE) != 0; }

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

// Bytes of the BF16 limb planes of one prepared operand (rows x K, row tile
// RT): six 2-byte planes per entry, rows and K padded to the tiles.
long long split_plane_bytes(long long rows, long long K, long long RT) {
  const long long r = (rows + RT - 1) / RT * RT, k = (K + 15) / 16 * 16;
  return 12 * r * k;
}

}  // namespace

extern "C" long long mpsgpu_request_footprint(const mpsgpu_request* r) {
  if (!r || r->L < 2 || r->D < 1) return 0;
  const int d = 2;
  const bool te = r->kind == MPSGPU_REQUEST_TIME_EVOLUTION;
  const int w = te ? 2 : (r->model == MPSGPU_MODEL_SCHWINGER ? 5 : 3);
  const std::vector<long long> b = bonds(r->L, d, r->D);
  long long mps = 0, env = 0, maxsite = 0;
  for (int k = 0; k < r->L; k++) {
    mps += (long long)d * b[k] * b[k + 1];
    env += 2LL * b[k] * b[k] * w;
    maxsite = std::max(maxsite, (long long)d * b[k] * b[k + 1]);
  }
  const long long D = r->D;
  const long long lanczos = te ? 0 : maxsite * 66;                // basis (m = 64) + work vector
  const long long lzstep = te ? 0 : maxsite + 4096;               // partial sums of the fused step
  const long long temps = 4 * D * D * w * d + 4 * d * D * D;      // contraction and QR workspaces
  const long long mpo = (long long)r->L * d * d * w * w * 5;      // tensor + leg matrices
  // time evolution: the state, its copy (the ket of optimize) and, for the
  // observables, w = 1 environments
  const long long states = te ? 3 * mps : 2 * mps;
  long long bytes = 16 * (states + env + lanczos + lzstep + temps + mpo) + (8 << 20);  // + scratch slack
  if (r->precision == 1) {
    // split-precision products of one site (ground state: every Lanczos
    // product; time evolution: the local vector): the limb planes of L and Rt
    // (made once per site) and of x and T2 (per product), the first product
    // in up to 4 K chunks (FP64), T2 (FP64), and the last product in up to 8
    // K chunks (FP64)
    bytes += split_plane_bytes(D * w, D, 128) + split_plane_bytes(D, D * w, 128) +
             split_plane_bytes(d * D, D, 128) + split_plane_bytes(D * d, D * w, 128) +
             16 * (4 * D * w * d * D + D * d * D * w + 8 * D * d * D);
  }
  return bytes;
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

  // first queued job that fits, under mu; a job passed over kMaxBypass times
  // blocks every later one
  std::deque<std::shared_ptr<Job>>::iterator pick() {
    for (auto it = queue.begin(); it != queue.end(); ++it) {
      if (in_use + (*it)->footprint <= budget) return it;
      if ((*it)->bypassed >= kMaxBypass) return queue.end();
    }
    return queue.end();
  }

  void worker(int wi) {
    mpsgpu_context* ctx = ctxs[wi];
    for (;;) {
      std::shared_ptr<Job> job;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] { return stop || pick() != queue.end(); });
        if (stop) return;
        auto it = pick();
        for (auto jt = queue.begin(); jt != it; ++jt) (*jt)->bypassed++;
        job = *it;
        queue.erase(it);
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

  static mpsgpu_options options_for(Job& job) {
    mpsgpu_options opt;
    mpsgpu_default_options(&opt);
    opt.convtol = job.req.convtol > 0 ? job.req.convtol : 1e-10;
    opt.precision = job.req.precision == 1 ? 1 : 0;
    opt.cancel_flag = &job.cancel;
    return opt;
  }

  int run_ground_state(mpsgpu_context* ctx, Job& job, mpsgpu_result& res) {
    const mpsgpu_request& r = job.req;
    mpsgpu_mpo* mpo = nullptr;
    mpsgpu_mps* mps = nullptr;
    mpsgpu_status st;
    if (r.model == MPSGPU_MODEL_ISING) st = mpsgpu_mpo_ising(ctx, r.L, r.p0, r.p1, r.p2, &mpo);
    else if (r.model == MPSGPU_MODEL_SCHWINGER) st = mpsgpu_mpo_schwinger(ctx, r.L, r.p0, r.p1, 0.0, r.p2, &mpo);
    else st = MPSGPU_INVALID;
    if (st == MPSGPU_OK) st = mpsgpu_mps_random_state(ctx, r.L, 2, r.D, r.seed, &mps);
    if (st == MPSGPU_OK) {
      const mpsgpu_options opt = options_for(job);
      mpsgpu_stats stats{};
      double e = 0.0;
      st = mpsgpu_find_ground_state(ctx, mpo, r.D, 0.0, &opt, mps, &e, &stats);
      res.energy = e;
      res.rounds = stats.rounds;
      res.matvecs = stats.matvecs;
      res.flops = stats.flops;
    }
    if (st == MPSGPU_OK && !job.result_file.empty()) st = mpsgpu_mps_export(ctx, mps, job.result_file.c_str());
    if (mps) mpsgpu_mps_free(ctx, mps);
    if (mpo) mpsgpu_mpo_free(ctx, mpo);
    return st;
  }

  // steps of IsingHamiltonian::getUMPO + Contractor::optimize from |0...0>
  // (the loop of the reference's programs, e.g. flatIsing.cpp:174-205)
  int run_time_evolution(mpsgpu_context* ctx, Job& job, mpsgpu_result& res) {
    const mpsgpu_request& r = job.req;
    if (r.model != MPSGPU_MODEL_ISING || r.steps < 0 || !(r.dt > 0.0)) return MPSGPU_INVALID;
    mpsgpu_mpo *U = nullptr, *H = nullptr;
    mpsgpu_mps* st_ = nullptr;
    mpsgpu_status st = mpsgpu_mpo_ising_evolution(ctx, r.L, r.p0, r.p1, r.p2, r.dt, r.imag, &U);
    if (st == MPSGPU_OK) st = mpsgpu_mpo_ising(ctx, r.L, r.p0, r.p1, r.p2, &H);
    if (st == MPSGPU_OK) st = mpsgpu_mps_product(ctx, r.L, 2, 1, &st_);
    const mpsgpu_options opt = options_for(job);
    const double sx[8] = {0.0, 0.0, 1.0, 0.0, 1.0, 0.0, 0.0, 0.0};  // [[0,1],[1,0]] column-major
    std::vector<double> ex(r.L);
    for (int step = 0; st == MPSGPU_OK && step < r.steps; step++) {
      if (is_cancelled(job)) {
        st = MPSGPU_CANCELLED;
        break;
      }
      mpsgpu_mps* aux = nullptr;
      st = mpsgpu_mps_copy(ctx, st_, &aux);
      mpsgpu_stats stats{};
      if (st == MPSGPU_OK) st = mpsgpu_optimize(ctx, U, aux, st_, r.D, &opt, nullptr, nullptr, &stats);
      if (aux) mpsgpu_mps_free(ctx, aux);
      res.rounds += stats.rounds;
      res.matvecs += stats.matvecs;
      res.flops += stats.flops;
      if (st == MPSGPU_OK && r.imag) st = mpsgpu_mps_gauge(ctx, st_, 'R');
      if (st == MPSGPU_OK && r.obs_sx) {
        st = mpsgpu_expectation_local(ctx, st_, sx, ex.data());
        if (st == MPSGPU_OK) r.obs_sx[step] = ex[r.L / 2];
      }
      if (st == MPSGPU_OK && r.obs_entropy) {
        st = mpsgpu_mps_gauge(ctx, st_, 'L');
        if (st == MPSGPU_OK) st = mpsgpu_entropy(ctx, st_, r.L / 2, &r.obs_entropy[step]);
      }
    }
    if (st == MPSGPU_OK) {
      double re = 0, im = 0, nr = 0, ni = 0;
      st = mpsgpu_contract(ctx, st_, H, st_, &re, &im);
      if (st == MPSGPU_OK) st = mpsgpu_contract(ctx, st_, nullptr, st_, &nr, &ni);
      res.energy = nr != 0.0 ? re / nr : re;
    }
    if (st == MPSGPU_OK && !job.result_file.empty()) st = mpsgpu_mps_export(ctx, st_, job.result_file.c_str());
    if (st_) mpsgpu_mps_free(ctx, st_);
    if (H) mpsgpu_mpo_free(ctx, H);
    if (U) mpsgpu_mpo_free(ctx, U);
    return st;
  }

  int run(mpsgpu_context* ctx, Job& job, mpsgpu_result& res) {
    if (is_cancelled(job)) return MPSGPU_CANCELLED;
    if (job.req.kind == MPSGPU_REQUEST_TIME_EVOLUTION) return run_time_evolution(ctx, job, res);
    if (job.req.kind != MPSGPU_REQUEST_GROUND_STATE) return MPSGPU_INVALID;
    return run_ground_state(ctx, job, res);
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
  if (req->kind != MPSGPU_REQUEST_GROUND_STATE && req->kind != MPSGPU_REQUEST_TIME_EVOLUTION) return MPSGPU_INVALID;
  const long long fp = mpsgpu_request_footprint(req);
  if (fp <= 0) return MPSGPU_BAD_SHAPE;
  if (fp > s->budget) return MPSGPU_OOM;  // can never be admitted
  auto job = std::make_shared<Job>();
  job->req = *req;
  if (req->result_file) job->result_file = req->result_file;
  job->req.result_file = nullptr;
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
      s->cv_work.notify_all();  // a job that blocked the queue may be gone
      return MPSGPU_OK;
    }
  }
  auto a = s->active.find(id);
  if (a == s->active.end()) return MPSGPU_INVALID;
  raise_cancel(*a->second);
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
    for (auto& kv : s->active) raise_cancel(*kv.second);
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
