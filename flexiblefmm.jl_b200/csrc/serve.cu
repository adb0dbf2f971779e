// A continuous-batching request server over the library's own entry points (no counterpart in
// the reference, which evaluates one FMM per call on one thread; this is the serving form of
// the matvec path).
//
// Requests (points, charges, tolerance) are admitted in arrival order onto `slots` worker
// threads, each owning a context (its own CUDA stream) and an operator cache per order that
// stays resident across requests. A request is admitted when a slot is free and its estimated
// device memory fits the budget left by the requests in flight; the front request waits for
// memory rather than being overtaken. Admitted requests build their tree, expansions and
// evaluation on their slot's stream, so the device work of different requests overlaps; device
// buffers come from the stream-ordered allocator, so no request's allocation or release
// synchronises another's stream. Every request's computation is independent of the others and
// deterministic (its box is snapped from its own points to a power-of-two width), so its results
// are the same alone and in any mix, on any slot.
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <tuple>
#include <unordered_map>

#include "passes.cuh"

namespace fmmb {
void set_last_error(const std::string& m);
void fix_cache_base_width(fmmb_cache* c, double w);
}

namespace {

using namespace fmmb;
using clk = std::chrono::steady_clock;

struct Job {
  fmmb_request r;
  int64_t id = 0;
  int p = 0, precision = 0, slot = -1;
  int64_t bytes = 0;
  clk::time_point t_submit, t_start, t_done;
  bool done = false;
  int status = FMMB_OK;
  std::string error;
};

// the order for a requested tolerance: the smallest p whose relative L2 error against direct sums
// stays below it. Laplace3D potential: measured with the CPU oracle (ppl = 64, uniform and
// 4-cluster points of 2·10⁵, uniform points of 10⁶ for p = 10..13; the worst of them).
// Stokeslet3D velocity: measured on the device path (ppl = 64 and 200, 2·10⁵ points uniform in
// the cube and on the jittered unit sphere; the worst of them). Yukawa3D takes the Laplace3D
// table (the screening only lowers the far field's share of the error).
int order_for_tol(double tol, int kernel) {
  static const double lap[PMAX + 1] = {1, 1, 9.5e-3, 3.1e-3, 1.0e-3, 3.6e-4, 1.3e-4, 5.6e-5, 2.4e-5, 7.6e-6, 3.8e-6,
                                       7.3e-7, 3.8e-7, 1.8e-7, 1.6e-7, 8.5e-8, 4.5e-8, 2.0e-8, 8.4e-9, 5.0e-9, 2.7e-9};
  static const double sto[PMAX + 1] = {1, 1, 3.7e-2, 1.3e-2, 4.8e-3, 1.9e-3, 7.5e-4, 3.4e-4, 1.4e-4, 6.9e-5, 3.1e-5,
                                       1.6e-5, 7.8e-6, 4.1e-6, 2.2e-6, 9.6e-7, 5.9e-7, 2.7e-7, 2.2e-7, 1.4e-7, 8.1e-8};
  const double* err = kernel == FMMB_KERNEL_STOKESLET3D ? sto : lap;
  for (int p = 2; p <= PMAX; ++p)
    if (err[p] <= tol) return p;
  return PMAX;
}

// an upper estimate of the device memory one request holds (tree, lists, expansions, staging);
// a Stokeslet request holds four expansions per node and three densities per point
int64_t bytes_estimate(int64_t n, int p, int ppl, int precision, int kernel) {
  const int64_t ld = ld_of(p), kp = (int64_t)((p + 1) * (p + 1) + 15) / 16 * 16;
  const int64_t nodes = 4 * n / std::max(ppl, 1) + 4096, nexp = kernel == FMMB_KERNEL_STOKESLET3D ? 4 : 1;
  int64_t b = n * (nexp == 4 ? 448 : 256);               // points in and sorted, keys, perm, densities, outputs
  b += nodes * (2 * nexp * ld * 8 + 27 * 4 + 64);        // multipoles, partial locals, colleagues, node arrays
  b += nodes * 190 * 8;                                  // far pairs
  if (nexp == 4) b += nodes / 8 * 4 * 8 * ld * 8;        // M2M / L2L staging of the largest level
  if (precision == FMMB_PRECISION_MIXED) b += nodes * kp * 8 + nodes * 4;   // FP16 copies, scales
  return b + (16 << 20);
}

double seconds(clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); }

}  // namespace

struct fmmb_server {
  int device = 0;
  int nslots = 1;
  int ppl = 64;
  int64_t budget = 0, in_use = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Job*> pending;
  std::unordered_map<int64_t, std::unique_ptr<Job>> jobs;
  int64_t next_id = 1;
  bool stop = false;      // no new submissions
  bool stop_now = false;  // the workers leave
  std::vector<fmmb_ctx*> ctx;
  std::vector<std::map<std::tuple<int, int, double>, fmmb_cache*>> caches;   // per slot, by (kernel, p, κ)
  std::vector<std::thread> workers;
};

namespace {

// one request on a slot: plan, state, matvec through the host-pointer entry points of the
// slot's context, then release; returns the status
int run_job(fmmb_server& S, int slot, Job& j, std::string& err) {
  const int kernel = j.r.kernel;
  fmmb_cache* cache = nullptr;
  {
    auto& cs = S.caches[slot];
    const double kappa = kernel == FMMB_KERNEL_YUKAWA3D ? j.r.kappa : 0.0;
    const auto key = std::make_tuple(kernel, j.p, kappa);
    auto it = cs.find(key);
    if (it == cs.end()) {
      fmmb_method_desc m{FMMB_METHOD_SPHERICAL_HARMONICS, kernel, j.p, 0, 0.0, kappa};
      int rc = fmmb_cache_create(S.ctx[slot], &m, &cache);
      if (rc) { err = fmmb_last_error(); return rc; }
      // a request's box depends on its own points only (not on which request the slot's cache
      // saw first), so its results are the same on any slot
      fix_cache_base_width(cache, 1.0);
      cs[key] = cache;
    } else {
      cache = it->second;
    }
  }
  fmmb_tree_opts o{};
  o.ppl = j.r.ppl > 0 ? j.r.ppl : S.ppl;
  o.max_levels = 30;
  fmmb_plan* plan = nullptr;
  fmmb_state* st = nullptr;
  int rc = fmmb_plan_create(cache, j.r.xyz, j.r.n, &o, &plan);
  if (!rc) rc = fmmb_state_create(plan, j.precision, &st);
  if (!rc) {
    if (kernel == FMMB_KERNEL_STOKESLET3D) rc = fmmb_stokes_eval(st, j.r.xyz, j.r.tau, j.r.n, j.r.pot);
    else rc = fmmb_matvec(st, j.r.xyz, j.r.tau, j.r.n, j.r.outputs, j.r.pot, j.r.grad);
  }
  if (rc) err = fmmb_last_error();
  if (st) fmmb_state_destroy(st);
  if (plan) fmmb_plan_destroy(plan);
  return rc;
}

void worker(fmmb_server* S, int slot) {
  for (;;) {
    Job* j = nullptr;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      // admission in arrival order: the front request waits for memory rather than being overtaken
      S->cv_work.wait(lk, [&] {
        return S->stop_now || (!S->pending.empty() &&
                               (S->in_use == 0 || S->in_use + S->pending.front()->bytes <= S->budget));
      });
      if (S->stop_now || (S->pending.empty() && S->stop)) return;
      j = S->pending.front();
      S->pending.pop_front();
      S->in_use += j->bytes;
      j->slot = slot;
      j->t_start = clk::now();
    }
    S->cv_work.notify_all();   // the next request may fit too
    std::string err;
    const int rc = run_job(*S, slot, *j, err);
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->in_use -= j->bytes;
      j->status = rc;
      j->error = err;
      j->t_done = clk::now();
      j->done = true;
    }
    S->cv_done.notify_all();
    S->cv_work.notify_all();
  }
}

}  // namespace

extern "C" {

int fmmb_server_create(int device, const fmmb_server_opts* opts, fmmb_server** out) {
  if (!opts || !out) return FMMB_ERR_ARGUMENT;
  if (opts->slots < 1 || opts->slots > 64 || opts->ppl < 1 || opts->hbm_budget < 0) return FMMB_ERR_ARGUMENT;
  std::unique_ptr<fmmb_server> S(new fmmb_server());
  S->device = device;
  S->nslots = opts->slots;
  S->ppl = opts->ppl;
  S->budget = opts->hbm_budget;
  if (S->budget == 0) {
    size_t fr = 0, tot = 0;
    if (cudaSetDevice(device) != cudaSuccess || cudaMemGetInfo(&fr, &tot) != cudaSuccess) return FMMB_ERR_DEVICE;
    S->budget = (int64_t)(0.8 * (double)fr);
  }
  for (int i = 0; i < S->nslots; ++i) {
    fmmb_ctx* c = nullptr;
    const int rc = fmmb_ctx_create(device, &c);
    if (rc) {
      for (auto* x : S->ctx) fmmb_ctx_destroy(x);
      return rc;
    }
    S->ctx.push_back(c);
  }
  S->caches.resize(S->nslots);
  for (int i = 0; i < S->nslots; ++i) S->workers.emplace_back(worker, S.get(), i);
  *out = S.release();
  return FMMB_OK;
}

int fmmb_server_submit(fmmb_server* S, const fmmb_request* r, int64_t* ticket) {
  if (!S || !r || !ticket) return FMMB_ERR_ARGUMENT;
  const bool stokes = r->kernel == FMMB_KERNEL_STOKESLET3D, yukawa = r->kernel == FMMB_KERNEL_YUKAWA3D;
  if (r->kernel != FMMB_KERNEL_LAPLACE3D && !stokes && !yukawa) return FMMB_ERR_UNSUPPORTED;
  if (yukawa && !(std::isfinite(r->kappa) && r->kappa > 0)) return FMMB_ERR_ARGUMENT;
  if (yukawa && r->precision == FMMB_PRECISION_MIXED) return FMMB_ERR_UNSUPPORTED;
  if (!r->xyz || !r->tau || r->n <= 0 || r->ppl < 0) return FMMB_ERR_ARGUMENT;
  if (stokes) {
    // Stokeslets in tau (3×n), velocities in pot (3×n), on the FP64 path
    if (!r->pot) return FMMB_ERR_ARGUMENT;
    if (r->precision == FMMB_PRECISION_MIXED) return FMMB_ERR_UNSUPPORTED;
  } else {
    if (r->outputs < 1 || r->outputs > 3) return FMMB_ERR_ARGUMENT;
    if (((r->outputs & FMMB_OUTPUT_POTENTIAL) && !r->pot) || ((r->outputs & FMMB_OUTPUT_GRADIENT) && !r->grad))
      return FMMB_ERR_ARGUMENT;
  }
  if (!(r->tol > 0 && r->tol < 1) && r->p == 0) return FMMB_ERR_ARGUMENT;
  std::unique_ptr<Job> j(new Job());
  j->r = *r;
  j->p = r->p > 0 ? r->p : order_for_tol(r->tol, r->kernel);
  if (j->p < 1 || j->p > PMAX) return FMMB_ERR_ARGUMENT;
  // the precision path: FP64 below 1e-8 (or where the mixed path has no kernel), mixed above
  if (stokes || yukawa) j->precision = FMMB_PRECISION_FP64;   // the paths these kernels have
  else
    j->precision = r->precision >= 0 ? r->precision
                                     : ((r->tol < 1e-8 || (j->p + 1) * (j->p + 1) > 144) ? FMMB_PRECISION_FP64 : FMMB_PRECISION_MIXED);
  j->bytes = bytes_estimate(r->n, j->p, r->ppl > 0 ? r->ppl : S->ppl, j->precision, r->kernel);
  j->t_submit = clk::now();
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->stop) return FMMB_ERR_ARGUMENT;
  j->id = S->next_id++;
  *ticket = j->id;
  S->pending.push_back(j.get());
  S->jobs[j->id] = std::move(j);
  S->cv_work.notify_one();
  return FMMB_OK;
}

int fmmb_server_wait(fmmb_server* S, int64_t ticket, double timeout_s, fmmb_request_info* info) {
  if (!S) return FMMB_ERR_ARGUMENT;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->jobs.find(ticket);
  if (it == S->jobs.end()) return FMMB_ERR_ARGUMENT;
  Job* j = it->second.get();
  auto pred = [&] { return j->done; };
  if (timeout_s < 0) S->cv_done.wait(lk, pred);
  else if (!S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred)) return FMMB_ERR_TIMEOUT;
  if (info) {
    info->status = j->status;
    info->p = j->p;
    info->precision = j->precision;
    info->slot = j->slot;
    info->queued_s = seconds(j->t_submit, j->t_start);
    info->run_s = seconds(j->t_start, j->t_done);
    info->latency_s = seconds(j->t_submit, j->t_done);
    info->bytes_estimate = j->bytes;
  }
  const int status = j->status;
  fmmb::set_last_error(j->error);
  S->jobs.erase(it);   // a ticket is waited for once
  return status;
}

int fmmb_server_destroy(fmmb_server* S) {
  if (!S) return FMMB_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;            // no new submissions; the queued requests still run
  }
  {
    std::unique_lock<std::mutex> lk(S->mu);
    S->cv_done.wait(lk, [&] { return S->pending.empty() && S->in_use == 0; });
    S->stop_now = true;
  }
  S->cv_work.notify_all();
  for (auto& t : S->workers) t.join();
  for (auto& cs : S->caches)
    for (auto& kv : cs) fmmb_cache_destroy(kv.second);
  for (auto* c : S->ctx) fmmb_ctx_destroy(c);
  delete S;
  return FMMB_OK;
}

}  // extern "C"
