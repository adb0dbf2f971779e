// A continuous-batching request server over the library's own entry points (no counterpart in
// the reference, which evaluates one FMM per call on one thread; this is the serving form of
// the matvec path).
//
// Requests (points, charges, tolerance) are admitted in arrival order onto `slots` worker
// threads, each owning a context (its own CUDA stream) and an operator cache per order that
// stays resident across requests. A request is admitted when a slot is free and its estimated
// device memory fits the budget left by the requests in flight; the front request waits for
// memory rather than being overtaken. A slot takes the front request together with later queued
// requests of the same kind (kernel, order, precision path, κ, ppl, outputs) that fit the budget,
// up to a request and point cap, and runs the group as one batch plan: one tree build, one list
// build and one launch per pass for all of them (the per-request cost of a plan, its host
// synchronisations and small launches, is paid once per group). Admitted groups build their
// trees, expansions and evaluations on their slot's stream, so the device work of different
// groups overlaps; device
// buffers come from the stream-ordered allocator, so no request's allocation or release
// synchronises another's stream. Every request's computation is independent of the others and
// deterministic (its box is snapped from its own points to a power-of-two width, and a batch
// plan computes each of its instances bitwise as the instance's own plan would), so its results
// are the same alone and in any mix or group, on any slot.
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
  int p = 0, precision = 0, slot = -1, ppl = 64;
  int64_t bytes = 0;
  clk::time_point t_submit, t_start, t_done;
  double plan_s = 0, matvec_s = 0, device_s = 0;
  int group = 1;
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

// the leaf size of a request that names none, by order and precision path (measured on the
// device, 2·10⁵ uniform and 4-cluster points, Laplace3D: the matvec time is flat or falling in ppl
// up to these and the error unchanged; at p = 20 on the FP64 path ppl = 512 takes 12.5 / 20.6 ms
// against 19.9 / 69.2 ms at 64, uniform / clustered). The mixed path's tensor-core M2L is cheap
// enough that 64 stays best.
int auto_ppl(int p, int precision) {
  if (precision == FMMB_PRECISION_MIXED || p <= 8) return 64;
  if (p <= 13) return 128;
  if (p <= 17) return 256;
  return 512;
}

double seconds(clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); }

}  // namespace

struct fmmb_server {
  int device = 0;
  int nslots = 1;
  int ppl = 64;
  int group_max = 64;
  int64_t group_points = 4000000;
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

// the kind of a request: requests of one kind can share a batch plan
std::tuple<int, int, int, double, int, int> kind(const fmmb_server& S, const Job& j) {
  return std::make_tuple(j.r.kernel, j.p, j.precision, j.r.kernel == FMMB_KERNEL_YUKAWA3D ? j.r.kappa : 0.0,
                         j.ppl, j.r.kernel == FMMB_KERNEL_STOKESLET3D ? 0 : j.r.outputs);
}

// a group of requests of one kind on a slot: one plan (a batch plan for more than one), one
// state, one matvec through the host-pointer entry points of the slot's context, the outputs
// copied to each request's buffers; then release. Returns the status
int run_group(fmmb_server& S, int slot, std::vector<Job*>& g, std::string& err) {
  Job& j0 = *g[0];
  const int kernel = j0.r.kernel;
  const bool stokes = kernel == FMMB_KERNEL_STOKESLET3D;
  fmmb_cache* cache = nullptr;
  {
    auto& cs = S.caches[slot];
    const double kappa = kernel == FMMB_KERNEL_YUKAWA3D ? j0.r.kappa : 0.0;
    const auto key = std::make_tuple(kernel, j0.p, kappa);
    auto it = cs.find(key);
    if (it == cs.end()) {
      fmmb_method_desc m{FMMB_METHOD_SPHERICAL_HARMONICS, kernel, j0.p, 0, 0.0, kappa};
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
  o.ppl = j0.ppl;
  o.max_levels = 30;
  // the group's inputs and outputs, concatenated in group order (one request: its own buffers)
  const size_t ng = g.size();
  const int dens = stokes ? 3 : 1;
  std::vector<int64_t> counts(ng);
  int64_t n = 0;
  for (size_t i = 0; i < ng; ++i) { counts[i] = g[i]->r.n; n += g[i]->r.n; }
  const int outputs = stokes ? 0 : j0.r.outputs;
  const int pot_w = stokes ? 3 : 1;
  cudaStream_t stream = nullptr;
  fmmb_ctx_stream(S.ctx[slot], (void**)&stream);
  // a group: its inputs copied request by request into device buffers on the slot's stream (no
  // host-side concatenation), its outputs copied back into each request's buffers
  double *dx = nullptr, *dt = nullptr, *dp = nullptr, *dg = nullptr;
  int rc = FMMB_OK;
  auto dev_alloc = [&](double** q, int64_t count) {
    if (!rc && cudaMallocAsync((void**)q, sizeof(double) * count, stream) != cudaSuccess) {
      rc = FMMB_ERR_DEVICE;
      err = "device memory for a request group";
    }
  };
  const bool want_pot = stokes || (outputs & FMMB_OUTPUT_POTENTIAL), want_grad = !stokes && (outputs & FMMB_OUTPUT_GRADIENT);
  if (ng > 1) {
    dev_alloc(&dx, 3 * n);
    dev_alloc(&dt, dens * n);
    if (want_pot) dev_alloc(&dp, pot_w * n);
    if (want_grad) dev_alloc(&dg, 3 * n);
    int64_t off = 0;
    for (Job* j : g) {
      if (!rc && (cudaMemcpyAsync(dx + 3 * off, j->r.xyz, sizeof(double) * 3 * j->r.n, cudaMemcpyHostToDevice, stream) ||
                  cudaMemcpyAsync(dt + dens * off, j->r.tau, sizeof(double) * dens * j->r.n, cudaMemcpyHostToDevice,
                                  stream))) {
        rc = FMMB_ERR_DEVICE;
        err = "copying a request's inputs";
      }
      off += j->r.n;
    }
  }
  fmmb_plan* plan = nullptr;
  fmmb_state* st = nullptr;
  const clk::time_point t0 = clk::now();
  if (!rc)
    rc = ng > 1 ? fmmb_batch_plan_create_dev(cache, dx, counts.data(), (int64_t)ng, &o, nullptr, &plan)
                : fmmb_plan_create(cache, j0.r.xyz, n, &o, &plan);
  if (!rc) rc = fmmb_state_create(plan, j0.precision, &st);
  const clk::time_point t1 = clk::now();
  double plan_s = seconds(t0, t1), matvec_s = 0, device_s = 0;
  if (!rc) {
    // the matvec's span on the slot's stream, beside its host time
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    const bool ev = cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess &&
                    cudaEventRecord(e0, stream) == cudaSuccess;
    if (ng == 1) {
      if (stokes) rc = fmmb_stokes_eval(st, j0.r.xyz, j0.r.tau, n, j0.r.pot);
      else rc = fmmb_matvec(st, j0.r.xyz, j0.r.tau, n, outputs, j0.r.pot, j0.r.grad);
    } else {
      if (stokes) rc = fmmb_stokes_eval_dev(st, dx, dt, n, dp);
      else rc = fmmb_matvec_dev(st, dx, dt, n, outputs, dp, dg);
      if (!rc) rc = fmmb_state_synchronize(st);
    }
    float ms = 0;
    if (ev && cudaEventRecord(e1, stream) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess &&
        cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess)
      device_s = ms * 1e-3;
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (!rc && ng > 1) {
      int64_t off = 0;
      for (Job* j : g) {
        if ((want_pot && cudaMemcpyAsync(j->r.pot, dp + pot_w * off, sizeof(double) * pot_w * j->r.n, cudaMemcpyDeviceToHost,
                                         stream)) ||
            (want_grad && cudaMemcpyAsync(j->r.grad, dg + 3 * off, sizeof(double) * 3 * j->r.n, cudaMemcpyDeviceToHost,
                                          stream))) {
          rc = FMMB_ERR_DEVICE;
          err = "copying a request's outputs";
          break;
        }
        off += j->r.n;
      }
      if (cudaStreamSynchronize(stream) != cudaSuccess && !rc) {
        rc = FMMB_ERR_DEVICE;
        err = "copying a request's outputs";
      }
    }
    matvec_s = seconds(t1, clk::now());
  }
  if (rc && err.empty()) err = fmmb_last_error();
  if (st) fmmb_state_destroy(st);
  if (plan) fmmb_plan_destroy(plan);
  for (double* q : {dx, dt, dp, dg})
    if (q) cudaFreeAsync(q, stream);
  for (Job* j : g) {
    j->plan_s = plan_s / ng;
    j->matvec_s = matvec_s / ng;
    j->device_s = device_s / ng;
    j->group = (int)ng;
  }
  return rc;
}

void worker(fmmb_server* S, int slot) {
  std::vector<Job*> group;
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
      group.assign(1, j);
      // later queued requests of the same kind join while they fit the caps and the budget
      int64_t pts = j->r.n;
      const auto k = kind(*S, *j);
      for (auto it = S->pending.begin(); it != S->pending.end() && (int)group.size() < S->group_max;) {
        Job* c = *it;
        if (kind(*S, *c) == k && pts + c->r.n <= S->group_points && S->in_use + c->bytes <= S->budget) {
          S->in_use += c->bytes;
          pts += c->r.n;
          group.push_back(c);
          it = S->pending.erase(it);
        } else {
          ++it;
        }
      }
      const clk::time_point now = clk::now();
      for (Job* c : group) { c->slot = slot; c->t_start = now; }
    }
    S->cv_work.notify_all();   // the next request may fit too
    std::string err;
    const int rc = run_group(*S, slot, group, err);
    {
      std::lock_guard<std::mutex> lk(S->mu);
      const clk::time_point now = clk::now();
      for (Job* c : group) {
        S->in_use -= c->bytes;
        c->status = rc;
        c->error = err;
        c->t_done = now;
        c->done = true;
      }
    }
    S->cv_done.notify_all();
    S->cv_work.notify_all();
  }
}

}  // namespace

extern "C" {

int fmmb_server_create(int device, const fmmb_server_opts* opts, fmmb_server** out) {
  if (!opts || !out) return FMMB_ERR_ARGUMENT;
  if (opts->slots < 1 || opts->slots > 64 || opts->ppl < 0 || opts->hbm_budget < 0) return FMMB_ERR_ARGUMENT;
  std::unique_ptr<fmmb_server> S(new fmmb_server());
  S->device = device;
  S->nslots = opts->slots;
  S->ppl = opts->ppl;
  S->budget = opts->hbm_budget;
  if (opts->group_max < 0 || opts->group_points < 0) return FMMB_ERR_ARGUMENT;
  S->group_max = opts->group_max > 0 ? opts->group_max : 64;
  S->group_points = opts->group_points > 0 ? opts->group_points : 4000000;
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
  if (stokes) j->precision = FMMB_PRECISION_FP64;   // the path this kernel has
  else
    j->precision = r->precision >= 0 ? r->precision
                                     : ((r->tol < 1e-8 || (j->p + 1) * (j->p + 1) > 144) ? FMMB_PRECISION_FP64 : FMMB_PRECISION_MIXED);
  j->ppl = r->ppl > 0 ? r->ppl : (S->ppl > 0 ? S->ppl : auto_ppl(j->p, j->precision));
  j->bytes = bytes_estimate(r->n, j->p, j->ppl, j->precision, r->kernel);
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
    info->plan_s = j->plan_s;
    info->matvec_s = j->matvec_s;
    info->device_s = j->device_s;
    info->group = j->group;
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
