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
// deterministic: its results are the same alone and in any mix.
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "passes.cuh"

namespace {

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

// the order for a requested tolerance: the smallest p whose relative L2 error against direct
// sums (uniform and clustered points, ppl = 64, the CPU oracle) stays below the tolerance
int order_for_tol(double tol) {
  static const double err[] = {0, 0, 1.2e-2, 4.9e-3, 2.1e-3, 9.6e-4, 4.5e-4, 2.2e-4, 1.0e-4, 4.9e-5, 2.3e-5,
                               1.1e-5, 5.3e-6, 2.5e-6, 1.2e-6, 5.7e-7, 2.7e-7, 1.3e-7, 6.2e-8, 3.0e-8, 1.4e-8};
  (void)err;
  return 0;
}

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
  bool stop = false;
  std::vector<fmmb_ctx*> ctx;
  std::vector<std::map<int, fmmb_cache*>> caches;
  std::vector<std::thread> workers;
};

// @@SERVER_BODY@@
