// spiffe_b200/csrc/batch.cu -- many independent problems at once.
//
// spiffe runs one problem per process (spiffe.c:85-365); a parameter scan or
// a stream of requests is many small problems, each of which leaves most of
// a B200 idle.  spiffe_gpu_batch_run advances a set of instances
// concurrently: every instance keeps its own stream and device state, host
// worker threads take instances from a shared round-robin queue and advance
// each by a chunk of integration steps, so the kernels of different
// instances overlap on the device while each instance's steps stay in
// order.  An instance is held by one thread at a time, so the per-instance
// host state needs no lock; the queue hand-over orders one chunk's host
// work before the next.
#include "../../include/spiffe_b200.h"

#include <algorithm>
#include <chrono>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

// the runtime's error channel (thread-local message)
extern "C" int spiffe_set_error(int code, const char *msg);

extern "C" int spiffe_gpu_batch_run(spiffe_gpu_instance *const *inst, int32_t n, const int64_t *steps,
                                    int32_t workers, int64_t chunk, double *done_ms)
{
  if (n < 0 || (n > 0 && (!inst || !steps)) || workers < 1)
    return spiffe_set_error(SPIFFE_ERR_INVALID, "bad argument");
  for (int32_t i = 0; i < n; i++)
    if (!inst[i] || steps[i] < 0)
      return spiffe_set_error(SPIFFE_ERR_INVALID, "null instance or negative step count");
  const auto t0 = std::chrono::steady_clock::now();
  const auto elapsed_ms = [&]() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  };
  std::vector<int64_t> left(steps, steps + n);
  std::deque<int32_t> queue;
  for (int32_t i = 0; i < n; i++) {
    if (left[i] > 0)
      queue.push_back(i);
    else if (done_ms)
      done_ms[i] = 0;
  }
  std::mutex mu;
  int first_rc = 0;
  std::string first_msg;
  auto worker = [&]() {
    for (;;) {
      int32_t i;
      int64_t k;
      {
        std::lock_guard<std::mutex> g(mu);
        if (queue.empty() || first_rc)
          return;
        i = queue.front();
        queue.pop_front();
        k = chunk > 0 ? std::min(chunk, left[i]) : left[i];
      }
      int rc = spiffe_gpu_run_steps(inst[i], k);
      bool finished = false;
      {
        std::lock_guard<std::mutex> g(mu);
        left[i] -= k;
        if (rc == 0 && left[i] > 0)
          queue.push_back(i);
        else
          finished = rc == 0;
      }
      if (finished) {
        rc = spiffe_gpu_synchronize(inst[i]);
        if (rc == 0 && done_ms)
          done_ms[i] = elapsed_ms();
      }
      if (rc) {
        std::lock_guard<std::mutex> g(mu);
        if (!first_rc) {
          first_rc = rc;
          first_msg = spiffe_gpu_last_error();
        }
        return;
      }
    }
  };
  const int32_t nw = std::max<int32_t>(1, std::min<int32_t>(workers, std::max<int32_t>(n, 1)));
  std::vector<std::thread> pool;
  for (int32_t w = 0; w < nw; w++)
    pool.emplace_back(worker);
  for (std::thread &t : pool)
    t.join();
  if (first_rc)
    return spiffe_set_error(first_rc, first_msg.c_str());
  return 0;
}
