// Serving loop: many RVE homogenisation solves resident on one GPU at once.
//
// Each of `max_slots` worker threads takes the oldest queued request that fits the
// device-memory budget, builds a solver handle for it (own buffers, own CUDA stream),
// runs the constant-rate time loop natively (ssfft_solve_constant_rates: Newton with
// device MINRES replayed from a CUDA graph per handle), copies the final stress out and
// posts a completion with its queue/start/end times.  Requests that arrive while others
// run start as soon as a slot and memory are free, and their kernels overlap on the GPU
// with those of the requests already running.
//
// Only the public C ABI of ssfft.h is used here, plus cudaMemGetInfo for admission.
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ssfft.h"

int ssfft_internal_fail(int code, const std::string &msg);

namespace {

struct Job {
  ssfft_request req;  // pointers below replace the caller's borrowed ones
  std::vector<double> rotations;
  std::vector<int32_t> orient, phase;
  double submit_time;
  size_t bytes;
};

size_t job_bytes(const ssfft_request &r) {
  int any_evp = 0, nslip = 0;
  for (int p = 0; p < r.n_phases; ++p)
    if (r.phases[p].kind == 1) {
      any_evp = 1;
      nslip = std::max(nslip, (int)r.phases[p].n_slip);
    }
  size_t b = 0;
  if (ssfft_estimate_bytes(&r.config, any_evp, nslip, &b) != 0) return 0;
  return b;
}

}  // namespace

struct PoolEntry {
  ssfft_handle *h;
  std::string key;
  size_t bytes;
  double last_used;
};

// Handles are reusable for any request of the same grid, precision and crystal-plasticity
// shape (ssfft_set_options / ssfft_set_microstructure rebind them).
std::string pool_key(const ssfft_request &r) {
  int any_evp = 0, nslip = 0;
  for (int p = 0; p < r.n_phases; ++p)
    if (r.phases[p].kind == 1) {
      any_evp = 1;
      nslip = std::max(nslip, (int)r.phases[p].n_slip);
    }
  return std::to_string(r.config.n[0]) + "x" + std::to_string(r.config.n[1]) + "x" +
         std::to_string(r.config.n[2]) + "/" + std::to_string(r.config.precision) + "/" +
         std::to_string(any_evp) + "/" + std::to_string(nslip);
}

struct ssfft_server {
  int device;
  size_t budget;
  std::chrono::steady_clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Job *> queue;
  std::vector<ssfft_completion> done;
  std::vector<std::thread> workers;
  size_t in_use = 0;  // bytes of every handle alive (running or idle in the pool)
  int running = 0;
  std::vector<PoolEntry> idle;
  long long outstanding = 0;  // submitted, not yet polled
  bool stopping = false;

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }

  // Called with mu held.  Grants the oldest job an idle pooled handle of its shape, or
  // room for a new one.  Idle handles of other shapes are evicted (destroyed outside the
  // lock, into `evict`) when the budget or the device's free memory is short.
  bool admit(Job *j, ssfft_handle **pooled, std::vector<ssfft_handle *> &evict) {
    const std::string key = pool_key(j->req);
    for (size_t k = 0; k < idle.size(); ++k)
      if (idle[k].key == key) {
        *pooled = idle[k].h;
        j->bytes = idle[k].bytes;
        idle.erase(idle.begin() + k);
        return true;
      }
    const size_t reserve = (size_t)512 << 20;  // headroom for the runtime and other users
    for (;;) {
      size_t free_b = 0, total_b = 0;
      const bool info = cudaMemGetInfo(&free_b, &total_b) == cudaSuccess;
      if (info && in_use + j->bytes <= budget && j->bytes + reserve <= free_b) {
        in_use += j->bytes;
        return true;
      }
      if (idle.empty()) return false;
      size_t lru = 0;
      for (size_t k = 1; k < idle.size(); ++k)
        if (idle[k].last_used < idle[lru].last_used) lru = k;
      in_use -= idle[lru].bytes;
      evict.push_back(idle[lru].h);
      idle.erase(idle.begin() + lru);
      if (!evict.empty()) return false;  // free them first, then look again
    }
  }

  void run_job(Job *j, int slot, ssfft_handle *h) {
    ssfft_completion c;
    memset(&c, 0, sizeof(c));
    c.tag = j->req.tag;
    c.slot = slot;
    c.submit_time = j->submit_time;
    c.start_time = now();
    c.device_bytes = j->bytes;
    ssfft_config cfg = j->req.config;
    cfg.device = device;
    int rc = h ? ssfft_set_options(h, &cfg) : ssfft_create(&cfg, &h);
    for (int p = 0; rc == 0 && p < j->req.n_phases; ++p) {
      const ssfft_phase &ph = j->req.phases[p];
      if (ph.kind == 0)
        rc = ssfft_set_phase_elastic(h, p, ph.stiffness);
      else
        rc = ssfft_set_phase_evp(h, p, ph.stiffness, ph.n_slip, ph.schmid,
                                 ph.reference_slip_rate, ph.rate_exponent, ph.slip_resistance,
                                 ph.hardening, ph.hardening_props, ph.n_props, ph.latent_ratio);
    }
    if (rc == 0)
      rc = ssfft_set_microstructure(h, j->req.n_orient, j->rotations.data(), j->orient.data(),
                                    j->phase.empty() ? nullptr : j->phase.data());
    if (rc == 0) rc = ssfft_solve_constant_rates(h, &j->req.schedule, &c.result);
    if (rc == 0 && j->req.stress_out) rc = ssfft_get_field(h, SSFFT_FIELD_STRESS, j->req.stress_out, 1);
    c.status = rc;
    if (rc != 0) {
      strncpy(c.message, ssfft_last_error(), sizeof(c.message) - 1);
      c.message[sizeof(c.message) - 1] = 0;
    }
    c.end_time = now();
    const std::string key = pool_key(j->req);
    const size_t bytes = j->bytes;
    if (rc != 0 && h) {  // a handle in an unknown state is not reused
      ssfft_destroy(h);
      h = nullptr;
    }
    std::lock_guard<std::mutex> lk(mu);
    if (h)
      idle.push_back(PoolEntry{h, key, bytes, c.end_time});
    else
      in_use -= bytes;
    --running;
    done.push_back(c);
    delete j;
    cv.notify_all();
  }

  void fail_job(Job *head, int slot, int code) {  // mu held
    ssfft_completion c;
    memset(&c, 0, sizeof(c));
    c.tag = head->req.tag;
    c.status = code;
    c.slot = slot;
    c.submit_time = head->submit_time;
    c.start_time = c.end_time = now();
    c.device_bytes = head->bytes;
    strncpy(c.message, "request does not fit the device-memory budget", sizeof(c.message) - 1);
    done.push_back(c);
    delete head;
  }

  void worker(int slot) {
    cudaSetDevice(device);
    for (;;) {
      Job *j = nullptr;
      ssfft_handle *pooled = nullptr;
      std::vector<ssfft_handle *> evict;
      {
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
          if (!queue.empty()) {
            Job *head = queue.front();
            if (head->bytes > budget) {  // can never fit: fail it now
              queue.pop_front();
              fail_job(head, slot, SSFFT_E_NOMEM);
              continue;
            }
            if (admit(head, &pooled, evict)) {
              j = head;
              queue.pop_front();
              ++running;
              break;
            }
            if (!evict.empty()) break;  // free evicted handles outside the lock, retry
            if (running == 0 && stopping) {  // nothing will free memory
              queue.pop_front();
              fail_job(head, slot, SSFFT_E_NOMEM);
              continue;
            }
          } else if (stopping) {
            break;
          }
          // wait for a submission or a completion (bounded, so the free-memory check of
          // cudaMemGetInfo is retried when other processes release memory)
          cv.wait_for(lk, std::chrono::milliseconds(50));
        }
      }
      for (ssfft_handle *e : evict) ssfft_destroy(e);
      if (j)
        run_job(j, slot, pooled);
      else if (evict.empty()) {
        std::lock_guard<std::mutex> lk(mu);
        if (stopping && queue.empty()) return;
      }
    }
  }

  void drain_pool() {
    for (PoolEntry &e : idle) ssfft_destroy(e.h);
    idle.clear();
  }
};

extern "C" int ssfft_server_create(int device, int max_slots, size_t hbm_budget_bytes,
                                   ssfft_server **out) {
  if (!out || max_slots < 1 || max_slots > 256)
    return ssfft_internal_fail(SSFFT_E_INVALID, "max_slots must be 1..256");
  *out = nullptr;
  // Many slot threads each wait on their own stream; spinning waits compete for the CPU
  // cores the other slots need to launch work.  SSFFT_SCHEDULE = spin | yield | blocking
  // selects the waiting mode of the process's CUDA context (before it is created).
  if (const char *sch = getenv("SSFFT_SCHEDULE")) {
    unsigned flags = cudaDeviceScheduleAuto;
    if (!strcmp(sch, "spin")) flags = cudaDeviceScheduleSpin;
    if (!strcmp(sch, "yield")) flags = cudaDeviceScheduleYield;
    if (!strcmp(sch, "blocking")) flags = cudaDeviceScheduleBlockingSync;
    cudaSetDevice(device);
    if (cudaSetDeviceFlags(flags) != cudaSuccess) cudaGetLastError();
  }
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return ssfft_internal_fail(SSFFT_E_CUDA, cudaGetErrorString(e));
  size_t free_b = 0, total_b = 0;
  e = cudaMemGetInfo(&free_b, &total_b);
  if (e != cudaSuccess) return ssfft_internal_fail(SSFFT_E_CUDA, cudaGetErrorString(e));
  ssfft_server *s = new ssfft_server();
  s->device = device;
  s->budget = hbm_budget_bytes ? hbm_budget_bytes : (size_t)(0.9 * (double)free_b);
  s->t0 = std::chrono::steady_clock::now();
  for (int k = 0; k < max_slots; ++k) s->workers.emplace_back(&ssfft_server::worker, s, k);
  *out = s;
  return 0;
}

extern "C" int ssfft_server_submit(ssfft_server *s, const ssfft_request *req) {
  if (!s || !req) return ssfft_internal_fail(SSFFT_E_INVALID, "null argument");
  const long long V = (long long)req->config.n[0] * req->config.n[1] * req->config.n[2];
  if (V <= 0 || req->n_orient < 1 || !req->rotations || !req->orient_of_point ||
      req->n_phases < 1 || req->n_phases > SSFFT_MAX_PHASES)
    return ssfft_internal_fail(SSFFT_E_INVALID, "incomplete request");
  Job *j = new Job();
  j->req = *req;
  j->rotations.assign(req->rotations, req->rotations + 9 * (size_t)req->n_orient);
  j->orient.assign(req->orient_of_point, req->orient_of_point + V);
  if (req->phase_of_point) j->phase.assign(req->phase_of_point, req->phase_of_point + V);
  j->req.rotations = nullptr;
  j->req.orient_of_point = nullptr;
  j->req.phase_of_point = nullptr;
  j->bytes = job_bytes(j->req);
  if (j->bytes == 0) {
    delete j;
    return ssfft_internal_fail(SSFFT_E_INVALID, "request configuration rejected");
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stopping) {
    delete j;
    return ssfft_internal_fail(SSFFT_E_INVALID, "server is shutting down");
  }
  j->submit_time = s->now();
  s->queue.push_back(j);
  ++s->outstanding;
  s->cv.notify_all();
  return 0;
}

extern "C" int ssfft_server_poll(ssfft_server *s, ssfft_completion *out, int max, int *n_out) {
  if (!s || !n_out || (max > 0 && !out)) return ssfft_internal_fail(SSFFT_E_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  int n = 0;
  while (n < max && !s->done.empty()) {
    out[n++] = s->done.front();
    s->done.erase(s->done.begin());
  }
  s->outstanding -= n;
  *n_out = n;
  return 0;
}

extern "C" int ssfft_server_pending(ssfft_server *s) {
  if (!s) return 0;
  std::lock_guard<std::mutex> lk(s->mu);
  return (int)s->outstanding;
}

extern "C" double ssfft_server_clock(ssfft_server *s) { return s ? s->now() : 0.0; }

extern "C" int ssfft_server_destroy(ssfft_server *s) {
  if (!s) return 0;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
    s->cv.notify_all();
  }
  for (auto &t : s->workers) t.join();
  for (Job *j : s->queue) delete j;
  s->drain_pool();
  delete s;
  return 0;
}
