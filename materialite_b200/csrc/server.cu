// Serving loop: many RVE homogenisation solves resident on one GPU, batched.
//
// Requests are sorted by class -- grid size, precision, tangent kind (elastic tables or
// per-voxel crystal-plasticity tangents), slip-system count, and whether the schedule has
// stress rates -- and each class has a group (group.cuh): up to `max_slots` requests that
// advance together, every kernel launch covering all of them.  A group's driver thread
// loads queued requests into free slots (a slot's device memory is allocated on its first
// use, when it fits both the server's budget and cudaMemGetInfo's free memory), runs the
// group's graph until some request finishes, returns the finished requests' results, and
// refills.  A request that arrives while its class runs with a free slot raises the
// group's wake flag, and the running graph returns at its next pass boundary (a few Krylov
// iterations) so that the request is loaded and joins the others; classes run
// concurrently on their own streams.
//
// A request's arithmetic does not depend on what else runs: every reduction of a slot is
// private to it and summed in a fixed order, so a result is bitwise the same alone and in
// any mix.
#include <cuda_runtime.h>

#include <atomic>
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

#include "../../include/ssfft.h"
#include "group_api.h"

int ssfft_internal_fail(int code, const std::string &msg);

namespace {

struct ClassInfo {
  bool voxel = false;
  int nslip = 0;
  bool rates = false;
  std::string key;
};

ClassInfo classify(const ssfft_request &r) {
  ClassInfo c;
  for (int p = 0; p < r.n_phases; ++p)
    if (r.phases[p].kind == 1) {
      c.voxel = true;
      c.nslip = std::max(c.nslip, (int)r.phases[p].n_slip);
    }
  for (int k = 0; k < 6; ++k)
    if (r.schedule.stress_rate[k] * r.config.stress_mask[k] != 0.0) c.rates = true;
  c.key = std::to_string(r.config.n[0]) + "x" + std::to_string(r.config.n[1]) + "x" +
          std::to_string(r.config.n[2]) + "/" + std::to_string(r.config.precision) + "/" +
          std::to_string(c.voxel) + "/" + std::to_string(c.nslip) + "/" + std::to_string(c.rates);
  return c;
}

size_t job_bytes(const ssfft_request &r, const ClassInfo &c) {
  size_t b = 0;
  if (ssfft_estimate_bytes(&r.config, c.voxel ? 1 : 0, c.nslip, &b) != 0) return 0;
  return b;
}

}  // namespace

struct GroupRunner;

struct ssfft_server {
  int device;
  int max_slots;
  size_t budget;
  std::chrono::steady_clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv;
  std::map<std::string, std::unique_ptr<GroupRunner>> runners;
  std::vector<ssfft_completion> done;
  size_t in_use = 0;           // bytes of allocated slots
  long long outstanding = 0;   // submitted, not yet polled
  bool stopping = false;

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  void post(const ssfft_completion &c) {
    std::lock_guard<std::mutex> lk(mu);
    done.push_back(c);
    cv.notify_all();
  }
};

struct GroupRunner {
  ssfft_server *srv;
  ClassInfo info;
  ssfft_config proto;
  Group *g = nullptr;
  std::atomic<Group *> gpub{nullptr};  // g once initialised, for the submitting threads
  int n_resident = 0;                  // occupied slots (guarded by srv->mu)
  bool init_failed = false;
  std::string init_message;
  std::deque<GroupJob *> queue;     // guarded by srv->mu
  std::vector<GroupJob *> resident; // by slot; touched by the runner thread only
  std::vector<double> start;        // admission time per slot
  std::vector<bool> counted;        // slot's bytes counted in srv->in_use
  std::atomic<long long> launches{0};  // kernels the group has launched (published per run)
  std::thread th;

  ~GroupRunner() {
    if (th.joinable()) th.join();
    for (GroupJob *j : queue) delete j;
    for (GroupJob *j : resident) delete j;
    if (g) group_delete(g);
  }

  ssfft_completion completion(const GroupJob *j, int slot, int status, const char *msg,
                              double start_time) {
    ssfft_completion c;
    memset(&c, 0, sizeof(c));
    c.tag = j->req.tag;
    c.status = status;
    c.slot = slot;
    c.submit_time = j->submit_time;
    c.start_time = start_time;
    c.end_time = srv->now();
    c.device_bytes = j->bytes;
    if (msg) {
      strncpy(c.message, msg, sizeof(c.message) - 1);
      c.message[sizeof(c.message) - 1] = 0;
    }
    return c;
  }

  // Take queued jobs into free slots (mu held).  A slot whose device memory is not yet
  // allocated is used only when the job fits the budget and the device's free memory.
  void admit(std::vector<int> &loaded) {
    const size_t reserve = (size_t)512 << 20;  // headroom for the runtime and other users
    for (int s = 0; s < srv->max_slots && !queue.empty(); ++s) {
      if (resident[s]) continue;
      GroupJob *j = queue.front();
      if (!counted[s]) {
        size_t free_b = 0, total_b = 0;
        const bool info_ok = cudaMemGetInfo(&free_b, &total_b) == cudaSuccess;
        if (!info_ok || srv->in_use + j->bytes > srv->budget || j->bytes + reserve > free_b)
          continue;  // try a slot that is already allocated
        srv->in_use += j->bytes;
        counted[s] = true;
      }
      queue.pop_front();
      resident[s] = j;
      ++n_resident;
      start[s] = srv->now();
      loaded.push_back(s);
    }
  }

  // Queued jobs that can never be admitted: larger than the whole budget, or, at shutdown,
  // with no slot allocated and nothing running (mu held).
  void reject_unfit() {
    while (!queue.empty()) {
      GroupJob *j = queue.front();
      bool any_alloc = false, any_res = false;
      for (int s = 0; s < srv->max_slots; ++s) {
        any_alloc = any_alloc || counted[s];
        any_res = any_res || resident[s];
      }
      const bool never = j->bytes > srv->budget || (!any_alloc && !any_res && srv->stopping);
      if (!never) return;
      queue.pop_front();
      srv->done.push_back(completion(j, -1, SSFFT_E_NOMEM,
                                     "request does not fit the device-memory budget", srv->now()));
      delete j;
    }
  }

  void run() {
    cudaSetDevice(srv->device);
    g = group_new();
    if (group_init(g, proto, srv->max_slots, info.voxel, info.rates, srv->device) != 0) {
      init_failed = true;
      init_message = ssfft_last_error();
    }
    resident.assign(srv->max_slots, nullptr);
    start.assign(srv->max_slots, 0.0);
    counted.assign(srv->max_slots, false);
    if (!init_failed) gpub.store(g);
    for (;;) {
      std::vector<int> loaded;
      {
        std::unique_lock<std::mutex> lk(srv->mu);
        for (;;) {
          if (init_failed) {
            while (!queue.empty()) {
              GroupJob *j = queue.front();
              queue.pop_front();
              srv->done.push_back(completion(j, -1, SSFFT_E_CUDA, init_message.c_str(), srv->now()));
              delete j;
            }
          } else {
            reject_unfit();
            admit(loaded);
            // submissions from here on find the slots as they are now
            if (g) group_clear_wake(g);
          }
          bool any = false;
          for (GroupJob *j : resident) any = any || j;
          if (any) break;
          if (srv->stopping && queue.empty()) {
            srv->cv.notify_all();
            return;
          }
          // wait for a submission (bounded, so that free memory is looked at again)
          srv->cv.wait_for(lk, std::chrono::milliseconds(20));
        }
      }
      for (int s : loaded) {
        if (group_load(g, s, *resident[s]) != 0) {
          srv->post(completion(resident[s], s, SSFFT_E_CUDA, ssfft_last_error(), start[s]));
          delete resident[s];
          resident[s] = nullptr;
          group_release_slot(g, s);
          std::lock_guard<std::mutex> lk(srv->mu);
          --n_resident;
        }
      }
      bool any = false;
      for (GroupJob *j : resident) any = any || j;
      if (!any) continue;
      const int rc = group_run(g);
      launches.store(group_launches(g));
      const std::string msg = rc ? ssfft_last_error() : "";
      for (int s = 0; s < srv->max_slots; ++s) {
        GroupJob *j = resident[s];
        if (!j) continue;
        const int st = group_slot_state(g, s);
        if (rc == 0 && st != GS_DONE && st != GS_FAILED) continue;
        ssfft_completion c = completion(j, s, 0, nullptr, start[s]);
        group_slot_result(g, s, &c.result);
        if (rc) {
          c.status = rc;
          strncpy(c.message, msg.c_str(), sizeof(c.message) - 1);
        } else if (st == GS_FAILED) {
          c.status = c.result.status ? c.result.status : SSFFT_E_INVALID;
          const char *m = c.status == SSFFT_E_NAN ? "non-finite value in the solve"
                                                  : "min time increment reached or singular mean tangent";
          strncpy(c.message, m, sizeof(c.message) - 1);
        } else if (j->req.stress_out) {
          if (group_read_stress(g, s, j->req.stress_out) != 0) {
            c.status = SSFFT_E_CUDA;
            strncpy(c.message, ssfft_last_error(), sizeof(c.message) - 1);
          }
        }
        c.result.device_seconds = srv->now() - start[s];
        c.end_time = srv->now();
        group_release_slot(g, s);
        delete j;
        resident[s] = nullptr;
        {
          std::lock_guard<std::mutex> lk(srv->mu);
          --n_resident;
        }
        srv->post(c);
      }
    }
  }
};

extern "C" int ssfft_server_create(int device, int max_slots, size_t hbm_budget_bytes,
                                   ssfft_server **out) {
  if (!out || max_slots < 1 || max_slots > 256)
    return ssfft_internal_fail(SSFFT_E_INVALID, "max_slots must be 1..256");
  *out = nullptr;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return ssfft_internal_fail(SSFFT_E_CUDA, cudaGetErrorString(e));
  size_t free_b = 0, total_b = 0;
  e = cudaMemGetInfo(&free_b, &total_b);
  if (e != cudaSuccess) return ssfft_internal_fail(SSFFT_E_CUDA, cudaGetErrorString(e));
  ssfft_server *s = new ssfft_server();
  s->device = device;
  s->max_slots = max_slots;
  s->budget = hbm_budget_bytes ? hbm_budget_bytes : (size_t)(0.9 * (double)free_b);
  s->t0 = std::chrono::steady_clock::now();
  *out = s;
  return 0;
}

extern "C" int ssfft_server_submit(ssfft_server *s, const ssfft_request *req) {
  if (!s || !req) return ssfft_internal_fail(SSFFT_E_INVALID, "null argument");
  const long long V = (long long)req->config.n[0] * req->config.n[1] * req->config.n[2];
  if (V <= 0 || req->n_orient < 1 || !req->rotations || !req->orient_of_point ||
      req->n_phases < 1 || req->n_phases > SSFFT_MAX_PHASES)
    return ssfft_internal_fail(SSFFT_E_INVALID, "incomplete request");
  for (int p = 0; p < req->n_phases; ++p)
    if (req->phases[p].kind != 0 && req->phases[p].kind != 1)
      return ssfft_internal_fail(SSFFT_E_INVALID, "request phases must be elastic or crystal EVP");
  const ClassInfo ci = classify(*req);
  GroupJob *j = new GroupJob();
  j->req = *req;
  j->rotations.assign(req->rotations, req->rotations + 9 * (size_t)req->n_orient);
  j->orient.assign(req->orient_of_point, req->orient_of_point + V);
  if (req->phase_of_point) j->phase.assign(req->phase_of_point, req->phase_of_point + V);
  j->req.rotations = nullptr;
  j->req.orient_of_point = nullptr;
  j->req.phase_of_point = nullptr;
  j->bytes = job_bytes(j->req, ci);
  if (j->bytes == 0) {
    delete j;
    return ssfft_internal_fail(SSFFT_E_INVALID, "request configuration rejected");
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stopping) {
    delete j;
    return ssfft_internal_fail(SSFFT_E_INVALID, "server is shutting down");
  }
  auto it = s->runners.find(ci.key);
  if (it == s->runners.end()) {
    auto r = std::make_unique<GroupRunner>();
    r->srv = s;
    r->info = ci;
    r->proto = j->req.config;
    r->proto.device = s->device;
    GroupRunner *rp = r.get();
    it = s->runners.emplace(ci.key, std::move(r)).first;
    rp->th = std::thread(&GroupRunner::run, rp);
  }
  j->submit_time = s->now();
  GroupRunner *r = it->second.get();
  r->queue.push_back(j);
  ++s->outstanding;
  // a free slot: the running graph of the class returns at its next pass to take it
  Group *g = r->gpub.load();
  if (g && r->n_resident < s->max_slots) group_wake(g);
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

extern "C" int ssfft_server_launches(ssfft_server *s, int64_t *kernel_launches) {
  if (!s || !kernel_launches) return ssfft_internal_fail(SSFFT_E_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  long long n = 0;
  for (auto &kv : s->runners) n += kv.second->launches.load();
  *kernel_launches = n;
  return 0;
}

extern "C" int ssfft_server_destroy(ssfft_server *s) {
  if (!s) return 0;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
    s->cv.notify_all();
  }
  for (auto &kv : s->runners)
    if (kv.second->th.joinable()) kv.second->th.join();
  s->runners.clear();
  delete s;
  return 0;
}
