// Serving loop for ensembles of independent suspensions (continuous batching).
//
// Requests (a configuration, a fiber layout, a step budget) are queued as they
// arrive; a dispatcher admits them in arrival order while a slot is free and
// the device memory their system needs (rf_device_bytes_estimate) fits the
// budget, so requests that arrive while others run start as soon as a slot
// and memory free up.  Each admitted request gets its own handle (device-
// resident fibers, Krylov state, previous-step velocities) and stream, driven
// by a worker thread; the streams of all running requests overlap on the
// device.  Small requests (at most pack_max_fibers fibers, mixed precision)
// instead join a pack: one worker thread steps all of them together, their
// systems solved by one launch per step and cluster size (rf_step_packed:
// one thread-block cluster per suspension); they join and leave the pack
// between steps.  Every kernel is
// deterministic (fixed-order reductions, no atomics), so a request's result
// does not depend on what runs beside it.
// The reference has no serving layer; this is the ensemble workload of the
// thesis' parameter studies run as a service.
#include <algorithm>
#include <cmath>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "rf_common.cuh"
#include "rf_kernels.cuh"
#include "rf_krylov.cuh"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  int64_t id = 0;
  rf_config cfg;
  int N = 0;
  int nsteps = 0;
  std::vector<double> pos, ori;       // inputs, then the final state
  std::vector<double> tvel, rvel;     // last velocities
  int64_t bytes = 0;                  // admission estimate
  int status = RF_REQ_QUEUED;
  int error = RF_OK;
  int steps_done = 0;
  bool cancel = false;
  double t_submit = 0, t_start = 0, t_ready = 0, t_end = 0;   // ready: handle and graphs built
  std::vector<double> step_ms;
  bool packed = false;                // stepped by the pack worker
  std::thread worker;
};

// a configuration the packed solve takes (rf_solve_packed's conditions)
bool packable(const rf_config& c, int N, int max_fibers) {
  return max_fibers > 0 && N <= std::min(max_fibers, rf::kPackMaxFibers) &&
         (c.precision == RF_PREC_MIXED_FP16 || c.precision == RF_PREC_MIXED_BF16) &&
         c.solver == RF_SOLVER_GMRES && c.number_of_terms_in_force_expansion == 5 &&
         c.number_of_quadrature_intervals == 8 && c.number_of_quadrature_points_per_interval == 3;
}

}  // namespace

struct rf_server {
  rf_server_config cfg;
  int device = 0;
  std::mutex mu;
  std::mutex setup_mu;               // handle creation and graph building: at most setup_lanes at once
  std::condition_variable setup_cv;
  int setup_lanes = 1, setup_busy = 0;
  std::condition_variable cv;        // dispatcher wake-up
  std::condition_variable done_cv;   // waiters
  std::deque<int64_t> queue;
  std::map<int64_t, std::unique_ptr<Request>> reqs;
  std::vector<std::thread> finished_workers;
  int64_t next_id = 1;
  int active = 0;
  int64_t bytes_in_use = 0;
  int64_t peak_bytes = 0;
  int peak_active = 0;
  bool stopping = false;
  std::thread dispatcher;
  // pack of small requests
  std::condition_variable pack_cv;
  std::vector<Request*> pack_pending;   // admitted, not yet in the pack
  int packed_active = 0;
  std::thread pack_worker;
  std::vector<double> all_step_ms;
  std::vector<double> pack_ms;          // wall time of each rf_step_packed call
  int64_t pack_member_steps = 0;        // suspensions stepped by those calls
  int64_t fiber_steps = 0;
  double t0 = 0, t_last = 0;
};

static double now_s() {
  return std::chrono::duration<double>(Clock::now().time_since_epoch()).count();
}

static void finish_locked(rf_server* s, Request* r, int rc, const std::vector<double>& lat);

// one of the server's setup lanes, held while a request is set up
struct SetupLane {
  rf_server* s;
  explicit SetupLane(rf_server* srv) : s(srv) {
    std::unique_lock<std::mutex> lk(s->setup_mu);
    s->setup_cv.wait(lk, [&] { return s->setup_busy < s->setup_lanes; });
    s->setup_busy += 1;
  }
  ~SetupLane() {
    std::lock_guard<std::mutex> lk(s->setup_mu);
    s->setup_busy -= 1;
    s->setup_cv.notify_one();
  }
};

static void run_request(rf_server* s, Request* r) {
  cudaSetDevice(s->device);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
  rf::set_coop_block_cap(std::max(1, sms / s->cfg.max_active));
  rf_handle* h = nullptr;
  int rc;
  {
    // A few requests at a time create their handles and build their step
    // graphs: the driver serialises stream, event and graph creation
    // internally, and sixteen threads doing it at once each took ~100x longer
    // than one alone (while slowing the others' launches).
    SetupLane lane(s);
    rc = rf_create(&r->cfg, r->N, r->pos.data(), r->ori.data(), &h);
    if (rc == RF_OK) {
      rf_set_host_wait(h, 1);
      rf_set_cuda_graphs(h, s->cfg.use_cuda_graphs);
      // whole-step graphs are built now, before the first step (a step then
      // is one graph launch from the first on)
      if (s->cfg.use_cuda_graphs == 1) rf_prepare_step_graphs(h, r->nsteps > 1 ? 3 : 1);
    }
  }
  std::vector<double> lat;
  if (rc == RF_OK) {
    {
      std::lock_guard<std::mutex> lk(s->mu);
      r->t_ready = now_s();
    }
    for (int t = 0; t < r->nsteps; ++t) {
      {
        std::lock_guard<std::mutex> lk(s->mu);
        if (r->cancel) break;
      }
      const auto a = Clock::now();
      rc = rf_step(h, t);
      const auto b = Clock::now();
      if (rc != RF_OK && rc != RF_E_NOCONV) break;
      rc = RF_OK;
      lat.push_back(std::chrono::duration<double, std::milli>(b - a).count());
      std::lock_guard<std::mutex> lk(s->mu);
      r->steps_done = t + 1;
    }
    if (rc == RF_OK) {
      rf_get_state(h, r->pos.data(), r->ori.data());
      if (r->steps_done > 0) rf_get_velocities(h, r->tvel.data(), r->rvel.data());
    }
    rf_destroy(h);
  }
  std::lock_guard<std::mutex> lk(s->mu);
  s->active -= 1;
  s->finished_workers.push_back(std::move(r->worker));
  finish_locked(s, r, rc, lat);
}

// record the end of a request (lock held)
static void finish_locked(rf_server* s, Request* r, int rc, const std::vector<double>& lat) {
  r->t_end = now_s();
  r->step_ms = lat;
  r->error = rc;
  r->status = rc != RF_OK ? RF_REQ_FAILED : (r->cancel ? RF_REQ_CANCELLED : RF_REQ_DONE);
  if (rc == RF_OK) {
    s->all_step_ms.insert(s->all_step_ms.end(), lat.begin(), lat.end());
    s->fiber_steps += (int64_t)r->N * (int64_t)lat.size();
  }
  s->t_last = r->t_end;
  s->bytes_in_use -= r->bytes;
  s->cv.notify_all();
  s->done_cv.notify_all();
}

// The pack: every small request admitted steps once per round; the
// suspensions of one restart length share an rf_step_packed call.
static void pack_loop(rf_server* s) {
  cudaSetDevice(s->device);
  struct Member {
    Request* r;
    rf_handle* h;
    int t;
    std::vector<double> lat;
  };
  std::vector<Member> mem;
  for (;;) {
    std::vector<Request*> joining;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      if (mem.empty() && s->pack_pending.empty()) {
        if (s->stopping) return;
        s->pack_cv.wait_for(lk, std::chrono::milliseconds(50));
        continue;
      }
      joining.swap(s->pack_pending);
    }
    // new members' handles, created from several host threads
    std::vector<rf_handle*> made(joining.size(), nullptr);
    std::vector<int> mrc(joining.size(), RF_OK);
    {
      const size_t nt = std::min<size_t>(8, joining.size());
      std::vector<std::thread> th;
      for (size_t k = 0; k < nt; ++k)
        th.emplace_back([&, k] {
          cudaSetDevice(s->device);
          for (size_t q = k; q < joining.size(); q += nt)
            mrc[q] = rf_create(&joining[q]->cfg, joining[q]->N, joining[q]->pos.data(), joining[q]->ori.data(),
                               &made[q]);
        });
      for (auto& x : th) x.join();
    }
    for (size_t q = 0; q < joining.size(); ++q) {
      Request* r = joining[q];
      if (mrc[q] != RF_OK) {
        std::lock_guard<std::mutex> lk(s->mu);
        finish_locked(s, r, mrc[q], {});
        s->packed_active -= 1;
        continue;
      }
      {
        std::lock_guard<std::mutex> lk(s->mu);
        r->t_ready = now_s();
      }
      mem.push_back({r, made[q], 0, {}});
    }
    // members that are done or cancelled leave before the step
    auto leave = [&](size_t k, int rc) {
      Member& q = mem[k];
      if (rc == RF_OK) {
        rf_get_state(q.h, q.r->pos.data(), q.r->ori.data());
        if (q.t > 0) rf_get_velocities(q.h, q.r->tvel.data(), q.r->rvel.data());
      }
      rf_destroy(q.h);
      std::lock_guard<std::mutex> lk(s->mu);
      finish_locked(s, q.r, rc, q.lat);
      s->packed_active -= 1;
      mem.erase(mem.begin() + (std::ptrdiff_t)k);
    };
    for (size_t k = mem.size(); k-- > 0;) {
      bool cancel;
      {
        std::lock_guard<std::mutex> lk(s->mu);
        cancel = mem[k].r->cancel;
      }
      if (cancel || mem[k].t >= mem[k].r->nsteps) leave(k, RF_OK);
    }
    if (mem.empty()) continue;
    // one packed step per restart length
    std::map<int, std::vector<size_t>> groups;
    for (size_t k = 0; k < mem.size(); ++k) {
      const rf_config& c = mem[k].r->cfg;
      groups[c.refinement_restart > 0 ? c.refinement_restart : c.gmres_restart].push_back(k);
    }
    std::vector<int> failed(mem.size(), RF_OK);
    for (auto& g : groups) {
      const size_t n = g.second.size();
      for (size_t a = 0; a < n; a += (size_t)s->cfg.pack_max_members) {
        const size_t nb = std::min(n - a, (size_t)s->cfg.pack_max_members);
        std::vector<rf_handle*> hs(nb);
        std::vector<int> ts(nb), st(nb, RF_OK);
        for (size_t q = 0; q < nb; ++q) {
          hs[q] = mem[g.second[a + q]].h;
          ts[q] = mem[g.second[a + q]].t;
        }
        const auto t0 = Clock::now();
        rf_step_packed(hs.data(), ts.data(), (int)nb, st.data());
        const double ms = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
        {
          std::lock_guard<std::mutex> lk(s->mu);
          s->pack_ms.push_back(ms);
          s->pack_member_steps += (int64_t)nb;
        }
        for (size_t q = 0; q < nb; ++q) {
          Member& mm = mem[g.second[a + q]];
          if (st[q] == RF_OK || st[q] == RF_E_NOCONV) {
            mm.t += 1;
            mm.lat.push_back(ms);
            std::lock_guard<std::mutex> lk(s->mu);
            mm.r->steps_done = mm.t;
          } else {
            failed[g.second[a + q]] = st[q];
          }
        }
      }
    }
    for (size_t k = mem.size(); k-- > 0;)
      if (failed[k] != RF_OK) leave(k, failed[k]);
  }
}

static void dispatch_loop(rf_server* s) {
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    // join workers that finished (their threads were moved here)
    while (!s->finished_workers.empty()) {
      std::thread t = std::move(s->finished_workers.back());
      s->finished_workers.pop_back();
      lk.unlock();
      if (t.joinable()) t.join();
      lk.lock();
    }
    if (s->stopping && s->active == 0 && s->packed_active == 0) return;
    bool admitted = false;
    while (!s->stopping && !s->queue.empty()) {
      Request* r = s->reqs[s->queue.front()].get();
      if (r->cancel) {
        r->status = RF_REQ_CANCELLED;
        s->queue.pop_front();
        s->done_cv.notify_all();
        continue;
      }
      const int running = s->active + s->packed_active;
      if (r->packed) {
        if (running > 0 && s->bytes_in_use + r->bytes > s->cfg.hbm_budget_bytes) break;   // wait for memory
        s->queue.pop_front();
        r->status = RF_REQ_RUNNING;
        r->t_start = now_s();
        s->packed_active += 1;
        s->bytes_in_use += r->bytes;
        s->peak_bytes = std::max(s->peak_bytes, s->bytes_in_use);
        s->peak_active = std::max(s->peak_active, s->active + s->packed_active);
        s->pack_pending.push_back(r);
        s->pack_cv.notify_all();
        admitted = true;
        continue;
      }
      if (s->active >= s->cfg.max_active) break;
      if (running > 0 && s->bytes_in_use + r->bytes > s->cfg.hbm_budget_bytes) break;   // wait for memory
      s->queue.pop_front();
      r->status = RF_REQ_RUNNING;
      r->t_start = now_s();
      s->active += 1;
      s->bytes_in_use += r->bytes;
      s->peak_bytes = std::max(s->peak_bytes, s->bytes_in_use);
      s->peak_active = std::max(s->peak_active, s->active + s->packed_active);
      r->worker = std::thread(run_request, s, r);
      admitted = true;
    }
    if (!admitted) s->cv.wait_for(lk, std::chrono::milliseconds(50));
  }
}

extern "C" {

int rf_server_config_default(rf_server_config* c) {
  if (!c) return RF_E_INPUT;
  std::memset(c, 0, sizeof(*c));
  // Requests of at most 128 fibers step in the pack, eight larger ones at once
  // on their own handles.  On the served ensemble (N log-uniform in [16, 1000],
  // 400 requests/s, one B200) this gave per-step p50 1.44 ms, p99 5.7 ms and
  // 1.05M fiber-steps/s, against 3.45 / 6.6 ms and 0.93M with no pack and
  // sixteen requests at once (fewer slots: shorter steps, longer queues).
  c->max_active = 8;
  // restart cycles only: with many requests sharing the GPU a step waits
  // mostly for the others' kernels, and building whole-step graphs at every
  // admission cost more aggregate rate (618k vs 881k fiber-steps/s on the
  // served ensemble) than it saved in launches
  c->use_cuda_graphs = 2;
  c->pack_max_fibers = rf::kPackSingleMaxFibers;
  c->pack_max_members = 148;
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) c->hbm_budget_bytes = (int64_t)(0.8 * (double)fr);
  else c->hbm_budget_bytes = (int64_t)64 << 30;
  c->reserve_bytes = c->hbm_budget_bytes / 4;
  return RF_OK;
}

int rf_server_create(const rf_server_config* cfg, rf_server** out) {
  if (!cfg || !out || cfg->max_active < 1 || cfg->hbm_budget_bytes <= 0 || cfg->pack_max_fibers < 0 ||
      (cfg->pack_max_fibers > 0 && cfg->pack_max_members < 1) || cfg->reserve_bytes < 0) {
    rf::set_last_error_str("rf_server_create: max_active >= 1, a positive memory budget, pack_max_members >= 1, "
                           "reserve_bytes >= 0");
    return RF_E_INPUT;
  }
  rf_server* s = new rf_server();
  s->cfg = *cfg;
  s->setup_lanes = std::max(1, cfg->max_active / 4);
  cudaGetDevice(&s->device);
  rf::pools_acquire();   // requests' memory stays in the handles' pool between requests
  const int64_t reserve = std::min(cfg->reserve_bytes, cfg->hbm_budget_bytes);
  if (reserve > 0) {
    // one allocation of the reserve, freed at once: the pool keeps it (its
    // release threshold is at the maximum while a server or handle lives)
    cudaMemPool_t pool = nullptr;
    cudaStream_t st = nullptr;
    void* p = nullptr;
    if (rf::handle_pool(s->device, &pool) == cudaSuccess &&
        cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess) {
      if (cudaMallocFromPoolAsync(&p, (size_t)reserve, pool, st) == cudaSuccess) cudaFreeAsync(p, st);
      cudaStreamSynchronize(st);
      cudaStreamDestroy(st);
    }
    cudaGetLastError();   // a reserve that does not fit only means growing on demand
  }
  s->t0 = now_s();
  s->dispatcher = std::thread(dispatch_loop, s);
  if (cfg->pack_max_fibers > 0) s->pack_worker = std::thread(pack_loop, s);
  *out = s;
  return RF_OK;
}

int rf_server_submit(rf_server* s, const rf_config* cfg, int N, const double* pos, const double* ori, int nsteps,
                     int64_t* id) {
  if (!s || !cfg || !pos || !ori || !id || N < 1 || nsteps < 0) return RF_E_INPUT;
  auto r = std::make_unique<Request>();
  r->cfg = *cfg;
  r->N = N;
  r->nsteps = nsteps;
  r->pos.assign(pos, pos + 3 * (size_t)N);
  r->ori.assign(ori, ori + 3 * (size_t)N);
  r->tvel.assign(3 * (size_t)N, 0.0);
  r->rvel.assign(3 * (size_t)N, 0.0);
  r->bytes = rf_device_bytes_estimate(cfg, N);   // also validates the configuration
  if (r->bytes < 0) return RF_E_INPUT;
  r->packed = packable(*cfg, N, s->cfg.pack_max_fibers);
  r->t_submit = now_s();
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stopping) return RF_E_STATE;
  if (r->bytes > s->cfg.hbm_budget_bytes) {
    rf::set_last_error_str("rf_server_submit: the request needs more device memory than the budget");
    return RF_E_OOM;
  }
  r->id = s->next_id++;
  *id = r->id;
  s->queue.push_back(r->id);
  s->reqs[r->id] = std::move(r);
  s->cv.notify_all();
  return RF_OK;
}

int rf_server_poll(rf_server* s, int64_t id, int* status, int* steps_done) {
  if (!s || !status) return RF_E_INPUT;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return RF_E_INPUT;
  *status = it->second->status;
  if (steps_done) *steps_done = it->second->steps_done;
  return RF_OK;
}

int rf_server_cancel(rf_server* s, int64_t id) {
  if (!s) return RF_E_INPUT;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return RF_E_INPUT;
  it->second->cancel = true;
  s->cv.notify_all();
  return RF_OK;
}

int rf_server_wait(rf_server* s, int64_t id, double timeout_s) {
  if (!s) return RF_E_INPUT;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return RF_E_INPUT;
  Request* r = it->second.get();
  const bool ok = s->done_cv.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] {
    return r->status == RF_REQ_DONE || r->status == RF_REQ_FAILED || r->status == RF_REQ_CANCELLED;
  });
  return ok ? RF_OK : RF_E_TIMEOUT;
}

int rf_server_drain(rf_server* s, double timeout_s) {
  if (!s) return RF_E_INPUT;
  std::unique_lock<std::mutex> lk(s->mu);
  const bool ok = s->done_cv.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                      [&] { return s->queue.empty() && s->active == 0 && s->packed_active == 0; });
  return ok ? RF_OK : RF_E_TIMEOUT;
}

int rf_server_result(rf_server* s, int64_t id, double* pos, double* ori, double* tvel, double* rvel,
                     rf_request_stats* st) {
  if (!s) return RF_E_INPUT;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return RF_E_INPUT;
  Request* r = it->second.get();
  if (r->status != RF_REQ_DONE && r->status != RF_REQ_CANCELLED && r->status != RF_REQ_FAILED) return RF_E_STATE;
  if (r->status == RF_REQ_FAILED) return r->error;
  const size_t n = 3 * (size_t)r->N;
  if (pos) std::memcpy(pos, r->pos.data(), n * sizeof(double));
  if (ori) std::memcpy(ori, r->ori.data(), n * sizeof(double));
  if (tvel) std::memcpy(tvel, r->tvel.data(), n * sizeof(double));
  if (rvel) std::memcpy(rvel, r->rvel.data(), n * sizeof(double));
  if (st) {
    std::memset(st, 0, sizeof(*st));
    st->steps_done = r->steps_done;
    st->queue_ms = 1000.0 * (r->t_start - r->t_submit);
    st->run_ms = 1000.0 * (r->t_end - r->t_start);
    double sum = 0;
    for (double v : r->step_ms) sum += v;
    st->mean_step_ms = r->step_ms.empty() ? 0.0 : sum / r->step_ms.size();
    st->device_bytes = r->bytes;
    st->setup_ms = r->t_ready > 0 ? 1000.0 * (r->t_ready - r->t_start) : 0.0;
  }
  return RF_OK;
}

int rf_server_step_times(rf_server* s, int64_t id, double* ms, int capacity, int* count) {
  if (!s || !count || capacity < 0) return RF_E_INPUT;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return RF_E_INPUT;
  const Request* r = it->second.get();
  if (r->status != RF_REQ_DONE && r->status != RF_REQ_CANCELLED && r->status != RF_REQ_FAILED) return RF_E_STATE;
  *count = (int)r->step_ms.size();
  if (ms) std::copy_n(r->step_ms.begin(), std::min<size_t>((size_t)capacity, r->step_ms.size()), ms);
  return RF_OK;
}

int rf_server_get_stats(rf_server* s, rf_server_stats* out) {
  if (!s || !out) return RF_E_INPUT;
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(out, 0, sizeof(*out));
  std::vector<double> v = s->all_step_ms;
  std::sort(v.begin(), v.end());
  auto pct = [&](double p) -> double {
    if (v.empty()) return 0.0;
    const size_t k = (size_t)std::min<double>(v.size() - 1, std::ceil(p * v.size()) - 1);
    return v[k];
  };
  out->steps = (int64_t)v.size();
  out->p50_step_ms = pct(0.50);
  out->p99_step_ms = pct(0.99);
  out->fiber_steps = s->fiber_steps;
  out->elapsed_s = s->t_last - s->t0;
  out->peak_active = s->peak_active;
  out->peak_bytes = s->peak_bytes;
  int done = 0, failed = 0, queued = 0;
  std::vector<double> su;
  for (auto& kv : s->reqs)
    if (kv.second->status == RF_REQ_DONE && kv.second->t_ready > 0)
      su.push_back(1000.0 * (kv.second->t_ready - kv.second->t_start));
  std::sort(su.begin(), su.end());
  if (!su.empty()) {
    auto sq = [&](double p) { return su[(size_t)std::min<double>(su.size() - 1, std::ceil(p * su.size()) - 1)]; };
    out->p50_setup_ms = sq(0.50);
    out->p99_setup_ms = sq(0.99);
  }
  for (auto& kv : s->reqs) {
    done += kv.second->status == RF_REQ_DONE;
    failed += kv.second->status == RF_REQ_FAILED;
    queued += kv.second->status == RF_REQ_QUEUED;
  }
  out->completed = done;
  out->failed = failed;
  out->queued = queued;
  out->active = s->active + s->packed_active;
  std::vector<double> pk = s->pack_ms;
  std::sort(pk.begin(), pk.end());
  out->pack_steps = (int64_t)pk.size();
  if (!pk.empty()) {
    auto pq = [&](double p) { return pk[(size_t)std::min<double>(pk.size() - 1, std::ceil(p * pk.size()) - 1)]; };
    out->pack_p50_ms = pq(0.50);
    out->pack_p99_ms = pq(0.99);
    out->pack_max_ms = pk.back();
    out->pack_mean_members = (double)s->pack_member_steps / (double)pk.size();
  }
  return RF_OK;
}

int rf_server_destroy(rf_server* s) {
  if (!s) return RF_E_INPUT;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
    for (auto& kv : s->reqs) kv.second->cancel = true;
    s->cv.notify_all();
  }
  if (s->dispatcher.joinable()) s->dispatcher.join();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->pack_cv.notify_all();
  }
  if (s->pack_worker.joinable()) s->pack_worker.join();
  for (auto& kv : s->reqs)
    if (kv.second->worker.joinable()) kv.second->worker.join();
  for (auto& t : s->finished_workers)
    if (t.joinable()) t.join();
  delete s;
  rf::pools_release();
  return RF_OK;
}

}  // extern "C"
