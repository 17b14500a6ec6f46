// server.cpp - continuous-batching solve server.
//
// Requests (aircraft shape, cell target, M, alpha, delta, fixed states) are queued by any host
// thread.  One scheduler thread owns the GPU work:
//   * admission: pending requests enter the active set in arrival order while the estimated
//     device memory of all resident cases stays under the budget and a slot is free;
//   * warm start: a finished case stays resident, keyed by its geometry; a later request with
//     the same key takes it over and starts from its converged state (src/air_cfd.js:521-537:
//     the reference's controller re-applies conditions without a reset);
//   * every round advances all active cases together by `chunk` iterations through one batch
//     (batch.cu: every case's own launches, concurrent in one CUDA graph), then checks each
//     case's FP64 density residual (src/air_cfd.js:552-555, every fluid cell) against its
//     first one;
//   * a case that dropped by the configured ratio or reached the iteration cap gets its FP64
//     forces and Trefftz drag and leaves; the next round already contains the newcomers;
//   * grid sequencing (src/app_cfd.js:271-278, 398-403), when configured: a cold request first
//     runs a coarse case of the same geometry in the batch; when that has dropped its residual
//     (or hit its cap) the requested case measures its own free-stream res0 over one chunk,
//     takes the coarse state interpolated onto its cells (interp.cu) and carries on in the
//     batch in the coarse case's place.
// Each case's arithmetic is the same in the mix as alone: the batched tile is the single-case
// tile, and every case checks its residual every `chunk` of its own iterations.
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>
#include "solver.cuh"

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
  int64_t id;
  a3d_request req;
  a3d_result res{};
  Clock::time_point t_submit, t_admit, t_done;
  a3d_solver* s = nullptr;
  double res0 = -1;
  long it_start = 0;
  bool done = false;
  size_t bytes = 0;
  a3d_solver* coarse = nullptr;  // grid sequencing: the coarse case while it runs
  size_t coarse_bytes = 0;
  double coarse_res0 = -1;
  long coarse_its = 0;
  bool planned_warm = false;  // admission promised it a cached case of its geometry
};

struct Cached {
  a3d_solver* s;
  size_t bytes;
  double res0;
  uint64_t last_use;
  bool reserved;  // promised to an admitted request: not evicted, not promised twice
};

size_t case_bytes(const int32_t dims[3]) {
  const double N = (double)dims[0] * dims[1] * dims[2];
  return (size_t)(N * 96.0) + (64u << 20);  // 3 x 20 B state, 21 B geometry, codes, snapshot, scratch
}

// Admission estimate of a request before its grid exists (target cells, plus the coarse case).
double request_bytes(const a3d_request& r, int sequence) {
  double b = r.cells * 96.0 + (64u << 20);
  if (sequence > 1) b += r.cells / sequence * 96.0 + (64u << 20);
  return b;
}

}  // namespace

struct a3d_server {
  a3d_server_config cfg;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Job>> pending;
  std::vector<std::shared_ptr<Job>> active;
  std::map<int64_t, std::shared_ptr<Job>> jobs;
  std::multimap<uint64_t, Cached> cache;  // geometry key -> idle resident case
  size_t resident = 0;                    // estimated device bytes of active + cached cases
  int64_t next_id = 1;
  uint64_t tick = 0;
  bool stop = false;
  std::thread th;
  Clock::time_point t0;
  int64_t completed = 0, warm_starts = 0, rounds = 0;
  int last_error = A3D_OK;
  std::string last_error_msg;
};

namespace {

double secs(a3d_server* sv, Clock::time_point t) { return std::chrono::duration<double>(t - sv->t0).count(); }

// Evicts least recently used idle cases (none promised to an admitted request) until `need`
// more bytes fit the budget.  Caller holds sv->mu.
void make_room(a3d_server* sv, size_t need) {
  while (sv->resident + need > (size_t)sv->cfg.hbm_budget_bytes) {
    auto lru = sv->cache.end();
    for (auto it = sv->cache.begin(); it != sv->cache.end(); ++it)
      if (!it->second.reserved && (lru == sv->cache.end() || it->second.last_use < lru->second.last_use)) lru = it;
    if (lru == sv->cache.end()) return;
    sv->resident -= lru->second.bytes;
    a3d_solver_destroy(lru->second.s);
    sv->cache.erase(lru);
  }
}

// The coarse case of a sequenced request: cells / sequence, same shape and delta, free stream.
// The per-case stage configuration of served cases: the paired-cell tile with the configured z
// run and one launch per stage.  The cases already run concurrently in the server's batch, so
// the z chunks that speed up a lone case only add launches here.  (64 uneven cases advanced
// together: 15.0 G cell-updates/s with this tile, 14.0 with the single-cell TMA tile.)
int configure_case(a3d_server* sv, a3d_solver* s) {
  int rc = a3d_solver_set_kernel(s, a3d::KERNEL_PAIR, sv->cfg.kz);
  if (rc == A3D_OK) rc = a3d_solver_set_chunks(s, 1);
  return rc;
}

int start_coarse(a3d_server* sv, Job& j) {
  const a3d_request& r = j.req;
  std::vector<double> xf(16384), yf(16384), zf(16384);
  int32_t dims[3];
  double h, core[5];
  int rc = a3d_grid_build(&r.shape, r.cells / sv->cfg.sequence, 16384, xf.data(), yf.data(), zf.data(), dims, &h,
                          core);
  if (rc != A3D_OK) return rc;
  if (dims[0] < 2 || dims[1] < 2 || dims[2] < 2) return A3D_OK;  // nothing to interpolate from: no sequencing
  const size_t bytes = case_bytes(dims);
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    make_room(sv, bytes);
    sv->resident += bytes;
  }
  rc = a3d_solver_create_shape(&r.shape, dims, xf.data(), yf.data(), zf.data(), h, r.delta_deg, sv->cfg.device,
                               &j.coarse);
  if (rc != A3D_OK) {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->resident -= bytes;
    return rc;
  }
  configure_case(sv, j.coarse);
  j.coarse_bytes = bytes;
  a3d_solver_set_free(j.coarse, r.F);
  a3d_solver_set_fix(j.coarse, r.fix);
  a3d_solver_reset(j.coarse);
  double dummy;
  return a3d_solver_residual(j.coarse, 1, &dummy);  // snapshot
}

// Frees the coarse case of a sequenced request.  Called without sv->mu: it takes the lock only
// to update the resident bytes.
void drop_coarse(a3d_server* sv, Job& j) {
  if (!j.coarse) return;
  a3d_solver_destroy(j.coarse);
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->resident -= j.coarse_bytes;
  }
  j.coarse = nullptr;
  j.coarse_bytes = 0;
}

// Coarse case done: the requested case measures its free-stream res0 over one chunk (on the
// batch's tile, so the value is the one a cold batched run gets), then starts from the
// coarse state.  The probe chunk counts towards the case's iterations.  Runs on the scheduler
// thread without sv->mu, so that submit, poll and stats are not held up by its GPU work.
int switch_to_target(a3d_server* sv, Job& j) {
  j.coarse_its = j.coarse->it;
  const int chunk = sv->cfg.chunk_iters;
  int rc = configure_case(sv, j.s);
  if (rc == A3D_OK) rc = a3d_solver_step(j.s, chunk);
  double r0 = -1, dummy;
  if (rc == A3D_OK) rc = a3d_solver_residual(j.s, 1, &r0);
  if (rc == A3D_OK) j.res0 = r0;
  if (rc == A3D_OK) rc = a3d_solver_interp_state(j.s, j.coarse);
  if (rc == A3D_OK) rc = a3d_solver_residual(j.s, 1, &dummy);  // snapshot of the interpolated start
  drop_coarse(sv, j);
  j.it_start = j.s->it - chunk;
  return rc;
}

// Starts an admitted request: takes the cached case admission promised it (warm start) or
// builds a new one.  Called without sv->mu; the lock covers only the cache and the resident
// bytes, the geometry build runs outside it.
int start_case(a3d_server* sv, Job& j) {
  const a3d_request& r = j.req;
  if (j.planned_warm) {
    std::lock_guard<std::mutex> lk(sv->mu);
    auto range = sv->cache.equal_range(r.geometry_key);
    for (auto it = range.first; it != range.second; ++it)
      if (it->second.reserved) {  // warm start: resident geometry and converged state
        j.s = it->second.s;
        j.res0 = it->second.res0;
        j.bytes = it->second.bytes;  // the cached case's bytes stay counted in `resident`
        sv->cache.erase(it);
        j.res.warm = 1;
        sv->warm_starts++;
        break;
      }
  }
  if (!j.res.warm) {
    std::vector<double> xf(16384), yf(16384), zf(16384);
    int32_t dims[3];
    double h, core[5];
    int rc = a3d_grid_build(&r.shape, r.cells, 16384, xf.data(), yf.data(), zf.data(), dims, &h, core);
    if (rc != A3D_OK) return rc;
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      j.bytes = case_bytes(dims);
      make_room(sv, j.bytes);
      sv->resident += j.bytes;
    }
    rc = a3d_solver_create_shape(&r.shape, dims, xf.data(), yf.data(), zf.data(), h, r.delta_deg, sv->cfg.device,
                                 &j.s);
    if (rc != A3D_OK) {
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->resident -= j.bytes;
      j.s = nullptr;
      return rc;
    }
    configure_case(sv, j.s);
  }
  a3d_solver_set_free(j.s, r.F);
  a3d_solver_set_fix(j.s, r.fix);
  if (!j.res.warm) a3d_solver_reset(j.s);
  j.it_start = j.s->it;
  double dummy;
  a3d_solver_residual(j.s, 1, &dummy);  // snapshot
  if (!j.res.warm && sv->cfg.sequence > 1) return start_coarse(sv, j);
  return A3D_OK;
}

// Completes a request: its FP64 forces and Trefftz drag (GPU work, without sv->mu), then under
// the lock the result, the cache and the resident bytes; a case that is not kept is freed
// after the lock is released.
void finish_case(a3d_server* sv, Job& j, int status) {
  a3d_result& o = j.res;
  o.status = status;
  o.iterations = j.s ? j.s->it - j.it_start : 0;
  if (status == A3D_OK) {
    const a3d_request& r = j.req;
    double f[3] = {0, 0, 0}, cdi = 0;
    int rc = a3d_solver_forces(j.s, r.alpha_deg, r.M < 0.05 ? 0.05 : r.M, r.ref_S, r.ref_xcg, r.ref_zcg, r.ref_c, f);
    if (rc == A3D_OK) rc = a3d_solver_trefftz(j.s, r.xT, r.alpha_deg, r.M, r.ref_S, &cdi);
    o.CL = f[0]; o.CD = f[1]; o.Cm = f[2]; o.CDi = cdi;
    o.status = rc;
  }
  o.res0 = j.res0;
  o.coarse_iterations = j.coarse_its;
  drop_coarse(sv, j);
  j.t_done = Clock::now();
  o.t_submit = secs(sv, j.t_submit);
  o.t_admit = secs(sv, j.t_admit);
  o.t_done = secs(sv, j.t_done);
  a3d_solver* discard = nullptr;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (j.s) {
      if (status == A3D_OK && sv->cfg.warm_start) {
        sv->cache.insert({j.req.geometry_key, Cached{j.s, j.bytes, j.res0, ++sv->tick, false}});
      } else {
        sv->resident -= j.bytes;
        discard = j.s;
      }
      j.s = nullptr;
    }
    j.done = true;
    sv->completed++;
  }
  if (discard) a3d_solver_destroy(discard);
}

void scheduler(a3d_server* sv) {
  cudaSetDevice(sv->cfg.device);
  a3d_batch* batch = nullptr;
  // The batch is keyed by (request id, coarse phase), never by solver address: a finished
  // case's solver is destroyed and the next one may be allocated at the same address, and a
  // batch kept for it would still hold the old case's device table (buffers, tensor maps).
  std::vector<std::pair<int64_t, int>> batch_key;
  for (;;) {
    std::vector<std::shared_ptr<Job>> admit;
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      sv->cv_work.wait_for(lk, std::chrono::milliseconds(50),
                           [&] { return sv->stop || !sv->pending.empty() || !sv->active.empty(); });
      if (sv->stop) break;
      // admission: arrival order, slot cap and memory budget.  A request is warm only while an
      // idle cached case of its geometry is still unpromised: it reserves that case (which
      // then cannot be evicted) and adds no bytes; every other request adds its estimate,
      // which must fit the budget once the unreserved idle cases are evicted.
      size_t planned = sv->resident, idle = 0;
      for (auto& c : sv->cache)
        if (!c.second.reserved) idle += c.second.bytes;
      while (!sv->pending.empty() && (int)(sv->active.size() + admit.size()) < sv->cfg.max_active) {
        auto& j = sv->pending.front();
        const double est = request_bytes(j->req, sv->cfg.sequence);
        Cached* hit = nullptr;
        if (sv->cfg.warm_start) {
          auto range = sv->cache.equal_range(j->req.geometry_key);
          for (auto it = range.first; it != range.second; ++it)
            if (!it->second.reserved) { hit = &it->second; break; }
        }
        if (!hit && planned + est > sv->cfg.hbm_budget_bytes + idle) break;  // wait for memory
        if (hit) {
          hit->reserved = true;
          idle -= hit->bytes;
          j->planned_warm = true;
        } else {
          planned += (size_t)est;
        }
        admit.push_back(j);
        sv->pending.pop_front();
      }
    }
    for (auto& j : admit) {
      j->t_admit = Clock::now();
      const int rc = start_case(sv, *j);
      if (rc != A3D_OK) {
        finish_case(sv, *j, rc);
        sv->cv_done.notify_all();
      } else {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->active.push_back(j);
      }
    }
    std::vector<std::shared_ptr<Job>> act;
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      act = sv->active;
    }
    if (act.empty()) continue;
    // one round: all active cases advance together
    std::vector<a3d_solver*> set;
    std::vector<std::pair<int64_t, int>> key;
    for (auto& j : act) {
      set.push_back(j->coarse ? j->coarse : j->s);
      key.emplace_back(j->id, j->coarse ? 1 : 0);
    }
    if (!batch || key != batch_key) {
      if (batch) a3d_batch_destroy(batch);
      batch = nullptr;
      if (a3d_batch_create(set.data(), (int)set.size(), &batch) != A3D_OK) {
        {
          std::lock_guard<std::mutex> lk(sv->mu);
          sv->last_error = A3D_ERR_CUDA;
          sv->last_error_msg = a3d_last_error();
        }
        for (auto& j : act) finish_case(sv, *j, A3D_ERR_CUDA);
        {
          std::lock_guard<std::mutex> lk(sv->mu);
          sv->active.clear();
        }
        sv->cv_done.notify_all();
        batch_key.clear();
        continue;
      }
      int32_t kz0 = 0, ct0 = 0;  // keep the batch's default CTAs per SM for its tile
      a3d_batch_get_schedule(batch, &kz0, &ct0, nullptr);
      a3d_batch_set_schedule(batch, sv->cfg.kz > 0 ? sv->cfg.kz : kz0, ct0);
      batch_key = key;
    }
    int rc = a3d_batch_step(batch, sv->cfg.chunk_iters);
    if (rc == A3D_OK) rc = a3d_batch_sync(batch);
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->rounds++;
    }
    std::vector<std::shared_ptr<Job>> still;
    for (auto& j : act) {
      double res = -1;
      int st = rc != A3D_OK ? rc : a3d_solver_residual(j->coarse ? j->coarse : j->s, 1, &res);
      if (st == A3D_OK && j->coarse) {  // sequencing: the coarse case's own stopping rule
        if (j->coarse_res0 <= 0 && res > 0) j->coarse_res0 = res;
        if ((j->coarse_res0 > 0 && res / j->coarse_res0 <= sv->cfg.sequence_drop) ||
            j->coarse->it >= sv->cfg.sequence_max_iters)
          st = switch_to_target(sv, *j);
        if (st == A3D_OK) {
          still.push_back(j);
          continue;
        }
      }
      const long its = j->s->it - j->it_start;
      bool fin = st != A3D_OK;
      if (!fin) {
        if (j->res0 <= 0 && res > 0) j->res0 = res;
        j->res.residual = res;
        fin = (j->res0 > 0 && res / j->res0 <= sv->cfg.residual_drop) || its >= sv->cfg.max_iters;
      }
      if (fin) {
        finish_case(sv, *j, st);
      } else {
        still.push_back(j);
      }
    }
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->active = still;
    }
    sv->cv_done.notify_all();
  }
  if (batch) a3d_batch_destroy(batch);
}

}  // namespace

using namespace a3d;

extern "C" int a3d_server_create(const a3d_server_config* cfg, a3d_server** out) {
  clear_error();
  A3D_ARG(cfg && out, "null pointer");
  A3D_ARG(cfg->chunk_iters >= 1 && cfg->max_iters >= 1 && cfg->max_active >= 1, "server limits");
  A3D_ARG(cfg->hbm_budget_bytes > 0 && cfg->residual_drop > 0, "server budget / residual drop");
  A3D_ARG(cfg->sequence <= 1 || (cfg->sequence_drop > 0 && cfg->sequence_max_iters >= 1), "sequencing limits");
  A3D_TRY(use_device(cfg->device));
  a3d_server* sv = new a3d_server();
  sv->cfg = *cfg;
  if (sv->cfg.kz <= 0) sv->cfg.kz = 16;
  sv->t0 = Clock::now();
  sv->th = std::thread(scheduler, sv);
  *out = sv;
  return A3D_OK;
}

extern "C" int a3d_server_submit(a3d_server* sv, const a3d_request* req, int64_t* id) {
  clear_error();
  A3D_ARG(sv && req && id, "null pointer");
  A3D_ARG(req->cells >= 8 && req->M > 0, "request");
  auto j = std::make_shared<Job>();
  j->req = *req;
  j->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (request_bytes(*req, sv->cfg.sequence) > sv->cfg.hbm_budget_bytes) {
      set_error("request needs about %.1f GB, above the %.1f GB budget", request_bytes(*req, sv->cfg.sequence) * 1e-9,
                sv->cfg.hbm_budget_bytes * 1e-9);
      return A3D_ERR_BUDGET;
    }
    j->id = sv->next_id++;
    sv->jobs[j->id] = j;
    sv->pending.push_back(j);
    *id = j->id;
  }
  sv->cv_work.notify_one();
  return A3D_OK;
}

extern "C" int a3d_server_poll(a3d_server* sv, int64_t id, a3d_result* out, int32_t* done) {
  clear_error();
  A3D_ARG(sv && out && done, "null pointer");
  std::lock_guard<std::mutex> lk(sv->mu);
  auto it = sv->jobs.find(id);
  A3D_ARG(it != sv->jobs.end(), "unknown request id");
  *done = it->second->done;
  if (*done) *out = it->second->res;
  return A3D_OK;
}

extern "C" int a3d_server_wait(a3d_server* sv, int64_t id, double timeout_s, a3d_result* out) {
  clear_error();
  A3D_ARG(sv && out, "null pointer");
  std::unique_lock<std::mutex> lk(sv->mu);
  auto it = sv->jobs.find(id);
  A3D_ARG(it != sv->jobs.end(), "unknown request id");
  auto j = it->second;
  if (!sv->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] { return j->done; })) {
    set_error("request %lld not finished after %.1f s", (long long)id, timeout_s);
    return A3D_ERR_TIMEOUT;
  }
  *out = j->res;
  return A3D_OK;
}

extern "C" int a3d_server_stats(a3d_server* sv, int64_t out[6]) {
  clear_error();
  A3D_ARG(sv && out, "null pointer");
  std::lock_guard<std::mutex> lk(sv->mu);
  out[0] = (int64_t)sv->pending.size();
  out[1] = (int64_t)sv->active.size();
  out[2] = sv->completed;
  out[3] = sv->warm_starts;
  out[4] = sv->rounds;
  out[5] = (int64_t)sv->resident;
  return A3D_OK;
}

extern "C" int a3d_server_destroy(a3d_server* sv) {
  if (!sv) return A3D_OK;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stop = true;
  }
  sv->cv_work.notify_all();
  if (sv->th.joinable()) sv->th.join();
  for (auto& j : sv->active)
    if (j->s) a3d_solver_destroy(j->s);
  for (auto& c : sv->cache) a3d_solver_destroy(c.second.s);
  delete sv;
  return A3D_OK;
}
