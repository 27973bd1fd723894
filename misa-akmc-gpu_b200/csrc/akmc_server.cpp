// akmc_server.cpp -- job server over the context API of include/akmc.h.
//
// Jobs queue in arrival order and are admitted oldest first, or smallest hop budget first.  Each lane (a host thread with its own context, hence its own
// CUDA stream) takes the queued jobs that fit the device-memory budget as one batch and runs
// them together in chunks of rounds.  A job's result is published, and its memory returned to
// the budget, as soon as that job is done.  When an eighth of a batch has finished and queued
// jobs fit, the lane refills: the running jobs are saved as restart snapshots, the context is
// rebuilt with them and the newly admitted jobs, and the snapshots are restored, so every
// job's trajectory is exactly the one it has alone.  A lane also refills, after 8 chunks, when
// at least as many jobs wait as it runs.  A lane whose live jobs are all single-block boxes, with
// none queued, runs them round by round in chunks 8 times longer: those jobs are the small boxes
// with large hop budgets that end a run, latency bound, and the dependency-driven schedule's
// launches (at most a time step each for budget jobs) cost more than their rounds; single-block
// jobs keep one another's pace in lockstep.  Both schedules give the same trajectory.  Lanes overlap on the GPU.  All shared state is under one mutex; the device work
// runs outside it.
#include <algorithm>
#include <chrono>
#include <climits>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/akmc.h"

namespace {

// Chunks of a batch's tail (single-block jobs only, empty queue): this many times the
// configured length.
constexpr int64_t kTailChunks = 8;

struct SJob {
  int64_t ticket = 0;
  akmc_job_config cfg{};
  bool has_eam = false;
  akmc_eam_tables eam{};
  std::vector<uint8_t> occ;
  int64_t bytes = 0;
  int state = 0;  // 0 queued, 1 running, 2 done
  akmc_job_result res{};
  std::vector<uint8_t> out;
  std::vector<uint8_t> snap;  // restart snapshot while the job moves to a rebuilt context
};

// Device bytes a job holds: occupancy, density cache, block records and lists, vacancies.
int64_t job_bytes(const akmc_job_config& c, int64_t nsites, int64_t nvac) {
  const int64_t nb = static_cast<int64_t>(std::max(1, c.blocks[0])) * std::max(1, c.blocks[1]) * std::max(1, c.blocks[2]);
  const int64_t per_site = c.energy_model == AKMC_MODEL_EAM ? 5 : 1;
  return nsites * per_site + nb * 1024 + nvac * 16 + (c.energy_model == AKMC_MODEL_EAM ? 400000 : 0);
}

}  // namespace

struct akmc_server {
  akmc_server_config cfg{};
  std::mutex m;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<SJob>> queue;
  std::unordered_map<int64_t, std::shared_ptr<SJob>> jobs;  // queued, running or done, not collected
  int64_t next_ticket = 1;
  int64_t held = 0;     // bytes of the jobs in running batches
  int64_t running = 0;  // jobs in running batches
  bool stopping = false;
  std::vector<std::thread> lanes;
  // profile, summed over lanes (under the mutex): seconds building contexts (create, add,
  // prepare, restore), running chunks (rounds and the job-state read), reading results, and
  // waiting for work; chunks run, live jobs summed over chunks, contexts built
  double t_build = 0, t_run = 0, t_publish = 0, t_wait = 0;
  double t_add = 0, t_prepare = 0, t_restore = 0, t_save = 0;  // parts of t_build
  int64_t n_chunks = 0, n_live = 0, n_builds = 0;
  void add_time(double& slot, std::chrono::steady_clock::time_point since) {
    const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - since).count();
    std::lock_guard<std::mutex> lk(m);
    slot += dt;
  }
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }

  // Under the lock: the job's result is final and its bytes go back to the budget.
  void publish(const std::shared_ptr<SJob>& j, int32_t status, akmc_ctx* ctx = nullptr) {
    char msg[sizeof(j->res.error)] = {0};
    if (status != AKMC_OK && ctx) akmc_last_error(ctx, msg, static_cast<int32_t>(sizeof(msg)));
    {
      std::lock_guard<std::mutex> lk(m);
      j->res.status = status;
      std::memcpy(j->res.error, msg, sizeof(msg));
      j->res.finish_s = now();
      j->state = 2;
      j->snap.clear();
      j->snap.shrink_to_fit();
      --running;
      held -= j->bytes;
    }
    cv_done.notify_all();
    cv_work.notify_all();
  }

  // The queued job admitted next: the oldest, or the one with the smallest hop budget (jobs
  // without a budget last, ties by arrival).
  std::deque<std::shared_ptr<SJob>>::const_iterator next_locked() const {
    if (cfg.order != AKMC_SERVE_SMALLEST_BUDGET || queue.empty()) return queue.begin();
    auto key = [](const std::shared_ptr<SJob>& j) {
      return j->cfg.hop_budget > 0 ? j->cfg.hop_budget : INT64_MAX;
    };
    auto best = queue.begin();
    for (auto it = queue.begin(); it != queue.end(); ++it)
      if (key(*it) < key(*best)) best = it;  // strictly smaller: the earliest of equals stays
    return best;
  }

  bool fits_locked() const {
    return !queue.empty() && held + (*next_locked())->bytes <= cfg.budget_bytes;
  }

  // Under the lock: moves queued jobs that fit into `live`.
  void take_locked(std::vector<std::shared_ptr<SJob>>& live) {
    while (fits_locked() && static_cast<int32_t>(live.size()) < cfg.max_batch_jobs) {
      const auto it = next_locked();
      auto j = *it;
      queue.erase(it);
      j->state = 1;
      j->res.start_s = now();
      held += j->bytes;
      ++running;
      live.push_back(j);
    }
  }

  // Runs `live` until every job is done, refilling from the queue on the way.
  void run_batch(std::vector<std::shared_ptr<SJob>>& live) {
    while (!live.empty()) {
      auto tb = std::chrono::steady_clock::now();
      akmc_context_config cc{};
      cc.device = cfg.device;
      cc.graph_rounds = cfg.chunk_rounds;
      akmc_ctx* ctx = nullptr;
      akmc_status st = akmc_create(&cc, &ctx);
      if (st != AKMC_OK) {
        for (auto& j : live) publish(j, st);
        live.clear();
        return;
      }
      auto tpart = std::chrono::steady_clock::now();
      std::vector<std::shared_ptr<SJob>> in;  // jobs of this context, by job id
      for (auto& j : live) {
        akmc_job_config c = j->cfg;
        c.eam = j->has_eam ? &j->eam : nullptr;
        int32_t id = -1;
        const akmc_status s = akmc_add_job(ctx, &c, j->occ.data(), static_cast<int64_t>(j->occ.size()), &id);
        if (s != AKMC_OK) publish(j, s, ctx);
        else in.push_back(j);
      }
      add_time(t_add, tpart);
      tpart = std::chrono::steady_clock::now();
      if (!in.empty()) st = akmc_prepare(ctx);
      add_time(t_prepare, tpart);
      tpart = std::chrono::steady_clock::now();
      for (size_t k = 0; st == AKMC_OK && k < in.size(); ++k)
        if (!in[k]->snap.empty())
          st = akmc_restore_snapshot(ctx, static_cast<int32_t>(k), in[k]->snap.data(),
                                     static_cast<int64_t>(in[k]->snap.size()));
      add_time(t_restore, tpart);
      add_time(t_build, tb);
      {
        std::lock_guard<std::mutex> lk(m);
        ++n_builds;
      }
      std::vector<bool> over(in.size(), false);
      std::vector<akmc_job_state> js(in.size());
      size_t left = in.size(), finished = 0, chunks_here = 0;
      const size_t refill_after = std::max<size_t>(1, in.size() / 8);
      bool refill = false;
      while (st == AKMC_OK && left > 0 && !refill) {
        auto tr = std::chrono::steady_clock::now();
        bool tail = chunks_here > 0;  // job states known
        for (size_t k = 0; tail && k < in.size(); ++k) tail = over[k] || js[k].n_blocks == 1;
        if (tail) {
          std::lock_guard<std::mutex> lk(m);
          tail = queue.empty();
        }
        st = akmc_set_round_schedule(ctx, tail ? AKMC_SCHEDULE_ROUNDS : AKMC_SCHEDULE_AUTO);
        if (st == AKMC_OK) st = akmc_run_rounds(ctx, tail ? kTailChunks * cfg.chunk_rounds : cfg.chunk_rounds);
        if (st == AKMC_OK) st = akmc_get_job_states(ctx, js.data(), static_cast<int32_t>(in.size()));
        add_time(t_run, tr);
        {
          std::lock_guard<std::mutex> lk(m);
          ++n_chunks;
          n_live += static_cast<int64_t>(left);
        }
        auto tp = std::chrono::steady_clock::now();
        for (size_t k = 0; st == AKMC_OK && k < in.size(); ++k) {
          if (over[k] || !js[k].done) continue;
          auto& j = in[k];
          j->out.resize(j->occ.size());
          st = akmc_get_occupancy(ctx, static_cast<int32_t>(k), j->out.data(), static_cast<int64_t>(j->out.size()));
          if (st != AKMC_OK) break;
          j->res.hops = js[k].hops;
          j->res.rounds = js[k].round;
          j->res.n_blocks = js[k].n_blocks;
          publish(j, AKMC_OK);
          over[k] = true;
          --left;
          ++finished;
        }
        add_time(t_publish, tp);
        ++chunks_here;
        if (st == AKMC_OK && left > 0) {
          // refill when an eighth of the batch is done, or when at least as many jobs wait as
          // run (a small early batch of long jobs must not hold the queue back)
          std::lock_guard<std::mutex> lk(m);
          const bool grow = queue.size() >= left && chunks_here >= 8;
          refill = !stopping && fits_locked() && static_cast<int32_t>(left) < cfg.max_batch_jobs &&
                   (finished >= refill_after || grow);
        }
      }
      live.clear();
      tb = std::chrono::steady_clock::now();
      for (size_t k = 0; k < in.size(); ++k) {
        if (over[k]) continue;
        if (st != AKMC_OK) {
          publish(in[k], st, ctx);
          continue;
        }
        // carried into the next context
        int64_t n = 0;
        st = akmc_snapshot_size(ctx, static_cast<int32_t>(k), &n);
        if (st == AKMC_OK) {
          in[k]->snap.resize(static_cast<size_t>(n));
          int64_t w = 0;
          st = akmc_save_snapshot(ctx, static_cast<int32_t>(k), in[k]->snap.data(), n, &w);
        }
        if (st != AKMC_OK) publish(in[k], st, ctx);
        else live.push_back(in[k]);
      }
      add_time(t_save, tb);
      akmc_destroy(ctx);
      add_time(t_build, tb);
      if (!live.empty()) {
        std::lock_guard<std::mutex> lk(m);
        take_locked(live);
      }
    }
  }

  void lane() {
    for (;;) {
      std::vector<std::shared_ptr<SJob>> live;
      {
        const auto tw = std::chrono::steady_clock::now();
        std::unique_lock<std::mutex> lk(m);
        cv_work.wait(lk, [&] { return stopping || fits_locked(); });
        t_wait += std::chrono::duration<double>(std::chrono::steady_clock::now() - tw).count();
        if (stopping) return;
        take_locked(live);
      }
      run_batch(live);
    }
  }
};

namespace {

bool collect(akmc_server* s, const std::shared_ptr<SJob>& j, akmc_job_result* res, uint8_t* occ_out, int64_t n) {
  if (res) *res = j->res;
  if (occ_out && !j->out.empty()) std::memcpy(occ_out, j->out.data(), static_cast<size_t>(std::min<int64_t>(n, static_cast<int64_t>(j->out.size()))));
  s->jobs.erase(j->ticket);
  return true;
}

}  // namespace

extern "C" {

AKMC_API akmc_status akmc_server_create(const akmc_server_config* cfg, akmc_server** out) {
  if (!out) return AKMC_EINVAL;
  *out = nullptr;
  akmc_server* s = new (std::nothrow) akmc_server();
  if (!s) return AKMC_ENOMEM;
  if (cfg) s->cfg = *cfg;
  if (s->cfg.lanes <= 0) s->cfg.lanes = 2;
  if (s->cfg.budget_bytes <= 0) s->cfg.budget_bytes = int64_t(8) << 30;
  if (s->cfg.max_batch_jobs <= 0) s->cfg.max_batch_jobs = 512;
  if (s->cfg.chunk_rounds <= 0) s->cfg.chunk_rounds = 16;
  try {
    for (int i = 0; i < s->cfg.lanes; ++i) s->lanes.emplace_back([s] { s->lane(); });
  } catch (...) {
    {
      std::lock_guard<std::mutex> lk(s->m);
      s->stopping = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->lanes) t.join();
    delete s;
    return AKMC_ENOMEM;
  }
  *out = s;
  return AKMC_OK;
}

AKMC_API akmc_status akmc_server_submit(akmc_server* s, const akmc_job_config* cfg, const uint8_t* occ,
                                        int64_t n_sites, int64_t* ticket) {
  if (!s || !cfg || !occ || !ticket) return AKMC_EINVAL;
  *ticket = 0;
  if (cfg->hop_budget <= 0 && cfg->max_rounds <= 0) return AKMC_EINVAL;  // the job would never end
  for (int d = 0; d < 3; ++d)
    if (cfg->box[d] < 8 || cfg->box[d] > (1 << 20)) return AKMC_EINVAL;
  if (n_sites != 2 * cfg->box[0] * cfg->box[1] * cfg->box[2]) return AKMC_EINVAL;
  if (cfg->energy_model == AKMC_MODEL_EAM && !cfg->eam) return AKMC_EINVAL;
  auto j = std::make_shared<SJob>();
  j->cfg = *cfg;
  j->has_eam = cfg->eam != nullptr;
  if (j->has_eam) j->eam = *cfg->eam;
  j->cfg.eam = nullptr;
  j->occ.assign(occ, occ + n_sites);
  const int64_t nvac = std::count(j->occ.begin(), j->occ.end(), static_cast<uint8_t>(AKMC_V));
  j->bytes = job_bytes(*cfg, n_sites, nvac);
  {
    std::lock_guard<std::mutex> lk(s->m);
    if (s->stopping) return AKMC_ESTATE;
    if (j->bytes > s->cfg.budget_bytes) return AKMC_EINVAL;
    j->ticket = s->next_ticket++;
    j->res.submit_s = s->now();
    s->jobs[j->ticket] = j;
    s->queue.push_back(j);
    *ticket = j->ticket;
  }
  s->cv_work.notify_one();
  return AKMC_OK;
}

AKMC_API akmc_status akmc_server_poll(akmc_server* s, int64_t ticket, akmc_job_result* res, uint8_t* occ_out,
                                      int64_t n_sites, int32_t* ready) {
  if (!s || !ready) return AKMC_EINVAL;
  *ready = 0;
  std::lock_guard<std::mutex> lk(s->m);
  auto it = s->jobs.find(ticket);
  if (it == s->jobs.end()) return AKMC_ENOTFOUND;
  auto j = it->second;
  if (j->state != 2) return AKMC_OK;
  if (occ_out && n_sites != static_cast<int64_t>(j->occ.size())) return AKMC_EINVAL;
  collect(s, j, res, occ_out, n_sites);
  *ready = 1;
  return AKMC_OK;
}

AKMC_API akmc_status akmc_server_wait(akmc_server* s, int64_t ticket, double timeout_s, akmc_job_result* res,
                                      uint8_t* occ_out, int64_t n_sites) {
  if (!s) return AKMC_EINVAL;
  std::unique_lock<std::mutex> lk(s->m);
  auto it = s->jobs.find(ticket);
  if (it == s->jobs.end()) return AKMC_ENOTFOUND;
  auto j = it->second;
  if (occ_out && n_sites != static_cast<int64_t>(j->occ.size())) return AKMC_EINVAL;
  const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(std::max(0.0, timeout_s)),
                                      [&] { return j->state == 2; });
  if (!ok) return AKMC_ETIMEOUT;
  collect(s, j, res, occ_out, n_sites);
  return AKMC_OK;
}

AKMC_API akmc_status akmc_server_stats(akmc_server* s, int64_t* queued, int64_t* running, int64_t* done) {
  if (!s) return AKMC_EINVAL;
  std::lock_guard<std::mutex> lk(s->m);
  int64_t d = 0;
  for (auto& kv : s->jobs) d += kv.second->state == 2 ? 1 : 0;
  if (queued) *queued = static_cast<int64_t>(s->queue.size());
  if (running) *running = s->running;
  if (done) *done = d;
  return AKMC_OK;
}

AKMC_API akmc_status akmc_server_profile(akmc_server* s, double* seconds8, int64_t* counts3) {
  if (!s || !seconds8 || !counts3) return AKMC_EINVAL;
  std::lock_guard<std::mutex> lk(s->m);
  seconds8[0] = s->t_build;
  seconds8[1] = s->t_run;
  seconds8[2] = s->t_publish;
  seconds8[3] = s->t_wait;
  seconds8[4] = s->t_add;
  seconds8[5] = s->t_prepare;
  seconds8[6] = s->t_restore;
  seconds8[7] = s->t_save;
  counts3[0] = s->n_chunks;
  counts3[1] = s->n_live;
  counts3[2] = s->n_builds;
  return AKMC_OK;
}

AKMC_API akmc_status akmc_server_shutdown(akmc_server* s) {
  if (!s) return AKMC_EINVAL;
  {
    std::lock_guard<std::mutex> lk(s->m);
    s->stopping = true;
    for (auto& j : s->queue) {
      j->state = 2;
      j->res.status = AKMC_ESTATE;
    }
    s->queue.clear();
  }
  s->cv_work.notify_all();
  for (auto& t : s->lanes) t.join();  // running batches finish first
  delete s;
  return AKMC_OK;
}

}  // extern "C"
