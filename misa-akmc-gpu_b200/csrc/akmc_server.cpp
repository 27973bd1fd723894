// akmc_server.cpp -- job server over the context API of include/akmc.h.
//
// Jobs queue in arrival order and are admitted oldest first, or smallest hop budget first.
// Each lane is a host thread with one context (hence one CUDA stream) for its whole life,
// created with room for many jobs (akmc_context_config.max_jobs).  Between chunks of rounds the
// lane admits queued jobs that fit the device-memory budget and the context's room
// (akmc_admit_job), runs one chunk of rounds of every live job, and publishes each job that is
// done -- its lattice read back, its slots and memory freed (akmc_retire_job) -- while the
// others keep running.  So a job's lattice, density cache, vacancies and random streams stay in
// device memory from admission to its end, and its trajectory is exactly the one it has alone.
// A chunk is one time-boxed launch (akmc_run_for, cfg.chunk_us): every live job advances as far
// as its own rounds allow in that time, so small jobs are not held to the pace of the largest;
// the queue is checked after every chunk.  Lanes overlap on the GPU.  All shared
// state is under one mutex; the device work runs outside it.
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

// Room of a lane's context: domain blocks and vacancies held at once, the largest block edge.
constexpr int64_t kLaneBlocks = 1 << 14;
constexpr int64_t kLaneVacancies = 1 << 18;
constexpr int32_t kLaneBlockEdge = 24;

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
  int32_t slot = -1;  // its job id in the lane's context while it runs
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
  // profile, summed over lanes (under the mutex): seconds changing the lanes' job sets
  // (creating the contexts, admitting and retiring jobs), running chunks (rounds and the
  // job-state read), reading results, and waiting for work; chunks run, live jobs summed over
  // chunks, contexts built
  double t_build = 0, t_run = 0, t_publish = 0, t_wait = 0;
  double t_admit = 0, t_create = 0, t_retire = 0;  // parts of t_build
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

  // Under the lock: the next queued job that fits the budget, moved to running.
  std::shared_ptr<SJob> take_one_locked() {
    if (stopping || !fits_locked()) return nullptr;
    const auto it = next_locked();
    auto j = *it;
    queue.erase(it);
    j->state = 1;
    j->res.start_s = now();
    held += j->bytes;
    ++running;
    return j;
  }
  // Under the lock: a job taken but not admitted (the context is full) goes back to the front.
  void put_back_locked(const std::shared_ptr<SJob>& j) {
    j->state = 0;
    held -= j->bytes;
    --running;
    queue.push_front(j);
  }

  // One lane: a context for the lane's life, jobs admitted and retired between chunks.
  void lane() {
    auto tc = std::chrono::steady_clock::now();
    akmc_context_config cc{};
    cc.device = cfg.device;
    cc.graph_rounds = cfg.chunk_rounds;
    cc.max_jobs = cfg.max_batch_jobs;
    cc.max_block_edge = kLaneBlockEdge;
    cc.max_blocks = kLaneBlocks;
    cc.max_vacancies = kLaneVacancies;
    akmc_ctx* ctx = nullptr;
    akmc_status st = akmc_create(&cc, &ctx);
    if (st == AKMC_OK) st = akmc_prepare(ctx);
    add_time(t_create, tc);
    add_time(t_build, tc);
    {
      std::lock_guard<std::mutex> lk(m);
      ++n_builds;
    }
    std::vector<std::shared_ptr<SJob>> slots;  // by job id of the context
    std::vector<akmc_job_state> js;
    size_t live = 0;
    if (st != AKMC_OK) {  // no context: every job this lane takes fails with the reason
      for (;;) {
        std::shared_ptr<SJob> j;
        {
          std::unique_lock<std::mutex> lk(m);
          cv_work.wait(lk, [&] { return stopping || fits_locked(); });
          if (stopping) break;
          j = take_one_locked();
        }
        if (j) publish(j, st, ctx);
      }
      if (ctx) akmc_destroy(ctx);
      return;
    }
    for (;;) {
      // admit what fits (budget and room), oldest (or smallest budget) first
      auto ta = std::chrono::steady_clock::now();
      while (st == AKMC_OK) {
        std::shared_ptr<SJob> j;
        {
          std::lock_guard<std::mutex> lk(m);
          if (static_cast<int32_t>(live) >= cfg.max_batch_jobs) break;
          j = take_one_locked();
        }
        if (!j) break;
        akmc_job_config c = j->cfg;
        c.eam = j->has_eam ? &j->eam : nullptr;
        int32_t id = -1;
        const akmc_status s = akmc_admit_job(ctx, &c, j->occ.data(), static_cast<int64_t>(j->occ.size()), &id);
        if (s == AKMC_EBUSY && live > 0) {  // no room until a running job ends
          std::lock_guard<std::mutex> lk(m);
          put_back_locked(j);
          break;
        }
        if (s != AKMC_OK) {
          publish(j, s, ctx);
          continue;
        }
        j->slot = id;
        if (static_cast<size_t>(id) >= slots.size()) slots.resize(static_cast<size_t>(id) + 1);
        slots[static_cast<size_t>(id)] = j;
        ++live;
      }
      add_time(t_admit, ta);
      add_time(t_build, ta);
      if (st != AKMC_OK) {  // the lane's context failed: its jobs fail, the lane stops
        for (auto& j : slots)
          if (j) publish(j, st, ctx);
        break;
      }
      if (live == 0) {
        const auto tw = std::chrono::steady_clock::now();
        std::unique_lock<std::mutex> lk(m);
        cv_work.wait(lk, [&] { return stopping || fits_locked(); });
        t_wait += std::chrono::duration<double>(std::chrono::steady_clock::now() - tw).count();
        if (stopping) break;
        continue;
      }
      // one chunk: every live job advances as far as it can in cfg.chunk_us
      auto tr = std::chrono::steady_clock::now();
      st = akmc_run_for(ctx, int64_t(1) << 40, cfg.chunk_us);
      js.resize(slots.size());
      if (st == AKMC_OK) st = akmc_get_job_states(ctx, js.data(), static_cast<int32_t>(js.size()));
      add_time(t_run, tr);
      {
        std::lock_guard<std::mutex> lk(m);
        ++n_chunks;
        n_live += static_cast<int64_t>(live);
      }
      // publish and retire the jobs that are done
      auto tp = std::chrono::steady_clock::now();
      for (size_t k = 0; st == AKMC_OK && k < slots.size(); ++k) {
        auto& j = slots[k];
        if (!j || !js[k].done) continue;
        j->out.resize(j->occ.size());
        st = akmc_get_occupancy(ctx, static_cast<int32_t>(k), j->out.data(), static_cast<int64_t>(j->out.size()));
        if (st != AKMC_OK) break;
        j->res.hops = js[k].hops;
        j->res.rounds = js[k].round;
        j->res.n_blocks = js[k].n_blocks;
        {
          const size_t nb = static_cast<size_t>(js[k].n_blocks);
          std::vector<double> evo(8 * nb);
          std::vector<int64_t> bh(nb);
          st = akmc_get_block_clocks(ctx, static_cast<int32_t>(k), evo.data(), bh.data(), js[k].n_blocks);
          if (st != AKMC_OK) break;
          uint64_t h = 0xCBF29CE484222325ull;
          auto mix = [&h](const void* p, size_t n) {
            const unsigned char* b = static_cast<const unsigned char*>(p);
            for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 0x100000001B3ull;
          };
          for (size_t b = 0; b < nb; ++b) {
            mix(evo.data() + 8 * b, 8 * sizeof(double));
            mix(&bh[b], sizeof(int64_t));
          }
          j->res.clocks_fnv = h;
        }
        auto tt = std::chrono::steady_clock::now();
        st = akmc_retire_job(ctx, static_cast<int32_t>(k));
        add_time(t_retire, tt);
        add_time(t_build, tt);
        publish(j, st == AKMC_OK ? AKMC_OK : st, ctx);
        j = nullptr;
        --live;
      }
      add_time(t_publish, tp);
      if (st != AKMC_OK) {
        for (auto& j : slots)
          if (j) publish(j, st, ctx);
        break;
      }
    }
    if (ctx) akmc_destroy(ctx);
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
  if (s->cfg.chunk_us <= 0) s->cfg.chunk_us = 2000;
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
  for (int d = 0; d < 3; ++d) {
    if (cfg->box[d] < 8 || cfg->box[d] > (1 << 20)) return AKMC_EINVAL;
    const int64_t nb = cfg->blocks[d] > 0 ? cfg->blocks[d] : 1;
    if ((cfg->box[d] + nb - 1) / nb > kLaneBlockEdge) return AKMC_EINVAL;  // blocks larger than a lane takes
  }
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
  seconds8[4] = s->t_admit;
  seconds8[5] = s->t_create;
  seconds8[6] = s->t_retire;
  seconds8[7] = 0.0;
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
