// Serving: a request loop with continuous batching. Requests (parameter set,
// seed, step count) queue on the host; each tick admits queued requests
// whose device footprint fits the HBM budget, advances every resident run by
// up to steps_per_tick fused steps in one batched launch sequence, copies out
// due snapshots and retires finished runs, freeing their memory for the
// queue. A run's result does not depend on which other runs share its
// launches: every kernel works per run, noise is keyed by (seed, particle,
// step) and all sums run in a fixed order.
//
// A request's initial positions (the reference's initialiser on the host,
// std::mt19937_64 seeded by the request) are drawn ahead of its admission by
// a host thread of the server, for the first requests of the queue, while the
// device steps the resident runs; admission then only allocates, uploads and
// sorts. The positions are those the run's own generator would draw, and the
// run's generator continues from the drawn state.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "bd_api.h"
#include "bd_engine.h"
#include "bd_host.h"

using bd::Engine;
using bd::RunHost;

namespace {
struct Request {
  long long id = 0;
  bd_params p{};
  uint64_t seed = 0;
  long long nsteps = 0;
  int snap_every = 0;
  int state = BD_REQ_QUEUED;
  long long done = 0;
  int snapshots = 0;
  double submit_s = 0, admit_s = 0, finish_s = 0;
  int error = 0;
  size_t bytes = 0;
  RunHost* run = nullptr;
  int C = 0;  // cells per side, to decode the records
  // final and last snapshot state as the device's cell-sorted records (one
  // copy each); converted to the reference layout only when asked for
  std::vector<bd::Rec> fin, snap;
  long long snap_step = -1;
  // initial positions drawn ahead of admission (prep: 0 not yet, 1 being
  // drawn, 2 ready with status prep_status) and the generator after drawing
  int prep = 0, prep_status = 0;
  std::vector<int32_t> g[2];
  std::vector<double> q[2];
  std::mt19937_64 gen;
};

// Draw the initial positions of a request with its own generator (seeded as
// the engine seeds a run's generator), into rq's buffers.
static void draw_positions(Request& rq) {
  rq.gen.seed(rq.seed);
  const int m = rq.p.startpos_methode == 2 ? 1 : rq.p.startpos_methode;
  rq.g[0].assign(2 * (size_t)rq.p.N1 + 2, 0);
  rq.g[1].assign(2 * (size_t)rq.p.N2 + 2, 0);
  rq.q[0].assign(2 * (size_t)rq.p.N1 + 2, 0.0);
  rq.q[1].assign(2 * (size_t)rq.p.N2 + 2, 0.0);
  int32_t* g[2] = {rq.g[0].data(), rq.g[1].data()};
  double* q[2] = {rq.q[0].data(), rq.q[1].data()};
  rq.prep_status = bd::init_positions_host(&rq.p, rq.gen, m, g, q);
}

// records -> git[N][2] / rel[N][2] of one species, in particle order
static void records_to_species(const std::vector<bd::Rec>& h, int N1, int C, int species, int32_t* git,
                               double* rel) {
  for (const bd::Rec& q : h) {
    const int s = q.pid >= N1;
    if (s != species) continue;
    const int i = s ? q.pid - N1 : q.pid;
    if (git) {
      git[2 * i] = q.cell / C;
      git[2 * i + 1] = q.cell % C;
    }
    if (rel) {
      rel[2 * i] = (double)q.ox;
      rel[2 * i + 1] = (double)q.oy;
    }
  }
}
}  // namespace

struct bd_server {
  Engine e;
  bd_serve_opts o{};
  std::string snapdir;
  size_t budget = 0, used = 0;
  std::deque<long long> queue;
  std::map<long long, Request> reqs;
  std::vector<long long> active;  // request id of e.runs[k]
  long long next_id = 1;
  std::chrono::steady_clock::time_point t0;
  std::vector<double> latencies;
  long long completed = 0;
  long long particle_steps = 0;
  double step_s = 0.0, tick_s = 0.0, admit_s = 0.0, plan_s = 0.0, fetch_s = 0.0;
  // the batch autotuner ran on a mix of this many particles (0: not yet); it
  // runs again once the resident mix has grown to twice that
  long long tuned_particles = 0;
  static constexpr long long TUNE_MIN_PARTICLES = 1 << 20;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  // the drawing thread: it takes the first queued requests without positions
  // (at most PREP_AHEAD ready ones ahead of admission). mu guards the queue,
  // the request map's structure and every request's prep fields.
  static constexpr int PREP_AHEAD = 32;
  std::thread drawer;
  std::mutex mu;
  std::condition_variable cv;
  bool stop = false;
};

// The next request the drawing thread should draw, or null (mu held).
static Request* next_to_draw(bd_server* s) {
  int ready = 0;
  for (long long id : s->queue) {
    auto it = s->reqs.find(id);
    if (it == s->reqs.end() || it->second.state != BD_REQ_QUEUED) continue;
    Request& rq = it->second;
    if (rq.prep == 0) return &rq;
    if (++ready >= bd_server::PREP_AHEAD) return nullptr;
  }
  return nullptr;
}

static void drawer_loop(bd_server* s) {
  for (;;) {
    Request* rq = nullptr;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv.wait(lk, [&] { return s->stop || (rq = next_to_draw(s)) != nullptr; });
      if (s->stop) return;
      rq->prep = 1;
    }
    draw_positions(*rq);
    {
      std::lock_guard<std::mutex> lk(s->mu);
      rq->prep = 2;
    }
    s->cv.notify_all();
  }
}

// The request's positions, drawn by the thread or here (mu not held).
static void take_positions(bd_server* s, Request& rq) {
  std::unique_lock<std::mutex> lk(s->mu);
  if (rq.prep == 0) {
    rq.prep = 1;
    lk.unlock();
    draw_positions(rq);
    lk.lock();
    rq.prep = 2;
    s->cv.notify_all();
    return;
  }
  s->cv.wait(lk, [&] { return rq.prep == 2; });
}

#define RK(x)                   \
  do {                          \
    int r_ = (x);               \
    if (r_ != BD_OK) return r_; \
  } while (0)

static int fetch_positions(Engine& e, size_t k, std::vector<bd::Rec>& out) {
  return e.get_records(k, out);
}

static int admit(bd_server* s, bool& changed) {
  for (;;) {
    if (s->o.max_runs > 0 && (int)s->active.size() >= s->o.max_runs) break;
    Request* head = nullptr;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      while (!s->queue.empty()) {
        auto it = s->reqs.find(s->queue.front());
        if (it != s->reqs.end() && it->second.state == BD_REQ_QUEUED) {
          head = &it->second;
          break;
        }
        s->queue.pop_front();
      }
    }
    if (!head) break;
    Request& rq = *head;
    if (s->used + rq.bytes > s->budget) break;  // first-come first-served
    RunHost* r = nullptr;
    int st = s->e.add_run(rq.p, rq.seed, &r);
    if (st == BD_ERR_NOMEM) break;  // device fuller than the budget says: retry later
    if (st == BD_OK) take_positions(s, rq);
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->queue.pop_front();
    }
    s->cv.notify_all();  // the drawing thread may take the next request
    if (st != BD_OK) {
      rq.state = BD_REQ_FAILED;
      rq.error = st;
      continue;
    }
    changed = true;
    s->used += rq.bytes;
    rq.run = r;
    rq.C = r->C;
    rq.state = BD_REQ_RUNNING;
    rq.admit_s = s->now();
    s->active.push_back(rq.id);
    const size_t k = s->e.runs.size() - 1;
    int32_t* g[2] = {rq.g[0].data(), rq.g[1].data()};
    double* q[2] = {rq.q[0].data(), rq.q[1].data()};
    st = rq.prep_status;
    r->gen = rq.gen;  // the run's generator continues after the drawn positions
    if (st == BD_OK) st = s->e.set_all_positions(k, g, q);
    for (int sp = 0; sp < 2; sp++) {  // converted into the engine's staging: not needed any more
      std::vector<int32_t>().swap(rq.g[sp]);
      std::vector<double>().swap(rq.q[sp]);
    }
    if (st != BD_OK) {
      // a run without a sorted state must not stay in the launch plan
      RK(s->e.remove_run(k));
      s->active.pop_back();
      s->used -= std::min(s->used, rq.bytes);
      rq.state = BD_REQ_FAILED;
      rq.error = st;
      rq.run = nullptr;
    }
  }
  return BD_OK;
}

static int retire(bd_server* s, size_t k, int state) {
  Request& rq = s->reqs[s->active[k]];
  rq.state = state;
  rq.finish_s = s->now();
  rq.run = nullptr;
  RK(s->e.remove_run(k));
  s->used -= std::min(s->used, rq.bytes);
  s->active.erase(s->active.begin() + k);
  if (state == BD_REQ_DONE) {
    s->completed++;
    s->latencies.push_back(rq.finish_s - rq.submit_s);
  }
  return BD_OK;
}

extern "C" {

int bd_serve_create(const bd_serve_opts* o, bd_server** out) {
  if (!o || !out) return BD_ERR_ARG;
  *out = nullptr;
  bd_server* s = new (std::nothrow) bd_server();
  if (!s) return BD_ERR_NOMEM;
  s->o = *o;
  if (s->o.steps_per_tick <= 0) s->o.steps_per_tick = 100;
  if (o->snapshot_dir) s->snapdir = o->snapshot_dir;
  s->o.snapshot_dir = nullptr;
  int st = s->e.init(o->device);
  if (st != BD_OK) {
    delete s;
    return st;
  }
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  s->budget = o->hbm_budget ? o->hbm_budget : (size_t)(0.8 * (double)fr);
  s->t0 = std::chrono::steady_clock::now();
  try {
    s->drawer = std::thread(drawer_loop, s);
  } catch (...) {
    delete s;
    return BD_ERR_NOMEM;
  }
  *out = s;
  return BD_OK;
}

int bd_serve_destroy(bd_server* s) {
  if (!s) return BD_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv.notify_all();
  if (s->drawer.joinable()) s->drawer.join();
  for (auto& e : s->ev)
    if (e) cudaEventDestroy(e);
  delete s;
  return BD_OK;
}

int bd_serve_submit(bd_server* s, const bd_params* p, uint64_t seed, long long nsteps,
                    int snapshot_every, long long* req_id) {
  if (!s || !p || nsteps < 0 || snapshot_every < 0) return BD_ERR_ARG;
  RK(bd::params_validate(p));
  if (p->max_reisedistanz < 1e20) return BD_ERR_UNSUPPORTED;  // serving steps with a fixed dt
  Request rq;
  rq.id = s->next_id++;
  rq.p = *p;
  rq.seed = seed;
  rq.nsteps = nsteps;
  rq.snap_every = snapshot_every;
  rq.submit_s = s->now();
  rq.bytes = s->e.footprint_of(*p);
  if (rq.bytes > s->budget) return BD_ERR_NOMEM;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->reqs[rq.id] = std::move(rq);
    s->queue.push_back(s->next_id - 1);
  }
  s->cv.notify_all();
  if (req_id) *req_id = s->next_id - 1;
  return BD_OK;
}

int bd_serve_cancel(bd_server* s, long long id) {
  if (!s) return BD_ERR_ARG;
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return BD_ERR_NOTFOUND;
  Request& rq = it->second;
  if (rq.state == BD_REQ_QUEUED) {
    std::lock_guard<std::mutex> lk(s->mu);
    rq.state = BD_REQ_CANCELLED;
    rq.finish_s = s->now();
    return BD_OK;
  }
  if (rq.state == BD_REQ_RUNNING) {
    for (size_t k = 0; k < s->active.size(); k++)
      if (s->active[k] == id) return retire(s, k, BD_REQ_CANCELLED);
  }
  return BD_ERR_STATE;
}

int bd_serve_poll(bd_server* s, long long id, bd_req_status* st) {
  if (!s || !st) return BD_ERR_ARG;
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return BD_ERR_NOTFOUND;
  const Request& rq = it->second;
  st->state = rq.state;
  st->steps_done = rq.done;
  st->steps_total = rq.nsteps;
  st->snapshots = rq.snapshots;
  st->submit_s = rq.submit_s;
  st->admit_s = rq.admit_s;
  st->finish_s = rq.finish_s;
  st->error = rq.error;
  return BD_OK;
}

static int serve_tick(bd_server* s, int* active);

int bd_serve_tick(bd_server* s, int* active) {
  if (!s) return BD_ERR_ARG;
  const double t0 = s->now();
  const int st = serve_tick(s, active);
  s->tick_s += s->now() - t0;
  return st;
}

static int serve_tick(bd_server* s, int* active) {
  bool changed = false;
  double t = s->now();
  RK(admit(s, changed));
  s->admit_s += s->now() - t;
  t = s->now();
  // runs with nothing left to do (nsteps == 0) retire at once
  for (size_t k = 0; k < s->active.size();) {
    Request& rq = s->reqs[s->active[k]];
    if (rq.done >= rq.nsteps) {
      RK(fetch_positions(s->e, k, rq.fin));
      RK(retire(s, k, BD_REQ_DONE));
      continue;
    }
    k++;
  }
  if (!s->active.empty()) {
    const long long K = s->o.steps_per_tick;
    std::vector<long long> budget(s->active.size());
    long long most = 0;
    for (size_t k = 0; k < s->active.size(); k++) {
      const Request& rq = s->reqs[s->active[k]];
      long long b = std::min(K, rq.nsteps - rq.done);
      if (rq.snap_every > 0) b = std::min(b, rq.snap_every - rq.done % rq.snap_every);
      budget[k] = b;
      most = std::max(most, b);
    }
    RK(s->e.set_steps_left_all(budget));
    // as many steps as the longest budget: launches past it would only skip
    // every run
    s->fetch_s += s->now() - t;
    t = s->now();
    RK(s->e.step(0));  // builds the plan first if the runs changed (device current), untimed
    // the plan's transform items and the particle kernel's shape are tuned
    // on the resident mix when it reaches 2^20 particles and again whenever
    // it has doubled since (a few times in a stream; every choice gives the
    // same bits, so results do not depend on when it ran)
    long long resident = 0;
    for (auto* r : s->e.runs) resident += r->N;
    if (resident >= bd_server::TUNE_MIN_PARTICLES && resident >= 2 * s->tuned_particles &&
        !s->e.uses_fused()) {
      bd_tune_result tr;
      const int st = s->e.autotune(2, &tr);
      if (st != BD_OK && st != BD_ERR_STATE) return st;
      s->tuned_particles = resident;
    }
    s->plan_s += s->now() - t;
    if (!s->ev[0]) {
      if (cudaEventCreate(&s->ev[0]) != cudaSuccess || cudaEventCreate(&s->ev[1]) != cudaSuccess)
        return BD_ERR_CUDA;
    }
    cudaEventRecord(s->ev[0], s->e.stream);
    RK(s->e.step(most));
    cudaEventRecord(s->ev[1], s->e.stream);
    std::vector<bd::RunDyn> y;
    RK(s->e.get_dyn_all(y));
    // a grid-barrier wait that gave up leaves the fused step's barrier words
    // set: the engine clears them and returns the run to its state before
    // the failed step (the request still ends with BD_ERR_TIMEOUT)
    for (const bd::RunDyn& d : y)
      if (d.err & bd::E_BARRIER_TIMEOUT) {
        s->e.sync_check();
        break;
      }
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, s->ev[0], s->ev[1]) == cudaSuccess) s->step_s += ms * 1e-3;
    t = s->now();
    for (size_t k = 0; k < s->active.size(); k++) {
      Request& rq = s->reqs[s->active[k]];
      const long long did = budget[k] - y[k].steps_left;
      rq.done += did;
      s->particle_steps += did * (long long)(rq.p.N1 + rq.p.N2);
      if (y[k].err & bd::E_NONFINITE) rq.error = BD_ERR_NONFINITE;
      if (y[k].err & bd::E_BARRIER_TIMEOUT) rq.error = BD_ERR_TIMEOUT;
      if (rq.snap_every > 0 && did > 0 && rq.done % rq.snap_every == 0) {
        RK(fetch_positions(s->e, k, rq.snap));
        rq.snap_step = rq.done;
        rq.snapshots++;
        if (!s->snapdir.empty()) {
          const double B = s->e.runs[k]->B;
          const int Ns[2] = {rq.p.N1, rq.p.N2};
          for (int sp = 0; sp < 2; sp++) {
            if (Ns[sp] == 0) continue;
            std::vector<int32_t> g(2 * (size_t)Ns[sp]);
            std::vector<double> q(2 * (size_t)Ns[sp]);
            records_to_species(rq.snap, rq.p.N1, rq.C, sp, g.data(), q.data());
            std::string path = s->snapdir + "/pos" + std::to_string(sp + 1) + "_" +
                               std::to_string(rq.id) + ".txt";
            bd::write_pos_frame(path.c_str(), rq.snapshots > 1, (double)rq.done * rq.p.dt_max, Ns[sp],
                                g.data(), q.data(), B);
          }
        }
      }
    }
    for (size_t k = 0; k < s->active.size();) {
      Request& rq = s->reqs[s->active[k]];
      if (rq.done >= rq.nsteps || rq.error) {
        RK(fetch_positions(s->e, k, rq.fin));
        RK(retire(s, k, rq.error ? BD_REQ_FAILED : BD_REQ_DONE));
        continue;
      }
      k++;
    }
  }
  s->fetch_s += s->now() - t;
  (void)changed;
  if (active) *active = (int)s->active.size();
  return BD_OK;
}

int bd_serve_result(bd_server* s, long long id, int species, int32_t* git, double* rel) {
  if (!s || species < 0 || species > 1) return BD_ERR_ARG;
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return BD_ERR_NOTFOUND;
  const Request& rq = it->second;
  if (rq.state != BD_REQ_DONE) return BD_ERR_STATE;
  records_to_species(rq.fin, rq.p.N1, rq.C, species, git, rel);
  return BD_OK;
}

int bd_serve_release(bd_server* s, long long id) {
  if (!s) return BD_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return BD_ERR_NOTFOUND;
  if (it->second.state == BD_REQ_RUNNING || it->second.state == BD_REQ_QUEUED) return BD_ERR_STATE;
  // a cancelled request may still be drawn by the server's thread
  s->cv.wait(lk, [&] { return it->second.prep != 1; });
  s->reqs.erase(it);
  return BD_OK;
}

int bd_serve_snapshot(bd_server* s, long long id, int species, long long* step, int32_t* git,
                      double* rel) {
  if (!s || species < 0 || species > 1) return BD_ERR_ARG;
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return BD_ERR_NOTFOUND;
  const Request& rq = it->second;
  if (rq.snap_step < 0) return BD_ERR_STATE;
  if (step) *step = rq.snap_step;
  records_to_species(rq.snap, rq.p.N1, rq.C, species, git, rel);
  return BD_OK;
}

int bd_serve_stats_get(bd_server* s, bd_serve_stats* st) {
  if (!s || !st) return BD_ERR_ARG;
  std::memset(st, 0, sizeof(*st));
  st->completed = s->completed;
  st->particle_steps = s->particle_steps;
  st->wall_s = s->now();
  std::vector<double> l = s->latencies;
  std::sort(l.begin(), l.end());
  auto q = [&](double f) {
    if (l.empty()) return 0.0;
    size_t i = (size_t)std::ceil(f * l.size()) - 1;
    return l[std::min(i, l.size() - 1)];
  };
  st->p50_latency_s = q(0.50);
  st->p99_latency_s = q(0.99);
  st->max_latency_s = l.empty() ? 0.0 : l.back();
  st->step_s = s->step_s;
  st->host_s = s->tick_s - s->step_s;
  st->admit_s = s->admit_s;
  st->plan_s = s->plan_s;
  st->fetch_s = s->fetch_s;
  st->active = (int)s->active.size();
  st->queued = 0;
  for (long long id : s->queue) {
    auto it = s->reqs.find(id);
    if (it != s->reqs.end() && it->second.state == BD_REQ_QUEUED) st->queued++;
  }
  st->hbm_in_use = s->used;
  return BD_OK;
}

}  // extern "C"
