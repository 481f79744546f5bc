// ausm_server_*: continuous batching of solve requests on one device.
//
// Requests wait in a FIFO until admission.  A round (pump) is:
//   1. admit queued requests in arrival order while a slot is free and the request's
//      device bytes fit the budget next to those already admitted (a request that does
//      not fit waits, and so do the ones behind it: no overtaking, so a large request
//      cannot starve);  admission creates the solver, generates its grid (multicolor
//      TTM sweeps), sets the initial state, takes the initial density-residual L2 and
//      adds it to the batch;
//   2. advance the batch by chunk_steps RK3 steps (one graph replay);
//   3. read every member's dt / wave speed and residual L2 (one synchronisation each),
//      and retire members that converged (residual_drop decades below the initial
//      norm), reached max_steps or diverged: forces and Cp are computed, the solver is
//      removed from the batch and destroyed, its bytes go back to the budget.
// With the worker running (ausm_server_start), admission is off the rounds' path: a
// second host thread, the admitter, prepares each admitted request (solver, grid,
// state, first norm) on the solver's own stream while the worker keeps stepping the
// batch on the batch stream, so their device work overlaps; the worker joins prepared
// requests to the batch at the start of its next round (the batch stream waits for the
// solver's stream).  A request holds its slot and budget from the moment it leaves the
// queue.  ausm_server_pump / drain without the worker admit on the calling thread.
// Submit and poll only touch host state under the server mutex.  Rounds are counted
// per request from its admission, so a request's dt sequence, residual checks and
// stopping step do not depend on what else is in the batch or when it joined.
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "ausm.h"
#include "solver_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Req {
  int64_t id = 0;
  AusmRequest r{};
  std::vector<double> body;  // copy of r.body_xy
  double bytes = 0.0;
  bool charged = false;   // bytes counted in the server's in_use
  bool retiring = false;  // counted in the server's retiring
  int state = AUSM_REQ_QUEUED;
  int stop = 0;
  int steps = 0;
  double l2_first = NAN, l2_last = NAN;
  double forces[6] = {NAN, NAN, NAN, NAN, NAN, NAN};
  std::vector<double> cp;
  Clock::time_point t_submit, t_admit, t_done;
  ausm_solver* h = nullptr;
  std::string err;
};

bool finite_params(const AusmParams& p) {
  const double v[] = {p.gamma, p.in_rho, p.in_pressure, p.mach, p.aoa_deg, p.K_p, p.K_u, p.cfl, p.ramp};
  for (double x : v)
    if (!std::isfinite(x)) return false;
  return !std::isnan(p.maxdt);
}

// Host-side validation of a request (no CUDA); empty string when it is acceptable.
std::string validate(const AusmRequest& r) {
  if (r.M < 4 || r.N < 2) return "grid must be at least 4 x 2 cells";
  if ((double)r.M * (r.N + 3) > 2.0e9) return "grid too large";
  if (!finite_params(r.params)) return "non-finite flow parameter";
  const AusmParams& p = r.params;
  if (!(p.gamma > 1.0 && p.in_rho > 0.0 && p.in_pressure > 0.0 && p.mach > 0.0 && p.cfl > 0.0 && p.maxdt > 0.0))
    return "need gamma > 1, in_rho > 0, in_pressure > 0, mach > 0, cfl > 0, maxdt > 0";
  if (p.ramp != 0.0) return "served requests start at full inflow speed (ramp must be 0)";
  if (p.scheme < 0 || p.scheme > 2) return "unknown scheme";
  if (p.muscl != 0 && p.muscl != 1) return "muscl must be 0 or 1";
  if (!r.body_xy && (r.naca4 < 0 || r.naca4 > 9999 || r.naca4 % 100 == 0)) return "bad NACA 4-digit code";
  if (!(std::isfinite(r.chord) && r.chord > 0.0)) return "chord must be > 0";
  if (!(std::isfinite(r.far_radius) && r.far_radius > r.chord)) return "far_radius must exceed the chord";
  if (!(std::isfinite(r.first_spacing) && r.first_spacing >= 0.0 && r.first_spacing < r.far_radius))
    return "first_spacing must be in [0, far_radius)";
  if (r.grid_iters < 0 || r.grid_iters > 1000000) return "grid_iters must be in [0, 1e6]";
  if (r.init_mode != AUSM_INIT_REST && r.init_mode != AUSM_INIT_FREESTREAM) return "unknown init mode";
  if (!(std::isfinite(r.residual_drop) && r.residual_drop >= 0.0)) return "residual_drop must be >= 0";
  if (r.max_steps < 1) return "max_steps must be >= 1";
  if (r.body_xy)
    for (int k = 0; k < 2 * r.M; k++)
      if (!std::isfinite(r.body_xy[k])) return "non-finite body vertex";
  return "";
}

// Device bytes of a fused-engine solver driven by the server: FP32 and FP64 vertices
// (8 + 16 per vertex), the two face-record arrays (16 per face), three state buffers
// (48 per cell), the Cp array, and a fixed 64 KiB for the per-solver scalars and the
// reduction scratch (2 x 2368 doubles), allocation rounding included.
double request_bytes(const AusmRequest& r) {
  const double M = r.M, N = r.N;
  return 40.0 * M * (N + 1) + 16.0 * M * N + 48.0 * M * N + 8.0 * M + 65536.0;
}

}  // namespace

struct ausm_server {
  double budget = 0.0;
  int max_active = 1, chunk = 100, flags = 0;
  int dev = -1;
  std::mutex mu;       // everything below except the CUDA objects
  std::mutex pump_mu;  // one round at a time
  std::condition_variable cv;
  std::deque<Req*> queue;
  std::vector<Req*> active;  // in batch member order
  std::deque<Req*> to_prepare;  // left the queue, waiting for the admitter
  std::deque<Req*> ready;       // prepared by the admitter, joining at the next round
  int preparing = 0;            // to_prepare + the one the admitter is working on
  bool async_admit = false;     // the admitter thread is running
  int retiring = 0;          // finished members whose forces / teardown are in progress
  int admitting = 0;         // requests taken off the queue whose admission is in progress
  std::unordered_map<int64_t, std::unique_ptr<Req>> reqs;
  int64_t next_id = 1;
  double in_use = 0.0, peak = 0.0, cell_updates = 0.0;
  int64_t submitted = 0, rejected = 0, admitted = 0, finished = 0, failed = 0, rounds = 0;
  ausm_batch* batch = nullptr;
  std::thread worker, admitter;
  std::condition_variable admit_cv;
  bool running = false, stopping = false;
  std::string err;
};

namespace {

int sfail(ausm_server* s, int code, const std::string& msg) {
  ausm::set_thread_error(msg);
  if (s) {
    std::lock_guard<std::mutex> lk(s->mu);
    s->err = msg;
  }
  return code;
}

// Ends a request (caller holds no lock); frees its solver.
void finish(ausm_server* s, Req* q, int state, int stop) {
  if (q->h) {
    if (q->h->batch) ausm_batch_remove(q->h->batch, q->h);
    ausm_destroy(q->h);
    q->h = nullptr;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (q->state == AUSM_REQ_QUEUED && q->charged) s->admitting--;  // its admission failed
  q->state = state;
  q->stop = stop;
  q->t_done = Clock::now();
  if (q->charged) s->in_use -= q->bytes;
  q->charged = false;
  if (q->retiring) {
    q->retiring = false;
    s->retiring--;
  }
  if (state == AUSM_REQ_DONE) s->finished++;
  else s->failed++;
}

// Creates the solver of q, its grid and state (on the solver's own stream); on failure
// the request ends with the library's status.
bool prepare(ausm_server* s, Req* q) {
  const AusmRequest& r = q->r;
  ausm_solver* h = nullptr;
  int rc = ausm_create(r.M, r.N, &h);
  auto fail_req = [&](int code) {
    q->err = h ? ausm_last_error(h) : ausm_last_error(nullptr);
    q->h = h;
    finish(s, q, code, 0);
    return false;
  };
  if (rc) return fail_req(rc);
  q->h = h;
  if ((rc = ausm_set_params(h, &r.params))) return fail_req(rc);
  if (q->body.empty())
    rc = ausm_set_body_naca4(h, r.naca4, 0.5 * r.chord, 0.0, r.closed_te);
  else
    rc = ausm_set_body_points(h, q->body.data(), r.M);
  if (rc) return fail_req(rc);
  if ((rc = ausm_set_outer(h, AUSM_OUTER_CIRCLE, r.far_radius, 0.0, 0.0))) return fail_req(rc);
  if (r.first_spacing > 0.0 && (rc = ausm_set_radial_stretch(h, r.first_spacing))) return fail_req(rc);
  if ((rc = ausm_generate_grid(h, r.grid_iters, AUSM_GRID_MULTICOLOR, 0.0, nullptr))) return fail_req(rc);
  if ((rc = ausm_init_state(h, r.init_mode))) return fail_req(rc);
  double l2 = NAN;
  if ((rc = ausm_residual_l2(h, &l2))) return fail_req(rc);
  q->cp.assign(r.M, NAN);
  q->l2_first = q->l2_last = l2;
  return true;
}

// Adds a prepared request to the batch (worker thread); it is active from now on.
bool join(ausm_server* s, Req* q) {
  int rc;
  if (!(s->flags & AUSM_SERVE_PLAIN) && (rc = ausm_batch_add(s->batch, q->h))) {
    q->err = ausm_batch_last_error(s->batch);
    finish(s, q, rc, 0);
    return false;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  q->state = AUSM_REQ_RUNNING;
  q->t_admit = Clock::now();
  s->admitted++;
  s->admitting--;
  s->active.push_back(q);
  return true;
}

bool admit(ausm_server* s, Req* q) { return prepare(s, q) && join(s, q); }

// The admitter thread: prepares requests the worker took off the queue.
void admitter_loop(ausm_server* s) {
  cudaSetDevice(s->dev);
  for (;;) {
    Req* q = nullptr;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->admit_cv.wait(lk, [&] { return s->stopping || !s->to_prepare.empty(); });
      if (s->stopping) return;
      q = s->to_prepare.front();
      s->to_prepare.pop_front();
    }
    const bool ok = prepare(s, q);
    std::lock_guard<std::mutex> lk(s->mu);
    s->preparing--;
    if (ok) s->ready.push_back(q);
    s->cv.notify_all();
  }
}

// Stop decision of one member after a round.
int classify(const Req* q, float wave, double l2) {
  if (!std::isfinite(wave) || !std::isfinite(l2)) return AUSM_STOP_DIVERGED;
  if (q->r.residual_drop > 0.0 && q->l2_first > 0.0 && l2 <= q->l2_first * std::pow(10.0, -q->r.residual_drop))
    return AUSM_STOP_CONVERGED;
  if (q->steps >= q->r.max_steps) return AUSM_STOP_MAX_STEPS;
  return 0;
}

void retire(ausm_server* s, Req* q, int stop) {
  int state = AUSM_REQ_DONE;
  if (stop == AUSM_STOP_DIVERGED) {
    state = AUSM_ERR_DIVERGED;
    q->err = "the solution diverged (non-finite wave speed or residual)";
  } else {
    int rc = ausm_forces(q->h, q->forces, q->cp.data());
    if (rc) {
      state = rc;
      q->err = ausm_last_error(q->h);
    }
  }
  finish(s, q, state, stop);
}

// A failed round: its batch members end with the round's status (a timed-out tile, a
// CUDA error); queued requests stay queued (a broken device fails them at their own
// admission).  Returns the status, as the round does.
int fail_round(ausm_server* s, const std::vector<Req*>& act, int rc, const std::string& why) {
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (Req* q : act)
      for (size_t k = 0; k < s->active.size(); k++)
        if (s->active[k] == q) {
          s->active.erase(s->active.begin() + k);
          break;
        }
  }
  for (Req* q : act) {
    q->err = why;
    finish(s, q, rc, 0);
  }
  return sfail(s, rc, why);
}

int pump_round(ausm_server* s, int* remaining) {
  std::lock_guard<std::mutex> pl(s->pump_mu);
  if (s->dev < 0) {
    int rc = cudaGetDevice(&s->dev) == cudaSuccess ? AUSM_OK : AUSM_ERR_CUDA;
    if (rc) {
      s->dev = -1;
      return sfail(s, rc, "no CUDA device");
    }
  } else {
    cudaSetDevice(s->dev);
  }
  if (!(s->flags & AUSM_SERVE_PLAIN) && !s->batch) {
    int rc = ausm_batch_create(&s->batch);
    if (rc) return sfail(s, rc, ausm_batch_last_error(nullptr));
    if (s->flags & AUSM_SERVE_NO_GRAPH) ausm_batch_set_graphs(s->batch, 0);
  }
  // 1. requests the admitter has prepared join the batch; then admission, in arrival
  // order, on this thread or handed to the admitter
  for (;;) {
    Req* q = nullptr;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      if (s->ready.empty()) break;
      q = s->ready.front();
      s->ready.pop_front();
    }
    join(s, q);
  }
  for (;;) {
    Req* q = nullptr;
    bool async;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      async = s->async_admit && !(s->flags & AUSM_SERVE_PLAIN);
      const int slots = (s->flags & AUSM_SERVE_PLAIN) ? 1 : s->max_active;
      const int held = (int)(s->active.size() + s->ready.size()) + s->preparing;
      if (s->queue.empty() || held >= slots) break;
      Req* f = s->queue.front();
      if (s->in_use + f->bytes > s->budget) break;
      s->queue.pop_front();
      s->in_use += f->bytes;
      f->charged = true;
      s->admitting++;  // neither queued nor active until it joins the batch
      if (s->in_use > s->peak) s->peak = s->in_use;
      q = f;
      if (async) {
        s->preparing++;
        s->to_prepare.push_back(q);
        s->admit_cv.notify_one();
      }
    }
    if (!async) admit(s, q);
  }
  std::vector<Req*> act;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    act = s->active;
  }
  if (!act.empty()) {
    // 2-3. one round of every active solve, then the stop checks
    const int n = (int)act.size();
    std::vector<float> dtw(2 * (size_t)n, NAN);
    std::vector<double> l2(n, NAN);
    if (s->flags & AUSM_SERVE_PLAIN) {
      for (int k = 0; k < n; k++) {
        float dt = NAN;
        int rc = ausm_step(act[k]->h, s->chunk, &dt);
        if (rc == AUSM_OK) {
          ausm_max_wave_speed(act[k]->h, &dtw[2 * k + 1]);
          rc = ausm_residual_l2(act[k]->h, &l2[k]);
          if (rc == AUSM_ERR_DIVERGED) l2[k] = NAN;
        }
        dtw[2 * k] = dt;
      }
    } else {
      int rc = ausm_batch_step(s->batch, s->chunk, dtw.data());
      if (rc != AUSM_OK && rc != AUSM_ERR_DIVERGED) return fail_round(s, act, rc, ausm_batch_last_error(s->batch));
      rc = ausm_batch_residual_l2(s->batch, l2.data());
      if (rc != AUSM_OK) return fail_round(s, act, rc, ausm_batch_last_error(s->batch));
    }
    std::vector<std::pair<Req*, int>> done;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->rounds++;
      for (int k = 0; k < n; k++) {
        Req* q = act[k];
        q->steps += s->chunk;
        q->l2_last = l2[k];
        s->cell_updates += (double)q->r.M * q->r.N * s->chunk;
        int stop = classify(q, dtw[2 * k + 1], l2[k]);
        if (stop) done.emplace_back(q, stop);
      }
      for (auto& d : done) {
        d.first->retiring = true;
        s->retiring++;
        for (size_t k = 0; k < s->active.size(); k++)
          if (s->active[k] == d.first) {
            s->active.erase(s->active.begin() + k);
            break;
          }
      }
    }
    for (auto& d : done) retire(s, d.first, d.second);
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (remaining) *remaining = (int)(s->queue.size() + s->active.size()) + s->retiring + s->admitting;
  s->cv.notify_all();
  return AUSM_OK;
}

void worker_loop(ausm_server* s) {
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(s->mu);
      // work: a batch to step, prepared requests to join, or queued requests a slot and
      // the budget admit (otherwise wait for a retirement, a preparation or a submit)
      auto work = [&] {
        if (s->stopping || !s->active.empty() || !s->ready.empty()) return true;
        if (s->queue.empty()) return false;
        const int slots = (s->flags & AUSM_SERVE_PLAIN) ? 1 : s->max_active;
        return (int)s->ready.size() + s->preparing < slots && s->in_use + s->queue.front()->bytes <= s->budget;
      };
      s->cv.wait(lk, work);
      if (s->stopping) return;
    }
    int left = 0;
    if (pump_round(s, &left) != AUSM_OK) {  // the round's members were ended by fail_round
      std::lock_guard<std::mutex> lk(s->mu);
      s->cv.notify_all();
    }
  }
}

}  // namespace

extern "C" {

int ausm_request_bytes(const AusmRequest* r, double* bytes) {
  if (!r || !bytes) return sfail(nullptr, AUSM_ERR_INVALID, "null argument");
  if (r->M < 1 || r->N < 1) return sfail(nullptr, AUSM_ERR_INVALID, "grid must be at least 1 x 1");
  *bytes = request_bytes(*r);
  return AUSM_OK;
}

int ausm_server_create(double hbm_budget_bytes, int max_active, int chunk_steps, int flags, ausm_server** out) {
  if (!out) return sfail(nullptr, AUSM_ERR_INVALID, "null output handle");
  *out = nullptr;
  if (!(hbm_budget_bytes > 0.0) || max_active < 1 || chunk_steps < 1 || (flags & ~3))
    return sfail(nullptr, AUSM_ERR_INVALID, "need budget > 0, max_active >= 1, chunk_steps >= 1, known flags");
  ausm_server* s = new ausm_server();
  s->budget = hbm_budget_bytes;
  s->max_active = max_active;
  s->chunk = chunk_steps;
  s->flags = flags;
  *out = s;
  return AUSM_OK;
}

int ausm_server_stop(ausm_server* s) {
  if (!s) return sfail(nullptr, AUSM_ERR_INVALID, "null handle");
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (!s->running) return AUSM_OK;
    s->stopping = true;
    s->cv.notify_all();
    s->admit_cv.notify_all();
  }
  s->worker.join();
  if (s->admitter.joinable()) s->admitter.join();
  std::lock_guard<std::mutex> lk(s->mu);
  s->running = false;
  s->stopping = false;
  s->async_admit = false;
  // requests handed to the admitter but not prepared go back to the front of the queue
  while (!s->to_prepare.empty()) {
    Req* q = s->to_prepare.back();
    s->to_prepare.pop_back();
    s->preparing--;
    s->admitting--;
    s->in_use -= q->bytes;
    q->charged = false;
    s->queue.push_front(q);
  }
  return AUSM_OK;
}

int ausm_server_destroy(ausm_server* s) {
  if (!s) return AUSM_OK;
  ausm_server_stop(s);
  if (s->dev >= 0) cudaSetDevice(s->dev);
  std::vector<Req*> held(s->active.begin(), s->active.end());
  held.insert(held.end(), s->ready.begin(), s->ready.end());
  for (Req* q : held)
    if (q->h) {
      if (q->h->batch) ausm_batch_remove(q->h->batch, q->h);
      ausm_destroy(q->h);
      q->h = nullptr;
    }
  if (s->batch) ausm_batch_destroy(s->batch);
  delete s;
  return AUSM_OK;
}

const char* ausm_server_last_error(const ausm_server* s) { return s ? s->err.c_str() : ausm_last_error(nullptr); }

int ausm_server_submit(ausm_server* s, const AusmRequest* r, int64_t* id) {
  if (!s || !r || !id) return sfail(s, AUSM_ERR_INVALID, "null argument");
  std::string why = validate(*r);
  if (!why.empty()) {
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->rejected++;
    }
    return sfail(s, AUSM_ERR_INVALID, "request rejected: " + why);
  }
  const double bytes = request_bytes(*r);
  if (bytes > s->budget) {
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->rejected++;
    }
    return sfail(s, AUSM_ERR_BUDGET, "request rejected: needs " + std::to_string(bytes) +
                                         " device bytes, above the whole budget of " + std::to_string(s->budget));
  }
  auto q = std::make_unique<Req>();
  q->r = *r;
  if (r->body_xy) q->body.assign(r->body_xy, r->body_xy + 2 * (size_t)r->M);
  q->r.body_xy = nullptr;
  q->bytes = bytes;
  q->t_submit = Clock::now();
  std::lock_guard<std::mutex> lk(s->mu);
  q->id = s->next_id++;
  *id = q->id;
  s->queue.push_back(q.get());
  s->reqs.emplace(q->id, std::move(q));
  s->submitted++;
  s->cv.notify_all();
  return AUSM_OK;
}

int ausm_server_pump(ausm_server* s, int* remaining) {
  if (!s) return sfail(nullptr, AUSM_ERR_INVALID, "null handle");
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->running) return sfail(nullptr, AUSM_ERR_STATE, "the worker thread is pumping this server");
  }
  return pump_round(s, remaining);
}

int ausm_server_start(ausm_server* s) {
  if (!s) return sfail(nullptr, AUSM_ERR_INVALID, "null handle");
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->running) return AUSM_OK;
  if (s->dev < 0 && cudaGetDevice(&s->dev) != cudaSuccess) {
    s->dev = -1;
    return sfail(nullptr, AUSM_ERR_CUDA, "no CUDA device");
  }
  s->running = true;
  s->async_admit = !(s->flags & AUSM_SERVE_PLAIN);
  s->worker = std::thread([s] {
    cudaSetDevice(s->dev);
    worker_loop(s);
  });
  if (s->async_admit) s->admitter = std::thread([s] { admitter_loop(s); });
  return AUSM_OK;
}

int ausm_server_poll(ausm_server* s, int64_t id, AusmResult* res, double* cp) {
  if (!s || !res) return sfail(nullptr, AUSM_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return sfail(nullptr, AUSM_ERR_NOT_FOUND, "unknown request id " + std::to_string(id));
  const Req* q = it->second.get();
  std::memset(res, 0, sizeof *res);
  res->id = q->id;
  res->state = q->state;
  res->stop = q->stop;
  res->M = q->r.M;
  res->N = q->r.N;
  res->steps = q->steps;
  res->l2_first = q->l2_first;
  res->l2_last = q->l2_last;
  const bool done = q->state != AUSM_REQ_QUEUED && q->state != AUSM_REQ_RUNNING;
  for (int k = 0; k < 6; k++) res->forces[k] = done ? q->forces[k] : NAN;
  const bool admitted = q->t_admit != Clock::time_point{};
  res->queue_ms = admitted ? ms_between(q->t_submit, q->t_admit) : NAN;
  res->run_ms = admitted && done ? ms_between(q->t_admit, q->t_done) : NAN;
  res->latency_ms = done ? ms_between(q->t_submit, q->t_done) : NAN;
  if (cp && done && q->state == AUSM_REQ_DONE) std::memcpy(cp, q->cp.data(), q->cp.size() * sizeof(double));
  if (done && !q->err.empty()) ausm::set_thread_error(q->err);  // why it failed, for ausm_last_error(NULL)
  return AUSM_OK;
}

int ausm_server_drain(ausm_server* s, double timeout_ms) {
  if (!s) return sfail(nullptr, AUSM_ERR_INVALID, "null handle");
  const auto t_end = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                        std::chrono::duration<double, std::milli>(timeout_ms < 0 ? 0.0 : timeout_ms));
  bool worker;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    worker = s->running;
  }
  if (worker) {
    std::unique_lock<std::mutex> lk(s->mu);
    auto idle = [&] { return s->queue.empty() && s->active.empty() && s->retiring == 0 && s->admitting == 0; };
    if (timeout_ms < 0) s->cv.wait(lk, idle);
    else if (!s->cv.wait_until(lk, t_end, idle)) return AUSM_ERR_TIMEOUT;
    return AUSM_OK;
  }
  for (;;) {
    int left = 0;
    int rc = pump_round(s, &left);
    if (rc) return rc;
    if (left == 0) return AUSM_OK;
    if (timeout_ms >= 0 && Clock::now() >= t_end) return sfail(s, AUSM_ERR_TIMEOUT, "drain timed out");
  }
}

int ausm_server_stats(ausm_server* s, AusmServerStats* st) {
  if (!s || !st) return sfail(nullptr, AUSM_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  st->submitted = s->submitted;
  st->rejected = s->rejected;
  st->admitted = s->admitted;
  st->finished = s->finished;
  st->failed = s->failed;
  st->rounds = s->rounds;
  st->pending = (int)s->queue.size();
  st->active = (int)s->active.size();
  st->bytes_in_use = s->in_use;
  st->peak_bytes = s->peak;
  st->cell_updates = s->cell_updates;
  return AUSM_OK;
}

}  // extern "C"
