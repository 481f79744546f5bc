// C ABI of libausm (include/ausm.h): solver handles, host geometry input, and the
// orchestration of the device kernels for the reference's operator surface.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "ausm.h"
#include "ausm_internal.h"
#include "solver_internal.h"

using namespace ausm;

static thread_local std::string g_err;

namespace ausm {
// error text for ausm_last_error(NULL) from entry points defined in other files
void set_thread_error(const std::string& msg) { g_err = msg; }

// Uniform values as the reference builds them (main.js:779-784, util.js:180-185), in
// double, rounded to f32; derived constants in f32 in the shaders' operation order.
void make_consts(ausm_solver* h) {
  const AusmParams& p = h->p;
  Consts c{};
  const float g = (float)p.gamma, inRho = (float)p.in_rho, inP = (float)p.in_pressure;
  double a = p.aoa_deg * M_PI / 180.0;
  double u = h->speed_now * std::cos(a), v = h->speed_now * std::sin(a);
  c.gamma = g; c.inRho = inRho; c.inP = inP;
  c.gm1 = g - 1.0f;
  c.gm1inv = 1.0f / (g - 1.0f);
  c.Kp = (float)p.K_p; c.Ku = (float)p.K_u; c.cfl = (float)p.cfl; c.maxdt = (float)p.maxdt;
  c.inflow = make_float2((float)u, (float)v);
  double rhoE = p.in_pressure / (p.gamma - 1.0) + 0.5 * (h->speed_now * h->speed_now) * p.in_rho;
  c.inState = make_float4(inRho, (float)(u * p.in_rho), (float)(v * p.in_rho), (float)rhoE);
  c.a2inf = (g * inP) / inRho;
  c.Vinf2 = c.inflow.x * c.inflow.x + c.inflow.y * c.inflow.y;
  c.Minf2 = c.Vinf2 / c.a2inf;
  c.gammaInP = g * inP;
  c.aStarK = (2.0f * c.gm1) / (g + 1.0f);
  c.ambE = inP / (g - 1.0f);
  c.h2k = (2.0f * g) / c.gm1;
  c.ask4 = 0.25f * c.aStarK;
  c.minfk = c.Vinf2 / c.gammaInP;
  c.hsg = 0.5f * std::sqrt(g);
  c.muscl = p.muscl;
  h->c = c;
  // FP64 constants from the FP64 parameters, in the oracle's operation order
  ex::ConstsR<double> d{};
  d.gamma = p.gamma; d.inRho = p.in_rho; d.inP = p.in_pressure;
  d.gm1 = p.gamma - 1.0;
  d.gm1inv = 1.0 / (p.gamma - 1.0);
  d.Kp = p.K_p; d.Ku = p.K_u; d.cfl = p.cfl; d.maxdt = p.maxdt;
  d.inflow = {u, v};
  d.inState = {p.in_rho, u * p.in_rho, v * p.in_rho, rhoE};
  d.a2inf = (p.gamma * p.in_pressure) / p.in_rho;
  d.Vinf2 = u * u + v * v;
  d.Minf2 = d.Vinf2 / d.a2inf;
  d.gammaInP = p.gamma * p.in_pressure;
  d.aStarK = (2.0 * d.gm1) / (p.gamma + 1.0);
  d.ambE = p.in_pressure / (p.gamma - 1.0);
  d.muscl = p.muscl;
  h->cd = d;
  if (h->f64) h->f64->c = d;
}

void ramp_after_steps(ausm_solver* h, int n) {
  if (h->p.ramp > 0.0 && n > 0) {
    double target = h->p.mach * std::sqrt(h->p.gamma * h->p.in_pressure / h->p.in_rho);
    h->speed_now += (target - h->speed_now) / (h->p.ramp / n * 50.0);
    make_consts(h);
  }
}

// ---- tile-height autotuner ----
// The TMA stage kernel exists for tile heights 8, 16 and 32 (32 x 4, 32 x 8 and 32 x 16
// threads; 8, 4 and 2 CTAs per SM).  Which is fastest depends on the grid (partial
// tiles at the edges, halo overhead, occupancy) and the scheme, so it is measured: a
// few stage-1 launches per candidate on the solve's own data, timed with CUDA events on
// its stream.  Stage 1 reads the current state and writes the next buffer, which is
// scratch until the next step's stage 1 overwrites it, so tuning has no effect on the
// solution.  Results are cached per (M, N, scheme) for the process.
namespace {
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int>, int> g_tune_cache;
}  // namespace

int tuned_tile_rows(ausm_solver* h, bool force, int* rows) {
  *rows = 16;
  if (!h->tma[1].ok) return AUSM_OK;  // per-thread kernels: 16 rows
  if (const char* e = std::getenv("AUSM_TILE_ROWS")) {
    const int r = std::atoi(e);
    if ((r == 8 || r == 16 || r == 32) && h->tma[tile_index(r)].ok) {
      *rows = r;
      return AUSM_OK;
    }
  }
  if (const char* e = std::getenv("AUSM_AUTOTUNE"))
    if (e[0] == '0') return AUSM_OK;
  if (!force && h->tile_rows) {
    *rows = h->tile_rows;
    return AUSM_OK;
  }
  const auto key = std::make_tuple(h->M, h->N, h->p.scheme);
  if (!force) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      *rows = h->tile_rows = it->second;
      return AUSM_OK;
    }
  }
  const int a = h->cur, b = (a + 1) % 3;
  const double cells = (double)h->M * h->N;
  // about 2 ms of launches per candidate and round; two rounds, each candidate's best
  // time counts (clock ramp-up and co-running work only ever make a run slower)
  const int reps = (int)std::max(5.0, std::min(100.0, 1.0e8 / std::max(cells, 1.0)));
  float best_ms[3] = {INFINITY, INFINITY, INFINITY};
  for (int round = 0; round < 2; round++)
    for (int k = 0; k < 3; k++) {
      const TmaMaps& tm = h->tma[k];
      if (!tm.ok) continue;
      const TmaMapsLaunch t = {tm.halo[a], tm.plain[a], tm.mi, tm.mj, tm.wrap[a]};
      auto launch = [&] {
        launch_fused_stage(h->p.scheme, 1, false, h->Q[a], nullptr, h->Q[b], h->Mi, h->Mj, h->dt, h->wave, 0, h->c,
                           h->M, h->N, &t, kTileHeights[k], h->err_flag, h->st);
      };
      launch();  // warm-up (first-launch attribute set-up, caches)
      cudaEventRecord(h->e0, h->st);
      for (int r = 0; r < reps; r++) launch();
      cudaEventRecord(h->e1, h->st);
      cudaError_t e = cudaEventSynchronize(h->e1);
      if (e == cudaSuccess) e = cudaGetLastError();
      if (e != cudaSuccess) {
        set_thread_error(std::string("tile autotuning: ") + cudaGetErrorString(e));
        h->err = std::string("tile autotuning: ") + cudaGetErrorString(e);
        return AUSM_ERR_CUDA;
      }
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, h->e0, h->e1);
      best_ms[k] = std::min(best_ms[k], ms);
    }
  int best_rows = 16;
  float best = INFINITY;
  for (int k = 0; k < 3; k++)
    if (best_ms[k] < best) {
      best = best_ms[k];
      best_rows = kTileHeights[k];
    }
  *rows = h->tile_rows = best_rows;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_cache[key] = best_rows;
  return AUSM_OK;
}

}  // namespace ausm


namespace {

int fail(ausm_solver* h, int code, const std::string& msg) {
  g_err = msg;
  if (h) h->err = msg;
  return code;
}
#define CU(h, call)                                                                   \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return fail(h, e_ == cudaErrorMemoryAllocation ? AUSM_ERR_OOM : AUSM_ERR_CUDA,  \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                \
  } while (0)
#define CHECK_LAUNCH(h) CU(h, cudaGetLastError())
#define NEED(h, cond, code, msg) \
  do {                           \
    if (!(cond)) return fail(h, code, msg); \
  } while (0)

template <class T> cudaError_t dalloc(T** p, size_t n) { return cudaMalloc((void**)p, n * sizeof(T)); }

int use_device(ausm_solver* h) {
  int d = -1;
  CU(h, cudaGetDevice(&d));
  if (d != h->dev) CU(h, cudaSetDevice(h->dev));
  return AUSM_OK;
}

double inflow_target(const AusmParams& p) { return p.mach * std::sqrt(p.gamma * p.in_pressure / p.in_rho); }

// Timeout reporting.  A TMA stage kernel whose bounded wait gave up sets *err_flag
// (device).  Every fused step queues a copy of the flag to pinned host memory; the next
// call that waits for the stream (this step when it returns dt, or a later state,
// force, norm, field, wave-speed, synchronize or timing call) reads it, clears the flag
// and returns AUSM_ERR_TIMEOUT, so no path steps past a timed-out tile unreported.
int queue_err_read(ausm_solver* h) {
  CU(h, cudaMemcpyAsync(h->h_wave + 2, h->err_flag, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  h->err_read_queued = true;
  return AUSM_OK;
}
// After the stream has been synchronised.
int take_timeout(ausm_solver* h) {
  if (!h->err_read_queued) return AUSM_OK;
  h->err_read_queued = false;
  if (h->h_wave[2] == 0) return AUSM_OK;
  h->h_wave[2] = 0;
  CU(h, cudaMemsetAsync(h->err_flag, 0, sizeof(int), h->st));
  return fail(h, AUSM_ERR_TIMEOUT, "a tile load did not arrive within the bounded wait");
}
// Synchronises h's stream and reports a queued timeout.
int sync_and_check(ausm_solver* h) {
  CU(h, cudaStreamSynchronize(h->st));
  return take_timeout(h);
}

int ensure_reference_buffers(ausm_solver* h) {
  if (h->S[0]) return AUSM_OK;
  size_t nref = (size_t)h->M * (h->N + 3), n = (size_t)h->M * h->N;
  for (auto& s : h->S) CU(h, dalloc(&s, nref));
  CU(h, dalloc(&h->fx, n));
  CU(h, dalloc(&h->fy, (size_t)h->M * (h->N + 1)));
  CU(h, dalloc(&h->res, n));
  CU(h, dalloc(&h->flen, n));
  CU(h, dalloc(&h->area, n));
  return AUSM_OK;
}
// staging: a float reference-layout state (M x (N+3) float4) followed by room for one
// M x N float field
int ensure_staging(ausm_solver* h) {
  if (!h->staging) CU(h, dalloc(&h->staging, (size_t)h->M * (h->N + 3) + ((size_t)h->M * h->N + 3) / 4));
  return AUSM_OK;
}

// current interior state (fused: Q[cur]; reference: rows 1..N of S[2])
const float4* interior(ausm_solver* h) {
  return h->engine == AUSM_ENGINE_FUSED ? h->Q[h->cur] : h->S[2] + h->M;
}

// The current state in the float reference layout, in staging.
int state_to_staging(ausm_solver* h) {
  int rc = ensure_staging(h);
  if (rc) return rc;
  if (h->engine == AUSM_ENGINE_FUSED)
    launch_to_ref_layout(h->Q[h->cur], h->staging, h->V, h->c, h->M, h->N, h->st);
  else if (h->engine == AUSM_ENGINE_REFERENCE)
    launch_ref_boundary(h->S[2], h->staging, h->V, h->c, h->M, h->N, h->st);
  else
    h->f64->to_f32(h->staging, h->Vd, h->st);
  CHECK_LAUNCH(h);
  return AUSM_OK;
}
// A float reference-layout state in staging becomes the current engine's state.
int staging_to_state(ausm_solver* h) {
  if (h->engine == AUSM_ENGINE_FUSED) {
    h->cur = 0;
    launch_from_ref_layout(h->staging, h->Q[0], h->M, h->N, h->st);
  } else if (h->engine == AUSM_ENGINE_REFERENCE) {
    CU(h, cudaMemcpyAsync(h->S[2], h->staging, (size_t)h->M * (h->N + 3) * sizeof(float4), cudaMemcpyDeviceToDevice,
                          h->st));
  } else {
    h->f64->from_f32(h->staging, h->st);
  }
  CHECK_LAUNCH(h);
  return AUSM_OK;
}
int ensure_f64(ausm_solver* h) {
  if (h->f64) return AUSM_OK;
  h->f64 = new F64Engine();
  cudaError_t e = h->f64->allocate(h->M, h->N);
  if (e != cudaSuccess) {
    delete h->f64;
    h->f64 = nullptr;
    return fail(h, e == cudaErrorMemoryAllocation ? AUSM_ERR_OOM : AUSM_ERR_CUDA,
                std::string("FP64 engine buffers: ") + cudaGetErrorString(e));
  }
  h->f64->c = h->cd;
  if (h->has_grid) h->f64->metrics(h->Vd, h->st);
  CHECK_LAUNCH(h);
  return AUSM_OK;
}

int refresh_wave(ausm_solver* h) {
  if (h->engine == AUSM_ENGINE_F64) {
    h->f64->wave_speed(h->st);
    CHECK_LAUNCH(h);
    return AUSM_OK;
  }
  CU(h, cudaMemsetAsync(h->wave, 0, sizeof(uint32_t), h->st));
  if (h->engine == AUSM_ENGINE_FUSED) {
    launch_wave_interior(h->Q[h->cur], h->Mj, h->c.gamma, h->M, h->N, h->wave, h->st);
  } else {
    launch_ref_wave(h->S[2], h->flen, h->area, h->c.gamma, h->M, h->N, h->wave, h->st);
  }
  CHECK_LAUNCH(h);
  return AUSM_OK;
}

int after_grid(ausm_solver* h) {
  launch_metrics_d(h->Vd, h->Mi, h->Mj, h->M, h->N, h->st);
  if (h->f64) h->f64->metrics(h->Vd, h->st);
  CHECK_LAUNCH(h);
  if (h->engine == AUSM_ENGINE_REFERENCE) {
    launch_ref_metrics(h->V, h->area, h->flen, h->M, h->N, h->st);
    CHECK_LAUNCH(h);
  }
  h->has_grid = true;
  if (h->has_state) return refresh_wave(h);
  return AUSM_OK;
}

// NACA 4-digit boundary vertex (grid.js:38-52), t = vertex index.
void naca4_point(int t_idx, int M, int naca4, double size, double xoff, double te, double& x, double& y) {
  const double exponent = 7.0 / 5.0;
  double t = t_idx / (M / 2.0);
  size *= 2;
  double thickness = naca4 % 100 / 100.0;
  double m = std::floor(naca4 / 1000.0) / 100.0;
  double p = (double)((int)std::floor(naca4 / 100.0) % 10) / 10.0;
  auto thick = [&](double s) {
    return 5 * thickness * (0.2969 * std::sqrt(s) - 0.126 * s - 0.3516 * s * s + 0.2843 * s * s * s + te * s * s * s * s);
  };
  auto camber = [&](double s) {
    return s < p ? (m / (p * p)) * (2 * p * s - s * s) : (m / ((1 - p) * (1 - p))) * ((1 - 2 * p) + 2 * p * s - s * s);
  };
  auto dcamber = [&](double s) { return (s < p ? (m / (p * p)) : (m / ((1 - p) * (1 - p)))) * (2 * p - 2 * s); };
  auto sym = [&](double s, double& sx, double& sy) {
    double d = dcamber(s);
    sx = thick(s) * -std::sin(std::atan(d));
    sy = thick(s) / std::sqrt(1 + d * d);
  };
  double s, sx, sy;
  if (t <= 1) {
    s = std::pow(1 - t, exponent);
    sym(s, sx, sy);
    x = (s - 0.5 + sx) * size + xoff;
    y = (camber(s) + sy) * size;
  } else {
    s = std::pow(t - 1, exponent);
    sym(s, sx, sy);
    x = (s - 0.5 - sx) * size + xoff;
    y = (camber(s) - sy) * size;
  }
}

}  // namespace

extern "C" {

int ausm_default_params(AusmParams* p) {
  if (!p) return fail(nullptr, AUSM_ERR_INVALID, "null params");
  p->gamma = 1.4;
  p->in_rho = 1.0;
  p->in_pressure = 1.0 / 1.4;
  p->mach = 3.8;  // inflowVel 3.8 with a_inf = 1 (util.js:87, 92-94)
  p->aoa_deg = 0.0;
  p->K_p = 0.0;
  p->K_u = 0.75;
  p->cfl = 1.5;
  p->maxdt = 1e-4;
  p->muscl = 1;
  p->scheme = AUSM_SLAU2;
  p->ramp = 0.0;
  return AUSM_OK;
}

const char* ausm_last_error(const ausm_solver* h) { return h ? h->err.c_str() : g_err.c_str(); }

int ausm_set_device(int device) {
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(nullptr, AUSM_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  return AUSM_OK;
}

int ausm_device_count(int* count) {
  if (!count) return fail(nullptr, AUSM_ERR_INVALID, "null output");
  cudaError_t e = cudaGetDeviceCount(count);
  if (e != cudaSuccess) {
    *count = 0;
    return fail(nullptr, AUSM_ERR_CUDA, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
  }
  return AUSM_OK;
}

int ausm_destroy(ausm_solver* h) {
  if (!h) return AUSM_OK;
  if (h->batch) ausm_batch_remove(h->batch, h);
  cudaSetDevice(h->dev);
  if (h->st) cudaStreamSynchronize(h->st);
  void* dptrs[] = {h->V, h->V2, h->Vd, h->Mi, h->Mj, h->Q[0], h->Q[1], h->Q[2], h->S[0], h->S[1], h->S[2], h->fx, h->fy, h->res,
                   h->flen, h->area, h->staging, h->cp, h->wave, h->dt, h->dacc, h->parts, h->move, h->err_flag};
  for (void* d : dptrs)
    if (d) cudaFree(d);
  delete h->f64;
  if (h->h_dt) cudaFreeHost(h->h_dt);
  if (h->h_wave) cudaFreeHost(h->h_wave);
  if (h->h_acc) cudaFreeHost(h->h_acc);
  if (h->e0) cudaEventDestroy(h->e0);
  if (h->e1) cudaEventDestroy(h->e1);
  if (h->own_st) cudaStreamDestroy(h->own_st);
  delete h;
  return AUSM_OK;
}

int ausm_create(int M, int N, ausm_solver** out) {
  if (!out) return fail(nullptr, AUSM_ERR_INVALID, "null output handle");
  *out = nullptr;
  if (M < 4 || N < 2) return fail(nullptr, AUSM_ERR_INVALID, "grid must be at least 4 x 2 cells");
  if ((double)M * (N + 3) > 2.0e9) return fail(nullptr, AUSM_ERR_INVALID, "grid too large");
  ausm_solver* h = new ausm_solver();
  h->M = M;
  h->N = N;
  int rc = AUSM_OK;
  auto bail = [&](int code) {
    std::string msg = h->err;
    ausm_destroy(h);
    g_err = msg;
    return code;
  };
  if (cudaGetDevice(&h->dev) != cudaSuccess) {
    h->err = "no CUDA device";
    return bail(AUSM_ERR_CUDA);
  }
#define TRY(x)                        \
  do {                                \
    cudaError_t e_ = (x);             \
    if (e_ != cudaSuccess) {          \
      h->err = std::string(#x) + ": " + cudaGetErrorString(e_); \
      return bail(e_ == cudaErrorMemoryAllocation ? AUSM_ERR_OOM : AUSM_ERR_CUDA); \
    }                                 \
  } while (0)
  TRY(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
  h->own_st = h->st;
  TRY(cudaEventCreate(&h->e0));
  TRY(cudaEventCreate(&h->e1));
  size_t n = (size_t)M * N;
  TRY(dalloc(&h->V, (size_t)M * (N + 1)));
  TRY(dalloc(&h->Vd, (size_t)M * (N + 1)));
  TRY(dalloc(&h->Mi, n));
  TRY(dalloc(&h->Mj, (size_t)M * (N + 1)));
  for (auto& q : h->Q) TRY(dalloc(&q, n));
  TRY(dalloc(&h->wave, 4));
  TRY(dalloc(&h->dt, 4));
  TRY(dalloc(&h->dacc, 4));
  TRY(dalloc(&h->parts, 2 * (size_t)kMaxParts));
  TRY(dalloc(&h->move, 4));
  TRY(dalloc(&h->err_flag, 1));
  TRY(cudaMemsetAsync(h->err_flag, 0, sizeof(int), h->st));
  TRY(cudaMallocHost((void**)&h->h_dt, 4 * sizeof(float)));
  TRY(cudaMallocHost((void**)&h->h_wave, 4 * sizeof(uint32_t)));
  TRY(cudaMallocHost((void**)&h->h_acc, 4 * sizeof(double)));
  TRY(cudaMemsetAsync(h->wave, 0, 4 * sizeof(uint32_t), h->st));
#undef TRY
  {
    const float4* qs[3] = {h->Q[0], h->Q[1], h->Q[2]};
    // a solve whose maps cannot be encoded steps with the per-thread staging kernel
    for (int k = 0; k < 3; k++) encode_tma_maps(qs, h->Mi, h->Mj, M, N, kTileHeights[k], &h->tma[k]);
  }
  ausm_default_params(&h->p);
  h->speed_now = inflow_target(h->p);
  make_consts(h);
  h->body.assign((size_t)M * 2, 0.0);
  h->outer.assign((size_t)M * 2, 0.0);
  (void)rc;
  *out = h;
  return AUSM_OK;
}

int ausm_dims(const ausm_solver* h, int* M, int* N) {
  if (!h) return fail(nullptr, AUSM_ERR_INVALID, "null handle");
  if (M) *M = h->M;
  if (N) *N = h->N;
  return AUSM_OK;
}

int ausm_set_engine(ausm_solver* h, int engine) {
  NEED(h, h, AUSM_ERR_INVALID, "null handle");
  NEED(h, engine == AUSM_ENGINE_FUSED || engine == AUSM_ENGINE_REFERENCE || engine == AUSM_ENGINE_F64,
       AUSM_ERR_INVALID, "unknown engine");
  if (engine == h->engine) return AUSM_OK;
  NEED(h, !h->batch, AUSM_ERR_STATE, "a batch member stays on the fused engine; remove it from the batch first");
  int rc = use_device(h);
  if (rc) return rc;
  if (engine == AUSM_ENGINE_REFERENCE) {
    rc = ensure_reference_buffers(h);
    if (rc) return rc;
    if (h->has_grid) {
      launch_ref_metrics(h->V, h->area, h->flen, h->M, h->N, h->st);
      CHECK_LAUNCH(h);
    }
  }
  if (engine == AUSM_ENGINE_F64 && (rc = ensure_f64(h))) return rc;
  if (h->has_state) {  // carry the state over through the float reference layout
    if ((rc = state_to_staging(h))) return rc;
    h->engine = engine;
    if ((rc = staging_to_state(h))) return rc;
    return refresh_wave(h);
  }
  h->engine = engine;
  return AUSM_OK;
}

int ausm_set_params(ausm_solver* h, const AusmParams* p) {
  NEED(h, h, AUSM_ERR_INVALID, "null handle");
  NEED(h, p, AUSM_ERR_INVALID, "null params");
  NEED(h, p->gamma > 1.0 && p->in_rho > 0.0 && p->in_pressure > 0.0, AUSM_ERR_INVALID,
       "need gamma > 1, in_rho > 0, in_pressure > 0");
  NEED(h, p->cfl > 0.0 && p->maxdt > 0.0 && p->mach >= 0.0 && p->ramp >= 0.0, AUSM_ERR_INVALID,
       "need cfl > 0, maxdt > 0, mach >= 0, ramp >= 0");
  NEED(h, p->scheme >= 0 && p->scheme <= 2, AUSM_ERR_INVALID, "unknown scheme");
  NEED(h, std::isfinite(p->aoa_deg) && std::isfinite(p->K_p) && std::isfinite(p->K_u), AUSM_ERR_INVALID,
       "non-finite parameter");
  int rc = use_device(h);
  if (rc) return rc;
  bool gamma_changed = p->gamma != h->p.gamma;
  if (p->scheme != h->p.scheme) h->tile_rows = 0;  // tuned per scheme
  h->p = *p;
  if (p->ramp <= 0.0) h->speed_now = inflow_target(*p);
  make_consts(h);
  if (gamma_changed && h->has_state && h->has_grid) return refresh_wave(h);
  return AUSM_OK;
}

int ausm_get_params(const ausm_solver* h, AusmParams* p) {
  if (!h || !p) return fail(nullptr, AUSM_ERR_INVALID, "null argument");
  *p = h->p;
  return AUSM_OK;
}

int ausm_set_scheme(ausm_solver* h, int scheme) {
  NEED(h, h, AUSM_ERR_INVALID, "null handle");
  NEED(h, scheme >= 0 && scheme <= 2, AUSM_ERR_INVALID, "unknown scheme");
  if (scheme != h->p.scheme) h->tile_rows = 0;  // tuned per scheme
  h->p.scheme = scheme;
  return AUSM_OK;
}

int ausm_naca4_points(int M, int digits, double size, double x_offset, int closed_te, double* xy) {
  if (!xy || M < 4) return fail(nullptr, AUSM_ERR_INVALID, "need M >= 4 and an output array");
  if (!(digits > 0 && digits <= 9999 && size > 0.0))
    return fail(nullptr, AUSM_ERR_INVALID, "NACA digits 1..9999 and size > 0");
  if (digits % 100 == 0) return fail(nullptr, AUSM_ERR_INVALID, "NACA thickness must be > 0");
  int mdig = digits / 1000, pdig = (digits / 100) % 10;
  if (mdig != 0 && pdig == 0)
    return fail(nullptr, AUSM_ERR_INVALID, "cambered NACA needs a camber position digit > 0");
  double te = closed_te ? -0.1036 : -0.1015;
  for (int i = 0; i < M; i++) naca4_point(i, M, digits, size, x_offset, te, xy[2 * i], xy[2 * i + 1]);
  return AUSM_OK;
}

int ausm_set_body_naca4(ausm_solver* h, int digits, double size, double x_offset, int closed_te) {
  NEED(h, h, AUSM_ERR_INVALID, "null handle");
  int rc = ausm_naca4_points(h->M, digits, size, x_offset, closed_te, h->body.data());
  if (rc) return fail(h, rc, g_err);
  h->has_body = true;
  return AUSM_OK;
}

int ausm_set_body_points(ausm_solver* h, const double* xy, int n) {
  NEED(h, h, AUSM_ERR_INVALID, "null handle");
  NEED(h, xy, AUSM_ERR_INVALID, "null points");
  NEED(h, n == h->M, AUSM_ERR_INVALID, "body needs exactly M points");
  for (int k = 0; k < 2 * n; k++) NEED(h, std::isfinite(xy[k]), AUSM_ERR_INVALID, "non-finite body point");
  std::memcpy(h->body.data(), xy, sizeof(double) * 2 * n);
  h->has_body = true;
  return AUSM_OK;
}

int ausm_outer_points(int M, int kind, double p0, double p1, double p2, double* xy) {
  if (!xy || M < 4) return fail(nullptr, AUSM_ERR_INVALID, "need M >= 4 and an output array");
  if (!(p0 > 0.0)) return fail(nullptr, AUSM_ERR_INVALID, "outer boundary size must be > 0");
  if (kind == AUSM_OUTER_RECT) {  // grid.js:238-255
    for (int i = 0; i < M; i++) {
      double t = (double)i / M;
      t = std::fmod(t + 0.125, 1.0);
      double x, y;
      if (t < 0.25) {
        t *= 4;
        x = p0; y = t * 2 - 1;
      } else if (t < 0.5) {
        t = (t - 0.25) * 4;
        x = ((1 - t) * 2 - 1) * p0; y = 1;
      } else if (t < 0.75) {
        t = (t - 0.5) * 4;
        x = -p0; y = (1 - t) * 2 - 1;
      } else {
        t = (t - 0.75) * 4;
        x = (t * 2 - 1) * p0; y = -1;
      }
      xy[2 * i] = x;
      xy[2 * i + 1] = y;
    }
  } else if (kind == AUSM_OUTER_CIRCLE) {  // grid.js:232-237, centred at (p1, p2)
    for (int i = 0; i < M; i++) {
      double t = (double)i / M;
      xy[2 * i] = p1 + p0 * std::cos(t * M_PI * 2);
      xy[2 * i + 1] = p2 + p0 * std::sin(t * M_PI * 2);
    }
  } else {
    return fail(nullptr, AUSM_ERR_INVALID, "unknown outer boundary kind");
  }
  return AUSM_OK;
}

int ausm_set_outer(ausm_solver* h, int kind, double p0, double p1, double p2) {
  NEED(h, h, AUSM_ERR_INVALID, "null handle");
  int rc = ausm_outer_points(h->M, kind, p0, p1, p2, h->outer.data());
  if (rc) return fail(h, rc, g_err);
  h->has_outer = true;
  return AUSM_OK;
}

int ausm_set_radial_stretch(ausm_solver* h, double first_spacing) {
  NEED(h, h, AUSM_ERR_INVALID, "null handle");
  NEED(h, std::isfinite(first_spacing), AUSM_ERR_INVALID, "non-finite spacing");
  h->stretch = first_spacing;
  return AUSM_OK;
}

int ausm_generate_grid(ausm_solver* h, int iters, int method, double tol, int* iters_done) {
  NEED(h, h, AUSM_ERR_INVALID, "null handle");
  NEED(h, h->has_body && h->has_outer, AUSM_ERR_STATE, "set the body and outer boundary first");
  NEED(h, iters >= 0, AUSM_ERR_INVALID, "iters must be >= 0");
  NEED(h, method == AUSM_GRID_JACOBI || method == AUSM_GRID_MULTICOLOR, AUSM_ERR_INVALID, "unknown grid method");
  int rc = use_device(h);
  if (rc) return rc;
  const int M = h->M, N = h->N;
  int done = 0;
  if (method == AUSM_GRID_JACOBI) {  // FP32, the reference's generator (shaders/grid.js:33-113)
    std::vector<float> v((size_t)M * (N + 1) * 2, 0.0f);
    for (int i = 0; i < M; i++) {
      v[2 * i] = (float)h->body[2 * i];
      v[2 * i + 1] = (float)h->body[2 * i + 1];
      size_t o = ((size_t)N * M + i) * 2;
      v[o] = (float)h->outer[2 * i];
      v[o + 1] = (float)h->outer[2 * i + 1];
    }
    CU(h, cudaMemcpyAsync(h->V, v.data(), v.size() * sizeof(float), cudaMemcpyHostToDevice, h->st));
    launch_grid_init(h->V, M, N, h->stretch, h->st);
    CHECK_LAUNCH(h);
    if (iters > 0) {
      if (!h->V2) CU(h, dalloc(&h->V2, (size_t)M * (N + 1)));
      CU(h, cudaMemcpyAsync(h->V2, h->V, (size_t)M * (N + 1) * sizeof(float2), cudaMemcpyDeviceToDevice, h->st));
      float2 *src = h->V, *dst = h->V2;
      for (int it = 0; it < iters; it++) {
        launch_grid_jacobi(src, dst, M, N, h->st);
        std::swap(src, dst);
      }
      CHECK_LAUNCH(h);
      if (src != h->V)
        CU(h, cudaMemcpyAsync(h->V, src, (size_t)M * (N + 1) * sizeof(float2), cudaMemcpyDeviceToDevice, h->st));
    }
    launch_f2d(h->V, h->Vd, (size_t)M * (N + 1), h->st);
    done = iters;
  } else {  // FP64 multicolor Gauss-Seidel from the FP64 boundaries
    std::vector<double> vd((size_t)M * (N + 1) * 2, 0.0);
    for (int i = 0; i < M; i++) {
      vd[2 * i] = h->body[2 * i];
      vd[2 * i + 1] = h->body[2 * i + 1];
      size_t o = ((size_t)N * M + i) * 2;
      vd[o] = h->outer[2 * i];
      vd[o + 1] = h->outer[2 * i + 1];
    }
    CU(h, cudaMemcpyAsync(h->Vd, vd.data(), vd.size() * sizeof(double), cudaMemcpyHostToDevice, h->st));
    launch_grid_init_d(h->Vd, M, N, h->stretch, h->st);
    CHECK_LAUNCH(h);
    const int ncol = (M & 1) ? 6 : 4;
    const int check_every = 25;
    for (int it = 0; it < iters; it++) {
      CU(h, cudaMemsetAsync(h->move, 0, sizeof(uint32_t), h->st));
      for (int col = 0; col < ncol; col++) launch_grid_multicolor_d(h->Vd, M, N, col, 1.0, h->move, h->st);
      done = it + 1;
      if (tol > 0.0 && (done % check_every == 0 || done == iters)) {
        CHECK_LAUNCH(h);
        CU(h, cudaMemcpyAsync(h->h_wave + 1, h->move, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->st));
        CU(h, cudaStreamSynchronize(h->st));
        float mv;
        std::memcpy(&mv, h->h_wave + 1, 4);
        if (mv <= tol) break;
      }
    }
    CHECK_LAUNCH(h);
    launch_d2f(h->Vd, h->V, (size_t)M * (N + 1), h->st);
  }
  CHECK_LAUNCH(h);
  if (iters_done) *iters_done = done;
  return after_grid(h);
}

int ausm_set_vertices(ausm_solver* h, const float* xy) {
  NEED(h, h, AUSM_ERR_INVALID, "null handle");
  NEED(h, xy, AUSM_ERR_INVALID, "null vertices");
  int rc = use_device(h);
  if (rc) return rc;
  CU(h, cudaMemcpyAsync(h->V, xy, (size_t)h->M * (h->N + 1) * sizeof(float2), cudaMemcpyHostToDevice, h->st));
  launch_f2d(h->V, h->Vd, (size_t)h->M * (h->N + 1), h->st);
  return after_grid(h);
}

int ausm_get_vertices(ausm_solver* h, float* xy) {
  NEED(h, h, AUSM_ERR_INVALID, "null handle");
  NEED(h, xy, AUSM_ERR_INVALID, "null vertices");
  NEED(h, h->has_grid, AUSM_ERR_STATE, "no grid yet");
  int rc = use_device(h);
  if (rc) return rc;
  CU(h, cudaMemcpyAsync(xy, h->V, (size_t)h->M * (h->N + 1) * sizeof(float2), cudaMemcpyDeviceToHost, h->st));
  CU(h, cudaStreamSynchronize(h->st));
  return AUSM_OK;
}

int ausm_init_state(ausm_solver* h, int mode) {
  NEED(h, h, AUSM_ERR_INVALID, "null handle");
  NEED(h, h->has_grid, AUSM_ERR_STATE, "no grid yet");
  NEED(h, mode == AUSM_INIT_REST || mode == AUSM_INIT_FREESTREAM, AUSM_ERR_INVALID, "unknown init mode");
  int rc = use_device(h);
  if (rc) return rc;
  if (h->p.ramp > 0.0) {  // prepareState restarts the ramp from rest (main.js:654)
    h->speed_now = 0.0;
    make_consts(h);
  }
  const Consts& c = h->c;
  float4 s = mode == AUSM_INIT_REST ? make_float4(c.inRho, 0.0f, 0.0f, c.inP / (c.gamma - 1.0f)) : c.inState;
  if (h->engine == AUSM_ENGINE_FUSED) {
    h->cur = 0;
    launch_fill(h->Q[0], s, (size_t)h->M * h->N, h->st);
  } else if (h->engine == AUSM_ENGINE_REFERENCE) {
    launch_fill(h->S[2], s, (size_t)h->M * (h->N + 3), h->st);
  } else {
    const ex::ConstsR<double>& d = h->cd;
    if (mode == AUSM_INIT_REST) h->f64->fill(d.inRho, 0.0, 0.0, d.inP / (d.gamma - 1.0), h->st);
    else h->f64->fill(d.inState.x, d.inState.y, d.inState.z, d.inState.w, h->st);
  }
  CHECK_LAUNCH(h);
  h->has_state = true;
  return refresh_wave(h);
}

int ausm_set_state(ausm_solver* h, const float* q) {
  NEED(h, h, AUSM_ERR_INVALID, "null handle");
  NEED(h, q, AUSM_ERR_INVALID, "null state");
  NEED(h, h->has_grid, AUSM_ERR_STATE, "no grid yet");
  int rc = use_device(h);
  if (rc) return rc;
  size_t bytes = (size_t)h->M * (h->N + 3) * sizeof(float4);
  if (h->engine == AUSM_ENGINE_REFERENCE) {
    CU(h, cudaMemcpyAsync(h->S[2], q, bytes, cudaMemcpyHostToDevice, h->st));
  } else {
    if ((rc = ensure_staging(h))) return rc;
    CU(h, cudaMemcpyAsync(h->staging, q, bytes, cudaMemcpyHostToDevice, h->st));
    if ((rc = staging_to_state(h))) return rc;
  }
  h->has_state = true;
  return refresh_wave(h);
}

int ausm_get_state(ausm_solver* h, float* q) {
  NEED(h, h, AUSM_ERR_INVALID, "null handle");
  NEED(h, q, AUSM_ERR_INVALID, "null state");
  NEED(h, h->has_state, AUSM_ERR_STATE, "no state yet");
  int rc = use_device(h);
  if (rc) return rc;
  if ((rc = state_to_staging(h))) return rc;
  CU(h, cudaMemcpyAsync(q, h->staging, (size_t)h->M * (h->N + 3) * sizeof(float4), cudaMemcpyDeviceToHost, h->st));
  return sync_and_check(h);
}

int ausm_get_state_f64(ausm_solver* h, double* q) {
  NEED(h, h, AUSM_ERR_INVALID, "null handle");
  NEED(h, q, AUSM_ERR_INVALID, "null state");
  NEED(h, h->has_state, AUSM_ERR_STATE, "no state yet");
  int rc = use_device(h);
  if (rc) return rc;
  const size_t n = (size_t)h->M * (h->N + 3);
  if (h->engine == AUSM_ENGINE_F64) {
    const void* src = h->f64->state_ref(h->Vd, h->st);
    CHECK_LAUNCH(h);
    CU(h, cudaMemcpyAsync(q, src, n * 4 * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CU(h, cudaStreamSynchronize(h->st));
    return AUSM_OK;
  }
  std::vector<float> f(n * 4);
  if ((rc = ausm_get_state(h, f.data()))) return rc;
  for (size_t k = 0; k < f.size(); k++) q[k] = f[k];
  return AUSM_OK;
}

}  // extern "C"

namespace {
// ausm_step; read_err: queue the read of the timeout flag (ausm_time_steps queues one
// after all its repetitions instead, so that its timed steps stay back to back).
int step_impl(ausm_solver* h, int n, float* dt_out, bool read_err) {
  NEED(h, h, AUSM_ERR_INVALID, "null handle");
  NEED(h, n >= 0, AUSM_ERR_INVALID, "n must be >= 0");
  NEED(h, h->has_grid && h->has_state, AUSM_ERR_STATE, "need a grid and a state");
  int rc = use_device(h);
  if (rc) return rc;
  const int M = h->M, N = h->N, sch = h->p.scheme;
  cudaStream_t s = h->st;
  if (h->engine == AUSM_ENGINE_F64) {
    h->f64->step(sch, n, h->Vd, s);
    CHECK_LAUNCH(h);
    ramp_after_steps(h, n);
    if (dt_out) {
      CU(h, cudaMemcpyAsync(h->h_acc, h->f64->dt, sizeof(double), cudaMemcpyDeviceToHost, s));
      CU(h, cudaMemcpyAsync(h->h_acc + 1, h->f64->wave, sizeof(double), cudaMemcpyDeviceToHost, s));
      CU(h, cudaStreamSynchronize(s));
      *dt_out = (float)h->h_acc[0];
      if (!std::isfinite(h->h_acc[1]) || !std::isfinite(h->h_acc[0]))
        return fail(h, AUSM_ERR_DIVERGED, "max wave speed is not finite: the solution diverged");
    }
    return AUSM_OK;
  }
  if (n == 0 || h->engine != AUSM_ENGINE_FUSED) launch_dt(h->wave, h->dt, h->c.maxdt, h->c.cfl, s);
  if (n > 0) {
    // fused: the first step's stage 1 computes dt from *wave and its stage 2 clears
    // *wave (dt_mode 1, 2), so a step is three launches
    if (h->engine != AUSM_ENGINE_FUSED) CU(h, cudaMemsetAsync(h->wave, 0, sizeof(uint32_t), s));
    if (h->engine == AUSM_ENGINE_FUSED) {
      int rows = 16;
      if ((rc = tuned_tile_rows(h, false, &rows))) return rc;
      for (int k = 0; k < n; k++) {
        int a = h->cur, b = (a + 1) % 3, c3 = (a + 2) % 3;
        TmaMapsLaunch t1, t2, t3;
        const TmaMapsLaunch *p1 = nullptr, *p2 = nullptr, *p3 = nullptr;
        const TmaMaps& tm = h->tma[tile_index(rows)];
        if (tm.ok) {
          t1 = {tm.halo[a], tm.plain[a], tm.mi, tm.mj, tm.wrap[a]};
          t2 = {tm.halo[b], tm.plain[a], tm.mi, tm.mj, tm.wrap[b]};
          t3 = {tm.halo[c3], tm.plain[a], tm.mi, tm.mj, tm.wrap[c3]};
          p1 = &t1; p2 = &t2; p3 = &t3;
        }
        launch_fused_stage(sch, 1, false, h->Q[a], nullptr, h->Q[b], h->Mi, h->Mj, h->dt, h->wave, k == 0 ? 1 : 0,
                           h->c, M, N, p1, rows, h->err_flag, s);
        launch_fused_stage(sch, 2, false, h->Q[b], h->Q[a], h->Q[c3], h->Mi, h->Mj, h->dt, h->wave, k == 0 ? 2 : 0,
                           h->c, M, N, p2, rows, h->err_flag, s);
        launch_fused_stage(sch, 3, k == n - 1, h->Q[c3], h->Q[a], h->Q[b], h->Mi, h->Mj, h->dt, h->wave, 0, h->c, M,
                           N, p3, rows, h->err_flag, s);
        h->cur = b;
      }
    } else {
      // texture ping-pong of main.js:744-777
      float4 **S = h->S;
      for (int k = 0; k < n; k++) {
        launch_ref_boundary(S[2], S[0], h->V, h->c, M, N, s);
        launch_ref_fluxes(sch, S[0], h->V, h->fx, h->fy, h->c, M, N, s);
        launch_ref_residual(h->fx, h->fy, h->flen, h->area, h->res, M, N, s);
        launch_ref_rk(1, h->res, S[0], nullptr, S[1], h->dt, M, N, s);
        launch_ref_boundary(S[1], S[2], h->V, h->c, M, N, s);
        launch_ref_fluxes(sch, S[2], h->V, h->fx, h->fy, h->c, M, N, s);
        launch_ref_residual(h->fx, h->fy, h->flen, h->area, h->res, M, N, s);
        launch_ref_rk(2, h->res, S[0], S[1], S[2], h->dt, M, N, s);
        launch_ref_boundary(S[2], S[1], h->V, h->c, M, N, s);
        launch_ref_fluxes(sch, S[1], h->V, h->fx, h->fy, h->c, M, N, s);
        launch_ref_residual(h->fx, h->fy, h->flen, h->area, h->res, M, N, s);
        launch_ref_rk(3, h->res, S[0], S[1], S[2], h->dt, M, N, s);
      }
      launch_ref_wave(S[2], h->flen, h->area, h->c.gamma, M, N, h->wave, s);
    }
  }
  CHECK_LAUNCH(h);
  ramp_after_steps(h, n);
  if (h->engine == AUSM_ENGINE_FUSED && n > 0 && (read_err || dt_out) && (rc = queue_err_read(h))) return rc;
  if (dt_out) {
    CU(h, cudaMemcpyAsync(h->h_dt, h->dt, sizeof(float), cudaMemcpyDeviceToHost, s));
    CU(h, cudaMemcpyAsync(h->h_wave, h->wave, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    if ((rc = sync_and_check(h))) return rc;
    *dt_out = h->h_dt[0];
    float w;
    std::memcpy(&w, h->h_wave, 4);
    if (!std::isfinite(w) || !std::isfinite(h->h_dt[0]))
      return fail(h, AUSM_ERR_DIVERGED, "max wave speed is not finite: the solution diverged");
  }
  return AUSM_OK;
}
}  // namespace

extern "C" {

int ausm_step(ausm_solver* h, int n, float* dt_out) { return step_impl(h, n, dt_out, true); }

int ausm_max_wave_speed(ausm_solver* h, float* out) {
  NEED(h, h, AUSM_ERR_INVALID, "null handle");
  NEED(h, out, AUSM_ERR_INVALID, "null output");
  int rc = use_device(h);
  if (rc) return rc;
  if (h->engine == AUSM_ENGINE_F64) {
    CU(h, cudaMemcpyAsync(h->h_acc, h->f64->wave, sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CU(h, cudaStreamSynchronize(h->st));
    *out = (float)h->h_acc[0];
    return AUSM_OK;
  }
  CU(h, cudaMemcpyAsync(h->h_wave, h->wave, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->st));
  if ((rc = sync_and_check(h))) return rc;
  std::memcpy(out, h->h_wave, 4);
  return AUSM_OK;
}

int ausm_forces(ausm_solver* h, double* out6, double* cp) {
  NEED(h, h, AUSM_ERR_INVALID, "null handle");
  NEED(h, h->has_state, AUSM_ERR_STATE, "no state yet");
  int rc = use_device(h);
  if (rc) return rc;
  const AusmParams& p = h->p;
  double a = p.aoa_deg * M_PI / 180.0;
  double vx = h->speed_now * std::cos(a), vy = h->speed_now * std::sin(a);
  double q_inf = 0.5 * p.in_rho * (vx * vx + vy * vy);
  if (cp && !h->cp) CU(h, dalloc(&h->cp, (size_t)h->M));
  if (h->engine == AUSM_ENGINE_F64)
    h->f64->forces(h->Vd, h->parts, h->dacc, cp ? h->cp : nullptr, q_inf, p.in_pressure, h->st);
  else
    launch_forces(interior(h), h->Vd, h->c, h->M, h->dacc, h->parts, cp ? h->cp : nullptr, q_inf, p.in_pressure,
                  h->st);
  CHECK_LAUNCH(h);
  CU(h, cudaMemcpyAsync(h->h_acc, h->dacc, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  if (cp) CU(h, cudaMemcpyAsync(cp, h->cp, (size_t)h->M * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  if ((rc = sync_and_check(h))) return rc;
  double Fx = h->h_acc[0], Fy = h->h_acc[1];
  double vl = std::sqrt(vx * vx + vy * vy);
  double nx = vx / vl, ny = vy / vl;
  double invQ = 1.0 / q_inf;
  double Cl = (Fx * -ny + Fy * nx) * invQ, Cd = (Fx * nx + Fy * ny) * invQ;
  double FV = Fx * nx + Fy * ny;
  if (out6) {
    out6[0] = Fx;
    out6[1] = Fy;
    out6[2] = std::sqrt(Fx * Fx + Fy * Fy) * (FV > 0 ? 1.0 : (FV < 0 ? -1.0 : 0.0));
    out6[3] = Cl;
    out6[4] = Cd;
    out6[5] = Cl / Cd;
  }
  return AUSM_OK;
}

int ausm_residual_l2(ausm_solver* h, double* l2) {
  NEED(h, h, AUSM_ERR_INVALID, "null handle");
  NEED(h, l2, AUSM_ERR_INVALID, "null output");
  NEED(h, h->has_grid && h->has_state, AUSM_ERR_STATE, "need a grid and a state");
  int rc = use_device(h);
  if (rc) return rc;
  const int M = h->M, N = h->N;
  const float4* R = nullptr;
  if (h->engine == AUSM_ENGINE_F64) {
    h->f64->residual(h->p.scheme, h->Vd, h->st);
    h->f64->sumsq_rho(h->parts, h->dacc, h->st);
  } else if (h->engine == AUSM_ENGINE_FUSED) {
    float4* scratch = h->Q[(h->cur + 1) % 3];
    launch_fused_stage(h->p.scheme, 0, false, h->Q[h->cur], nullptr, scratch, h->Mi, h->Mj, h->dt, h->wave, 0, h->c, M,
                       N, nullptr, 16, h->err_flag, h->st);
    R = scratch;
  } else {
    launch_ref_boundary(h->S[2], h->S[0], h->V, h->c, M, N, h->st);
    launch_ref_fluxes(h->p.scheme, h->S[0], h->V, h->fx, h->fy, h->c, M, N, h->st);
    launch_ref_residual(h->fx, h->fy, h->flen, h->area, h->res, M, N, h->st);
    R = h->res;
  }
  if (R) launch_sumsq_rho(R, (size_t)M * N, h->dacc, h->parts, h->st);
  CHECK_LAUNCH(h);
  CU(h, cudaMemcpyAsync(h->h_acc, h->dacc, sizeof(double), cudaMemcpyDeviceToHost, h->st));
  if ((rc = sync_and_check(h))) return rc;
  *l2 = std::sqrt(h->h_acc[0] / ((double)M * N));
  if (!std::isfinite(*l2)) return fail(h, AUSM_ERR_DIVERGED, "residual norm is not finite: the solution diverged");
  return AUSM_OK;
}

int ausm_field(ausm_solver* h, int kind, float* out) {
  NEED(h, h, AUSM_ERR_INVALID, "null handle");
  NEED(h, out, AUSM_ERR_INVALID, "null output");
  NEED(h, kind >= 0 && kind <= AUSM_FIELD_WAVE_SPEED, AUSM_ERR_INVALID, "unknown field");
  NEED(h, h->has_grid && h->has_state, AUSM_ERR_STATE, "need a grid and a state");
  int rc = use_device(h);
  if (rc) return rc;
  rc = ensure_staging(h);
  if (rc) return rc;
  const float4* q;
  float* buf = reinterpret_cast<float*>(h->staging);
  if (h->engine == AUSM_ENGINE_F64) {  // rounded to f32 into staging; the field goes past it
    if ((rc = state_to_staging(h))) return rc;
    q = h->staging + h->M;
    buf = reinterpret_cast<float*>(h->staging + (size_t)h->M * (h->N + 3));
  } else {
    q = interior(h);
  }
  launch_field(q, h->V, h->c, kind, h->M, h->N, buf, h->st);
  CHECK_LAUNCH(h);
  CU(h, cudaMemcpyAsync(out, buf, (size_t)h->M * h->N * sizeof(float), cudaMemcpyDeviceToHost, h->st));
  return sync_and_check(h);
}

int ausm_stream(ausm_solver* h, void** stream) {
  NEED(h, h, AUSM_ERR_INVALID, "null handle");
  NEED(h, stream, AUSM_ERR_INVALID, "null output");
  *stream = (void*)h->st;
  return AUSM_OK;
}

int ausm_synchronize(ausm_solver* h) {
  NEED(h, h, AUSM_ERR_INVALID, "null handle");
  return sync_and_check(h);
}

int ausm_debug_set_wait_polls(unsigned polls) {
  NEED(nullptr, polls <= 65536u, AUSM_ERR_INVALID, "polls must be in [0, 65536] (the default bound)");
  // the solvers' streams do not synchronise with the copy to the constant: let the work
  // already queued run with the bound it was queued under, and the next launches see the new one
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = set_wait_polls_fused(polls);
  if (e == cudaSuccess) e = set_wait_polls_batch(polls);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return fail(nullptr, AUSM_ERR_CUDA, std::string("wait polls: ") + cudaGetErrorString(e));
  return AUSM_OK;
}

int ausm_autotune(ausm_solver* h, int force, int* rows) {
  NEED(h, h, AUSM_ERR_INVALID, "null handle");
  NEED(h, h->has_grid && h->has_state, AUSM_ERR_STATE, "need a grid and a state");
  int rc = use_device(h);
  if (rc) return rc;
  int r = 16;
  if (h->engine == AUSM_ENGINE_FUSED) {
    launch_dt(h->wave, h->dt, h->c.maxdt, h->c.cfl, h->st);
    if ((rc = tuned_tile_rows(h, force != 0, &r))) return rc;
  }
  if (rows) *rows = r;
  return AUSM_OK;
}

int ausm_time_steps(ausm_solver* h, int n, int reps, float* ms_out) {
  NEED(h, h, AUSM_ERR_INVALID, "null handle");
  NEED(h, ms_out && reps > 0 && n > 0, AUSM_ERR_INVALID, "need n > 0, reps > 0 and an output");
  int rc = use_device(h);
  if (rc) return rc;
  CU(h, cudaEventRecord(h->e0, h->st));
  for (int r = 0; r < reps; r++) {
    rc = step_impl(h, n, nullptr, false);
    if (rc) return rc;
  }
  CU(h, cudaEventRecord(h->e1, h->st));
  if (h->engine == AUSM_ENGINE_FUSED && (rc = queue_err_read(h))) return rc;
  CU(h, cudaEventSynchronize(h->e1));
  CU(h, cudaEventElapsedTime(ms_out, h->e0, h->e1));
  return sync_and_check(h);
}

}  // extern "C"
