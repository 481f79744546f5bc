// Host-side state of a solver handle, shared by the C-ABI files (api.cu, batch.cu).
#pragma once
#include <string>
#include <vector>

#include "ausm.h"
#include "ausm_internal.h"

struct ausm_solver {
  int M = 0, N = 0, dev = 0;
  int engine = AUSM_ENGINE_FUSED;
  AusmParams p{};
  double speed_now = 0.0;  // current inflow speed (ramped when p.ramp > 0)
  ausm::Consts c{};
  ausm::ex::ConstsR<double> cd{};  // the same constants in FP64 (F64 engine)
  ausm::F64Engine* f64 = nullptr;  // buffers of the F64 engine, once selected
  cudaStream_t st = nullptr;      // the stream calls run on (the batch's while a member)
  cudaStream_t own_st = nullptr;  // the handle's own stream
  ausm_batch* batch = nullptr;    // batch this solver belongs to, if any
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  std::vector<double> body, outer;  // M x 2
  bool has_body = false, has_outer = false, has_grid = false, has_state = false;
  double stretch = 0.0;
  float2* V = nullptr;    // vertices, FP32 (reference layout, API, reference engine)
  float2* V2 = nullptr;   // Jacobi ping-pong
  double2* Vd = nullptr;  // vertices, FP64 (multicolor generator, metrics, forces)
  float4* Mi = nullptr;   // FP64-computed face records, i-faces [N][M]
  float4* Mj = nullptr;   // ... j-faces [N+1][M]
  float4* Q[3] = {nullptr, nullptr, nullptr};
  int cur = 0;
  float4* S[3] = {nullptr, nullptr, nullptr};
  float4 *fx = nullptr, *fy = nullptr, *res = nullptr, *flen = nullptr;
  float* area = nullptr;
  float4* staging = nullptr;
  double* cp = nullptr;
  uint32_t* wave = nullptr;
  float* dt = nullptr;
  double* dacc = nullptr;
  double* parts = nullptr;  // 2 * kMaxParts per-block partial sums
  uint32_t* move = nullptr;
  int* err_flag = nullptr;  // set by a kernel whose bounded wait gave up
  bool err_read_queued = false;  // a copy of *err_flag to h_wave[2] is queued on st (api.cu)
  ausm::TmaMaps tma[3];  // per tile height kTileHeights[k]
  int tile_rows = 0;      // tile height of the TMA stage kernel; 0 until tuned
  float* h_dt = nullptr;
  uint32_t* h_wave = nullptr;
  double* h_acc = nullptr;
  std::string err;
};

namespace ausm {
// Reference-order f32 uniforms of h's parameters and current inflow speed (api.cu).
void make_consts(ausm_solver* h);
// Inflow speed update of a ramped start after n steps (main.js:779), api.cu.
void ramp_after_steps(ausm_solver* h, int n);
void set_thread_error(const std::string& msg);
// Tile height for h's fused steps: AUSM_TILE_ROWS, the process-wide tuning cache for
// (M, N, scheme), or a tuning run (api.cu).  Enqueues work on h's stream; must not run
// inside a stream capture.
int tuned_tile_rows(ausm_solver* h, bool force, int* rows);
inline int tile_index(int rows) { return rows == 8 ? 0 : (rows == 32 ? 2 : 1); }
}  // namespace ausm
