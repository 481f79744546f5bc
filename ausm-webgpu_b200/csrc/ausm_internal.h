// Internal declarations shared by the CUDA kernels and the C-ABI layer.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstdlib>

#include "physics.cuh"
#include "physics_exact.cuh"

namespace ausm {

// Block sizes must be multiples of 32 threads.
// Block-wide max of non-negative float bit patterns (u32 order == float order for
// x >= 0; NaN bit patterns compare above +inf, so a NaN wave speed propagates and the
// host reports divergence).  One atomicMax per block into *dst.  All threads call it.
// Launch with programmatic stream serialization: the kernel may start while its
// stream predecessor is still running and waits for it with grid_dep_wait (tma.cuh)
// before reading anything that kernel writes.  AUSM_PDL=0 launches plainly (A/B
// timing).
inline bool pdl_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("AUSM_PDL");
    return !(e && e[0] == '0');
  }();
  return on;
}
template <class... KArgs, class... Args>
cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, static_cast<Args&&>(args)...);
}

__device__ __forceinline__ void block_max_to(uint32_t* dst, uint32_t v) {
  __shared__ uint32_t warp_max[32];
  v = __reduce_max_sync(0xffffffffu, v);
  const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int lane = t & 31, w = t >> 5;
  if (lane == 0) warp_max[w] = v;
  __syncthreads();
  if (w == 0) {
    const int nw = (blockDim.x * blockDim.y * blockDim.z + 31) >> 5;
    uint32_t x = lane < nw ? warp_max[lane] : 0u;
    x = __reduce_max_sync(0xffffffffu, x);
    if (lane == 0) atomicMax(dst, x);
  }
}

// Block-wide sum of doubles, stored by one thread into *dst (a per-block slot; the
// slots are then summed in a fixed order by launch_sum_parts, so the total does not
// depend on block timing).  All threads call it.
__device__ __forceinline__ void block_sum_store(double* dst, double v) {
  __shared__ double warp_sum[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int lane = t & 31, w = t >> 5;
  if (lane == 0) warp_sum[w] = v;
  __syncthreads();
  if (w == 0) {
    const int nw = (blockDim.x * blockDim.y * blockDim.z + 31) >> 5;
    double x = lane < nw ? warp_sum[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) *dst = x;
  }
}
// Per-block partial sums of a reduction (at most kMaxParts blocks per quantity).
constexpr int kMaxParts = 148 * 16;

// ---- fused engine (kernels_fused.cu) ----
// TMA descriptors of one solve for one tile height ty: per state buffer the halo box
// (36 x (ty+4) cells), the plain box (32 x ty cells) and the seam box (2 x (ty+4)
// cells: the two columns a tile at the seam wraps to), and the face-record boxes
// (33 x ty i-faces, 32 x (ty+1) j-faces).
struct TmaMaps {
  CUtensorMap halo[3];
  CUtensorMap plain[3];
  CUtensorMap mi, mj;
  CUtensorMap wrap[3];
  bool ok = false;
};
struct TmaMapsLaunch {  // the five a stage launch reads
  CUtensorMap qs;
  CUtensorMap qn;
  CUtensorMap mi, mj;
  CUtensorMap wrap;  // seam box of the buffer qs reads
};
// Tile heights of the TMA tile kernels (the autotuner's candidates) and their index.
constexpr int kTileHeights[3] = {8, 16, 32};
bool encode_tma_maps(const float4* const Q[3], const float4* Mi, const float4* Mj, int M, int N, int ty,
                     TmaMaps* out);
// stage 1..3: RK stage; stage 0: write dQ/dt of Qs to Qo.  emit (stage 3 only):
// atomicMax the new state's wave speed bits into *wave (cleared before, see dt_mode).
// With tm != nullptr the TMA kernel runs and sets *err on a bounded-wait timeout.
// Mi, Mj: the FP64-computed face records (launch_metrics_d).
// ty: tile height of the TMA tile kernel (8, 16 or 32; tm must come from maps of that
// height); the per-thread kernel uses 16.
// dt_mode: 0 the stage reads *dt; 1 (stage 1 of a call's first step) dt = min(maxdt,
// cfl / *wave) is computed and stored to *dt; 2 (stage 2 of that step) *wave is
// cleared.  The TMA tile kernel does both in the kernel; for the others a dt kernel or
// a memset runs before the stage.
void launch_fused_stage(int scheme, int stage, bool emit, const float4* Qs, const float4* Qn, float4* Qo,
                        const float4* Mi, const float4* Mj, float* dt, uint32_t* wave, int dt_mode, const Consts& c,
                        int M, int N, const TmaMapsLaunch* tm, int ty, int* err, cudaStream_t s);
void launch_wave_interior(const float4* Q, const float4* Mj, float gamma, int M, int N, uint32_t* wave,
                          cudaStream_t s);
// Polls of the first bounded wait of each TMA box in the single-solve and batched stage
// kernels (ausm_debug_set_wait_polls), on the current device.
cudaError_t set_wait_polls_fused(unsigned polls);
cudaError_t set_wait_polls_batch(unsigned polls);

// ---- batched engine (kernels_batch.cu) ----
// One solve of a batch as the device sees it.  Its tiles are work items
// tile0 .. tile0 + tiles_x * tiles_y - 1 of the batch; cur is the index of the buffer
// holding the current state (the RK3 buffers rotate by one per step).
struct BatchSolve {
  float4* Q[3];
  const float4* Mi;
  const float4* Mj;
  const CUtensorMap* maps;  // in device memory: halo[0..2], plain[0..2], mi, mj; null without TMA
  float* dt;
  uint32_t* wave;
  Consts c;
  int M, N, scheme, tiles_x, tile0, cur;  // scheme: the work-list group key (scheme, + 4 with MUSCL on)
  int chunk0;  // first residual-norm chunk (512 cells) of the solve
};
// Tensor maps per batch member, in this order: halo[0..2], plain[0..2], mi, mj,
// wrap[0..2] (TmaMaps of the batch's tile height).
constexpr int kBatchMaps = 11;
// One work item (tile) of a batch: its solve's descriptor index, that solve's buffer
// rotation when the table was written, the tile's column | row << 16, and the solve's
// M (what the tile's loads need, in one 16-byte load).
struct alignas(16) BatchItem {
  int solve, cur, tile, M;
};
// All launches go to stream s.  rot: steps already taken since the descriptors' cur.
// Stage 0 writes the residual dQ/dt of the current state into the solve's next buffer.
// A stage launch covers the work items [t_lo, t_hi) of one scheme group; *steps counts
// the steps the batch has taken since the item table was written (so a solve's current
// buffer is (items[t].cur + *steps + rot) % 3); maps holds kBatchMaps tensor maps per
// descriptor.
void launch_batch_dt(BatchSolve* d, int nsolves, cudaStream_t s);
// rows: tile height (8, 16, 32) the descriptors' work items were laid out with.  With
// err != nullptr (every solve of the launch has maps for that height) stages 1-3 stage
// their tiles by TMA and a bounded-wait timeout sets *err; without TMA rows must be 16.
void launch_batch_stage(int scheme, int stage, bool emit, const BatchSolve* d, const BatchItem* items,
                        const int* steps, const CUtensorMap* maps, int t_lo, int t_hi, int rot, int rows, int* err,
                        cudaStream_t s);
// advances every descriptor's cur and the batch's step counter *taken by `steps`
void launch_batch_advance(BatchSolve* d, int nsolves, int steps, int* taken, cudaStream_t s);
// out[2 s] = dt, out[2 s + 1] = max wave speed of solve s
void launch_batch_gather(const BatchSolve* d, int nsolves, float* out, cudaStream_t s);
// l2[s] = sqrt(mean over solve s's cells of (d rho / dt)^2), from the stage-0 residual;
// part holds one double per norm chunk (512 cells of one solve; chunk0 in the
// descriptors).  Summation order depends only on the solve's own grid.
void launch_batch_residual_norm(const BatchSolve* d, int nsolves, int total_chunks, double* part, double* l2,
                                cudaStream_t s);

// ---- full-FP64 engine (kernels_f64.cu, built with -fmad=false) ----
// The reference-shaped engine in double on its own buffers; vertices are the solver's
// FP64 vertices.  S[2] holds the current state in the reference layout.
struct F64Engine {
  int M = 0, N = 0;
  ex::ConstsR<double> c{};
  ex::V4<double>* S[3] = {nullptr, nullptr, nullptr};
  ex::V4<double>*fx = nullptr, *fy = nullptr, *res = nullptr, *flen = nullptr;
  double* area = nullptr;
  unsigned long long* wave = nullptr;  // max wave speed, double bits
  double* dt = nullptr;
  ~F64Engine();
  cudaError_t allocate(int M, int N);
  void metrics(const double2* Vd, cudaStream_t s);
  void from_f32(const float4* ref, cudaStream_t s);  // a float reference-layout state -> S[2]
  void to_f32(float4* ref, const double2* Vd, cudaStream_t s);
  void fill(double rho, double ru, double rv, double E, cudaStream_t s);
  const void* state_ref(const double2* Vd, cudaStream_t s);  // S[2] with its ghost rows, in S[0]
  void wave_speed(cudaStream_t s);
  void step(int scheme, int n, const double2* Vd, cudaStream_t s);
  void residual(int scheme, const double2* Vd, cudaStream_t s);  // dQ/dt of S[2] into res
  void sumsq_rho(double* parts, double* acc, cudaStream_t s);
  void forces(const double2* Vd, double* parts, double* acc, double* cp, double q_inf, double p_inf, cudaStream_t s);
};
// out[q] = fixed-order sum of parts[q * kMaxParts + 0 .. nb - 1], q < nq (kernels_misc.cu)
void launch_sum_parts(const double* parts, int nb, int nq, double* out, cudaStream_t s);

// ---- reference-shaped engine (kernels_reference.cu, built with -fmad=false) ----
// States use the reference layout [N+3][M] (row 0 wall ghost).
void launch_ref_metrics(const float2* V, float* area, float4* flen, int M, int N, cudaStream_t s);
void launch_ref_boundary(const float4* in, float4* out, const float2* V, const Consts& c, int M, int N,
                         cudaStream_t s);
void launch_ref_fluxes(int scheme, const float4* st, const float2* V, float4* fx, float4* fy, const Consts& c, int M,
                       int N, cudaStream_t s);
void launch_ref_residual(const float4* fx, const float4* fy, const float4* flen, const float* area, float4* res, int M,
                         int N, cudaStream_t s);
void launch_ref_rk(int stage, const float4* res, const float4* s0, const float4* s1, float4* out, const float* dt,
                   int M, int N, cudaStream_t s);
void launch_ref_wave(const float4* st, const float4* flen, const float* area, float gamma, int M, int N,
                     uint32_t* wave, cudaStream_t s);
void launch_dt(const uint32_t* wave, float* dt, float maxdt, float cfl, cudaStream_t s);

// ---- grid, layout, forces, norms (kernels_misc.cu) ----
void launch_to_ref_layout(const float4* Qint, float4* ref, const float2* V, const Consts& c, int M, int N,
                          cudaStream_t s);
void launch_from_ref_layout(const float4* ref, float4* Qint, int M, int N, cudaStream_t s);
void launch_fill(float4* Q, float4 v, size_t n, cudaStream_t s);
void launch_grid_init(float2* V, int M, int N, double first_spacing, cudaStream_t s);
void launch_grid_jacobi(const float2* src, float2* dst, int M, int N, cudaStream_t s);
// parts: 2 * kMaxParts doubles of scratch; acc gets the sums, in a fixed order.
// FP64 grid and face records (kernels_misc.cu): see k_metrics_d for the record layout.
void launch_grid_init_d(double2* V, int M, int N, double first_spacing, cudaStream_t s);
void launch_grid_multicolor_d(double2* V, int M, int N, int color, double omega, uint32_t* move, cudaStream_t s);
void launch_d2f(const double2* a, float2* b, size_t n, cudaStream_t s);
void launch_f2d(const float2* a, double2* b, size_t n, cudaStream_t s);
void launch_metrics_d(const double2* V, float4* Mi, float4* Mj, int M, int N, cudaStream_t s);
void launch_forces(const float4* row0, const double2* V, const Consts& c, int M, double* acc /*2*/, double* parts,
                   double* cp, double q_inf, double p_inf, cudaStream_t s);
void launch_sumsq_rho(const float4* R, size_t n, double* acc, double* parts, cudaStream_t s);
void launch_field(const float4* Qint, const float2* V, const Consts& c, int kind, int M, int N, float* out,
                  cudaStream_t s);

}  // namespace ausm
