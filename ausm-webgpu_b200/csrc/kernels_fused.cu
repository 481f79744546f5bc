// Fused TVD-RK3 stage kernels: one launch per stage does the work of the reference's
// five dispatches (boundary ausm.js:23, j-flux + i-flux ausm.js:271/345, residual
// ausm.js:402, RK stage ausm.js:441/470/501).
//
// Work decomposition: a CTA of 32 x TY/2 threads handles a 32 x TY tile of interior
// cells (TY = 8, 16 or 32, stage_tile.cuh); thread (x, y) owns cells (x, y) and
// (x, y + TY/2) and keeps their conserved state in registers.  Per tile, shared memory
// holds
//   - P: primitives of the tile plus a 2-cell MUSCL halo on every side (corners
//     unused), with the periodic seam wrapped in i and the ghost rows (wall j=-1,-2,
//     far field j=N,N+1) computed from the interior,
//   - Ti/Tj: the FP64-computed face records of the tile's 33 x TY i-faces and
//     32 x (TY+1) j-faces (normal, half length, 1/A or the wave-speed factor),
//     overwritten by the flux x length of each face, evaluated once,
// and each thread then assembles the residual and the stage combination of its two
// cells and stores the new conserved states as float4.  The last stage-3 launch of a
// step(n) call also reduces the new state's CFL wave speed (block max, one atomicMax
// on the float bits, as cflReductionShaderCode ausm.js:535-581); the first step's
// stage 1 turns it into dt.
//
// k_fused_tile_tma stages its tile with TMA (cp.async.bulk.tensor, each CTA its own boxes;
// tile_tma.cuh), one tile per CTA, launched with programmatic dependent launch.
// k_fused_stage loads 32 x 16 tiles with per-thread loads: it evaluates the residual
// alone (stage 0) and steps a solve whose tensor maps could not be encoded.  Every
// mbarrier wait is bounded; on a timeout the CTA sets *err and stops.
//
// HBM layout: interior state float4 [N][M] (row-major, no ghost rows), face records
// float4 Mi [N][M] and Mj [N+1][M].  Traffic per cell and stage: 16 B state in, 16 B
// out, 16 B Qn in (stages 2 and 3), 32 B of face records.
#include "ausm_internal.h"
#include "stage_tile.cuh"
#include "tile_tma.cuh"

namespace ausm {

#ifndef AUSM_FUSED_MIN_BLOCKS
#define AUSM_FUSED_MIN_BLOCKS 4  // resident CTAs per SM the register budget is sized for
#endif

using namespace tile;

// tile height of the per-thread kernel
constexpr int TYD = 16;
using GD = Geo<TYD>;

// ---- per-thread staging, one tile per CTA (the residual, and solves without tensor maps) ----
template <int SCHEME, int STAGE, bool EMIT>
__global__ void __launch_bounds__(GD::NT, AUSM_FUSED_MIN_BLOCKS)
    k_fused_stage(const float4* __restrict__ Qs, const float4* __restrict__ Qn, float4* __restrict__ Qo,
                  const float4* __restrict__ Mi, const float4* __restrict__ Mj, const float* __restrict__ dtp,
                  uint32_t* __restrict__ wave, const Consts c, const int M, const int N) {
  __shared__ float4 P[GD::PH][GD::PW];
  __shared__ float4 Ti[TYD][TX + 1];
  __shared__ float4 Tj[TYD + 1][TX];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TYD;
  float4 qa, qb;
  stage_tile_ldg<TYD>(Qs, Mi, Mj, c, P, Ti, Tj, i0, j0, M, N, tx, ty, qa, qb);
  __syncthreads();
  const FaceW w = own_weights<TYD>(Ti, Tj, tx, ty);
  faces_phase<SCHEME, TYD>(P, Ti, Tj, c, i0, j0, M, N, tx, ty);
  __syncthreads();
  auto qn = [&](int h) { return __ldg(&Qn[(size_t)(j0 + ty + GD::NWY * h) * M + i0 + tx]); };
  uint32_t wmax = combine_phase<STAGE, EMIT, TYD>(Ti, Tj, w, qa, qb, qn, Qo, *dtp, c, i0, j0, M, N, tx, ty);
  if constexpr (EMIT) block_max_to(wave, wmax);
}

// ---- TMA-staged, one tile per CTA (the default; TY chosen by the autotuner) ----
template <int SCHEME, int STAGE, bool EMIT, int TY>
__global__ void __launch_bounds__(Geo<TY>::NT, Geo<TY>::MIN_BLOCKS)
    k_fused_tile_tma(const __grid_constant__ TmaMapsLaunch tm, const float4* __restrict__ Qs,
                     float4* __restrict__ Qo, const float4* __restrict__ Mi, const float4* __restrict__ Mj,
                     float* __restrict__ dtp, uint32_t* __restrict__ wave, const int dt_mode, int* __restrict__ err,
                     const Consts c, const int M, const int N) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  uint32_t wmax = 0u;
  if (!tile_tma_body<SCHEME, STAGE, EMIT, TY>(smem, &tm.qs, &tm.qn, &tm.mi, &tm.mj, &tm.wrap, Qs, Qo, Mi, Mj, dtp, wave,
                                              dt_mode, c, M, N, blockIdx.x * TX, blockIdx.y * TY, err, wmax))
    return;
  if constexpr (EMIT) block_max_to(wave, wmax);
}

// ---- launchers ----
namespace {
template <int S, int ST, bool E, int TY>
void launch_tile(const float4* Qs, float4* Qo, const float4* Mi, const float4* Mj, float* dt, uint32_t* wave,
                 int dt_mode, const Consts& c, int M, int N, const TmaMapsLaunch* tm, int* err, cudaStream_t s) {
  auto kern = k_fused_tile_tma<S, ST, E, TY>;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, T1<TY>::SMEM);
    attr = true;
  }
  const dim3 grid((M + TX - 1) / TX, (N + TY - 1) / TY);
  launch_pdl(kern, grid, dim3(NWX, Geo<TY>::NWY), T1<TY>::SMEM, s, *tm, Qs, Qo, Mi, Mj, dt, wave, dt_mode, err, c, M,
             N);
}

template <int S, int ST, bool E>
void launch_t(const float4* Qs, const float4* Qn, float4* Qo, const float4* Mi, const float4* Mj, float* dt,
              uint32_t* wave, int dt_mode, const Consts& c, int M, int N, const TmaMapsLaunch* tm, int ty, int* err,
              cudaStream_t s) {
  if constexpr (ST != 0) {
    if (tm) {
      if (ty == 8) launch_tile<S, ST, E, 8>(Qs, Qo, Mi, Mj, dt, wave, dt_mode, c, M, N, tm, err, s);
      else if (ty == 32) launch_tile<S, ST, E, 32>(Qs, Qo, Mi, Mj, dt, wave, dt_mode, c, M, N, tm, err, s);
      else launch_tile<S, ST, E, 16>(Qs, Qo, Mi, Mj, dt, wave, dt_mode, c, M, N, tm, err, s);
      return;
    }
  }
  const int tilesX = (M + TX - 1) / TX, tilesY = (N + TYD - 1) / TYD;
  k_fused_stage<S, ST, E><<<dim3(tilesX, tilesY), dim3(NWX, GD::NWY), 0, s>>>(Qs, Qn, Qo, Mi, Mj, dt, wave, c, M, N);
}
template <int S>
void launch_s(int stage, bool emit, const float4* Qs, const float4* Qn, float4* Qo, const float4* Mi,
              const float4* Mj, float* dt, uint32_t* wave, int dt_mode, const Consts& c, int M, int N,
              const TmaMapsLaunch* tm, int ty, int* err, cudaStream_t s) {
  switch (stage) {
    case 0: launch_t<S, 0, false>(Qs, Qn, Qo, Mi, Mj, dt, wave, dt_mode, c, M, N, tm, ty, err, s); break;
    case 1: launch_t<S, 1, false>(Qs, Qn, Qo, Mi, Mj, dt, wave, dt_mode, c, M, N, tm, ty, err, s); break;
    case 2: launch_t<S, 2, false>(Qs, Qn, Qo, Mi, Mj, dt, wave, dt_mode, c, M, N, tm, ty, err, s); break;
    default:
      if (emit) launch_t<S, 3, true>(Qs, Qn, Qo, Mi, Mj, dt, wave, dt_mode, c, M, N, tm, ty, err, s);
      else launch_t<S, 3, false>(Qs, Qn, Qo, Mi, Mj, dt, wave, dt_mode, c, M, N, tm, ty, err, s);
  }
}
}  // namespace

void launch_fused_stage(int scheme, int stage, bool emit, const float4* Qs, const float4* Qn, float4* Qo,
                        const float4* Mi, const float4* Mj, float* dt, uint32_t* wave, int dt_mode, const Consts& c,
                        int M, int N, const TmaMapsLaunch* tm, int ty, int* err, cudaStream_t s) {
  if (dt_mode != 0 && !(tm && stage != 0)) {  // kernels without the in-kernel time step
    if (dt_mode == 1) launch_dt(wave, dt, c.maxdt, c.cfl, s);
    else cudaMemsetAsync(wave, 0, sizeof(uint32_t), s);
    dt_mode = 0;
  }
  // TMA stage kernels with MUSCL on are instantiated with it known (scheme + 4)
  const int sf = scheme + (c.muscl > 0 && tm && stage != 0 ? 4 : 0);
  switch (sf) {
    case 0: launch_s<0>(stage, emit, Qs, Qn, Qo, Mi, Mj, dt, wave, dt_mode, c, M, N, tm, ty, err, s); break;
    case 1: launch_s<1>(stage, emit, Qs, Qn, Qo, Mi, Mj, dt, wave, dt_mode, c, M, N, tm, ty, err, s); break;
    case 2: launch_s<2>(stage, emit, Qs, Qn, Qo, Mi, Mj, dt, wave, dt_mode, c, M, N, tm, ty, err, s); break;
    case 4: launch_s<4>(stage, emit, Qs, Qn, Qo, Mi, Mj, dt, wave, dt_mode, c, M, N, tm, ty, err, s); break;
    case 5: launch_s<5>(stage, emit, Qs, Qn, Qo, Mi, Mj, dt, wave, dt_mode, c, M, N, tm, ty, err, s); break;
    default: launch_s<6>(stage, emit, Qs, Qn, Qo, Mi, Mj, dt, wave, dt_mode, c, M, N, tm, ty, err, s); break;
  }
}

// Polls of the TMA stage kernels' first bounded waits (tma.cuh c_wait_polls).
cudaError_t set_wait_polls_fused(unsigned polls) { return cudaMemcpyToSymbol(c_wait_polls, &polls, sizeof polls); }

// Tensor maps of the TMA kernels for tile height ty: state buffers as 2-D float tensors
// of 4M x N (row pitch 16 M bytes) with the halo box 144 x (ty+4) and the Qn box
// 128 x ty and the seam box 8 x (ty+4); face records Mi as 4M x N with the box
// 132 x ty, Mj as 4M x (N+1) with the box 128 x (ty+1).  Every box's row is a multiple
// of 16 bytes and every x coordinate a multiple of 4 floats (16 bytes).
bool encode_tma_maps(const float4* const Q[3], const float4* Mi, const float4* Mj, int M, int N, int ty,
                     TmaMaps* out) {
  out->ok = false;
  using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static Encode encode = nullptr;
  if (!encode) {
    cudaDriverEntryPointQueryResult q;
    void* fn = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return false;
    encode = reinterpret_cast<Encode>(fn);
  }
  const cuuint32_t estr[2] = {1, 1};
  auto enc = [&](CUtensorMap* m, const void* ptr, cuuint64_t w, cuuint64_t h, cuuint64_t pitch, cuuint32_t bw,
                 cuuint32_t bh) {
    const cuuint64_t dims[2] = {w, h};
    const cuuint64_t strides[1] = {pitch};
    const cuuint32_t box[2] = {bw, bh};
    return encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(ptr), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  };
  const cuuint32_t bty = (cuuint32_t)ty;
  for (int b = 0; b < 3; b++) {
    if (!enc(&out->halo[b], Q[b], 4ull * M, N, 16ull * M, 4 * (TX + 4), bty + 4)) return false;
    if (!enc(&out->plain[b], Q[b], 4ull * M, N, 16ull * M, 4 * TX, bty)) return false;
  }
  for (int b = 0; b < 3; b++)
    if (!enc(&out->wrap[b], Q[b], 4ull * M, N, 16ull * M, 8, bty + 4)) return false;
  if (!enc(&out->mi, Mi, 4ull * M, N, 16ull * M, 4 * (TX + 1), bty)) return false;
  if (!enc(&out->mj, Mj, 4ull * M, N + 1, 16ull * M, 4 * TX, bty + 1)) return false;
  out->ok = true;
  return true;
}

// Wave speed + max of an interior state from the cells' wave-speed factors (seeds dt
// after init_state / set_state, main.js:649-652).
__global__ void k_wave_interior(const float4* __restrict__ Q, const float4* __restrict__ Mj, float gamma, int M, int N,
                                uint32_t* wave) {
  uint32_t wm = 0u;
  size_t total = (size_t)M * N;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
    float w = wave_speed_w<false>(Q[k], Mj[k].w, gamma);
    wm = max(wm, __float_as_uint(w));
  }
  block_max_to(wave, wm);
}

void launch_wave_interior(const float4* Q, const float4* Mj, float gamma, int M, int N, uint32_t* wave,
                          cudaStream_t s) {
  int blocks = (int)std::min<size_t>(((size_t)M * N + 255) / 256, 148 * 8);
  k_wave_interior<<<blocks, 256, 0, s>>>(Q, Mj, gamma, M, N, wave);
}

}  // namespace ausm
