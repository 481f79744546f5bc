// Reference-shaped engine: the reference's five dispatches per RK stage, one CUDA
// kernel each, on the reference's buffer layout (main.js:110-125):
//   boundary  ausm.js:23-120   M x (N+3)   ghost rows + pass-through copy
//   j-flux    ausm.js:128-392  M x (N+1)   faces below each interior cell
//   i-flux    ausm.js:128-392  M x N       faces left of each interior cell (the
//                                          reference's extra column i=M is never read,
//                                          ausm.js:420, and is not computed)
//   residual  ausm.js:402-436  M x N
//   RK stage  ausm.js:441-527  M x N       interior rows only
// plus the wave-speed max reduction (ausm.js:617-630, 535-581) and the grid metrics
// (shaders/grid.js:115-147).  This translation unit is compiled with -fmad=false and
// uses the exact (FAST=false) arithmetic, so it matches the float oracle bit for bit.
// It is the plain one-launch-per-dispatch baseline of the benchmarks.
#include "ausm_internal.h"

namespace ausm {

__device__ __forceinline__ float4 ref_load(const float4* __restrict__ st, int M, int i, int j) {
  // loadState (ausm.js:138-143): i wraps, interior index + 1, clamped at the wall ghost
  int ii = (i + M) % M;
  int jj = max(j + 1, 0);
  return st[(size_t)jj * M + ii];
}

__global__ void k_ref_metrics(const float2* __restrict__ V, float* __restrict__ area, float4* __restrict__ flen,
                              int M, int N) {
  int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= M || j >= N) return;
  int r = (i + 1) % M;
  float2 a = V[(size_t)j * M + i], b = V[(size_t)j * M + r], c = V[(size_t)(j + 1) * M + i],
         d = V[(size_t)(j + 1) * M + r];
  size_t k = (size_t)j * M + i;
  area[k] = quad_area(a, b, c, d);
  float4 l;
  l.x = sqrtf((a.x - c.x) * (a.x - c.x) + (a.y - c.y) * (a.y - c.y));
  l.y = sqrtf((b.x - d.x) * (b.x - d.x) + (b.y - d.y) * (b.y - d.y));
  l.z = sqrtf((c.x - d.x) * (c.x - d.x) + (c.y - d.y) * (c.y - d.y));
  l.w = sqrtf((a.x - b.x) * (a.x - b.x) + (a.y - b.y) * (a.y - b.y));
  flen[k] = l;
}

__global__ void k_ref_boundary(const float4* __restrict__ in, float4* __restrict__ out,
                               const float2* __restrict__ V, const Consts c, int M, int N) {
  int i = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= M || y >= N + 3) return;
  int r = (i + 1) % M;
  if (y == 0) {
    out[i] = wall_ghost<false>(in[(size_t)M + i], V[i], V[r]);
  } else if (y > N) {
    float4 g1, g2;
    far_ghosts<false>(in[(size_t)N * M + i], V[(size_t)N * M + i], V[(size_t)N * M + r], c, g1, g2);
    out[(size_t)y * M + i] = (y == N + 1) ? g1 : g2;
  } else {
    out[(size_t)y * M + i] = in[(size_t)y * M + i];
  }
}

template <int SCHEME>
__global__ void k_ref_flux_j(const float4* __restrict__ st, const float2* __restrict__ V, float4* __restrict__ fy,
                             const Consts c, int M, int N) {
  int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= M || j > N) return;
  float nx, ny, len;
  edge_normal<false>(V[(size_t)j * M + i], V[(size_t)j * M + (i + 1) % M], nx, ny, len);
  const float gm1 = c.gm1;
  float4 f = face_flux<SCHEME>(to_prim<false>(ref_load(st, M, i, j - 2), gm1),
                                      to_prim<false>(ref_load(st, M, i, j - 1), gm1),
                                      to_prim<false>(ref_load(st, M, i, j), gm1),
                                      to_prim<false>(ref_load(st, M, i, j + 1), gm1), nx, ny, c);
  fy[(size_t)j * M + i] = f;
}

template <int SCHEME>
__global__ void k_ref_flux_i(const float4* __restrict__ st, const float2* __restrict__ V, float4* __restrict__ fx,
                             const Consts c, int M, int N) {
  int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= M || j >= N) return;
  float nx, ny, len;
  edge_normal<false>(V[(size_t)(j + 1) * M + i], V[(size_t)j * M + i], nx, ny, len);
  const float gm1 = c.gm1;
  float4 f = face_flux<SCHEME>(to_prim<false>(ref_load(st, M, i - 2, j), gm1),
                                      to_prim<false>(ref_load(st, M, i - 1, j), gm1),
                                      to_prim<false>(ref_load(st, M, i, j), gm1),
                                      to_prim<false>(ref_load(st, M, i + 1, j), gm1), nx, ny, c);
  fx[(size_t)j * M + i] = f;
}

__global__ void k_ref_residual(const float4* __restrict__ fx, const float4* __restrict__ fy,
                               const float4* __restrict__ flen, const float* __restrict__ area,
                               float4* __restrict__ res, int M, int N) {
  int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= M || j >= N) return;
  size_t k = (size_t)j * M + i;
  float4 xl = fx[k], xr = fx[(size_t)j * M + (i + 1) % M], yu = fy[(size_t)(j + 1) * M + i], yd = fy[k];
  float4 l = flen[k];
  float A = area[k];
  float4 R;
  R.x = -(xr.x * l.y - xl.x * l.x + yu.x * l.z - yd.x * l.w) / A;
  R.y = -(xr.y * l.y - xl.y * l.x + yu.y * l.z - yd.y * l.w) / A;
  R.z = -(xr.z * l.y - xl.z * l.x + yu.z * l.z - yd.z * l.w) / A;
  R.w = -(xr.w * l.y - xl.w * l.x + yu.w * l.z - yd.w * l.w) / A;
  res[k] = R;
}

template <int STAGE>
__global__ void k_ref_rk(const float4* __restrict__ res, const float4* __restrict__ s0, const float4* __restrict__ s1,
                         float4* __restrict__ out, const float* __restrict__ dtp, int M, int N) {
  int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= M || j >= N) return;
  const float dt = *dtp;
  size_t k = (size_t)j * M + i, o = (size_t)(j + 1) * M + i;
  float4 R = res[k], Q = s0[o], o4;
  if constexpr (STAGE == 1) {
    o4 = make_float4(Q.x + dt * R.x, Q.y + dt * R.y, Q.z + dt * R.z, Q.w + dt * R.w);
  } else if constexpr (STAGE == 2) {
    float4 Q1 = s1[o];
    o4 = make_float4(0.75f * Q.x + 0.25f * (Q1.x + dt * R.x), 0.75f * Q.y + 0.25f * (Q1.y + dt * R.y),
                     0.75f * Q.z + 0.25f * (Q1.z + dt * R.z), 0.75f * Q.w + 0.25f * (Q1.w + dt * R.w));
  } else {
    float4 Q2 = s1[o];
    o4 = make_float4((Q.x + 2.0f * (Q2.x + dt * R.x)) / 3.0f, (Q.y + 2.0f * (Q2.y + dt * R.y)) / 3.0f,
                     (Q.z + 2.0f * (Q2.z + dt * R.z)) / 3.0f, (Q.w + 2.0f * (Q2.w + dt * R.w)) / 3.0f);
  }
  out[o] = o4;
}

__global__ void k_ref_wave(const float4* __restrict__ st, const float4* __restrict__ flen,
                           const float* __restrict__ area, float gamma, int M, int N, uint32_t* wave) {
  uint32_t wm = 0u;
  size_t total = (size_t)M * N;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
    float4 l = flen[k];
    float w = wave_speed<false>(st[k + M], ((l.x + l.y) + l.z) + l.w, area[k], gamma);
    wm = max(wm, __float_as_uint(w));
  }
  block_max_to(wave, wm);
}

// dt = min(maxdt, cfl / maxWaveSpeed) (ausm.js:457)
__global__ void k_dt(const uint32_t* __restrict__ wave, float* __restrict__ dt, float maxdt, float cfl) {
  dt[0] = fminf(maxdt, cfl / __uint_as_float(wave[0]));
}

// ---- launchers ----
static inline dim3 grid16(int w, int h) { return dim3((w + 15) / 16, (h + 15) / 16); }
static const dim3 B16(16, 16);

void launch_ref_metrics(const float2* V, float* area, float4* flen, int M, int N, cudaStream_t s) {
  k_ref_metrics<<<grid16(M, N), B16, 0, s>>>(V, area, flen, M, N);
}
void launch_ref_boundary(const float4* in, float4* out, const float2* V, const Consts& c, int M, int N,
                         cudaStream_t s) {
  k_ref_boundary<<<grid16(M, N + 3), B16, 0, s>>>(in, out, V, c, M, N);
}
void launch_ref_fluxes(int scheme, const float4* st, const float2* V, float4* fx, float4* fy, const Consts& c, int M,
                       int N, cudaStream_t s) {
  switch (scheme) {
    case 0:
      k_ref_flux_j<0><<<grid16(M, N + 1), B16, 0, s>>>(st, V, fy, c, M, N);
      k_ref_flux_i<0><<<grid16(M, N), B16, 0, s>>>(st, V, fx, c, M, N);
      break;
    case 1:
      k_ref_flux_j<1><<<grid16(M, N + 1), B16, 0, s>>>(st, V, fy, c, M, N);
      k_ref_flux_i<1><<<grid16(M, N), B16, 0, s>>>(st, V, fx, c, M, N);
      break;
    default:
      k_ref_flux_j<2><<<grid16(M, N + 1), B16, 0, s>>>(st, V, fy, c, M, N);
      k_ref_flux_i<2><<<grid16(M, N), B16, 0, s>>>(st, V, fx, c, M, N);
      break;
  }
}
void launch_ref_residual(const float4* fx, const float4* fy, const float4* flen, const float* area, float4* res, int M,
                         int N, cudaStream_t s) {
  k_ref_residual<<<grid16(M, N), B16, 0, s>>>(fx, fy, flen, area, res, M, N);
}
void launch_ref_rk(int stage, const float4* res, const float4* s0, const float4* s1, float4* out, const float* dt,
                   int M, int N, cudaStream_t s) {
  if (stage == 1) k_ref_rk<1><<<grid16(M, N), B16, 0, s>>>(res, s0, s1, out, dt, M, N);
  else if (stage == 2) k_ref_rk<2><<<grid16(M, N), B16, 0, s>>>(res, s0, s1, out, dt, M, N);
  else k_ref_rk<3><<<grid16(M, N), B16, 0, s>>>(res, s0, s1, out, dt, M, N);
}
void launch_ref_wave(const float4* st, const float4* flen, const float* area, float gamma, int M, int N,
                     uint32_t* wave, cudaStream_t s) {
  int blocks = (int)std::min<size_t>(((size_t)M * N + 255) / 256, 148 * 8);
  k_ref_wave<<<blocks, 256, 0, s>>>(st, flen, area, gamma, M, N, wave);
}
void launch_dt(const uint32_t* wave, float* dt, float maxdt, float cfl, cudaStream_t s) {
  k_dt<<<1, 1, 0, s>>>(wave, dt, maxdt, cfl);
}

}  // namespace ausm
