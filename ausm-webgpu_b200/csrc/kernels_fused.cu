// Fused TVD-RK3 stage kernel: one launch per stage does the work of the reference's
// five dispatches (boundary ausm.js:23, j-flux + i-flux ausm.js:271/345, residual
// ausm.js:402, RK stage ausm.js:441/470/501).
//
// A CTA of 32 x 8 threads owns a TX=32 x TY=16 tile of interior cells; thread (x, y)
// owns cells (x, y) and (x, y+8) and keeps their conserved state in registers.  The
// CTA stages into shared memory
//   - primitives of the tile plus a 2-cell MUSCL halo on every side (corners
//     skipped), the periodic seam wrapped in i, and the ghost rows (wall j=-1,-2 and
//     far field j=N,N+1) computed in place from the interior,
//   - the (TX+1) x (TY+1) vertices of the tile,
// evaluates every i-face and j-face of the tile exactly once (flux x face length in
// shared memory; warp w evaluates face rows w and w+8 of each direction, warps 0 and 1
// the extra top row and right column), then per owned cell assembles the residual and
// the stage combination and stores the new conserved state as one float4.  The last
// stage-3 launch of a step(n) call also reduces the new state's CFL wave speed (block
// max, one atomicMax on the float bits, as cflReductionShaderCode ausm.js:535-581).
//
// HBM layout: interior state float4 [N][M] (row-major, no ghost rows), vertices
// float2 [N+1][M].  Algorithmic traffic per cell and stage: 16 B state in, 16 B out,
// 16 B Qn in (stages 2 and 3), 8 B vertex.
#include "ausm_internal.h"

namespace ausm {

#ifndef AUSM_FUSED_MIN_BLOCKS
#define AUSM_FUSED_MIN_BLOCKS 4  // resident CTAs per SM the register budget is sized for
#endif

namespace {
constexpr int TX = 32, TY = 16, NWX = 32, NWY = 8;
constexpr int PW = TX + 4, PH = TY + 4;

// i in [-2, M + TX + 2) -> [0, M); the last branch only runs for M < TX + 3
__device__ __forceinline__ int wrap_i(int i, int M) {
  if (i < 0) i += M;
  if (i >= M) i -= M;
  if (i >= M) i %= M;
  return i;
}

// Conserved state of tile cell (i, j) with j in [-2, N+1]: interior cells are loaded,
// ghost rows are computed from the adjacent interior row (boundary pass ausm.js:34-120,
// loadState clamp ausm.js:141 maps j = -1 and -2 to the wall ghost).
__device__ __forceinline__ float4 tile_cell(const float4* __restrict__ Qs, const float2* __restrict__ V,
                                            const Consts& c, int M, int N, int i, int j) {
  if (j >= 0 && j < N) return __ldg(&Qs[(size_t)j * M + i]);
  int r = i + 1 == M ? 0 : i + 1;
  if (j < 0) return wall_ghost<true>(__ldg(&Qs[i]), __ldg(&V[i]), __ldg(&V[r]));
  if (j <= N + 1) {
    float4 g1, g2;
    size_t vb = (size_t)N * M;
    far_ghosts<true>(__ldg(&Qs[(size_t)(N - 1) * M + i]), __ldg(&V[vb + i]), __ldg(&V[vb + r]), c, g1, g2);
    return j == N ? g1 : g2;
  }
  return make_float4(1.0f, 0.0f, 0.0f, 1.0f);  // beyond the far field: never read
}
}  // namespace

template <int SCHEME, int STAGE, bool EMIT>
__global__ void __launch_bounds__(NWX* NWY, AUSM_FUSED_MIN_BLOCKS)
    k_fused_stage(const float4* __restrict__ Qs, const float4* __restrict__ Qn, float4* __restrict__ Qo,
                  const float2* __restrict__ V, const float* __restrict__ dtp, uint32_t* __restrict__ wave,
                  const Consts c, const int M, const int N) {
  __shared__ float4 P[PH][PW];
  __shared__ float2 Vs[TY + 1][TX + 1];
  __shared__ float4 Fi[TY][TX + 1];
  __shared__ float4 Fj[TY + 1][TX];

  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int ic = wrap_i(i0 + tx, M);  // column of the owned cells (wrapped when i0+tx >= M)
  const int ja = j0 + ty, jb = j0 + ty + 8;

  // ---- stage the tile ----
  // owned cells (tile rows ty+2, ty+10, column tx+2), kept in registers
  const float4 qa = tile_cell(Qs, V, c, M, N, ic, ja);
  const float4 qb = tile_cell(Qs, V, c, M, N, ic, jb);
  // halo rows (warps 0-3: rows 0, 1, TY+2, TY+3, columns 2..TX+1) and halo columns
  // (warps 4-5: columns 0, 1, TX+2, TX+3, rows 2..TY+1)
  float4 qh = make_float4(1.0f, 0.0f, 0.0f, 1.0f);
  int hr = -1, hc = -1;
  if (ty < 4) {
    hr = ty < 2 ? ty : TY + ty;
    hc = tx + 2;
  } else if (ty < 6) {
    int k = (ty - 4) * 32 + tx;  // 0..63
    int sel = k >> 4;            // 0..3
    hc = sel < 2 ? sel : TX + sel;
    hr = 2 + (k & 15);
  }
  if (hr >= 0) qh = tile_cell(Qs, V, c, M, N, wrap_i(i0 - 2 + hc, M), j0 - 2 + hr);
  // vertices: rows ty, ty+8, ty+16 (ty = 0), columns tx and (lane 0) TX
  for (int r = ty; r <= TY; r += NWY) {
    int j = j0 + r;
    if (j <= N) {
      Vs[r][tx] = __ldg(&V[(size_t)j * M + ic]);
      if (tx == 0) Vs[r][TX] = __ldg(&V[(size_t)j * M + wrap_i(i0 + TX, M)]);
    }
  }
  P[ty + 2][tx + 2] = to_prim<true>(qa, c.gm1);
  P[ty + 10][tx + 2] = to_prim<true>(qb, c.gm1);
  if (hr >= 0) P[hr][hc] = to_prim<true>(qh, c.gm1);
  __syncthreads();

  // ---- faces: flux x length, each face once ----
  // i-faces of rows ty and ty+8 (and, on warp 1, the right column TX); j-faces of rows
  // ty and ty+8 (and, on warp 0, the top row TY).  Strides are compile-time.
  {
    const int nI = ty == 1 && tx < TY ? 3 : 2;
    for (int t = 0; t < nI; t++) {
      const int r = t < 2 ? ty + 8 * t : tx;
      const int cc = t < 2 ? tx : TX;
      if (j0 + r < N && cc <= M - i0) {
        float nx, ny, len;
        edge_normal<true>(Vs[r + 1][cc], Vs[r][cc], nx, ny, len);  // tangent V(i,j+1)-V(i,j)
        const float4* b = &P[r + 2][cc];
        float4 f = face_flux<SCHEME, true>(b[0], b[1], b[2], b[3], nx, ny, c);
        Fi[r][cc] = make_float4(f.x * len, f.y * len, f.z * len, f.w * len);
      }
    }
    const int nJ = ty == 0 ? 3 : 2;
    for (int t = 0; t < nJ; t++) {
      const int r = t < 2 ? ty + 8 * t : TY;
      const int cc = tx;
      if (j0 + r <= N && i0 + cc < M) {
        float nx, ny, len;
        edge_normal<true>(Vs[r][cc], Vs[r][cc + 1], nx, ny, len);  // tangent V(i,j)-V(i+1,j)
        const float4* b = &P[r][cc + 2];
        float4 f = face_flux<SCHEME, true>(b[0], b[PW], b[2 * PW], b[3 * PW], nx, ny, c);
        Fj[r][cc] = make_float4(f.x * len, f.y * len, f.z * len, f.w * len);
      }
    }
  }
  __syncthreads();

  // ---- residual + stage combination for the owned cells ----
  const float dt = *dtp;
  uint32_t wmax = 0u;
  const int i = i0 + tx;
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int r = ty + 8 * h;
    const int j = j0 + r;
    if (i < M && j < N) {
      const float4 q = h ? qb : qa;
      float2 a = Vs[r][tx], b = Vs[r][tx + 1], cv = Vs[r + 1][tx], d = Vs[r + 1][tx + 1];
      float iA = frcp<true>(quad_area(a, b, cv, d));
      float4 fl = Fi[r][tx], fr = Fi[r][tx + 1], fd = Fj[r][tx], fu = Fj[r + 1][tx];
      float4 R;
      R.x = -(((fr.x - fl.x) + fu.x) - fd.x) * iA;
      R.y = -(((fr.y - fl.y) + fu.y) - fd.y) * iA;
      R.z = -(((fr.z - fl.z) + fu.z) - fd.z) * iA;
      R.w = -(((fr.w - fl.w) + fu.w) - fd.w) * iA;
      size_t o = (size_t)j * M + i;
      float4 out;
      if constexpr (STAGE == 0) {  // residual only (dQ/dt)
        out = R;
      } else if constexpr (STAGE == 1) {
        out = make_float4(q.x + dt * R.x, q.y + dt * R.y, q.z + dt * R.z, q.w + dt * R.w);
      } else if constexpr (STAGE == 2) {
        float4 n = __ldg(&Qn[o]);
        out = make_float4(0.75f * n.x + 0.25f * (q.x + dt * R.x), 0.75f * n.y + 0.25f * (q.y + dt * R.y),
                          0.75f * n.z + 0.25f * (q.z + dt * R.z), 0.75f * n.w + 0.25f * (q.w + dt * R.w));
      } else {
        float4 n = __ldg(&Qn[o]);
        const float third = 1.0f / 3.0f;
        out = make_float4((n.x + 2.0f * (q.x + dt * R.x)) * third, (n.y + 2.0f * (q.y + dt * R.y)) * third,
                          (n.z + 2.0f * (q.z + dt * R.z)) * third, (n.w + 2.0f * (q.w + dt * R.w)) * third);
      }
      Qo[o] = out;
      if constexpr (EMIT) {
        float ll = sqrtf((a.x - cv.x) * (a.x - cv.x) + (a.y - cv.y) * (a.y - cv.y));
        float lr = sqrtf((b.x - d.x) * (b.x - d.x) + (b.y - d.y) * (b.y - d.y));
        float lu = sqrtf((cv.x - d.x) * (cv.x - d.x) + (cv.y - d.y) * (cv.y - d.y));
        float ld = sqrtf((a.x - b.x) * (a.x - b.x) + (a.y - b.y) * (a.y - b.y));
        float w = wave_speed<true>(out, ((ll + lr) + lu) + ld, quad_area(a, b, cv, d), c.gamma);
        wmax = max(wmax, __float_as_uint(w));
      }
    }
  }
  if constexpr (EMIT) block_max_to(wave, wmax);
}

// ---- launchers ----
namespace {
template <int S, int ST, bool E>
void launch_t(const float4* Qs, const float4* Qn, float4* Qo, const float2* V, const float* dt, uint32_t* wave,
              const Consts& c, int M, int N, cudaStream_t s) {
  dim3 grid((M + TX - 1) / TX, (N + TY - 1) / TY);
  k_fused_stage<S, ST, E><<<grid, dim3(NWX, NWY), 0, s>>>(Qs, Qn, Qo, V, dt, wave, c, M, N);
}
template <int S>
void launch_s(int stage, bool emit, const float4* Qs, const float4* Qn, float4* Qo, const float2* V,
              const float* dt, uint32_t* wave, const Consts& c, int M, int N, cudaStream_t s) {
  switch (stage) {
    case 0: launch_t<S, 0, false>(Qs, Qn, Qo, V, dt, wave, c, M, N, s); break;
    case 1: launch_t<S, 1, false>(Qs, Qn, Qo, V, dt, wave, c, M, N, s); break;
    case 2: launch_t<S, 2, false>(Qs, Qn, Qo, V, dt, wave, c, M, N, s); break;
    default:
      if (emit) launch_t<S, 3, true>(Qs, Qn, Qo, V, dt, wave, c, M, N, s);
      else launch_t<S, 3, false>(Qs, Qn, Qo, V, dt, wave, c, M, N, s);
  }
}
}  // namespace

void launch_fused_stage(int scheme, int stage, bool emit, const float4* Qs, const float4* Qn, float4* Qo,
                        const float2* V, const float* dt, uint32_t* wave, const Consts& c, int M, int N,
                        cudaStream_t s) {
  switch (scheme) {
    case 0: launch_s<0>(stage, emit, Qs, Qn, Qo, V, dt, wave, c, M, N, s); break;
    case 1: launch_s<1>(stage, emit, Qs, Qn, Qo, V, dt, wave, c, M, N, s); break;
    default: launch_s<2>(stage, emit, Qs, Qn, Qo, V, dt, wave, c, M, N, s); break;
  }
}

// Wave speed + max of an interior state with metrics recomputed from the vertices
// (seeds dt after init_state / set_state, main.js:649-652).
__global__ void k_wave_interior(const float4* __restrict__ Q, const float2* __restrict__ V, float gamma, int M, int N,
                                uint32_t* wave) {
  uint32_t wm = 0u;
  size_t total = (size_t)M * N;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
    int j = (int)(k / M), i = (int)(k - (size_t)j * M);
    int r = (i + 1) % M;
    float2 a = V[(size_t)j * M + i], b = V[(size_t)j * M + r], cv = V[(size_t)(j + 1) * M + i],
           d = V[(size_t)(j + 1) * M + r];
    float ll = sqrtf((a.x - cv.x) * (a.x - cv.x) + (a.y - cv.y) * (a.y - cv.y));
    float lr = sqrtf((b.x - d.x) * (b.x - d.x) + (b.y - d.y) * (b.y - d.y));
    float lu = sqrtf((cv.x - d.x) * (cv.x - d.x) + (cv.y - d.y) * (cv.y - d.y));
    float ld = sqrtf((a.x - b.x) * (a.x - b.x) + (a.y - b.y) * (a.y - b.y));
    float w = wave_speed<false>(Q[k], ((ll + lr) + lu) + ld, quad_area(a, b, cv, d), gamma);
    wm = max(wm, __float_as_uint(w));
  }
  block_max_to(wave, wm);
}

void launch_wave_interior(const float4* Q, const float2* V, float gamma, int M, int N, uint32_t* wave,
                          cudaStream_t s) {
  int blocks = (int)std::min<size_t>(((size_t)M * N + 255) / 256, 148 * 8);
  k_wave_interior<<<blocks, 256, 0, s>>>(Q, V, gamma, M, N, wave);
}

}  // namespace ausm
