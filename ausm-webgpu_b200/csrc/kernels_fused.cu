// Fused TVD-RK3 stage kernel: one launch per stage does the work of the reference's
// five dispatches (boundary ausm.js:23, j-flux + i-flux ausm.js:271/345, residual
// ausm.js:402, RK stage ausm.js:441/470/501).
//
// A CTA owns a TX x TY tile of interior cells.  It stages into shared memory
//   - the primitive variables of the tile plus a 2-cell MUSCL halo on every side
//     (corners skipped), with the periodic seam wrapped in i and the ghost rows
//     (wall j=-1,-2 and far field j=N,N+1) computed in place from the interior,
//   - the (TX+1) x (TY+1) vertices of the tile,
// evaluates every i-face and j-face of the tile once (flux x face length kept in
// shared memory), then per cell assembles the residual and the stage combination and
// writes the new conserved state with one float4 store.  The last stage-3 launch of a
// step(n) call also reduces the new state's CFL wave speed (block max + one atomicMax
// on the float bits, as the reference's cflReductionShaderCode ausm.js:535-581).
//
// HBM layout: interior state float4 [N][M] (row-major, no ghost rows), vertices
// float2 [N+1][M].  Algorithmic traffic per cell and stage: 16 B state in, 16 B out,
// 16 B Qn in (stages 2 and 3), 8 B vertex.
#include "ausm_internal.h"

namespace ausm {

template <int TX, int TY, int NT, int SCHEME, int STAGE, bool EMIT>
__global__ void __launch_bounds__(NT, 2)
    k_fused_stage(const float4* __restrict__ Qs, const float4* __restrict__ Qn, float4* __restrict__ Qo,
                  const float2* __restrict__ V, const float* __restrict__ dtp, uint32_t* __restrict__ wave,
                  const Consts c, const int M, const int N) {
  constexpr int PW = TX + 4, PH = TY + 4;
  constexpr int NFI = TY * (TX + 1);
  constexpr int NFI_PAD = (NFI + 31) / 32 * 32;  // j-faces start warp-aligned
  constexpr int NFJ = (TY + 1) * TX;
  __shared__ float4 P[PH][PW];
  __shared__ float2 Vs[TY + 1][TX + 1];
  __shared__ float4 Fi[TY][TX + 1];
  __shared__ float4 Fj[TY + 1][TX];

  const int tid = threadIdx.x;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;

  // ---- vertices of the tile (i wraps mod M) ----
  for (int k = tid; k < (TY + 1) * (TX + 1); k += NT) {
    int r = k / (TX + 1), cc = k - r * (TX + 1);
    int j = j0 + r;
    int i = (i0 + cc) % M;
    if (j <= N) Vs[r][cc] = V[(size_t)j * M + i];
  }
  // ---- primitives with halo and ghost rows ----
  for (int k = tid; k < PH * PW; k += NT) {
    int r = k / PW, cc = k - r * PW;
    bool rh = (r < 2) | (r >= TY + 2), ch = (cc < 2) | (cc >= TX + 2);
    if (rh & ch) continue;
    int j = j0 - 2 + r;
    int i = i0 - 2 + cc;
    i = (i % M + M) % M;
    float4 q;
    if (j >= 0 && j < N) {
      q = Qs[(size_t)j * M + i];
    } else if (j < 0) {  // wall ghost (rows -1 and -2 both map to it, ausm.js:141)
      q = wall_ghost<true>(Qs[i], V[i], V[(i + 1) % M]);
    } else if (j <= N + 1) {
      float4 g1, g2;
      size_t vb = (size_t)N * M;
      far_ghosts<true>(Qs[(size_t)(N - 1) * M + i], V[vb + i], V[vb + (i + 1) % M], c, g1, g2);
      q = (j == N) ? g1 : g2;
    } else {
      q = make_float4(1.0f, 0.0f, 0.0f, 1.0f);  // beyond the far field: never read
    }
    P[r][cc] = to_prim<true>(q, c.gm1);
  }
  __syncthreads();

  // ---- faces: flux x length ----
  for (int k = tid; k < NFI_PAD + NFJ; k += NT) {
    if (k < NFI) {
      int r = k / (TX + 1), cc = k - r * (TX + 1);
      if (j0 + r < N && cc <= M - i0) {
        float nx, ny, len;
        edge_normal<true>(Vs[r + 1][cc], Vs[r][cc], nx, ny, len);  // tangent V(i,j+1)-V(i,j)
        float4 f = face_flux<SCHEME, true>(P[r + 2][cc], P[r + 2][cc + 1], P[r + 2][cc + 2], P[r + 2][cc + 3],
                                           nx, ny, c);
        Fi[r][cc] = make_float4(f.x * len, f.y * len, f.z * len, f.w * len);
      }
    } else if (k >= NFI_PAD) {
      int kk = k - NFI_PAD;
      int r = kk / TX, cc = kk - r * TX;
      if (j0 + r <= N && i0 + cc < M) {
        float nx, ny, len;
        edge_normal<true>(Vs[r][cc], Vs[r][cc + 1], nx, ny, len);  // tangent V(i,j)-V(i+1,j)
        float4 f = face_flux<SCHEME, true>(P[r][cc + 2], P[r + 1][cc + 2], P[r + 2][cc + 2], P[r + 3][cc + 2],
                                           nx, ny, c);
        Fj[r][cc] = make_float4(f.x * len, f.y * len, f.z * len, f.w * len);
      }
    }
  }
  __syncthreads();

  // ---- residual + stage combination ----
  const float dt = *dtp;
  uint32_t wmax = 0u;
  for (int k = tid; k < TX * TY; k += NT) {
    int r = k / TX, cc = k - r * TX;
    int i = i0 + cc, j = j0 + r;
    if (i < M && j < N) {
      float2 a = Vs[r][cc], b = Vs[r][cc + 1], cv = Vs[r + 1][cc], d = Vs[r + 1][cc + 1];
      float iA = frcp<true>(quad_area(a, b, cv, d));
      float4 fl = Fi[r][cc], fr = Fi[r][cc + 1], fd = Fj[r][cc], fu = Fj[r + 1][cc];
      float4 R;
      R.x = -(((fr.x - fl.x) + fu.x) - fd.x) * iA;
      R.y = -(((fr.y - fl.y) + fu.y) - fd.y) * iA;
      R.z = -(((fr.z - fl.z) + fu.z) - fd.z) * iA;
      R.w = -(((fr.w - fl.w) + fu.w) - fd.w) * iA;
      size_t o = (size_t)j * M + i;
      float4 q = Qs[o];
      float4 out;
      if constexpr (STAGE == 0) {  // residual only (dQ/dt)
        out = R;
      } else if constexpr (STAGE == 1) {
        out = make_float4(q.x + dt * R.x, q.y + dt * R.y, q.z + dt * R.z, q.w + dt * R.w);
      } else if constexpr (STAGE == 2) {
        float4 n = Qn[o];
        out = make_float4(0.75f * n.x + 0.25f * (q.x + dt * R.x), 0.75f * n.y + 0.25f * (q.y + dt * R.y),
                          0.75f * n.z + 0.25f * (q.z + dt * R.z), 0.75f * n.w + 0.25f * (q.w + dt * R.w));
      } else {
        float4 n = Qn[o];
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
constexpr int FTX = 32, FTY = 16, FNT = 256;

template <int S, int ST, bool E>
void launch_t(const float4* Qs, const float4* Qn, float4* Qo, const float2* V, const float* dt, uint32_t* wave,
              const Consts& c, int M, int N, cudaStream_t s) {
  dim3 grid((M + FTX - 1) / FTX, (N + FTY - 1) / FTY);
  k_fused_stage<FTX, FTY, FNT, S, ST, E><<<grid, FNT, 0, s>>>(Qs, Qn, Qo, V, dt, wave, c, M, N);
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
