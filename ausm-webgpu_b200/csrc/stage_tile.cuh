// Tile compute shared by the single-solve and batched stage kernels: tile geometry,
// staging of a tile's cells (interior loads, seam wrap, ghost rows), the face phase
// (flux x length of every face of the tile, each once) and the combine phase (residual
// and RK stage combination of the two cells a thread owns).  See kernels_fused.cu for
// the work decomposition.
#pragma once
#include "ausm_internal.h"

namespace ausm {
namespace tile {
constexpr int TX = 32, TY = 16, NWX = 32, NWY = 8, NT = NWX * NWY;
constexpr int PW = TX + 4, PH = TY + 4;
constexpr int VW_TMA = TX + 2;  // vertex box width: 34 x 8 B = 272 B, a multiple of 16 B

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
  return make_float4(1.0f, 0.0f, 0.0f, 1.0f);  // beyond the far field: never read by a valid face
}

// halo entry of thread (tx, ty): warps 0-3 take primitive rows 0, 1, TY+2, TY+3
// (columns 2..TX+1), warps 4-5 columns 0, 1, TX+2, TX+3 (rows 2..TY+1)
__device__ __forceinline__ void halo_entry(int tx, int ty, int& hr, int& hc) {
  hr = -1;
  hc = -1;
  if (ty < 4) {
    hr = ty < 2 ? ty : TY + ty;
    hc = tx + 2;
  } else if (ty < 6) {
    int k = (ty - 4) * 32 + tx;  // 0..63
    int sel = k >> 4;            // 0..3
    hc = sel < 2 ? sel : TX + sel;
    hr = 2 + (k & 15);
  }
}

// Flux x length of every face of the tile.  Vs is the vertex tile with row width VW.
template <int SCHEME, int VW>
__device__ __forceinline__ void faces_phase(const float4 (*P)[PW], const float2* Vs, float4 (*Fi)[TX + 1],
                                            float4 (*Fj)[TX], const Consts& c, int i0, int j0, int M, int N, int tx,
                                            int ty) {
  const int nI = ty == 1 && tx < TY ? 3 : 2;
  for (int t = 0; t < nI; t++) {
    const int r = t < 2 ? ty + 8 * t : tx;
    const int cc = t < 2 ? tx : TX;
    if (j0 + r < N && cc <= M - i0) {
      float nx, ny, len;
      edge_normal<true>(Vs[(r + 1) * VW + cc], Vs[r * VW + cc], nx, ny, len);  // tangent V(i,j+1)-V(i,j)
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
      edge_normal<true>(Vs[r * VW + cc], Vs[r * VW + cc + 1], nx, ny, len);  // tangent V(i,j)-V(i+1,j)
      const float4* b = &P[r][cc + 2];
      float4 f = face_flux<SCHEME, true>(b[0], b[PW], b[2 * PW], b[3 * PW], nx, ny, c);
      Fj[r][cc] = make_float4(f.x * len, f.y * len, f.z * len, f.w * len);
    }
  }
}

// Residual and stage combination of the two owned cells; returns the max wave-speed
// bits of the new state when EMIT.  qn(h) fetches Qn of owned cell h (stages 2, 3).
template <int STAGE, bool EMIT, int VW, class QnFetch>
__device__ __forceinline__ uint32_t combine_phase(const float2* Vs, const float4 (*Fi)[TX + 1],
                                                  const float4 (*Fj)[TX], float4 qa, float4 qb, QnFetch qn,
                                                  float4* __restrict__ Qo, float dt, const Consts& c, int i0, int j0,
                                                  int M, int N, int tx, int ty) {
  uint32_t wmax = 0u;
  const int i = i0 + tx;
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int r = ty + 8 * h;
    const int j = j0 + r;
    if (i < M && j < N) {
      const float4 q = h ? qb : qa;
      float2 a = Vs[r * VW + tx], b = Vs[r * VW + tx + 1], cv = Vs[(r + 1) * VW + tx], d = Vs[(r + 1) * VW + tx + 1];
      float A = quad_area(a, b, cv, d);
      float iA = frcp<true>(A);
      float4 fl = Fi[r][tx], fr = Fi[r][tx + 1], fd = Fj[r][tx], fu = Fj[r + 1][tx];
      float4 R;
      R.x = -(((fr.x - fl.x) + fu.x) - fd.x) * iA;
      R.y = -(((fr.y - fl.y) + fu.y) - fd.y) * iA;
      R.z = -(((fr.z - fl.z) + fu.z) - fd.z) * iA;
      R.w = -(((fr.w - fl.w) + fu.w) - fd.w) * iA;
      float4 out;
      if constexpr (STAGE == 0) {  // residual only (dQ/dt)
        out = R;
      } else if constexpr (STAGE == 1) {
        out = make_float4(q.x + dt * R.x, q.y + dt * R.y, q.z + dt * R.z, q.w + dt * R.w);
      } else if constexpr (STAGE == 2) {
        float4 n = qn(h);
        out = make_float4(0.75f * n.x + 0.25f * (q.x + dt * R.x), 0.75f * n.y + 0.25f * (q.y + dt * R.y),
                          0.75f * n.z + 0.25f * (q.z + dt * R.z), 0.75f * n.w + 0.25f * (q.w + dt * R.w));
      } else {
        float4 n = qn(h);
        const float third = 1.0f / 3.0f;
        out = make_float4((n.x + 2.0f * (q.x + dt * R.x)) * third, (n.y + 2.0f * (q.y + dt * R.y)) * third,
                          (n.z + 2.0f * (q.z + dt * R.z)) * third, (n.w + 2.0f * (q.w + dt * R.w)) * third);
      }
      Qo[(size_t)j * M + i] = out;
      if constexpr (EMIT) {
        float ll = sqrtf((a.x - cv.x) * (a.x - cv.x) + (a.y - cv.y) * (a.y - cv.y));
        float lr = sqrtf((b.x - d.x) * (b.x - d.x) + (b.y - d.y) * (b.y - d.y));
        float lu = sqrtf((cv.x - d.x) * (cv.x - d.x) + (cv.y - d.y) * (cv.y - d.y));
        float ld = sqrtf((a.x - b.x) * (a.x - b.x) + (a.y - b.y) * (a.y - b.y));
        float w = wave_speed<true>(out, ((ll + lr) + lu) + ld, A, c.gamma);
        wmax = max(wmax, __float_as_uint(w));
      }
    }
  }
  return wmax;
}
}  // namespace tile
}  // namespace ausm
