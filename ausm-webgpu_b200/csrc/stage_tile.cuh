// Tile compute shared by the single-solve and batched stage kernels: tile geometry,
// staging of a tile's cells (interior loads, seam wrap, ghost rows), the face phase
// (flux x length of every face of the tile, each once) and the combine phase (residual
// and RK stage combination of the two cells a thread owns).
//
// A tile is TX = 32 cells wide (one warp per tile row) and TY = 8, 16 or 32 cells high,
// handled by 32 x TY/2 threads; thread (tx, ty) owns cells (tx, ty) and (tx, ty + TY/2).
// The tile height is a template parameter chosen per solve (or batch) by the autotuner.
//
// Geometry comes from the FP64-computed face records (k_metrics_d): Mi[j][i] =
// (nx, ny, len/2, 1/A) of the face left of cell (i, j), Mj[j][i] = (nx, ny, len/2, W)
// of the face below it, W the cell's wave-speed factor.  A tile stages the records of its
// faces in shared memory (Ti: TY rows x 33 faces, Tj: TY+1 rows x 32 faces); the face
// phase reads a face's record and overwrites it with that face's flux x length, so the
// flux tiles share that memory.  Each face is read and written by one thread only, and
// the thread that owns a cell computes that cell's left and lower faces, so it keeps
// the cell's 1/A and W in registers (FaceW) before the records are overwritten.
#pragma once
#include "ausm_internal.h"

namespace ausm {
namespace tile {
constexpr int TX = 32, NWX = 32;

template <int TY> struct Geo {
  static_assert(TY == 8 || TY == 16 || TY == 32, "tile height");
  static constexpr int NWY = TY / 2;           // warps (= tile rows per owned-cell row)
  static constexpr int NT = NWX * NWY;         // threads
  static constexpr int PW = TX + 4, PH = TY + 4;  // primitive tile with its 2-cell halo
  static constexpr int HALO = 4 * TX + 4 * TY;    // halo entries (corners unused)
  // CTAs per SM the register budget is sized for: 64 registers per thread, except 9
  // CTAs (56 registers) for 8-row tiles, which measured slightly faster than 8
  static constexpr int MIN_BLOCKS = TY == 8 ? 9 : 1024 / NT;
};

// i in [-2, M + TX + 2) -> [0, M); the last branch only runs for M < TX + 3
__device__ __forceinline__ int wrap_i(int i, int M) {
  if (i < 0) i += M;
  if (i >= M) i -= M;
  if (i >= M) i %= M;
  return i;
}

// Conserved state of tile cell (i, j) with j in [-2, N+1]: interior cells are loaded,
// ghost rows are computed from the adjacent interior row and the wall / outer face
// normal (boundary pass ausm.js:34-120, loadState clamp ausm.js:141 maps j = -1 and -2
// to the wall ghost).
__device__ __forceinline__ float4 tile_cell(const float4* __restrict__ Qs, const float4* __restrict__ Mj,
                                            const Consts& c, int M, int N, int i, int j) {
  if (j >= 0 && j < N) return __ldg(&Qs[(size_t)j * M + i]);
  if (j < 0) {
    const float4 f = __ldg(&Mj[i]);
    return wall_ghost_n<true>(__ldg(&Qs[i]), f.x, f.y);
  }
  if (j <= N + 1) {
    const float4 f = __ldg(&Mj[(size_t)N * M + i]);
    float4 g1, g2;
    far_ghosts_n<true>(__ldg(&Qs[(size_t)(N - 1) * M + i]), f.x, f.y, c, g1, g2);
    return j == N ? g1 : g2;
  }
  return make_float4(1.0f, 0.0f, 0.0f, 1.0f);  // beyond the far field: never read by a valid face
}

// Halo entry k of the primitive tile (k < HALO): first the rows 0, 1, TY+2, TY+3
// (columns 2..TX+1), then the columns 0, 1, TX+2, TX+3 (rows 2..TY+1).
template <int TY> __device__ __forceinline__ void halo_entry(int k, int& hr, int& hc) {
  if (k < 4 * TX) {
    const int r = k / TX;
    hr = r < 2 ? r : TY + r;
    hc = 2 + k % TX;
  } else {
    const int k2 = k - 4 * TX, sel = k2 / TY;
    hc = sel < 2 ? sel : TX + sel;
    hr = 2 + k2 % TY;
  }
}

// Face records of the tile from global memory (per-thread loads; the TMA kernels load
// the same boxes with the tensor engine).  Ti[r][cc] = Mi[j0+r][i0+cc] (cc = TX wraps
// through the seam), Tj[r][cc] = Mj[j0+r][i0+cc]; rows past the grid are left unset.
template <int TY>
__device__ __forceinline__ void stage_faces(const float4* __restrict__ Mi, const float4* __restrict__ Mj,
                                            float4 (*Ti)[TX + 1], float4 (*Tj)[TX], int i0, int j0, int ic, int M,
                                            int N, int tx, int ty) {
  constexpr int NWY = Geo<TY>::NWY;
#pragma unroll
  for (int r = ty; r < TY; r += NWY) {
    const int j = j0 + r;
    if (j < N) {
      Ti[r][tx] = __ldg(&Mi[(size_t)j * M + ic]);
      if (tx == 0) Ti[r][TX] = __ldg(&Mi[(size_t)j * M + wrap_i(i0 + TX, M)]);
    }
  }
  for (int r = ty; r <= TY; r += NWY) {
    const int j = j0 + r;
    if (j <= N) Tj[r][tx] = __ldg(&Mj[(size_t)j * M + ic]);
  }
}

// 1/A and wave-speed factor of the two owned cells, read before the face phase
// overwrites the records
struct FaceW {
  float iA[2], W[2];
};
template <int TY>
__device__ __forceinline__ FaceW own_weights(const float4 (*Ti)[TX + 1], const float4 (*Tj)[TX], int tx, int ty) {
  constexpr int NWY = Geo<TY>::NWY;
  FaceW w;
  w.iA[0] = Ti[ty][tx].w;
  w.iA[1] = Ti[ty + NWY][tx].w;
  w.W[0] = Tj[ty][tx].w;
  w.W[1] = Tj[ty + NWY][tx].w;
  return w;
}

// Flux x length of every face of the tile, written over the face's record.  Face rows
// ty and ty + TY/2 of each direction per thread; warp 1 also takes the right face
// column (rows 0..TY-1), warp 0 the top face row.  INNER: the tile with its halo lies
// inside the grid away from the seam, so every face exists and no bound is tested.
template <int SCHEME, int TY, bool INNER = false>
__device__ __forceinline__ void faces_phase(const float4 (*P)[TX + 4], float4 (*Ti)[TX + 1], float4 (*Tj)[TX],
                                            const Consts& c, int i0, int j0, int M, int N, int tx, int ty) {
  constexpr int NWY = Geo<TY>::NWY, PW = Geo<TY>::PW;
  auto iface = [&](int r, int cc) {
    if (INNER || (j0 + r < N && cc <= M - i0)) {
      const float4 m = Ti[r][cc];
      const float4* b = &P[r + 2][cc];
      Ti[r][cc] = face_flux_len<SCHEME>(b[0], b[1], b[2], b[3], m.x, m.y, m.z, c);
    }
  };
  auto jface = [&](int r, int cc) {
    if (INNER || (j0 + r <= N && i0 + cc < M)) {
      const float4 m = Tj[r][cc];
      const float4* b = &P[r][cc + 2];
      Tj[r][cc] = face_flux_len<SCHEME>(b[0], b[PW], b[2 * PW], b[3 * PW], m.x, m.y, m.z, c);
    }
  };
#pragma unroll
  for (int t = 0; t < 2; t++) iface(ty + NWY * t, tx);
  if (ty == 1 && tx < TY) iface(tx, TX);
#pragma unroll
  for (int t = 0; t < 2; t++) jface(ty + NWY * t, tx);
  if (ty == 0) jface(TY, tx);
}

// x / 3 correctly rounded (in all but rare halfway cases), as the reference's division:
// q = x * fl(1/3), then the exact remainder x - 3 q and one correction.  A plain product
// with fl(1/3) = 1/3 (1 + 3e-8) would scale the whole state by that factor every step,
// a bias that compounds over thousands of steps.
__device__ __forceinline__ float2 div3(float2 x) {
  const float2 t = make_float2(1.0f / 3.0f, 1.0f / 3.0f), m3 = make_float2(-3.0f, -3.0f);
  const float2 q = mul2(x, t);
  return fma2(fma2(m3, q, x), t, q);
}

// Residual and stage combination of the two owned cells from the face fluxes Fi (over
// Ti) and Fj (over Tj); returns the max wave-speed bits of the new state when EMIT.
// qn(h) fetches Qn of owned cell h (stages 2, 3).
template <int STAGE, bool EMIT, int TY, bool INNER = false, class QnFetch>
__device__ __forceinline__ uint32_t combine_phase(const float4 (*Fi)[TX + 1], const float4 (*Fj)[TX], const FaceW& w,
                                                  float4 qa, float4 qb, QnFetch qn, float4* __restrict__ Qo, float dt,
                                                  const Consts& c, int i0, int j0, int M, int N, int tx, int ty) {
  constexpr int NWY = Geo<TY>::NWY;
  uint32_t wmax = 0u;
  const int i = i0 + tx;
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int r = ty + NWY * h;
    const int j = j0 + r;
    if (INNER || (i < M && j < N)) {
      const float4 q = h ? qb : qa;
      const float2 niA = make_float2(-w.iA[h], -w.iA[h]), m1 = make_float2(-1.0f, -1.0f);
      const float4 fl = Fi[r][tx], fr = Fi[r][tx + 1], fd = Fj[r][tx], fu = Fj[r + 1][tx];
      // R = -(((fr - fl) + fu) - fd) / A, two components per f32x2 operation
      const float2 R01 = mul2(fma2(lo2(fd), m1, add2(fma2(lo2(fl), m1, lo2(fr)), lo2(fu))), niA);
      const float2 R23 = mul2(fma2(hi2(fd), m1, add2(fma2(hi2(fl), m1, hi2(fr)), hi2(fu))), niA);
      const float2 dt2 = make_float2(dt, dt);
      float2 o01, o23;
      if constexpr (STAGE == 0) {  // residual only (dQ/dt)
        o01 = R01;
        o23 = R23;
      } else if constexpr (STAGE == 1) {
        o01 = fma2(dt2, R01, lo2(q));
        o23 = fma2(dt2, R23, hi2(q));
      } else if constexpr (STAGE == 2) {
        const float4 n = qn(h);
        const float2 c25 = make_float2(0.25f, 0.25f), c75 = make_float2(0.75f, 0.75f);
        o01 = fma2(c75, lo2(n), mul2(c25, fma2(dt2, R01, lo2(q))));
        o23 = fma2(c75, hi2(n), mul2(c25, fma2(dt2, R23, hi2(q))));
      } else {
        const float4 n = qn(h);
        const float2 two = make_float2(2.0f, 2.0f);
        o01 = div3(fma2(two, fma2(dt2, R01, lo2(q)), lo2(n)));
        o23 = div3(fma2(two, fma2(dt2, R23, hi2(q)), hi2(n)));
      }
      const float4 out = make_float4(o01.x, o01.y, o23.x, o23.y);
      Qo[(size_t)j * M + i] = out;
      if constexpr (EMIT) wmax = max(wmax, __float_as_uint(wave_speed_w<true>(out, w.W[h], c.gamma)));
    }
  }
  return wmax;
}

// Per-thread staging of a whole tile (the kernels without TMA): the owned cells and the
// halo into P (as primitives), the face records into Ti / Tj.  Returns the owned
// conserved states.
template <int TY>
__device__ __forceinline__ void stage_tile_ldg(const float4* __restrict__ Qs, const float4* __restrict__ Mi,
                                               const float4* __restrict__ Mj, const Consts& c, float4 (*P)[TX + 4],
                                               float4 (*Ti)[TX + 1], float4 (*Tj)[TX], int i0, int j0, int M, int N,
                                               int tx, int ty, float4& qa, float4& qb) {
  constexpr int NWY = Geo<TY>::NWY, NT = Geo<TY>::NT, HALO = Geo<TY>::HALO;
  const int ic = wrap_i(i0 + tx, M);
  qa = tile_cell(Qs, Mj, c, M, N, ic, j0 + ty);
  qb = tile_cell(Qs, Mj, c, M, N, ic, j0 + ty + NWY);
  const int tid = ty * NWX + tx;
  float4 qh[(HALO + NT - 1) / NT];
#pragma unroll
  for (int e = 0; e < (HALO + NT - 1) / NT; e++) {
    const int k = tid + e * NT;
    if (k < HALO) {
      int hr, hc;
      halo_entry<TY>(k, hr, hc);
      qh[e] = tile_cell(Qs, Mj, c, M, N, wrap_i(i0 - 2 + hc, M), j0 - 2 + hr);
    }
  }
  stage_faces<TY>(Mi, Mj, Ti, Tj, i0, j0, ic, M, N, tx, ty);
  P[ty + 2][tx + 2] = to_prim<true>(qa, c.gm1);
  P[ty + NWY + 2][tx + 2] = to_prim<true>(qb, c.gm1);
#pragma unroll
  for (int e = 0; e < (HALO + NT - 1) / NT; e++) {
    const int k = tid + e * NT;
    if (k < HALO) {
      int hr, hc;
      halo_entry<TY>(k, hr, hc);
      P[hr][hc] = to_prim<true>(qh[e], c.gm1);
    }
  }
}
}  // namespace tile
}  // namespace ausm
