// TMA staging of one stage tile (one tile per CTA): the state box with its 2-cell halo
// (36 x (TY+4) float4), the face-record boxes (33 x TY i-faces, 32 x (TY+1) j-faces),
// for stages 2 and 3 the Qn box (32 x TY) and, for a tile at the seam, the two columns
// its halo wraps to (2 x (TY+4)) land in shared memory by cp.async.bulk.tensor copies
// (each CTA fetching its own) completing on three mbarriers; the threads then fill the ghost rows
// the boxes cannot hold and run the tile compute of stage_tile.cuh.  Used by the single-solve kernel (tensor maps as a kernel
// parameter) and the batched kernel (per-solve tensor maps in global memory, written
// by the host before the launch).
#pragma once
#include "stage_tile.cuh"
#include "tma.cuh"

namespace ausm {
namespace tile {

constexpr int r128(int x) { return (x + 127) / 128 * 128; }

// Box sizes and the dynamic shared memory layout of one tile (offsets multiples of
// 128 B from a 128-B aligned base).
template <int TY> struct T1 {
  static constexpr int SQ = (TX + 4) * (TY + 4) * 16;  // state box
  static constexpr int SI = TY * (TX + 1) * 16;        // i-face box
  static constexpr int SJ = (TY + 1) * TX * 16;        // j-face box
  static constexpr int SN = TY * TX * 16;              // Qn box
  static constexpr int SW = (TY + 4) * 2 * 16;         // seam box
  static constexpr int OFF_I = r128(SQ), OFF_J = OFF_I + r128(SI), OFF_N = OFF_J + r128(SJ);
  static constexpr int OFF_W = OFF_N + r128(SN);       // left and right seam boxes
  static constexpr int OFF_BAR = OFF_W + 2 * r128(SW);
  static constexpr int SMEM = OFF_BAR + 128 + 128;  // 3 mbarriers + alignment slack of the base
};

// The tile's loads, issued by thread 0 in two parts: first the barriers and the
// face-record boxes (barrier 1; the records never change, so this part may run before
// the previous stage has finished), then, once the previous stage's writes are
// visible (tile_tma_issue's caller waits for them), the state box and the seam boxes
// (barrier 0) and Qn (stages 2, 3; barrier 2), so each phase waits only for what it
// reads.  Seam boxes: a tile whose halo starts left of column 0 gets columns M-2, M-1
// (left box), one whose halo reaches column M gets columns 0, 1 (right box).
template <int TY>
__device__ __forceinline__ void tile_tma_issue_records(const CUtensorMap* mi, const CUtensorMap* mj,
                                                       unsigned char* smem, int i0, int j0) {
  using L = T1<TY>;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + L::OFF_BAR);
  mbar_init(&bar[0], 1);
  mbar_init(&bar[1], 1);
  mbar_init(&bar[2], 1);
  mbar_fence_init();
  mbar_expect_tx(&bar[1], L::SI + L::SJ);
  tma_load_2d(smem + L::OFF_I, mi, 4 * i0, j0, &bar[1]);
  tma_load_2d(smem + L::OFF_J, mj, 4 * i0, j0, &bar[1]);
}
template <int STAGE, int TY>
__device__ __forceinline__ void tile_tma_issue_state(const CUtensorMap* qs, const CUtensorMap* qn,
                                                     const CUtensorMap* wr, unsigned char* smem, int i0, int j0,
                                                     int M) {
  using L = T1<TY>;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + L::OFF_BAR);
  const bool wl = i0 == 0, wrr = i0 + TX + 2 > M;
  mbar_expect_tx(&bar[0], L::SQ + (wl ? L::SW : 0) + (wrr ? L::SW : 0));
  tma_load_2d(smem, qs, 4 * (i0 - 2), j0 - 2, &bar[0]);
  if (wl) tma_load_2d(smem + L::OFF_W, wr, 4 * (M - 2), j0 - 2, &bar[0]);
  if (wrr) tma_load_2d(smem + L::OFF_W + r128(L::SW), wr, 0, j0 - 2, &bar[0]);
  if constexpr (STAGE >= 2) {
    mbar_expect_tx(&bar[2], L::SN);
    tma_load_2d(smem + L::OFF_N, qn, 4 * i0, j0, &bar[2]);
  }
}

// Thread 0 polls barrier q (bounded); the other threads wait at the CTA barrier, which
// issues no instructions while the box lands, so co-resident CTAs keep the issue
// slots.  The mbarrier wait acquires the async-proxy writes for thread 0 and the CTA
// barrier passes them on to the rest.  Returns false for every thread on a timeout,
// after thread 0 has set *err and given the copies still in flight a second bounded
// wait.  Every thread of the CTA calls it.
template <int STAGE, int TY>
__device__ __forceinline__ bool tile_tma_wait(unsigned char* smem, int q, int tid, int* err) {
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + T1<TY>::OFF_BAR);
  bool ok = true;
  if (tid == 0) ok = mbar_wait(&bar[q], 0, c_wait_polls);
  if (__syncthreads_or(!ok)) {
    if (tid == 0) {
      atomicExch(err, 1);
      for (int k = q; k < (STAGE >= 2 ? 3 : 2); k++) mbar_wait(&bar[k], 0);
    }
    return false;
  }
  return true;
}

// The tile's compute once its state box has landed: ghost rows, seam columns and
// conversion to primitives, then (after the face records) the face phase, then (after
// Qn) the combine.  INNER: tile and halo inside the grid, clear of the seam, so the
// state box holds every entry and no bound is tested.
template <int SCHEME, int STAGE, bool EMIT, int TY, bool INNER>
__device__ __forceinline__ bool tile_tma_compute(unsigned char* smem, const float4* __restrict__ Qs,
                                                 float4* __restrict__ Qo, const float4* __restrict__ Mi,
                                                 const float4* __restrict__ Mj, float dt, const Consts& c, int M,
                                                 int N, int i0, int j0, int* err, uint32_t& wmax) {
  using L = T1<TY>;
  constexpr int NWY = Geo<TY>::NWY, NT = Geo<TY>::NT, HALO = Geo<TY>::HALO;
  float4(*P)[TX + 4] = reinterpret_cast<float4(*)[TX + 4]>(smem);
  float4(*Ti)[TX + 1] = reinterpret_cast<float4(*)[TX + 1]>(smem + L::OFF_I);
  float4(*Tj)[TX] = reinterpret_cast<float4(*)[TX]>(smem + L::OFF_J);
  float4(*SN)[TX] = reinterpret_cast<float4(*)[TX]>(smem + L::OFF_N);
  float4(*WL)[2] = reinterpret_cast<float4(*)[2]>(smem + L::OFF_W);             // columns M-2, M-1
  float4(*WR)[2] = reinterpret_cast<float4(*)[2]>(smem + L::OFF_W + r128(L::SW));  // columns 0, 1
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * NWX + tx;

  // take the seam columns from the seam boxes, keep the owned conserved states, convert
  // to primitives in place (the face records are landing); ghost rows are filled once
  // the records have landed (below)
  auto stage_entry = [&](int pr, int pc) {
    float4 q;
    if constexpr (INNER) {
      q = P[pr][pc];
    } else {
      const int ig = i0 - 2 + pc, j = j0 - 2 + pr;
      const float4 none = make_float4(1.0f, 0.0f, 0.0f, 1.0f);  // never read by a face of the grid
      if (j >= 0 && j < N) q = ig < 0 ? WL[pr][ig + 2] : (ig < M ? P[pr][pc] : (ig < M + 2 ? WR[pr][ig - M] : none));
      else q = none;  // a ghost row (set below) or beyond it
    }
    P[pr][pc] = to_prim<true>(q, c.gm1);
    return q;
  };
  const float4 qa = stage_entry(ty + 2, tx + 2);
  const float4 qb = stage_entry(ty + NWY + 2, tx + 2);
#pragma unroll
  for (int e = 0; e < (HALO + NT - 1) / NT; e++) {
    const int k = tid + e * NT;
    if (k < HALO) {
      int hr, hc;
      halo_entry<TY>(k, hr, hc);
      stage_entry(hr, hc);
    }
  }
  if (!tile_tma_wait<STAGE, TY>(smem, 1, tid, err)) return false;  // also orders the P writes
  if constexpr (!INNER) {
    // ghost rows (boundary pass ausm.js:34-120; loadState's clamp ausm.js:141 maps rows
    // -2 and -1 to the wall ghost), each computed once per column by the thread that
    // holds the adjacent interior cell, with the face normal from the landed records
    const bool wall = j0 == 0, far = j0 + TY + 2 > N, seam = i0 + TX >= M;  // uniform per CTA
    const int i = i0 + tx;
    if (wall && ty == 0 && i < M) {
      const float4 g = to_prim<true>(wall_ghost_n<true>(qa, Tj[0][tx].x, Tj[0][tx].y), c.gm1);
      P[0][tx + 2] = g;
      P[1][tx + 2] = g;
    }
    if (far && i < M) {
      const int r = N - 1 - j0;  // tile row of the last interior row; r == TY: the halo row above
      const bool mine = r < TY && ty == (r < NWY ? r : r - NWY);
      if (mine || (r == TY && ty == 0)) {
        const float4 s = r < TY ? (r < NWY ? qa : qb) : __ldg(&Qs[(size_t)(N - 1) * M + i]);
        const float4 f = N - j0 <= TY ? Tj[N - j0][tx] : __ldg(&Mj[(size_t)N * M + i]);
        float4 g1, g2;
        far_ghosts_n<true>(s, f.x, f.y, c, g1, g2);
        P[r + 3][tx + 2] = to_prim<true>(g1, c.gm1);
        if (r + 4 <= TY + 3) P[r + 4][tx + 2] = to_prim<true>(g2, c.gm1);
      }
    }
    if (seam && tx == 0)  // the face column past the seam (zero-filled by the box)
      for (int r = ty; r < TY; r += NWY)
        if (j0 + r < N) Ti[r][M - i0] = __ldg(&Mi[(size_t)(j0 + r) * M]);
    if (wall || far || seam) __syncthreads();
  }
  const FaceW w = own_weights<TY>(Ti, Tj, tx, ty);
  faces_phase<SCHEME, TY, INNER>(P, Ti, Tj, c, i0, j0, M, N, tx, ty);
  if constexpr (STAGE >= 2) {
    if (!tile_tma_wait<STAGE, TY>(smem, 2, tid, err)) return false;  // also orders the flux writes
  } else {
    __syncthreads();
  }
  auto qnf = [&](int h) { return SN[ty + NWY * h][tx]; };
  wmax = combine_phase<STAGE, EMIT, TY, INNER>(Ti, Tj, w, qa, qb, qnf, Qo, dt, c, i0, j0, M, N, tx, ty);
  return true;
}

// The stage of tile (i0, j0) after thread 0 has issued its loads;
// wmax gets the tile's max wave-speed bits (EMIT).  Returns false (nothing written)
// when one of the tile's loads timed out.
template <int SCHEME, int STAGE, bool EMIT, int TY>
__device__ __forceinline__ bool tile_tma_run(unsigned char* smem, const float4* __restrict__ Qs,
                                             float4* __restrict__ Qo, const float4* __restrict__ Mi,
                                             const float4* __restrict__ Mj, float dt, const Consts& c, int M, int N,
                                             int i0, int j0, int* err, uint32_t& wmax) {
  const int tid = threadIdx.y * NWX + threadIdx.x;
  if (!tile_tma_wait<STAGE, TY>(smem, 0, tid, err)) return false;
  const bool inner = i0 >= 2 && i0 + TX + 2 <= M && j0 >= 2 && j0 + TY + 2 <= N;  // uniform per CTA
  if (inner) return tile_tma_compute<SCHEME, STAGE, EMIT, TY, true>(smem, Qs, Qo, Mi, Mj, dt, c, M, N, i0, j0, err, wmax);
  return tile_tma_compute<SCHEME, STAGE, EMIT, TY, false>(smem, Qs, Qo, Mi, Mj, dt, c, M, N, i0, j0, err, wmax);
}

// The time step of a single-solve stage launch, read after the wait for the previous
// stage.  mode 0: *dtp.  mode 1 (stage 1 of the first step of an ausm_step call):
// dt = min(maxdt, cfl / max wave speed) (ausm.js:457) from the wave-speed bits the
// previous call's last stage left, computed by every CTA alike and stored to *dtp by
// the CTA at the origin for stages 2 and 3.  mode 2 (stage 2 of that step): *dtp, and
// the CTA at the origin clears the wave-speed accumulator (stage 1 has read it) for
// this call's last stage 3.
__device__ __forceinline__ float stage_dt(float* dtp, uint32_t* wave, int mode, const Consts& c, bool lead) {
  const bool origin = lead && blockIdx.x == 0 && blockIdx.y == 0;
  if (mode == 1) {
    const float dt = fminf(c.maxdt, c.cfl / __uint_as_float(*wave));
    if (origin) *dtp = dt;
    return dt;
  }
  if (mode == 2 && origin) *wave = 0u;
  return *dtp;
}

// The whole stage of tile (i0, j0): the record loads, the wait for the previous stage
// (programmatic dependent launch), the state loads and the time step (stage_dt), then
// tile_tma_run.
template <int SCHEME, int STAGE, bool EMIT, int TY>
__device__ __forceinline__ bool tile_tma_body(unsigned char* smem, const CUtensorMap* qs, const CUtensorMap* qn,
                                              const CUtensorMap* mi, const CUtensorMap* mj, const CUtensorMap* wr,
                                              const float4* __restrict__ Qs, float4* __restrict__ Qo,
                                              const float4* __restrict__ Mi, const float4* __restrict__ Mj,
                                              float* dtp, uint32_t* wave, int dt_mode, const Consts& c, int M, int N,
                                              int i0, int j0, int* err, uint32_t& wmax) {
  const bool lead = threadIdx.y * NWX + threadIdx.x == 0;
  if (lead) tile_tma_issue_records<TY>(mi, mj, smem, i0, j0);
  grid_dep_wait();
  grid_dep_launch();
  if (lead) tile_tma_issue_state<STAGE, TY>(qs, qn, wr, smem, i0, j0, M);
  const float dt = stage_dt(dtp, wave, dt_mode, c, lead);
  return tile_tma_run<SCHEME, STAGE, EMIT, TY>(smem, Qs, Qo, Mi, Mj, dt, c, M, N, i0, j0, err, wmax);
}

}  // namespace tile
}  // namespace ausm
