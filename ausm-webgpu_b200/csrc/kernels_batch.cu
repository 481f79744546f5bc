// Batched stage kernel: one launch per RK stage and scheme advances every solve of that
// scheme in a batch of independent O-grids of any sizes (stage 0: residual only).  The
// work list is the concatenation of all solves' 32 x TY tiles, grouped by scheme; each
// CTA takes one work item, reads its solve, the solve's buffer rotation and its tile
// coordinates from the item table (one load; a binary search over the first-tile
// offsets took a chain of dependent loads), issues its TMA boxes through the solve's
// tensor maps before it reads anything else of the solve's descriptor, and runs the
// same tile compute as the single-solve kernel
// (stage_tile.cuh) with that solve's buffers, constants and dt; with TMA (every solve
// has tensor maps) its boxes are loaded through the solve's maps (tile_tma.cuh).  The
// tile height TY (8, 16 or 32) is chosen per batch by the autotuner (batch.cu).  The
// scheme is a template parameter: a run-time scheme switch inside one kernel holds all
// three flux variants' registers at once and spills at the 64-register budget.  One
// CTA per item rather than a persistent grid-stride loop: the hardware block scheduler
// hands out items dynamically, and on B200 the persistent form ran 8% slower.  Each
// solve's dt comes from its own max wave speed, so a solve's arithmetic is the same
// alone or in any batch.  The buffer rotation lives in the descriptors (cur, advanced
// on the device after a step sequence), so one captured CUDA graph of n steps can be
// replayed for any number of rounds.
#include <algorithm>

#include "stage_tile.cuh"
#include "tile_tma.cuh"

namespace ausm {
using namespace tile;

// dynamic shared memory of the per-thread-load kernel: P, Ti, Tj
template <int TY> struct LdgSmem {
  static constexpr int OFF_I = (TX + 4) * (TY + 4) * 16;
  static constexpr int OFF_J = OFF_I + TY * (TX + 1) * 16;
  static constexpr int BYTES = OFF_J + (TY + 1) * TX * 16;
};

// Work item t0 + blockIdx.x of the item table: its solve, the index of the solve's
// current buffer and its tile origin.  The buffer index is the solve's rotation when
// the table was written plus the steps the batch has taken since (*steps) plus rot.
struct ItemTile {
  int s, a, i0, j0, M;
};
template <int TY>
__device__ __forceinline__ ItemTile item_tile(const BatchItem* __restrict__ items, const int* __restrict__ steps,
                                              int item, int rot) {
  const BatchItem it = items[item];
  return {it.solve, (it.cur + *steps + rot) % 3, (it.tile & 0xffff) * TX, (it.tile >> 16) * TY, it.M};
}

// One CTA per work item of one scheme group; per-thread loads.
template <int SCHEME, int STAGE, bool EMIT, int TY>
__global__ void __launch_bounds__(Geo<TY>::NT, Geo<TY>::MIN_BLOCKS)
    k_batch_stage(const BatchSolve* __restrict__ solves, const BatchItem* __restrict__ items,
                  const int* __restrict__ steps, const int t0, const int rot) {
  using G = Geo<TY>;
  extern __shared__ __align__(16) unsigned char smem_ldg[];  // P, Ti, Tj (LdgSmem<TY>)
  float4(*P)[G::PW] = reinterpret_cast<float4(*)[G::PW]>(smem_ldg);
  float4(*Ti)[TX + 1] = reinterpret_cast<float4(*)[TX + 1]>(smem_ldg + LdgSmem<TY>::OFF_I);
  float4(*Tj)[TX] = reinterpret_cast<float4(*)[TX]>(smem_ldg + LdgSmem<TY>::OFF_J);
  const int tx = threadIdx.x, ty = threadIdx.y;
  const ItemTile w0 = item_tile<TY>(items, steps, t0 + blockIdx.x, rot);
  grid_dep_wait();  // the previous stage (and the dt of this step) complete
  grid_dep_launch();
  const BatchSolve& d = solves[w0.s];
  const Consts c = d.c;
  const int M = d.M, N = d.N, i0 = w0.i0, j0 = w0.j0;
  const int a = w0.a, b = (a + 1) % 3, c3 = (a + 2) % 3;
  const float4* Qs = d.Q[STAGE <= 1 ? a : (STAGE == 2 ? b : c3)];
  const float4* Qn = d.Q[a];
  float4* Qo = d.Q[STAGE == 2 ? c3 : b];
  float4 qa, qb;
  stage_tile_ldg<TY>(Qs, d.Mi, d.Mj, c, P, Ti, Tj, i0, j0, M, N, tx, ty, qa, qb);
  __syncthreads();
  const FaceW w = own_weights<TY>(Ti, Tj, tx, ty);
  faces_phase<SCHEME, TY>(P, Ti, Tj, c, i0, j0, M, N, tx, ty);
  __syncthreads();
  auto qn = [&](int h) { return __ldg(&Qn[(size_t)(j0 + ty + G::NWY * h) * M + i0 + tx]); };
  uint32_t wv = combine_phase<STAGE, EMIT, TY>(Ti, Tj, w, qa, qb, qn, Qo, *d.dt, c, i0, j0, M, N, tx, ty);
  if constexpr (EMIT) block_max_to(d.wave, wv);
}

// TMA-staged form (stages 1-3): the tile's boxes come through the solve's own tensor
// maps (in global memory, kBatchMaps per solve in descriptor order, for this tile
// height).
template <int SCHEME, int STAGE, bool EMIT, int TY>
__global__ void __launch_bounds__(Geo<TY>::NT, Geo<TY>::MIN_BLOCKS)
    k_batch_stage_tma(const BatchSolve* __restrict__ solves, const BatchItem* __restrict__ items,
                      const int* __restrict__ steps, const CUtensorMap* __restrict__ maps, const int t0,
                      const int rot, int* __restrict__ err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  const ItemTile w0 = item_tile<TY>(items, steps, t0 + blockIdx.x, rot);
  const int a = w0.a, b = (a + 1) % 3, c3 = (a + 2) % 3;
  const int s_in = STAGE == 1 ? a : (STAGE == 2 ? b : c3);
  const CUtensorMap* mp = maps + kBatchMaps * (size_t)w0.s;
  const bool lead = threadIdx.y * NWX + threadIdx.x == 0;
  if (lead) tile_tma_issue_records<TY>(&mp[6], &mp[7], smem, w0.i0, w0.j0);
  grid_dep_wait();  // the previous stage (and the dt of this step) complete
  grid_dep_launch();
  if (lead) tile_tma_issue_state<STAGE, TY>(&mp[s_in], &mp[3 + a], &mp[8 + s_in], smem, w0.i0, w0.j0, w0.M);
  const BatchSolve& d = solves[w0.s];  // read while the boxes land
  const Consts c = d.c;
  uint32_t wmax = 0u;
  if (!tile_tma_run<SCHEME, STAGE, EMIT, TY>(smem, d.Q[s_in], d.Q[STAGE == 2 ? c3 : b], d.Mi, d.Mj, *d.dt, c, d.M,
                                             d.N, w0.i0, w0.j0, err, wmax))
    return;
  if constexpr (EMIT) block_max_to(d.wave, wmax);
}

// dt = min(maxdt, cfl / max wave speed) per solve (ausm.js:457), then the wave-speed
// accumulator is cleared for the step sequence's last stage 3.
__global__ void k_batch_dt(BatchSolve* __restrict__ solves, int n) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  BatchSolve& d = solves[s];
  d.dt[0] = fminf(d.c.maxdt, d.c.cfl / __uint_as_float(d.wave[0]));
  d.wave[0] = 0u;
}
__global__ void k_batch_advance(BatchSolve* __restrict__ solves, int n, int steps, int* __restrict__ taken) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) solves[s].cur = (solves[s].cur + steps) % 3;
  if (s == 0) *taken += steps;
}

__global__ void k_batch_gather(const BatchSolve* __restrict__ solves, int n, float* __restrict__ out) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  out[2 * s] = solves[s].dt[0];
  out[2 * s + 1] = __uint_as_float(solves[s].wave[0]);
}

// Residual norms in a fixed order that depends only on each solve's own size: one CTA
// per chunk of kNormChunk consecutive cells (row-major) of one solve, strided per-thread
// sums and a shared-memory tree into part[chunk]; then one warp per solve adds its
// chunks' partial sums (lane-strided, then a fixed butterfly).  The tile height of the
// batch does not enter, so a solve's norm is the same in any batch.
constexpr int kNormChunk = 512;

__global__ void __launch_bounds__(256) k_batch_chunk_sumsq(const BatchSolve* __restrict__ solves, int nsolves,
                                                           double* __restrict__ part) {
  const int chunk = blockIdx.x;
  int lo = 0, hi = nsolves - 1;  // the last solve whose first chunk is <= chunk
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (solves[mid].chunk0 <= chunk) lo = mid;
    else hi = mid - 1;
  }
  const BatchSolve& d = solves[lo];
  const float4* R = d.Q[(d.cur + 1) % 3];
  const size_t n = (size_t)d.M * d.N, k0 = (size_t)(chunk - d.chunk0) * kNormChunk;
  double acc = 0.0;
  for (int k = threadIdx.x; k < kNormChunk; k += 256)
    if (k0 + k < n) {
      double r = R[k0 + k].x;
      acc += r * r;
    }
  __shared__ double sh[256];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[chunk] = sh[0];
}

__global__ void k_batch_norm(const BatchSolve* __restrict__ solves, int nsolves, const double* __restrict__ part,
                             double* __restrict__ l2) {
  const int s = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (s >= nsolves) return;
  const BatchSolve& d = solves[s];
  const size_t n = (size_t)d.M * d.N;
  const int nchunks = (int)((n + kNormChunk - 1) / kNormChunk);
  double acc = 0.0;
  for (int t = lane; t < nchunks; t += 32) acc += part[d.chunk0 + t];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) l2[s] = sqrt(acc / (double)n);
}

void launch_batch_gather(const BatchSolve* d, int nsolves, float* out, cudaStream_t s) {
  k_batch_gather<<<(nsolves + 127) / 128, 128, 0, s>>>(d, nsolves, out);
}
void launch_batch_residual_norm(const BatchSolve* d, int nsolves, int total_chunks, double* part, double* l2,
                                cudaStream_t s) {
  if (total_chunks <= 0) return;
  k_batch_chunk_sumsq<<<total_chunks, 256, 0, s>>>(d, nsolves, part);
  k_batch_norm<<<(nsolves + 3) / 4, 128, 0, s>>>(d, nsolves, part, l2);
}

cudaError_t set_wait_polls_batch(unsigned polls) { return cudaMemcpyToSymbol(c_wait_polls, &polls, sizeof polls); }

void launch_batch_dt(BatchSolve* d, int nsolves, cudaStream_t s) {
  k_batch_dt<<<(nsolves + 127) / 128, 128, 0, s>>>(d, nsolves);
}
void launch_batch_advance(BatchSolve* d, int nsolves, int steps, int* taken, cudaStream_t s) {
  k_batch_advance<<<(nsolves + 127) / 128, 128, 0, s>>>(d, nsolves, steps, taken);
}

namespace {
template <int SC, int ST, bool E, int TY>
void launch_b(const BatchSolve* d, const BatchItem* items, const int* steps, const CUtensorMap* maps, int t_lo, int t_hi, int rot, int* err, cudaStream_t s) {
  const dim3 block(NWX, Geo<TY>::NWY);
  if constexpr (ST != 0) {
    if (err) {
      static bool attr = false;
      if (!attr) {
        cudaFuncSetAttribute(k_batch_stage_tma<SC, ST, E, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             T1<TY>::SMEM);
        attr = true;
      }
      launch_pdl(k_batch_stage_tma<SC, ST, E, TY>, dim3(t_hi - t_lo), block, T1<TY>::SMEM, s, d, items, steps, maps,
                 t_lo, rot, err);
      return;
    }
  }
  // per-thread loads: the residual (any height) and batches without TMA (height 16)
  if constexpr (ST == 0 || TY == 16) {
    static bool attr = false;
    if (!attr) {
      cudaFuncSetAttribute(k_batch_stage<SC, ST, E, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           LdgSmem<TY>::BYTES);
      attr = true;
    }
    launch_pdl(k_batch_stage<SC, ST, E, TY>, dim3(t_hi - t_lo), block, LdgSmem<TY>::BYTES, s, d, items, steps, t_lo,
               rot);
  }
}
template <int SC, int TY>
void launch_scheme(int stage, bool emit, const BatchSolve* d, const BatchItem* items, const int* steps, const CUtensorMap* maps, int t_lo, int t_hi, int rot,
                   int* err, cudaStream_t s) {
  if (stage == 0) launch_b<SC, 0, false, TY>(d, items, steps, maps, t_lo, t_hi, rot, nullptr, s);
  else if (stage == 1) launch_b<SC, 1, false, TY>(d, items, steps, maps, t_lo, t_hi, rot, err, s);
  else if (stage == 2) launch_b<SC, 2, false, TY>(d, items, steps, maps, t_lo, t_hi, rot, err, s);
  else if (emit) launch_b<SC, 3, true, TY>(d, items, steps, maps, t_lo, t_hi, rot, err, s);
  else launch_b<SC, 3, false, TY>(d, items, steps, maps, t_lo, t_hi, rot, err, s);
}
template <int TY>
void launch_rows(int scheme, int stage, bool emit, const BatchSolve* d, const BatchItem* items, const int* steps, const CUtensorMap* maps, int t_lo, int t_hi,
                 int rot, int* err, cudaStream_t s) {
  switch (scheme) {  // scheme + 4: MUSCL known on
    case 0: launch_scheme<0, TY>(stage, emit, d, items, steps, maps, t_lo, t_hi, rot, err, s); break;
    case 1: launch_scheme<1, TY>(stage, emit, d, items, steps, maps, t_lo, t_hi, rot, err, s); break;
    case 2: launch_scheme<2, TY>(stage, emit, d, items, steps, maps, t_lo, t_hi, rot, err, s); break;
    case 4: launch_scheme<4, TY>(stage, emit, d, items, steps, maps, t_lo, t_hi, rot, err, s); break;
    case 5: launch_scheme<5, TY>(stage, emit, d, items, steps, maps, t_lo, t_hi, rot, err, s); break;
    default: launch_scheme<6, TY>(stage, emit, d, items, steps, maps, t_lo, t_hi, rot, err, s); break;
  }
}
}  // namespace

void launch_batch_stage(int scheme, int stage, bool emit, const BatchSolve* d, const BatchItem* items,
                        const int* steps, const CUtensorMap* maps, int t_lo,
                        int t_hi, int rot, int rows, int* err, cudaStream_t s) {
  if (t_hi <= t_lo) return;
  if (rows == 8) launch_rows<8>(scheme, stage, emit, d, items, steps, maps, t_lo, t_hi, rot, err, s);
  else if (rows == 32) launch_rows<32>(scheme, stage, emit, d, items, steps, maps, t_lo, t_hi, rot, err, s);
  else launch_rows<16>(scheme, stage, emit, d, items, steps, maps, t_lo, t_hi, rot, err, s);
}

}  // namespace ausm
