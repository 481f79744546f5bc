// Full-FP64 engine: the reference's dispatch structure (boundary, j-flux, i-flux,
// residual, RK stage per stage; wave-speed max once per step(n) call, main.js:744-791)
// on FP64 buffers, with FP64 metrics from the FP64 vertices and every operation in
// double (physics_exact.cuh; compiled with -fmad=false).  It exists to state the FP32
// engines' error against an FP64 solution of the same problem on the same grid.
//
// Layout as the reference engine, in double: state double4 [N+3][M] (row 0 wall ghost,
// rows N+1, N+2 far field), fluxes double4 [N][M] (i) and [N+1][M] (j), residual
// double4 [N][M], face lengths double4 and cell areas double [N][M].
#include "ausm_internal.h"
#include "physics_exact.cuh"

namespace ausm {

using ex::ConstsR;
using ex::V2;
using ex::V4;
using R = double;

namespace {

__device__ __forceinline__ V4<R> ld(const V4<R>* st, int M, int i, int j) {  // loadState, ausm.js:138-143
  int ii = (i + M) % M;
  int jj = max(j + 1, 0);
  return st[(size_t)jj * M + ii];
}

__global__ void k_ex_metrics(const V2<R>* __restrict__ V, R* __restrict__ area, V4<R>* __restrict__ flen, int M,
                             int N) {
  int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= M || j >= N) return;
  int r = (i + 1) % M;
  V2<R> a = V[(size_t)j * M + i], b = V[(size_t)j * M + r], c = V[(size_t)(j + 1) * M + i],
        d = V[(size_t)(j + 1) * M + r];
  size_t k = (size_t)j * M + i;
  area[k] = ex::quad_area(a, b, c, d);
  flen[k] = {sqrt((a.x - c.x) * (a.x - c.x) + (a.y - c.y) * (a.y - c.y)),
             sqrt((b.x - d.x) * (b.x - d.x) + (b.y - d.y) * (b.y - d.y)),
             sqrt((c.x - d.x) * (c.x - d.x) + (c.y - d.y) * (c.y - d.y)),
             sqrt((a.x - b.x) * (a.x - b.x) + (a.y - b.y) * (a.y - b.y))};
}

__global__ void k_ex_boundary(const V4<R>* __restrict__ in, V4<R>* __restrict__ out, const V2<R>* __restrict__ V,
                              const ConstsR<R> c, int M, int N) {
  int i = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= M || y >= N + 3) return;
  int r = (i + 1) % M;
  if (y == 0) {
    out[i] = ex::wall_ghost(in[(size_t)M + i], V[i], V[r]);
  } else if (y > N) {
    V4<R> g1, g2;
    ex::far_ghosts(in[(size_t)N * M + i], V[(size_t)N * M + i], V[(size_t)N * M + r], c, g1, g2);
    out[(size_t)y * M + i] = (y == N + 1) ? g1 : g2;
  } else {
    out[(size_t)y * M + i] = in[(size_t)y * M + i];
  }
}

template <int SCHEME>
__global__ void k_ex_flux_j(const V4<R>* __restrict__ st, const V2<R>* __restrict__ V, V4<R>* __restrict__ fy,
                            const ConstsR<R> c, int M, int N) {
  int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= M || j > N) return;
  R nx, ny, len;
  ex::edge_normal(V[(size_t)j * M + i], V[(size_t)j * M + (i + 1) % M], nx, ny, len);
  fy[(size_t)j * M + i] = ex::face_flux<SCHEME>(ex::to_prim(ld(st, M, i, j - 2), c.gm1),
                                                ex::to_prim(ld(st, M, i, j - 1), c.gm1),
                                                ex::to_prim(ld(st, M, i, j), c.gm1),
                                                ex::to_prim(ld(st, M, i, j + 1), c.gm1), nx, ny, c);
}

template <int SCHEME>
__global__ void k_ex_flux_i(const V4<R>* __restrict__ st, const V2<R>* __restrict__ V, V4<R>* __restrict__ fx,
                            const ConstsR<R> c, int M, int N) {
  int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= M || j >= N) return;
  R nx, ny, len;
  ex::edge_normal(V[(size_t)(j + 1) * M + i], V[(size_t)j * M + i], nx, ny, len);
  fx[(size_t)j * M + i] = ex::face_flux<SCHEME>(ex::to_prim(ld(st, M, i - 2, j), c.gm1),
                                                ex::to_prim(ld(st, M, i - 1, j), c.gm1),
                                                ex::to_prim(ld(st, M, i, j), c.gm1),
                                                ex::to_prim(ld(st, M, i + 1, j), c.gm1), nx, ny, c);
}

__global__ void k_ex_residual(const V4<R>* __restrict__ fx, const V4<R>* __restrict__ fy,
                              const V4<R>* __restrict__ flen, const R* __restrict__ area, V4<R>* __restrict__ res,
                              int M, int N) {
  int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= M || j >= N) return;
  size_t k = (size_t)j * M + i;
  V4<R> xl = fx[k], xr = fx[(size_t)j * M + (i + 1) % M], yu = fy[(size_t)(j + 1) * M + i], yd = fy[k];
  V4<R> l = flen[k];
  R A = area[k];
  res[k] = {-(xr.x * l.y - xl.x * l.x + yu.x * l.z - yd.x * l.w) / A,
            -(xr.y * l.y - xl.y * l.x + yu.y * l.z - yd.y * l.w) / A,
            -(xr.z * l.y - xl.z * l.x + yu.z * l.z - yd.z * l.w) / A,
            -(xr.w * l.y - xl.w * l.x + yu.w * l.z - yd.w * l.w) / A};
}

template <int STAGE>
__global__ void k_ex_rk(const V4<R>* __restrict__ res, const V4<R>* __restrict__ s0, const V4<R>* __restrict__ s1,
                        V4<R>* __restrict__ out, const R* __restrict__ dtp, int M, int N) {
  int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= M || j >= N) return;
  const R dt = *dtp;
  size_t k = (size_t)j * M + i, o = (size_t)(j + 1) * M + i;
  V4<R> Rr = res[k], Q = s0[o], o4;
  if constexpr (STAGE == 1) {
    o4 = {Q.x + dt * Rr.x, Q.y + dt * Rr.y, Q.z + dt * Rr.z, Q.w + dt * Rr.w};
  } else if constexpr (STAGE == 2) {
    V4<R> Q1 = s1[o];
    o4 = {R(0.75) * Q.x + R(0.25) * (Q1.x + dt * Rr.x), R(0.75) * Q.y + R(0.25) * (Q1.y + dt * Rr.y),
          R(0.75) * Q.z + R(0.25) * (Q1.z + dt * Rr.z), R(0.75) * Q.w + R(0.25) * (Q1.w + dt * Rr.w)};
  } else {
    V4<R> Q2 = s1[o];
    o4 = {(Q.x + R(2) * (Q2.x + dt * Rr.x)) / R(3), (Q.y + R(2) * (Q2.y + dt * Rr.y)) / R(3),
          (Q.z + R(2) * (Q2.z + dt * Rr.z)) / R(3), (Q.w + R(2) * (Q2.w + dt * Rr.w)) / R(3)};
  }
  out[o] = o4;
}

// max of the FP64 wave speed: positive doubles order like their bit patterns
__global__ void k_ex_wave(const V4<R>* __restrict__ st, const V4<R>* __restrict__ flen, const R* __restrict__ area,
                          R gamma, int M, int N, unsigned long long* wave) {
  __shared__ unsigned long long red[8];
  unsigned long long wm = 0ull;
  size_t total = (size_t)M * N;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
    V4<R> l = flen[k];
    R w = ex::wave_speed(st[k + M], ((l.x + l.y) + l.z) + l.w, area[k], gamma);
    wm = max(wm, (unsigned long long)__double_as_longlong(w));
  }
  for (int o = 16; o > 0; o >>= 1) wm = max(wm, __shfl_down_sync(0xffffffffu, wm, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = wm;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) wm = max(wm, red[w]);
    atomicMax(wave, wm);
  }
}

__global__ void k_ex_dt(const unsigned long long* __restrict__ wave, R* __restrict__ dt, R maxdt, R cfl) {
  dt[0] = fmin(maxdt, cfl / __longlong_as_double((long long)wave[0]));
}

__global__ void k_ex_fill(V4<R>* __restrict__ a, V4<R> v, size_t n) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) a[k] = v;
}
__global__ void k_ex_to_f32(const V4<R>* __restrict__ a, float4* __restrict__ b, size_t n) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    V4<R> v = a[k];
    b[k] = make_float4((float)v.x, (float)v.y, (float)v.z, (float)v.w);
  }
}
__global__ void k_ex_from_f32(const float4* __restrict__ a, V4<R>* __restrict__ b, size_t n) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    float4 v = a[k];
    b[k] = {v.x, v.y, v.z, v.w};
  }
}

// surface force from the FP64 state (pressure of interior row 1, graphs.js:5-41),
// per-block partial sums; Cp per wall face
__global__ void k_ex_forces(const V4<R>* __restrict__ row1, const V2<R>* __restrict__ V, R gamma, int M,
                            double* parts, double* cp, double q_inf, double p_inf) {
  double fx = 0.0, fy = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M; i += gridDim.x * blockDim.x) {
    V4<R> s = row1[i];
    R rho = s.x, u = s.y / rho, v = s.z / rho;
    R p = (s.w - R(0.5) * rho * (u * u + v * v)) * (gamma - R(1));
    V2<R> a = V[i], b = V[(i + 1) % M];
    R dx = b.x - a.x, dy = b.y - a.y;
    R len = sqrt(dx * dx + dy * dy);
    R nx = dy / len, ny = -dx / len;
    fx += -p * len * nx;
    fy += -p * len * ny;
    if (cp) cp[i] = (p - p_inf) / q_inf;
  }
  block_sum_store(parts + blockIdx.x, fx);
  __syncthreads();
  block_sum_store(parts + kMaxParts + blockIdx.x, fy);
}

__global__ void k_ex_sumsq_rho(const V4<R>* __restrict__ res, size_t n, double* parts) {
  double s = 0.0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    s += res[k].x * res[k].x;
  block_sum_store(parts + blockIdx.x, s);
}

inline dim3 grid16(int w, int h) { return dim3((w + 15) / 16, (h + 15) / 16); }
const dim3 B16(16, 16);
inline int grid1d(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }

template <int SCHEME>
void fluxes(const V4<R>* st, const V2<R>* V, V4<R>* fx, V4<R>* fy, const ConstsR<R>& c, int M, int N,
            cudaStream_t s) {
  k_ex_flux_j<SCHEME><<<grid16(M, N + 1), B16, 0, s>>>(st, V, fy, c, M, N);
  k_ex_flux_i<SCHEME><<<grid16(M, N), B16, 0, s>>>(st, V, fx, c, M, N);
}

}  // namespace

F64Engine::~F64Engine() {
  void* p[] = {S[0], S[1], S[2], fx, fy, res, flen, area, wave, dt};
  for (void* q : p)
    if (q) cudaFree(q);
}

cudaError_t F64Engine::allocate(int M_, int N_) {
  M = M_;
  N = N_;
  const size_t nref = (size_t)M * (N + 3), n = (size_t)M * N;
  cudaError_t e = cudaSuccess;
  for (auto& s : S)
    if (e == cudaSuccess) e = cudaMalloc((void**)&s, nref * sizeof(V4<R>));
  if (e == cudaSuccess) e = cudaMalloc((void**)&fx, n * sizeof(V4<R>));
  if (e == cudaSuccess) e = cudaMalloc((void**)&fy, (size_t)M * (N + 1) * sizeof(V4<R>));
  if (e == cudaSuccess) e = cudaMalloc((void**)&res, n * sizeof(V4<R>));
  if (e == cudaSuccess) e = cudaMalloc((void**)&flen, n * sizeof(V4<R>));
  if (e == cudaSuccess) e = cudaMalloc((void**)&area, n * sizeof(R));
  if (e == cudaSuccess) e = cudaMalloc((void**)&wave, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc((void**)&dt, sizeof(R));
  return e;
}

void F64Engine::metrics(const double2* Vd, cudaStream_t s) {
  k_ex_metrics<<<grid16(M, N), B16, 0, s>>>(reinterpret_cast<const V2<R>*>(Vd), area, flen, M, N);
}
void F64Engine::from_f32(const float4* ref, cudaStream_t s) {
  const size_t n = (size_t)M * (N + 3);
  k_ex_from_f32<<<grid1d(n), 256, 0, s>>>(ref, S[2], n);
}
void F64Engine::to_f32(float4* ref, const double2* Vd, cudaStream_t s) {
  // boundary pass into S[0] (the reference layout with its ghost rows), then rounded
  k_ex_boundary<<<grid16(M, N + 3), B16, 0, s>>>(S[2], S[0], reinterpret_cast<const V2<R>*>(Vd), c, M, N);
  const size_t n = (size_t)M * (N + 3);
  k_ex_to_f32<<<grid1d(n), 256, 0, s>>>(S[0], ref, n);
}
void F64Engine::fill(double rho, double ru, double rv, double E, cudaStream_t s) {
  const size_t n = (size_t)M * (N + 3);
  k_ex_fill<<<grid1d(n), 256, 0, s>>>(S[2], V4<R>{rho, ru, rv, E}, n);
}
const void* F64Engine::state_ref(const double2* Vd, cudaStream_t s) {
  k_ex_boundary<<<grid16(M, N + 3), B16, 0, s>>>(S[2], S[0], reinterpret_cast<const V2<R>*>(Vd), c, M, N);
  return S[0];
}
void F64Engine::wave_speed(cudaStream_t s) {
  cudaMemsetAsync(wave, 0, sizeof(unsigned long long), s);
  int blocks = (int)std::min<size_t>(((size_t)M * N + 255) / 256, 148 * 8);
  k_ex_wave<<<blocks, 256, 0, s>>>(S[2], flen, area, c.gamma, M, N, wave);
}
void F64Engine::step(int scheme, int n, const double2* Vd_, cudaStream_t s) {
  const V2<R>* Vd = reinterpret_cast<const V2<R>*>(Vd_);
  k_ex_dt<<<1, 1, 0, s>>>(wave, dt, c.maxdt, c.cfl);
  auto flux = [&](const V4<R>* st) {
    if (scheme == 0) fluxes<0>(st, Vd, fx, fy, c, M, N, s);
    else if (scheme == 1) fluxes<1>(st, Vd, fx, fy, c, M, N, s);
    else fluxes<2>(st, Vd, fx, fy, c, M, N, s);
    k_ex_residual<<<grid16(M, N), B16, 0, s>>>(fx, fy, flen, area, res, M, N);
  };
  const dim3 gb = grid16(M, N + 3), gi = grid16(M, N);
  for (int k = 0; k < n; k++) {  // the texture ping-pong of main.js:744-777
    k_ex_boundary<<<gb, B16, 0, s>>>(S[2], S[0], Vd, c, M, N);
    flux(S[0]);
    k_ex_rk<1><<<gi, B16, 0, s>>>(res, S[0], nullptr, S[1], dt, M, N);
    k_ex_boundary<<<gb, B16, 0, s>>>(S[1], S[2], Vd, c, M, N);
    flux(S[2]);
    k_ex_rk<2><<<gi, B16, 0, s>>>(res, S[0], S[1], S[2], dt, M, N);
    k_ex_boundary<<<gb, B16, 0, s>>>(S[2], S[1], Vd, c, M, N);
    flux(S[1]);
    k_ex_rk<3><<<gi, B16, 0, s>>>(res, S[0], S[1], S[2], dt, M, N);
  }
  if (n > 0) wave_speed(s);
}
void F64Engine::residual(int scheme, const double2* Vd_, cudaStream_t s) {
  const V2<R>* Vd = reinterpret_cast<const V2<R>*>(Vd_);
  k_ex_boundary<<<grid16(M, N + 3), B16, 0, s>>>(S[2], S[0], Vd, c, M, N);
  if (scheme == 0) fluxes<0>(S[0], Vd, fx, fy, c, M, N, s);
  else if (scheme == 1) fluxes<1>(S[0], Vd, fx, fy, c, M, N, s);
  else fluxes<2>(S[0], Vd, fx, fy, c, M, N, s);
  k_ex_residual<<<grid16(M, N), B16, 0, s>>>(fx, fy, flen, area, res, M, N);
}
void F64Engine::sumsq_rho(double* parts, double* acc, cudaStream_t s) {
  const size_t n = (size_t)M * N;
  const int blocks = grid1d(n);
  k_ex_sumsq_rho<<<blocks, 256, 0, s>>>(res, n, parts);
  launch_sum_parts(parts, blocks, 1, acc, s);
}
void F64Engine::forces(const double2* Vd, double* parts, double* acc, double* cp, double q_inf, double p_inf,
                       cudaStream_t s) {
  int blocks = std::min((M + 255) / 256, 148);
  k_ex_forces<<<blocks, 256, 0, s>>>(S[2] + M, reinterpret_cast<const V2<R>*>(Vd), c.gamma, M, parts, cp, q_inf,
                                     p_inf);
  launch_sum_parts(parts, blocks, 2, acc, s);
}

}  // namespace ausm
