// Grid generation, layout conversion, surface forces, residual norms and field output.
#include "ausm_internal.h"

namespace ausm {

// ---- reference layout <-> interior layout ----
// ref: float4 [N+3][M] with row 0 the wall ghost and rows N+1, N+2 the far field,
// filled with the boundary pass of the interior (ausm.js:34-120).
__global__ void k_to_ref_layout(const float4* __restrict__ Q, float4* __restrict__ ref, const float2* __restrict__ V,
                                const Consts c, int M, int N) {
  int i = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= M || y >= N + 3) return;
  int r = (i + 1) % M;
  if (y == 0) {
    ref[i] = wall_ghost<false>(Q[i], V[i], V[r]);
  } else if (y > N) {
    float4 g1, g2;
    far_ghosts<false>(Q[(size_t)(N - 1) * M + i], V[(size_t)N * M + i], V[(size_t)N * M + r], c, g1, g2);
    ref[(size_t)y * M + i] = (y == N + 1) ? g1 : g2;
  } else {
    ref[(size_t)y * M + i] = Q[(size_t)(y - 1) * M + i];
  }
}
__global__ void k_from_ref_layout(const float4* __restrict__ ref, float4* __restrict__ Q, size_t n, int M) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    Q[k] = ref[k + M];
}
__global__ void k_fill(float4* __restrict__ Q, float4 v, size_t n) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) Q[k] = v;
}

// ---- grid ----
// Initial guess (shaders/grid.js:18-27): mix(body, outer, t) along each i line,
// t = j/N (reference) or a geometric progression with first cell height `h1` relative
// to the body-outer distance of that line.
__global__ void k_grid_init(float2* __restrict__ V, int M, int N, double first_spacing) {
  int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= M || j > N || j == 0 || j == N) return;
  float2 a = V[i], b = V[(size_t)N * M + i];
  float t;
  if (first_spacing <= 0.0) {
    t = float(j) / float(N);
  } else {
    double L = sqrt((double)(b.x - a.x) * (b.x - a.x) + (double)(b.y - a.y) * (b.y - a.y));
    double h = first_spacing / L;  // first step as a fraction of the line length
    // growth ratio q solves h (q^N - 1)/(q - 1) = 1 (bisection, fixed iteration count)
    double lo = 1.0 + 1e-12, hi = 2.0;
    if (h * N >= 1.0) { lo = 1e-6; hi = 1.0 - 1e-12; }
    for (int it = 0; it < 200; it++) {
      double q = 0.5 * (lo + hi);
      double s = h * (pow(q, (double)N) - 1.0) / (q - 1.0);
      if ((s > 1.0) == (h * N < 1.0)) hi = q; else lo = q;
    }
    double q = 0.5 * (lo + hi);
    t = (float)(h * (pow(q, (double)j) - 1.0) / (q - 1.0));
  }
  V[(size_t)j * M + i] = make_float2(a.x * (1.0f - t) + b.x * t, a.y * (1.0f - t) + b.y * t);
}

// TTM/Winslow update with P = Q = 0, omega = 1, applied only where the Jacobian is
// negative (shaders/grid.js:55-108); i wraps through the seam.
__device__ __forceinline__ float2 ttm_point(const float2* __restrict__ s, int M, int i, int j, float omega) {
  int l = i == 0 ? M - 1 : i - 1, r = i == M - 1 ? 0 : i + 1;
  size_t rj = (size_t)j * M, ru = (size_t)(j + 1) * M, rd = (size_t)(j - 1) * M;
  float2 c = s[rj + i], L = s[rj + l], R = s[rj + r], D = s[rd + i], U = s[ru + i];
  float2 DL = s[rd + l], DR = s[rd + r], UL = s[ru + l], UR = s[ru + r];
  float xix = 0.5f * (R.x - L.x), xiy = 0.5f * (R.y - L.y);
  float etx = 0.5f * (U.x - D.x), ety = 0.5f * (U.y - D.y);
  float xex = 0.25f * (UR.x + DL.x - UL.x - DR.x), xey = 0.25f * (UR.y + DL.y - UL.y - DR.y);
  float alpha = etx * etx + ety * ety, gam = xix * xix + xiy * xiy, beta = xix * etx + xiy * ety;
  const float Pc = 0.0f, Qc = 0.0f;
  float den = 2.0f * (alpha + gam);
  float npx = (alpha * (L.x + R.x + Pc * xix) + gam * (D.x + U.x + Qc * etx) - 2.0f * beta * xex) / den;
  float npy = (alpha * (L.y + R.y + Pc * xiy) + gam * (D.y + U.y + Qc * ety) - 2.0f * beta * xey) / den;
  float jac = xix * ety - xiy * etx;
  if (jac < 0.0f) return make_float2(c.x * (1.0f - omega) + npx * omega, c.y * (1.0f - omega) + npy * omega);
  return c;
}
__global__ void k_grid_jacobi(const float2* __restrict__ src, float2* __restrict__ dst, int M, int N) {
  int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= M || j < 1 || j >= N) return;
  dst[(size_t)j * M + i] = ttm_point(src, M, i, j, 1.0f);
}

// ---- FP64 grid (multicolor TTM generator of the fused engine) and FP64 metrics ----
__global__ void k_grid_init_d(double2* __restrict__ V, int M, int N, double first_spacing) {
  int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= M || j > N || j == 0 || j == N) return;
  double2 a = V[i], b = V[(size_t)N * M + i];
  double t;
  if (first_spacing <= 0.0) {
    t = (double)j / (double)N;
  } else {
    double L = sqrt((b.x - a.x) * (b.x - a.x) + (b.y - a.y) * (b.y - a.y));
    double h = first_spacing / L;
    double lo = 1.0 + 1e-12, hi = 2.0;
    if (h * N >= 1.0) { lo = 1e-6; hi = 1.0 - 1e-12; }
    for (int it = 0; it < 200; it++) {
      double q = 0.5 * (lo + hi);
      double s = h * (pow(q, (double)N) - 1.0) / (q - 1.0);
      if ((s > 1.0) == (h * N < 1.0)) hi = q; else lo = q;
    }
    double q = 0.5 * (lo + hi);
    t = h * (pow(q, (double)j) - 1.0) / (q - 1.0);
  }
  V[(size_t)j * M + i] = make_double2(a.x * (1.0 - t) + b.x * t, a.y * (1.0 - t) + b.y * t);
}

__device__ __forceinline__ double2 ttm_point_d(const double2* __restrict__ s, int M, int i, int j, double omega) {
  int l = i == 0 ? M - 1 : i - 1, r = i == M - 1 ? 0 : i + 1;
  size_t rj = (size_t)j * M, ru = (size_t)(j + 1) * M, rd = (size_t)(j - 1) * M;
  double2 c = s[rj + i], L = s[rj + l], R = s[rj + r], D = s[rd + i], U = s[ru + i];
  double2 DL = s[rd + l], DR = s[rd + r], UL = s[ru + l], UR = s[ru + r];
  double xix = 0.5 * (R.x - L.x), xiy = 0.5 * (R.y - L.y);
  double etx = 0.5 * (U.x - D.x), ety = 0.5 * (U.y - D.y);
  double xex = 0.25 * (UR.x + DL.x - UL.x - DR.x), xey = 0.25 * (UR.y + DL.y - UL.y - DR.y);
  double alpha = etx * etx + ety * ety, gam = xix * xix + xiy * xiy, beta = xix * etx + xiy * ety;
  double den = 2.0 * (alpha + gam);
  double npx = (alpha * (L.x + R.x) + gam * (D.x + U.x) - 2.0 * beta * xex) / den;
  double npy = (alpha * (L.y + R.y) + gam * (D.y + U.y) - 2.0 * beta * xey) / den;
  double jac = xix * ety - xiy * etx;
  if (jac < 0.0) return make_double2(c.x * (1.0 - omega) + npx * omega, c.y * (1.0 - omega) + npy * omega);
  return c;
}
// One colour of the FP64 multicolour Gauss-Seidel sweep: colour (i&1)*2 + (j&1); with odd
// M the seam column i = M-1 is coloured 4 + (j&1) so no two points of a colour touch
// (9-point stencil, periodic in i).  Records the max vertex move (float bits).
__global__ void k_grid_multicolor_d(double2* __restrict__ V, int M, int N, int color, double omega, uint32_t* move) {
  int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  uint32_t mv = 0u;
  if (i < M && j >= 1 && j < N) {
    int col = ((M & 1) && i == M - 1) ? 4 + (j & 1) : (i & 1) * 2 + (j & 1);
    if (col == color) {
      double2 p = ttm_point_d(V, M, i, j, omega);
      double2 o = V[(size_t)j * M + i];
      mv = __float_as_uint((float)fmax(fabs(p.x - o.x), fabs(p.y - o.y)));
      V[(size_t)j * M + i] = p;
    }
  }
  block_max_to(move, mv);
}
__global__ void k_d2f(const double2* __restrict__ a, float2* __restrict__ b, size_t n) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    b[k] = make_float2((float)a[k].x, (float)a[k].y);
}
__global__ void k_f2d(const float2* __restrict__ a, double2* __restrict__ b, size_t n) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    b[k] = make_double2(a[k].x, a[k].y);
}

// Face records in FP64, rounded once to FP32 (shaders/grid.js:115-147 computes them in
// FP32 from FP32 vertices).  Mi[j][i]: face between cells (i-1, j) and (i, j), tangent
// V(i, j+1) - V(i, j), unit normal (-t.y, t.x), half its length (the fused flux takes
// twice the mass flux and pressure), and 1 / area of cell (i, j).  Mj[j][i],
// j = 0..N: face between cells (i, j-1) and (i, j), tangent V(i, j) - V(i+1, j),
// normal, half length, and for j < N the wave-speed factor
// (l_l + l_r + l_u + l_d) / (2 A) of cell (i, j) (ausm.js:617-630).
__global__ void k_metrics_d(const double2* __restrict__ V, float4* __restrict__ Mi, float4* __restrict__ Mj, int M,
                            int N) {
  int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= M || j > N) return;
  const int r = i + 1 == M ? 0 : i + 1;
  const double2 a = V[(size_t)j * M + i], b = V[(size_t)j * M + r];
  double tx = a.x - b.x, ty = a.y - b.y;
  double ld = sqrt(tx * tx + ty * ty);
  float w = 0.0f;
  if (j < N) {
    const double2 c = V[(size_t)(j + 1) * M + i], d = V[(size_t)(j + 1) * M + r];
    double ux = c.x - a.x, uy = c.y - a.y;
    double ll = sqrt(ux * ux + uy * uy);
    double lr = sqrt((d.x - b.x) * (d.x - b.x) + (d.y - b.y) * (d.y - b.y));
    double lu = sqrt((c.x - d.x) * (c.x - d.x) + (c.y - d.y) * (c.y - d.y));
    double A = 0.5 * fabs((d.x - a.x) * (c.y - b.y) - (c.x - b.x) * (d.y - a.y));
    w = (float)((ll + lr + lu + ld) / (2.0 * A));
    Mi[(size_t)j * M + i] = make_float4((float)(-uy / ll), (float)(ux / ll), (float)(0.5 * ll), (float)(1.0 / A));
  }
  Mj[(size_t)j * M + i] = make_float4((float)(-ty / ld), (float)(tx / ld), (float)(0.5 * ld), w);
}

// ---- surface force (graphs.js:5-41, summed as graphs.js:43-103): FP32 pressure of the first interior cell,
// FP64 face length, normal and sum; also Cp per wall face ----
__global__ void k_forces(const float4* __restrict__ row0, const double2* __restrict__ V, const Consts c, int M,
                         double* parts, double* cp, double q_inf, double p_inf) {
  double fx = 0.0, fy = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M; i += gridDim.x * blockDim.x) {
    float4 s = row0[i];
    float rho = s.x, u = s.y / rho, v = s.z / rho;
    float p = (s.w - 0.5f * rho * (u * u + v * v)) * (c.gamma - 1.0f);
    double2 a = V[i], b = V[(i + 1) % M];
    double dx = b.x - a.x, dy = b.y - a.y;
    double len = sqrt(dx * dx + dy * dy);
    double nx = dy / len, ny = -dx / len;  // (vtx2.y - vtx1.y, vtx1.x - vtx2.x) / length
    fx += -(double)p * len * nx;
    fy += -(double)p * len * ny;
    if (cp) cp[i] = ((double)p - p_inf) / q_inf;
  }
  block_sum_store(parts + blockIdx.x, fx);
  __syncthreads();
  block_sum_store(parts + kMaxParts + blockIdx.x, fy);
}

__global__ void k_sumsq_rho(const float4* __restrict__ R, size_t n, double* parts) {
  double s = 0.0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    double r = R[k].x;
    s += r * r;
  }
  block_sum_store(parts + blockIdx.x, s);
}

// out[q] = sum of parts[q * kMaxParts + 0 .. nb - 1], in a fixed order (one block of
// 256 threads per quantity q: strided partial sums, then a shared-memory tree).
__global__ void k_sum_parts(const double* __restrict__ parts, int nb, double* __restrict__ out) {
  __shared__ double sh[256];
  const int t = threadIdx.x;
  const double* p = parts + (size_t)blockIdx.x * kMaxParts;
  double a = 0.0;
  for (int k = t; k < nb; k += 256) a += p[k];
  sh[t] = a;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (t < w) sh[t] += sh[t + w];
    __syncthreads();
  }
  if (t == 0) out[blockIdx.x] = sh[0];
}

// ---- headless field output (ausm.js:617-707 without the colour map) ----
__global__ void k_field(const float4* __restrict__ Q, const float2* __restrict__ V, const Consts c, int kind, int M,
                        int N, float* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= M || j >= N) return;
  size_t k = (size_t)j * M + i;
  float4 s = Q[k];
  float rho = s.x, u = s.y / rho, v = s.z / rho;
  float p = (s.w - 0.5f * rho * (u * u + v * v)) * (c.gamma - 1.0f);
  float T = p / rho;
  float a = sqrtf(c.gamma * T);
  float speed = sqrtf(u * u + v * v);
  float r;
  switch (kind) {
    case 0: r = rho; break;
    case 1: r = p; break;
    case 2: r = T; break;
    case 3: r = speed / a; break;
    case 4: r = logf(p / powf(rho, c.gamma)); break;
    default: {
      int rr = (i + 1) % M;
      float2 A = V[k], B = V[(size_t)j * M + rr], C = V[(size_t)(j + 1) * M + i], D = V[(size_t)(j + 1) * M + rr];
      float ll = sqrtf((A.x - C.x) * (A.x - C.x) + (A.y - C.y) * (A.y - C.y));
      float lr = sqrtf((B.x - D.x) * (B.x - D.x) + (B.y - D.y) * (B.y - D.y));
      float lu = sqrtf((C.x - D.x) * (C.x - D.x) + (C.y - D.y) * (C.y - D.y));
      float ld = sqrtf((A.x - B.x) * (A.x - B.x) + (A.y - B.y) * (A.y - B.y));
      r = wave_speed<false>(s, ((ll + lr) + lu) + ld, quad_area(A, B, C, D), c.gamma);
    }
  }
  out[k] = r;
}

// ---- launchers ----
static inline dim3 grid16(int w, int h) { return dim3((w + 15) / 16, (h + 15) / 16); }
static const dim3 B16(16, 16);
static inline int grid1d(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }

void launch_to_ref_layout(const float4* Qint, float4* ref, const float2* V, const Consts& c, int M, int N,
                          cudaStream_t s) {
  k_to_ref_layout<<<grid16(M, N + 3), B16, 0, s>>>(Qint, ref, V, c, M, N);
}
void launch_from_ref_layout(const float4* ref, float4* Qint, int M, int N, cudaStream_t s) {
  size_t n = (size_t)M * N;
  k_from_ref_layout<<<grid1d(n), 256, 0, s>>>(ref, Qint, n, M);
}
void launch_fill(float4* Q, float4 v, size_t n, cudaStream_t s) { k_fill<<<grid1d(n), 256, 0, s>>>(Q, v, n); }
void launch_grid_init(float2* V, int M, int N, double first_spacing, cudaStream_t s) {
  k_grid_init<<<grid16(M, N + 1), B16, 0, s>>>(V, M, N, first_spacing);
}
void launch_grid_jacobi(const float2* src, float2* dst, int M, int N, cudaStream_t s) {
  k_grid_jacobi<<<grid16(M, N + 1), B16, 0, s>>>(src, dst, M, N);
}
void launch_forces(const float4* row0, const double2* V, const Consts& c, int M, double* acc, double* parts,
                   double* cp, double q_inf, double p_inf, cudaStream_t s) {
  int blocks = std::min((M + 255) / 256, 148);
  k_forces<<<blocks, 256, 0, s>>>(row0, V, c, M, parts, cp, q_inf, p_inf);
  k_sum_parts<<<2, 256, 0, s>>>(parts, blocks, acc);
}
void launch_sumsq_rho(const float4* R, size_t n, double* acc, double* parts, cudaStream_t s) {
  const int blocks = grid1d(n);  // <= kMaxParts
  k_sumsq_rho<<<blocks, 256, 0, s>>>(R, n, parts);
  k_sum_parts<<<1, 256, 0, s>>>(parts, blocks, acc);
}
void launch_grid_init_d(double2* V, int M, int N, double first_spacing, cudaStream_t s) {
  k_grid_init_d<<<grid16(M, N + 1), B16, 0, s>>>(V, M, N, first_spacing);
}
void launch_grid_multicolor_d(double2* V, int M, int N, int color, double omega, uint32_t* move, cudaStream_t s) {
  k_grid_multicolor_d<<<grid16(M, N + 1), B16, 0, s>>>(V, M, N, color, omega, move);
}
void launch_d2f(const double2* a, float2* b, size_t n, cudaStream_t s) { k_d2f<<<grid1d(n), 256, 0, s>>>(a, b, n); }
void launch_f2d(const float2* a, double2* b, size_t n, cudaStream_t s) { k_f2d<<<grid1d(n), 256, 0, s>>>(a, b, n); }
void launch_metrics_d(const double2* V, float4* Mi, float4* Mj, int M, int N, cudaStream_t s) {
  k_metrics_d<<<grid16(M, N + 1), B16, 0, s>>>(V, Mi, Mj, M, N);
}
void launch_sum_parts(const double* parts, int nb, int nq, double* out, cudaStream_t s) {
  k_sum_parts<<<nq, 256, 0, s>>>(parts, nb, out);
}
void launch_field(const float4* Qint, const float2* V, const Consts& c, int kind, int M, int N, float* out,
                  cudaStream_t s) {
  k_field<<<grid16(M, N), B16, 0, s>>>(Qint, V, c, kind, M, N, out);
}

}  // namespace ausm
