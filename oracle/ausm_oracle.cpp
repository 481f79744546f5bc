// ORACLE — test infrastructure only.
//
// CPU restatement of the explicit TVD-RK3 time step of the AUSM-family O-grid
// Euler solver (huj31415/ausm-webgpu), written from the reference's WGSL
// shaders and host dispatch order.  It is the checker for the CUDA library: only
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
// It is never the product path.
//
// Every expression keeps the reference's operation order so that, built with
// -ffp-contract=off (no fused multiply-add), the float instantiation reproduces the
// reference arithmetic bit for bit in IEEE single precision.  The double
// instantiation is the FP64 oracle of the precision study.
//
// Parity pin: oracle/wgsl_ref/ compiles the reference's own WGSL source for the CPU
// (mechanical WGSL->C++ translation of src/shaders/*.js, never committed); the
// golden fixtures in tests/golden/ come from that build, and tests check this file
// against them bit-exactly in float.
//
// Layout (reference, main.js:110-125, util.js:51-54):
//   vertices  float2  M x (N+1)   row j=0 body, j=N outer, i wraps mod M (no seam copy)
//   state     float4  M x (N+3)   row 0 wall ghost, rows 1..N interior, N+1,N+2 far field
//   area      float   M x N;  face lengths float4 (left,right,up,down) M x N
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

template <class T> struct V2 { T x, y; };
template <class T> struct V4 { T x, y, z, w; };

// WGSL builtins with the reference's semantics (WGSL spec definitions).
template <class T> inline T wmax(T a, T b) { return std::fmax(a, b); }
template <class T> inline T wmin(T a, T b) { return std::fmin(a, b); }
template <class T> inline T wclamp01(T e) { return wmin(wmax(e, T(0)), T(1)); }  // saturate
template <class T> inline T wsign(T e) { return e > T(0) ? T(1) : (e < T(0) ? T(-1) : T(0)); }
template <class T> inline T wstep(T edge, T x) { return edge <= x ? T(1) : T(0); }
template <class T> inline T wmix(T a, T b, T t) { return a * (T(1) - t) + b * t; }
template <class T> inline T dot2(V2<T> a, V2<T> b) { return a.x * b.x + a.y * b.y; }
template <class T> inline T len2(V2<T> a) { return std::sqrt(dot2(a, a)); }
template <class T> inline V2<T> normalize2(V2<T> a) {
  T l = len2(a);
  return {a.x / l, a.y / l};
}
template <class T> inline V2<T> sub2(V2<T> a, V2<T> b) { return {a.x - b.x, a.y - b.y}; }

struct OrcParams {  // mirrors the reference uniform fields used on the path (util.js:1-29)
  double gamma, in_rho, in_pressure;
  double inflow[2];    // uni.inflowV
  double in_state[4];  // uni.inState
  double K_p, K_u, cfl, maxdt;
  int muscl;           // uni.muscl > 0 enables MUSCL (ausm.js:240)
  int scheme;          // 0 SLAU2, 1 SLAU, 2 AUSM+-up (util.js:114-118)
};

template <class T> struct Oracle {
  int M, N;
  std::vector<T> vtx;     // M*(N+1)*2
  std::vector<T> area;    // M*N
  std::vector<T> flen;    // M*N*4
  std::vector<T> q;       // M*(N+3)*4, current state ("state2" of main.js)
  std::vector<T> qn, q1, qs, fx, fy, res, ws;  // work arrays
  T gamma = T(1.4), inRho = T(1), inP = T(1.0 / 1.4), Kp = T(0), Ku = T(0.75), cfl = T(1.5),
    maxdt = T(1e-4);
  V2<T> inflow{T(0), T(0)};
  V4<T> inState{T(0), T(0), T(0), T(0)};
  int muscl = 1, scheme = 0;
  T maxWave = T(0);

  Oracle(int M_, int N_) : M(M_), N(N_) {
    vtx.assign((size_t)M * (N + 1) * 2, T(0));
    area.assign((size_t)M * N, T(0));
    flen.assign((size_t)M * N * 4, T(0));
    size_t ns = (size_t)M * (N + 3) * 4;
    q.assign(ns, T(0)); qn = q1 = qs = q;
    fx.assign((size_t)M * N * 4, T(0));
    fy.assign((size_t)M * (N + 1) * 4, T(0));
    res.assign((size_t)M * N * 4, T(0));
    ws.assign((size_t)M * N, T(0));
  }

  void set_params(const OrcParams& p) {
    gamma = T(p.gamma); inRho = T(p.in_rho); inP = T(p.in_pressure);
    inflow = {T(p.inflow[0]), T(p.inflow[1])};
    inState = {T(p.in_state[0]), T(p.in_state[1]), T(p.in_state[2]), T(p.in_state[3])};
    Kp = T(p.K_p); Ku = T(p.K_u); cfl = T(p.cfl); maxdt = T(p.maxdt);
    muscl = p.muscl; scheme = p.scheme;
  }

  V2<T> V(int i, int j) const {
    size_t k = ((size_t)j * M + i) * 2;
    return {vtx[k], vtx[k + 1]};
  }
  static V4<T> ld4(const std::vector<T>& a, size_t cell) {
    const T* p = &a[cell * 4];
    return {p[0], p[1], p[2], p[3]};
  }
  static void st4(std::vector<T>& a, size_t cell, V4<T> v) {
    T* p = &a[cell * 4];
    p[0] = v.x; p[1] = v.y; p[2] = v.z; p[3] = v.w;
  }

  // ---- grid finalize: cell area and face lengths (shaders/grid.js:115-147) ----
  void metrics() {
#pragma omp parallel for schedule(static)
    for (int j = 0; j < N; j++)
      for (int i = 0; i < M; i++) {
        int r = (i + 1) % M;
        V2<T> a = V(i, j), b = V(r, j), c = V(i, j + 1), d = V(r, j + 1);
        size_t k = (size_t)j * M + i;
        area[k] = T(0.5) * std::fabs((d.x - a.x) * (c.y - b.y) - (c.x - b.x) * (d.y - a.y));
        flen[k * 4 + 0] = len2(sub2(a, c));  // left
        flen[k * 4 + 1] = len2(sub2(b, d));  // right
        flen[k * 4 + 2] = len2(sub2(c, d));  // up
        flen[k * 4 + 3] = len2(sub2(a, b));  // down
      }
  }

  // ---- initial state (ausm.js:1-17 at rest; freestream = uni.inState, main.js:783-784) ----
  void init_state(int mode) {
    V4<T> s;
    if (mode == 0) s = {inRho, T(0), T(0), inP / (gamma - T(1))};
    else s = inState;
    for (size_t c = 0; c < (size_t)M * (N + 3); c++) st4(q, c, s);
    wave_speed_max(q);
  }

  // ---- ghost cells (ausm.js:34-120): returns the full array with ghost rows filled ----
  void boundary(const std::vector<T>& in, std::vector<T>& out) {
    if (&in != &out) out = in;  // pass-through copy (ausm.js:55)
    const T g = gamma;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < M; i++) {
      int r = (i + 1) % M;
      {  // object boundary: row 0 reflects row 1 about the wall normal (ausm.js:57-64)
        V2<T> t = normalize2(sub2(V(i, 0), V(r, 0)));
        V2<T> n{-t.y, t.x};
        V4<T> s = ld4(in, (size_t)1 * M + i);
        T rho = s.x;
        V2<T> u{s.y / rho, s.z / rho};
        T dn = T(2) * dot2(n, u);
        V2<T> gu{u.x - dn * n.x, u.y - dn * n.y};
        st4(out, i, V4<T>{rho, gu.x * rho, gu.y * rho, s.w});
      }
      // outer boundary: rows N+1, N+2 from row N (ausm.js:65-117)
      V2<T> t = normalize2(sub2(V(i, N), V(r, N)));
      V2<T> n{-t.y, t.x};
      V4<T> s = ld4(in, (size_t)N * M + i);
      T rho = s.x;
      V2<T> u{s.y / rho, s.z / rho};
      T inout = dot2(n, inflow);
      V4<T> g1, g2;
      if (inout < T(0)) {
        g1 = g2 = inState;
      } else {
        T gm1inv = T(1) / (g - T(1));
        T u2 = dot2(u, u);
        T P = (s.w - T(0.5) * u2 * rho) * (g - T(1));
        T a2 = (g * P) / rho;
        T a2inf = (g * inP / inRho);
        T Mint = u2 / a2;
        T Minf2 = dot2(inflow, inflow) / a2inf;
        if (Mint < T(1) && Minf2 < T(1)) {
          T un_int = dot2(u, n);
          T un_inf = inout;
          T a_int = std::sqrt(a2), a_inf = std::sqrt(a2inf);
          T J_int = un_int + T(2) * a_int * gm1inv;
          T J_ext = un_inf - T(2) * a_inf * gm1inv;
          T un_g = T(0.5) * (J_int + J_ext);
          T a_g = wmax(a_int * T(0.1), T(0.25) * (J_int - J_ext) * (g - T(1)));
          T X = wmax(T(1e-6), a_g / a_int);
          T X2 = X * X;
          T rho_g = wmax(T(1e-6), rho * X2 * X2 * X);
          T dun = un_g - un_int;
          V2<T> vg{dun * n.x + u.x, dun * n.y + u.y};
          T E_g = wmax(T(1e-6), (rho_g * a_g * a_g) / g) * gm1inv + T(0.5) * rho_g * dot2(vg, vg);
          g1 = {rho_g, vg.x * rho_g, vg.y * rho_g, E_g};
        } else if (Minf2 > T(1)) {
          T ambE = inP / (g - T(1)) + T(0.5) * rho * u2;
          g1 = {s.x, s.y, s.z, ambE};
        } else {
          g1 = s;
        }
        g2 = {T(2) * g1.x - s.x, T(2) * g1.y - s.y, T(2) * g1.z - s.z, T(2) * g1.w - s.w};
      }
      st4(out, (size_t)(N + 1) * M + i, g1);
      st4(out, (size_t)(N + 2) * M + i, g2);
    }
  }

  // loadState (ausm.js:138-143): i wraps, interior index shifted by +1, clamped at the wall ghost
  V4<T> load(const std::vector<T>& Q, int i, int j) const {
    int ii = (i + M) % M;
    int jj = std::max(j + 1, 0);
    return ld4(Q, (size_t)jj * M + ii);
  }
  // toPrimitive (ausm.js:145-150)
  V4<T> prim(V4<T> Q) const {
    T rho = Q.x;
    T u = Q.y / rho, v = Q.z / rho;
    T p = wmax(T(1e-7), (Q.w - T(0.5) * rho * (u * u + v * v)) * (gamma - T(1)));
    return {rho, u, v, p};
  }
  static T vanAlbada(T r) {  // ausm.js:168-171
    T r2 = r * r;
    return (r2 + r) / (r2 + T(1));
  }

  // One face: MUSCL interface states (ausm.js:201-266) and the selected flux.
  V4<T> face_flux(V4<T> QL2, V4<T> QL, V4<T> QR, V4<T> QR2, V2<T> n) const {
    const T gm1 = gamma - T(1);
    const T eps = T(1e-6);
    V4<T> L2 = prim(QL2), L = prim(QL), R = prim(QR), R2 = prim(QR2);
    V4<T> Lm = L, Rm = R;
    if (muscl > 0) {
      T* pl2 = &L2.x; T* pl = &L.x; T* pr = &R.x; T* pr2 = &R2.x; T* ol = &Lm.x; T* orr = &Rm.x;
      for (int k = 0; k < 4; k++) {
        T dL = pl[k] - pl2[k], dF = pr[k] - pl[k], dR = pr2[k] - pr[k];
        T rL = (dL * dF + eps) / (dF * dF + eps);
        T rR = (dF * dR + eps) / (dF * dF + eps);
        ol[k] = ol[k] + T(0.5) * vanAlbada(rL) * dF;
        orr[k] = orr[k] - T(0.5) * vanAlbada(rR) * dF;
      }
    }
    T rhoL = Lm.x, rhoR = Rm.x;
    V2<T> vL{Lm.y, Lm.z}, vR{Rm.y, Rm.z};
    T uL = dot2(vL, n), uR = dot2(vR, n);
    T pL = Lm.w, pR = Rm.w;
    T hL = pL / (gm1 * rhoL) + T(0.5) * dot2(vL, vL) + pL / rhoL;
    T hR = pR / (gm1 * rhoR) + T(0.5) * dot2(vR, vR) + pR / rhoR;
    T mdot, P;
    if (scheme == 2) {  // AUSM+-up (ausm.js:271-336)
      T Minf2 = dot2(inflow, inflow) / (gamma * inP / rhoL);
      T sigma = T(1);
      T ht = T(0.5) * (hL + hR);
      T aStar = std::sqrt(wmax(T(1e-6), T(2) * gm1 / (gamma + T(1)) * ht));
      T aHL = aStar * aStar / wmax(uL, aStar);
      T aHR = aStar * aStar / wmax(-uR, aStar);
      T a = wmin(aHL, aHR);
      T ML = uL / a, MR = uR / a;
      T a2 = a * a;
      T Mbar2 = (uL * uL + uR * uR) / (a2 * T(2));
      T Mo2 = wmin(T(1), wmax(Mbar2, Minf2));
      T fa = Mo2 * (T(2) - Mo2);
      T rhoI = T(0.5) * (rhoL + rhoR);
      T Mp1L = ML + T(1), Mp1R = MR + T(1);
      T Mm1L = ML - T(1), Mm1R = MR - T(1);
      T M2pL = T(0.25) * Mp1L * Mp1L, M2pR = T(0.25) * Mp1R * Mp1R;
      T M2mL = T(-0.25) * Mm1L * Mm1L, M2mR = T(-0.25) * Mm1R * Mm1R;
      T M4subL = M2pL * (T(1) + T(2) * M2mL);
      T M4subR = M2mR * (T(1) - T(2) * M2pR);
      T supL = wstep(T(1), std::fabs(ML)), supR = wstep(T(1), std::fabs(MR));
      T M4L = wmix(M4subL, wmax(T(0), ML), supL);
      T M4R = wmix(M4subR, wmin(T(0), MR), supR);
      T Mi = M4L + M4R - Kp / fa * wmax(T(1) - sigma * Mbar2, T(0)) * (pR - pL) / (rhoI * a2);
      T alpha4 = T(0.75) * (T(-4) + T(5) * fa * fa);
      T P5subL = M2pL * ((T(2) - ML) + alpha4 * ML * M2mL);
      T P5subR = M2mR * ((T(-2) - MR) - alpha4 * MR * M2pR);
      T P5L = wmix(P5subL, wstep(T(0), ML), supL);
      T P5R = wmix(P5subR, wstep(T(0), -MR), supR);
      P = (P5L * pL + P5R * pR) - Ku * P5L * P5R * (rhoL + rhoR) * fa * a * (uR - uL);
      mdot = a * Mi * (Mi > T(0) ? rhoL : rhoR);
    } else {  // SLAU2 / SLAU (ausm.js:345-392)
      T aL = std::sqrt(gamma * wmax(pL, T(1e-10)) / wmax(rhoL, T(1e-10)));
      T aR = std::sqrt(gamma * wmax(pR, T(1e-10)) / wmax(rhoR, T(1e-10)));
      T a = (aL + aR) * T(0.5);
      T ML = uL / a, MR = uR / a;
      T Uarc = std::sqrt(T(0.5) * (dot2(vL, vL) + dot2(vR, vR)));
      T Marc = wmin(T(1), Uarc / a);
      T X = (T(1) - Marc) * (T(1) - Marc);
      T mpL = ML + T(1), mmR = MR - T(1);
      T sqL = T(0.5) * mpL * mpL, sqR = T(0.5) * mmR * mmR;
      T supL = wstep(T(1), std::fabs(ML)), supR = wstep(T(1), std::fabs(MR));
      T fpp = wclamp01(T(0.5) * wmix(sqL * (T(2) - T(1) * ML), T(1) + T(1) * wsign(ML), supL));
      T fpm = wclamp01(T(0.5) * wmix(sqR * (T(2) - T(-1) * MR), T(1) + T(-1) * wsign(MR), supR));
      if (scheme == 0)
        P = T(0.5) * ((fpp - fpm) * (pL - pR) + (pL + pR) + (Uarc * (fpp + fpm - T(1)) * (rhoL + rhoR) * a));
      else
        P = T(0.5) * ((fpp - fpm) * (pL - pR) + (T(1) + (T(1) - X) * (fpp + fpm - T(1))) * (pL + pR));
      T dp = pR - pL;
      T ubar = (rhoL * std::fabs(uL) + rhoR * std::fabs(uR)) / (rhoL + rhoR);
      T gg = wclamp01(-ML) * wclamp01(MR);
      T ubp = wmix(ubar, std::fabs(uL), gg);
      T ubm = wmix(ubar, std::fabs(uR), gg);
      mdot = T(0.5) * ((rhoL * (uL + ubp) + rhoR * (uR - ubm)) * (T(1) - gg) - X / a * dp);
    }
    // phi * mdot + (0, n*P, 0)  (ausm.js:329-334, 386-391)
    bool left = mdot > T(0);
    T p0 = T(1), p1 = left ? vL.x : vR.x, p2 = left ? vL.y : vR.y, p3 = left ? hL : hR;
    return {p0 * mdot + T(0), p1 * mdot + n.x * P, p2 * mdot + n.y * P, p3 * mdot + T(0)};
  }

  // vertical (j-) faces: M x (N+1), face (i,j) lies below interior cell (i,j)
  void flux_j(const std::vector<T>& Q) {
#pragma omp parallel for schedule(static)
    for (int j = 0; j <= N; j++)
      for (int i = 0; i < M; i++) {
        V2<T> t = normalize2(sub2(V(i, j), V((i + 1) % M, j)));
        V2<T> n{-t.y, t.x};
        V4<T> f = face_flux(load(Q, i, j - 2), load(Q, i, j - 1), load(Q, i, j), load(Q, i, j + 1), n);
        st4(fy, (size_t)j * M + i, f);
      }
  }
  // horizontal (i-) faces: face (i,j) lies left of interior cell (i,j); the reference's
  // extra column i=M is never read (ausm.js:420) and is not computed here.
  void flux_i(const std::vector<T>& Q) {
#pragma omp parallel for schedule(static)
    for (int j = 0; j < N; j++)
      for (int i = 0; i < M; i++) {
        V2<T> t = normalize2(sub2(V(i, j + 1), V(i, j)));
        V2<T> n{-t.y, t.x};
        V4<T> f = face_flux(load(Q, i - 2, j), load(Q, i - 1, j), load(Q, i, j), load(Q, i + 1, j), n);
        st4(fx, (size_t)j * M + i, f);
      }
  }
  // residual (ausm.js:415-436)
  void residual() {
#pragma omp parallel for schedule(static)
    for (int j = 0; j < N; j++)
      for (int i = 0; i < M; i++) {
        size_t k = (size_t)j * M + i;
        int r = (i + 1) % M;
        const T* xl = &fx[k * 4];
        const T* xr = &fx[((size_t)j * M + r) * 4];
        const T* yu = &fy[((size_t)(j + 1) * M + i) * 4];
        const T* yd = &fy[k * 4];
        T lf = flen[k * 4 + 0], rf = flen[k * 4 + 1], uf = flen[k * 4 + 2], df = flen[k * 4 + 3];
        T A = area[k];
        for (int c = 0; c < 4; c++)
          res[k * 4 + c] = -(xr[c] * rf - xl[c] * lf + yu[c] * uf - yd[c] * df) / A;
      }
  }
  void eval_residual(const std::vector<T>& Q) {
    boundary(Q, qs);
    flux_j(qs);
    flux_i(qs);
    residual();
  }

  // wave speed (ausm.js:617-630) + max reduction (ausm.js:535-581): max is order-free
  T wave_speed_max(const std::vector<T>& Q) {
    T m = T(0);
#pragma omp parallel for schedule(static) reduction(max : m)
    for (int j = 0; j < N; j++)
      for (int i = 0; i < M; i++) {
        size_t k = (size_t)j * M + i;
        V4<T> s = ld4(Q, (size_t)(j + 1) * M + i);
        T rho = s.x;
        V2<T> vel{s.y / rho, s.z / rho};
        T p = (s.w - T(0.5) * rho * dot2(vel, vel)) * (gamma - T(1));
        T temp = p / rho;
        T a = std::sqrt(gamma * temp);
        T speed = len2(vel);
        T fsum = flen[k * 4 + 0] + flen[k * 4 + 1] + flen[k * 4 + 2] + flen[k * 4 + 3];
        T w = (speed + a) * fsum / (T(2) * area[k]);
        ws[k] = w;
        m = wmax(m, w);
      }
    maxWave = m;
    return m;
  }

  T dt() const { return wmin(maxdt, cfl / maxWave); }

  // One TVD-RK3 step (ausm.js:441-527, dispatch order main.js:744-777), interior rows only.
  void rk3(T dt) {
    const size_t off = (size_t)M * 4;  // skip wall ghost row
    const size_t n = (size_t)M * N * 4;
    qn = q;
    eval_residual(qn);
    q1 = qn;
#pragma omp parallel for schedule(static)
    for (long long x = 0; x < (long long)n; x++) q1[off + x] = qn[off + x] + dt * res[x];
    eval_residual(q1);
    std::vector<T>& q2 = q;  // reuse
    q2 = q1;
#pragma omp parallel for schedule(static)
    for (long long x = 0; x < (long long)n; x++)
      q2[off + x] = T(0.75) * qn[off + x] + T(0.25) * (q1[off + x] + dt * res[x]);
    eval_residual(q2);
#pragma omp parallel for schedule(static)
    for (long long x = 0; x < (long long)n; x++)
      q[off + x] = (qn[off + x] + T(2) * (q2[off + x] + dt * res[x])) / T(3);
  }

  // step(n): dt fixed from the state at entry (main.js:744-791), refreshed after the n steps.
  T step(int nsteps) {
    T d = dt();
    for (int s = 0; s < nsteps; s++) rk3(d);
    wave_speed_max(q);
    return d;
  }

  // surface force (graphs.js:5-41) and its 256-lane tree sum (graphs.js:43-103)
  void forces(double* out /* Fx, Fy, |F|sign(F.V), Cl, Cd, Cl/Cd */) {
    std::vector<V2<T>> f(M);
    for (int i = 0; i < M; i++) {
      V4<T> s = ld4(q, (size_t)1 * M + i);
      T rho = s.x;
      V2<T> vel{s.y / rho, s.z / rho};
      T p = (s.w - T(0.5) * rho * dot2(vel, vel)) * (gamma - T(1));
      V2<T> v1 = V(i, 0), v2 = V((i + 1) % M, 0);
      T fl = len2(sub2(v2, v1));
      V2<T> nn{(v2.y - v1.y) / fl, (v1.x - v2.x) / fl};
      T pf = p * fl;
      f[i] = {pf * -nn.x, pf * -nn.y};
    }
    V2<T> lane[256];
    for (int l = 0; l < 256; l++) {
      V2<T> acc{T(0), T(0)};
      for (int i = l; i < M; i += 256) { acc.x = acc.x + f[i].x; acc.y = acc.y + f[i].y; }
      lane[l] = acc;
    }
    for (int s = 128; s > 0; s >>= 1)
      for (int l = 0; l < s; l++) { lane[l].x = lane[l].x + lane[l + s].x; lane[l].y = lane[l].y + lane[l + s].y; }
    V2<T> F = lane[0];
    V2<T> vN = normalize2(inflow);
    T invQ = T(1) / (T(0.5) * inRho * dot2(inflow, inflow));
    T Cl = dot2(F, V2<T>{-vN.y, vN.x}) * invQ;
    T Cd = dot2(F, vN) * invQ;
    out[0] = (double)F.x; out[1] = (double)F.y;
    out[2] = (double)(len2(F) * wsign(dot2(F, vN)));
    out[3] = (double)Cl; out[4] = (double)Cd; out[5] = (double)(Cl / Cd);
  }

  // ---- grid generation (shaders/grid.js:4-110, driver main.js:658-699) ----
  // Linear interpolation in j between body (row 0) and outer (row N) vertices.
  void grid_interpolate() {
    const std::vector<T> src = vtx;  // the shader reads gridPoints0 and writes gridPoints1
    auto P = [&](int ii, int jj) { size_t k = ((size_t)jj * M + ii) * 2; return V2<T>{src[k], src[k + 1]}; };
    for (int j = 0; j <= N; j++) {
      T t = T(j) / T(N);
      for (int i = 0; i < M; i++) {
        V2<T> a = P(i, 0), b = P(i, N);
        size_t k = ((size_t)j * M + i) * 2;
        vtx[k] = wmix(a.x, b.x, t);
        vtx[k + 1] = wmix(a.y, b.y, t);
      }
    }
  }
  // TTM/Winslow update of one vertex from the source array (P=Q=0, omega=1, only if jac<0)
  V2<T> ttm_point(const std::vector<T>& s, int i, int j) const {
    auto P = [&](int ii, int jj) { size_t k = ((size_t)jj * M + ii) * 2; return V2<T>{s[k], s[k + 1]}; };
    int l = i == 0 ? M - 1 : i - 1;
    int r = i == M - 1 ? 0 : i + 1;
    int u = j + 1, d = j - 1;
    V2<T> c = P(i, j), L = P(l, j), R = P(r, j), D = P(i, d), U = P(i, u);
    V2<T> DL = P(l, d), DR = P(r, d), UL = P(l, u), UR = P(r, u);
    V2<T> xi{T(0.5) * (R.x - L.x), T(0.5) * (R.y - L.y)};
    V2<T> eta{T(0.5) * (U.x - D.x), T(0.5) * (U.y - D.y)};
    V2<T> xe{T(0.25) * (UR.x + DL.x - UL.x - DR.x), T(0.25) * (UR.y + DL.y - UL.y - DR.y)};
    T alpha = dot2(eta, eta), gam = dot2(xi, xi), beta = dot2(xi, eta);
    const T Pc = T(0), Qc = T(0), omega = T(1);
    T den = T(2) * (alpha + gam);
    V2<T> np{(alpha * (L.x + R.x + Pc * xi.x) + gam * (D.x + U.x + Qc * eta.x) - T(2) * beta * xe.x) / den,
             (alpha * (L.y + R.y + Pc * xi.y) + gam * (D.y + U.y + Qc * eta.y) - T(2) * beta * xe.y) / den};
    T jac = xi.x * eta.y - xi.y * eta.x;
    if (jac < T(0)) return V2<T>{wmix(c.x, np.x, omega), wmix(c.y, np.y, omega)};
    return c;
  }
  // Jacobi sweeps with ping-pong buffers; rows 0 and N are fixed.  Returns the final
  // iterate in vtx and (if prev != nullptr) the previous iterate.
  void grid_jacobi(int iters, std::vector<T>* prev) {
    std::vector<T> a = vtx, b = vtx;
    std::vector<T>* src = &a; std::vector<T>* dst = &b;
    for (int it = 0; it < iters; it++) {
#pragma omp parallel for schedule(static)
      for (int j = 1; j < N; j++)
        for (int i = 0; i < M; i++) {
          V2<T> p = ttm_point(*src, i, j);
          size_t k = ((size_t)j * M + i) * 2;
          (*dst)[k] = p.x; (*dst)[k + 1] = p.y;
        }
      std::swap(src, dst);
    }
    if (prev) *prev = *dst;
    vtx = *src;
  }
  // Multicolour Gauss-Seidel (new, not in the reference): four colours (i&1, j&1) decouple
  // the 9-point stencil; when M is odd the seam column i=M-1 gets its own two colours.
  // Sweeps until the max vertex move is <= tol or iters is reached; returns sweeps done.
  int grid_multicolor(int iters, T tol, T* last_move) {
    int odd = M & 1;
    int sweeps = 0;
    T mv = T(0);
    for (int it = 0; it < iters; it++) {
      mv = T(0);
      int ncol = odd ? 6 : 4;
      for (int c = 0; c < ncol; c++) {
        // the points of one colour do not touch each other: any order gives the same result
        T cmv = T(0);
#pragma omp parallel for schedule(static) reduction(max : cmv)
        for (int j = 1; j < N; j++)
          for (int i = 0; i < M; i++) {
            int col;
            if (odd && i == M - 1) col = 4 + (j & 1);
            else col = (i & 1) * 2 + (j & 1);
            if (col != c) continue;
            V2<T> p = ttm_point(vtx, i, j);
            size_t k = ((size_t)j * M + i) * 2;
            T d = wmax(std::fabs(p.x - vtx[k]), std::fabs(p.y - vtx[k + 1]));
            cmv = wmax(cmv, d);
            vtx[k] = p.x; vtx[k + 1] = p.y;
          }
        mv = wmax(mv, cmv);
      }
      sweeps++;
      if (mv <= tol) break;
    }
    if (last_move) *last_move = mv;
    return sweeps;
  }
  // density-residual L2 norm sqrt(mean(R_rho^2)) of the current state (new, FP64 sum)
  double residual_l2() {
    eval_residual(q);
    double s = 0;
    for (size_t k = 0; k < (size_t)M * N; k++) s += (double)res[k * 4] * (double)res[k * 4];
    return std::sqrt(s / ((double)M * N));
  }
};

template <class T> Oracle<T>* O(void* h) { return static_cast<Oracle<T>*>(h); }

}  // namespace

#define ORC_API(SUF, T)                                                                          \
  extern "C" void* orc_create_##SUF(int M, int N) { return new Oracle<T>(M, N); }                \
  extern "C" void orc_destroy_##SUF(void* h) { delete O<T>(h); }                                 \
  extern "C" void orc_set_params_##SUF(void* h, const OrcParams* p) { O<T>(h)->set_params(*p); } \
  extern "C" void orc_set_vertices_##SUF(void* h, const T* xy) {                                 \
    auto* o = O<T>(h); std::memcpy(o->vtx.data(), xy, o->vtx.size() * sizeof(T));               \
  }                                                                                              \
  extern "C" void orc_get_vertices_##SUF(void* h, T* xy) {                                       \
    auto* o = O<T>(h); std::memcpy(xy, o->vtx.data(), o->vtx.size() * sizeof(T));               \
  }                                                                                              \
  extern "C" void orc_metrics_##SUF(void* h) { O<T>(h)->metrics(); }                             \
  extern "C" void orc_get_metrics_##SUF(void* h, T* area, T* flen) {                             \
    auto* o = O<T>(h);                                                                           \
    if (area) std::memcpy(area, o->area.data(), o->area.size() * sizeof(T));                     \
    if (flen) std::memcpy(flen, o->flen.data(), o->flen.size() * sizeof(T));                     \
  }                                                                                              \
  extern "C" void orc_init_state_##SUF(void* h, int mode) { O<T>(h)->init_state(mode); }         \
  extern "C" void orc_set_state_##SUF(void* h, const T* q) {                                     \
    auto* o = O<T>(h); std::memcpy(o->q.data(), q, o->q.size() * sizeof(T));                     \
    o->wave_speed_max(o->q);                                                                     \
  }                                                                                              \
  extern "C" void orc_get_state_##SUF(void* h, T* q) {                                           \
    auto* o = O<T>(h); std::memcpy(q, o->q.data(), o->q.size() * sizeof(T));                     \
  }                                                                                              \
  extern "C" void orc_fill_ghosts_##SUF(void* h) { auto* o = O<T>(h); o->boundary(o->q, o->q); } \
  extern "C" double orc_step_##SUF(void* h, int n) { return (double)O<T>(h)->step(n); }          \
  extern "C" double orc_max_wave_##SUF(void* h) { return (double)O<T>(h)->maxWave; }             \
  extern "C" void orc_get_wave_speeds_##SUF(void* h, T* w) {                                     \
    auto* o = O<T>(h); std::memcpy(w, o->ws.data(), o->ws.size() * sizeof(T));                   \
  }                                                                                              \
  extern "C" void orc_eval_residual_##SUF(void* h, T* r) {                                       \
    auto* o = O<T>(h); o->eval_residual(o->q);                                                   \
    std::memcpy(r, o->res.data(), o->res.size() * sizeof(T));                                   \
  }                                                                                              \
  extern "C" void orc_get_fluxes_##SUF(void* h, T* fx, T* fy) {                                  \
    auto* o = O<T>(h);                                                                           \
    std::memcpy(fx, o->fx.data(), o->fx.size() * sizeof(T));                                     \
    std::memcpy(fy, o->fy.data(), o->fy.size() * sizeof(T));                                     \
  }                                                                                              \
  extern "C" void orc_forces_##SUF(void* h, double* out) { O<T>(h)->forces(out); }               \
  extern "C" double orc_residual_l2_##SUF(void* h) { return O<T>(h)->residual_l2(); }            \
  extern "C" void orc_grid_interpolate_##SUF(void* h) { O<T>(h)->grid_interpolate(); }           \
  extern "C" void orc_grid_jacobi_##SUF(void* h, int iters, T* prev) {                           \
    auto* o = O<T>(h);                                                                           \
    if (prev) {                                                                                  \
      std::vector<T> p; o->grid_jacobi(iters, &p);                                               \
      std::memcpy(prev, p.data(), p.size() * sizeof(T));                                         \
    } else o->grid_jacobi(iters, nullptr);                                                       \
  }                                                                                              \
  extern "C" int orc_grid_multicolor_##SUF(void* h, int iters, double tol, double* mv) {         \
    T m; int s = O<T>(h)->grid_multicolor(iters, T(tol), &m); if (mv) *mv = (double)m; return s; \
  }

ORC_API(f32, float)
ORC_API(f64, double)

extern "C" int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
extern "C" void orc_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
