// The solver's arithmetic in a generic real type R, spelled operation by operation as
// the reference writes it (IEEE division and square root; the translation units that
// include it are compiled with -fmad=false).  R = double is the full-FP64 engine
// (kernels_f64.cu) used to state the FP32 path's error; the operation order and
// literals are those of the FP32 exact path in physics.cuh (FAST = false), which
// reproduces the reference bit for bit, so R = double follows the same algorithm as
// the FP64 CPU oracle.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ausm {
namespace ex {

template <class R> struct alignas(2 * sizeof(R)) V2 { R x, y; };
template <class R> struct alignas(4 * sizeof(R)) V4 { R x, y, z, w; };

// Per-solve constants in R, derived in R from the FP64 parameters.
template <class R> struct ConstsR {
  R gamma, gm1, gm1inv, inRho, inP, Kp, Ku, cfl, maxdt;
  V2<R> inflow;
  V4<R> inState;
  R a2inf, Minf2, Vinf2, gammaInP, aStarK, ambE;
  int muscl;
};

template <class R> __device__ __forceinline__ R rmax(R a, R b) { return fmax(a, b); }
template <class R> __device__ __forceinline__ R rmin(R a, R b) { return fmin(a, b); }
template <class R> __device__ __forceinline__ R sat(R x) { return rmin(rmax(x, R(0)), R(1)); }
template <class R> __device__ __forceinline__ R wsign(R x) { return x > R(0) ? R(1) : (x < R(0) ? R(-1) : R(0)); }

template <class R> __device__ __forceinline__ void edge_normal(V2<R> a, V2<R> b, R& nx, R& ny, R& len) {
  R dx = a.x - b.x, dy = a.y - b.y;
  len = sqrt(dx * dx + dy * dy);
  R tx = dx / len, ty = dy / len;
  nx = -ty;
  ny = tx;
}

template <class R> __device__ __forceinline__ V4<R> to_prim(V4<R> Q, R gm1) {
  R rho = Q.x, u = Q.y / rho, v = Q.z / rho;
  R p = rmax(R(1e-7), (Q.w - R(0.5) * rho * (u * u + v * v)) * gm1);
  return {rho, u, v, p};
}

template <class R> __device__ __forceinline__ V4<R> wall_ghost(V4<R> s, V2<R> a, V2<R> b) {
  R nx, ny, len;
  edge_normal(a, b, nx, ny, len);
  R rho = s.x, u = s.y / rho, v = s.z / rho;
  R dn = R(2) * (nx * u + ny * v);
  R gu = u - dn * nx, gv = v - dn * ny;
  return {rho, gu * rho, gv * rho, s.w};
}

template <class R>
__device__ __forceinline__ void far_ghosts(V4<R> s, V2<R> a, V2<R> b, const ConstsR<R>& c, V4<R>& g1, V4<R>& g2) {
  R nx, ny, len;
  edge_normal(a, b, nx, ny, len);
  R rho = s.x, u = s.y / rho, v = s.z / rho;
  R inout = nx * c.inflow.x + ny * c.inflow.y;
  if (inout < R(0)) {
    g1 = c.inState;
    g2 = c.inState;
    return;
  }
  const R g = c.gamma;
  R u2 = u * u + v * v;
  R P = (s.w - R(0.5) * u2 * rho) * (g - R(1));
  R a2 = g * P / rho;
  R Mint = u2 / a2;
  if (Mint < R(1) && c.Minf2 < R(1)) {
    R un_int = u * nx + v * ny;
    R a_int = sqrt(a2), a_inf = sqrt(c.a2inf);
    R J_int = un_int + R(2) * a_int * c.gm1inv;
    R J_ext = inout - R(2) * a_inf * c.gm1inv;
    R un_g = R(0.5) * (J_int + J_ext);
    R a_g = rmax(a_int * R(0.1), R(0.25) * (J_int - J_ext) * (g - R(1)));
    R X = rmax(R(1e-6), a_g / a_int);
    R X2 = X * X;
    R rho_g = rmax(R(1e-6), rho * X2 * X2 * X);
    R dun = un_g - un_int;
    R vgx = dun * nx + u, vgy = dun * ny + v;
    R E_g = rmax(R(1e-6), rho_g * a_g * a_g / g) * c.gm1inv + R(0.5) * rho_g * (vgx * vgx + vgy * vgy);
    g1 = {rho_g, vgx * rho_g, vgy * rho_g, E_g};
  } else if (c.Minf2 > R(1)) {
    g1 = {s.x, s.y, s.z, c.ambE + R(0.5) * rho * u2};
  } else {
    g1 = s;
  }
  g2 = {R(2) * g1.x - s.x, R(2) * g1.y - s.y, R(2) * g1.z - s.z, R(2) * g1.w - s.w};
}

template <class R> __device__ __forceinline__ void muscl1(R l2, R l, R r, R r2, R& lo, R& ro) {
  const R eps = R(1e-6);
  R dL = l - l2, dF = r - l, dR = r2 - r;
  R den = dF * dF + eps;
  R rL = (dL * dF + eps) / den, rR = (dF * dR + eps) / den;
  R r2L = rL * rL, r2R = rR * rR;
  lo = l + R(0.5) * ((r2L + rL) / (r2L + R(1))) * dF;
  ro = r - R(0.5) * ((r2R + rR) / (r2R + R(1))) * dF;
}

template <int SCHEME, class R>
__device__ __forceinline__ V4<R> face_flux(V4<R> L2, V4<R> L, V4<R> R_, V4<R> R2, R nx, R ny,
                                           const ConstsR<R>& c) {
  V4<R> Lm = L, Rm = R_;
  if (c.muscl > 0) {
    muscl1(L2.x, L.x, R_.x, R2.x, Lm.x, Rm.x);
    muscl1(L2.y, L.y, R_.y, R2.y, Lm.y, Rm.y);
    muscl1(L2.z, L.z, R_.z, R2.z, Lm.z, Rm.z);
    muscl1(L2.w, L.w, R_.w, R2.w, Lm.w, Rm.w);
  }
  const R gm1 = c.gm1;
  R rhoL = Lm.x, rhoR = Rm.x, pL = Lm.w, pR = Rm.w;
  R vxL = Lm.y, vyL = Lm.z, vxR = Rm.y, vyR = Rm.z;
  R uL = vxL * nx + vyL * ny, uR = vxR * nx + vyR * ny;
  R kL = vxL * vxL + vyL * vyL, kR = vxR * vxR + vyR * vyR;
  R hL = pL / (gm1 * rhoL) + R(0.5) * kL + pL / rhoL;
  R hR = pR / (gm1 * rhoR) + R(0.5) * kR + pR / rhoR;
  R mdot, P;
  if constexpr (SCHEME == 2) {
    R Minf2 = c.Vinf2 / (c.gammaInP / rhoL);
    const R sigma = R(1);
    R ht = R(0.5) * (hL + hR);
    R aStar = sqrt(rmax(R(1e-6), c.aStarK * ht));
    R as2 = aStar * aStar;
    R aHL = as2 / rmax(uL, aStar);
    R aHR = as2 / rmax(-uR, aStar);
    R a = rmin(aHL, aHR);
    R ML = uL / a, MR = uR / a;
    R a2 = a * a;
    R Mbar2 = (uL * uL + uR * uR) / (a2 * R(2));
    R Mo2 = rmin(R(1), rmax(Mbar2, Minf2));
    R fa = Mo2 * (R(2) - Mo2);
    R rhoI = R(0.5) * (rhoL + rhoR);
    R Mp1L = ML + R(1), Mp1R = MR + R(1), Mm1L = ML - R(1), Mm1R = MR - R(1);
    R M2pL = R(0.25) * Mp1L * Mp1L, M2pR = R(0.25) * Mp1R * Mp1R;
    R M2mL = R(-0.25) * Mm1L * Mm1L, M2mR = R(-0.25) * Mm1R * Mm1R;
    bool supL = R(1) <= fabs(ML), supR = R(1) <= fabs(MR);
    R M4L = supL ? rmax(R(0), ML) : M2pL * (R(1) + R(2) * M2mL);
    R M4R = supR ? rmin(R(0), MR) : M2mR * (R(1) - R(2) * M2pR);
    R Mi = M4L + M4R - c.Kp / fa * rmax(R(1) - sigma * Mbar2, R(0)) * (pR - pL) / (rhoI * a2);
    R alpha4 = R(0.75) * (R(-4) + R(5) * fa * fa);
    R P5L = supL ? (R(0) <= ML ? R(1) : R(0)) : M2pL * ((R(2) - ML) + alpha4 * ML * M2mL);
    R P5R = supR ? (R(0) <= -MR ? R(1) : R(0)) : M2mR * ((R(-2) - MR) - alpha4 * MR * M2pR);
    P = (P5L * pL + P5R * pR) - c.Ku * P5L * P5R * (rhoL + rhoR) * fa * a * (uR - uL);
    mdot = a * Mi * (Mi > R(0) ? rhoL : rhoR);
  } else {
    R aL = sqrt(c.gamma * rmax(pL, R(1e-10)) / rmax(rhoL, R(1e-10)));
    R aR = sqrt(c.gamma * rmax(pR, R(1e-10)) / rmax(rhoR, R(1e-10)));
    R a = (aL + aR) * R(0.5);
    R ML = uL / a, MR = uR / a;
    R Uarc = sqrt(R(0.5) * (kL + kR));
    R Marc = rmin(R(1), Uarc / a);
    R X = (R(1) - Marc) * (R(1) - Marc);
    R mpL = ML + R(1), mmR = MR - R(1);
    R sqL = R(0.5) * mpL * mpL, sqR = R(0.5) * mmR * mmR;
    bool supL = R(1) <= fabs(ML), supR = R(1) <= fabs(MR);
    R fpp = sat(R(0.5) * (supL ? R(1) + R(1) * wsign(ML) : sqL * (R(2) - R(1) * ML)));
    R fpm = sat(R(0.5) * (supR ? R(1) + R(-1) * wsign(MR) : sqR * (R(2) - R(-1) * MR)));
    if constexpr (SCHEME == 0)
      P = R(0.5) * ((fpp - fpm) * (pL - pR) + (pL + pR) + (Uarc * (fpp + fpm - R(1)) * (rhoL + rhoR) * a));
    else
      P = R(0.5) * ((fpp - fpm) * (pL - pR) + (R(1) + (R(1) - X) * (fpp + fpm - R(1))) * (pL + pR));
    R dp = pR - pL;
    R ubar = (rhoL * fabs(uL) + rhoR * fabs(uR)) / (rhoL + rhoR);
    R g = sat(-ML) * sat(MR);
    R ubp = ubar * (R(1) - g) + fabs(uL) * g;
    R ubm = ubar * (R(1) - g) + fabs(uR) * g;
    mdot = R(0.5) * ((rhoL * (uL + ubp) + rhoR * (uR - ubm)) * (R(1) - g) - X / a * dp);
  }
  bool left = mdot > R(0);
  R p1 = left ? vxL : vxR, p2 = left ? vyL : vyR, p3 = left ? hL : hR;
  return {R(1) * mdot + R(0), p1 * mdot + nx * P, p2 * mdot + ny * P, p3 * mdot + R(0)};
}

template <class R> __device__ __forceinline__ R wave_speed(V4<R> s, R lsum, R area, R gamma) {
  R rho = s.x, u = s.y / rho, v = s.z / rho;
  R p = (s.w - R(0.5) * rho * (u * u + v * v)) * (gamma - R(1));
  R T = p / rho;
  R a = sqrt(gamma * T);
  R speed = sqrt(u * u + v * v);
  return (speed + a) * lsum / (R(2) * area);
}

template <class R> __device__ __forceinline__ R quad_area(V2<R> a, V2<R> b, V2<R> c, V2<R> d) {
  return R(0.5) * fabs((d.x - a.x) * (c.y - b.y) - (c.x - b.x) * (d.y - a.y));
}

}  // namespace ex
}  // namespace ausm
