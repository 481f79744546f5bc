// Device arithmetic of the AUSM-family solver: primitive conversion, ghost cells,
// MUSCL/van Albada interface states and the SLAU2 / SLAU / AUSM+-up fluxes.
//
// Functions with a template flag FAST: FAST=false spells each operation as the
// reference writes it (IEEE division and square root, same operation order), and
// face_flux / muscl1 are that form only; the reference-shaped engine reproduces the CPU
// oracle bit for bit with them.  FAST=true, muscl2_packed and face_flux_len are the
// fused engines' arithmetic: approximate reciprocal and square root (one MUFU
// instruction each, about 1 ulp), shared reciprocals, an algebraically equal van
// Albada form and every fused multiply-add written out (fmaf / packed f32x2); its
// parity bound against the oracle is tested at 1e-5.
//
// Every translation unit that includes this file is compiled with -fmad=false, so the
// compiler contracts nothing on its own: the rounding of each expression is fixed by
// its source, not by the code around an inlined copy, and two kernels that compute the
// same face or cell (for instance tiles of different heights) give the same bits.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ausm {

// Per-solve constants, f32 like the reference's uniform buffer (util.js:1-29).  The
// derived values are computed on the host in f32 in the reference's operation order.
struct Consts {
  float gamma, gm1, gm1inv, inRho, inP, Kp, Ku, cfl, maxdt;
  float2 inflow;   // uni.inflowV
  float4 inState;  // uni.inState
  float a2inf;     // (gamma*inP)/inRho                  ausm.js:81
  float Minf2;     // dot(inflow,inflow)/a2inf            ausm.js:83
  float Vinf2;     // dot(inflow,inflow)                  ausm.js:273
  float gammaInP;  // gamma*inP                           ausm.js:273
  float aStarK;    // (2*gm1)/(gamma+1)                   ausm.js:278
  float ambE;      // inP/(gamma-1)                       ausm.js:108
  float h2k;       // 2 gamma/(gamma-1): twice the total enthalpy is h2k p/rho + |v|^2 (FAST only)
  float ask4;      // aStarK/4: the AUSM+-up a*^2 from twice the enthalpies (FAST only)
  float minfk;     // Vinf2/gammaInP: the AUSM+-up M_inf^2 from rho_L is rho_L * minfk (FAST only)
  float hsg;       // sqrt(gamma)/2: the SLAU mean sound speed is hsg (sqrt(p_L/rho_L) + sqrt(p_R/rho_R)) (FAST only)
  int muscl;
};

// FAST: the hardware's approximate reciprocal, square root and reciprocal square root
// (PTX rcp.approx.ftz / sqrt.approx.ftz / rsqrt.approx.ftz, one instruction each, relative error about 1 ulp; subnormal inputs and
// results flush to zero, which no state of the solver reaches).
__device__ __forceinline__ float rcp_approx(float b) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(b));
  return r;
}
__device__ __forceinline__ float rsqrt_approx(float b) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(b));
  return r;
}
template <bool FAST> __device__ __forceinline__ float fdiv(float a, float b) {
  if constexpr (FAST) return a * rcp_approx(b);
  else return a / b;
}
template <bool FAST> __device__ __forceinline__ float frcp(float b) {
  if constexpr (FAST) return rcp_approx(b);
  else return 1.0f / b;
}
template <bool FAST> __device__ __forceinline__ float fsqrt(float a) {
  if constexpr (FAST) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
    return r;
  } else {
    return sqrtf(a);
  }
}
__device__ __forceinline__ float sat(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }
// a * b + c and a * b rounded once and clamped to [0, 1] (PTX .sat, one instruction each)
__device__ __forceinline__ float fma_sat(float a, float b, float c) {
  float r;
  asm("fma.rn.sat.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
__device__ __forceinline__ float mul_sat(float a, float b) {
  float r;
  asm("mul.rn.sat.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
  return r;
}

// Packed FP32 (sm_100 f32x2): two IEEE-rounded operations per instruction.
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }
__device__ __forceinline__ float wsign(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }

// unit normal (-t.y, t.x) of the tangent t = normalize(a - b), and |a - b|
template <bool FAST>
__device__ __forceinline__ void edge_normal(float2 a, float2 b, float& nx, float& ny, float& len) {
  float dx = a.x - b.x, dy = a.y - b.y;
  float l2 = dx * dx + dy * dy;
  if constexpr (FAST) {
    float ri = rsqrtf(l2);
    len = l2 * ri;
    float tx = dx * ri, ty = dy * ri;
    nx = -ty; ny = tx;
  } else {
    len = sqrtf(l2);
    float tx = dx / len, ty = dy / len;
    nx = -ty; ny = tx;
  }
}

// toPrimitive (ausm.js:145-150): (rho, u, v, p), p >= 1e-7
template <bool FAST> __device__ __forceinline__ float4 to_prim(float4 Q, float gm1) {
  float rho = Q.x;
  if constexpr (FAST) {
    // rho |v|^2 as (rho u) u + (rho v) v
    const float ir = frcp<true>(rho);
    const float u = Q.y * ir, v = Q.z * ir;
    const float k = fmaf(Q.z, v, Q.y * u);
    return make_float4(rho, u, v, fmaxf(1e-7f, fmaf(-0.5f, k, Q.w) * gm1));
  } else {
    float u = Q.y / rho, v = Q.z / rho;
    float p = fmaxf(1e-7f, (Q.w - 0.5f * rho * (u * u + v * v)) * gm1);
    return make_float4(rho, u, v, p);
  }
}

// Wall ghost (ausm.js:57-64): velocity of the first interior cell reflected about the
// wall normal (nx, ny); rho and rhoE kept.
template <bool FAST> __device__ __forceinline__ float4 wall_ghost_n(float4 s, float nx, float ny) {
  float rho = s.x;
  float u = fdiv<FAST>(s.y, rho), v = fdiv<FAST>(s.z, rho);
  float dn = 2.0f * (nx * u + ny * v);
  float gu = u - dn * nx, gv = v - dn * ny;
  return make_float4(rho, gu * rho, gv * rho, s.w);
}
// ... with the normal of the wall face between vertices a=(i,0), b=(i+1,0)
template <bool FAST> __device__ __forceinline__ float4 wall_ghost(float4 s, float2 a, float2 b) {
  float nx, ny, len;
  edge_normal<FAST>(a, b, nx, ny, len);
  return wall_ghost_n<FAST>(s, nx, ny);
}

// Far-field ghosts (ausm.js:65-117) from the last interior cell s and the unit normal
// (nx, ny) of the outer face.  g1 = row N+1, g2 = row N+2.
template <bool FAST>
__device__ __forceinline__ void far_ghosts_n(float4 s, float nx, float ny, const Consts& c, float4& g1, float4& g2) {
  float rho = s.x;
  float u = fdiv<FAST>(s.y, rho), v = fdiv<FAST>(s.z, rho);
  float inout = nx * c.inflow.x + ny * c.inflow.y;
  if (inout < 0.0f) {  // inflow
    g1 = c.inState;
    g2 = c.inState;
    return;
  }
  const float g = c.gamma;
  float u2 = u * u + v * v;
  float P = (s.w - 0.5f * u2 * rho) * (g - 1.0f);
  float a2 = fdiv<FAST>(g * P, rho);
  float Mint = fdiv<FAST>(u2, a2);
  if (Mint < 1.0f && c.Minf2 < 1.0f) {  // subsonic: Riemann invariants
    float un_int = u * nx + v * ny;
    float a_int = fsqrt<FAST>(a2), a_inf = fsqrt<FAST>(c.a2inf);
    float J_int = un_int + 2.0f * a_int * c.gm1inv;
    float J_ext = inout - 2.0f * a_inf * c.gm1inv;
    float un_g = 0.5f * (J_int + J_ext);
    float a_g = fmaxf(a_int * 0.1f, 0.25f * (J_int - J_ext) * (g - 1.0f));
    float X = fmaxf(1e-6f, fdiv<FAST>(a_g, a_int));
    float X2 = X * X;
    float rho_g = fmaxf(1e-6f, rho * X2 * X2 * X);
    float dun = un_g - un_int;
    float vgx = dun * nx + u, vgy = dun * ny + v;
    float E_g = fmaxf(1e-6f, fdiv<FAST>(rho_g * a_g * a_g, g)) * c.gm1inv + 0.5f * rho_g * (vgx * vgx + vgy * vgy);
    g1 = make_float4(rho_g, vgx * rho_g, vgy * rho_g, E_g);
  } else if (c.Minf2 > 1.0f) {  // ambient pressure
    g1 = make_float4(s.x, s.y, s.z, c.ambE + 0.5f * rho * u2);
  } else {  // supersonic outflow: copy
    g1 = s;
  }
  g2 = make_float4(2.0f * g1.x - s.x, 2.0f * g1.y - s.y, 2.0f * g1.z - s.z, 2.0f * g1.w - s.w);
}
// ... with the normal of the outer face between vertices a=(i,N), b=(i+1,N)
template <bool FAST>
__device__ __forceinline__ void far_ghosts(float4 s, float2 a, float2 b, const Consts& c, float4& g1, float4& g2) {
  float nx, ny, len;
  edge_normal<FAST>(a, b, nx, ny, len);
  far_ghosts_n<FAST>(s, nx, ny, c, g1, g2);
}

// van Albada-limited MUSCL on two primitive components at once (packed f32x2), the
// FAST form of muscl1: phi(r) = n (n + d) / (n^2 + d^2) with r = n / d, one reciprocal
// per side and none for r itself.  The right side takes the reciprocal of -q (the
// same magnitude), so both sides add phi x dF/2 with one shared dF/2.
__device__ __forceinline__ void muscl2_packed(float2 l2, float2 l, float2 r, float2 r2, float2& lo, float2& ro) {
  const float2 eps = make_float2(1e-6f, 1e-6f), m1 = make_float2(-1.0f, -1.0f);
  const float2 half = make_float2(0.5f, 0.5f);
  // differences as x*(-1) + y: exact products, one rounding, no separate negation
  const float2 dL = fma2(l2, m1, l), dF = fma2(l, m1, r), dR = fma2(r, m1, r2);
  const float2 den = fma2(dF, dF, eps);
  const float2 nL = fma2(dL, dF, eps), nR = fma2(dF, dR, eps);
  const float2 d2 = mul2(den, den);
  const float2 qL = fma2(nL, nL, d2), qR = fma2(nR, nR, d2);
  const float2 rqL = make_float2(rcp_approx(qL.x), rcp_approx(qL.y));
  const float2 rqR = make_float2(rcp_approx(-qR.x), rcp_approx(-qR.y));
  const float2 tL = mul2(nL, add2(nL, den)), tR = mul2(nR, add2(nR, den));
  const float2 hdF = mul2(half, dF);
  lo = fma2(mul2(tL, rqL), hdF, l);
  ro = fma2(mul2(tR, rqR), hdF, r);
}

// van Albada-limited MUSCL update of one primitive component (ausm.js:238-249).
__device__ __forceinline__ void muscl1(float l2, float l, float r, float r2, float& lo, float& ro) {
  const float eps = 1e-6f;
  float dL = l - l2, dF = r - l, dR = r2 - r;
  float den = dF * dF + eps;
  float nL = dL * dF + eps, nR = dF * dR + eps;
  float rL = nL / den, rR = nR / den;
  float r2L = rL * rL, r2R = rR * rR;
  lo = l + 0.5f * ((r2L + rL) / (r2L + 1.0f)) * dF;
  ro = r - 0.5f * ((r2R + rR) / (r2R + 1.0f)) * dF;
}

// Flux per unit face length through a face with unit normal (nx, ny) pointing from
// L to R, from the primitive states of the four cells along the face normal line
// (fluxInterfaceStateCode ausm.js:201-266 + SLAUFluxShaderCode ausm.js:348-391 /
// AUSMupFluxShaderCode ausm.js:273-334).
template <int SCHEME>
__device__ __forceinline__ float4 face_flux(float4 L2, float4 L, float4 R, float4 R2, float nx, float ny,
                                            const Consts& c) {
  float4 Lm = L, Rm = R;
  if (c.muscl > 0) {
    muscl1(L2.x, L.x, R.x, R2.x, Lm.x, Rm.x);
    muscl1(L2.y, L.y, R.y, R2.y, Lm.y, Rm.y);
    muscl1(L2.z, L.z, R.z, R2.z, Lm.z, Rm.z);
    muscl1(L2.w, L.w, R.w, R2.w, Lm.w, Rm.w);
  }
  const float gm1 = c.gm1;
  float rhoL = Lm.x, rhoR = Rm.x, pL = Lm.w, pR = Rm.w;
  float vxL = Lm.y, vyL = Lm.z, vxR = Rm.y, vyR = Rm.z;
  float uL = vxL * nx + vyL * ny, uR = vxR * nx + vyR * ny;
  float kL = vxL * vxL + vyL * vyL, kR = vxR * vxR + vyR * vyR;
  float hL = pL / (gm1 * rhoL) + 0.5f * kL + pL / rhoL;
  float hR = pR / (gm1 * rhoR) + 0.5f * kR + pR / rhoR;
  float mdot, P;
  if constexpr (SCHEME == 2) {  // AUSM+-up, Liou 2006 eqs. 28-30, 69-76
    float Minf2 = c.Vinf2 / (c.gammaInP / rhoL);
    const float sigma = 1.0f;
    float ht = 0.5f * (hL + hR);
    float aStar = sqrtf(fmaxf(1e-6f, c.aStarK * ht));
    float as2 = aStar * aStar;
    float aHL = as2 / fmaxf(uL, aStar);
    float aHR = as2 / fmaxf(-uR, aStar);
    float a = fminf(aHL, aHR);
    float ML = uL / a, MR = uR / a;
    float a2 = a * a;
    float Mbar2 = (uL * uL + uR * uR) / (a2 * 2.0f);
    float Mo2 = fminf(1.0f, fmaxf(Mbar2, Minf2));
    float fa = Mo2 * (2.0f - Mo2);
    float rhoI = 0.5f * (rhoL + rhoR);
    float Mp1L = ML + 1.0f, Mp1R = MR + 1.0f, Mm1L = ML - 1.0f, Mm1R = MR - 1.0f;
    float M2pL = 0.25f * Mp1L * Mp1L, M2pR = 0.25f * Mp1R * Mp1R;
    float M2mL = -0.25f * Mm1L * Mm1L, M2mR = -0.25f * Mm1R * Mm1R;
    bool supL = 1.0f <= fabsf(ML), supR = 1.0f <= fabsf(MR);
    float M4L = supL ? fmaxf(0.0f, ML) : M2pL * (1.0f + 2.0f * M2mL);
    float M4R = supR ? fminf(0.0f, MR) : M2mR * (1.0f - 2.0f * M2pR);
    float Mi = M4L + M4R - (c.Kp / fa * fmaxf(1.0f - sigma * Mbar2, 0.0f) * (pR - pL)) / (rhoI * a2);
    float alpha4 = 0.75f * (-4.0f + 5.0f * fa * fa);
    float P5L = supL ? (0.0f <= ML ? 1.0f : 0.0f) : M2pL * ((2.0f - ML) + alpha4 * ML * M2mL);
    float P5R = supR ? (0.0f <= -MR ? 1.0f : 0.0f) : M2mR * ((-2.0f - MR) - alpha4 * MR * M2pR);
    P = (P5L * pL + P5R * pR) - c.Ku * P5L * P5R * (rhoL + rhoR) * fa * a * (uR - uL);
    mdot = a * Mi * (Mi > 0.0f ? rhoL : rhoR);
  } else {  // SLAU2 (SCHEME 0, Kitamura-Shima 2013) / SLAU (SCHEME 1, Shima-Kitamura 2011)
    float aL = sqrtf(c.gamma * fmaxf(pL, 1e-10f) / fmaxf(rhoL, 1e-10f));
    float aR = sqrtf(c.gamma * fmaxf(pR, 1e-10f) / fmaxf(rhoR, 1e-10f));
    float a = (aL + aR) * 0.5f;
    float Uarc = sqrtf(0.5f * (kL + kR));
    float ML = uL / a, MR = uR / a;
    float Marc = fminf(1.0f, Uarc / a);
    float X = (1.0f - Marc) * (1.0f - Marc);
    float mpL = ML + 1.0f, mmR = MR - 1.0f;
    float sqL = 0.5f * mpL * mpL, sqR = 0.5f * mmR * mmR;
    bool supL = 1.0f <= fabsf(ML), supR = 1.0f <= fabsf(MR);
    float fpp = sat(0.5f * (supL ? 1.0f + 1.0f * wsign(ML) : sqL * (2.0f - 1.0f * ML)));
    float fpm = sat(0.5f * (supR ? 1.0f + -1.0f * wsign(MR) : sqR * (2.0f - -1.0f * MR)));
    if constexpr (SCHEME == 0)
      P = 0.5f * ((fpp - fpm) * (pL - pR) + (pL + pR) + (Uarc * (fpp + fpm - 1.0f) * (rhoL + rhoR) * a));
    else
      P = 0.5f * ((fpp - fpm) * (pL - pR) + (1.0f + (1.0f - X) * (fpp + fpm - 1.0f)) * (pL + pR));
    float dp = pR - pL;
    float ubar = (rhoL * fabsf(uL) + rhoR * fabsf(uR)) / (rhoL + rhoR);
    float g = sat(-ML) * sat(MR);
    float ubp = ubar * (1.0f - g) + fabsf(uL) * g;
    float ubm = ubar * (1.0f - g) + fabsf(uR) * g;
    mdot = 0.5f * ((rhoL * (uL + ubp) + rhoR * (uR - ubm)) * (1.0f - g) - X / a * dp);
  }
  bool left = mdot > 0.0f;
  float p1 = left ? vxL : vxR, p2 = left ? vyL : vyR, p3 = left ? hL : hR;
  return make_float4(1.0f * mdot + 0.0f, p1 * mdot + nx * P, p2 * mdot + ny * P, p3 * mdot + 0.0f);
}

// FAST flux x face length (the fused engines), from the face's half length hl: the
// arithmetic of face_flux with approximate reciprocals and square roots, every fused
// multiply-add written out, and these algebraic rewrites:
//  - the length folded into the mass flux and pressure; SLAU / SLAU2 compute twice
//    the mass flux and twice the pressure and multiply them by hl (two multiplies by
//    0.5 fewer), AUSM+-up multiplies by hl + hl;
//  - twice the total enthalpy h2 = h2k p / rho + |v|^2, so that no 0.5 |v|^2 is
//    formed; the energy flux is h2 x (mass flux x hl);
//  - no "+ 0" terms (those keep the reference's sign of zero in the exact path);
//  - SLAU / SLAU2: 1/rho guarded by one max; one guarded p / rho per side serves both
//    the speed of sound, a = sqrt(gamma) / 2 (sqrt(p_L / rho_L) + sqrt(p_R / rho_R)),
//    and the enthalpy (the enthalpy takes the guarded pressure, which differs from the
//    reference only for p < 1e-10); the pressure-split functions as the smoothstep
//    s^2 (3 - 2 s) of s = (M + 1) / 2 clamped to [0, 1] by one saturating fused
//    multiply-add from the normal velocity and a / 2: that is the cubic
//    f(M) = (M+1)^2 (2-M) / 4 of the clamped Mach number, which is exactly the
//    reference's branch (|M| >= 1 gives 1 or 0, the cubic is 1 at M = 1, 0 at M = -1
//    and within [0, 1] between, so its saturate is a no-op); 1 - min(1, Uarc / a) and
//    sat(-ML), sat(MR) as single saturating operations;
//  - AUSM+-up: M_inf^2 from rho_L as rho_L Vinf^2 / (gamma p_inf); a*^2 as
//    (aStarK / 4) (h2L + h2R), used as computed (not the square of its square root);
//    the interface speed of sound min(a*^2 / max(uL, a*), a*^2 / max(-uR, a*)) as
//    a*^2 / max(uL, -uR, a*) and its reciprocal as max(uL, -uR, a*) / a*^2, with a* and
//    1 / a*^2 from one reciprocal square root (two MUFU operations instead of four);
//    Mbar^2 = (ML^2 + MR^2) / 2 from the face Mach numbers; the K_p pressure-diffusion
//    term only when K_p != 0 (uniform per solve; the reference's default is 0).
// SCHEME_FLAGS: the scheme (bits 0-1), plus 4 when the launch knows MUSCL is on, so the
// kernel has no per-face branch on it (c.muscl is read at run time otherwise).
template <int SCHEME_FLAGS>
__device__ __forceinline__ float4 face_flux_len(float4 L2, float4 L, float4 R, float4 R2, float nx, float ny,
                                                float hl, const Consts& c) {
  constexpr int SCHEME = SCHEME_FLAGS & 3;
  constexpr bool MUSCL_ON = (SCHEME_FLAGS & 4) != 0;  // MUSCL known on at compile time
  float4 Lm = L, Rm = R;
  if (MUSCL_ON || c.muscl > 0) {
    float2 a, b;
    muscl2_packed(lo2(L2), lo2(L), lo2(R), lo2(R2), a, b);
    Lm.x = a.x; Lm.y = a.y; Rm.x = b.x; Rm.y = b.y;
    muscl2_packed(hi2(L2), hi2(L), hi2(R), hi2(R2), a, b);
    Lm.z = a.x; Lm.w = a.y; Rm.z = b.x; Rm.w = b.y;
  }
  const float rhoL = Lm.x, rhoR = Rm.x, pL = Lm.w, pR = Rm.w;
  const float vxL = Lm.y, vyL = Lm.z, vxR = Rm.y, vyR = Rm.z;
  const float uL = fmaf(vyL, ny, vxL * nx), uR = fmaf(vyR, ny, vxR * nx);
  const float kL = fmaf(vyL, vyL, vxL * vxL), kR = fmaf(vyR, vyR, vxR * vxR);
  if constexpr (SCHEME == 2) {  // AUSM+-up, Liou 2006 eqs. 28-30, 69-76
    const float irL = frcp<true>(rhoL), irR = frcp<true>(rhoR);
    const float h2L = fmaf(c.h2k * pL, irL, kL), h2R = fmaf(c.h2k * pR, irR, kR);
    const float Minf2 = rhoL * c.minfk;
    const float as2 = fmaxf(1e-6f, c.ask4 * (h2L + h2R));
    // a = min(a*^2 / max(uL, a*), a*^2 / max(-uR, a*)) = a*^2 / max(uL, -uR, a*), and
    // 1 / a = max(uL, -uR, a*) / a*^2 with 1 / a*^2 = (1 / a*)^2 from one rsqrt
    const float rs = rsqrt_approx(as2);
    const float mx = fmaxf(fmaxf(uL, -uR), as2 * rs);
    const float ia = mx * (rs * rs);
    const float a = as2 * frcp<true>(mx);
    const float ML = uL * ia, MR = uR * ia;
    const float Mbar2 = 0.5f * fmaf(MR, MR, ML * ML);
    const float Mo2 = fminf(1.0f, fmaxf(Mbar2, Minf2));
    const float fa = Mo2 * (2.0f - Mo2);
    // M2+(M) = (M+1)^2/4 = ((M+1)/2)^2, M2-(M) = -((M-1)/2)^2
    const float hpL = fmaf(0.5f, ML, 0.5f), hpR = fmaf(0.5f, MR, 0.5f);
    const float hmL = fmaf(0.5f, ML, -0.5f), hmR = fmaf(0.5f, MR, -0.5f);
    const float M2pL = hpL * hpL, M2pR = hpR * hpR, M2mL = -(hmL * hmL), M2mR = -(hmR * hmR);
    const bool supL = 1.0f <= fabsf(ML), supR = 1.0f <= fabsf(MR);
    const float M4L = supL ? fmaxf(0.0f, ML) : M2pL * fmaf(2.0f, M2mL, 1.0f);
    const float M4R = supR ? fminf(0.0f, MR) : M2mR * fmaf(-2.0f, M2pR, 1.0f);
    float Mi = M4L + M4R;
    if (c.Kp != 0.0f) {
      const float rhoI = 0.5f * (rhoL + rhoR);
      Mi -= c.Kp * frcp<true>(fa) * fmaxf(1.0f - Mbar2, 0.0f) * (pR - pL) * frcp<true>(rhoI * a * a);
    }
    const float alpha4 = 0.75f * fmaf(5.0f * fa, fa, -4.0f);
    const float P5L = supL ? (0.0f <= ML ? 1.0f : 0.0f) : M2pL * fmaf(alpha4 * ML, M2mL, 2.0f - ML);
    const float P5R = supR ? (0.0f <= -MR ? 1.0f : 0.0f) : M2mR * fmaf(-alpha4 * MR, M2pR, -2.0f - MR);
    const float P = fmaf(-c.Ku * P5L * P5R * (rhoL + rhoR) * fa * a, uR - uL, fmaf(P5L, pL, P5R * pR));
    const float mdot = a * Mi * (Mi > 0.0f ? rhoL : rhoR);
    const bool left = mdot > 0.0f;
    const float len = hl + hl;
    const float ml = mdot * len, Pl = P * len, mlh = mdot * hl;
    const float p1 = left ? vxL : vxR, p2 = left ? vyL : vyR, p3 = left ? h2L : h2R;
    return make_float4(ml, fmaf(p1, ml, nx * Pl), fmaf(p2, ml, ny * Pl), p3 * mlh);
  } else {  // SLAU2 (SCHEME 0, Kitamura-Shima 2013) / SLAU (SCHEME 1, Shima-Kitamura 2011)
    const float irL = frcp<true>(fmaxf(rhoL, 1e-10f)), irR = frcp<true>(fmaxf(rhoR, 1e-10f));
    // guarded p / rho: the speed of sound is sqrt(gamma p / rho), twice the enthalpy h2k p / rho + |v|^2
    const float tL = fmaxf(pL, 1e-10f) * irL, tR = fmaxf(pR, 1e-10f) * irR;
    const float h2L = fmaf(c.h2k, tL, kL), h2R = fmaf(c.h2k, tR, kR);
    const float a = c.hsg * (fsqrt<true>(tL) + fsqrt<true>(tR));  // (a_L + a_R) / 2
    const float ia = frcp<true>(a), hia = 0.5f * ia;
    const float Uarc = fsqrt<true>(0.5f * (kL + kR));
    const float omM = fma_sat(-Uarc, ia, 1.0f);  // 1 - min(1, Uarc / a)
    const float X = omM * omM;
    // f(M) = (M+1)^2 (2-M) / 4 for |M| < 1, 0 or 1 beyond, is the smoothstep s^2 (3 - 2 s)
    // of s = (M + 1) / 2 clamped to [0, 1]; f(ML) and f(-MR)
    const float sL = fma_sat(uL, hia, 0.5f), sR = fma_sat(-uR, hia, 0.5f);
    const float fpp = (sL * sL) * fmaf(-2.0f, sL, 3.0f);
    const float fpm = (sR * sR) * fmaf(-2.0f, sR, 3.0f);
    const float rs = rhoL + rhoR;
    const float dpLR = pL - pR, s1 = (fpp + fpm) - 1.0f;
    float P2;  // 2 P
    if constexpr (SCHEME == 0)
      P2 = fmaf(Uarc * s1 * rs, a, fmaf(fpp - fpm, dpLR, pL + pR));
    else
      P2 = fmaf(fpp - fpm, dpLR, fmaf(1.0f - X, s1, 1.0f) * (pL + pR));
    const float ubar = fmaf(rhoL, fabsf(uL), rhoR * fabsf(uR)) * frcp<true>(rs);
    const float g = mul_sat(-uL, ia) * mul_sat(uR, ia);  // sat(-ML) sat(MR)
    const float omg = 1.0f - g;
    const float ubo = ubar * omg;
    const float ubp = fmaf(fabsf(uL), g, ubo), ubm = fmaf(fabsf(uR), g, ubo);
    // 2 mdot = (rhoL (uL + ubp) + rhoR (uR - ubm)) (1 - g) - X/a (pR - pL)
    const float md2 = fmaf(X * ia, dpLR, fmaf(rhoL, uL + ubp, rhoR * (uR - ubm)) * omg);
    const bool left = md2 > 0.0f;
    const float ml = md2 * hl, Pl = P2 * hl;
    const float p1 = left ? vxL : vxR, p2 = left ? vyL : vyR, p3 = left ? h2L : h2R;
    return make_float4(ml, fmaf(p1, ml, nx * Pl), fmaf(p2, ml, ny * Pl), p3 * (0.5f * ml));
  }
}

// Cell wave speed for the CFL condition (ausm.js:617-630): (|v| + a) * sum(l) / (2 A).
template <bool FAST> __device__ __forceinline__ float wave_speed(float4 s, float lsum, float area, float gamma) {
  float rho = s.x;
  float u = fdiv<FAST>(s.y, rho), v = fdiv<FAST>(s.z, rho);
  float p = (s.w - 0.5f * rho * (u * u + v * v)) * (gamma - 1.0f);
  float T = fdiv<FAST>(p, rho);
  float a = fsqrt<FAST>(gamma * T);
  float speed = fsqrt<FAST>(u * u + v * v);
  return fdiv<FAST>((speed + a) * lsum, 2.0f * area);
}

// ... with the cell's precomputed factor W = sum(l) / (2 A)
template <bool FAST> __device__ __forceinline__ float wave_speed_w(float4 s, float W, float gamma) {
  float rho = s.x;
  if constexpr (FAST) {
    const float ir = frcp<true>(rho);
    const float u = s.y * ir, v = s.z * ir;
    const float k = fmaf(v, v, u * u);
    const float p = fmaf(-0.5f * rho, k, s.w) * (gamma - 1.0f);
    return (fsqrt<true>(k) + fsqrt<true>(gamma * (p * ir))) * W;
  } else {
    float u = s.y / rho, v = s.z / rho;
    float p = (s.w - 0.5f * rho * (u * u + v * v)) * (gamma - 1.0f);
    float T = p / rho;
    float a = sqrtf(gamma * T);
    float speed = sqrtf(u * u + v * v);
    return (speed + a) * W;
  }
}

// Cell area of the quad a=(i,j), b=(i+1,j), c=(i,j+1), d=(i+1,j+1) (shaders/grid.js:140).
__device__ __forceinline__ float quad_area(float2 a, float2 b, float2 c, float2 d) {
  return 0.5f * fabsf((d.x - a.x) * (c.y - b.y) - (c.x - b.x) * (d.y - a.y));
}

}  // namespace ausm
