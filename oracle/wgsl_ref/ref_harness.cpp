// ORACLE — test infrastructure only.
//
// Host side for the reference's own compute shaders compiled for the CPU (translate.py).
// It plays the part of src/main.js: it creates the same textures and buffers
// (main.js:110-151), binds them exactly as the reference's bind groups do
// (main.js:190-441, 543-565) and issues the dispatches in the reference's order and
// sizes (main.js:604-612, 631-707, 744-791, 808-810).  Host geometry input
// (updateGridBoundaries, grid.js:267-296) is restated here; the body and outer
// boundary coordinates themselves are inputs.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "uniforms_gen.h"
#include "wgsl_rt.h"

#define DECL_MOD(n)                                    \
  extern "C" void n##_bind(int, void*);                \
  extern "C" void n##_dispatch(unsigned, unsigned, unsigned);
DECL_MOD(prepareStateShaderCode)
DECL_MOD(boundaryShaderCode)
DECL_MOD(SLAU2_verticalFluxShaderCode)
DECL_MOD(SLAU2_horizontalFluxShaderCode)
DECL_MOD(SLAU_verticalFluxShaderCode)
DECL_MOD(SLAU_horizontalFluxShaderCode)
DECL_MOD(AUSMup_verticalFluxShaderCode)
DECL_MOD(AUSMup_horizontalFluxShaderCode)
DECL_MOD(residualShaderCode)
DECL_MOD(integrationStage1ShaderCode)
DECL_MOD(integrationStage2ShaderCode)
DECL_MOD(integrationStage3ShaderCode)
DECL_MOD(cflReductionShaderCode)
DECL_MOD(visualizationShaderCode)
DECL_MOD(visualizationFieldProbe)
DECL_MOD(gridInterpolationShaderCode)
DECL_MOD(gridEllipticPoissonShaderCode)
DECL_MOD(gridFinalizeShaderCode)
DECL_MOD(forceCalcShaderCode)
DECL_MOD(forceIntegrationShaderCode)

namespace {
using namespace wgsl;
struct Mod {
  void (*bind)(int, void*);
  void (*dispatch)(unsigned, unsigned, unsigned);
};
#define MOD(n) Mod{&n##_bind, &n##_dispatch}

struct RefUniforms {  // the path's uniform fields (util.js:1-29), host doubles
  double gamma, in_rho, in_pressure;
  double inflow[2];
  double in_state[4];
  double K_p, K_u, cfl, maxdt;
  int muscl, scheme;
};

struct RefSim {
  int M, N;
  unsigned WG = 16;  // main.js:34
  TexData gridPoints0, gridPoints1, gridBoundaries, gridArea, faceLengths, cellDistances;
  TexData state0, state1, state2, fluxX, fluxY, residual, vis;
  std::vector<float> waveSpeeds, forceValues, ring;
  uint32_t maxWaveSpeed = 0;
  float forceVector[2] = {0, 0};
  Uniforms uni{};
  GraphUniforms guni{};
  std::vector<float> gridVtxData;        // grid.js:33
  std::vector<int16_t> gridBoundaryData; // grid.js:34
  Mod vflux, hflux;

  RefSim(int M_, int N_) : M(M_), N(N_) {
    gridPoints0.init(M, N + 1, 2, TEX_F32);
    gridPoints1.init(M, N + 1, 2, TEX_F32);
    gridBoundaries.init(M, N + 1, 2, TEX_S16);
    gridArea.init(M, N, 1, TEX_F32);
    faceLengths.init(M, N, 4, TEX_F32);
    cellDistances.init(M, N, 4, TEX_F32);
    state0.init(M, N + 3, 4, TEX_F32);
    state1.init(M, N + 3, 4, TEX_F32);
    state2.init(M, N + 3, 4, TEX_F32);
    fluxX.init(M + 1, N, 4, TEX_F32);
    fluxY.init(M, N + 1, 4, TEX_F32);
    residual.init(M, N, 4, TEX_F32);
    vis.init(M, N, 4, TEX_F32);
    waveSpeeds.assign((size_t)M * N, 0.0f);
    forceValues.assign((size_t)M * 2, 0.0f);
    ring.assign(256 * 4, 0.0f);
    gridVtxData.assign((size_t)M * (N + 1) * 2, 0.0f);
    gridBoundaryData.assign((size_t)M * (N + 1) * 2, 0);
    // main.js:874-887 and util.js defaults for the non-path fields
    uni.zoom = 1.0f;
    uni.simDomain = vec2f(float(M), float(N));
    uni.contourCompression = 1.001f;
    uni.visMultiplier = 1.0f;
    uni.simDisplayMode = 0.0f;
    guni.nPoints = 256.0f;
    guni.writeHead = 0.0f;
    vflux = MOD(SLAU2_verticalFluxShaderCode);
    hflux = MOD(SLAU2_horizontalFluxShaderCode);
  }

  unsigned wg(int n) const { return (unsigned)((n + (int)WG - 1) / (int)WG); }

  void set_uniforms(const RefUniforms& u) {
    uni.gamma = float(u.gamma);
    uni.inRho = float(u.in_rho);
    uni.inPressure = float(u.in_pressure);
    uni.inflowV = vec2f(float(u.inflow[0]), float(u.inflow[1]));
    uni.inState = vec4f(float(u.in_state[0]), float(u.in_state[1]), float(u.in_state[2]), float(u.in_state[3]));
    uni.K_p = float(u.K_p);
    uni.K_u = float(u.K_u);
    uni.cflFactor = float(u.cfl);
    uni.maxdt = float(u.maxdt);
    uni.muscl = float(u.muscl);
    set_scheme(u.scheme);
  }
  // updateSolver (main.js:629, pipelines main.js:314-327)
  void set_scheme(int s) {
    if (s == 0) { vflux = MOD(SLAU2_verticalFluxShaderCode); hflux = MOD(SLAU2_horizontalFluxShaderCode); }
    if (s == 1) { vflux = MOD(SLAU_verticalFluxShaderCode); hflux = MOD(SLAU_horizontalFluxShaderCode); }
    if (s == 2) { vflux = MOD(AUSMup_verticalFluxShaderCode); hflux = MOD(AUSMup_horizontalFluxShaderCode); }
  }

  // updateGridBoundaries (grid.js:267-296)
  void set_boundaries(const float* body, const float* outer) {
    for (int x = 0; x < M; x++) {
      size_t o = (size_t)x * 2;
      gridVtxData[o] = body[2 * x];
      gridVtxData[o + 1] = body[2 * x + 1];
      size_t b = ((size_t)N * M + x) * 2;
      gridVtxData[b] = outer[2 * x];
      gridVtxData[b + 1] = outer[2 * x + 1];
    }
    for (int y = 0; y <= N; y++) {
      size_t l = ((size_t)y * M + 0) * 2, r = ((size_t)y * M + (M - 1)) * 2;
      gridBoundaryData[l] = int16_t(M - 1);
      gridBoundaryData[l + 1] = int16_t(y);
      gridBoundaryData[r] = 0;
      gridBoundaryData[r + 1] = int16_t(y);
    }
  }

  void finalize(TexData& pts) {  // gridFinalizeBindGroup (main.js:218-234)
    Mod m = MOD(gridFinalizeShaderCode);
    m.bind(0, &uni); m.bind(1, &pts); m.bind(2, &gridBoundaries); m.bind(3, &gridArea);
    m.bind(4, &faceLengths); m.bind(5, &cellDistances);
    m.dispatch(wg(M), wg(N), 1);
  }

  // prepareGrid (main.js:658-705), grid part
  void prepare_grid(int iters) {
    std::memcpy(gridPoints0.f.data(), gridVtxData.data(), gridVtxData.size() * sizeof(float));
    std::memcpy(gridBoundaries.s.data(), gridBoundaryData.data(), gridBoundaryData.size() * sizeof(int16_t));
    Mod in = MOD(gridInterpolationShaderCode);
    in.bind(0, &uni); in.bind(1, &gridPoints0); in.bind(2, &gridPoints1); in.bind(3, &gridBoundaries);
    in.dispatch(wg(M), wg(N + 1), 1);
    gridPoints0.f = gridPoints1.f;  // copyTextureToTexture gp1 -> gp0
    Mod el = MOD(gridEllipticPoissonShaderCode);
    int pp = 0;
    for (int i = 0; i < iters; i++) {
      TexData& src = pp == 0 ? gridPoints1 : gridPoints0;
      TexData& dst = pp == 0 ? gridPoints0 : gridPoints1;
      el.bind(0, &uni); el.bind(1, &src); el.bind(2, &dst); el.bind(3, &gridBoundaries);
      el.dispatch(wg(M), wg(N + 1), 1);
      pp = 1 - pp;
    }
    finalize(pp == 0 ? gridPoints1 : gridPoints0);
  }
  // Parity injection: the same grid in both vertex textures, then the metrics.
  void set_grid(const float* xy) {
    std::memcpy(gridPoints0.f.data(), xy, gridPoints0.f.size() * sizeof(float));
    std::memcpy(gridPoints1.f.data(), xy, gridPoints1.f.size() * sizeof(float));
    for (int y = 0; y <= N; y++) {
      size_t l = ((size_t)y * M + 0) * 2, r = ((size_t)y * M + (M - 1)) * 2;
      gridBoundaries.s[l] = int16_t(M - 1); gridBoundaries.s[l + 1] = int16_t(y);
      gridBoundaries.s[r] = 0; gridBoundaries.s[r + 1] = int16_t(y);
    }
    finalize(gridPoints1);
  }

  void post() {  // visualization + CFL reduction on state2 (main.js:649-652, 789-792)
    Mod v = MOD(visualizationShaderCode);
    v.bind(0, &uni); v.bind(1, &state2); v.bind(2, &faceLengths); v.bind(3, &gridArea);
    v.bind(4, &vis); v.bind(5, waveSpeeds.data());
    v.dispatch(wg(M), wg(N), 1);
    Mod c = MOD(cflReductionShaderCode);
    c.bind(0, &uni); c.bind(1, waveSpeeds.data()); c.bind(2, &maxWaveSpeed);
    c.dispatch((unsigned)(((long long)M * N + 255) / 256), 1, 1);
  }
  // Raw field value of display mode `mode` (2 density, 3 temperature, 4 pressure,
  // 5 Mach, 8 entropy) of state2 from the visualization shader's own arithmetic
  // (translate.py's field probe), M x N floats.
  void field(int mode, float* out) {
    std::vector<float> buf((size_t)M * N, 0.0f);
    Uniforms u = uni;
    u.simDisplayMode = (float)mode;
    Mod v = MOD(visualizationFieldProbe);
    v.bind(0, &u); v.bind(1, &state2); v.bind(2, &faceLengths); v.bind(3, &gridArea);
    v.bind(4, &vis); v.bind(5, buf.data());
    v.dispatch(wg(M), wg(N), 1);
    std::memcpy(out, buf.data(), buf.size() * sizeof(float));
  }
  // prepareState (main.js:631-655); mode 1 starts from uni.inState everywhere instead of
  // the reference's fluid at rest (new option for freestream starts).
  void prepare_state(int mode) {
    if (mode == 0) {
      Mod m = MOD(prepareStateShaderCode);
      m.bind(0, &uni); m.bind(1, &state0);
      m.dispatch(wg(M), wg(N + 3), 1);
    } else {
      for (size_t c = 0; c < (size_t)M * (N + 3); c++)
        for (int k = 0; k < 4; k++) state0.f[c * 4 + k] = uni.inState[k];
    }
    state1.f = state0.f;
    state2.f = state0.f;
    post();
  }
  void set_state(const float* q) {
    std::memcpy(state2.f.data(), q, state2.f.size() * sizeof(float));
    post();
  }

  void boundary(TexData& in, TexData& out) {
    Mod b = MOD(boundaryShaderCode);
    b.bind(0, &uni); b.bind(1, &gridPoints0); b.bind(2, &gridBoundaries); b.bind(3, &in); b.bind(4, &out);
    b.dispatch(wg(M), wg(N + 3), 1);
  }
  void fluxes(TexData& s) {
    vflux.bind(0, &uni); vflux.bind(1, &gridPoints0); vflux.bind(2, &gridBoundaries); vflux.bind(3, &s);
    vflux.bind(4, &fluxY);
    vflux.dispatch(wg(M), wg(N + 1), 1);
    hflux.bind(0, &uni); hflux.bind(1, &gridPoints0); hflux.bind(2, &gridBoundaries); hflux.bind(3, &s);
    hflux.bind(4, &fluxX);
    hflux.dispatch(wg(M + 1), wg(N), 1);
  }
  void residual_pass() {
    Mod r = MOD(residualShaderCode);
    r.bind(0, &uni); r.bind(1, &fluxX); r.bind(2, &fluxY); r.bind(3, &residual); r.bind(4, &faceLengths);
    r.bind(5, &gridArea);
    r.dispatch(wg(M), wg(N), 1);
  }
  // One frame of the hot loop (main.js:744-791) without the inflow ramp.
  float frame(int steps) {
    float dt = std::fmin(uni.maxdt, uni.cflFactor / bitcast_f32(maxWaveSpeed));
    Mod s1 = MOD(integrationStage1ShaderCode), s2 = MOD(integrationStage2ShaderCode),
        s3 = MOD(integrationStage3ShaderCode);
    for (int i = 0; i < steps; i++) {
      boundary(state2, state0);
      fluxes(state0);
      residual_pass();
      s1.bind(0, &uni); s1.bind(1, &residual); s1.bind(2, &state0); s1.bind(3, &state1); s1.bind(4, &maxWaveSpeed);
      s1.dispatch(wg(M), wg(N), 1);
      boundary(state1, state2);
      fluxes(state2);
      residual_pass();
      s2.bind(0, &uni); s2.bind(1, &residual); s2.bind(2, &state0); s2.bind(3, &state1); s2.bind(4, &state2);
      s2.bind(5, &maxWaveSpeed);
      s2.dispatch(wg(M), wg(N), 1);
      boundary(state2, state1);
      fluxes(state1);
      residual_pass();
      s3.bind(0, &uni); s3.bind(1, &residual); s3.bind(2, &state0); s3.bind(3, &state1); s3.bind(4, &state2);
      s3.bind(5, &maxWaveSpeed);
      s3.dispatch(wg(M), wg(N), 1);
    }
    post();
    return dt;
  }
  // Residual of the current state2 without advancing it (boundary into state0).
  void eval_residual() {
    boundary(state2, state0);
    fluxes(state0);
    residual_pass();
  }
  // force calc + integration (main.js:808-810, graphs.js:5-103)
  void forces(double* out) {
    Mod f = MOD(forceCalcShaderCode);
    f.bind(0, &uni); f.bind(1, &state2); f.bind(2, &gridPoints0); f.bind(3, forceValues.data());
    f.dispatch((unsigned)((M + 15) / 16), 1, 1);
    Mod g = MOD(forceIntegrationShaderCode);
    g.bind(0, &uni); g.bind(1, &guni); g.bind(2, forceValues.data()); g.bind(3, ring.data());
    g.bind(4, forceVector);
    g.dispatch(1, 1, 1);
    out[0] = forceVector[0]; out[1] = forceVector[1];
    for (int k = 0; k < 4; k++) out[2 + k] = ring[k];
  }
  TexData* tex(int which) {
    switch (which) {
      case 0: return &gridPoints0; case 1: return &gridPoints1; case 2: return &gridArea;
      case 3: return &faceLengths; case 4: return &state0; case 5: return &state1; case 6: return &state2;
      case 7: return &fluxX; case 8: return &fluxY; case 9: return &residual;
      default: return nullptr;
    }
  }
};
}  // namespace

extern "C" {
void* ref_create(int M, int N) { return new RefSim(M, N); }
void ref_destroy(void* h) { delete static_cast<RefSim*>(h); }
void ref_set_uniforms(void* h, const RefUniforms* u) { static_cast<RefSim*>(h)->set_uniforms(*u); }
void ref_set_boundaries(void* h, const float* body, const float* outer) { static_cast<RefSim*>(h)->set_boundaries(body, outer); }
void ref_prepare_grid(void* h, int iters) { static_cast<RefSim*>(h)->prepare_grid(iters); }
void ref_set_grid(void* h, const float* xy) { static_cast<RefSim*>(h)->set_grid(xy); }
void ref_prepare_state(void* h, int mode) { static_cast<RefSim*>(h)->prepare_state(mode); }
void ref_set_state(void* h, const float* q) { static_cast<RefSim*>(h)->set_state(q); }
double ref_frame(void* h, int steps) { return static_cast<RefSim*>(h)->frame(steps); }
void ref_eval_residual(void* h) { static_cast<RefSim*>(h)->eval_residual(); }
void ref_forces(void* h, double* out) { static_cast<RefSim*>(h)->forces(out); }
uint32_t ref_max_wave_bits(void* h) { return static_cast<RefSim*>(h)->maxWaveSpeed; }
void ref_field(void* h, int mode, float* out) { static_cast<RefSim*>(h)->field(mode, out); }
void ref_get_wave_speeds(void* h, float* w) {
  auto* r = static_cast<RefSim*>(h);
  std::memcpy(w, r->waveSpeeds.data(), r->waveSpeeds.size() * sizeof(float));
}
// which: 0 gridPoints0, 1 gridPoints1, 2 gridArea, 3 faceLengths, 4-6 state0-2, 7 fluxX, 8 fluxY, 9 residual
long long ref_texture_size(void* h, int which) {
  TexData* t = static_cast<RefSim*>(h)->tex(which);
  return t ? (long long)t->w * t->h * t->ch : -1;
}
void ref_get_texture(void* h, int which, float* out) {
  TexData* t = static_cast<RefSim*>(h)->tex(which);
  if (t) std::memcpy(out, t->f.data(), t->f.size() * sizeof(float));
}
}
