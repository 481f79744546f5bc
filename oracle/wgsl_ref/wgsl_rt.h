// ORACLE — test infrastructure only.
//
// CPU runtime for WGSL compute shaders translated to C++ by translate.py.  It gives
// the WGSL built-in types and functions the meaning the WGSL specification defines
// (component-wise vector arithmetic, mix = e1*(1-e3)+e2*e3, step(edge,x) = x>=edge,
// normalize = e/length(e), reflect = e1-2*dot(e2,e1)*e2, textureLoad/textureStore on
// 2-D texel arrays with zero for out-of-range loads and dropped out-of-range stores),
// in IEEE single precision with no contraction.  Dispatches run each workgroup's
// invocations; shaders that call workgroupBarrier() are C++20 coroutines resumed
// invocation by invocation between barriers, workgroup 0 first.
#pragma once
#include <atomic>
#include <cmath>
#include <coroutine>
#include <cstdint>
#include <cstring>
#include <exception>
#include <type_traits>
#include <vector>

namespace wgsl {
using f32 = float;
using u32 = uint32_t;
using i32 = int32_t;

template <class T> struct vec2;
template <class T> struct vec3;
template <class T> struct vec4;
template <class T> struct is_vec : std::false_type {};
template <class T> struct is_vec<vec2<T>> : std::true_type {};
template <class T> struct is_vec<vec3<T>> : std::true_type {};
template <class T> struct is_vec<vec4<T>> : std::true_type {};
template <class T> constexpr bool is_vec_v = is_vec<std::decay_t<T>>::value;

template <class T, class A> inline void flat_push(T* out, int& n, const A& a) {
  if constexpr (is_vec_v<A>) {
    for (int k = 0; k < A::N; k++) out[n++] = T(a[k]);
  } else {
    out[n++] = T(a);
  }
}

#define WGSL_VEC_COMMON(CLS, NN)                                                        \
  static constexpr int N = NN;                                                     \
  T& operator[](int k) { return (&x)[k]; }                                         \
  const T& operator[](int k) const { return (&x)[k]; }                             \
  template <class A0, class... A, class = std::enable_if_t<!(sizeof...(A) == 0 &&  \
            std::is_same_v<std::decay_t<A0>, CLS<T>>)>>                            \
  explicit CLS(const A0& a0, const A&... a) {                                     \
    T buf[NN] = {};                                                                \
    int n = 0;                                                                     \
    flat_push(buf, n, a0);                                                         \
    (flat_push(buf, n, a), ...);                                                   \
    if (n == 1)                                                                    \
      for (int k = 0; k < NN; k++) (*this)[k] = buf[0];                            \
    else                                                                           \
      for (int k = 0; k < NN; k++) (*this)[k] = buf[k];                            \
  }

template <class T> struct vec2 {
  T x{}, y{};
  vec2() = default;
  vec2(const vec2&) = default;
  vec2& operator=(const vec2&) = default;
  WGSL_VEC_COMMON(vec2, 2)
  vec2<T> xy() const { return vec2<T>(x, y); }
};
template <class T> struct vec3 {
  T x{}, y{}, z{};
  vec3() = default;
  vec3(const vec3&) = default;
  vec3& operator=(const vec3&) = default;
  WGSL_VEC_COMMON(vec3, 3)
  vec2<T> xy() const { return vec2<T>(x, y); }
  vec2<T> yz() const { return vec2<T>(y, z); }
};
template <class T> struct vec4 {
  T x{}, y{}, z{}, w{};
  vec4() = default;
  vec4(const vec4&) = default;
  vec4& operator=(const vec4&) = default;
  WGSL_VEC_COMMON(vec4, 4)
  vec2<T> xy() const { return vec2<T>(x, y); }
  vec2<T> yz() const { return vec2<T>(y, z); }
  vec2<T> zw() const { return vec2<T>(z, w); }
  vec3<T> xyz() const { return vec3<T>(x, y, z); }
};

using vec2f = vec2<f32>; using vec3f = vec3<f32>; using vec4f = vec4<f32>;
using vec2u = vec2<u32>; using vec3u = vec3<u32>; using vec4u = vec4<u32>;
using vec2i = vec2<i32>; using vec3i = vec3<i32>; using vec4i = vec4<i32>;

// Common type of a concrete operand and an abstract-int literal (C++ int): a WGSL
// literal takes the type of the other operand.
template <class A, class B> struct ct {
  using type = std::conditional_t<std::is_same_v<A, B>, A, std::conditional_t<std::is_same_v<A, int>, B, A>>;
};
template <class A, class B> using ct_t = typename ct<std::decay_t<A>, std::decay_t<B>>::type;

template <class V> struct elem { using type = V; };
template <class T> struct elem<vec2<T>> { using type = T; };
template <class T> struct elem<vec3<T>> { using type = T; };
template <class T> struct elem<vec4<T>> { using type = T; };
template <class V> using elem_t = typename elem<std::decay_t<V>>::type;

template <class V, class R> struct rebind;
template <class T, class R> struct rebind<vec2<T>, R> { using type = vec2<R>; };
template <class T, class R> struct rebind<vec3<T>, R> { using type = vec3<R>; };
template <class T, class R> struct rebind<vec4<T>, R> { using type = vec4<R>; };

// ---- component-wise operators ----
#define WGSL_BINOP(OP)                                                                          \
  template <class V, std::enable_if_t<is_vec_v<V>, int> = 0>                                    \
  inline V operator OP(const V& a, const V& b) {                                                \
    V r; for (int k = 0; k < V::N; k++) r[k] = a[k] OP b[k]; return r;                          \
  }                                                                                             \
  template <class V, class S, std::enable_if_t<is_vec_v<V> && std::is_arithmetic_v<S>, int> = 0> \
  inline V operator OP(const V& a, S s) {                                                       \
    V r; for (int k = 0; k < V::N; k++) r[k] = a[k] OP elem_t<V>(s); return r;                  \
  }                                                                                             \
  template <class V, class S, std::enable_if_t<is_vec_v<V> && std::is_arithmetic_v<S>, int> = 0> \
  inline V operator OP(S s, const V& a) {                                                       \
    V r; for (int k = 0; k < V::N; k++) r[k] = elem_t<V>(s) OP a[k]; return r;                  \
  }                                                                                             \
  template <class V, class B, std::enable_if_t<is_vec_v<V>, int> = 0>                           \
  inline V& operator OP##=(V& a, const B& b) { a = a OP b; return a; }
WGSL_BINOP(+)
WGSL_BINOP(-)
WGSL_BINOP(*)
WGSL_BINOP(/)
WGSL_BINOP(%)
#undef WGSL_BINOP
template <class V, std::enable_if_t<is_vec_v<V>, int> = 0> inline V operator-(const V& a) {
  V r; for (int k = 0; k < V::N; k++) r[k] = -a[k]; return r;
}
#define WGSL_CMP(OP)                                                                             \
  template <class V, std::enable_if_t<is_vec_v<V>, int> = 0>                                     \
  inline typename rebind<V, bool>::type operator OP(const V& a, const V& b) {                    \
    typename rebind<V, bool>::type r; for (int k = 0; k < V::N; k++) r[k] = a[k] OP b[k]; return r; \
  }
WGSL_CMP(==)
WGSL_CMP(!=)
WGSL_CMP(<)
WGSL_CMP(<=)
WGSL_CMP(>)
WGSL_CMP(>=)
#undef WGSL_CMP
template <class V, std::enable_if_t<is_vec_v<V>, int> = 0> inline bool any(const V& v) {
  for (int k = 0; k < V::N; k++) if (v[k]) return true; return false;
}
template <class V, std::enable_if_t<is_vec_v<V>, int> = 0> inline bool all(const V& v) {
  for (int k = 0; k < V::N; k++) if (!v[k]) return false; return true;
}

// ---- scalar built-ins ----
inline f32 abs(f32 e) { return std::fabs(e); }
inline i32 abs(i32 e) { return e < 0 ? -e : e; }
inline f32 sqrt(f32 e) { return std::sqrt(e); }
inline f32 exp(f32 e) { return std::exp(e); }
inline f32 log(f32 e) { return std::log(e); }
inline f32 pow(f32 a, f32 b) { return std::pow(a, b); }
inline f32 sign(f32 e) { return e > 0.0f ? 1.0f : (e < 0.0f ? -1.0f : 0.0f); }
template <class T> inline T smax(T a, T b) {
  if constexpr (std::is_floating_point_v<T>) return std::fmax(a, b); else return a < b ? b : a;
}
template <class T> inline T smin(T a, T b) {
  if constexpr (std::is_floating_point_v<T>) return std::fmin(a, b); else return b < a ? b : a;
}
template <class A, class B, std::enable_if_t<!is_vec_v<A> && !is_vec_v<B>, int> = 0>
inline ct_t<A, B> max(A a, B b) { using R = ct_t<A, B>; return smax<R>(R(a), R(b)); }
template <class A, class B, std::enable_if_t<!is_vec_v<A> && !is_vec_v<B>, int> = 0>
inline ct_t<A, B> min(A a, B b) { using R = ct_t<A, B>; return smin<R>(R(a), R(b)); }
template <class A, class B, class C, std::enable_if_t<!is_vec_v<A>, int> = 0>
inline auto clamp(A e, B lo, C hi) { using R = ct_t<ct_t<A, B>, C>; return smin<R>(smax<R>(R(e), R(lo)), R(hi)); }
inline f32 saturate(f32 e) { return smin<f32>(smax<f32>(e, 0.0f), 1.0f); }
inline f32 step(f32 edge, f32 x) { return edge <= x ? 1.0f : 0.0f; }
inline f32 mix(f32 a, f32 b, f32 t) { return a * (1.0f - t) + b * t; }
template <class T, std::enable_if_t<!is_vec_v<T>, int> = 0> inline T select(T f, T t, bool c) { return c ? t : f; }
inline f32 select(double f, f32 t, bool c) { return c ? t : f32(f); }
inline f32 bitcast_f32(u32 u) { f32 f; std::memcpy(&f, &u, 4); return f; }
inline u32 bitcast_u32(f32 f) { u32 u; std::memcpy(&u, &f, 4); return u; }

// ---- vector built-ins ----
template <class V, std::enable_if_t<is_vec_v<V>, int> = 0> inline V abs(const V& v) {
  V r; for (int k = 0; k < V::N; k++) r[k] = abs(v[k]); return r;
}
template <class V, std::enable_if_t<is_vec_v<V>, int> = 0> inline V sign(const V& v) {
  V r; for (int k = 0; k < V::N; k++) r[k] = sign(v[k]); return r;
}
template <class V, std::enable_if_t<is_vec_v<V>, int> = 0> inline V saturate(const V& v) {
  V r; for (int k = 0; k < V::N; k++) r[k] = saturate(v[k]); return r;
}
template <class V, std::enable_if_t<is_vec_v<V>, int> = 0> inline V max(const V& a, const V& b) {
  V r; for (int k = 0; k < V::N; k++) r[k] = smax(a[k], b[k]); return r;
}
template <class V, std::enable_if_t<is_vec_v<V>, int> = 0> inline V min(const V& a, const V& b) {
  V r; for (int k = 0; k < V::N; k++) r[k] = smin(a[k], b[k]); return r;
}
template <class V, std::enable_if_t<is_vec_v<V>, int> = 0> inline V step(const V& e, const V& x) {
  V r; for (int k = 0; k < V::N; k++) r[k] = step(e[k], x[k]); return r;
}
template <class V, std::enable_if_t<is_vec_v<V>, int> = 0> inline V mix(const V& a, const V& b, const V& t) {
  V r; for (int k = 0; k < V::N; k++) r[k] = mix(a[k], b[k], t[k]); return r;
}
template <class V, std::enable_if_t<is_vec_v<V>, int> = 0> inline V mix(const V& a, const V& b, f32 t) {
  V r; for (int k = 0; k < V::N; k++) r[k] = mix(a[k], b[k], t); return r;
}
template <class V, std::enable_if_t<is_vec_v<V>, int> = 0> inline V select(const V& f, const V& t, bool c) {
  return c ? t : f;
}
template <class V, class BV, std::enable_if_t<is_vec_v<V> && is_vec_v<BV>, int> = 0>
inline V select(const V& f, const V& t, const BV& c) {
  V r; for (int k = 0; k < V::N; k++) r[k] = c[k] ? t[k] : f[k]; return r;
}
template <class V, std::enable_if_t<is_vec_v<V>, int> = 0> inline elem_t<V> dot(const V& a, const V& b) {
  elem_t<V> s = a[0] * b[0];
  for (int k = 1; k < V::N; k++) s = s + a[k] * b[k];
  return s;
}
template <class V, std::enable_if_t<is_vec_v<V>, int> = 0> inline f32 length(const V& v) { return std::sqrt(dot(v, v)); }
inline f32 length(f32 e) { return std::fabs(e); }
template <class V, std::enable_if_t<is_vec_v<V>, int> = 0> inline V normalize(const V& v) { return v / length(v); }
template <class V, std::enable_if_t<is_vec_v<V>, int> = 0> inline V reflect(const V& e1, const V& e2) {
  return e1 - 2.0f * dot(e2, e1) * e2;
}

// ---- resources ----
enum TexKind { TEX_F32 = 0, TEX_S16 = 1 };
struct TexData {
  int w = 0, h = 0, ch = 4, kind = TEX_F32;
  std::vector<float> f;     // w*h*ch floats
  std::vector<int16_t> s;   // w*h*ch int16
  void init(int w_, int h_, int ch_, int kind_) {
    w = w_; h = h_; ch = ch_; kind = kind_;
    if (kind == TEX_F32) f.assign((size_t)w * h * ch, 0.0f); else s.assign((size_t)w * h * ch, 0);
  }
};
struct TexF { TexData* t = nullptr; };  // texture_2d<f32>
struct TexI { TexData* t = nullptr; };  // texture_2d<i32>
struct TexW { TexData* t = nullptr; };  // texture_storage_2d<format, write>

template <class C> inline bool tex_in(const TexData* t, const C& c) {
  return (long long)c.x >= 0 && (long long)c.y >= 0 && (long long)c.x < t->w && (long long)c.y < t->h;
}
template <class C> inline vec4f textureLoad(const TexF& tx, const C& c, int) {
  const TexData* t = tx.t;
  vec4f r(0.0f, 0.0f, 0.0f, 1.0f);
  if (!tex_in(t, c)) return vec4f(0.0f);
  size_t b = ((size_t)c.y * t->w + (size_t)c.x) * t->ch;
  for (int k = 0; k < t->ch; k++) r[k] = t->f[b + k];
  return r;
}
template <class C> inline vec4i textureLoad(const TexI& tx, const C& c, int) {
  const TexData* t = tx.t;
  vec4i r(0, 0, 0, 1);
  if (!tex_in(t, c)) return vec4i(0);
  size_t b = ((size_t)c.y * t->w + (size_t)c.x) * t->ch;
  for (int k = 0; k < t->ch; k++) r[k] = t->s[b + k];
  return r;
}
template <class C> inline void textureStore(const TexW& tx, const C& c, const vec4f& v) {
  TexData* t = tx.t;
  if (!tex_in(t, c)) return;
  size_t b = ((size_t)c.y * t->w + (size_t)c.x) * t->ch;
  for (int k = 0; k < t->ch; k++) t->f[b + k] = v[k];
}
template <class T> struct Storage {  // var<storage> array<T>
  T* p = nullptr;
  T& operator[](u32 i) const { return p[i]; }
};
template <class T> struct Ref {  // var<storage> T (non-array)
  T* p = nullptr;
  Ref& operator=(const T& v) { *p = v; return *this; }
  operator T() const { return *p; }
};
struct AtomicU32 { u32* p = nullptr; };
inline void atomicStore(AtomicU32* a, u32 v) { std::atomic_ref<u32>(*a->p).store(v); }
inline u32 atomicMax(AtomicU32* a, u32 v) {
  std::atomic_ref<u32> r(*a->p);
  u32 cur = r.load();
  while (cur < v && !r.compare_exchange_weak(cur, v)) {}
  return cur;
}

// ---- dispatch ----
struct Task {
  struct promise_type {
    Task get_return_object() { return Task{std::coroutine_handle<promise_type>::from_promise(*this)}; }
    std::suspend_always initial_suspend() noexcept { return {}; }
    std::suspend_always final_suspend() noexcept { return {}; }
    void return_void() {}
    void unhandled_exception() { std::terminate(); }
  };
  std::coroutine_handle<promise_type> h;
  explicit Task(std::coroutine_handle<promise_type> hh) : h(hh) {}
  Task(Task&& o) noexcept : h(o.h) { o.h = {}; }
  Task(const Task&) = delete;
  ~Task() { if (h) h.destroy(); }
};

using InvokeFn = void (*)(vec3u gid, vec3u lid, vec3u nwg, vec3u wid);
using TaskFn = Task (*)(vec3u gid, vec3u lid, vec3u nwg, vec3u wid);

inline void run_plain(InvokeFn fn, u32 wx, u32 wy, u32 wz, u32 nx, u32 ny, u32 nz) {
  vec3u nwg(nx, ny, nz);
  long long total = (long long)nx * ny * nz;
#pragma omp parallel for schedule(dynamic, 16)
  for (long long w = 0; w < total; w++) {
    vec3u wid(u32(w % nx), u32((w / nx) % ny), u32(w / ((long long)nx * ny)));
    for (u32 lz = 0; lz < wz; lz++)
      for (u32 ly = 0; ly < wy; ly++)
        for (u32 lx = 0; lx < wx; lx++) {
          vec3u lid(lx, ly, lz);
          vec3u gid(wid.x * wx + lx, wid.y * wy + ly, wid.z * wz + lz);
          fn(gid, lid, nwg, wid);
        }
  }
}
inline void run_workgroup_tasks(TaskFn fn, void (*reset)(), u32 wx, u32 wy, u32 wz, vec3u wid, vec3u nwg) {
  reset();
  std::vector<Task> tasks;
  tasks.reserve((size_t)wx * wy * wz);
  for (u32 lz = 0; lz < wz; lz++)
    for (u32 ly = 0; ly < wy; ly++)
      for (u32 lx = 0; lx < wx; lx++) {
        vec3u lid(lx, ly, lz);
        vec3u gid(wid.x * wx + lx, wid.y * wy + ly, wid.z * wz + lz);
        tasks.push_back(fn(gid, lid, nwg, wid));
      }
  bool live = true;
  while (live) {  // one round = every invocation runs to its next barrier (or its end)
    live = false;
    for (auto& t : tasks)
      if (!t.h.done()) { t.h.resume(); if (!t.h.done()) live = true; }
  }
}
inline void run_barrier(TaskFn fn, void (*reset)(), u32 wx, u32 wy, u32 wz, u32 nx, u32 ny, u32 nz) {
  vec3u nwg(nx, ny, nz);
  long long total = (long long)nx * ny * nz;
  if (total == 0) return;
  run_workgroup_tasks(fn, reset, wx, wy, wz, vec3u(0u), nwg);  // workgroup 0 first
#pragma omp parallel for schedule(dynamic, 4)
  for (long long w = 1; w < total; w++) {
    vec3u wid(u32(w % nx), u32((w / nx) % ny), u32(w / ((long long)nx * ny)));
    run_workgroup_tasks(fn, reset, wx, wy, wz, wid, nwg);
  }
}
}  // namespace wgsl
