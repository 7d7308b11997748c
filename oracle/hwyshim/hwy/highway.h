/* Project-written, single-target stand-in for the small part of the Highway
 * SIMD library that the reference CPU engine calls.  It exists only so that
 * the reference's own C/C++ sources can be compiled, unmodified, into the
 * test oracle under oracle/_ref.  It is test infrastructure: nothing in the
 * product links it.
 *
 * One target is generated: 16 float lanes as a GCC vector extension.  The
 * compiler lowers it to AVX-512 when built with -mavx512f and to pairs of
 * AVX2 registers otherwise.  Multiply-add is always a true fused multiply-add
 * (the FMA intrinsics), never a contraction left to the compiler, so the
 * result bits do not depend on the optimiser.
 *
 * Semantics of each operation follow Highway's published documentation
 * (g3doc/quick_reference.md): lane-wise arithmetic, masks from comparisons,
 * IfThenElse(mask, yes, no), whole-vector interleaves and so on.
 */
#ifndef APOGEE_HWYSHIM_HIGHWAY_H_
#define APOGEE_HWYSHIM_HIGHWAY_H_

#include <stdint.h>
#include <string.h>
#include <math.h>
#include <vector>
#include <immintrin.h>

#ifndef HWY_SHIM_TARGET_NAME
#define HWY_SHIM_TARGET_NAME "SHIM16"
#endif

#define HWY_NAMESPACE N_SHIM16
#define HWY_STATIC_NAMESPACE N_SHIM16
#define HWY_SHIM16 (1LL << 10)
#define HWY_AVX2 (1LL << 20)      /* a different value: the AVX2-only code stays out */
#define HWY_TARGET HWY_SHIM16
#define HWY_BEFORE_NAMESPACE() static_assert(true, "")
#define HWY_AFTER_NAMESPACE() static_assert(true, "")
#define HWY_ATTR
#define HWY_INLINE inline __attribute__((always_inline))
#define HWY_MAX_LANES_D(D) (D::kLanes)
#define HWY_EXPORT(name) static_assert(true, "")
#define HWY_DYNAMIC_DISPATCH(name) HWY_NAMESPACE::name
#define HWY_STATIC_DISPATCH(name) HWY_NAMESPACE::name

namespace hwy {

inline const char *TargetName(int64_t t) {
  return t == HWY_SHIM16 ? HWY_SHIM_TARGET_NAME : "unknown";
}
inline int64_t &shim_forced_target() { static int64_t v = 0; return v; }
inline std::vector<int64_t> SupportedAndGeneratedTargets() {
  return std::vector<int64_t>{HWY_SHIM16};
}
inline void SetSupportedTargetsForTest(int64_t t) { shim_forced_target() = t; }

namespace HWY_NAMESPACE {

template <typename T, int N> struct Simd {
  typedef T type;
  static constexpr int kLanes = N;
};
template <typename T, int N> using CappedTag = Simd<T, N>;

template <typename T, int N> struct VecT;
template <int N> struct VecT<float, N> {
  typedef float raw __attribute__((vector_size(4 * N)));
  raw v;
};
template <int N> struct VecT<int32_t, N> {
  typedef int32_t raw __attribute__((vector_size(4 * N)));
  raw v;
};
template <int N> struct MaskT {
  typedef int32_t raw __attribute__((vector_size(4 * N)));
  raw m;   /* all ones where true */
};

template <class D> using Vec = VecT<typename D::type, D::kLanes>;
template <class D> using RebindToSigned = Simd<int32_t, D::kLanes>;

template <class D> HWY_INLINE Vec<D> Zero(D) {
  Vec<D> r; memset(&r, 0, sizeof r); return r;
}
template <class D> HWY_INLINE Vec<D> Set(D, typename D::type x) {
  Vec<D> r; r.v = (typename Vec<D>::raw){} + x; return r;
}
template <class D> HWY_INLINE Vec<D> LoadU(D, const typename D::type *p) {
  Vec<D> r; memcpy(&r.v, p, sizeof r.v); return r;
}
template <class D> HWY_INLINE void StoreU(Vec<D> v, D, typename D::type *p) {
  memcpy(p, &v.v, sizeof v.v);
}
template <typename T, int N> HWY_INLINE VecT<T, N> Add(VecT<T, N> a, VecT<T, N> b) {
  VecT<T, N> r; r.v = a.v + b.v; return r;
}
template <typename T, int N> HWY_INLINE VecT<T, N> Sub(VecT<T, N> a, VecT<T, N> b) {
  VecT<T, N> r; r.v = a.v - b.v; return r;
}
template <typename T, int N> HWY_INLINE VecT<T, N> Mul(VecT<T, N> a, VecT<T, N> b) {
  VecT<T, N> r; r.v = a.v * b.v; return r;
}
/* a*b + c, a*b - c, -a*b + c, -a*b - c; each one rounding (a true FMA). */
#if defined(__AVX512F__)
#define HWY_SHIM_FMA4(NAME, EXPR)                                               \
  template <int N> HWY_INLINE VecT<float, N> NAME(VecT<float, N> a, VecT<float, N> b, VecT<float, N> c) { \
    static_assert(N == 16, "shim vectors are 16 lanes");                        \
    __m512 x, y, z; memcpy(&x, &a, 64); memcpy(&y, &b, 64); memcpy(&z, &c, 64); \
    __m512 w = EXPR; VecT<float, N> r; memcpy(&r, &w, 64); return r; }
HWY_SHIM_FMA4(MulAdd, _mm512_fmadd_ps(x, y, z))
HWY_SHIM_FMA4(MulSub, _mm512_fmsub_ps(x, y, z))
HWY_SHIM_FMA4(NegMulAdd, _mm512_fnmadd_ps(x, y, z))
HWY_SHIM_FMA4(NegMulSub, _mm512_fnmsub_ps(x, y, z))
#elif defined(__FMA__)
#define HWY_SHIM_FMA4(NAME, F)                                                  \
  template <int N> HWY_INLINE VecT<float, N> NAME(VecT<float, N> a, VecT<float, N> b, VecT<float, N> c) { \
    static_assert(N % 8 == 0, "shim vectors are whole AVX registers");          \
    VecT<float, N> r;                                                           \
    for (int h = 0; h < N / 8; h++) {                                           \
      __m256 x, y, z; memcpy(&x, (const float *)&a + 8 * h, 32);                \
      memcpy(&y, (const float *)&b + 8 * h, 32); memcpy(&z, (const float *)&c + 8 * h, 32); \
      __m256 w = F(x, y, z); memcpy((float *)&r + 8 * h, &w, 32); }            \
    return r; }
HWY_SHIM_FMA4(MulAdd, _mm256_fmadd_ps)
HWY_SHIM_FMA4(MulSub, _mm256_fmsub_ps)
HWY_SHIM_FMA4(NegMulAdd, _mm256_fnmadd_ps)
HWY_SHIM_FMA4(NegMulSub, _mm256_fnmsub_ps)
#else
#error "the Highway shim needs FMA (build with -mfma)"
#endif
template <class D, typename T, int N> HWY_INLINE Vec<D> BitCast(D, VecT<T, N> v) {
  static_assert(sizeof(Vec<D>) == sizeof(v), "BitCast size");
  Vec<D> r; memcpy(&r, &v, sizeof r); return r;
}
template <typename T, int N> HWY_INLINE VecT<T, N> Xor(VecT<T, N> a, VecT<T, N> b) {
  VecT<int32_t, N> x, y; memcpy(&x, &a, sizeof x); memcpy(&y, &b, sizeof y);
  x.v ^= y.v; VecT<T, N> r; memcpy(&r, &x, sizeof r); return r;
}
template <typename T, int N> HWY_INLINE MaskT<N> Gt(VecT<T, N> a, VecT<T, N> b) {
  MaskT<N> m; m.m = (a.v > b.v); return m;
}
template <typename T, int N> HWY_INLINE VecT<T, N> IfThenElse(MaskT<N> m, VecT<T, N> yes, VecT<T, N> no) {
  VecT<T, N> r; r.v = m.m ? yes.v : no.v; return r;
}
template <class D, int N> HWY_INLINE MaskT<N> RebindMask(D, MaskT<N> m) { return m; }
template <class D, int N> HWY_INLINE bool AllFalse(D, MaskT<N> m) {
#if defined(__AVX512F__)
  if (N == 16) { __m512i x; memcpy(&x, &m.m, 64); return _mm512_test_epi32_mask(x, x) == 0; }
#endif
  int32_t acc = 0; for (int i = 0; i < N; i++) acc |= m.m[i]; return acc == 0;
}
template <class D> HWY_INLINE MaskT<D::kLanes> LoadMaskBits(D, const uint8_t *bits) {
  MaskT<D::kLanes> m;
  for (int i = 0; i < D::kLanes; i++) m.m[i] = ((bits[i >> 3] >> (i & 7)) & 1) ? -1 : 0;
  return m;
}
template <class D> HWY_INLINE typename D::type ReduceMax(D, Vec<D> v) {
  typename D::type r = v.v[0];
  for (int i = 1; i < D::kLanes; i++) r = v.v[i] > r ? v.v[i] : r;
  return r;
}
template <class D> HWY_INLINE void LoadInterleaved2(D, const typename D::type *p, Vec<D> &a, Vec<D> &b) {
  static_assert(D::kLanes == 16, "shim vectors are 16 lanes");
  Vec<D> x, y; memcpy(&x.v, p, sizeof x.v); memcpy(&y.v, p + 16, sizeof y.v);
  a.v = __builtin_shufflevector(x.v, y.v, 0, 2, 4, 6, 8, 10, 12, 14, 16, 18, 20, 22, 24, 26, 28, 30);
  b.v = __builtin_shufflevector(x.v, y.v, 1, 3, 5, 7, 9, 11, 13, 15, 17, 19, 21, 23, 25, 27, 29, 31);
}
template <class D> HWY_INLINE void StoreInterleaved2(Vec<D> a, Vec<D> b, D, typename D::type *p) {
  static_assert(D::kLanes == 16, "shim vectors are 16 lanes");
  Vec<D> x, y;
  x.v = __builtin_shufflevector(a.v, b.v, 0, 16, 1, 17, 2, 18, 3, 19, 4, 20, 5, 21, 6, 22, 7, 23);
  y.v = __builtin_shufflevector(a.v, b.v, 8, 24, 9, 25, 10, 26, 11, 27, 12, 28, 13, 29, 14, 30, 15, 31);
  memcpy(p, &x.v, sizeof x.v); memcpy(p + 16, &y.v, sizeof y.v);
}
/* Whole-vector interleave of the lower (upper) halves: a0 b0 a1 b1 ... */
template <class D> HWY_INLINE Vec<D> InterleaveWholeLower(D, Vec<D> a, Vec<D> b) {
  static_assert(D::kLanes == 16, "shim vectors are 16 lanes");
  Vec<D> r;
  r.v = __builtin_shufflevector(a.v, b.v, 0, 16, 1, 17, 2, 18, 3, 19, 4, 20, 5, 21, 6, 22, 7, 23);
  return r;
}
template <class D> HWY_INLINE Vec<D> InterleaveWholeUpper(D, Vec<D> a, Vec<D> b) {
  static_assert(D::kLanes == 16, "shim vectors are 16 lanes");
  Vec<D> r;
  r.v = __builtin_shufflevector(a.v, b.v, 8, 24, 9, 25, 10, 26, 11, 27, 12, 28, 13, 29, 14, 30, 15, 31);
  return r;
}

}  // namespace HWY_NAMESPACE
}  // namespace hwy

#endif
