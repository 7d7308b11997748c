// In-register inverse DFT butterflies (radix 2, 4, 8, 16) for the fused
// matched-filter kernels.  "Inverse" means X[k] = sum_n x[n] * exp(+2*pi*i*n*k/R),
// unnormalised: the correlation z[k] = sum_f D[f] conj(H[f]) exp(+2*pi*i*f*k/n)
// is an inverse transform of the conjugate product (the convention of
// python/matchedfilter/matchedfilter.h:35-52 in the reference).
//
// Each butterfly works on a compile-time strided view of a register array so
// that one thread can run several small butterflies over its 16 values.  The
// 8- and 16-point transforms are two-level Cooley-Tukey splits with the inner
// twiddles as literal constants (cos/sin of multiples of pi/8, written out to
// double precision and rounded once to float).
#pragma once
#include <cuda_runtime.h>

namespace mfb {

struct cf { float x, y; };

__device__ __forceinline__ cf cadd(cf a, cf b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ cf csub(cf a, cf b) { return {a.x - b.x, a.y - b.y}; }
// a * b
__device__ __forceinline__ cf cmul(cf a, cf b) {
  return {fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x)};
}
// a * i
__device__ __forceinline__ cf cmul_i(cf a) { return {-a.y, a.x}; }

constexpr float kSqrtHalf = 0.70710678118654752440f;
constexpr float kCos1_16 = 0.92387953251128675613f;   // cos(pi/8)
constexpr float kSin1_16 = 0.38268343236508977173f;   // sin(pi/8)

// a * exp(+2*pi*i*e/16) for the exponents the 16-point split needs.
template <int E>
__device__ __forceinline__ cf tw16(cf a) {
  constexpr int e = E & 15;
  if constexpr (e == 0) return a;
  else if constexpr (e == 4) return cmul_i(a);
  else if constexpr (e == 8) return {-a.x, -a.y};
  else if constexpr (e == 12) return {a.y, -a.x};
  else if constexpr (e == 2) return {kSqrtHalf * (a.x - a.y), kSqrtHalf * (a.x + a.y)};
  else if constexpr (e == 6) return {-kSqrtHalf * (a.x + a.y), kSqrtHalf * (a.x - a.y)};
  else if constexpr (e == 10) return {kSqrtHalf * (a.y - a.x), -kSqrtHalf * (a.x + a.y)};
  else if constexpr (e == 14) return {kSqrtHalf * (a.x + a.y), kSqrtHalf * (a.y - a.x)};
  else {
    // odd multiples of pi/8: c = cos(e*pi/8), s = sin(e*pi/8)
    constexpr float c = (e == 1 || e == 15) ? kCos1_16 : (e == 3 || e == 13) ? kSin1_16
                       : (e == 5 || e == 11) ? -kSin1_16 : -kCos1_16;
    constexpr float s = (e == 1 || e == 7) ? kSin1_16 : (e == 3 || e == 5) ? kCos1_16
                       : (e == 9 || e == 15) ? -kSin1_16 : -kCos1_16;
    return {fmaf(a.x, c, -a.y * s), fmaf(a.x, s, a.y * c)};
  }
}

// 2-point: v[O], v[O+S]
template <int O, int S>
__device__ __forceinline__ void dft2(cf *v) {
  cf a = v[O], b = v[O + S];
  v[O] = cadd(a, b);
  v[O + S] = csub(a, b);
}

// 4-point inverse DFT in place on v[O + S*q], q = 0..3, natural order.
template <int O, int S>
__device__ __forceinline__ void dft4(cf *v) {
  cf x0 = v[O], x1 = v[O + S], x2 = v[O + 2 * S], x3 = v[O + 3 * S];
  cf a = cadd(x0, x2), b = csub(x0, x2);
  cf c = cadd(x1, x3), d = cmul_i(csub(x1, x3));
  v[O] = cadd(a, c);
  v[O + 2 * S] = csub(a, c);
  v[O + S] = cadd(b, d);
  v[O + 3 * S] = csub(b, d);
}

// 8-point inverse DFT in place on v[O + S*q], q = 0..7, natural order.
// n = 2*n1 + n2, k = k1 + 4*k2: two 4-point DFTs, twiddle w8^(n2*k1), 2-point DFTs.
template <int O, int S>
__device__ __forceinline__ void dft8(cf *v) {
  dft4<O, 2 * S>(v);          // n2 = 0: x[0], x[2], x[4], x[6] -> A0[k1] at slots 0,2,4,6
  dft4<O + S, 2 * S>(v);      // n2 = 1: x[1], x[3], x[5], x[7] -> A1[k1] at slots 1,3,5,7
  cf a0 = v[O], a1 = v[O + 2 * S], a2 = v[O + 4 * S], a3 = v[O + 6 * S];
  cf b0 = v[O + S], b1 = tw16<2>(v[O + 3 * S]), b2 = tw16<4>(v[O + 5 * S]),
     b3 = tw16<6>(v[O + 7 * S]);
  v[O] = cadd(a0, b0);          v[O + 4 * S] = csub(a0, b0);
  v[O + S] = cadd(a1, b1);      v[O + 5 * S] = csub(a1, b1);
  v[O + 2 * S] = cadd(a2, b2);  v[O + 6 * S] = csub(a2, b2);
  v[O + 3 * S] = cadd(a3, b3);  v[O + 7 * S] = csub(a3, b3);
}

// 16-point inverse DFT in place on v[q], q = 0..15, natural order.
// n = 4*n1 + n2, k = k1 + 4*k2: four 4-point DFTs over n1 (per n2), twiddle
// w16^(n2*k1), then four 4-point DFTs over n2 (per k1).
__device__ __forceinline__ void dft16(cf *v) {
  dft4<0, 4>(v);  // n2 = 0 -> A[0][k1] at slots 0,4,8,12
  dft4<1, 4>(v);  // n2 = 1 -> A[1][k1] at slots 1,5,9,13
  dft4<2, 4>(v);
  dft4<3, 4>(v);
  v[5] = tw16<1>(v[5]);  v[9] = tw16<2>(v[9]);   v[13] = tw16<3>(v[13]);
  v[6] = tw16<2>(v[6]);  v[10] = tw16<4>(v[10]); v[14] = tw16<6>(v[14]);
  v[7] = tw16<3>(v[7]);  v[11] = tw16<6>(v[11]); v[15] = tw16<9>(v[15]);
  // slots 4*k1 + n2 hold A[n2][k1]; DFT over n2 for each k1 -> X[k1 + 4*k2]
  dft4<0, 1>(v);
  dft4<4, 1>(v);
  dft4<8, 1>(v);
  dft4<12, 1>(v);
  // now slot 4*k1 + k2 holds X[k1 + 4*k2]; transpose the 4x4 to natural order
  cf t;
  t = v[1]; v[1] = v[4]; v[4] = t;
  t = v[2]; v[2] = v[8]; v[8] = t;
  t = v[3]; v[3] = v[12]; v[12] = t;
  t = v[6]; v[6] = v[9]; v[9] = t;
  t = v[7]; v[7] = v[13]; v[13] = t;
  t = v[11]; v[11] = v[14]; v[14] = t;
}

// R-point inverse DFT on v[O + S*q], q = 0..R-1 (R in 2,4,8,16; O=0,S=1 for 16).
template <int R, int O, int S>
__device__ __forceinline__ void dftR(cf *v) {
  if constexpr (R == 2) dft2<O, S>(v);
  else if constexpr (R == 4) dft4<O, S>(v);
  else if constexpr (R == 8) dft8<O, S>(v);
  else {
    static_assert(R == 16 && O == 0 && S == 1, "radix-16 runs on a whole register file");
    dft16(v);
  }
}

}  // namespace mfb
