// Fused matched filter at n = 4096 with two pairs per thread (packed FP32x2).
//
// Same pair transform as flat_kernel<4096, MODE_PEAKS> (conjugate product ->
// unnormalised inverse FFT -> per-bin argmax, src/balanced-inl.h:1102-1113 in
// the reference), restructured for sm_100a's packed FP32 instructions: every
// thread carries the same butterfly of TWO pairs at once, lane A and lane B of
// float2 registers (X = (re_A, re_B), Y = (im_A, im_B)), so each add, multiply
// or FMA of the radix-16 Stockham passes is one FADD2 / FMUL2 / FFMA2 for both
// pairs.  The butterflies' operations, their order and their roundings are
// those of the scalar kernel; the packed form halves the FP32 instructions
// and the barriers per pair.
//
// Layout:
//  * a CTA of 256 threads = one pair slot of T = n/16 threads, two pairs per
//    item (pairs 2i and 2i+1 of the dense block or of the row list);
//  * the exchange buffer holds float4 records (re_A, re_B, im_A, im_B) with
//    the scalar kernel's padding (one record per 16), 69.6 KB, so two CTAs fit
//    on an SM;
//  * inter-pass twiddles are float4 (wr, wr, wi, wi) -- the same FP64-built
//    values as the scalar tables, duplicated for the two lanes; six of the
//    fifteen per pass are read, the others are products of two of those
//    (pass_twiddles), which halves the kernel's L1 traffic for twiddles at
//    the cost of about one float ulp in nine of them; the one-pair kernels
//    form theirs the same way, so the outputs stay bit-identical.
// Scope: n = 4096, MODE_PEAKS, the whole lag window with bins a multiple of
// 32 lags and at most KEYCAP bins (the benchmark's and the refine's layout);
// the launcher sends every other run to flat_kernel / rows_kernel.
#pragma once
#include <cstdint>
#include "flat_kernel.cuh"

namespace mfb {

namespace p2 {

__device__ __forceinline__ float2 add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub(float2 a, float2 b) {
  float2 r;
  asm("sub.rn.f32x2 %0, %1, %2;"
      : "=l"(*reinterpret_cast<unsigned long long *>(&r))
      : "l"(*reinterpret_cast<const unsigned long long *>(&a)),
        "l"(*reinterpret_cast<const unsigned long long *>(&b)));
  return r;
}
__device__ __forceinline__ float2 mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 dup(float x) { return make_float2(x, x); }

// 4-point inverse DFT on (X,Y)[O + S*q]; I2: input 2 is first multiplied by i.
// Scalar form: a = x0+x2, b = x0-x2, c = x1+x3, d = i(x1-x3); a+c, b+d, a-c, b-d.
template <int O, int S, bool I2 = false>
__device__ __forceinline__ void dft4(float2 *X, float2 *Y) {
  const float2 x0 = X[O], y0 = Y[O], x1 = X[O + S], y1 = Y[O + S];
  const float2 x3 = X[O + 3 * S], y3 = Y[O + 3 * S];
  float2 ax, ay, bx, by;
  if constexpr (I2) {   // x2 <- i * x2 = (-y2, x2)
    const float2 x2 = X[O + 2 * S], y2 = Y[O + 2 * S];
    ax = sub(x0, y2); ay = add(y0, x2);
    bx = add(x0, y2); by = sub(y0, x2);
  } else {
    const float2 x2 = X[O + 2 * S], y2 = Y[O + 2 * S];
    ax = add(x0, x2); ay = add(y0, y2);
    bx = sub(x0, x2); by = sub(y0, y2);
  }
  const float2 cx = add(x1, x3), cy = add(y1, y3);
  const float2 ex = sub(x1, x3), ey = sub(y1, y3);   // d = i*e = (-ey, ex)
  X[O] = add(ax, cx);          Y[O] = add(ay, cy);
  X[O + 2 * S] = sub(ax, cx);  Y[O + 2 * S] = sub(ay, cy);
  X[O + S] = sub(bx, ey);      Y[O + S] = add(by, ex);
  X[O + 3 * S] = add(bx, ey);  Y[O + 3 * S] = sub(by, ex);
}

// (X,Y)[i] *= exp(+2 pi i e / 16) for the exponents dft16 uses (e != 4).
template <int E>
__device__ __forceinline__ void tw16(float2 *X, float2 *Y, int i) {
  constexpr int e = E & 15;
  const float2 x = X[i], y = Y[i];
  if constexpr (e == 2) {
    X[i] = mul(dup(kSqrtHalf), sub(x, y));
    Y[i] = mul(dup(kSqrtHalf), add(x, y));
  } else if constexpr (e == 6) {
    X[i] = mul(dup(-kSqrtHalf), add(x, y));
    Y[i] = mul(dup(kSqrtHalf), sub(x, y));
  } else {
    static_assert(e == 1 || e == 3 || e == 9, "odd exponents of dft16");
    constexpr float c = (e == 1) ? kCos1_16 : (e == 3) ? kSin1_16 : -kCos1_16;
    constexpr float s = (e == 1) ? kSin1_16 : (e == 3) ? kCos1_16 : -kSin1_16;
    // scalar: {fmaf(x, c, -y*s), fmaf(x, s, y*c)}
    X[i] = fma(x, dup(c), mul(y, dup(-s)));
    Y[i] = fma(x, dup(s), mul(y, dup(c)));
  }
}

// 16-point inverse DFT of (X,Y)[0..15], natural order (the scalar dft16).
__device__ __forceinline__ void dft16(float2 *X, float2 *Y) {
  dft4<0, 4>(X, Y);
  dft4<1, 4>(X, Y);
  dft4<2, 4>(X, Y);
  dft4<3, 4>(X, Y);
  tw16<1>(X, Y, 5);  tw16<2>(X, Y, 9);  tw16<3>(X, Y, 13);
  tw16<2>(X, Y, 6);                     tw16<6>(X, Y, 14);
  tw16<3>(X, Y, 7);  tw16<6>(X, Y, 11); tw16<9>(X, Y, 15);
  dft4<0, 1>(X, Y);
  dft4<4, 1>(X, Y);
  dft4<8, 1, true>(X, Y);    // slot 10 carries the twiddle i
  dft4<12, 1>(X, Y);
  float2 t;
#define P2_SWAP(a, b) t = X[a]; X[a] = X[b]; X[b] = t; t = Y[a]; Y[a] = Y[b]; Y[b] = t;
  P2_SWAP(1, 4) P2_SWAP(2, 8) P2_SWAP(3, 12) P2_SWAP(6, 9) P2_SWAP(7, 13) P2_SWAP(11, 14)
#undef P2_SWAP
}

// (X, Y) *= w for a twiddle w = (wr, wi) shared by both lanes, given as the
// record (wr, wr, wi, wi); scalar cmul: {fmaf(x, wr, -y*wi), fmaf(x, wi, y*wr)}.
__device__ __forceinline__ void twiddle(float2 &x, float2 &y, float4 w) {
  const float2 wr = make_float2(w.x, w.y), wi = make_float2(w.z, w.w);
  const float2 nx = fma(x, wr, mul(y, make_float2(-wi.x, -wi.y)));
  const float2 ny = fma(x, wi, mul(y, wr));
  x = nx;
  y = ny;
}

// Product of two twiddle records (both lanes carry the same value).
__device__ __forceinline__ float4 tw_mul(float4 a, float4 b) {
  float2 x = make_float2(a.x, a.y), y = make_float2(a.z, a.w);
  twiddle(x, y, b);
  return make_float4(x.x, x.y, y.x, y.y);
}

// Read-only 16-byte load kept inside the pair loop: the twiddle tables are
// loop-invariant, and hoisted into registers they would crowd out the
// transform's 64 values.
__device__ __forceinline__ float4 ldg4(const float4 *p) {
  float4 r;
  asm volatile("ld.global.nc.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w) : "l"(p));
  return r;
}

// (X, Y)[q] *= w^q, q = 1..15, for one pass: w^1, w^2, w^3, w^4, w^8, w^12
// come from the FP64-built table (entry q at tw[(q-1)*stride]), the other
// nine are one product of two of those (w^(4a+b) = w^(4a) w^b), a rounding
// error of about one float ulp beside the table's half ulp.
__device__ __forceinline__ void pass_twiddles(float2 *X, float2 *Y, const float4 *tw, int stride) {
  const float4 w1 = ldg4(tw), w2 = ldg4(tw + stride), w3 = ldg4(tw + 2 * stride);
  const float4 w4 = ldg4(tw + 3 * stride), w8 = ldg4(tw + 7 * stride);
  const float4 w12 = ldg4(tw + 11 * stride);
  twiddle(X[1], Y[1], w1);
  twiddle(X[2], Y[2], w2);
  twiddle(X[3], Y[3], w3);
  twiddle(X[4], Y[4], w4);
  twiddle(X[5], Y[5], tw_mul(w4, w1));
  twiddle(X[6], Y[6], tw_mul(w4, w2));
  twiddle(X[7], Y[7], tw_mul(w4, w3));
  twiddle(X[8], Y[8], w8);
  twiddle(X[9], Y[9], tw_mul(w8, w1));
  twiddle(X[10], Y[10], tw_mul(w8, w2));
  twiddle(X[11], Y[11], tw_mul(w8, w3));
  twiddle(X[12], Y[12], w12);
  twiddle(X[13], Y[13], tw_mul(w12, w1));
  twiddle(X[14], Y[14], tw_mul(w12, w2));
  twiddle(X[15], Y[15], tw_mul(w12, w3));
}

}  // namespace p2

struct Flat2Geo {
  static constexpr int N = 4096;
  static constexpr int T = 256;                 // threads per pair slot
  static constexpr int BUF = N + N / 16;        // padded float4 records
  static constexpr int KEYS = 2 * 2 * KEYCAP;   // two pairs, double-buffered
  static constexpr int SMEM = BUF * 16 + KEYS * 8;
  static constexpr int TW = 15 * 16 + 15 * 256; // float4 twiddles of passes 1 and 2
};

// Items [ibeg, iend) of a launch: item i = pairs 2i, 2i+1 of the dense block
// (row = d*nt + t) or of the row list.  a.twid points at Flat2Geo::TW float4
// records: pass 1 at (q-1)*16 + k, pass 2 at 240 + (q-1)*256 + k.
template <int MODE>
__global__ void __launch_bounds__(256, 2)
flat2_kernel(const FlatArgs a) {
  static_assert(MODE == MODE_PEAKS, "peaks only");
  using Geo = Flat2Geo;
  constexpr int T = Geo::T;
  extern __shared__ __align__(16) float4 smem4[];
  float4 *buf = smem4;
  unsigned long long *kslots = reinterpret_cast<unsigned long long *>(smem4 + Geo::BUF);
  const float4 *tw4 = reinterpret_cast<const float4 *>(a.twid);

  const int t = threadIdx.x;
  const int lane = t & 31;
  const long long total = a.list ? (long long)(*a.list_count) : (long long)a.nd * a.nt;
  if (a.list && a.trig_total && blockIdx.x == 0 && threadIdx.x == 0)
    *a.trig_total += (unsigned long long)total;
  const long long items = (total + 1) / 2;
  const long long per = items / gridDim.x, extra = items % gridDim.x;
  const long long ibeg = blockIdx.x * per + (blockIdx.x < extra ? blockIdx.x : extra);
  const long long iend = ibeg + per + (blockIdx.x < extra ? 1 : 0);

  const int bs = a.binsize;
  const float inv_bs = 1.0f / (float)bs;
  const int nb = a.nb;
  const unsigned linv = 31u - (unsigned)lane;
  for (int b = t; b < Geo::KEYS; b += T) kslots[b] = 0ull;
  __syncthreads();

  for (long long item = ibeg; item < iend; ++item) {
    const long long pa = 2 * item, pb = 2 * item + 1;
    const bool live_b = pb < total;
    int row_a = a.list ? a.list[pa] : (int)pa;
    int row_b = live_b ? (a.list ? a.list[pb] : (int)pb) : row_a;
    const int da = row_a / a.nt, ta = row_a - da * a.nt;
    const int db = row_b / a.nt, tb = row_b - db * a.nt;
    // ---- pass 0: loads, conjugate products (scalar, into the two lanes) ------
    float2 X[16], Y[16];
    {
      const float2 *ha = a.tmpl + (long long)(a.t0 + ta) * a.tmpl_stride + t;
      const float2 *hb = a.tmpl + (long long)(a.t0 + tb) * a.tmpl_stride + t;
      const float2 *dpa = a.data + (long long)(a.d0 + da) * a.data_stride + t;
      const float2 *dpb = a.data + (long long)(a.d0 + db) * a.data_stride + t;
      if (da == db) {
#pragma unroll
        for (int s = 0; s < 16; s++) {
          const float2 d = __ldg(dpa + T * s);
          const float2 h = __ldg(ha + T * s), g = __ldg(hb + T * s);
          X[s].x = fmaf(d.x, h.x, d.y * h.y);
          Y[s].x = fmaf(d.y, h.x, -d.x * h.y);
          X[s].y = fmaf(d.x, g.x, d.y * g.y);
          Y[s].y = fmaf(d.y, g.x, -d.x * g.y);
        }
      } else {
#pragma unroll
        for (int s = 0; s < 16; s++) {
          const float2 d = __ldg(dpa + T * s), e = __ldg(dpb + T * s);
          const float2 h = __ldg(ha + T * s), g = __ldg(hb + T * s);
          X[s].x = fmaf(d.x, h.x, d.y * h.y);
          Y[s].x = fmaf(d.y, h.x, -d.x * h.y);
          X[s].y = fmaf(e.x, g.x, e.y * g.y);
          Y[s].y = fmaf(e.y, g.x, -e.x * g.y);
        }
      }
    }
    p2::dft16(X, Y);
    __syncthreads();           // the previous item's parks and keys are read
    {
      float4 *p0 = buf + pad16(t * 16);
#pragma unroll
      for (int q = 0; q < 16; q++) p0[q] = make_float4(X[q].x, X[q].y, Y[q].x, Y[q].y);
    }
    __syncthreads();
    // ---- pass 1 (span 16) ------------------------------------------------------
    {
      const float4 *pl = buf + pad16(t);
#pragma unroll
      for (int q = 0; q < 16; q++) {
        const float4 r = pl[q * (T + T / 16)];
        X[q] = make_float2(r.x, r.y);
        Y[q] = make_float2(r.z, r.w);
      }
      const int k = t & 15;
      p2::pass_twiddles(X, Y, tw4 + k, 16);
      p2::dft16(X, Y);
      __syncthreads();
      float4 *ps = buf + pad16((t >> 4) * 256 + k);
#pragma unroll
      for (int q = 0; q < 16; q++) ps[q * 17] = make_float4(X[q].x, X[q].y, Y[q].x, Y[q].y);
      __syncthreads();
    }
    // ---- pass 2 (span 256) -----------------------------------------------------
    {
      const float4 *pl = buf + pad16(t);
#pragma unroll
      for (int q = 0; q < 16; q++) {
        const float4 r = pl[q * (T + T / 16)];
        X[q] = make_float2(r.x, r.y);
        Y[q] = make_float2(r.z, r.w);
      }
      p2::pass_twiddles(X, Y, tw4 + 240 + t, 256);
      p2::dft16(X, Y);
      __syncthreads();         // buf is free: parks go there
    }
    // Thread t holds z[t + 256 q] of pair A in lane x, of pair B in lane y.
    // ---- per-bin argmax: one redux per slot, warp and pair ---------------------
    unsigned long long *keys = kslots + (int)(item & 1) * 2 * KEYCAP;   // [2][KEYCAP]
    {
      float2 *park = reinterpret_cast<float2 *>(buf);
      // lane q keeps pair A's slot-q maximum, lane 16 + q pair B's
      unsigned my = 0u;
#pragma unroll
      for (int q = 0; q < 16; q++) {
        const float2 m2 = p2::fma(X[q], X[q], p2::mul(Y[q], Y[q]));
        const unsigned ka = (m2.x > a.t2) ? ((__float_as_uint(m2.x) & ~31u) | linv) : 0u;
        const unsigned kb = (live_b && m2.y > a.t2) ? ((__float_as_uint(m2.y) & ~31u) | linv) : 0u;
        const unsigned xa = __reduce_max_sync(0xffffffffu, ka);
        const unsigned xb = __reduce_max_sync(0xffffffffu, kb);
        const int at = 2 * pad16(t + T * q);
        if (ka != 0u && ka == xa) park[at] = make_float2(X[q].x, Y[q].x);
        if (kb != 0u && kb == xb) park[at + 1] = make_float2(X[q].y, Y[q].y);
        my = ((lane & 15) == q) ? (lane < 16 ? xa : xb) : my;
      }
      if (my != 0u) {
        const int q = lane & 15;
        const int k = ((t & ~31) | (31 - (int)(my & 31u))) + T * q;
        const int bin = bin_of((t & ~31) + T * q, bs, inv_bs);
        atomicMax(keys + (lane >> 4) * KEYCAP + bin,
                  ((unsigned long long)(my & ~31u) << 32) | (unsigned)(~k));
      }
    }
    __syncthreads();
    // ---- outputs: threads [0, nb) pair A, [128, 128 + nb) pair B ----------------
    {
      const int sel = t >> 7, b = t & 127;
      const bool mine = b < nb && (sel == 0 || live_b);
      if (mine) {
        const unsigned long long kk = keys[sel * KEYCAP + b];
        const long long row = sel ? row_b : row_a;
        long long ix = -1;
        float2 val = make_float2(0.f, 0.f);
        if (kk != 0ull) {
          const int k = (int)(~(unsigned)kk);
          ix = k;
          val = reinterpret_cast<const float2 *>(buf)[2 * pad16(k) + sel];
        }
        const long long o = row * nb + b;
        a.out_idx[o * a.rs] = ix;
        a.out_val[o * a.rs] = val;
        if (a.host_rec)   // 16-byte store over the host link into the host table
          a.host_rec[o] = make_int4((int)(unsigned)(unsigned long long)ix,
                                    (int)(unsigned)((unsigned long long)ix >> 32),
                                    __float_as_int(val.x), __float_as_int(val.y));
        if (a.out_cnt && kk != 0ull) atomicAdd(a.out_cnt + row, 1);
      }
      // clear the other parity's keys for the next item (not read before the
      // next item's first barrier)
      unsigned long long *nxt = kslots + (int)((item + 1) & 1) * 2 * KEYCAP;
      if (b < nb && (sel == 0 || live_b)) nxt[sel * KEYCAP + b] = 0ull;
    }
  }
}

}  // namespace mfb
