// Fused matched-filter kernel for one CTA-resident transform (n <= 16384).
//
// For every (data d, template t) pair it forms P[f] = D[f] * conj(H[f]),
// runs the unnormalised inverse FFT of P, and reduces each bin of the lag
// window to its loudest sample, so the correlation series never leaves the
// SM.  This is the reference's fused pair transform (python/matchedfilter/
// matchedfilter.h:35-52; src/balanced-inl.h:1102-1113 on the CPU,
// src/gpu/tierb.slang:591-775 on its GPU backends), re-designed for sm_100a:
//
//  * Stockham autosort FFT, radix 16 (first pass radix 2/4/8/16), one
//    butterfly per thread per pass.  A thread keeps 16 complex values in
//    registers; passes exchange through padded shared memory.
//  * The conjugate product is formed while the first pass loads: the
//    template spectrum streams from HBM/L2 with coalesced 8-byte loads, the
//    data spectrum a thread needs sits in its registers for as long as the
//    CTA stays on that data row.
//  * Thread t ends holding z[t + T*q], q = 0..15 (T = n/16).  The per-bin
//    argmax is a warp redux on |z|^2 bit patterns followed by one 64-bit
//    shared-memory atomicMax per warp and bin on the key
//    (|z|^2 bits << 32) | ~lag, which makes the lowest lag win exact ties.
//  * Persistent CTAs walk a contiguous range of pairs, data row outer,
//    template inner, so the data spectrum is reloaded only when the row
//    changes and concurrent CTAs on different rows share templates in L2.
//
// Threshold contract (src/balanced-inl.h:804-886): a bin reports the lag of
// max |z|^2 iff that |z|^2 > thr^2 (thr <= 0 -> > 0, so zero is never a
// peak); otherwise index -1 and value 0.  |z|^2 is fmaf(re, re, im*im) as
// the reference computes it.
//
// MODE_GATE is the hierarchical coarse pass of src/hmf.c:241-300: one bin
// over the coarse window, and instead of writing the peak the pair either
// joins the refine list (coarse max reported and sqrt(max) >= gate) or has
// its full-size output rows written as (-1, 0) right away.
#pragma once
#include <cstdint>
#include "fft_radix.cuh"

namespace mfb {

enum { MODE_PEAKS = 0, MODE_GATE = 1 };

struct FlatArgs {
  const float2 *data;     // row r at data + r*data_stride (first n values used)
  const float2 *tmpl;     // row r at tmpl + r*tmpl_stride
  long long data_stride, tmpl_stride;
  const float2 *twid;     // inter-pass twiddles, layout of twiddle_offset()
  int d0, nd, t0, nt;     // pair block [d0,d0+nd) x [t0,t0+nt); output row = (d-d0)*nt + (t-t0)
  const int32_t *list;    // listed mode: output rows to run; nullptr = dense block
  const int32_t *list_count;  // device count for listed mode
  int ws, we, binsize, nb;    // lag window [ws,we), bins
  float t2;                   // threshold squared (0 if threshold <= 0)
  long long *out_idx;         // [rows][nb], element i at out_idx[i*rs]
  float2 *out_val;            // [rows][nb], element i at out_val[i*rs]
  int rs;                     // 1: separate arrays; 2: interleaved 16-byte (index, value) records
  int32_t *out_cnt;           // [rows] or nullptr (must be zeroed before the launch)
  // MODE_GATE only:
  float gate;                 // fire iff coarse max reported and sqrtf(m2) >= gate
  int32_t *fire_list;         // appended output rows that fired
  int32_t *fire_count;        // device counter (zeroed before the launch)
  int full_nb;                // bins of the full-size output written as (-1,0) when dismissed
  float *coarse_out;          // if set: write max |z| over the window per row instead of gating
  int data_cg;                // 1: data rows were written in this launch (coherent loads)
  // listed mode: if set, the launch adds the row count to this running total
  // (the hierarchical plan's trigger count) -- one thread, once
  unsigned long long *trig_total;
  // if set (record output, rs == 2): every output record is also stored here,
  // the caller's pinned host table seen from the device (flat2_kernel only)
  int4 *host_rec;
};

template <int N>
struct FlatGeo {
  static constexpr int LOG2N = (N == 64) ? 6 : (N == 128) ? 7 : (N == 256) ? 8 : (N == 512) ? 9
                             : (N == 1024) ? 10 : (N == 2048) ? 11 : (N == 4096) ? 12
                             : (N == 8192) ? 13 : (N == 16384) ? 14 : -1;
  static_assert(LOG2N > 0, "single-CTA kernel covers n = 64 .. 16384");
  static constexpr int T = N / 16;                       // threads per pair
  static constexpr int PASSES = (LOG2N + 3) / 4;
  static constexpr int R0 = N >> (4 * (PASSES - 1));     // radix of the first pass
  static constexpr int CTA = T >= 256 ? T : 256;
  static constexpr int G = CTA / T;                      // pairs in flight per CTA
  static constexpr int BUF = N + N / 16;                 // padded float2 per pair
  // + double-buffered key slots (KEYCAP = 64) + per-warp slot staging
  static constexpr int SMEM = G * BUF * 8 + G * 2 * 64 * 8 + G * (T >= 32 ? T / 32 : 1) * 16 * 4;
};

__host__ __device__ constexpr int pad16(int i) { return i + (i >> 4); }

// Span (product of radices already applied) before pass p.
template <int N>
__host__ __device__ constexpr int span_before(int p) {
  return p == 0 ? 1 : FlatGeo<N>::R0 << (4 * (p - 1));
}
// Offset of pass p's table (p >= 1): entries (q-1)*Ns + k for q = 1..15, k < Ns.
template <int N>
__host__ __device__ constexpr int twiddle_offset(int p) {
  int off = 0;
  for (int i = 1; i < p; i++) off += 15 * span_before<N>(i);
  return off;
}
template <int N>
__host__ __device__ constexpr int twiddle_count() { return twiddle_offset<N>(FlatGeo<N>::PASSES); }

constexpr int KEYCAP = 64;   // bins kept in the double-buffered key slots

// floor(x / bs) for any sign of x (bs > 0), through one float reciprocal and
// an exact integer correction; |x| < 2^22 here, so one step suffices.
__device__ __forceinline__ int bin_of(int x, int bs, float inv_bs) {
  int q = __float2int_rz((float)x * inv_bs);
  const int r = x - q * bs;
  q += (r >= bs) ? 1 : 0;
  q -= (r < 0) ? 1 : 0;
  return q;
}
__device__ __forceinline__ int bin_floor(int x, int bs) {
  return x >= 0 ? x / bs : -((-x + bs - 1) / bs);
}

__device__ __forceinline__ void group_sync(int T) {
  // A pair slot of at most one warp only needs the warp itself in step:
  // every shared-memory region the kernel uses belongs to one slot.
  if (T > 32) __syncthreads(); else __syncwarp();
}

// Synchronise a pair slot, or the whole CTA when the slot's threads are
// spread across warps (the column transforms of the large-n kernels).
template <bool CTA_SYNC>
__device__ __forceinline__ void pass_sync(int T) {
  if constexpr (CTA_SYNC) __syncthreads(); else group_sync(T);
}

// v[q] *= w^q, q = 1..15, for one radix-16 pass: w^1, w^2, w^3, w^4, w^8 and
// w^12 come from the FP64-built table (entry q at tw[(q-1)*stride]), the other
// nine are one product of two of those (w^(4a+b) = w^(4a) w^b), a rounding
// error of about one float ulp beside the table's half ulp.  The packed
// two-pair kernel forms its twiddles with the same operations in the same
// order, so the two kernels give bit-identical outputs.
__device__ __forceinline__ void pass_twiddles(cf *v, const float2 *tw, int stride) {
  auto ld = [&](int q) {
    const float2 w = __ldg(tw + (q - 1) * stride);
    return cf{w.x, w.y};
  };
  const cf w1 = ld(1), w2 = ld(2), w3 = ld(3), w4 = ld(4), w8 = ld(8), w12 = ld(12);
  v[1] = cmul(v[1], w1);
  v[2] = cmul(v[2], w2);
  v[3] = cmul(v[3], w3);
  v[4] = cmul(v[4], w4);
  v[5] = cmul(v[5], cmul(w4, w1));
  v[6] = cmul(v[6], cmul(w4, w2));
  v[7] = cmul(v[7], cmul(w4, w3));
  v[8] = cmul(v[8], w8);
  v[9] = cmul(v[9], cmul(w8, w1));
  v[10] = cmul(v[10], cmul(w8, w2));
  v[11] = cmul(v[11], cmul(w8, w3));
  v[12] = cmul(v[12], w12);
  v[13] = cmul(v[13], cmul(w12, w1));
  v[14] = cmul(v[14], cmul(w12, w2));
  v[15] = cmul(v[15], cmul(w12, w3));
}

// Unnormalised inverse FFT of the n values x[t + T*s] = v[s] held by the T
// threads of one pair slot (Stockham autosort: pass 0 radix R0, then radix
// 16).  On return v[q] = X[t + T*q].  buf is this slot's padded shared buffer;
// the function synchronises the slot before its first store, so buf may
// still be in use by the caller on entry, and it is free again on return.
template <int N, bool CTA_SYNC = false>
__device__ __forceinline__ void inverse_passes(cf *v, float2 *buf, const float2 *twid, int t) {
  using Geo = FlatGeo<N>;
  constexpr int T = Geo::T, R0 = Geo::R0, PASSES = Geo::PASSES;
  constexpr int B0 = 16 / R0;   // butterflies per thread in pass 0
#pragma unroll
  for (int b = 0; b < B0; b++) {
    if constexpr (R0 == 16) dftR<16, 0, 1>(v);
    else if constexpr (R0 == 8) { if (b == 0) dftR<8, 0, 2>(v); else dftR<8, 1, 2>(v); }
    else if constexpr (R0 == 4) {
      if (b == 0) dftR<4, 0, 4>(v); else if (b == 1) dftR<4, 1, 4>(v);
      else if (b == 2) dftR<4, 2, 4>(v); else dftR<4, 3, 4>(v);
    } else {
      switch (b) {   // R0 == 2: slots b and b + 8
        case 0: dft2<0, 8>(v); break; case 1: dft2<1, 8>(v); break;
        case 2: dft2<2, 8>(v); break; case 3: dft2<3, 8>(v); break;
        case 4: dft2<4, 8>(v); break; case 5: dft2<5, 8>(v); break;
        case 6: dft2<6, 8>(v); break; default: dft2<7, 8>(v); break;
      }
    }
  }
  pass_sync<CTA_SYNC>(T);
  // Pass 0 output j*R0 + q (j = t + T*b, q < R0): R0 divides 16, so the
  // 16-block of t*R0 holds every q, and T*R0 is a multiple of 16.
  {
    float2 *p0 = buf + pad16(t * R0);
#pragma unroll
    for (int b = 0; b < B0; b++)
#pragma unroll
      for (int q = 0; q < R0; q++) {
        const cf x = v[b + B0 * q];
        p0[q + b * (T * R0 + T * R0 / 16)] = make_float2(x.x, x.y);
      }
  }
  pass_sync<CTA_SYNC>(T);
#pragma unroll
  for (int p = 1; p < PASSES; p++) {
    const int Ns = span_before<N>(p);
    if constexpr (T % 16 == 0) {
      const float2 *pl = buf + pad16(t);
#pragma unroll
      for (int q = 0; q < 16; q++) {
        const float2 x = pl[q * (T + T / 16)];
        v[q] = {x.x, x.y};
      }
    } else {
#pragma unroll
      for (int q = 0; q < 16; q++) {
        const float2 x = buf[pad16(t + T * q)];
        v[q] = {x.x, x.y};
      }
    }
    const int k = t & (Ns - 1);
    pass_twiddles(v, twid + twiddle_offset<N>(p) + k, Ns);
    dftR<16, 0, 1>(v);
    pass_sync<CTA_SYNC>(T);
    if (p < PASSES - 1) {
      const int base = (t / Ns) * Ns * 16 + k;
      if (Ns % 16 == 0) {
        float2 *ps = buf + pad16(base);
#pragma unroll
        for (int q = 0; q < 16; q++) ps[q * (Ns + Ns / 16)] = make_float2(v[q].x, v[q].y);
      } else {
#pragma unroll
        for (int q = 0; q < 16; q++) buf[pad16(base + q * Ns)] = make_float2(v[q].x, v[q].y);
      }
      pass_sync<CTA_SYNC>(T);
    }
  }
}

// Items [ibeg, iend) of one launch's pairs (item i = pairs i*G .. i*G+G-1 of
// the dense block or the list), processed by one CTA of FlatGeo<N>::CTA
// threads with `smem` its dynamic shared memory.  CACHE_D keeps a data row
// in registers while consecutive pairs share it (long static ranges); without
// it the data spectrum is loaded beside each template (short dynamic ranges,
// 32 registers fewer).  Used by the batched kernel (ranges handed out at run
// time); synchronises the CTA on entry, so smem may still be in use then.
template <int N, int MODE, bool CACHE_D = true>
__device__ __forceinline__ void flat_range(const FlatArgs &a, long long ibeg, long long iend,
                                           float2 *smem) {
  using Geo = FlatGeo<N>;
  constexpr int T = Geo::T, G = Geo::G;
  const int g = threadIdx.x / T;          // pair slot inside the CTA
  const int t = threadIdx.x % T;          // thread inside the pair
  float2 *buf = smem + g * Geo::BUF;
  const long long total = a.list ? (long long)(*a.list_count) : (long long)a.nd * a.nt;
  __syncthreads();

  cf dreg[CACHE_D ? 16 : 1];   // the data row, kept while consecutive pairs share it
  int cur_d = -1;
  const int lane = threadIdx.x & 31;

  // Bin bookkeeping, once per launch.
  const int W = a.we - a.ws;
  const int bs = (MODE == MODE_GATE) ? W : a.binsize;
  const float inv_bs = 1.0f / (float)bs;
  const int Tdiv = T / bs, Tmod = T - Tdiv * bs;
  const unsigned gmask = (T >= 32) ? 0xffffffffu : (((1u << T) - 1u) << (lane & ~(T - 1)));
  const int wlo = (T >= 32) ? (t & ~31) : 0;   // first thread of this warp (or pair slot)
  const int wn = (T >= 32) ? 32 : T;           // threads sharing one redux
  const int gbase = (T >= 32) ? 0 : (lane & ~(T - 1));   // first lane of this redux group
  const unsigned linv = 31u - (unsigned)lane;
  int b_lo0 = bin_floor(wlo - a.ws, bs), r_lo0 = (wlo - a.ws) - b_lo0 * bs;
  // Per-thread slot masks, fixed for the launch: slot q in the window, and
  // slot q's warp-wide lag range inside the window and inside one bin.
  unsigned inmask = 0u, unimask = 0u;
  {
    int blo = b_lo0, rlo = r_lo0;
    for (int q = 0; q < 16; q++) {
      const int x = t + T * q - a.ws, xlo = wlo + T * q - a.ws;
      if (x >= 0 && x < W) inmask |= 1u << q;
      if (xlo >= 0 && xlo + wn - 1 < W && rlo + wn - 1 < bs) unimask |= 1u << q;
      blo += Tdiv;
      rlo += Tmod;
      if (rlo >= bs) { rlo -= bs; blo++; }
    }
  }
  const int nbins = (MODE == MODE_GATE) ? 1 : a.nb;
  const bool small_keys = nbins <= KEYCAP;
  unsigned long long *kslots = reinterpret_cast<unsigned long long *>(smem + G * Geo::BUF);
  // Per-warp staging of the 16 slot winners (fast layout only).
  unsigned *stage = reinterpret_cast<unsigned *>(kslots + G * 2 * KEYCAP) + g * (T >= 32 ? T / 32 : 1) * 16;
  // Fast layout: T >= 32, window = [0, n), bins a multiple of 32 lags, few bins.
  const bool fast = T >= 32 && a.ws == 0 && a.we == N && (bs & 31) == 0 &&
                    nbins <= KEYCAP;
  float2 *const pl_park = buf + pad16(t);   // z[t + T*q] parks at pl_park[q*(T + T/16)]
  if (small_keys) {
    for (int b = t; b < 2 * KEYCAP; b += T) kslots[g * 2 * KEYCAP + b] = 0ull;
  }

  for (long long item = ibeg; item < iend; ++item) {
    const long long pi = item * G + g;
    const bool live = pi < total;
    int row = 0, d = 0, tt = 0;
    if (live) {
      row = a.list ? a.list[pi] : (int)pi;
      d = row / a.nt;
      tt = row - d * a.nt;
    }
    // ---- pass 0: load, conjugate product, radix-R0 butterflies ----------
    cf v[16];
    if (live) {
      const float2 *hp = a.tmpl + (long long)(a.t0 + tt) * a.tmpl_stride;
      const float2 *dp = a.data + (long long)(a.d0 + d) * a.data_stride;
      if constexpr (CACHE_D) {
        if (d != cur_d) {
          if (a.data_cg) {   // data written earlier in the same launch
#pragma unroll
            for (int s = 0; s < 16; s++) {
              float2 x = __ldcg(dp + t + T * s);
              dreg[s] = {x.x, x.y};
            }
          } else {
#pragma unroll
            for (int s = 0; s < 16; s++) {
              float2 x = __ldg(dp + t + T * s);
              dreg[s] = {x.x, x.y};
            }
          }
          cur_d = d;
        }
#pragma unroll
        for (int s = 0; s < 16; s++) {
          float2 h = __ldg(hp + t + T * s);
          // D * conj(H)
          v[s].x = fmaf(dreg[s].x, h.x, dreg[s].y * h.y);
          v[s].y = fmaf(dreg[s].y, h.x, -dreg[s].x * h.y);
        }
      } else {
#pragma unroll
        for (int s = 0; s < 16; s++) {
          const float2 x = a.data_cg ? __ldcg(dp + t + T * s) : __ldg(dp + t + T * s);
          const float2 h = __ldg(hp + t + T * s);
          v[s].x = fmaf(x.x, h.x, x.y * h.y);
          v[s].y = fmaf(x.y, h.x, -x.x * h.y);
        }
      }
    } else {
#pragma unroll
      for (int s = 0; s < 16; s++) v[s] = {0.f, 0.f};
    }
    inverse_passes<N>(v, buf, a.twid, t);
    // Thread t now holds z[t + T*q] in v[q].
    // Keys: a double-buffered slot array when the bins fit, else buf itself.
    const int nb = (MODE == MODE_GATE) ? 1 : a.nb;
    unsigned long long *keys;
    if (small_keys) {
      keys = kslots + ((g * 2 + (int)(item & 1)) * KEYCAP);
    } else {
      keys = reinterpret_cast<unsigned long long *>(buf);
      for (int b = t; b < nb; b += T) keys[b] = 0ull;
      group_sync(T);
    }
    // ---- per-bin argmax ------------------------------------------------------
    // Keys are |z|^2 bit patterns with the low 5 mantissa bits replaced by
    // (31 - lane): ordering is by |z|^2 to within 2^-18 relative, and among
    // values that close the lower lag wins.  The same truncation is used for
    // every comparison, across warps too, so the result is deterministic.
    unsigned cand = 0u;
    if (fast) {
      // Whole window, bins a multiple of 32 lags: every warp slot is one bin.
      if (live) {
        unsigned mxs[16];
#pragma unroll
        for (int q = 0; q < 16; q++) {
          const float m2 = fmaf(v[q].x, v[q].x, v[q].y * v[q].y);
          const unsigned key = (m2 > a.t2) ? ((__float_as_uint(m2) & ~31u) | linv) : 0u;
          const unsigned mx = __reduce_max_sync(0xffffffffu, key);
          mxs[q] = mx;
          if (key != 0u && key == mx) pl_park[q * (T + T / 16)] = make_float2(v[q].x, v[q].y);
        }
        unsigned *st = stage + (t >> 5) * 16;
        if (lane == 0) {
          reinterpret_cast<uint4 *>(st)[0] = make_uint4(mxs[0], mxs[1], mxs[2], mxs[3]);
          reinterpret_cast<uint4 *>(st)[1] = make_uint4(mxs[4], mxs[5], mxs[6], mxs[7]);
          reinterpret_cast<uint4 *>(st)[2] = make_uint4(mxs[8], mxs[9], mxs[10], mxs[11]);
          reinterpret_cast<uint4 *>(st)[3] = make_uint4(mxs[12], mxs[13], mxs[14], mxs[15]);
        }
        __syncwarp();
        if (lane < 16) {
          const unsigned my = st[lane];
          if (my != 0u) {
            const int k = ((t & ~31) | (31 - (int)(my & 31u))) + T * lane;
            const int bin = bin_of((t & ~31) + T * lane, bs, inv_bs);
            atomicMax(keys + bin, ((unsigned long long)(my & ~31u) << 32) | (unsigned)(~k));
          }
        }
      }
    } else if (small_keys) {
      // Fast path: one redux per slot and warp; the winning lane parks z[k]
      // at buf[k] (free after the last pass); 16 lanes then publish the warp's
      // 16 slot winners to the per-bin keys with parallel atomics.
      unsigned mxs[16];
#pragma unroll
      for (int q = 0; q < 16; q++) {
        const int kq = t + T * q;
        const float m2 = fmaf(v[q].x, v[q].x, v[q].y * v[q].y);
        const bool ok = live && ((inmask >> q) & 1u) && m2 > a.t2;
        const unsigned key = ok ? ((__float_as_uint(m2) & ~31u) | linv) : 0u;
        mxs[q] = 0u;
        if ((unimask >> q) & 1u) {
          const unsigned mx = __reduce_max_sync(gmask, key);
          mxs[q] = mx;
          if (key != 0u && key == mx) buf[pad16(kq)] = make_float2(v[q].x, v[q].y);
        } else if (key != 0u) {
          const int bin = bin_of(kq - a.ws, bs, inv_bs);
          atomicMax(keys + bin, ((unsigned long long)(key & ~31u) << 32) | (unsigned)(~kq));
          buf[pad16(kq)] = make_float2(v[q].x, v[q].y);
        }
      }
      for (int j = lane - gbase; j < 16; j += wn) {
        unsigned my = 0u;
#pragma unroll
        for (int q = 0; q < 16; q++) my = (j == q) ? mxs[q] : my;
        if (my != 0u && ((unimask >> j) & 1u)) {
          const int wl = 31 - (int)(my & 31u);                       // winning lane
          const int tw = (T >= 32) ? ((t & ~31) | wl) : (wl & (T - 1));
          const int k = tw + T * j;
          const int bin = bin_of(wlo + T * j - a.ws, bs, inv_bs);
          atomicMax(keys + bin, ((unsigned long long)(my & ~31u) << 32) | (unsigned)(~k));
        }
      }
    } else {
      // Many bins (keys occupy buf): per-lane atomics, winners write back below.
#pragma unroll
      for (int q = 0; q < 16; q++) {
        const int kq = t + T * q;
        const float m2 = fmaf(v[q].x, v[q].x, v[q].y * v[q].y);
        const bool ok = live && ((inmask >> q) & 1u) && m2 > a.t2;
        if (ok) {
          const unsigned key = (__float_as_uint(m2) & ~31u) | linv;
          const int bin = bin_of(kq - a.ws, bs, inv_bs);
          atomicMax(keys + bin, ((unsigned long long)(key & ~31u) << 32) | (unsigned)(~kq));
          cand |= 1u << q;
        }
      }
    }
    group_sync(T);
    if (live) {
      if constexpr (MODE == MODE_PEAKS) {
        const long long obase = (long long)row * nb;
        if (small_keys) {
          int cnt = 0;
          for (int b = t; b < nb; b += T) {
            const unsigned long long kk = keys[b];
            long long ix = -1;
            float2 val = make_float2(0.f, 0.f);
            if (kk != 0ull) {
              const int k = (int)(~(unsigned)kk);
              ix = k;
              val = buf[pad16(k)];
              cnt++;
            }
            a.out_idx[(obase + b) * a.rs] = ix;
            a.out_val[(obase + b) * a.rs] = val;
          }
          if (a.out_cnt) {
            const int c = __reduce_add_sync(gmask, cnt);
            if (c && lane == (T >= 32 ? 0 : (lane & ~(T - 1)))) atomicAdd(a.out_cnt + row, c);
          }
        } else {
          // Many bins: keys live in buf, so the lane holding each winner writes it.
#pragma unroll
          for (int q = 0; q < 16; q++) {
            if (cand & (1u << q)) {
              const int kq = t + T * q;
              const int bin = bin_of(kq - a.ws, bs, inv_bs);
              const unsigned long long kk = keys[bin];
              if ((unsigned)(~(unsigned)kk) == (unsigned)kq) {
                a.out_idx[(obase + bin) * a.rs] = kq;
                a.out_val[(obase + bin) * a.rs] = make_float2(v[q].x, v[q].y);
              }
            }
          }
          int cnt = 0;
          for (int b = t; b < nb; b += T) {
            if (keys[b] == 0ull) {
              a.out_idx[(obase + b) * a.rs] = -1;
              a.out_val[(obase + b) * a.rs] = make_float2(0.f, 0.f);
            } else {
              cnt++;
            }
          }
          if (a.out_cnt) {
            const int c = __reduce_add_sync(gmask, cnt);
            if (c && lane == (T >= 32 ? 0 : (lane & ~(T - 1)))) atomicAdd(a.out_cnt + row, c);
          }
        }
      } else {
        const unsigned long long kk = keys[0];
        const float m2 = __uint_as_float((unsigned)(kk >> 32));
        const bool fire = kk != 0ull && sqrtf(m2) >= a.gate;
        if (a.coarse_out) {
          if (t == 0) a.coarse_out[row] = kk != 0ull ? sqrtf(m2) : 0.f;
        } else if (fire) {
          if (t == 0) a.fire_list[atomicAdd(a.fire_count, 1)] = row;
        } else {
          const long long obase = (long long)row * a.full_nb;
          for (int b = t; b < a.full_nb; b += T) {
            a.out_idx[(obase + b) * a.rs] = -1;
            a.out_val[(obase + b) * a.rs] = make_float2(0.f, 0.f);
          }
        }
      }
    }
    if (small_keys) {
      // Clear the other parity's slots for the next pair; they are not read
      // again before this pair's last barrier has passed.
      unsigned long long *nxt = kslots + ((g * 2 + (int)((item + 1) & 1)) * KEYCAP);
      for (int b = t; b < nb; b += T) nxt[b] = 0ull;
    }
  }
}

// The standalone kernel keeps its own copy of the pair loop instead of
// calling flat_range: written as a call (same code, ranges passed in) it
// measured 6% slower on the B200 (246 vs 232 us for 16 x 1024 pairs at
// n = 4096, CUDA events, L2 flushed), while flat_range's short dynamic ranges
// in the batched kernel need the entry barrier and the coherent-load switch.
template <int N, int MODE>
__global__ void __launch_bounds__(FlatGeo<N>::CTA, FlatGeo<N>::CTA <= 256 ? 2 : 1)
flat_kernel(const FlatArgs a) {
  using Geo = FlatGeo<N>;
  constexpr int T = Geo::T, G = Geo::G;
  extern __shared__ __align__(16) float2 smem[];

  const int g = threadIdx.x / T;          // pair slot inside the CTA
  const int t = threadIdx.x % T;          // thread inside the pair
  float2 *buf = smem + g * Geo::BUF;

  // Work: dense block or a device list of output rows.
  const long long total = a.list ? (long long)(*a.list_count) : (long long)a.nd * a.nt;
  const long long items = (total + G - 1) / G;
  const long long per = items / gridDim.x, extra = items % gridDim.x;
  const long long ibeg = blockIdx.x * per + (blockIdx.x < extra ? blockIdx.x : extra);
  const long long iend = ibeg + per + (blockIdx.x < extra ? 1 : 0);

  cf dreg[16];
  int cur_d = -1;
  const int lane = threadIdx.x & 31;

  // Bin bookkeeping, once per launch.
  const int W = a.we - a.ws;
  const int bs = (MODE == MODE_GATE) ? W : a.binsize;
  const float inv_bs = 1.0f / (float)bs;
  const int Tdiv = T / bs, Tmod = T - Tdiv * bs;
  const unsigned gmask = (T >= 32) ? 0xffffffffu : (((1u << T) - 1u) << (lane & ~(T - 1)));
  const int wlo = (T >= 32) ? (t & ~31) : 0;   // first thread of this warp (or pair slot)
  const int wn = (T >= 32) ? 32 : T;           // threads sharing one redux
  const int gbase = (T >= 32) ? 0 : (lane & ~(T - 1));   // first lane of this redux group
  const unsigned linv = 31u - (unsigned)lane;
  int b_lo0 = bin_floor(wlo - a.ws, bs), r_lo0 = (wlo - a.ws) - b_lo0 * bs;
  // Per-thread slot masks, fixed for the launch: slot q in the window, and
  // slot q's warp-wide lag range inside the window and inside one bin.
  unsigned inmask = 0u, unimask = 0u;
  {
    int blo = b_lo0, rlo = r_lo0;
    for (int q = 0; q < 16; q++) {
      const int x = t + T * q - a.ws, xlo = wlo + T * q - a.ws;
      if (x >= 0 && x < W) inmask |= 1u << q;
      if (xlo >= 0 && xlo + wn - 1 < W && rlo + wn - 1 < bs) unimask |= 1u << q;
      blo += Tdiv;
      rlo += Tmod;
      if (rlo >= bs) { rlo -= bs; blo++; }
    }
  }
  const int nbins = (MODE == MODE_GATE) ? 1 : a.nb;
  const bool small_keys = nbins <= KEYCAP;
  unsigned long long *kslots = reinterpret_cast<unsigned long long *>(smem + G * Geo::BUF);
  // Per-warp staging of the 16 slot winners (fast layout only).
  unsigned *stage = reinterpret_cast<unsigned *>(kslots + G * 2 * KEYCAP) + g * (T >= 32 ? T / 32 : 1) * 16;
  // Fast layout: T >= 32, window = [0, n), bins a multiple of 32 lags, few bins.
  const bool fast = T >= 32 && a.ws == 0 && a.we == N && (bs & 31) == 0 &&
                    nbins <= KEYCAP;
  float2 *const pl_park = buf + pad16(t);   // z[t + T*q] parks at pl_park[q*(T + T/16)]
  if (small_keys) {
    for (int b = t; b < 2 * KEYCAP; b += T) kslots[g * 2 * KEYCAP + b] = 0ull;
  }

  for (long long item = ibeg; item < iend; ++item) {
    const long long pi = item * G + g;
    const bool live = pi < total;
    int row = 0, d = 0, tt = 0;
    if (live) {
      row = a.list ? a.list[pi] : (int)pi;
      d = row / a.nt;
      tt = row - d * a.nt;
    }
    // ---- pass 0: load, conjugate product, radix-R0 butterflies ----------
    cf v[16];
    if (live) {
      if (d != cur_d) {
        const float2 *dp = a.data + (long long)(a.d0 + d) * a.data_stride;
#pragma unroll
        for (int s = 0; s < 16; s++) {
          float2 x = __ldg(dp + t + T * s);
          dreg[s] = {x.x, x.y};
        }
        cur_d = d;
      }
      const float2 *hp = a.tmpl + (long long)(a.t0 + tt) * a.tmpl_stride;
#pragma unroll
      for (int s = 0; s < 16; s++) {
        float2 h = __ldg(hp + t + T * s);
        // D * conj(H)
        v[s].x = fmaf(dreg[s].x, h.x, dreg[s].y * h.y);
        v[s].y = fmaf(dreg[s].y, h.x, -dreg[s].x * h.y);
      }
    } else {
#pragma unroll
      for (int s = 0; s < 16; s++) v[s] = {0.f, 0.f};
    }
    inverse_passes<N>(v, buf, a.twid, t);
    // Thread t now holds z[t + T*q] in v[q].
    // Keys: a double-buffered slot array when the bins fit, else buf itself.
    const int nb = (MODE == MODE_GATE) ? 1 : a.nb;
    unsigned long long *keys;
    if (small_keys) {
      keys = kslots + ((g * 2 + (int)(item & 1)) * KEYCAP);
    } else {
      keys = reinterpret_cast<unsigned long long *>(buf);
      for (int b = t; b < nb; b += T) keys[b] = 0ull;
      group_sync(T);
    }
    // ---- per-bin argmax ------------------------------------------------------
    // Keys are |z|^2 bit patterns with the low 5 mantissa bits replaced by
    // (31 - lane): ordering is by |z|^2 to within 2^-18 relative, and among
    // values that close the lower lag wins.  The same truncation is used for
    // every comparison, across warps too, so the result is deterministic.
    unsigned cand = 0u;
    if (fast) {
      // Whole window, bins a multiple of 32 lags: every warp slot is one bin.
      if (live) {
        unsigned mxs[16];
#pragma unroll
        for (int q = 0; q < 16; q++) {
          const float m2 = fmaf(v[q].x, v[q].x, v[q].y * v[q].y);
          const unsigned key = (m2 > a.t2) ? ((__float_as_uint(m2) & ~31u) | linv) : 0u;
          const unsigned mx = __reduce_max_sync(0xffffffffu, key);
          mxs[q] = mx;
          if (key != 0u && key == mx) pl_park[q * (T + T / 16)] = make_float2(v[q].x, v[q].y);
        }
        unsigned *st = stage + (t >> 5) * 16;
        if (lane == 0) {
          reinterpret_cast<uint4 *>(st)[0] = make_uint4(mxs[0], mxs[1], mxs[2], mxs[3]);
          reinterpret_cast<uint4 *>(st)[1] = make_uint4(mxs[4], mxs[5], mxs[6], mxs[7]);
          reinterpret_cast<uint4 *>(st)[2] = make_uint4(mxs[8], mxs[9], mxs[10], mxs[11]);
          reinterpret_cast<uint4 *>(st)[3] = make_uint4(mxs[12], mxs[13], mxs[14], mxs[15]);
        }
        __syncwarp();
        if (lane < 16) {
          const unsigned my = st[lane];
          if (my != 0u) {
            const int k = ((t & ~31) | (31 - (int)(my & 31u))) + T * lane;
            const int bin = bin_of((t & ~31) + T * lane, bs, inv_bs);
            atomicMax(keys + bin, ((unsigned long long)(my & ~31u) << 32) | (unsigned)(~k));
          }
        }
      }
    } else if (small_keys) {
      // Fast path: one redux per slot and warp; the winning lane parks z[k]
      // at buf[k] (free after the last pass); 16 lanes then publish the warp's
      // 16 slot winners to the per-bin keys with parallel atomics.
      unsigned mxs[16];
#pragma unroll
      for (int q = 0; q < 16; q++) {
        const int kq = t + T * q;
        const float m2 = fmaf(v[q].x, v[q].x, v[q].y * v[q].y);
        const bool ok = live && ((inmask >> q) & 1u) && m2 > a.t2;
        const unsigned key = ok ? ((__float_as_uint(m2) & ~31u) | linv) : 0u;
        mxs[q] = 0u;
        if ((unimask >> q) & 1u) {
          const unsigned mx = __reduce_max_sync(gmask, key);
          mxs[q] = mx;
          if (key != 0u && key == mx) buf[pad16(kq)] = make_float2(v[q].x, v[q].y);
        } else if (key != 0u) {
          const int bin = bin_of(kq - a.ws, bs, inv_bs);
          atomicMax(keys + bin, ((unsigned long long)(key & ~31u) << 32) | (unsigned)(~kq));
          buf[pad16(kq)] = make_float2(v[q].x, v[q].y);
        }
      }
      for (int j = lane - gbase; j < 16; j += wn) {
        unsigned my = 0u;
#pragma unroll
        for (int q = 0; q < 16; q++) my = (j == q) ? mxs[q] : my;
        if (my != 0u && ((unimask >> j) & 1u)) {
          const int wl = 31 - (int)(my & 31u);                       // winning lane
          const int tw = (T >= 32) ? ((t & ~31) | wl) : (wl & (T - 1));
          const int k = tw + T * j;
          const int bin = bin_of(wlo + T * j - a.ws, bs, inv_bs);
          atomicMax(keys + bin, ((unsigned long long)(my & ~31u) << 32) | (unsigned)(~k));
        }
      }
    } else {
      // Many bins (keys occupy buf): per-lane atomics, winners write back below.
#pragma unroll
      for (int q = 0; q < 16; q++) {
        const int kq = t + T * q;
        const float m2 = fmaf(v[q].x, v[q].x, v[q].y * v[q].y);
        const bool ok = live && ((inmask >> q) & 1u) && m2 > a.t2;
        if (ok) {
          const unsigned key = (__float_as_uint(m2) & ~31u) | linv;
          const int bin = bin_of(kq - a.ws, bs, inv_bs);
          atomicMax(keys + bin, ((unsigned long long)(key & ~31u) << 32) | (unsigned)(~kq));
          cand |= 1u << q;
        }
      }
    }
    group_sync(T);
    if (live) {
      if constexpr (MODE == MODE_PEAKS) {
        const long long obase = (long long)row * nb;
        if (small_keys) {
          int cnt = 0;
          for (int b = t; b < nb; b += T) {
            const unsigned long long kk = keys[b];
            long long ix = -1;
            float2 val = make_float2(0.f, 0.f);
            if (kk != 0ull) {
              const int k = (int)(~(unsigned)kk);
              ix = k;
              val = buf[pad16(k)];
              cnt++;
            }
            a.out_idx[(obase + b) * a.rs] = ix;
            a.out_val[(obase + b) * a.rs] = val;
          }
          if (a.out_cnt) {
            const int c = __reduce_add_sync(gmask, cnt);
            if (c && lane == (T >= 32 ? 0 : (lane & ~(T - 1)))) atomicAdd(a.out_cnt + row, c);
          }
        } else {
          // Many bins: keys live in buf, so the lane holding each winner writes it.
#pragma unroll
          for (int q = 0; q < 16; q++) {
            if (cand & (1u << q)) {
              const int kq = t + T * q;
              const int bin = bin_of(kq - a.ws, bs, inv_bs);
              const unsigned long long kk = keys[bin];
              if ((unsigned)(~(unsigned)kk) == (unsigned)kq) {
                a.out_idx[(obase + bin) * a.rs] = kq;
                a.out_val[(obase + bin) * a.rs] = make_float2(v[q].x, v[q].y);
              }
            }
          }
          int cnt = 0;
          for (int b = t; b < nb; b += T) {
            if (keys[b] == 0ull) {
              a.out_idx[(obase + b) * a.rs] = -1;
              a.out_val[(obase + b) * a.rs] = make_float2(0.f, 0.f);
            } else {
              cnt++;
            }
          }
          if (a.out_cnt) {
            const int c = __reduce_add_sync(gmask, cnt);
            if (c && lane == (T >= 32 ? 0 : (lane & ~(T - 1)))) atomicAdd(a.out_cnt + row, c);
          }
        }
      } else {
        const unsigned long long kk = keys[0];
        const float m2 = __uint_as_float((unsigned)(kk >> 32));
        const bool fire = kk != 0ull && sqrtf(m2) >= a.gate;
        if (a.coarse_out) {
          if (t == 0) a.coarse_out[row] = kk != 0ull ? sqrtf(m2) : 0.f;
        } else if (fire) {
          if (t == 0) a.fire_list[atomicAdd(a.fire_count, 1)] = row;
        } else {
          const long long obase = (long long)row * a.full_nb;
          for (int b = t; b < a.full_nb; b += T) {
            a.out_idx[(obase + b) * a.rs] = -1;
            a.out_val[(obase + b) * a.rs] = make_float2(0.f, 0.f);
          }
        }
      }
    }
    if (small_keys) {
      // Clear the other parity's slots for the next pair; they are not read
      // again before this pair's last barrier has passed.
      unsigned long long *nxt = kslots + ((g * 2 + (int)((item + 1) & 1)) * KEYCAP);
      for (int b = t; b < nb; b += T) nxt[b] = 0ull;
    }
  }
}

// Listed mode on its own: the output rows of a device row list (the
// hierarchical refine, mfb_run_rows).  Survivor lists are short and in
// arbitrary order, so the run is latency bound (a few pairs per CTA, each
// loading its own data row): without the data-row cache the kernel fits in
// 80 registers and three 256-thread CTAs per SM, 444 pairs in flight instead
// of 296 on 148 SMs.
template <int N>
__global__ void __launch_bounds__(FlatGeo<N>::CTA, FlatGeo<N>::CTA <= 256 ? 3 : 1)
rows_kernel(const FlatArgs a) {
  using Geo = FlatGeo<N>;
  extern __shared__ __align__(16) float2 smem[];
  const long long total = *a.list_count;
  if (a.trig_total && blockIdx.x == 0 && threadIdx.x == 0) *a.trig_total += (unsigned long long)total;
  const long long items = (total + Geo::G - 1) / Geo::G;
  const long long per = items / gridDim.x, extra = items % gridDim.x;
  const long long ibeg = blockIdx.x * per + (blockIdx.x < extra ? blockIdx.x : extra);
  const long long iend = ibeg + per + (blockIdx.x < extra ? 1 : 0);
  flat_range<N, MODE_PEAKS, false>(a, ibeg, iend, smem);
}

}  // namespace mfb
