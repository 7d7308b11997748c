// Band-16384 coarse pass of the hierarchical filter on the tensor cores, as a
// four-step around the 512-point tensor-core pass (coarse_tc.cu).
//
// The coarse value of a pair is max |z_c[j]| over the coarse window, with
// z_c[j] = sum_{f < m} D[f] conj(ct[f]) exp(+2 pi i f j / m) the m-point
// inverse DFT of the band-limited product (src/hmf.c:241-251, m = band).  For
// m = 16384 = 512 * 32, with f = f1 + 512 f2 and j = 32 k1 + k2 (f1, k1 < 512;
// f2, k2 < 32):
//
//   z_c[32 k1 + k2] = sum_f1 W512^(f1 k1) [ W_m^(f1 k2) sum_f2 P[f1 + 512 f2] W32^(f2 k2) ]
//
//   band_col_kernel   per (pair, column f1): the conjugate product gathered
//                     along f2, the 32-point inverse DFT in FP32 registers,
//                     the twiddle W_m^(f1 k2) (product of two FP64-built
//                     128-entry tables, both resident in L1), stored as
//                     row k2 of the pair's 32 x 512 scratch;
//   tc_coarse_rows    every scratch row through the split-precision 512-point
//                     tensor-core pass, max |z|^2 per row over the lags of
//                     the window that row holds;
//   band_gate_kernel  max over the pair's 32 rows and the gate of
//                     src/hmf.c:264-300 (fire -> refine list; dismissed ->
//                     its full-size output rows (-1, 0)), or the coarse value.
#pragma once
#include <cstdint>
#include "fft_radix.cuh"

namespace mfb {

constexpr int BAND_BIG = 16384;      // the band this four-step covers
constexpr int BAND_COLS = 512;       // the tensor-core DFT length (columns f1)
constexpr int BAND_ROWS = 32;        // rows k2 per pair

struct BandColArgs {
  const float2 *data;        // full-length data rows, stride data_stride; first 16384 bins used
  long long data_stride;
  const float2 *ct;          // coarse templates [nt_total][16384]
  int d0, nd, t0, nt;        // pair block (dense, row = d * nt + t)
  long long pair0;           // first pair of this batch
  int batch;                 // pairs in this batch
  const float2 *w32;         // W32^k, k = 0..15
  const float2 *wm;          // W_16384^m = wm[128 + (m >> 7)] * wm[m & 127] (two 128-entry tables)
  float2 *Y;                 // scratch [batch][32][512]
};

// 256 threads = 256 columns of one pair; two CTAs per pair.
static __global__ void __launch_bounds__(256)
band_col_kernel(const BandColArgs a) {
  const long long work = (long long)a.batch * 2;
  const long long total = (long long)a.nd * a.nt;
  for (long long w = blockIdx.x; w < work; w += gridDim.x) {
    const int bp = (int)(w >> 1);
    const long long pi = a.pair0 + bp;
    const int f1 = (int)(w & 1) * 256 + threadIdx.x;
    cf e[16], o[16];
    if (pi < total) {
      const int d = (int)(pi / a.nt), t = (int)(pi - (long long)d * a.nt);
      const float2 *dp = a.data + (long long)(a.d0 + d) * a.data_stride + f1;
      const float2 *hp = a.ct + (long long)(a.t0 + t) * BAND_BIG + f1;
#pragma unroll
      for (int m = 0; m < 16; m++) {
        const float2 x0 = __ldg(dp + BAND_COLS * (2 * m)), h0 = __ldg(hp + BAND_COLS * (2 * m));
        const float2 x1 = __ldg(dp + BAND_COLS * (2 * m + 1)), h1 = __ldg(hp + BAND_COLS * (2 * m + 1));
        e[m] = {fmaf(x0.x, h0.x, x0.y * h0.y), fmaf(x0.y, h0.x, -x0.x * h0.y)};
        o[m] = {fmaf(x1.x, h1.x, x1.y * h1.y), fmaf(x1.y, h1.x, -x1.x * h1.y)};
      }
    } else {
#pragma unroll
      for (int m = 0; m < 16; m++) { e[m] = {0.f, 0.f}; o[m] = {0.f, 0.f}; }
    }
    // 32-point inverse DFT: X[k] = E[k] + W32^k O[k], X[k + 16] = E[k] - W32^k O[k]
    dft16(e);
    dft16(o);
    float2 *yp = a.Y + (long long)bp * BAND_ROWS * BAND_COLS + f1;
#pragma unroll
    for (int k = 0; k < 16; k++) {
      const float2 w = __ldg(a.w32 + k);
      const cf wo = cmul(o[k], cf{w.x, w.y});
      const cf lo = cadd(e[k], wo), hi = csub(e[k], wo);
      const unsigned m_lo = ((unsigned)f1 * (unsigned)k) & (BAND_BIG - 1);
      const unsigned m_hi = ((unsigned)f1 * (unsigned)(k + 16)) & (BAND_BIG - 1);
      const float2 al = __ldg(a.wm + 128 + (m_lo >> 7)), bl = __ldg(a.wm + (m_lo & 127));
      const float2 ah = __ldg(a.wm + 128 + (m_hi >> 7)), bh = __ldg(a.wm + (m_hi & 127));
      const cf tl = cmul(cf{al.x, al.y}, cf{bl.x, bl.y}), th = cmul(cf{ah.x, ah.y}, cf{bh.x, bh.y});
      const cf yl = cmul(lo, tl), yh = cmul(hi, th);
      yp[(long long)k * BAND_COLS] = make_float2(yl.x, yl.y);
      yp[(long long)(k + 16) * BAND_COLS] = make_float2(yh.x, yh.y);
    }
  }
}

struct BandGateArgs {
  const float *m2;           // [batch][32] row maxima of |z|^2
  long long pair0;
  int batch;
  int nt;                    // templates of the block: output row = pair index (d * nt + t)
  long long total;           // pairs of the block
  float t2, gate;
  long long *out_idx;        // full-size outputs: rows of dismissed pairs get (-1, 0)
  float2 *out_val;
  int rs, full_nb;
  int32_t *fire_list, *fire_count;
  float *coarse_out;         // if set: sqrt of the pair's maximum instead of gating
};

// One warp per pair: lane k2 holds row k2's maximum.
static __global__ void __launch_bounds__(256)
band_gate_kernel(const BandGateArgs a) {
  const int lane = threadIdx.x & 31;
  const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long bp = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
       bp < a.batch; bp += nwarps) {
    const long long pi = a.pair0 + bp;
    if (pi >= a.total) continue;
    // |z|^2 >= 0: the IEEE bit patterns order as unsigned integers
    const unsigned mb = __reduce_max_sync(0xffffffffu, __float_as_uint(a.m2[bp * BAND_ROWS + lane]));
    const float best = __uint_as_float(mb);
    const int row = (int)pi;
    if (a.coarse_out) {
      if (lane == 0) a.coarse_out[row] = sqrtf(best);
      continue;
    }
    const bool fire = best > a.t2 && sqrtf(best) >= a.gate;
    if (fire) {
      if (lane == 0) a.fire_list[atomicAdd(a.fire_count, 1)] = row;
    } else {
      const long long obase = (long long)row * a.full_nb;
      for (int b = lane; b < a.full_nb; b += 32) {
        a.out_idx[(obase + b) * a.rs] = -1;
        a.out_val[(obase + b) * a.rs] = make_float2(0.f, 0.f);
      }
    }
  }
}

}  // namespace mfb
