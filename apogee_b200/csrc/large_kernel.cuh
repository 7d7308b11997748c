// Fused matched filter for transforms larger than one CTA holds
// (n = 32768 ... 1048576): a two-pass four-step through an L2-sized scratch.
//
// With n = N1 * N2, f = f1 + N1 f2 and k = N2 k1 + k2 (f1, k1 < N1; f2, k2 < N2):
//
//   z[N2 k1 + k2] = sum_f1 W_N1^(f1 k1) [ W_n^(f1 k2) sum_f2 P[f1 + N1 f2] W_N2^(f2 k2) ]
//
//   pass A  per (pair, column f1): conjugate product P = D conj(H) gathered along
//           f2, N2-point inverse FFT, twiddle W_n^(f1 k2), store Y[k2][f1];
//           16 adjacent columns per CTA so every load and store is coalesced.
//   pass B  per (pair, row k2): N1-point inverse FFT of Y[k2][.], giving the lags
//           N2 k1 + k2; per-bin argmax: shared-memory atomicMax inside the CTA on
//           (|z|^2 bits << 32 | ~lag), then one 128-bit atomic compare-and-swap per
//           (CTA, bin) that carries the winner's value with its key, so the
//           correlation series is never written.
//   finalize  candidate records -> (index, value) outputs and crossing counts.
//
// Pairs run in batches whose scratch (batch x n x 8 bytes, <= 64 MiB) stays
// resident in the 126 MB L2; pairs are ordered template-major so the data rows
// of one template share its spectrum in L2.  This is the unshipped "Tier C"
// two-dispatch four-step of the reference (src/gpu/tierb.slang:1043-1150) and
// the CPU plan of src/balanced-inl.h:174-386 for n up to 2^20, fused with the
// product and the argmax as the single-CTA kernel is.
#pragma once
#include "flat_kernel.cuh"

namespace mfb {

constexpr int LARGE_MAX_BINS = 4096;
constexpr int LARGE_SMALL_BINS = 512;   // pass-B launches with this many key slots or fewer
constexpr int LARGE_COLS = 16;          // columns per pass-A CTA

// Shared-memory stride between the column buffers of a pass-A CTA: one float2
// more than a column needs, so that the same offset in consecutive columns
// (what the threads of a half-warp touch together) falls in distinct banks.
template <int N2>
__host__ __device__ constexpr int col_buf() { return FlatGeo<N2>::BUF + 1; }

struct LargeArgs {
  const float2 *data, *tmpl;            // rows of n complex64
  int n, N1, N2;
  int d0, nd, t0, nt;                   // pair block; output row = (d-d0)*nt + (t-t0)
  const int32_t *list;                  // listed output rows, or nullptr (dense block)
  const int32_t *list_count;            // cluster kernel: the list's length on the device
  long long total;                      // pairs in the dense block or the list
  long long pair0;                      // first pair of this batch
  int batch;                            // pairs in this batch
  float2 *Y;                            // scratch [batch][N2][N1]
  uint4 *rec;                           // [batch][nb] records {re, im, ~lag, |z|^2 bits}
  const float2 *tw1, *tw2;              // inverse-pass twiddles of the N1- and N2-point FFTs
  const float2 *tw_hi, *tw_lo;          // W_n^m = tw_hi[m >> lo_bits] * tw_lo[m & lo_mask]
  int lo_bits;
  int ws, we, binsize, nb;
  int seg;                              // pass B: threads per bin segment (bin_lanes), 0: per point
  float t2;
  long long *out_idx;
  float2 *out_val;
  int rs;
  int32_t *out_cnt;
};

// Output row and (d, t) of the pair with index pi (dense: template-major).
__device__ __forceinline__ void large_pair(const LargeArgs &a, long long pi, int &row, int &d,
                                           int &t) {
  if (a.list) {
    row = a.list[pi];
    d = row / a.nt;
    t = row - d * a.nt;
  } else {
    t = (int)(pi / a.nd);
    d = (int)(pi - (long long)t * a.nd);
    row = d * a.nt + t;
  }
}

// W_n^m from the two-level table (FP64-built halves, one product).
__device__ __forceinline__ cf wn_table(const LargeArgs &a, unsigned m) {
  const float2 wh = __ldg(a.tw_hi + (m >> a.lo_bits));
  const float2 wl = __ldg(a.tw_lo + (m & ((1u << a.lo_bits) - 1u)));
  return cmul(cf{wh.x, wh.y}, cf{wl.x, wl.y});
}

// Pass A's twiddle: v[q] *= W_n^(f1 k2), k2 = t + T2 q.  The factor comes
// from the table at q = 0, 4, 8, 12 and from up to three steps of
// W_n^(f1 T2) in between (10 table reads instead of 32; the three products
// add at most a few float ulps).
template <int T2>
__device__ __forceinline__ void pass_a_twiddle(cf *v, const LargeArgs &a, int f1, int t) {
  const unsigned nm = (unsigned)(a.n - 1);
  const cf step = wn_table(a, ((unsigned)f1 * (unsigned)T2) & nm);
  cf w;
#pragma unroll
  for (int q = 0; q < 16; q++) {
    if ((q & 3) == 0) w = wn_table(a, ((unsigned)f1 * (unsigned)(t + T2 * q)) & nm);
    else w = cmul(w, step);
    v[q] = cmul(v[q], w);
  }
}

template <int N2>
__global__ void __launch_bounds__(N2 >= 256 ? N2 : 256, N2 >= 1024 ? 1 : (N2 >= 512 ? 2 : 3))
large_pass_a(const LargeArgs a) {
  constexpr int T2 = N2 / 16, C = LARGE_COLS;
  static_assert(T2 * C == N2, "pass A runs one thread per (column, point group)");
  extern __shared__ __align__(16) float2 smem[];
  const int c = threadIdx.x % C, t = threadIdx.x / C;
  float2 *buf = smem + c * col_buf<N2>();
  const int tiles = a.N1 / C;
  const long long work = (long long)a.batch * tiles;
  for (long long w = blockIdx.x; w < work; w += gridDim.x) {
    const int bp = (int)(w / tiles), tile = (int)(w - (long long)bp * tiles);
    const long long pi = a.pair0 + bp;
    const int f1 = tile * C + c;
    cf v[16];
    if (pi < a.total) {
      int row, d, tt;
      large_pair(a, pi, row, d, tt);
      const float2 *dp = a.data + (long long)(a.d0 + d) * a.n;
      const float2 *hp = a.tmpl + (long long)(a.t0 + tt) * a.n;
#pragma unroll
      for (int s = 0; s < 16; s++) {
        const long long f = f1 + (long long)a.N1 * (t + T2 * s);
        const float2 x = __ldg(dp + f), h = __ldg(hp + f);
        v[s].x = fmaf(x.x, h.x, x.y * h.y);
        v[s].y = fmaf(x.y, h.x, -x.x * h.y);
      }
    } else {
#pragma unroll
      for (int s = 0; s < 16; s++) v[s] = {0.f, 0.f};
    }
    inverse_passes<N2, true>(v, buf, a.tw2, t);
    pass_a_twiddle<T2>(v, a, f1, t);
    float2 *yp = a.Y + (long long)bp * a.N2 * a.N1 + f1;
#pragma unroll
    for (int q = 0; q < 16; q++)
      yp[(long long)(t + T2 * q) * a.N1] = make_float2(v[q].x, v[q].y);
  }
}

// 128-bit max on the high 64 bits (the key); the low 64 bits (value) travel
// with it.  Keys only grow, so a key already >= ours settles it with one plain
// (single-copy atomic, 64-bit) read; otherwise compare-and-swap from the key
// and value read separately -- if they were inconsistent the first swap fails
// and returns the true record.
__device__ __forceinline__ void rec_max(uint4 *slot, uint4 mine) {
  const unsigned long long mkey = ((unsigned long long)mine.w << 32) | mine.z;
  const unsigned long long *q = reinterpret_cast<const unsigned long long *>(slot);
  const unsigned long long k0 = __ldcg(q + 1);
  if (k0 >= mkey) return;
  unsigned __int128 *p = reinterpret_cast<unsigned __int128 *>(slot);
  const unsigned __int128 m = ((unsigned __int128)mkey << 64) |
                              (((unsigned long long)mine.y << 32) | mine.x);
  unsigned __int128 old = ((unsigned __int128)k0 << 64) | __ldcg(q);
  for (;;) {
    const unsigned __int128 prev = atomicCAS(p, old, m);
    if (prev == old) break;
    old = prev;
    if ((unsigned long long)(old >> 64) >= mkey) break;
  }
}

// Pass-B keys: (|z|^2 bits with the low 5 mantissa bits cleared) << 32 | ~lag,
// so a bin keeps its largest |z|^2 to within 2^-18 relative and, among values
// that close, the lowest lag -- the order the single-CTA kernels use.
//
// Lanes of a warp that share a bin: a warp holds 32 / T1 rows k2 (T1 < 32) or
// 32 threads of one row, thread t at k1 = t + T1 q.  With binsize = m N2 (m a
// power of two) and the window starting on a multiple of binsize, lag
// N2 k1 + k2 (k2 < N2) falls in bin floor(k1 / m) less a constant, so the
// lanes sharing a bin are the aligned blocks of min(m, T1, 32) threads t of
// every row in the warp.  Returns that block size when it spans the warp
// (every lane of a warp then shares one bin), else 0.
__host__ __device__ inline int bin_lanes(int binsize, int ws, int N1, int N2) {
  if (binsize % N2 != 0 || ws % binsize != 0) return 0;
  const int m = binsize / N2;
  if ((m & (m - 1)) != 0) return 0;
  const int T1 = N1 / 16, cap = T1 < 32 ? T1 : 32;
  return m >= cap ? cap : 0;   // whole-warp segments only: several per warp measured slower
}

// Per-thread constants of pass_b_key for T1 threads per row and seg > 0:
// the lanes of this lane's bin segment, and its rank among them in lag order
// (t first, then the row).
__device__ __forceinline__ void bin_segment(int T1, int seg, unsigned &mask, unsigned &rank) {
  const int lane = threadIdx.x & 31;
  if (T1 >= 32) {
    mask = seg >= 32 ? 0xffffffffu : ((1u << seg) - 1u) << (lane & ~(seg - 1));
    rank = (unsigned)lane;
  } else {
    const int rows = 32 / T1, t = lane % T1, row = lane / T1;
    const unsigned block = ((1u << seg) - 1u) << (t & ~(seg - 1));
    mask = 0u;
    for (int r = 0; r < rows; r++) mask |= block << (r * T1);
    rank = (unsigned)(t * rows + row);
  }
}

// One step of pass B: this thread's z = v at `lag` (a candidate when `cand`).
// With seg > 0 the warp first reduces each bin segment (one redux; the winner,
// unique by rank, parks its value and publishes the segment's key); otherwise
// every candidate parks and publishes.  `park` is where the value goes.
__device__ __forceinline__ void pass_b_key(unsigned long long *keys, float2 *park, cf v, float m2,
                                           int lag, bool cand, int seg, unsigned mask,
                                           unsigned rank, int ws, int bs, float inv_bs) {
  const unsigned mt = __float_as_uint(m2) & ~31u;
  if (seg > 0) {
    if (!__any_sync(mask, cand)) return;   // the usual case above a threshold
    const unsigned k32 = cand ? (mt | (31u - rank)) : 0u;
    const unsigned mx = __reduce_max_sync(mask, k32);
    if (k32 != 0u && k32 == mx) {
      *park = make_float2(v.x, v.y);
      atomicMax(keys + bin_of(lag - ws, bs, inv_bs), ((unsigned long long)mt << 32) | (unsigned)(~lag));
    }
  } else if (cand) {
    *park = make_float2(v.x, v.y);
    atomicMax(keys + bin_of(lag - ws, bs, inv_bs), ((unsigned long long)mt << 32) | (unsigned)(~lag));
  }
}

template <int N1>
__global__ void __launch_bounds__(FlatGeo<N1>::CTA, 4)   // 64 registers: four CTAs per SM
large_pass_b(const LargeArgs a) {
  using Geo = FlatGeo<N1>;
  constexpr int T1 = Geo::T, G = Geo::G;
  extern __shared__ __align__(16) float2 smem[];
  const int g = threadIdx.x / T1, t = threadIdx.x % T1;
  float2 *buf = smem + g * Geo::BUF;
  unsigned long long *keys = reinterpret_cast<unsigned long long *>(smem + G * Geo::BUF);
  const int bs = a.binsize;
  const float inv_bs = 1.0f / (float)bs;
  unsigned smask = 0u, srank = 0u;
  if (a.seg > 0) bin_segment(T1, a.seg, smask, srank);
  const long long work = (long long)a.batch * a.N2 / G;
  for (long long w = blockIdx.x; w < work; w += gridDim.x) {
    const long long r0 = w * G;                       // first row of this CTA
    const int bp = (int)(r0 / a.N2), k2base = (int)(r0 - (long long)bp * a.N2);
    const int k2 = k2base + g;
    const bool live = a.pair0 + bp < a.total;
    cf v[16];
    const float2 *yp = a.Y + ((long long)bp * a.N2 + k2) * a.N1;
#pragma unroll
    for (int s = 0; s < 16; s++) {
      const float2 x = yp[t + T1 * s];
      v[s] = {x.x, x.y};
    }
    for (int b = threadIdx.x; b < a.nb; b += blockDim.x) keys[b] = 0ull;
    __syncthreads();
    inverse_passes<N1>(v, buf, a.tw1, t);
    // thread t holds z[N2 k1 + k2] for k1 = t + T1 q
#pragma unroll
    for (int q = 0; q < 16; q++) {
      const int k1 = t + T1 * q;
      const int lag = a.N2 * k1 + k2;
      const float m2 = fmaf(v[q].x, v[q].x, v[q].y * v[q].y);
      pass_b_key(keys, buf + pad16(k1), v[q], m2, lag,
                 live && lag >= a.ws && lag < a.we && m2 > a.t2, a.seg, smask, srank, a.ws, bs,
                 inv_bs);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < a.nb; b += blockDim.x) {
      const unsigned long long kk = keys[b];
      if (kk == 0ull) continue;
      const int lag = (int)(~(unsigned)kk);
      const int gw = (lag % a.N2) - k2base, k1w = lag / a.N2;
      const float2 val = smem[gw * Geo::BUF + pad16(k1w)];
      rec_max(a.rec + (long long)bp * a.nb + b,
              make_uint4(__float_as_uint(val.x), __float_as_uint(val.y), (unsigned)kk,
                         (unsigned)(kk >> 32)));
    }
    __syncthreads();
  }
}

// Forward transforms of series blocks for n > 16384 (run_series): the same
// two passes over block b = pair0 + bp of the series, conjugated and scaled by
// 1/n on the way in (FFT(x) = conj(IFFT(conj(x)))), written back conjugated
// in natural order: spectra row b, frequency N2*k1 + k2.
struct LargeFwd {
  const float2 *series;
  long long nseries;
  const unsigned long long *starts;   // [blocks]
  float2 *spectra;                    // [blocks][n]
  float scale;                        // 1/n
};

template <int N2>
__global__ void __launch_bounds__(N2 >= 256 ? N2 : 256)
large_fwd_a(const LargeArgs a, const LargeFwd s) {
  constexpr int T2 = N2 / 16, C = LARGE_COLS;
  extern __shared__ __align__(16) float2 smem[];
  const int c = threadIdx.x % C, t = threadIdx.x / C;
  float2 *buf = smem + c * col_buf<N2>();
  const int tiles = a.N1 / C;
  const long long work = (long long)a.batch * tiles;
  const unsigned lo_mask = (1u << a.lo_bits) - 1u;
  for (long long w = blockIdx.x; w < work; w += gridDim.x) {
    const int bp = (int)(w / tiles), tile = (int)(w - (long long)bp * tiles);
    const long long blk = a.pair0 + bp;
    const int f1 = tile * C + c;
    cf v[16];
    if (blk < a.total) {
      const long long s0 = (long long)s.starts[blk];
#pragma unroll
      for (int q = 0; q < 16; q++) {
        const long long e = s0 + f1 + (long long)a.N1 * (t + T2 * q);
        float2 x = make_float2(0.f, 0.f);
        if (e < s.nseries) x = __ldg(s.series + e);
        v[q] = {x.x * s.scale, -x.y * s.scale};
      }
    } else {
#pragma unroll
      for (int q = 0; q < 16; q++) v[q] = {0.f, 0.f};
    }
    inverse_passes<N2, true>(v, buf, a.tw2, t);
    float2 *yp = a.Y + (long long)bp * a.N2 * a.N1 + f1;
#pragma unroll
    for (int q = 0; q < 16; q++) {
      const int k2 = t + T2 * q;
      const unsigned m = ((unsigned)f1 * (unsigned)k2) & (unsigned)(a.n - 1);
      const float2 wh = __ldg(a.tw_hi + (m >> a.lo_bits)), wl = __ldg(a.tw_lo + (m & lo_mask));
      const cf y = cmul(v[q], cmul(cf{wh.x, wh.y}, cf{wl.x, wl.y}));
      yp[(long long)k2 * a.N1] = make_float2(y.x, y.y);
    }
  }
}

template <int N1>
__global__ void __launch_bounds__(FlatGeo<N1>::CTA)
large_fwd_b(const LargeArgs a, const LargeFwd s) {
  using Geo = FlatGeo<N1>;
  constexpr int T1 = Geo::T, G = Geo::G;
  extern __shared__ __align__(16) float2 smem[];
  const int g = threadIdx.x / T1, t = threadIdx.x % T1;
  float2 *buf = smem + g * Geo::BUF;
  const long long work = (long long)a.batch * a.N2 / G;
  for (long long w = blockIdx.x; w < work; w += gridDim.x) {
    const long long r0 = w * G;
    const int bp = (int)(r0 / a.N2), k2 = (int)(r0 - (long long)bp * a.N2) + g;
    const long long blk = a.pair0 + bp;
    const float2 *yp = a.Y + ((long long)bp * a.N2 + k2) * a.N1;
    cf v[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
      const float2 x = yp[t + T1 * q];
      v[q] = {x.x, x.y};
    }
    inverse_passes<N1>(v, buf, a.tw1, t);
    if (blk < a.total) {
      float2 *o = s.spectra + blk * a.n + k2;
#pragma unroll
      for (int q = 0; q < 16; q++)
        o[(long long)a.N2 * (t + T1 * q)] = make_float2(v[q].x, -v[q].y);
    }
  }
}

__global__ void large_finalize(const LargeArgs a) {
  const long long n_out = (long long)a.batch * a.nb;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_out;
       i += (long long)gridDim.x * blockDim.x) {
    const int bp = (int)(i / a.nb), b = (int)(i - (long long)bp * a.nb);
    const long long pi = a.pair0 + bp;
    if (pi >= a.total) continue;
    int row, d, t;
    large_pair(a, pi, row, d, t);
    const uint4 r = a.rec[i];
    const long long o = ((long long)row * a.nb + b) * a.rs;
    if (r.w == 0u && r.z == 0u) {
      a.out_idx[o] = -1;
      a.out_val[o] = make_float2(0.f, 0.f);
    } else {
      a.out_idx[o] = (long long)(int)(~r.z);
      a.out_val[o] = make_float2(__uint_as_float(r.x), __uint_as_float(r.y));
      if (a.out_cnt) atomicAdd(a.out_cnt + row, 1);
    }
  }
}

}  // namespace mfb
