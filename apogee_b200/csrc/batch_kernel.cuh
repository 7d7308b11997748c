// Many uneven matched-filter jobs in one persistent launch.
//
// A job is one (data, templates, binsize, threshold, window) block of any
// power-of-two n from 64 to 2^20, or a run_series job whose data rows are the
// forward transforms of time-series blocks.  Every CTA (256 threads, two per
// SM, all resident) takes tickets from one atomic counter; a ticket is one
// unit of work inside a segment of a host-built segment table:
//
//   SEG_SMALL      n <= 4096: `unit_items` items of the single-CTA fused
//                  filter (flat_range, G = 4096/n pairs per item).
//   SEG_FWD_SMALL  n <= 4096 series job: G blocks' forward transforms.
//   SEG_A / SEG_B  n >= 8192: the two passes of the four-step split
//                  n = N1 * N2 (N2 in {64, 128, 256}, N1 in [64, 4096]) for
//                  one batch of pairs, through a scratch slot:
//                  A = N2-point column transforms of the conjugate product,
//                  twiddled, into Y[pair][k2][f1]; B = N1-point row
//                  transforms and the per-bin argmax, merged across CTAs
//                  into the job's 16-byte output records with a 128-bit
//                  compare-and-swap; the last B unit of a batch rewrites that
//                  batch's records in PEAK_DTYPE layout.
//   SEG_FA / SEG_FB the same two passes as a forward transform of series
//                  blocks, writing spectra instead of peaks.
//
// Dependencies are counters with bounded waits: B(q) waits for every A(q)
// unit, A(q) waits until the B units of the batch that last used its slot
// (q - nslots) are done, and a series job's pair units wait for its forward
// units.  The host orders segments so that every wait is on units with
// smaller tickets; since all CTAs are resident and tickets are taken in
// order, the unfinished unit with the smallest ticket never waits, so the
// launch always makes progress.  A wait that runs out sets the error word;
// every CTA then stops taking tickets.
//
// The reference runs one plan per shape (src/matchfilt.c:73-147 ap_mf_create
// and ap_mf_run; src/matchfilt.c:437-490 run_series); it has no batched form.
#pragma once
#include <cstdint>
#include "flat_kernel.cuh"
#include "large_kernel.cuh"

namespace mfb {

constexpr int BATCH_CTA = 256;
constexpr int BATCH_MAX_BINS = LARGE_MAX_BINS;
constexpr unsigned BATCH_SPIN_LIMIT = 1u << 22;

enum { SEG_SMALL = 0, SEG_FWD_SMALL = 1, SEG_A = 2, SEG_B = 3, SEG_FA = 4, SEG_FB = 5 };
enum { BATCH_ERR_WAIT = 1 };

struct BatchJob {
  const float2 *data;                 // [nd][n] spectra (a series job: its workspace)
  float2 *spec;                       // series job: workspace written by the forward units
  const float2 *tmpl;                 // [nt][n]
  uint4 *rec;                         // [nd*nt][nb] output records, PEAK_DTYPE layout
  const float2 *twid;                 // n <= 4096: inter-pass table of n
  const float2 *tw1, *tw2;            // n >= 8192: tables of N1 and N2
  const float2 *tw_hi, *tw_lo;        // n >= 8192: W_n^m = hi[m >> lo_bits] * lo[m & mask]
  const float2 *series;               // series job: complex64 samples
  const unsigned long long *starts;   // series job: [nd] block starts
  long long nseries;
  int n, nd, nt, nb, binsize, ws, we;
  float t2;
  int N1, N2, lo_bits;
  int batch_pairs;                    // n >= 8192: pairs (blocks) per scratch batch
  int unit_items;                     // n <= 4096: items per ticket
  int fwd_units;                      // series job: forward units to wait for, else 0
  int fwd_ctr;                        // series job: its counter in fwd_done
  float scale;                        // 1/n
};

struct BatchSeg {
  long long t0;                       // first ticket
  int job, kind;
  int q;                              // global batch (slot user) index, SEG_A/B/FA/FB
  int q_local;                        // batch index inside the job
  int units;                          // tickets
  int pairs;                          // pairs (blocks) in this batch
  int raw;                            // A/B/FA/FB: work units (4096 points each)
  int per;                            // A/B/FA/FB: work units per ticket
};

struct BatchArgs {
  const BatchSeg *segs;
  int nseg;
  long long total;                    // tickets
  unsigned long long *ticket;
  unsigned *a_done, *b_done;          // [nbatches]
  const unsigned *a_total, *b_total;  // [nbatches]
  unsigned *fwd_done;                 // [njobs]
  int *err;
  float2 *slots;
  long long slot_elems;               // float2 per slot
  int nslots;
};

// The launch's arguments and job descriptors live in constant memory: every
// field a unit reads is re-read from the constant cache on demand (as a
// kernel parameter would be) instead of holding registers across the
// transform.  One table per device: a run refreshes it from the plan's
// device copy right before the launch, on the same stream.
constexpr int BATCH_MAX_JOBS = 300;
struct BatchTable {
  BatchArgs args;
  BatchJob jobs[BATCH_MAX_JOBS];
};
__constant__ BatchTable c_batch;

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Wait (thread 0, bounded) until *ctr >= target; false for every thread of
// the CTA if the wait ran out or another CTA reported an error.
__device__ __forceinline__ bool batch_wait(const unsigned *ctr, unsigned target, int *err) {
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    int ok = 1;
    unsigned spins = 0;
    while (ld_acquire(ctr) < target) {
      if (*(volatile int *)err) { ok = 0; break; }
      if (++spins > BATCH_SPIN_LIMIT) {
        atomicCAS(err, 0, BATCH_ERR_WAIT);
        ok = 0;
        break;
      }
      __nanosleep(256);
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Publish this ticket's global writes and count its `count` units; true for
// every thread of the CTA when they were the last of `total` counted on ctr.
__device__ __forceinline__ bool batch_done(unsigned *ctr, unsigned total, unsigned count = 1u) {
  __shared__ int s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(ctr, count) == total - count);
  __syncthreads();
  return s_last != 0;
}

// Pair pi of a two-pass job, template-major so that a batch shares templates.
__device__ __forceinline__ void batch_pair(const BatchJob &j, long long pi, int &row, int &d,
                                           int &t) {
  t = (int)(pi / j.nd);
  d = (int)(pi - (long long)t * j.nd);
  row = d * j.nt + t;
}

template <int N>
__device__ __forceinline__ void small_unit(int jid, int u, float2 *smem) {
  const BatchArgs &a = c_batch.args;
  const BatchJob &j = c_batch.jobs[jid];
  if (j.fwd_units && !batch_wait(a.fwd_done + j.fwd_ctr, (unsigned)j.fwd_units, a.err)) return;
  constexpr int G = FlatGeo<N>::G;
  FlatArgs f = {};
  f.data = j.data;
  f.tmpl = j.tmpl;
  f.data_stride = N;
  f.tmpl_stride = N;
  f.twid = j.twid;
  f.nd = j.nd;
  f.nt = j.nt;
  f.ws = j.ws;
  f.we = j.we;
  f.binsize = j.binsize;
  f.nb = j.nb;
  f.t2 = j.t2;
  f.out_idx = reinterpret_cast<long long *>(j.rec);
  f.out_val = reinterpret_cast<float2 *>(reinterpret_cast<char *>(j.rec) + 8);
  f.rs = 2;
  f.data_cg = j.fwd_units != 0;
  const long long items = ((long long)j.nd * j.nt + G - 1) / G;
  const long long ibeg = (long long)u * j.unit_items;
  const long long iend = min(items, ibeg + j.unit_items);
  flat_range<N, MODE_PEAKS, false>(f, ibeg, iend, smem);
}

template <int N>
__device__ __noinline__ void fwd_small_unit(int jid, int u, float2 *smem) {
  const BatchArgs &a = c_batch.args;
  const BatchJob &j = c_batch.jobs[jid];
  using Geo = FlatGeo<N>;
  constexpr int T = Geo::T, G = Geo::G;
  const int g = threadIdx.x / T, t = threadIdx.x % T;
  float2 *buf = smem + g * Geo::BUF;
  const int b = u * G + g;
  const bool live = b < j.nd;
  cf v[16];
  if (live) {
    const long long s0 = (long long)j.starts[b];
#pragma unroll
    for (int s = 0; s < 16; s++) {
      const long long e = s0 + t + T * s;
      float2 x = make_float2(0.f, 0.f);
      if (e < j.nseries) x = __ldg(j.series + e);
      v[s] = {x.x * j.scale, -x.y * j.scale};
    }
  } else {
#pragma unroll
    for (int s = 0; s < 16; s++) v[s] = {0.f, 0.f};
  }
  __syncthreads();   // the previous unit's readers of smem are done
  inverse_passes<N>(v, buf, j.twid, t);
  if (live) {
    float2 *o = j.spec + (long long)b * N;
#pragma unroll
    for (int q = 0; q < 16; q++) o[t + T * q] = make_float2(v[q].x, -v[q].y);
  }
  batch_done(a.fwd_done + j.fwd_ctr, (unsigned)j.fwd_units);
}

// Column pass: C = 4096/N2 adjacent columns f1 of one pair (or block), the
// N2-point inverse transform of column f1 over f2, times W_n^(f1 k2).
template <int N2, bool FWD>
__device__ __noinline__ void a_unit(int jid, int segi, int u, float2 *smem) {
  const BatchArgs &a = c_batch.args;
  const BatchJob &j = c_batch.jobs[jid];
  const BatchSeg sg = a.segs[segi];
  constexpr int T2 = N2 / 16, C = BATCH_CTA / T2;
  if (sg.q >= a.nslots &&
      !batch_wait(a.b_done + (sg.q - a.nslots), a.b_total[sg.q - a.nslots], a.err))
    return;
  if (!FWD && j.fwd_units && !batch_wait(a.fwd_done + j.fwd_ctr, (unsigned)j.fwd_units, a.err))
    return;
  const int c = threadIdx.x % C, t = threadIdx.x / C;
  float2 *buf = smem + c * col_buf<N2>();
  const int tiles = j.N1 / C;
  const int w0 = u * sg.per, w1 = min(sg.raw, w0 + sg.per);
  for (int w = w0; w < w1; w++) {
  const int bp = w / tiles, tile = w - bp * tiles;
  const long long pi = (long long)sg.q_local * j.batch_pairs + bp;
  const int f1 = tile * C + c;
  cf v[16];
  if (FWD) {
    const long long s0 = (long long)j.starts[pi];
#pragma unroll
    for (int s = 0; s < 16; s++) {
      const long long e = s0 + f1 + (long long)j.N1 * (t + T2 * s);
      float2 x = make_float2(0.f, 0.f);
      if (e < j.nseries) x = __ldg(j.series + e);
      v[s] = {x.x * j.scale, -x.y * j.scale};
    }
  } else {
    int row, d, tt;
    batch_pair(j, pi, row, d, tt);
    const float2 *dp = j.data + (long long)d * j.n;
    const float2 *hp = j.tmpl + (long long)tt * j.n;
#pragma unroll
    for (int s = 0; s < 16; s++) {
      const long long f = f1 + (long long)j.N1 * (t + T2 * s);
      const float2 x = j.fwd_units ? __ldcg(dp + f) : __ldg(dp + f), h = __ldg(hp + f);
      v[s].x = fmaf(x.x, h.x, x.y * h.y);
      v[s].y = fmaf(x.y, h.x, -x.x * h.y);
    }
  }
  inverse_passes<N2, true>(v, buf, j.tw2, t);
  const unsigned lo_mask = (1u << j.lo_bits) - 1u;
  float2 *yp = a.slots + (long long)(sg.q % a.nslots) * a.slot_elems + (long long)bp * j.n + f1;
#pragma unroll
  for (int q = 0; q < 16; q++) {
    const int k2 = t + T2 * q;
    const unsigned m = ((unsigned)f1 * (unsigned)k2) & (unsigned)(j.n - 1);
    const float2 wh = __ldg(j.tw_hi + (m >> j.lo_bits)), wl = __ldg(j.tw_lo + (m & lo_mask));
    const cf y = cmul(v[q], cmul(cf{wh.x, wh.y}, cf{wl.x, wl.y}));
    yp[(long long)k2 * j.N1] = make_float2(y.x, y.y);
  }
  }
  batch_done(a.a_done + sg.q, a.a_total[sg.q], (unsigned)(w1 - w0));
}

// Row pass: G1 = 4096/N1 rows k2 of one pair (or block), the N1-point inverse
// transform over f1, giving lags N2*k1 + k2; then the per-bin argmax merged
// into the output records (or, forward, the spectrum written out).
template <int N1, bool FWD>
__device__ __noinline__ void b_unit(int jid, int segi, int u, float2 *smem) {
  const BatchArgs &a = c_batch.args;
  const BatchJob &j = c_batch.jobs[jid];
  const BatchSeg sg = a.segs[segi];
  using Geo = FlatGeo<N1>;
  constexpr int T1 = Geo::T, G1 = Geo::G;
  if (!batch_wait(a.a_done + sg.q, a.a_total[sg.q], a.err)) return;
  const int g = threadIdx.x / T1, t = threadIdx.x % T1;
  float2 *buf = smem + g * Geo::BUF;
  unsigned long long *keys = reinterpret_cast<unsigned long long *>(smem + G1 * Geo::BUF);
  const int rgroups = j.N2 / G1;
  const int w0 = u * sg.per, w1 = min(sg.raw, w0 + sg.per);
  for (int w = w0; w < w1; w++) {
  __syncthreads();   // the previous unit's readers of keys and rows are done
  const int bp = w / rgroups, rg = w - bp * rgroups;
  const int k2base = rg * G1, k2 = k2base + g;
  const long long pi = (long long)sg.q_local * j.batch_pairs + bp;
  const float2 *yp = a.slots + (long long)(sg.q % a.nslots) * a.slot_elems +
                     ((long long)bp * j.N2 + k2) * j.N1;
  cf v[16];
#pragma unroll
  for (int s = 0; s < 16; s++) {
    const float2 x = __ldcg(yp + t + T1 * s);
    v[s] = {x.x, x.y};
  }
  if (!FWD)
    for (int b = threadIdx.x; b < j.nb; b += BATCH_CTA) keys[b] = 0ull;
  __syncthreads();
  inverse_passes<N1>(v, buf, j.tw1, t);
  if (FWD) {
    float2 *o = j.spec + pi * j.n + k2;
#pragma unroll
    for (int q = 0; q < 16; q++)
      o[(long long)j.N2 * (t + T1 * q)] = make_float2(v[q].x, -v[q].y);
    continue;
  }
  int row, d, tt;
  batch_pair(j, pi, row, d, tt);
  const float inv_bs = 1.0f / (float)j.binsize;
#pragma unroll
  for (int q = 0; q < 16; q++) {
    const int k1 = t + T1 * q;
    const int lag = j.N2 * k1 + k2;
    const float m2 = fmaf(v[q].x, v[q].x, v[q].y * v[q].y);
    if (lag >= j.ws && lag < j.we && m2 > j.t2) {
      const int bin = bin_of(lag - j.ws, j.binsize, inv_bs);
      atomicMax(keys + bin, ((unsigned long long)(__float_as_uint(m2) & ~31u) << 32) | (unsigned)(~lag));
      buf[pad16(k1)] = make_float2(v[q].x, v[q].y);
    }
  }
  __syncthreads();
  uint4 *rec = j.rec + (long long)row * j.nb;
  for (int b = threadIdx.x; b < j.nb; b += BATCH_CTA) {
    const unsigned long long kk = keys[b];
    if (kk == 0ull) continue;
    const int lag = (int)(~(unsigned)kk);
    const int gw = (lag % j.N2) - k2base, k1w = lag / j.N2;
    const float2 val = smem[gw * Geo::BUF + pad16(k1w)];
    rec_max(rec + b, make_uint4(__float_as_uint(val.x), __float_as_uint(val.y), (unsigned)kk,
                                (unsigned)(kk >> 32)));
  }
  }
  if (FWD) {
    batch_done(a.b_done + sg.q, a.b_total[sg.q], (unsigned)(w1 - w0));
    if (threadIdx.x == 0) atomicAdd(a.fwd_done + j.fwd_ctr, (unsigned)(w1 - w0));
    return;
  }
  if (batch_done(a.b_done + sg.q, a.b_total[sg.q], (unsigned)(w1 - w0))) {
    // Last row unit of the batch: records {re, im, ~lag, |z|^2 bits} become
    // {int64 index, re, im}, or {-1, 0, 0} where nothing was reported.
    const long long n_out = (long long)sg.pairs * j.nb;
    for (long long i = threadIdx.x; i < n_out; i += BATCH_CTA) {
      const int p = (int)(i / j.nb), b = (int)(i - (long long)p * j.nb);
      int r2, d2, t2;
      batch_pair(j, (long long)sg.q_local * j.batch_pairs + p, r2, d2, t2);
      uint4 *slot = j.rec + (long long)r2 * j.nb + b;
      const uint4 x = __ldcg(slot);
      long long ix = -1;
      float2 val = make_float2(0.f, 0.f);
      if (x.z != 0u || x.w != 0u) {
        ix = (long long)(int)(~x.z);
        val = make_float2(__uint_as_float(x.x), __uint_as_float(x.y));
      }
      *reinterpret_cast<longlong2 *>(slot) =
          make_longlong2(ix, (long long)(((unsigned long long)__float_as_uint(val.y) << 32) |
                                         __float_as_uint(val.x)));
    }
  }
}

// Index of the segment holding ticket tk: forward from the CTA's last one
// (tickets a CTA takes only grow), then bisection.
__device__ __forceinline__ int find_seg(long long tk, int from) {
  const BatchArgs &a = c_batch.args;
  int s = from;
  for (int i = 0; i < 8; i++) {
    if (s + 1 >= a.nseg || a.segs[s + 1].t0 > tk) return s;
    s++;
  }
  int lo = s, hi = a.nseg - 1;   // segs[lo].t0 <= tk
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (a.segs[mid].t0 <= tk) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__global__ void __launch_bounds__(BATCH_CTA, 2) batch_kernel() {
  const BatchArgs &a = c_batch.args;
  extern __shared__ __align__(16) float2 smem[];
  __shared__ long long s_tk;
  __shared__ int s_seg;
  int seg = 0;
  for (;;) {
    __syncthreads();   // the previous unit is done with s_tk, s_seg and smem
    if (threadIdx.x == 0) {
      long long tk = a.total;
      if (*(volatile int *)a.err == 0) tk = (long long)atomicAdd(a.ticket, 1ull);
      if (tk < a.total) seg = find_seg(tk, seg);
      s_tk = tk;
      s_seg = seg;
    }
    __syncthreads();
    const long long tk = s_tk;
    if (tk >= a.total) break;
    const int segi = s_seg;
    const BatchSeg sg = a.segs[segi];
    const int jid = sg.job;
    const int n = c_batch.jobs[jid].n;
    const int u = (int)(tk - sg.t0);
    switch (sg.kind) {
      case SEG_SMALL:
        switch (n) {
          case 64: small_unit<64>(jid, u, smem); break;
          case 128: small_unit<128>(jid, u, smem); break;
          case 256: small_unit<256>(jid, u, smem); break;
          case 512: small_unit<512>(jid, u, smem); break;
          case 1024: small_unit<1024>(jid, u, smem); break;
          case 2048: small_unit<2048>(jid, u, smem); break;
          default: small_unit<4096>(jid, u, smem); break;
        }
        break;
      case SEG_FWD_SMALL:
        switch (n) {
          case 64: fwd_small_unit<64>(jid, u, smem); break;
          case 128: fwd_small_unit<128>(jid, u, smem); break;
          case 256: fwd_small_unit<256>(jid, u, smem); break;
          case 512: fwd_small_unit<512>(jid, u, smem); break;
          case 1024: fwd_small_unit<1024>(jid, u, smem); break;
          case 2048: fwd_small_unit<2048>(jid, u, smem); break;
          default: fwd_small_unit<4096>(jid, u, smem); break;
        }
        break;
      case SEG_A:
      case SEG_FA: {
        const int N2 = c_batch.jobs[jid].N2;
        if (sg.kind == SEG_A) {
          if (N2 == 64) a_unit<64, false>(jid, segi, u, smem);
          else if (N2 == 128) a_unit<128, false>(jid, segi, u, smem);
          else a_unit<256, false>(jid, segi, u, smem);
        } else {
          if (N2 == 64) a_unit<64, true>(jid, segi, u, smem);
          else if (N2 == 128) a_unit<128, true>(jid, segi, u, smem);
          else a_unit<256, true>(jid, segi, u, smem);
        }
        break;
      }
      default: {
        const int N1 = c_batch.jobs[jid].N1;
        if (sg.kind == SEG_B) {
          switch (N1) {
            case 64: b_unit<64, false>(jid, segi, u, smem); break;
            case 128: b_unit<128, false>(jid, segi, u, smem); break;
            case 256: b_unit<256, false>(jid, segi, u, smem); break;
            case 512: b_unit<512, false>(jid, segi, u, smem); break;
            case 1024: b_unit<1024, false>(jid, segi, u, smem); break;
            case 2048: b_unit<2048, false>(jid, segi, u, smem); break;
            default: b_unit<4096, false>(jid, segi, u, smem); break;
          }
        } else {
          switch (N1) {
            case 64: b_unit<64, true>(jid, segi, u, smem); break;
            case 128: b_unit<128, true>(jid, segi, u, smem); break;
            case 256: b_unit<256, true>(jid, segi, u, smem); break;
            case 512: b_unit<512, true>(jid, segi, u, smem); break;
            case 1024: b_unit<1024, true>(jid, segi, u, smem); break;
            case 2048: b_unit<2048, true>(jid, segi, u, smem); break;
            default: b_unit<4096, true>(jid, segi, u, smem); break;
          }
        }
        break;
      }
    }
  }
}

// Dynamic shared memory the batched kernel needs: the largest unit.
constexpr int batch_smem_bytes() {
  int m = 0;
  const int small[7] = {FlatGeo<64>::SMEM, FlatGeo<128>::SMEM, FlatGeo<256>::SMEM,
                        FlatGeo<512>::SMEM, FlatGeo<1024>::SMEM, FlatGeo<2048>::SMEM,
                        FlatGeo<4096>::SMEM};
  for (int i = 0; i < 7; i++) m = small[i] > m ? small[i] : m;
  const int a_units[3] = {(BATCH_CTA / 4) * col_buf<64>() * 8,
                          (BATCH_CTA / 8) * col_buf<128>() * 8,
                          (BATCH_CTA / 16) * col_buf<256>() * 8};
  for (int i = 0; i < 3; i++) m = a_units[i] > m ? a_units[i] : m;
  const int b_units[7] = {FlatGeo<64>::G * FlatGeo<64>::BUF, FlatGeo<128>::G * FlatGeo<128>::BUF,
                          FlatGeo<256>::G * FlatGeo<256>::BUF, FlatGeo<512>::G * FlatGeo<512>::BUF,
                          FlatGeo<1024>::G * FlatGeo<1024>::BUF,
                          FlatGeo<2048>::G * FlatGeo<2048>::BUF,
                          FlatGeo<4096>::G * FlatGeo<4096>::BUF};
  for (int i = 0; i < 7; i++) {
    const int b = b_units[i] * 8 + BATCH_MAX_BINS * 8;
    m = b > m ? b : m;
  }
  return m;
}

}  // namespace mfb
