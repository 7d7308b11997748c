// Fused matched filter for n = 32768 and 65536 on a thread-block cluster:
// the four-step split of the two-pass kernels (large_kernel.cuh) with the
// transpose between the passes carried through distributed shared memory
// instead of an HBM/L2 scratch.
//
// n = N1 * N2, f = f1 + N1 f2, k = N2 k1 + k2:
//
//   z[N2 k1 + k2] = sum_f1 W_N1^(f1 k1) [ W_n^(f1 k2) sum_f2 P[f1 + N1 f2] W_N2^(f2 k2) ]
//
// A cluster of C CTAs (n / C points per CTA, 16 per thread) takes one pair
// at a time:
//   pass A   CTA r forms the conjugate product for columns f1 in
//            [r N1/C, (r+1) N1/C) (a half-warp loads 16 adjacent columns:
//            128-byte rows), runs their N2-point inverse FFTs and the twiddle
//            W_n^(f1 k2), and stores Y[k2][f1] straight into the shared memory
//            of the CTA that owns row k2 (rows [r N2/C, (r+1) N2/C) belong to
//            CTA r; a half-warp's 16 stores are one 128-byte row segment);
//   pass B   each CTA runs the N1-point inverse FFTs of its rows, keeps the
//            per-bin maximum of the pass-B keys (pass_b_key) with shared atomics
//            and parks every candidate's value in place; CTA r then takes bins
//            r, r + C, ...: the maximum over the CTAs' keys and the winner's
//            value, read from the other CTAs' shared memory (plain loads: no
//            atomics across the cluster), and writes the outputs.
// Three cluster barriers per pair order the steps (every CTA done reading the
// previous pair -> rows written -> every CTA's keys final); one more before
// exit keeps every CTA's shared memory alive while the others read from it.
// Clusters of 8 or 16 CTAs of 256 threads (4096 points each, three CTAs per
// SM) or of 4 / 8 CTAs of 512 threads (8192 points, one per SM).  Measured
// on a B200 against the two-pass kernels (the default): 0.35 vs 0.31 us per
// pair at n = 32768 and 0.82 vs 0.60 at 65536 on dense blocks with binsize
// n/16 (pass B takes ~45% of a CTA's time, the three barriers ~20%),
// faster on short row lists at n = 32768, where the two-pass path reads the
// row count on the host.  The arithmetic (products, FFT passes,
// twiddles, key order) is that of large_pass_a / large_pass_b, so the outputs
// equal the two-pass kernels'.  Clusters walk the pairs template-major with a
// stride of the cluster count, so clusters running at the same time share a
// template spectrum in L2.
#pragma once
#include <cooperative_groups.h>
#include "large_kernel.cuh"

namespace mfb {

// Cluster barrier without release semantics (barrier.cluster.wait still
// acquires): for a barrier that only orders reads before later writes.
__device__ __forceinline__ void cluster_sync_relaxed() {
  asm volatile("barrier.cluster.arrive.relaxed.aligned;\n\tbarrier.cluster.wait.aligned;" ::: "memory");
}

template <int N1, int N2, int C>
struct ClusterGeo {
  static constexpr int N = N1 * N2;
  static constexpr int TH = N / (16 * C);             // threads per CTA
  static constexpr int CA = N1 / C;                   // pass-A columns per CTA
  static constexpr int T2 = N2 / 16;                  // threads per column
  static constexpr int RB = N2 / C;                   // pass-B rows per CTA
  static constexpr int T1 = N1 / 16;                  // threads per row
  static constexpr int BUF1 = FlatGeo<N1>::BUF;       // float2 per received row
  static constexpr int COLS = CA * col_buf<N2>();     // float2, pass-A column buffers
  static constexpr int ROWS = RB * BUF1;              // float2, rows of pass B
  static constexpr int SMEM_FIXED = (COLS + ROWS) * 8;
  static constexpr int MINB = TH == 256 ? 3 : 1;      // CTAs per SM the registers allow
  static_assert(CA * T2 == TH && RB * T1 == TH, "both passes use every thread");
  static_assert(TH == 256 || TH == 512, "256 or 512 threads per CTA");
  static_assert(CA % 16 == 0, "a half-warp covers 16 adjacent columns");
};

template <int N1, int N2, int C>
__global__ void __launch_bounds__(ClusterGeo<N1, N2, C>::TH, ClusterGeo<N1, N2, C>::MINB)
cluster_kernel(const LargeArgs a) {
  namespace cg = cooperative_groups;
  using Geo = ClusterGeo<N1, N2, C>;
  constexpr int TH = Geo::TH, CA = Geo::CA, T2 = Geo::T2, RB = Geo::RB, T1 = Geo::T1;
  constexpr int BUF1 = Geo::BUF1;
  extern __shared__ __align__(16) float2 smem[];
  float2 *cols = smem;                                   // pass A
  float2 *rows = smem + Geo::COLS;                       // pass B (written by every CTA)
  unsigned long long *keys = reinterpret_cast<unsigned long long *>(rows + Geo::ROWS);
  cg::cluster_group cluster = cg::this_cluster();
  if (cluster.num_blocks() != (unsigned)C || gridDim.x % C != 0) return;   // every CTA alike
  const int rank = (int)cluster.block_rank();
  const int nclusters = (int)(gridDim.x / C);
  const int cid = (int)(blockIdx.x / C);
  const int tid = threadIdx.x;
  const long long total = a.list_count ? (long long)(*a.list_count) : a.total;
  const int bs = a.binsize;
  const float inv_bs = 1.0f / (float)bs;
  unsigned smask = 0u, srank = 0u;
  if (a.seg > 0) bin_segment(T1, a.seg, smask, srank);

  // pass-A geometry: column c of this CTA, point group t
  const int c = tid % CA, t = tid / CA;
  const int f1 = rank * CA + c;
  float2 *cbuf = cols + c * col_buf<N2>();
  // pass-B geometry: row g of this CTA (k2 = rank*RB + g), thread t1
  const int g = tid / T1, t1 = tid % T1;
  const int k2b = rank * RB + g;
  float2 *rbuf = rows + g * BUF1;

  for (long long pi = cid; pi < total; pi += nclusters) {
    int orow, d, tt;
    large_pair(a, pi, orow, d, tt);
    // ---- pass A: product, N2-point inverse FFT per column, twiddle ----------
    cf v[16];
    {
      const float2 *dp = a.data + (long long)(a.d0 + d) * a.n;
      const float2 *hp = a.tmpl + (long long)(a.t0 + tt) * a.n;
#pragma unroll
      for (int s = 0; s < 16; s++) {
        const int f = f1 + N1 * (t + T2 * s);
        const float2 x = __ldg(dp + f), h = __ldg(hp + f);
        v[s].x = fmaf(x.x, h.x, x.y * h.y);
        v[s].y = fmaf(x.y, h.x, -x.x * h.y);
      }
    }
    inverse_passes<N2, true>(v, cbuf, a.tw2, t);
    pass_a_twiddle<T2>(v, a, f1, t);
    // every CTA has read the previous pair's keys and parked values (the
    // values read were consumed before this barrier: no release needed)
    cluster_sync_relaxed();
    for (int b = tid; b < a.nb; b += TH) keys[b] = 0ull;
#pragma unroll
    for (int q = 0; q < 16; q++) {
      const int k2 = t + T2 * q;
      float2 *dst = cluster.map_shared_rank(rows, k2 / RB);
      dst[(k2 % RB) * BUF1 + f1] = make_float2(v[q].x, v[q].y);
    }
    cluster.sync();
    // ---- pass B: N1-point inverse FFT per row, per-bin maxima ----------------
#pragma unroll
    for (int s = 0; s < 16; s++) {
      const float2 x = rbuf[t1 + T1 * s];
      v[s] = {x.x, x.y};
    }
    inverse_passes<N1>(v, rbuf, a.tw1, t1);
    // thread t1 holds z[N2 k1 + k2b] for k1 = t1 + T1 q; rbuf is free
#pragma unroll
    for (int q = 0; q < 16; q++) {
      const int k1 = t1 + T1 * q;
      const int lag = N2 * k1 + k2b;
      const float m2 = fmaf(v[q].x, v[q].x, v[q].y * v[q].y);
      pass_b_key(keys, rbuf + pad16(k1), v[q], m2, lag, lag >= a.ws && lag < a.we && m2 > a.t2,
                 a.seg, smask, srank, a.ws, bs, inv_bs);
    }
    cluster.sync();
    // ---- outputs: CTA r takes bins r, r + C, ...: maximum over the CTAs' keys -----
    {
      for (int b = rank + C * tid; b < a.nb; b += C * TH) {
        unsigned long long kk = 0ull;
#pragma unroll
        for (int r = 0; r < C; r++) {
          const unsigned long long kr = cluster.map_shared_rank(keys, r)[b];
          kk = kr > kk ? kr : kk;
        }
        const long long o = ((long long)orow * a.nb + b) * a.rs;
        if (kk == 0ull) {
          a.out_idx[o] = -1;
          a.out_val[o] = make_float2(0.f, 0.f);
        } else {
          const int lag = (int)(~(unsigned)kk);
          const int k2 = lag & (N2 - 1), k1 = lag / N2;
          const float2 *src = cluster.map_shared_rank(rows, k2 / RB);
          a.out_idx[o] = lag;
          a.out_val[o] = src[(k2 % RB) * BUF1 + pad16(k1)];
          if (a.out_cnt) atomicAdd(a.out_cnt + orow, 1);
        }
      }
    }
  }
  // other CTAs may still read this one's keys and parked values
  cluster.sync();
}

}  // namespace mfb
