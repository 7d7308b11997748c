// Adjoint of the fused filter's peak values at fixed lags.
//
// A reported peak of pair (d, t) in bin b is z = sum_f D[d,f] conj(H[t,f]) W^(f k)
// with W = exp(2 pi i / n) and k its lag.  With g the upstream gradient of z in
// torch's convention (dL/dRe z + i dL/dIm z), z is holomorphic in D and
// antiholomorphic in H, so
//
//   grad_D[d, f] = sum_t sum_b  g_dtb       H[t, f] W^(-f k_dtb)
//   grad_H[t, f] = sum_d sum_b  conj(g_dtb) D[d, f] W^(+f k_dtb)
//
// One kernel serves both: "own" rows are the ones written (d for grad_D, t for
// grad_H), "other" rows are summed over.  Each thread owns frequencies f and
// f + n/2, whose twiddles differ by (-1)^k, and OC own rows; the (lag,
// gradient) entries of the CTA's rows are staged in shared memory in rounds,
// read as broadcasts.  Twiddles come from FP64-built hi/lo tables in shared
// memory: W^m = hi[m >> lo_bits] * lo[m & (2^lo_bits - 1)].  The lags are the
// forward pass's argmax lags; nothing of the correlation series is stored.
#pragma once
#include <cstdint>
#include "fft_radix.cuh"

namespace mfb {

constexpr int ADJ_THREADS = 256;
constexpr int ADJ_CAP = 2048;   // staged (lag, gradient) entries per round
constexpr int ADJ_TW = 1024;    // entries of each twiddle half-table (n <= 2^20)

struct AdjArgs {
  const float2 *src;      // other rows [other][n]: templates (grad_D) or data (grad_H)
  const int64_t *idx;     // [nd][nt][nb] lags; < 0 where no peak was reported
  const float2 *gz;       // [nd][nt][nb] upstream gradient of the peak value
  float2 *out;            // [own][n]
  int n, nd, nt, nb;
  int own, other;
  int rows_per_round, bins_per_round;
  int other_per_split;    // other rows per blockIdx.z
  const float2 *tw_hi, *tw_lo;
  int lo_bits, hi_count;
  int accumulate;         // 1: atomicAdd into a zeroed out (other split over blockIdx.z)
};

template <int OC, bool GRAD_DATA>
__global__ void __launch_bounds__(ADJ_THREADS) adjoint_kernel(const AdjArgs a) {
  __shared__ float2 s_hi[ADJ_TW], s_lo[ADJ_TW];
  __shared__ int s_k[ADJ_CAP];
  __shared__ float2 s_g[ADJ_CAP];
  const int half = a.n >> 1;
  const int f = blockIdx.x * ADJ_THREADS + threadIdx.x;
  const int j0 = blockIdx.y * OC;
  const int ob = blockIdx.z * a.other_per_split;
  const int oe = min(a.other, ob + a.other_per_split);
  const unsigned mask_n = (unsigned)a.n - 1u, lo_mask = (1u << a.lo_bits) - 1u;
  for (int i = threadIdx.x; i < a.hi_count; i += ADJ_THREADS) s_hi[i] = a.tw_hi[i];
  for (int i = threadIdx.x; i <= (int)lo_mask; i += ADJ_THREADS) s_lo[i] = a.tw_lo[i];
  cf acc0[OC], acc1[OC];
#pragma unroll
  for (int j = 0; j < OC; j++) acc0[j] = acc1[j] = cf{0.f, 0.f};

  for (int o0 = ob; o0 < oe; o0 += a.rows_per_round) {
    const int rr = min(a.rows_per_round, oe - o0);
    for (int b0 = 0; b0 < a.nb; b0 += a.bins_per_round) {
      const int bc = min(a.bins_per_round, a.nb - b0);
      const int per_row = OC * bc, total = rr * per_row;
      __syncthreads();   // the previous round's readers are done (and the tables are in)
      for (int e = threadIdx.x; e < total; e += ADJ_THREADS) {
        const int ol = e / per_row, rem = e - ol * per_row;
        const int jj = rem / bc, bl = rem - jj * bc;
        int k = 0;
        float2 g = make_float2(0.f, 0.f);
        const int own_row = j0 + jj;
        if (own_row < a.own) {
          const int o = o0 + ol;
          const int d = GRAD_DATA ? own_row : o, t = GRAD_DATA ? o : own_row;
          const long long i = ((long long)d * a.nt + t) * a.nb + b0 + bl;
          const long long kk = a.idx[i];
          if (kk >= 0) {
            k = (int)kk;
            g = a.gz[i];
            if (!GRAD_DATA) g.y = -g.y;   // conj(g)
          }
        }
        s_k[e] = k;
        s_g[e] = g;
      }
      __syncthreads();
      if (f < half) {
        for (int ol = 0; ol < rr; ol++) {
          const float2 *sp = a.src + (long long)(o0 + ol) * a.n;
          const float2 s0 = __ldg(sp + f), s1 = __ldg(sp + f + half);
#pragma unroll
          for (int jj = 0; jj < OC; jj++) {
            cf u0 = {0.f, 0.f}, u1 = {0.f, 0.f};
            const int eb = (ol * OC + jj) * bc;
            for (int bl = 0; bl < bc; bl++) {
              const int k = s_k[eb + bl];
              const float2 g = s_g[eb + bl];
              const unsigned m = ((unsigned)f * (unsigned)k) & mask_n;
              const float2 wh = s_hi[m >> a.lo_bits], wl = s_lo[m & lo_mask];
              const float wr = fmaf(wh.x, wl.x, -wh.y * wl.y);
              const float wi = fmaf(wh.x, wl.y, wh.y * wl.x);
              float tr, ti;
              if (GRAD_DATA) {           // g * conj(W^(fk))
                tr = fmaf(g.x, wr, g.y * wi);
                ti = fmaf(g.y, wr, -g.x * wi);
              } else {                   // conj(g) * W^(fk)
                tr = fmaf(g.x, wr, -g.y * wi);
                ti = fmaf(g.x, wi, g.y * wr);
              }
              const float sgn = (k & 1) ? -1.f : 1.f;   // W^((f + n/2) k) = (-1)^k W^(fk)
              u0.x += tr;
              u0.y += ti;
              u1.x = fmaf(sgn, tr, u1.x);
              u1.y = fmaf(sgn, ti, u1.y);
            }
            acc0[jj].x = fmaf(s0.x, u0.x, fmaf(-s0.y, u0.y, acc0[jj].x));
            acc0[jj].y = fmaf(s0.x, u0.y, fmaf(s0.y, u0.x, acc0[jj].y));
            acc1[jj].x = fmaf(s1.x, u1.x, fmaf(-s1.y, u1.y, acc1[jj].x));
            acc1[jj].y = fmaf(s1.x, u1.y, fmaf(s1.y, u1.x, acc1[jj].y));
          }
        }
      }
    }
  }
  if (f < half) {
#pragma unroll
    for (int jj = 0; jj < OC; jj++) {
      if (j0 + jj >= a.own) break;
      float2 *op = a.out + (long long)(j0 + jj) * a.n;
      if (a.accumulate) {
        atomicAdd(&op[f].x, acc0[jj].x);
        atomicAdd(&op[f].y, acc0[jj].y);
        atomicAdd(&op[f + half].x, acc1[jj].x);
        atomicAdd(&op[f + half].y, acc1[jj].y);
      } else {
        op[f] = make_float2(acc0[jj].x, acc0[jj].y);
        op[f + half] = make_float2(acc1[jj].x, acc1[jj].y);
      }
    }
  }
}

}  // namespace mfb
