// Coarse-gate model on the device: the reference's Monte-Carlo gate
// (python/matchedfilter/gatemodel.py:63-140) with its FP64 parts -- profile
// sums, lag covariances A(d) = sum_k q_k exp(2 pi i k d / n) of the full and
// in-band profile, their Cholesky factors -- and its FP32 parts -- noise
// transforms of the draws, coarse and fine maxima -- all on the GPU.  The
// Gaussian draws themselves come from the caller (the model's seeded numpy
// stream), so the estimator is the reference's draw for draw.
#pragma once
#include <cstdint>

namespace mfb {

constexpr int GATE_K = 16;          // lags per sub-grid offset (taus), at most
constexpr int GATE_GRID = 9;        // coarse grid lags (-4 .. 4 steps)

struct GateArgs {
  const double *power;              // [n] profile (any scale)
  int n, band, dmax;                // lag table covers d in [-dmax, dmax]
  double *sums;                     // [2]: total, in-band
  double2 *a_full, *a_band;         // [2*dmax+1]
  int step, per, has_out;
  const int *taus;                  // [step][GATE_K]
  const int *ntaus;                 // [step]
  const int *on_grid;               // [step][GATE_GRID] indices into taus
  float2 *l_in, *l_out;             // [step][GATE_K][GATE_K] complex64 factors
  float2 *s_full, *s_band;          // [step][GATE_K]
  const float2 *draw_in, *draw_out; // [step][per][GATE_K]
  float snr;
  float *coarse, *fine;             // [step][per]
};

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide FP64 sum (blockDim.x a multiple of 32, <= 1024); every thread gets it.
__device__ double block_sum(double v) {
  __shared__ double part[32];
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) part[w] = v;
  __syncthreads();
  double s = 0.0;
  for (int i = 0; i < (int)(blockDim.x >> 5); i++) s += part[i];
  return s;
}

// sums[0] = sum power, sums[1] = sum of the lowest `band` bins (one block).
__global__ void gate_sums_kernel(const GateArgs a) {
  double t = 0.0, lo = 0.0;
  for (int k = threadIdx.x; k < a.n; k += blockDim.x) {
    const double p = a.power[k];
    t += p;
    if (k < a.band) lo += p;
  }
  t = block_sum(t);
  lo = block_sum(lo);
  if (threadIdx.x == 0) {
    a.sums[0] = t;
    a.sums[1] = lo;
  }
}

// One block per lag d: A_full(d) and A_band(d) in FP64.
__global__ void gate_lags_kernel(const GateArgs a) {
  const int d = (int)blockIdx.x - a.dmax;
  const double total = a.sums[0];
  double f = a.sums[1] / total;
  f = f < 0.0 ? 0.0 : (f > 1.0 ? 1.0 : f);
  double fr = 0.0, fi = 0.0, br = 0.0, bi = 0.0;
  for (int k = threadIdx.x; k < a.n; k += blockDim.x) {
    const double q = a.power[k] / total;
    long long m = ((long long)k * d) % a.n;
    if (m < 0) m += a.n;
    double s, c;
    sincospi(2.0 * (double)m / (double)a.n, &s, &c);
    fr += q * c;
    fi += q * s;
    if (k < a.band) {
      br += q * c;
      bi += q * s;
    }
  }
  fr = block_sum(fr);
  fi = block_sum(fi);
  br = block_sum(br);
  bi = block_sum(bi);
  if (threadIdx.x == 0) {
    a.a_full[blockIdx.x] = make_double2(fr, fi);
    a.a_band[blockIdx.x] = f > 0.0 ? make_double2(br / f, bi / f) : make_double2(0.0, 0.0);
  }
}

// Lower Cholesky factor of the Hermitian matrix (c + c^H)/2 + 1e-9 I, FP64.
__device__ void chol16(double2 (*c)[GATE_K], int K, float2 *out) {
  double2 L[GATE_K][GATE_K];
  for (int i = 0; i < K; i++)
    for (int j = 0; j < K; j++) {
      const double2 x = c[i][j], y = c[j][i];
      L[i][j] = make_double2(0.5 * (x.x + y.x), 0.5 * (x.y - y.y));
    }
  for (int i = 0; i < K; i++) L[i][i].x += 1e-9;
  for (int j = 0; j < K; j++) {
    double dsum = L[j][j].x;
    for (int k = 0; k < j; k++) dsum -= L[j][k].x * L[j][k].x + L[j][k].y * L[j][k].y;
    const double djj = sqrt(dsum > 0.0 ? dsum : 0.0);
    L[j][j] = make_double2(djj, 0.0);
    for (int i = j + 1; i < K; i++) {
      double re = L[i][j].x, im = L[i][j].y;
      for (int k = 0; k < j; k++) {   // - L[i][k] * conj(L[j][k])
        re -= L[i][k].x * L[j][k].x + L[i][k].y * L[j][k].y;
        im -= L[i][k].y * L[j][k].x - L[i][k].x * L[j][k].y;
      }
      L[i][j] = djj > 0.0 ? make_double2(re / djj, im / djj) : make_double2(0.0, 0.0);
    }
    for (int i = 0; i < j; i++) L[i][j] = make_double2(0.0, 0.0);
  }
  for (int i = 0; i < GATE_K; i++)
    for (int j = 0; j < GATE_K; j++)
      out[i * GATE_K + j] = (i < K && j < K) ? make_float2((float)L[i][j].x, (float)L[i][j].y)
                                             : make_float2(0.f, 0.f);
}

__device__ __forceinline__ double2 lag_at(const double2 *table, int dmax, int d) {
  return table[d + dmax];
}

// One thread per sub-grid offset: covariances at the offset's lag
// differences, their factors, and the signal shapes at taus - offset.
__global__ void gate_chol_kernel(const GateArgs a) {
  const int off = blockIdx.x * blockDim.x + threadIdx.x;
  if (off >= a.step) return;
  const int K = a.ntaus[off];
  const int *tau = a.taus + off * GATE_K;
  double f = a.sums[1] / a.sums[0];
  f = f < 0.0 ? 0.0 : (f > 1.0 ? 1.0 : f);
  double2 c[GATE_K][GATE_K];
  for (int i = 0; i < K; i++)
    for (int j = 0; j < K; j++) c[i][j] = lag_at(a.a_band, a.dmax, tau[i] - tau[j]);
  chol16(c, K, a.l_in + (size_t)off * GATE_K * GATE_K);
  if (a.has_out) {
    for (int i = 0; i < K; i++)
      for (int j = 0; j < K; j++) {
        const double2 af = lag_at(a.a_full, a.dmax, tau[i] - tau[j]);
        const double2 ab = lag_at(a.a_band, a.dmax, tau[i] - tau[j]);
        c[i][j] = make_double2((af.x - f * ab.x) / (1.0 - f), (af.y - f * ab.y) / (1.0 - f));
      }
    chol16(c, K, a.l_out + (size_t)off * GATE_K * GATE_K);
  }
  for (int i = 0; i < GATE_K; i++) {
    float2 sf = make_float2(0.f, 0.f), sb = sf;
    if (i < K) {
      const double2 xf = lag_at(a.a_full, a.dmax, tau[i] - off);
      const double2 xb = lag_at(a.a_band, a.dmax, tau[i] - off);
      sf = make_float2((float)xf.x, (float)xf.y);
      sb = make_float2((float)xb.x, (float)xb.y);
    }
    a.s_full[off * GATE_K + i] = sf;
    a.s_band[off * GATE_K + i] = sb;
  }
}

// One thread per draw: noise = draw @ L^T (times sqrt 2), the fine maximum
// over all taus of |snr s_full + sqrt(f) n_in + sqrt(1-f) n_out| and the
// coarse maximum over the grid lags of |snr sqrt(f) s_band + n_in|, in FP32.
__global__ void gate_draw_kernel(const GateArgs a) {
  const int off = blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.per) return;
  const int K = a.ntaus[off];
  double f = a.sums[1] / a.sums[0];
  f = f < 0.0 ? 0.0 : (f > 1.0 ? 1.0 : f);
  const float sq_in = (float)sqrt(f), sq_out = (float)sqrt(1.0 - f);
  const float cs = (float)((double)a.snr * sqrt(f));
  const float scale = (float)sqrt(2.0);
  const float2 *L = a.l_in + (size_t)off * GATE_K * GATE_K;
  const float2 *Lo = a.l_out + (size_t)off * GATE_K * GATE_K;
  const float2 *w = a.draw_in + ((size_t)off * a.per + i) * GATE_K;
  const float2 *wo = a.has_out ? a.draw_out + ((size_t)off * a.per + i) * GATE_K : nullptr;
  float2 din[GATE_K], dout[GATE_K];
#pragma unroll
  for (int b = 0; b < GATE_K; b++) {
    din[b] = b < K ? w[b] : make_float2(0.f, 0.f);
    dout[b] = (wo && b < K) ? wo[b] : make_float2(0.f, 0.f);
  }
  const int *grid = a.on_grid + off * GATE_GRID;
  float fine = 0.f, coarse = 0.f;
  for (int r = 0; r < K; r++) {
    float nr = 0.f, ni = 0.f, orr = 0.f, oi = 0.f;
#pragma unroll
    for (int b = 0; b < GATE_K; b++) {
      const float2 l = L[r * GATE_K + b];
      nr = fmaf(din[b].x, l.x, fmaf(-din[b].y, l.y, nr));
      ni = fmaf(din[b].x, l.y, fmaf(din[b].y, l.x, ni));
      if (wo) {
        const float2 lo = Lo[r * GATE_K + b];
        orr = fmaf(dout[b].x, lo.x, fmaf(-dout[b].y, lo.y, orr));
        oi = fmaf(dout[b].x, lo.y, fmaf(dout[b].y, lo.x, oi));
      }
    }
    nr *= scale; ni *= scale; orr *= scale; oi *= scale;
    const float2 sf = a.s_full[off * GATE_K + r], sb = a.s_band[off * GATE_K + r];
    const float fr = a.snr * sf.x + sq_in * nr + sq_out * orr;
    const float fi = a.snr * sf.y + sq_in * ni + sq_out * oi;
    fine = fmaxf(fine, sqrtf(fr * fr + fi * fi));
    bool on = false;
    for (int g = 0; g < GATE_GRID; g++) on |= (grid[g] == r);
    if (on) {
      const float cr = cs * sb.x + nr, ci = cs * sb.y + ni;
      coarse = fmaxf(coarse, sqrtf(cr * cr + ci * ci));
    }
  }
  a.coarse[(size_t)off * a.per + i] = coarse;
  a.fine[(size_t)off * a.per + i] = fine;
}

}  // namespace mfb
