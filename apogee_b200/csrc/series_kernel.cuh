// Forward transform of time-series blocks for run_series.
//
// Block b covers series[start_b .. start_b + n), zero-padded past the end of
// the series, and its spectrum is FFT(x / n), unnormalised forward transform
// of the 1/n-scaled block (src/matchfilt.c:454-470; GPU form
// src/gpu/series_forward.slang:8-33).  n is a power of two, so the 1/n scale
// is exact and applying it on the way in is bit-identical to applying it to
// the spectrum.  The forward transform is the inverse one conjugated on both
// sides: FFT(x) = conj(IFFT(conj(x))), so it reuses inverse_passes.
#pragma once
#include "flat_kernel.cuh"

namespace mfb {

struct SeriesArgs {
  const float2 *series;            // complex64 samples
  long long nseries;
  const unsigned long long *starts;   // [nblocks] sample offsets
  int nblocks;
  float2 *out;                     // spectra, row b at out + b*out_stride
  long long out_stride;
  const float2 *twid;
  float scale;                     // 1/n
};

template <int N>
__global__ void __launch_bounds__(FlatGeo<N>::CTA)
series_forward_kernel(const SeriesArgs a) {
  using Geo = FlatGeo<N>;
  constexpr int T = Geo::T, G = Geo::G;
  extern __shared__ __align__(16) float2 smem[];
  const int g = threadIdx.x / T, t = threadIdx.x % T;
  float2 *buf = smem + g * Geo::BUF;
  const int rounds = (a.nblocks + G * gridDim.x - 1) / (G * gridDim.x);
  for (int r = 0; r < rounds; r++) {
    const int b = (r * gridDim.x + blockIdx.x) * G + g;
    const bool live = b < a.nblocks;
    cf v[16];
    if (live) {
      const long long s0 = (long long)a.starts[b];
#pragma unroll
      for (int s = 0; s < 16; s++) {
        const long long e = s0 + t + T * s;
        float2 x = make_float2(0.f, 0.f);
        if (e < a.nseries) x = __ldg(a.series + e);
        v[s] = {x.x * a.scale, -x.y * a.scale};
      }
    } else {
#pragma unroll
      for (int s = 0; s < 16; s++) v[s] = {0.f, 0.f};
    }
    inverse_passes<N>(v, buf, a.twid, t);
    if (live) {
      float2 *o = a.out + (long long)b * a.out_stride;
#pragma unroll
      for (int q = 0; q < 16; q++) o[t + T * q] = make_float2(v[q].x, -v[q].y);
    }
  }
}

}  // namespace mfb
