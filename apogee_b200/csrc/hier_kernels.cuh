// Hierarchical-filter support kernels: FP64 band fractions and coarse
// template scaling (src/hmf.c:118-156), plus the interface of the tensor-core
// coarse pass (coarse_tc.cu).
#pragma once
#include <type_traits>
#include <cuda_runtime.h>
#include <cstdint>

namespace mfb {

struct HierFpowArgs {
  const float2 *tmpl;   // [nt][n]
  int n, m, t0, count;
  float *fpow;          // [nt]
};
struct HierScaleArgs {
  const float2 *tmpl;   // [nt][n]
  int n, m, t0, count;
  int ref_on;
  float ref_f;
  const float *fpow;
  float2 *ct;           // [nt][m]
};

// Band fraction of each template, sum_{k<m}|H_k|^2 / sum_k |H_k|^2, with both
// sums in FP64 and the ratio rounded to float (src/hmf.c:144-153).
static __global__ void hier_fpow_kernel(const HierFpowArgs a) {
  const int t = a.t0 + blockIdx.x;
  const float2 *h = a.tmpl + (long long)t * a.n;
  double low = 0.0, total = 0.0;
  for (int k = threadIdx.x; k < a.n; k += blockDim.x) {
    const float2 x = h[k];
    const double p = (double)x.x * x.x + (double)x.y * x.y;
    total += p;
    if (k < a.m) low += p;
  }
  __shared__ double sl[32], st[32];
  for (int o = 16; o; o >>= 1) {
    low += __shfl_xor_sync(0xffffffffu, low, o);
    total += __shfl_xor_sync(0xffffffffu, total, o);
  }
  if ((threadIdx.x & 31) == 0) { sl[threadIdx.x >> 5] = low; st[threadIdx.x >> 5] = total; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double L = 0.0, S = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) { L += sl[w]; S += st[w]; }
    a.fpow[t] = S > 0.0 ? (float)(L / S) : 0.f;
  }
}

// ct[t][k] = (float)(H[t][k] * (1/sqrt(f))) in double, f the reference
// fraction or the row's own; f <= 0 gives a zero coarse template
// (src/hmf.c:118-124).
static __global__ void hier_scale_kernel(const HierScaleArgs a) {
  const int t = a.t0 + blockIdx.x;
  const double f = a.ref_on ? (double)a.ref_f : (double)a.fpow[t];
  const double sc = f > 0.0 ? 1.0 / sqrt(f) : 0.0;
  const float2 *h = a.tmpl + (long long)t * a.n;
  float2 *c = a.ct + (long long)t * a.m;
  for (int k = threadIdx.x; k < a.m; k += blockDim.x) {
    const float2 x = h[k];
    c[k] = make_float2((float)((double)x.x * sc), (float)((double)x.y * sc));
  }
}

inline cudaError_t launch_hier_fpow(const HierFpowArgs &a, cudaStream_t s) {
  hier_fpow_kernel<<<a.count, 256, 0, s>>>(a);
  return cudaGetLastError();
}
inline cudaError_t launch_hier_scale(const HierScaleArgs &a, cudaStream_t s) {
  hier_scale_kernel<<<a.count, 256, 0, s>>>(a);
  return cudaGetLastError();
}

// The hierarchical run's table written straight into a caller's pinned host
// table (mapped memory, stores over the host link).  Every row the gate
// dismisses is all empty records (index -1, value 0), so when the host table
// holds the previous run's result only the rows that change cross the link:
// the rows refined now are written, and the rows refined last time but not
// now are reset to empty.  Three launches:
//   hier_mark_kernel     marks the rows of this run's list (bit p of
//                        mark[row], p the run's parity), after the coarse pass;
//   hier_unwrite_kernel  resets the rows of the previous list that carry no
//                        mark of this run, clears the previous run's mark bit,
//                        stores this run's list for the next one (list store
//                        p) and, in its last block, flips the parity -- these
//                        two on a second stream while the refine runs (the
//                        rows they touch are not the refined ones);
//   hier_write_kernel    writes the refined rows after the refine, unless the
//                        refine kernel stored them into the table itself.
// State on the device (so that a CUDA graph of the run replays correctly):
// mark[rows], list_store[2][rows], count_store[2], ctl = {parity, blocks
// done, rows reset}.
struct HierHostArgs {
  const int4 *records;        // device table [rows][nb]
  int4 *table;                // host table [rows][nb] (device-visible pointer)
  long long nb;
  const int32_t *list, *count;        // this run's refined rows
  uint32_t *mark;             // [rows]
  int32_t *list_store;        // [2][rows]
  int32_t *count_store;       // [2]
  unsigned *ctl;              // [3]
  long long rows;
  unsigned long long *total;  // plan's trigger total
  long long *info;            // host [2] (device-visible) or null: refined rows, bytes written
  int write_rows;             // 0: the table was copied whole, only bookkeeping
  long long full_bytes;       // bytes of that whole copy
};

// Marks this run's rows (bit p of mark[row]); runs before hier_unwrite_kernel,
// which needs the marks, and may run beside the refine: neither reads the
// refined values.
static __global__ void hier_mark_kernel(const HierHostArgs a) {
  const long long c = *a.count;
  const uint32_t bit = 1u << (a.ctl[0] & 1u);
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  for (long long i = t0; i < c; i += stride) a.mark[a.list[i]] |= bit;   // rows are unique
}

// Copies this run's refined rows into the host table (after the refine;
// not needed when the refine kernel stored them there itself).
static __global__ void hier_write_kernel(const HierHostArgs a) {
  const long long c = *a.count;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (a.write_rows)
    for (long long e = t0; e < c * a.nb; e += stride) {
      const long long i = e / a.nb;
      const long long at = (long long)a.list[i] * a.nb + (e - i * a.nb);
      a.table[at] = a.records[at];
    }
}

static __global__ void hier_unwrite_kernel(const HierHostArgs a) {
  const unsigned p = a.ctl[0] & 1u, q = p ^ 1u;
  const uint32_t now = 1u << p, old = 1u << q;
  const long long c = *a.count;
  const long long pc = a.count_store[q];
  const int32_t *prev = a.list_store + q * a.rows;
  int32_t *keep = a.list_store + p * a.rows;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int4 empty = make_int4(-1, -1, 0, 0);
  unsigned reset = 0;
  if (a.write_rows)
    for (long long e = t0; e < pc * a.nb; e += stride) {
      const long long i = e / a.nb, j = e - i * a.nb;
      const int32_t r = prev[i];
      if (!(a.mark[r] & now)) {
        a.table[(long long)r * a.nb + j] = empty;
        if (j == 0) reset++;
      }
    }
  __syncthreads();     // every thread of the block has read the marks it needs
  for (long long i = t0; i < pc; i += stride) {
    // the previous run's bit goes; a row refined again keeps this run's bit
    // (its stale check above only reads `now`), the grid's other blocks read
    // only rows of the previous list, each owned by one (i) here
    atomicAnd(a.mark + prev[i], ~old);
  }
  for (long long i = t0; i < c; i += stride) keep[i] = a.list[i];
  if (reset) atomicAdd(a.ctl + 2, reset);
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(a.ctl + 1, 1u) == gridDim.x - 1) {     // last block of the grid
      __threadfence();
      const unsigned rs = atomicAdd(a.ctl + 2, 0u);
      a.count_store[p] = (int32_t)c;
      *a.total += (unsigned long long)c;
      if (a.info) {
        a.info[0] = c;
        a.info[1] = a.write_rows ? ((long long)rs + c) * a.nb * 16 : a.full_bytes;
      }
      a.ctl[2] = 0;
      a.ctl[1] = 0;
      __threadfence();
      a.ctl[0] = q;                                    // the next run's parity
    }
  }
}

// The lowest `cols` bins (as 8-byte complex values) of `rows` data rows read
// straight from pinned, mapped host memory by the device: many 8- or 16-byte
// reads in flight at once, where a strided copy would move the 16 short rows
// one after another.  VEC = 2: 16-byte accesses (src 16-byte aligned).
template <int VEC>
static __global__ void band_gather_kernel(float2 *dst, long long dst_row, const float2 *src,
                                          long long src_row, int cols, int rows) {
  using V = typename std::conditional<VEC == 2, float4, float2>::type;
  const int cv = cols / VEC;
  const long long total = (long long)rows * cv;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / cv), c = (int)(i - (long long)r * cv);
    reinterpret_cast<V *>(dst + r * dst_row)[c] = reinterpret_cast<const V *>(src + r * src_row)[c];
  }
}

inline int hier_host_grid(long long max_elems, int sms) {
  long long blocks = (max_elems + 255) / 256;
  if (blocks > 2ll * sms) blocks = 2ll * sms;
  return blocks < 1 ? 1 : (int)blocks;
}

static __global__ void reference_sum_kernel(const float *p, int n, int m, double *out) {
  double low = 0.0, total = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const double x = (double)p[k];
    total += x;
    if (k < m) low += x;
  }
  __shared__ double sl[32], st[32];
  for (int o = 16; o; o >>= 1) {
    low += __shfl_xor_sync(0xffffffffu, low, o);
    total += __shfl_xor_sync(0xffffffffu, total, o);
  }
  if ((threadIdx.x & 31) == 0) { sl[threadIdx.x >> 5] = low; st[threadIdx.x >> 5] = total; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double L = 0.0, S = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) { L += sl[w]; S += st[w]; }
    out[0] = L;
    out[1] = S;
  }
}

// FP64 in-band and total sums of a host reference profile, on the device
// (src/hmf.c:125-136).  Synchronous; returns a cudaError_t value.
inline int reference_fraction_fp64(const float *power_host, size_t n, size_t m, double *low,
                                   double *total, cudaStream_t s) {
  float *dp = nullptr;
  double *dout = nullptr;
  cudaError_t e = cudaMalloc(&dp, n * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&dout, 2 * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyAsync(dp, power_host, n * sizeof(float), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) { reference_sum_kernel<<<1, 1024, 0, s>>>(dp, (int)n, (int)m, dout); e = cudaGetLastError(); }
  double h[2] = {0, 0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, dout, sizeof h, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(dp);
  cudaFree(dout);
  *low = h[0];
  *total = h[1];
  return (int)e;
}

// ---- tensor-core coarse pass (coarse_tc.cu) --------------------------------
struct TcCoarse;
struct TcRunArgs {
  const float2 *data;   // full-length data rows [nd_total][n]; the first m bins are used
  const float2 *ct;     // coarse templates [nt_total][m]
  int n;
  int d0, nd, t0, nt;
  int ws, we;           // coarse window [ws, we) on the m-point grid
  float gate;
  long long *out_idx;   // full-size outputs: rows of dismissed pairs get (-1, 0)
  float2 *out_val;
  int rs;               // record stride of out_idx/out_val in 8-byte units (1 or 2)
  int full_nb;
  int32_t *fire_list, *fire_count;
  float *coarse_out;    // if set: write max |z| per pair here instead of gating
};
int tc_coarse_create(TcCoarse **out, int m, int ntmpl, int ndata, int fp16);
void tc_coarse_destroy(TcCoarse *c);
int tc_coarse_pack_templates(TcCoarse *c, const float2 *ct, int t0, int count, cudaStream_t s);
int tc_coarse_run(TcCoarse *c, const TcRunArgs &a, cudaStream_t s);
// Rows mode of the same pass: max |z|^2 of the 512-point inverse DFT of each
// of `nrows` already-formed rows (stride 512), row r being column r % n2 of a
// band of 512 * n2 points whose lags n2 * j + (r % n2) are kept in [cs, ce).
int tc_coarse_rows(TcCoarse *c, const float2 *rows, long long nrows, int n2, int cs, int ce,
                   float *m2_out, cudaStream_t s);
const char *tc_coarse_error();
// 0, or -1 if a run timed out waiting for the tensor cores (synchronous).
int tc_coarse_check(TcCoarse *c);

}  // namespace mfb
