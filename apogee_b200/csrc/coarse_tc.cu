// Tensor-core coarse pass of the hierarchical filter (tcgen05, sm_100a).
//
// The coarse value of a pair is max_j |z_c[j]| over the coarse window, where
// z_c[j] = sum_{f<m} D[f] conj(ct[f]) exp(+2 pi i f j / m) is the m-point
// inverse DFT of the band-limited conjugate product (src/hmf.c:241-251: the
// reference runs the flat filter at length m).  Here the m = 512 point DFT is
// factored m = 16 x 32 (f = 32 f1 + f2, j = j1 + 16 j2):
//
//   stage 1  Y[j1, f2] = sum_f1 W16^(f1 j1) P[32 f1 + f2]          (GEMM)
//   twiddle  Y'[j1, f2] = Y[j1, f2] W512^(f2 j1)                      (CUDA cores)
//   stage 2  Z[j1 + 16 j2] = sum_f2 W32^(f2 j2) Y'[j1, f2]           (GEMM)
//
// Both stages are real GEMMs on the 5th-generation tensor cores: complex
// values are realified (re, im interleaved along K), and every operand is
// split into hi + lo halves of BF16 (or FP16) with the products
// hi*hi + hi*lo + lo*hi accumulated in FP32 in tensor memory, which keeps
// about 16 significant bits (BF16) of the FP32 inputs.  Pairs are batched
// along M: stage 1 rows are (pair, f2) -- 4 pairs per 128-row tile -- and
// stage 2 rows are (pair, j1) -- 8 pairs per tile.
//
// Per item (8 pairs): the conjugate product and its split are written by the
// CUDA cores as the stage-1 A operand (K-major, no swizzle); one thread
// issues 12 MMAs (M128 N32 K16) into TMEM; the accumulators come back with
// tcgen05.ld, are twiddled, split and written transposed as the stage-2 A
// operand (K-major, 128-byte swizzle, so a warp's 32 stores to one row hit 32
// different banks); 12 more MMAs (M128 N64 K16); then |z|^2 over the window,
// max over the pair's 16 rows, and the gate of src/hmf.c:264-300.  The three
// steps run in separate warp roles on consecutive items (see
// coarse_tc_ws_kernel).  The DFT matrices (B operands) and the 512-point
// twiddles are built once on the host in FP64 and copied into shared memory
// at kernel start.
//
// Every wait on an mbarrier is bounded; on timeout the kernel records an
// error flag, stops issuing work, releases its tensor memory and returns.
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cmath>
#include <climits>
#include <cstring>
#include <vector>
#include "hier_kernels.cuh"

namespace mfb {

namespace tc {
constexpr int BAND = 512;
constexpr int PAIRS = 8;          // pairs per item; producer warp w works on pair w
// constant operands at the start of shared memory (1024-byte aligned base)
constexpr int OFF_B2 = 0;         // 2 splits x 8 KB, 128B swizzle (64 rows x 128 B)
constexpr int OFF_B1 = 16384;     // 2 splits x 2 k-steps x 1 KB, no swizzle
constexpr int OFF_TW = 20480;     // 512 float2 twiddles W512^(f2 j1), [j1][f2]
constexpr int CONST_BYTES = 24576;
constexpr unsigned SPIN_LIMIT = 1u << 22;

__host__ __device__ constexpr uint32_t idesc(int n, int fp16) {
  // kind::f16 instruction descriptor: D = F32, A = B = BF16 (or F16), both
  // K-major, N >> 3 at bit 17, M >> 4 at bit 24 (M = 128).
  return (1u << 4) | ((fp16 ? 0u : 1u) << 7) | ((fp16 ? 0u : 1u) << 10) |
         ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo, uint32_t layout) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) | ((uint64_t)layout << 61);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mma(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :: "r"(dtmem), "l"(a), "l"(b), "r"(id), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :: "r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
  for (unsigned i = 0; i < SPIN_LIMIT; i++) {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}\n" : "=r"(ok) : "r"(bar), "r"(phase) : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

#define MFB_TMEM_LD32(taddr, r)                                                                    \
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "                                            \
               "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"                             \
               "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"            \
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),          \
                 "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),        \
                 "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]),    \
                 "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),    \
                 "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),    \
                 "=r"(r[30]), "=r"(r[31])                                                          \
               : "r"(taddr))

#define MFB_TMEM_LD16(taddr, r)                                                                    \
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "                                            \
               "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"                     \
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),          \
                 "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),        \
                 "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])                                \
               : "r"(taddr))

__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// hi + lo split of x into two 16-bit floats, packed (re in the low half).
template <int FP16>
__device__ __forceinline__ void split2(float re, float im, uint32_t &hi, uint32_t &lo) {
  if constexpr (FP16) {
    const __half2 h = __floats2half2_rn(re, im);
    const float2 hf = __half22float2(h);
    const __half2 l = __floats2half2_rn(re - hf.x, im - hf.y);
    hi = *reinterpret_cast<const uint32_t *>(&h);
    lo = *reinterpret_cast<const uint32_t *>(&l);
  } else {
    // hi: the upper 16 bits of each FP32 (BF16 by truncation, one byte
    // permute for both); lo: the exact remainder, rounded to BF16 by one
    // packed conversion.  |lo| < 2^-7 |x|, so hi + lo carries ~16 bits.
    const uint32_t rb = __float_as_uint(re), ib = __float_as_uint(im);
    hi = __byte_perm(rb, ib, 0x7632);
    const float rr = re - __uint_as_float(rb & 0xFFFF0000u);
    const float ri = im - __uint_as_float(ib & 0xFFFF0000u);
    const __nv_bfloat162 l = __floats2bfloat162_rn(rr, ri);
    lo = *reinterpret_cast<const uint32_t *>(&l);
  }
}
}  // namespace tc

struct TcKernelArgs {
  const float2 *data;        // full-length rows, stride n; first BAND bins used
  long long data_stride;
  const float2 *ct;          // coarse templates [nt][BAND]
  const uint4 *consts;       // CONST_BYTES image: B2 | B1 | twiddles
  int d0, nd, t0, nt;
  int ws, we;
  float t2, gate;
  long long *out_idx;
  float2 *out_val;
  int rs, full_nb;
  int32_t *fire_list, *fire_count;
  float *coarse_out;
  int *err;
  // Rows mode (the band-16384 four-step): "pairs" are rows r of a scratch of
  // already-formed 512-point products (data = the scratch, nd = rows, nt = 1,
  // no template), row r is column k2 = r % rows_n2 of a longer band whose
  // lags are rows_n2 * j + k2; the window [cs, ce) is on that longer grid,
  // and coarse_out receives max |z|^2 of the row (no gate).
  int rows_n2, cs, ce;
};

// Warp-specialised form of the same pass: three roles in one 512-thread CTA
// (one per SM) work on consecutive items at once, handing operands over
// through NSLOT shared-memory and tensor-memory slots per stage:
//   warps 0-7   producers: warp w owns pair w of the item (lane = f2); the
//               conjugate product and split -> stage-1 A (slot k), inputs for
//               the next item already in flight; thread 0 issues the stage-1
//               MMAs into TMEM S1[k];
//   warps 8-11  stage-1 epilogue: quadrant q reads pairs q and 4 + q from
//               S1[k] -> twiddle, split, transposed store -> stage-2 A
//               (slot k); thread 256 issues the stage-2 MMAs into S2[k];
//   warps 12-15 stage-2 epilogue: S2[k] -> |z|^2 over the window, max per
//               pair with warp shuffles, gate.
// Hand-offs are mbarriers: full_s1[k] / full_s2[k] (MMA commits) and
// free_s1[k] / free_s2[k] (the epilogue warps have read the accumulators).
// A slot is reused every NSLOT items, so each wait is on the phase of the
// item NSLOT back and no role can run two phases ahead of a waiter.  Waits
// are bounded; a failed wait sets the error flag, every later wait returns
// at once and the roles run out their loops without issuing MMAs (no thread
// leaves a loop early, so the role barriers always fill).
namespace tcw {
constexpr int NSLOT = 2;
constexpr int THREADS = 512;
constexpr int TMEM_COLS = 256;                      // S1[2] x 64 + S2[2] x 64
constexpr int S2_COL = NSLOT * 64;
constexpr int SLOT = 32768;
constexpr int OFF_A2 = 24576;                       // NSLOT x 32 KB (2 splits x 16 KB, 128B swizzle)
constexpr int OFF_A1 = OFF_A2 + NSLOT * SLOT;       // NSLOT x 32 KB (2 tiles x 2 splits x 2 k-steps x 4 KB)
constexpr int OFF_BAR = OFF_A1 + NSLOT * SLOT;      // 4 NSLOT mbarriers, TMEM slot, abort flag
constexpr int SMEM_BYTES = OFF_BAR + 128 + 1024;
constexpr int B_FULL1 = 0, B_FULL2 = NSLOT, B_FREE1 = 2 * NSLOT, B_FREE2 = 3 * NSLOT;
}  // namespace tcw

__device__ __forceinline__ void role_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" :: "r"(id), "r"(nthreads) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(bar) : "memory");
}
// Bounded wait that gives up at once when another thread has given up.
__device__ __forceinline__ bool mbar_wait_ab(uint32_t bar, uint32_t phase, volatile int *abort_flag,
                                             int *err) {
  for (unsigned i = 0; i < tc::SPIN_LIMIT; i++) {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}\n" : "=r"(ok) : "r"(bar), "r"(phase) : "memory");
    if (ok) return true;
    if (*abort_flag) return false;
  }
  *err = 1;
  *abort_flag = 1;
  return false;
}

template <int FP16>
__global__ void __launch_bounds__(tcw::THREADS, 1)
coarse_tc_ws_kernel(const TcKernelArgs a) {
  using namespace tc;
  using tcw::NSLOT;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *sm = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t sbase = smem_u32(sm);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint64_t *bars = reinterpret_cast<uint64_t *>(sm + tcw::OFF_BAR);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + tcw::OFF_BAR + 8 * 4 * NSLOT);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(sm + tcw::OFF_BAR + 8 * 4 * NSLOT + 8);
  for (int i = tid; i < CONST_BYTES / 16; i += tcw::THREADS)
    reinterpret_cast<uint4 *>(sm)[i] = a.consts[i];
  if (tid == 0) {
    for (int i = 0; i < 4 * NSLOT; i++) {   // commits: 1 arrival; epilogue reads: 1 per warp (4)
      const int cnt = i < tcw::B_FREE1 ? 1 : 4;
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&bars[i])), "r"(cnt));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *abort_flag = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(tslot)), "r"(tcw::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_async_smem();
  tc_before_sync();
  __syncthreads();
  tc_after_sync();
  const uint32_t tmem = *tslot;
  const float2 *tw512 = reinterpret_cast<const float2 *>(sm + OFF_TW);
  const uint32_t id1 = idesc(32, FP16), id2 = idesc(64, FP16);
  const long long total = (long long)a.nd * a.nt;
  const long long items = (total + PAIRS - 1) / PAIRS;
  const long long per = items / gridDim.x, extra = items % gridDim.x;
  const long long ibeg = blockIdx.x * per + (blockIdx.x < extra ? blockIdx.x : extra);
  const int nit = (int)(per + (blockIdx.x < extra ? 1 : 0));
  auto bar = [&](int i) { return smem_u32(&bars[i]); };

  if (warp < 8) {
    // ---- producers: warp w owns pair w of the item, lane = f2 ----------------
    const int prow = 32 * (warp & 3) + lane, ptile = warp >> 2;
    float2 pd[16], ph[16];
    auto issue_loads = [&](int it) {
      const long long pi = (ibeg + it) * PAIRS + warp;
      if (it < nit && pi < total && a.rows_n2 > 0) {
        // rows mode: the product is already formed (times conj(1) below, exact)
        const float2 *dp = a.data + pi * (long long)a.data_stride;
#pragma unroll
        for (int f1 = 0; f1 < 16; f1++) { pd[f1] = __ldg(dp + 32 * f1 + lane); ph[f1] = make_float2(1.f, 0.f); }
      } else if (it < nit && pi < total) {
        const int d = (int)(pi / a.nt), t = (int)(pi - (long long)d * a.nt);
        const float2 *dp = a.data + (long long)(a.d0 + d) * a.data_stride;
        const float2 *hp = a.ct + (long long)(a.t0 + t) * BAND;
#pragma unroll
        for (int f1 = 0; f1 < 16; f1++) { pd[f1] = __ldg(dp + 32 * f1 + lane); ph[f1] = __ldg(hp + 32 * f1 + lane); }
      } else {
#pragma unroll
        for (int f1 = 0; f1 < 16; f1++) { pd[f1] = make_float2(0.f, 0.f); ph[f1] = make_float2(0.f, 0.f); }
      }
    };
    int last = -1;
    issue_loads(0);
    for (int it = 0; it < nit; it++) {
      const int k = it % NSLOT;
      const uint32_t u = (uint32_t)(it / NSLOT);
      if (it >= NSLOT) mbar_wait_ab(bar(tcw::B_FULL1 + k), (u - 1) & 1, abort_flag, a.err);  // A1[k] consumed
      uint8_t *a1 = sm + tcw::OFF_A1 + k * tcw::SLOT;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        uint32_t hh[4], ll[4];
#pragma unroll
        for (int v = 0; v < 4; v++) {
          const float2 x = pd[4 * q + v], h = ph[4 * q + v];
          split2<FP16>(fmaf(x.x, h.x, x.y * h.y), fmaf(x.y, h.x, -x.x * h.y), hh[v], ll[v]);
        }
        const int ks = q >> 1, cc = q & 1;
        const int off = (prow >> 3) * 256 + cc * 128 + (prow & 7) * 16;
        *reinterpret_cast<uint4 *>(a1 + ((ptile * 2 + 0) * 2 + ks) * 4096 + off) = make_uint4(hh[0], hh[1], hh[2], hh[3]);
        *reinterpret_cast<uint4 *>(a1 + ((ptile * 2 + 1) * 2 + ks) * 4096 + off) = make_uint4(ll[0], ll[1], ll[2], ll[3]);
      }
      issue_loads(it + 1);
      fence_async_smem();
      tc_before_sync();
      role_sync(1, 256);
      if (tid == 0) {
        bool ok = !*abort_flag;
        if (ok && it >= NSLOT)
          ok = mbar_wait_ab(bar(tcw::B_FREE1 + k), (u - 1) & 1, abort_flag, a.err);   // S1[k] read
        if (ok) {
          tc_after_sync();
          const uint32_t a1s = sbase + tcw::OFF_A1 + k * tcw::SLOT;
#pragma unroll
          for (int s = 0; s < 2; s++) {
            int first = 1;
#pragma unroll
            for (int c = 0; c < 3; c++) {
              const int ha = (c == 2) ? 1 : 0, hb = (c == 1) ? 1 : 0;
#pragma unroll
              for (int ks = 0; ks < 2; ks++) {
                const uint64_t ad = sdesc(a1s + ((s * 2 + ha) * 2 + ks) * 4096, 128, 256, 0);
                const uint64_t bd = sdesc(sbase + OFF_B1 + (hb * 2 + ks) * 1024, 128, 256, 0);
                mma(tmem + k * 64 + s * 32, ad, bd, id1, first ? 0u : 1u);
                first = 0;
              }
            }
          }
          commit(bar(tcw::B_FULL1 + k));
          last = it;
        }
      }
    }
    if (tid == 0 && last >= 0)   // own MMAs complete before the accumulators are freed
      mbar_wait(bar(tcw::B_FULL1 + last % NSLOT), (uint32_t)(last / NSLOT) & 1);
  } else if (warp < 12) {
    // ---- stage-1 epilogue: quadrant q, pairs q (tile 0) and 4 + q (tile 1), f2 = lane
    const int q = warp & 3, f2 = lane;
    float2 tw[16];                 // W512^(f2 j1), j1 = 0..15: the same for every item
#pragma unroll
    for (int j1 = 0; j1 < 16; j1++) tw[j1] = tw512[j1 * 32 + f2];
    int last = -1;
    for (int it = 0; it < nit; it++) {
      const int k = it % NSLOT;
      const uint32_t u = (uint32_t)(it / NSLOT);
      mbar_wait_ab(bar(tcw::B_FULL1 + k), u & 1, abort_flag, a.err);                       // S1[k] full
      tc_after_sync();
      uint32_t vv[16];
      if (it >= NSLOT) mbar_wait_ab(bar(tcw::B_FULL2 + k), (u - 1) & 1, abort_flag, a.err);  // A2[k] consumed
      uint8_t *a2 = sm + tcw::OFF_A2 + k * tcw::SLOT;
#pragma unroll
      for (int hh = 0; hh < 4; hh++) {
        // 16 accumulator columns (8 values j1 of one tile) at a time: few
        // registers live, so the compiler can overlap the elements' chains
        const int s = hh >> 1, p = 4 * s + q;
        MFB_TMEM_LD16(tmem + ((uint32_t)(32 * q) << 16) + k * 64 + 16 * hh, vv);
        tmem_wait_ld();
        if (hh == 3) {   // both tiles read: S1[k] is free
          tc_before_sync();
          if (lane == 0) mbar_arrive(bar(tcw::B_FREE1 + k));
        }
#pragma unroll
        for (int jj = 0; jj < 8; jj++) {
          const int j1 = 8 * (hh & 1) + jj;
          const float yr = __uint_as_float(vv[2 * jj]), yi = __uint_as_float(vv[2 * jj + 1]);
          const float2 w = tw[j1];
          const float zr = fmaf(yr, w.x, -yi * w.y), zi = fmaf(yr, w.y, yi * w.x);
          uint32_t hi, lo;
          split2<FP16>(zr, zi, hi, lo);
          const int R = p * 16 + j1;
          const int off = (R >> 3) * 1024 + (R & 7) * 128 + (((f2 >> 2) ^ (R & 7)) << 4) + (f2 & 3) * 4;
          *reinterpret_cast<uint32_t *>(a2 + off) = hi;
          *reinterpret_cast<uint32_t *>(a2 + 16384 + off) = lo;
        }
      }
      fence_async_smem();
      tc_before_sync();
      role_sync(2, 128);
      if (tid == 256) {
        bool ok = !*abort_flag;
        if (ok && it >= NSLOT)
          ok = mbar_wait_ab(bar(tcw::B_FREE2 + k), (u - 1) & 1, abort_flag, a.err);   // S2[k] read
        if (ok) {
          tc_after_sync();
          const uint32_t a2s = sbase + tcw::OFF_A2 + k * tcw::SLOT;
          int first = 1;
#pragma unroll
          for (int c = 0; c < 3; c++) {
            const int ha = (c == 2) ? 1 : 0, hb = (c == 1) ? 1 : 0;
#pragma unroll
            for (int ks = 0; ks < 4; ks++) {
              const uint64_t ad = sdesc(a2s + ha * 16384 + ks * 32, 16, 1024, 2);
              const uint64_t bd = sdesc(sbase + OFF_B2 + hb * 8192 + ks * 32, 16, 1024, 2);
              mma(tmem + tcw::S2_COL + k * 64, ad, bd, id2, first ? 0u : 1u);
              first = 0;
            }
          }
          commit(bar(tcw::B_FULL2 + k));
          last = it;
        }
      }
    }
    if (tid == 256 && last >= 0)
      mbar_wait(bar(tcw::B_FULL2 + last % NSLOT), (uint32_t)(last / NSLOT) & 1);
  } else {
    // ---- stage-2 epilogue: quadrant q, rows R = 32 q + lane = (pair R / 16, j1 = R % 16)
    const int q = warp & 3, R = 32 * q + lane, j1 = R & 15;
    for (int it = 0; it < nit; it++) {
      const int k = it % NSLOT;
      const uint32_t u = (uint32_t)(it / NSLOT);
      mbar_wait_ab(bar(tcw::B_FULL2 + k), u & 1, abort_flag, a.err);                       // S2[k] full
      tc_after_sync();
      int ws = a.ws, we = a.we;
      if (a.rows_n2 > 0) {
        // lags rows_n2 * j + k2 of the longer band inside [cs, ce)
        const long long pi = (ibeg + it) * PAIRS + (R >> 4);
        const int k2 = (int)(pi % a.rows_n2);
        ws = a.cs > k2 ? (a.cs - k2 + a.rows_n2 - 1) / a.rows_n2 : 0;
        we = a.ce > k2 ? (a.ce - k2 + a.rows_n2 - 1) / a.rows_n2 : 0;
      }
      float best = 0.f;
#pragma unroll
      for (int half = 0; half < 2; half++) {
        uint32_t v[32];
        MFB_TMEM_LD32(tmem + ((uint32_t)(32 * q) << 16) + tcw::S2_COL + k * 64 + 32 * half, v);
        tmem_wait_ld();
#pragma unroll
        for (int jj = 0; jj < 16; jj++) {
          const float zr = __uint_as_float(v[2 * jj]), zi = __uint_as_float(v[2 * jj + 1]);
          const int j = j1 + 16 * (16 * half + jj);
          const float m2 = fmaf(zr, zr, zi * zi);
          if (j >= ws && j < we && m2 > best) best = m2;
        }
      }
      tc_before_sync();
      if (lane == 0) mbar_arrive(bar(tcw::B_FREE2 + k));
#pragma unroll
      for (int o = 8; o; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, o));
      const int pr = R >> 4;
      const long long pi = (ibeg + it) * PAIRS + pr;
      if (pi < total && !*abort_flag) {
        const int row = (int)pi;
        if (a.rows_n2 > 0) {
          if ((lane & 15) == 0) a.coarse_out[pi] = best;
        } else if (a.coarse_out) {
          if ((lane & 15) == 0) a.coarse_out[row] = sqrtf(best);
        } else {
          const bool fire = best > a.t2 && sqrtf(best) >= a.gate;
          if (fire) {
            if ((lane & 15) == 0) a.fire_list[atomicAdd(a.fire_count, 1)] = row;
          } else {
            const long long obase = (long long)row * a.full_nb;
            for (int b = lane & 15; b < a.full_nb; b += 16) {
              a.out_idx[(obase + b) * a.rs] = -1;
              a.out_val[(obase + b) * a.rs] = make_float2(0.f, 0.f);
            }
          }
        }
      }
    }
  }
  tc_before_sync();
  __syncthreads();
  tc_after_sync();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(tcw::TMEM_COLS));
}

// ------------------------------------------------------------------- host side
struct TcCoarse {
  int m = 0, fp16 = 0, grid = 0, blocks_per_sm = 0;
  uint4 *consts = nullptr;
  int *err = nullptr;
};

static thread_local const char *g_tc_err = "";

static double dcos2pi(long long m, long long M) {   // cos(2 pi m / M), exact at quarter turns
  m %= M;
  if (m < 0) m += M;
  if ((4 * m) % M == 0) { const long long q = 4 * m / M; return q == 0 ? 1.0 : q == 2 ? -1.0 : 0.0; }
  return std::cos(2.0 * M_PI * (double)m / (double)M);
}
static double dsin2pi(long long m, long long M) { return dcos2pi(m - M / 4, M); }

template <int FP16>
static uint16_t to16(double x) {
  if (FP16) return __half_as_ushort(__float2half_rn((float)x));
  return __bfloat16_as_ushort(__float2bfloat16_rn((float)x));
}
template <int FP16>
static double from16(uint16_t u) {
  if (FP16) return (double)__half2float(__ushort_as_half(u));
  return (double)__bfloat162float(__ushort_as_bfloat16(u));
}

// Realified inverse-DFT matrix entry: output (j, co), input (f, ci) of an R-point DFT.
static double realified(int j, int co, int f, int ci, int R) {
  const double C = dcos2pi((long long)f * j, R), S = dsin2pi((long long)f * j, R);
  if (co == 0) return ci == 0 ? C : -S;
  return ci == 0 ? S : C;
}

template <int FP16>
static void build_consts(std::vector<uint8_t> &img) {
  using namespace tc;
  img.assign(CONST_BYTES, 0);
  auto put = [&](size_t off, uint16_t v) { memcpy(&img[off], &v, 2); };
  for (int h = 0; h < 2; h++) {
    // B2: 64 rows (n = 2 j2 + co) x 64 K (k = 2 f2 + ci), 128B swizzle
    for (int n = 0; n < 64; n++)
      for (int k = 0; k < 64; k++) {
        const double x = realified(n >> 1, n & 1, k >> 1, k & 1, 32);
        const uint16_t hi = to16<FP16>(x);
        const uint16_t v = h == 0 ? hi : to16<FP16>(x - from16<FP16>(hi));
        const int kb = 2 * k;
        const size_t off = OFF_B2 + h * 8192 + (n >> 3) * 1024 + (n & 7) * 128 +
                           (((kb >> 4) ^ (n & 7)) << 4) + (kb & 15);
        put(off, v);
      }
    // B1: 32 rows (n = 2 j1 + co) x 32 K (k = 2 f1 + ci), 2 k-steps, no swizzle
    for (int n = 0; n < 32; n++)
      for (int k = 0; k < 32; k++) {
        const double x = realified(n >> 1, n & 1, k >> 1, k & 1, 16);
        const uint16_t hi = to16<FP16>(x);
        const uint16_t v = h == 0 ? hi : to16<FP16>(x - from16<FP16>(hi));
        const int ks = k >> 4, kk = k & 15;
        const size_t off = OFF_B1 + (h * 2 + ks) * 1024 + (n >> 3) * 256 + (kk >> 3) * 128 +
                           (n & 7) * 16 + (kk & 7) * 2;
        put(off, v);
      }
  }
  // twiddles W512^(f2 j1) laid out [j1][f2], so a warp (f2 = lane) reads 32
  // consecutive entries
  for (int j1 = 0; j1 < 16; j1++)
    for (int f2 = 0; f2 < 32; f2++) {
      const float w[2] = {(float)dcos2pi((long long)f2 * j1, BAND), (float)dsin2pi((long long)f2 * j1, BAND)};
      memcpy(&img[OFF_TW + 8 * (j1 * 32 + f2)], w, 8);
    }
}

int tc_coarse_create(TcCoarse **out, int m, int ntmpl, int ndata, int fp16) {
  (void)ntmpl; (void)ndata;
  *out = nullptr;
  if (m != tc::BAND) { g_tc_err = "tensor-core coarse pass supports band 512"; return -1; }
  TcCoarse *c = new TcCoarse;
  c->m = m;
  c->fp16 = fp16;
  std::vector<uint8_t> img;
  if (fp16) build_consts<1>(img); else build_consts<0>(img);
  cudaError_t e = cudaMalloc(&c->consts, img.size());
  if (e == cudaSuccess) e = cudaMemcpy(c->consts, img.data(), img.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&c->err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(c->err, 0, sizeof(int));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(coarse_tc_ws_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, tcw::SMEM_BYTES);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(coarse_tc_ws_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, tcw::SMEM_BYTES);
  int dev = 0, sms = 0, smem_sm = 0;
  if (e == cudaSuccess) e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  if (e != cudaSuccess || smem_sm < tcw::SMEM_BYTES + 1024) {
    g_tc_err = e != cudaSuccess ? cudaGetErrorString(e) : "coarse kernel cannot be resident";
    tc_coarse_destroy(c);
    return -1;
  }
  // One 512-thread CTA per SM (all 128 registers x 512 threads; 256 TMEM columns).
  c->grid = sms;
  c->blocks_per_sm = 1;
  *out = c;
  return 0;
}

void tc_coarse_destroy(TcCoarse *c) {
  if (!c) return;
  cudaFree(c->consts);
  cudaFree(c->err);
  delete c;
}

int tc_coarse_pack_templates(TcCoarse *, const float2 *, int, int, cudaStream_t) { return 0; }

int tc_coarse_run(TcCoarse *c, const TcRunArgs &r, cudaStream_t s) {
  if (!c) { g_tc_err = "no tensor-core coarse state"; return -1; }
  TcKernelArgs a;
  memset(&a, 0, sizeof a);
  a.data = r.data;
  a.data_stride = r.n;
  a.ct = r.ct;
  a.consts = c->consts;
  a.d0 = r.d0; a.nd = r.nd; a.t0 = r.t0; a.nt = r.nt;
  a.ws = r.ws; a.we = r.we;
  a.t2 = r.gate > 0.f ? r.gate * r.gate : 0.f;
  a.gate = r.gate;
  a.out_idx = r.out_idx;
  a.out_val = r.out_val;
  a.rs = r.rs;
  a.full_nb = r.full_nb;
  a.fire_list = r.fire_list;
  a.fire_count = r.fire_count;
  a.coarse_out = r.coarse_out;
  a.err = c->err;
  if (c->fp16) coarse_tc_ws_kernel<1><<<c->grid, tcw::THREADS, tcw::SMEM_BYTES, s>>>(a);
  else coarse_tc_ws_kernel<0><<<c->grid, tcw::THREADS, tcw::SMEM_BYTES, s>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { g_tc_err = cudaGetErrorString(e); return -1; }
  return 0;
}

int tc_coarse_rows(TcCoarse *c, const float2 *rows, long long nrows, int n2, int cs, int ce,
                   float *m2_out, cudaStream_t s) {
  if (!c) { g_tc_err = "no tensor-core coarse state"; return -1; }
  if (nrows < 1 || nrows > INT_MAX || n2 < 1) { g_tc_err = "invalid row count"; return -1; }
  TcKernelArgs a;
  memset(&a, 0, sizeof a);
  a.data = rows;
  a.data_stride = tc::BAND;
  a.consts = c->consts;
  a.d0 = 0; a.nd = (int)nrows; a.t0 = 0; a.nt = 1;
  a.coarse_out = m2_out;
  a.err = c->err;
  a.rows_n2 = n2; a.cs = cs; a.ce = ce;
  if (c->fp16) coarse_tc_ws_kernel<1><<<c->grid, tcw::THREADS, tcw::SMEM_BYTES, s>>>(a);
  else coarse_tc_ws_kernel<0><<<c->grid, tcw::THREADS, tcw::SMEM_BYTES, s>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { g_tc_err = cudaGetErrorString(e); return -1; }
  return 0;
}

int tc_coarse_check(TcCoarse *c) {
  if (!c) return 0;
  int err = 0;
  if (cudaMemcpy(&err, c->err, sizeof err, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
  if (err) g_tc_err = "tensor-core coarse pass timed out waiting for the tensor cores";
  return err ? -1 : 0;
}

const char *tc_coarse_error() { return g_tc_err; }

}  // namespace mfb
