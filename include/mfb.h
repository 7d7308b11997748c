/* mfb.h -- C ABI of the B200 fused matched-filter library (libmfb.so).
 *
 * This is the drop-in seam for the device backends of the reference
 * (ahnitz/Apogee, package `matchedfilter`):
 *   - the transform backend vtable `ap_backend` (src/backend.h:6-55) and its
 *     plan wrapper `ap_plan` (src/dispatch.c:17-192), and
 *   - the GPU context duck-type `Context.peaks / hier_peaks / forward`
 *     (python/matchedfilter/_vkcompute.py:962,534,855),
 * behind the same filter-level contract as the reference C API
 * (python/matchedfilter/matchedfilter.h).  Plain C types only: pointers,
 * sizes and a CUDA stream passed as void*.
 *
 * Conventions (restated from the reference):
 *   - Correlation z[k] = sum_f D[f] conj(H[f]) exp(+2 pi i f k / n), unnormalised.
 *   - Bins: nb = ceil((end-start)/binsize) after clamping end to n; bin j covers
 *     lags [start + j*binsize, min(start + (j+1)*binsize, end)).
 *   - A bin reports the lag of max |z|^2 iff |z|^2 > threshold^2 (threshold <= 0
 *     means > 0); otherwise index -1 and value 0.  Exact ties: lowest lag.
 *   - Output rows: (d-d0)*nt + (t-t0), nb entries per row.
 *
 * Memory: spectra are copied into plan-owned device memory at ingest
 * (source may be host or device memory; cudaMemcpyDefault decides).  Output
 * pointers (idx, val, counts) are DEVICE pointers.  Runs are asynchronous on
 * the plan's stream; errors in arguments are reported before anything is
 * enqueued.
 *
 * Return values: 0 (MFB_OK) or a negative MFB_ERR_*; mfb_last_error() gives
 * the message for the calling thread.  A plan is not safe for concurrent use
 * from several threads (as src/matchfilt.c plans are not).
 */
#ifndef MFB_H
#define MFB_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define MFB_OK               0
#define MFB_ERR_ARG         -1   /* invalid argument or shape        -> ValueError   */
#define MFB_ERR_INDEX       -2   /* row index out of range           -> IndexError   */
#define MFB_ERR_CUDA        -3   /* CUDA runtime failure              -> RuntimeError */
#define MFB_ERR_UNSUPPORTED -4   /* transform length not implemented  -> ValueError   */
#define MFB_ERR_STATE       -5   /* plan not ready (e.g. no gate set) -> RuntimeError */

#define MFB_COARSE_FP32   0      /* coarse pass = flat FP32 filter at length band      */
#define MFB_COARSE_BF16X3 1      /* coarse pass = BF16 hi+lo tensor-core contraction    */
#define MFB_COARSE_FP16X3 2      /* coarse pass = FP16 hi+lo tensor-core contraction    */

typedef struct mfb_plan mfb_plan;
typedef struct mfb_hplan mfb_hplan;

/* ---- flat matched filter ------------------------------------------------ */

/* Replaces ap_mf_create (src/matchfilt.c:73-133; matchedfilter.h:53).  n is a
   power of two, 64 .. 2^20 (above 16384 the two-pass four-step); device is a
   CUDA ordinal.  *out = NULL on error. */
int mfb_create(mfb_plan **out, size_t n, int ndata, int ntmpl, int device);
/* Replaces ap_mf_destroy (src/matchfilt.c:135-146). */
int mfb_destroy(mfb_plan *p);
/* Stream for every later enqueue on this plan (a cudaStream_t, NULL = legacy). */
int mfb_set_stream(mfb_plan *p, void *stream);
/* Replaces ap_mf_set_data / ap_mf_set_template (src/matchfilt.c:179-215):
   copy `count` spectra of n complex64 (interleaved re,im) into rows d0.. / t0.. */
int mfb_set_data(mfb_plan *p, int d0, int count, const void *spec);
int mfb_set_templates(mfb_plan *p, int t0, int count, const void *spec);
/* Replaces ap_mf_run (src/matchfilt.c:411-420; matchedfilter.h:66-70).
   idx: int64 [nd*nt*nb]; val: complex64 [nd*nt*nb]; counts: int32 [nd*nt] or NULL.
   Returns 0, not the total of threshold crossings that ap_mf_run returns
   (matchedfilter.h:66-71): the run is only enqueued here, and the total would
   need a host synchronisation.  Sum `counts` after synchronising instead. */
int mfb_run(mfb_plan *p, int d0, int nd, int t0, int nt, size_t binsize, float threshold,
            size_t start, size_t end, int64_t *idx, void *val, int32_t *counts);
/* Same as mfb_run, but the output is one array of 16-byte records laid out
   as the reference's PEAK_DTYPE = [("index","<i8"),("value","<c8")]
   (python/matchedfilter/__init__.py:45), so a host copy of it IS the
   structured result (the assembly of __init__.py:155-173 happens on the
   device). records: DEVICE [nd*nt*nb] x 16 bytes. */
int mfb_run_records(mfb_plan *p, int d0, int nd, int t0, int nt, size_t binsize, float threshold,
                    size_t start, size_t end, void *records, int32_t *counts);
/* Kernel choice for n = 4096 (no counterpart in the reference, whose CPU
   engine picks its own code path per shape): on (the default), runs whose
   lag window is [0, n) with bins a multiple of 32 lags and at most 64 bins
   use the kernel that carries two pairs per thread in packed FP32x2
   arithmetic; off, they use the one-pair-per-thread kernel.  Both compute
   the same operations in the same order and give bit-identical results;
   the switch lets a caller compare or time the two. */
int mfb_set_packed(mfb_plan *p, int on);
/* Kernel choice for n = 32768 and 65536 (no counterpart in the reference,
   whose CPU engine always runs its four-step plan through memory): mode 0
   runs the two-pass kernels through the plan's L2-sized scratch; mode 1 runs
   each pair on one thread-block cluster whose distributed shared memory
   holds the whole spectrum between the two passes of the four-step split --
   8 (n = 32768) or 16 (n = 65536) CTAs of 256 threads, three CTAs per SM --
   in one launch with no scratch and no host decision (listed runs read their
   row count on the device, so a hierarchical run at these lengths is
   replayed as one CUDA graph); mode 2 the same with 4 / 8 CTAs of 512
   threads, one per SM.  Same arithmetic, identical results.  The default is
   the faster on a B200: mode 1 at n = 32768 (on a par with mode 0 on dense
   blocks, faster on short row lists), mode 0 at 65536 (mode 1 is 1.3x
   slower there). */
int mfb_set_cluster(mfb_plan *p, int mode);
/* Replaces ap_mf_run_sel (src/matchfilt.c:492-503) in list form: run only the
   output rows rows[0..*nrows) of the block [d0,d0+nd) x [t0,t0+nt), where a row
   is (d-d0)*nt + (t-t0) and the row count lives in DEVICE memory (nrows), so a
   survivor list made on the GPU needs no host round trip.  The caller keeps
   *nrows <= max_rows.  Every kernel reads the count on the device, except the
   two-pass kernels (n >= 65536, and n = 32768 in cluster mode 0), which size
   their batches on the host: there the call reads the count, synchronises the
   plan's stream and refuses a count above max_rows. */
int mfb_run_rows(mfb_plan *p, int d0, int nd, int t0, int nt, const int32_t *rows,
                 const int32_t *nrows, int max_rows, size_t binsize, float threshold,
                 size_t start, size_t end, int64_t *idx, void *val, int32_t *counts);
/* Replaces ap_mf_run_series (src/matchfilt.c:437-490; matchedfilter.h:98-103);
   returns 0, not the crossings total (see mfb_run).
   series: complex64 [nseries] (device or host); starts/win_start/win_end:
   host arrays of nblocks.  Every block's window must give the same bin count
   (MFB_ERR_ARG otherwise).  Block b's spectrum is FFT(series[start..start+n)/n),
   zero-padded past nseries.  Output [nblocks][nt][nb] in caller order.
   The plan's data rows are used as scratch: set_data again before run(). */
int mfb_run_series(mfb_plan *p, const void *series, size_t nseries, const uint64_t *starts,
                   const uint64_t *win_start, const uint64_t *win_end, int nblocks,
                   int t0, int nt, size_t binsize, float threshold,
                   int64_t *idx, void *val, int32_t *counts);
/* Forward spectra of blocks, FFT(series[start..start+n)/n) zero-padded past
   nseries, into spectra [nblocks][n] (DEVICE).  Replaces the GPU forward
   stage Context.forward (python/matchedfilter/_vkcompute.py:855-906). */
int mfb_forward(mfb_plan *p, const void *series, size_t nseries, const uint64_t *starts_dev,
                int nblocks, void *spectra);
/* Replaces ap_mf_nbins / ap_nbins (src/dispatch.c:62-67). */
size_t mfb_nbins(size_t n, size_t binsize, size_t start, size_t end);
/* Message of the last error on this thread ("" if none). */
const char *mfb_last_error(void);
/* 1 if n is a supported transform length (replaces ap_supported, matchedfilter.h:208). */
int mfb_supported(size_t n);

/* ---- hierarchical matched filter ----------------------------------------- */

/* Replaces ap_hmf_create_ex (src/hmf.c:33-70): full plan at n plus a coarse
   pass over the lowest `band` bins (band a power of two, 64 <= band < n). */
int mfb_hier_create(mfb_hplan **out, size_t n, int ndata, int ntmpl, size_t band,
                    int coarse_kind, int device);
int mfb_hier_destroy(mfb_hplan *p);
/* mfb_set_packed for the plan's refine (and its flat filter). */
int mfb_hier_set_packed(mfb_hplan *p, int on);
/* mfb_set_cluster for the plan's refine. */
int mfb_hier_set_cluster(mfb_hplan *p, int mode);
int mfb_hier_set_stream(mfb_hplan *p, void *stream);
/* Replaces ap_hmf_set_data / ap_hmf_set_template (src/hmf.c:139-156).  The
   template's band fraction is summed in FP64 on the device. */
int mfb_hier_set_data(mfb_hplan *p, int d0, int count, const void *spec);
int mfb_hier_set_templates(mfb_hplan *p, int t0, int count, const void *spec);
/* Replaces ap_hmf_set_reference (src/hmf.c:125-138): power is HOST float32[n]
   or NULL (use each template's own band fraction).  FP64 sums on the device. */
int mfb_hier_set_reference(mfb_hplan *p, const float *power);
/* Replaces ap_hmf_set_threshold (src/hmf.c:107-110): finite; negative marks
   the plan unconfigured and runs then fail with MFB_ERR_STATE. */
int mfb_hier_set_threshold(mfb_hplan *p, float coarse_threshold);
/* Replaces ap_hmf_run (src/hmf.c:222-328): coarse pass, gate, and a refine of
   the survivors with the flat kernel, all enqueued on the stream with no host
   decision in between.  Same arguments and output as mfb_run; returns 0,
   not the crossings total of ap_hmf_run (see mfb_run). */
int mfb_hier_run(mfb_hplan *p, int d0, int nd, int t0, int nt, size_t binsize, float threshold,
                 size_t start, size_t end, int64_t *idx, void *val, int32_t *counts);
/* mfb_hier_run with PEAK_DTYPE record output, as mfb_run_records. */
int mfb_hier_run_records(mfb_hplan *p, int d0, int nd, int t0, int nt, size_t binsize,
                         float threshold, size_t start, size_t end, void *records,
                         int32_t *counts);
/* mfb_hier_run_records whose table lands in the caller's HOST memory.
   records: DEVICE workspace of nd*nt*nb 16-byte records (16-byte aligned),
   left holding the table as mfb_hier_run_records writes it.  table: pinned,
   mapped host memory (cudaHostAlloc / cudaMallocHost / cudaHostRegister) of
   nd*nt*nb records, written by the device on the plan's stream.  Every row
   the gate dismisses is all empty records (index -1, value 0), so when
   `table` is the one this plan wrote last with the same nd*nt and nb, only
   the rows that change cross the host link: the rows refined now are
   written, and the rows refined last time but not now are reset to empty.
   Any other table is copied whole.  The caller must not write into the table between calls.
   info: pinned host int64[2] or NULL; receives the refined rows and the
   bytes written into the table.  data: NULL, or all ndata data spectra
   (ndata x n complex64) in host memory, copied into the plan's data rows
   first -- the lowest band bins of every row ahead of the coarse pass, the
   rest on a second stream while the coarse pass runs -- so the memory must
   stay unchanged until the run has completed (pinned memory makes both
   copies asynchronous).  Read table and info after synchronising the
   stream.  The plan's trigger total is updated as by mfb_hier_run.
   Same contract as ap_hmf_run (src/hmf.c:222-328) for the table itself. */
int mfb_hier_run_host(mfb_hplan *p, int d0, int nd, int t0, int nt, size_t binsize,
                      float threshold, size_t start, size_t end, const void *data,
                      void *records, void *table, int64_t *info);
/* mfb_hier_run split for measurement: phase 1 enqueues only the coarse pass
   and gate (dismissed rows written, survivor list built), phase 2 only the
   refine of the list phase 1 built; phase 0 is the whole run.  Lets a caller
   time the two kernels of one run separately with events between them. */
int mfb_hier_run_phase(mfb_hplan *p, int phase, int d0, int nd, int t0, int nt, size_t binsize,
                       float threshold, size_t start, size_t end, int64_t *idx, void *val,
                       int32_t *counts);
/* Survivors of the last mfb_hier_run (synchronises the plan's stream). */
int mfb_hier_last_triggers(mfb_hplan *p, int64_t *triggers);
/* Replaces ap_hmf_run_series (src/hmf.c:158-220): runs of blocks with equal
   windows, at most ndata at a time, are forward-transformed on the device
   into the plan's data rows (FFT(block/n), zero past nseries) and run through
   mfb_hier_run.  Arguments and output as mfb_run_series; the plan's data rows
   are scratch afterwards. */
int mfb_hier_run_series(mfb_hplan *p, const void *series, size_t nseries, const uint64_t *starts,
                        const uint64_t *win_start, const uint64_t *win_end, int nblocks,
                        int t0, int nt, size_t binsize, float threshold,
                        int64_t *idx, void *val, int32_t *counts);
/* Replaces ap_hmf_stats (src/hmf.c:84-103): pairs and triggers since creation
   (synchronises the plan's stream).  Triggers are summed on the device, so
   runs need no host round trip and can be captured in a CUDA graph. */
int mfb_hier_stats(mfb_hplan *p, int64_t *pairs, int64_t *triggers);
/* Replaces ap_hmf_config (src/hmf.c:104-106). */
int mfb_hier_config(mfb_hplan *p, size_t *band, int *coarse_kind);
/* Coarse maxima only (gate calibration, diagnostics, the precision study):
   for every pair of the block, the maximum |coarse z| over the coarse
   window, float32 [nd*nt] DEVICE (0 where every coarse sample is 0).  Uses
   the plan's coarse kind. */
int mfb_hier_coarse_values(mfb_hplan *p, int d0, int nd, int t0, int nt, size_t start,
                           size_t end, float *out);

/* ---- batched uneven jobs --------------------------------------------------- */

/* One job of a batch: a (data or series, templates) block of any supported n,
   its own binsize, threshold and lag window (the same for every row). */
typedef struct mfb_job {
  size_t n;                 /* power of two, 64 ... 2^20 */
  int nd, nt;               /* data rows (series blocks) and templates */
  const void *data;         /* DEVICE complex64 [nd][n] spectra; NULL for a series job */
  const void *templates;    /* DEVICE complex64 [nt][n] */
  const void *series;       /* series job: DEVICE complex64 [nseries] samples, else NULL */
  size_t nseries;
  const uint64_t *starts;   /* series job: HOST [nd] block starts; block b is
                               series[starts[b] .. starts[b]+n), zero past the end,
                               transformed as FFT(x/n) (src/matchfilt.c:454-470) */
  size_t binsize;
  float threshold;
  size_t start, end;        /* lag window, clamped to [0, n] */
  void *records;            /* DEVICE output [nd][nt][nb] 16-byte records in PEAK_DTYPE
                               layout {int64 index; complex64 value}, 16-byte aligned */
  int split;                /* n >= 8192: N2 of the four-step split n = N1*N2, one of
                               64, 128, 256 (0 = 256 for n >= 16384, else 128) */
  int unit_items;           /* n <= 4096: items (of 4096/n pairs) per ticket (0 = 1) */
} mfb_job;

typedef struct mfb_batch_opts {
  size_t slot_bytes;        /* two-pass scratch per slot (0 = 64 MiB) */
  int slots;                /* scratch slots, 2 ... 64 (0 = 3) */
} mfb_batch_opts;

typedef struct mfb_batch mfb_batch;

/* No single counterpart: the reference runs one plan per shape
   (ap_mf_create / ap_mf_run, src/matchfilt.c:73-147,411-420; run_series,
   src/matchfilt.c:437-490).  Plans a batch of jobs for ONE persistent launch:
   validates every job, builds the twiddle tables, the segment table and the
   scratch slots (allocates; do it before any capture).  Outputs are the
   callers' `records`; inputs stay the callers' and must outlive the batch. */
int mfb_batch_create(mfb_batch **out, int device, const mfb_job *jobs, int njobs,
                     const mfb_batch_opts *opts);
/* Clears the counters and the two-pass outputs and launches the persistent
   kernel on `stream`.  No allocation, no host synchronisation: capturable
   in a CUDA graph and replayable. */
int mfb_batch_run(mfb_batch *b, void *stream);
/* Synchronises `stream`; MFB_ERR_CUDA if a dependency wait inside the last
   run ran out (the results of that run are then not valid). */
int mfb_batch_status(mfb_batch *b, void *stream);
/* Failure-detection test hook: adds delta (+1 or -1) to the pass-A unit
   count that pass B of the first four-step batch waits for.  With +1 that
   count is never reached: the next run's bounded dependency wait runs out
   (a few seconds), the launch stops taking tickets and returns, and
   mfb_batch_status reports MFB_ERR_CUDA; -1 restores the plan.  No GPU
   fault, trap or hang is involved.  MFB_ERR_STATE if the batch has no
   four-step pass.  Synchronous. */
int mfb_batch_test_wait_limit(mfb_batch *b, int delta);
/* Tickets, grid, segments, scratch batches and scratch bytes of the plan. */
int mfb_batch_info(mfb_batch *b, int64_t *tickets, int *grid, int *segments, int *batches,
                   size_t *scratch_bytes);
int mfb_batch_destroy(mfb_batch *b);

/* ---- adjoint --------------------------------------------------------------- */

/* No counterpart in the reference (it has no gradients).  Adjoint of the peak
   values at their fixed lags: with k = idx[d][t][b] (skipped when < 0) and g =
   gz[d][t][b] the upstream gradient of the complex peak value in torch's
   convention (dL/dRe z + i dL/dIm z),
     grad_data[d][f] = sum_t sum_b g       * templates[t][f] * exp(-2 pi i f k / n)
     grad_tmpl[t][f] = sum_d sum_b conj(g) * data[d][f]      * exp(+2 pi i f k / n)
   data [nd][n], templates [nt][n], gz, grad_*: complex64; idx int64
   [nd][nt][nb]; all DEVICE pointers of `device`.  Either gradient may be NULL;
   each given one is overwritten.  FP32 arithmetic with FP64-built twiddles.
   Queued on `stream` (NULL = default); the first call for an n builds its
   twiddle tables (allocates, synchronises). */
int mfb_adjoint(int device, size_t n, const void *data, int nd, const void *templates, int nt,
                size_t nb, const int64_t *idx, const void *gz, void *grad_data, void *grad_tmpl,
                void *stream);

/* ---- large transforms with no allocation --------------------------------- */

/* Size of the file-scope device array that mfb_run_large_static uses as its
   scratch: 8 MiB per device, reserved when the library's device code loads on
   that device.  With CUDA's lazy module loading (the default) that load, and
   so the reservation, happens at the first kernel launch of any mfb_* entry
   point on the device -- which is the first mfb_run_large_static call itself
   when nothing else has run there -- and the kernels a call launches may be
   loaded (their code placed in device memory) at their own first launch.
   Make one earlier call on the device, or set CUDA_MODULE_LOADING=EAGER, if
   even that first reservation must happen before a given point. */
#define MFB_STATIC_SCRATCH_BYTES (8u << 20)

/* No counterpart in the reference.  The two-pass filter of mfb_run for
   power-of-two n = 32768 ... 524288 with no plan and no allocation of any
   kind, for callers that cannot let a library allocate device memory (their
   own pool owns HBM, or the device-wide synchronisation of cudaMalloc/cudaFree
   would stall their other streams).
   data [nd][n], templates [nt][n]: complex64 rows in DEVICE memory of `device`.
   idx int64 / val complex64 [nd][nt][nb] DEVICE outputs with
   nb = mfb_nbins(n, binsize, start, end) <= 4096; counts int32 [nd*nt] or
   NULL.  Results, threshold and window mean what they mean for mfb_run.  Work
   is queued on `stream` (a cudaStream_t of `device`; NULL = default stream).
   Limit: one pair needs n*8 bytes of rows plus nb*16 bytes of records
   (rounded up to 256); that must fit MFB_STATIC_SCRATCH_BYTES, so n = 1048576
   is refused with MFB_ERR_UNSUPPORTED and a message giving the bytes needed.
   Pairs run in as many batches as the scratch needs.
   Zeroing: the records must be zero when each batch's second pass starts;
   the call clears them on `stream` itself, and clears counts, so nothing the
   caller passes has to start at zero and nothing carries over between calls.
   Set-up: the first call on a device takes the scratch's device address
   (cudaGetSymbolAddress, with that device current), uploads the twiddles and
   sets the kernel attributes, synchronously; make that first call before any
   stream capture.
   Races: the scratch is one per device, so calls on one device that overlap
   in time (two streams without an ordering between them, or two host
   threads) overwrite each other's scratch and return wrong results; order
   them on one stream or with events. */
int mfb_run_large_static(int device, size_t n, const void *data, int nd, const void *templates,
                         int nt, size_t binsize, float threshold, size_t start, size_t end,
                         int64_t *idx, void *val, int32_t *counts, void *stream);

/* ---- coarse-gate model ------------------------------------------------------ */

/* Replaces the numerics of the reference's gate model joint_maxima
   (python/matchedfilter/gatemodel.py:63-140) on the device: FP64 profile sums,
   lag covariances of the full and in-band profile and their Cholesky factors,
   then the FP32 noise transforms and the coarse / fine maxima of every draw.
   HOST arguments: power [n] (FP64); step = n/band sub-grid offsets; taus [step][16]
   (the offset's lags, ntaus[step] of them, ascending); on_grid [step][9] (the
   coarse grid lags' positions in taus); draw_in / draw_out complex64
   [step][per][16] (the model's standard normal draws / sqrt 2, zero past
   ntaus; draw_out ignored unless has_out).  Outputs HOST coarse, fine
   [step][per] and sums_out[2] = (sum power, sum of the lowest band bins). */
int mfb_gate_maxima(int device, const double *power, size_t n, size_t band, float snr, int step,
                    int per, int has_out, const int32_t *taus, const int32_t *ntaus,
                    const int32_t *on_grid, const void *draw_in, const void *draw_out,
                    float *coarse, float *fine, double *sums_out);

/* ---- measurement --------------------------------------------------------- */

/* Measured FP32 FMA throughput of `device` in FLOP/s (2 per FMA), from a
   register-resident FMA loop over every SM, timed with CUDA events.  The
   roofline denominator for the FP32 kernels. */
int mfb_fp32_peak(int device, double *flops_per_s);

#ifdef __cplusplus
}
#endif
#endif
