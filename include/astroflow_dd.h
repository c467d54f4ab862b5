/* astroflow_dd.h — C ABI of the B200 dedispersion library (libastroflow_dd.so).
 *
 * This is the drop-in boundary for astroflow's dedispersion hot path: every
 * entry point takes plain pointers, sizes and PODs, returns a status code and
 * never exits the process.  It replaces, for the Python pipeline, the compute
 * that the reference binds through pybind11 in src/bindpy:
 *
 *   _astroflow_core._dedisperse_spec      -> dd_plan_create + dd_run[_host]
 *       (src/bindpy/bindings.cpp:43-57, src/bindpy/pyapi.cpp:284-309,
 *        src/core/dedispered.cu:988-1304 gpucal::dedisperse_spec<T>)
 *   _astroflow_core._dedispered_fil       -> dd_plan_create(freq_mode = DD_FREQ_FIL,
 *        algorithm = DD_ALGO_SUBBAND for target 1 / DD_ALGO_BRUTE for target 0)
 *       (src/bindpy/bindings.cpp:25-29, src/bindpy/pyapi.cpp:6-51,
 *        src/core/dedispered.cu:483-986, include/cpucal.hpp:75-201)
 *
 * and the stage functions the reference keeps in src/core and src/rfi
 * (include/iqrmcuda.h, include/rfimarker.h), whose results are exposed for
 * parity checks through dd_run_ex.
 *
 * Pointers passed to dd_run / dd_run_ex are device pointers on the plan's
 * device; dd_run_host takes host pointers (pinned or pageable) and stages the
 * copies on the given stream.  `stream` is a cudaStream_t (NULL = the legacy
 * default stream).  All functions are thread-compatible: one plan must not be
 * used by two threads at once; different plans are independent.
 */
#ifndef ASTROFLOW_DD_H
#define ASTROFLOW_DD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DD_ABI_VERSION 2

/* Status codes.  DD_ERR_INVALID corresponds to the reference's
 * std::invalid_argument (Python ValueError), e.g. a frequency range outside
 * the band (dedispered.cu:1009-1027); the others to std::runtime_error
 * (Python RuntimeError).  The reference exits the process on CUDA errors
 * (dedispered.cu:76-84); this library returns DD_ERR_CUDA instead. */
enum dd_status {
  DD_OK = 0,
  DD_ERR_INVALID = 1,
  DD_ERR_RUNTIME = 2,
  DD_ERR_CUDA = 3,
  DD_ERR_NOMEM = 4,
  DD_ERR_TIMEOUT = 5,
  DD_ERR_UNSUPPORTED = 6
};

/* Filterbank header: the fields of the reference's Header (include/data.h:24-50)
 * and Filterbank (include/filterbank.h:66-88).  The _dedisperse_spec path's
 * Header holds float fields; callers pass those floats widened to double (an
 * exact conversion) and the library rounds them back to float wherever the
 * reference computes in float (freq_mode DD_FREQ_HEADER).  The filename path
 * (DD_FREQ_FIL) uses them as the double values the SIGPROC reader produces. */
typedef struct dd_header {
  double mjd;
  double tsamp;    /* seconds */
  double fch1;     /* MHz, lowest channel (data are in ascending frequency order) */
  double foff;     /* MHz, > 0 */
  int32_t nbits;   /* 8, 16 or 32 */
  int32_t nchans;
  int64_t ndata;   /* time samples */
} dd_header;

/* IQRM parameters, the reference's iqrmconfig (include/rfi.h:12-39). */
typedef struct dd_iqrm_config {
  int32_t mode;        /* 0 = per-channel mean, 1 = per-channel standard deviation */
  float radius_frac;
  float nsigma;
  double geofactor;
  double win_sec;      /* 0 = one window over the whole chunk */
  double hop_sec;
  int32_t include_tail;
} dd_iqrm_config;

/* RFI stage switches, the reference's rficonfig (include/rfi.h:41-57). */
typedef struct dd_rfi_config {
  int32_t use_mask;     /* zero the channels listed in the mask file */
  int32_t use_zero_dm;  /* zero-DM filter */
  int32_t use_iqrm;     /* IQRM channel masking */
  dd_iqrm_config iqrm;
} dd_rfi_config;

enum dd_algorithm {
  DD_ALGO_SUBBAND = 0, /* two-stage subband sums of the reference GPU path (dedispered.cu:416-476) */
  DD_ALGO_BRUTE = 1    /* direct sums with the CPU path's semantics (cpucal.hpp:75-201) */
};

enum dd_zero_dm_mode {
  /* The filter as the reference calls it (dedispered.cu:1107): the 4-argument
   * call resolves to zero_dm_filter(T*, num_channels, num_samples, alpha), so it
   * is a no-op when chan_start == 0 and otherwise filters the first
   * chan_start*chan_end elements as [chan_end][chan_start] with
   * alpha = down_ndata (rfimarker.cu:130-169). */
  DD_ZDM_CALLSITE = 0,
  /* The range filter the call site intends (rfimarker.cu:257-305): per sample,
   * subtract the mean of the non-zero values of [chan_start, chan_end) from
   * those channels and clip at zero, with the mean taken exactly
   * (v -> max(0, v - ceil(sum/count))). */
  DD_ZDM_RANGE = 1,
  /* The same range filter in the arithmetic of the reference's range kernels
   * (rfimarker.cu:172-305): per sample a float sum of the non-zero values in
   * the kernels' order (256 threads, channel-strided partial sums, pairwise
   * tree), the mean by the fast-math float divide, then
   * v -> trunc(max(0, float(v) - mean)).  Equal to DD_ZDM_RANGE while the float
   * sums are exact and the quotient rounds the same way; it differs where the
   * sums pass 2^24 (16-bit samples over thousands of channels). */
  DD_ZDM_RANGE_REF = 2
};

enum dd_table_mode {
  /* Delay tables with the reference path's own arithmetic: for the subband
   * algorithm the single-precision device expressions of dedispered.cu:318-335
   * and 385-413 evaluated on the GPU with the same fast-math flags; for the
   * brute-force algorithm the float expression of cpucal.hpp:124-131 compiled
   * with the reference's host flags (-Ofast, FMA, AVX2), which reproduces the
   * reference build's table on the same host CPU (its vector reciprocal is
   * CPU-dependent at rounding ties). */
  DD_TABLE_REFERENCE = 0,
  /* round(4148.808*DM*(f^-2 - fref^-2)/tsamp) evaluated in FP64 on the host. */
  DD_TABLE_FP64 = 1,
  /* Brute force only: the float expression of cpucal.hpp:124-131 in strict
   * IEEE single precision (no contraction, exact reciprocals); host-independent,
   * and a few entries per ten thousand away from the reference build at ties. */
  DD_TABLE_IEEE = 2
};

enum dd_freq_mode {
  DD_FREQ_HEADER = 0, /* freq[i] = fch1 + i*foff in float (dedispered.cu:1004-1005) */
  DD_FREQ_FIL = 1     /* freq[i] = fch1 + i*foff in double (filterbank.cpp:445-449) */
};

typedef struct dd_plan_params {
  float dm_low;
  float dm_high;
  float dm_step;
  float freq_start;          /* MHz, >= lowest channel frequency */
  float freq_end;            /* MHz, <= highest channel frequency */
  int32_t time_downsample;   /* >= 1 */
  float t_sample;            /* seconds per slice of the brute-force path (cpucal.hpp:141) */
  int32_t algorithm;         /* dd_algorithm */
  int32_t subband_width;     /* channels per subband (AF_SUBBAND_SIZE_CH, default 32) */
  int32_t ndm0;              /* fine DMs per nominal DM (AF_SUBBAND_NDM0, default 32) */
  int32_t zero_dm_mode;      /* dd_zero_dm_mode */
  int32_t table_mode;        /* dd_table_mode */
  int32_t freq_mode;         /* dd_freq_mode */
  const double* freq_table;  /* optional [nchans] channel frequencies (DD_FREQ_FIL; a
                                SIGPROC file's own table, filterbank.cpp:376-383), or NULL */
} dd_plan_params;

typedef struct dd_plan_info {
  int64_t chan_start;        /* first channel of the band */
  int64_t chan_end;          /* last channel (inclusive for subband, exclusive for brute force) */
  int64_t dm_steps;          /* DM trials = output rows */
  int64_t nsamp_in;          /* input time samples */
  int64_t nsamp_binned;      /* samples after time binning (subband) */
  int64_t out_cols;          /* output columns per DM row */
  int64_t out_elem_bytes;    /* 4 (uint32) or 8 (uint64 for 32-bit input) */
  int64_t nsb;               /* subbands (subband algorithm) */
  int64_t ndm_nom;           /* nominal DMs (subband algorithm) */
  int64_t max_delay;         /* largest stage-1 or brute-force delay, samples */
  int64_t max_residual;      /* largest stage-2 shift, samples */
  int64_t nslices;           /* brute force: slices of t_sample */
  int64_t n_iqrm_windows;    /* IQRM windows (0 when IQRM is off) */
  int64_t workspace_bytes;   /* device workspace the plan holds */
  int64_t delay_rows;        /* rows of the delay table (ndm_nom or dm_steps) */
  int64_t delay_cols;        /* columns of the delay table (channels) */
  int64_t table_mismatch_fp64; /* delay entries where the table differs from the FP64 table */
  int64_t tile_samples;      /* time samples per stage-1/stage-2 launch (subband) */
  double adds_per_run;       /* algorithmic integer additions per dd_run */
  int64_t subband_sum_copies; /* copies of each stage-1 sum in device memory: 2 when stage 1
                                 also writes the one-sample-shifted twin stage 2 reads, else 1 */
} dd_plan_info;

typedef struct dd_plan dd_plan;

/* Build a plan: validates the arguments with the reference's rules (band
 * edges, channel range, DM count, dedispered.cu:1003-1031 / cpucal.hpp:85-116),
 * builds the delay tables, and reserves the device workspace on `device`
 * (the reference's target_id, dedispered.cu:997-1001).  bad_channels is the
 * list the reference reads from its mask file (rfimarker.cu:441-467); it may
 * be NULL when n_bad == 0. */
int dd_plan_create(const dd_header* header, const dd_plan_params* params,
                   const dd_rfi_config* rfi, const int32_t* bad_channels, int32_t n_bad,
                   int32_t device, dd_plan** plan);
int dd_plan_destroy(dd_plan* plan);
/* Destroy a plan without a device-wide synchronisation: its device memory is
 * released stream-ordered on `stream`, so every use of the plan must have been
 * issued on `stream` (or be complete).  For servers that retire plans while
 * other requests run (dd_plan_destroy waits for the whole device first, as
 * cudaFree does). */
int dd_plan_destroy_async(dd_plan* plan, void* stream);
int dd_plan_get_info(const dd_plan* plan, dd_plan_info* info);

/* Copy the plan's delay tables to host memory: delay is [delay_rows][delay_cols]
 * int32; residual is [dm_steps][nsb] int32 (subband only, may be NULL). */
int dd_plan_get_tables(const dd_plan* plan, int32_t* delay, int32_t* residual);

/* The brute-force delay table of the reference's CPU path (cpucal.hpp:119-132)
 * without a plan or a GPU: table[m][c - chan_start] for DM trial m of
 * dm_low + m*dm_step (m < dm_steps) and channel c of [chan_start, chan_end), with
 * freq[] the channel frequencies (ascending) and the reference frequency
 * freq[ref_channel] taken as float.  mode: DD_TABLE_REFERENCE, DD_TABLE_IEEE or
 * DD_TABLE_FP64 as above.  *mismatch_fp64 (may be NULL) receives the number of
 * entries that differ from the FP64 evaluation.  Host memory only. */
int dd_brute_delay_table(const double* freq, int64_t chan_start, int64_t chan_end,
                         int64_t ref_channel, float dm_low, float dm_step, int64_t dm_steps,
                         double tsamp, int32_t mode, int32_t* table, int64_t* mismatch_fp64);

/* Replace the brute-force delay table ([dm_steps][delay_cols] int32, host). */
int dd_plan_set_delay_table(dd_plan* plan, const int32_t* delay);

/* Dedisperse one chunk.  input: [nsamp_in][nchans] samples of header.nbits
 * (device).  output: [dm_steps][out_cols] uint32 (uint64 for 32-bit input),
 * device.  Brute force writes the slices of t_sample back to back: slice s
 * occupies columns [s*cols0, s*cols0 + cols_s) of every row. */
int dd_run(dd_plan* plan, const void* input, void* output, void* stream);

/* dd_run with the intermediate results exposed for parity checks (device
 * pointers, each may be NULL): iqrm_masks [n_iqrm_windows][nchans] uint8 and
 * iqrm_bounds [n_iqrm_windows][2] uint32 (t0, t1) as in iqrm_omp::WindowMask
 * (include/iqrm.hpp:162-166); prepped [nsamp_binned][nchans] samples after
 * binning and all RFI stages, the input the dedispersion sums read. */
int dd_run_ex(dd_plan* plan, const void* input, void* output, uint8_t* iqrm_masks,
              uint32_t* iqrm_bounds, void* prepped, void* stream);

/* dd_run from host memory: copies input in, runs, copies the output back and
 * synchronises the stream.  Host buffers may be pageable or pinned (pinned
 * buffers let the output of each time tile travel while the next tile is
 * summed).  The device-side input and output buffers are kept by the plan for
 * later calls and released with it. */
int dd_run_host(dd_plan* plan, const void* h_input, void* h_output, void* stream);

/* dd_run_host without waiting: queues the input copy, the run and the output
 * copies and returns.  It has no counterpart in the reference (whose call,
 * dedispered.cu:988-1304, blocks until its output is on the host); it serves
 * callers that stream chunk after chunk: one chunk's output copy (device to
 * host) overlaps the next chunk's input copy (host to device) and RFI stages,
 * and each time tile's sums of the next chunk wait only for the copy of the
 * output columns they overwrite.  h_input may be reused once the call's input copy is done (the
 * stream reaches it), h_output holds the result once dd_run_host_join has made
 * a stream wait for it and that stream has reached that point; pinned host
 * buffers are needed for the copies to overlap.  The calls of one plan must use
 * one stream. */
int dd_run_host_async(dd_plan* plan, const void* h_input, void* h_output, void* stream);

/* Makes `stream` wait (without blocking the host) for every output copy the
 * plan's dd_run_host_async calls have queued; with sync != 0 it also
 * synchronises the stream and reports a device-side failure of those runs
 * (a bounded wait that gave up) as dd_run_host does. */
int dd_run_host_join(dd_plan* plan, void* stream, int32_t sync);

/* Device-time breakdown of one run, measured with CUDA events on the run's
 * stream (the role of the reference's AF_DEBUG stage timers,
 * dedispered.cu:41-73, without their device-wide synchronisations). */
typedef struct dd_run_stats {
  float total_ms;          /* the whole run */
  float prep_ms;           /* binning, RFI stages and layout */
  float stage1_ms;         /* subband stage 1, all time tiles */
  float stage2_ms;         /* subband stage 2 or brute-force sums, all time tiles */
  int32_t launches;        /* kernels this library launched */
  int32_t stage1_launches;
  int32_t stage2_launches;
} dd_run_stats;

/* Autotuner of the subband path's launch shape.  Results do not depend on it:
 * the time tiling and the staging depth only change how the same sums are
 * scheduled.  dd_plan_autotune times dd_run of `plan` on the caller's chunk
 * (device `input`, `output` overwritten) for each candidate pair of subband-sum
 * budget per time tile (0.5, 1, 2 and 4 GiB, candidates giving the same tile
 * length skipped) and staged source pairs in flight (4, 6, 8, and as many as
 * fit; at most what leaves two blocks per SM), `reps` timed runs each after one
 * warm-up, keeps the fastest and reports it.  Candidates whose buffers do not
 * fit in device memory are skipped.  Synchronises the stream.  Batches built
 * from the plan earlier pick the new shape up at their next run. */
typedef struct dd_tune_report {
  int64_t candidates;       /* shapes timed */
  int64_t best_budget_bytes;
  int64_t best_tile_samples;
  int32_t best_stages;      /* 0: as many as fit */
  int32_t pad;
  double best_ms;           /* mean dd_run time of the chosen shape */
  double default_ms;        /* mean dd_run time of the shape the plan was built with */
} dd_tune_report;
int dd_plan_autotune(dd_plan* plan, const void* input, void* output, int32_t reps, void* stream,
                     dd_tune_report* report);

/* Kernels this library has launched from the calling thread (monotonic). */
int dd_launch_count(int64_t* count);

/* dd_run that also fills `stats`; synchronises the stream before returning. */
int dd_run_profiled(dd_plan* plan, const void* input, void* output, void* stream,
                    dd_run_stats* stats);

/* Measures this GPU's sustained 32-bit integer addition rate (additions per
 * second, a three-input add counted as two) with a register-resident kernel;
 * the denominator of the add-bound roofline of the dedispersion sums. */
int dd_measure_int_add_rate(int32_t device, double* adds_per_second);

/* IQRM channel masks of one chunk computed without allocating any device
 * memory.  It has no counterpart in the reference (whose IQRM, iqrm.cu:203-345,
 * allocates and frees device buffers on every call); it serves callers that
 * cannot allocate while they run, such as real-time pipelines whose deadlines
 * forbid cudaMalloc/cudaFree (both may synchronise the device) and host
 * frameworks that have already reserved the GPU's memory for their own pools.
 *
 * input: device [nsamp][nchans] samples of nbits (the chunk as the IQRM stage
 * sees it, after any time binning); channels [chan_start, chan_end) are
 * examined (chan_end exclusive, as the reference's IQRM takes it); tsamp is the
 * sampling time of `input` in seconds.  Outputs (device, caller-owned): masks
 * [max_windows][nchans] uint8 and bounds [max_windows][2] uint32 (t0, t1), the
 * same values dd_run_ex reports; *n_windows (host) receives the window count.
 * Runs on the calling thread's current device, on `stream`.
 *
 * All working memory comes from an 8 MiB array that the library keeps in a
 * GPU's memory from the first call on that GPU until the process exits;
 * requests whose working set exceeds it, and bands wider than the per-window
 * sort's shared memory holds, fail with DD_ERR_INVALID.  The first call on a
 * device resolves the array's address with that device current: make it before
 * any stream capture.  The library's device code loads lazily, so that first
 * call is also when the array takes its 8 MiB: a host that reserves most of the
 * GPU's memory for its own pools should make one small call before reserving
 * it.  Do not call it again on a device after cudaDeviceReset.  Calls share the
 * array, so calls whose GPU work overlaps race with each other and must be
 * serialised by the caller. */
int dd_iqrm_masks_noalloc(const void* input, int32_t nbits, int64_t nsamp, int32_t nchans,
                          int32_t chan_start, int32_t chan_end, double tsamp,
                          const dd_iqrm_config* cfg, uint8_t* masks, uint32_t* bounds,
                          int32_t max_windows, int32_t* n_windows, void* stream);

/* ---- Single-DM dedispersed spectrum of a time window (candidate plots):
 * cpucal::dedisperse_spec_with_dm (include/cpucal.hpp:341-483) with
 * freq_mode DD_FREQ_HEADER, cpucal::dedispered_fil_with_dm (cpucal.hpp:203-339)
 * with DD_FREQ_FIL.  Channels [chan_start, chan_start + nchans) selected by the
 * reference's linear frequency map; out[t][c] = x[t_start + t + delay(c)][chan_start + c],
 * delay(c) = lround(4148.808*dm*(1/f_c^2 - 1/f_high^2)/tsamp) in float.  IQRM and
 * the mask file (rfi->use_iqrm, rfi->use_mask) run first on the rows
 * [rfi_t0, rfi_t0 + rfi_len) as the reference does; the reference zeroes those
 * rows of the caller's array, here they are left untouched and, when
 * masked_rows is not NULL, written there instead ([rfi_len][nchans]). */
typedef struct dd_single_dm_params {
  float tstart;              /* seconds from the chunk's first sample */
  float tend;
  float dm;
  float freq_start;          /* MHz */
  float freq_end;
  int32_t freq_mode;         /* dd_freq_mode: Header (float) or Filterbank (double) arithmetic */
  const double* freq_table;  /* DD_FREQ_FIL: the file's channel frequencies, or NULL */
} dd_single_dm_params;
typedef struct dd_single_dm_info {
  int64_t t_start;           /* input sample of output row 0 */
  int64_t ntimes;            /* output rows */
  int64_t chan_start;        /* first selected channel */
  int64_t nchans;            /* selected channels = output columns */
  int64_t rfi_t0;            /* first input row of the RFI slice */
  int64_t rfi_len;           /* rows of the RFI slice */
  float tend;                /* tstart + ntimes * tsamp */
  float freq_start;          /* lowest selected frequency */
  float freq_end;            /* highest selected frequency */
  int32_t pad;
} dd_single_dm_info;
/* Host-only: validate and report the output geometry. */
int dd_single_dm_geometry(const dd_header* header, const dd_single_dm_params* params,
                          dd_single_dm_info* info);
/* input: device [ndata][nchans]; output: device [ntimes][nchans (selected)]. */
int dd_single_dm_run(const dd_header* header, const dd_single_dm_params* params,
                     const dd_rfi_config* rfi, const int32_t* bad_channels, int32_t n_bad,
                     const void* input, void* output, void* masked_rows, void* stream);

/* ---- DM-time images: the image step of the reference's GPU path
 * (preprocess_typed_dedisperseddata_with_slicing, include/data.h:620-727) and of
 * its CPU path (preprocess_dedisperseddata, data.h:299-369), on the GPU.  Each
 * slice (columns [col_start[i], col_start[i] + col_count[i]) of every row) is
 * converted to float, resized to target x target (INTER_AREA when both of its
 * dimensions exceed target, else INTER_LANCZOS4, with OpenCV's float rounding),
 * min-max normalised to uint8 and colored through lut_bgr (256 BGR triples, e.g.
 * OpenCV's COLORMAP_VIRIDIS of a gray ramp).  dm_time: device [nrows][row_pitch]
 * of uint32 (elem_bytes 4) or uint64 (8).  Outputs (device, either may be NULL
 * but not both): images [nslices][target][target][3] uint8 (B, G, R) and
 * resized [nslices][target][target] float.  col_start, col_count and lut_bgr are
 * host arrays.  target <= 1024. */
int dd_images(const void* dm_time, int32_t elem_bytes, int64_t nrows, int64_t row_pitch,
              int32_t nslices, const int64_t* col_start, const int64_t* col_count,
              int32_t target, const uint8_t* lut_bgr, uint8_t* images, float* resized,
              void* stream);

/* ---- Ingest: data into device memory in the plans' layout ([time][channel],
 * ascending frequency), through pinned staging blocks that worker threads fill
 * while earlier blocks are copied and transformed on the device.
 *
 * dd_fil_read_header parses a SIGPROC header as the reference's Filterbank does
 * (src/data/filterbank.cpp:319-452: keywords, FREQUENCY_START/fchannel tables,
 * sample count from the file size) and reports it after the reference's channel
 * flip (filterbank.cpp:793-842: foff < 0 -> ascending order, fch1 = lowest
 * frequency, foff = |foff|; a file with a frequency table keeps fch1 = foff = 0);
 * freq_table (optional, cap entries) receives the frequency table in that order.
 * dd_fil_read streams samples [t0, t0 + nsamp) of a single-IF file into
 * device_out ([nsamp][nchans], nbits/8 bytes per sample), flipping the channel
 * order on the device when the file's foff < 0.  dd_ingest_host does the same
 * from a host array [nsamp][npol][nchans]: npol 1 copies (DD_INGEST_FLIP
 * reverses the channels), npol >= 2 averages polarisations 0 and 1 as the
 * reference's PSRFITS reader does (python/astroflow/io/psrfits.py:44-51:
 * ((a + b) / 2).astype(dtype), the sum wrapping in the sample type, the
 * halving truncating toward zero; DD_INGEST_SIGNED for signed samples), then
 * flips if asked.  Both return when the copies are done; work queued on
 * `stream` afterwards sees the data. */
typedef struct dd_fil_header {
  double tsamp, fch1, foff, tstart;
  int64_t ndata;          /* samples in the file */
  int64_t header_bytes;
  int32_t nbits, nchans, nifs;
  int32_t flipped;        /* the file's channels run downwards; reads reverse them */
  int32_t has_freq_table;
  int32_t pad;
} dd_fil_header;
#define DD_INGEST_FLIP 1
#define DD_INGEST_SIGNED 2
int dd_fil_read_header(const char* path, dd_fil_header* out, double* freq_table, int32_t cap);
int dd_fil_read(const char* path, int64_t t0, int64_t nsamp, void* device_out, void* stream);
int dd_ingest_host(const void* host, int64_t nsamp, int32_t npol, int32_t nchans,
                   int32_t elem_bytes, int32_t flags, void* device_out, void* stream);

/* ---- Batches: many chunks of different geometries dedispersed together.
 * The reference dedisperses one chunk per call (gpucal::dedisperse_spec,
 * src/core/dedispered.cu:988-1304).  A batch runs one chunk through each of its
 * plans: each plan's binning/RFI/layout kernels, then the dedispersion sums of
 * all plans batched, either as one launch per (time tile, stage, kernel
 * variant) over that stage of every plan (default), or with DD_BATCH_PERSISTENT
 * as a single persistent launch over all of them whose blocks are handed out in
 * order and whose dependent stages wait (bounded) on completion counters.
 * Results equal dd_run of each plan on its chunk.  With DD_BATCH_GRAPH the run
 * is captured into a CUDA graph on the batch's own stream and replayed while
 * the same buffers are passed; new buffers (or a plan whose tables were
 * replaced) cause one new capture.  Plans must stay alive and unused elsewhere
 * while the batch runs.  Plans whose sums cannot be batched (32-bit samples,
 * delay spreads wider than the staged windows) run their own kernels inside the
 * same run. */
#define DD_BATCH_GRAPH 1
#define DD_BATCH_PERSISTENT 2
typedef struct dd_batch dd_batch;
typedef struct dd_batch_info {
  int64_t nplans;
  int64_t groups;          /* batched staged sums */
  int64_t blocks;          /* blocks of all batched sum launches */
  int64_t sum_launches;    /* batched sum launches per run */
  int64_t launches;        /* kernels one run launches (all of them) */
  int64_t own_plans;       /* plans that run their own kernels */
  int32_t graph;           /* runs replay a captured CUDA graph */
  int32_t persistent;      /* sums in one persistent launch */
  int32_t graph_captures;  /* graphs captured so far */
  int32_t pad;
} dd_batch_info;
/* flags: DD_BATCH_GRAPH | DD_BATCH_PERSISTENT. */
int dd_batch_create(dd_plan* const* plans, int32_t nplans, int32_t flags, dd_batch** batch);
/* inputs[i], outputs[i]: device buffers of plan i as for dd_run.  Asynchronous
 * with respect to the host; ordered after earlier work on `stream`, and later
 * work on `stream` is ordered after it. */
int dd_batch_run(dd_batch* batch, const void* const* inputs, void* const* outputs, void* stream);
/* Waits for the batch's work and reports a bounded device wait that gave up. */
int dd_batch_status(dd_batch* batch);
int dd_batch_get_info(const dd_batch* batch, dd_batch_info* info);
int dd_batch_destroy(dd_batch* batch);

/* ---- Streams: a beam dedispersed chunk by chunk (no reference counterpart:
 * the reference treats every call's chunk as standalone and drops the terms
 * with t + delay >= N, dedispered.cu:444 and 473).  A stream keeps the beam's
 * last `tail_samples` input samples on the device, tail = the plan's largest
 * total delay (stage-1 delay plus stage-2 shift) in input samples, and runs each
 * push as the plain subband call (all RFI stages included) on [tail | chunk],
 * returning its first chunk/time_downsample output columns, the columns whose
 * delayed samples all lie in the buffer.  Push k's column t is the beam's
 * binned time (samples pushed before push k - tail)/time_downsample + t; the
 * first pushes read a zero-filled tail.  header.ndata is the chunk length (a
 * multiple of time_downsample); params must select DD_ALGO_SUBBAND.  Pushes of
 * one stream must be ordered (one CUDA stream, or serialised). */
typedef struct dd_stream dd_stream;
typedef struct dd_stream_info {
  int64_t dm_steps;        /* output rows */
  int64_t out_cols;        /* output columns per push */
  int64_t chunk_samples;   /* input samples per push */
  int64_t tail_samples;    /* input samples kept between pushes */
  int64_t pushed_samples;  /* input samples pushed so far */
  int64_t workspace_bytes; /* device memory the stream holds */
  double adds_per_push;    /* algorithmic integer additions per push */
} dd_stream_info;
int dd_stream_open(const dd_header* header, const dd_plan_params* params,
                   const dd_rfi_config* rfi, const int32_t* bad_channels, int32_t n_bad,
                   int32_t device, dd_stream** stream_out);
/* chunk: device [chunk_samples][nchans]; output: device [dm_steps][out_cols]. */
int dd_stream_push(dd_stream* s, const void* chunk, void* output, void* stream);
int dd_stream_get_info(const dd_stream* s, dd_stream_info* info);
/* The plan a stream runs (owned by the stream): its info and tables. */
int dd_stream_plan(const dd_stream* s, dd_plan** plan);
int dd_stream_close(dd_stream* s);

/* Last error message of the calling thread ("" if none). */
const char* dd_last_error(void);
int dd_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* ASTROFLOW_DD_H */
