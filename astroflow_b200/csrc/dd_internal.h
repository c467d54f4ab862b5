// Internal declarations of the B200 dedispersion library (not part of the ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/astroflow_dd.h"

namespace dd {

// ---------------------------------------------------------------- errors
void set_error(const std::string& msg);
struct Error {
  int code;
  std::string msg;
};
#define DD_CUDA_TRY(call)                                                          \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess)                                                         \
      throw ::dd::Error{DD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
  } while (0)

// Kernel launches made by this library on the calling thread (monotonic).
long long& launch_count();
#define DD_COUNT_LAUNCH() (++::dd::launch_count())
// After a kernel launch: count it and surface launch errors.
#define DD_LAUNCHED()                           \
  do {                                          \
    DD_COUNT_LAUNCH();                          \
    DD_CUDA_TRY(cudaGetLastError());            \
  } while (0)

// ---------------------------------------------------------------- device buffer
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void alloc(size_t n);
  void release();
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

// Geometry of one IQRM segment: the samples [t0, t1) are covered by the same
// set of IQRM windows, whose masks are OR-ed into seg_mask[segment][nchans].
struct IqrmSeg {
  uint32_t t0, t1;
};

}  // namespace dd

struct dd_plan {
  dd_header hdr{};
  dd_plan_params p{};
  dd_rfi_config rfi{};
  int device = 0;
  int nbits = 8;
  int elem = 1;  // bytes per input sample

  std::vector<double> freq;  // channel frequencies (ascending)
  int64_t cs = 0, ce = 0;    // band: [cs, ce] subband, [cs, ce) brute force
  int64_t dm_steps = 0;
  int64_t nin = 0;           // input samples
  int64_t nbin = 0;          // binned samples (subband) / input samples (brute)
  int64_t nout = 0;          // subband: output columns (nbin, or fewer for a stream's plan)
  float ref_freq = 0.f;
  double tsamp = 0;          // sampling time as the reference path uses it

  // subband geometry
  int64_t dch = 0, nsb = 0, ndm_nom = 0;
  int sbw = 32, ndm0 = 32;
  int max_delay = 0, max_res = 0;
  int inter16 = 0;           // stage-1 sums stored as uint16 (8-bit input, narrow subbands)
  int twin = 0;              // stage 1 also writes the one-sample-shifted twin of its uint16 sums
  int64_t tile = 0;          // time tile of the stage-1 -> stage-2 pipeline
  int64_t tile_pitch = 0;    // row pitch of the inter tile (elements)
  int64_t xpitch = 0;        // row pitch of the channel-major prepared input (elements)
  int win1 = 0, win2 = 0;    // staged window bytes of the shared-memory sums (0: not used)

  // brute-force geometry (CPU path semantics)
  int64_t nc = 0;            // channels summed, [cs, ce)
  int64_t sps = 0;           // samples per slice
  int64_t nslices = 0;
  int64_t cols0 = 0;         // columns of a full slice
  std::vector<int64_t> slice_cols;
  int64_t out_cols = 0;
  int64_t phase_len = 0;     // padded length of one phase row of the brute-force layout
  bool phases_merge = true;  // slices share one phase pattern (sps % ds == 0)
  int winb = 0;              // staged window bytes of the brute-force sums (0: not used)

  // tables (host copies)
  std::vector<int32_t> h_delay;  // [ndm_nom][dch] (subband) or [dm_steps][nc] (brute)
  std::vector<int32_t> h_res;    // [dm_steps][nsb]
  int64_t table_mismatch_fp64 = 0;

  // IQRM
  std::vector<uint32_t> win_t0, win_t1;
  std::vector<int32_t> lags;
  std::vector<dd::IqrmSeg> segs;
  int iqrm_variant = 0;
  std::vector<int32_t> bad;

  // device state
  dd::DevBuf d_delay, d_res, d_lags, d_bad_keep, d_win, d_seg_t0;
  dd::DevBuf d_binned;   // binned / working copy of the input [nbin][nchans]
  dd::DevBuf d_x;        // prepared channel-major input
  dd::DevBuf d_host_in, d_host_out;  // device side of dd_run_host (kept across calls)
  cudaStream_t copy_stream = nullptr; // dd_run_host: output copies overlapping the sums
  cudaEvent_t host_done = nullptr;    // the last host-path output copy enqueued
  bool host_pending = false;          // host_done marks copies a later run must wait for
  std::vector<cudaEvent_t> host_tile_copied;  // per time tile: its output copy of the last run
  int64_t host_tile = 0;                      // the time tile those copies were made with
  dd::DevBuf d_inter;    // stage-1 tile (two buffers in a DD_PAIR_STAGES build)
  dd::DevBuf d_bin_lut;  // full-bin values of the time binning (8/16-bit samples, ds > 1)
  int64_t inter_bytes = 0; // bytes of one buffer
  int64_t inter_budget = 0; // subband-sum bytes per time tile the tiling was set for
  int stages_override = 0;  // staged source pairs in flight (0: as many as fit)
  dd::DevBuf d_stats;    // IQRM sums [nwin][2][csub] uint64
  dd::DevBuf d_iqrm_scratch;
  dd::DevBuf d_masks;    // IQRM window masks [nwin][nchans]
  dd::DevBuf d_segmask;  // [nseg][nchans]
  dd::DevBuf d_zdm;      // per-sample zero-DM offsets [nbin]
  dd::DevBuf d_desc1, d_desc2, d_descb;  // staging descriptors: stage 1, stage 2, brute force
  dd::DevBuf d_err;      // device error word of the staged sums (0: no error)
  double adds = 0;
  int64_t generation = 0;  // bumped whenever device tables are replaced
  std::vector<cudaEvent_t> events;  // timing events of dd_run_profiled
  ~dd_plan() {
    for (cudaEvent_t e : events) cudaEventDestroy(e);
    if (copy_stream) {
      cudaStreamSynchronize(copy_stream);
      cudaStreamDestroy(copy_stream);
    }
    if (host_done) cudaEventDestroy(host_done);
    for (cudaEvent_t e : host_tile_copied) cudaEventDestroy(e);
  }
};

namespace dd {

// ---- fast-math translation unit (dd_fastmath.cu) ----
void launch_subband_tables(const double* d_freq, int64_t cs, int64_t ce, float dm_low,
                           float dm_step, int64_t dm_steps, int sbw, int ndm0, float ref_freq,
                           double tsamp, int ds, int32_t* d_delay1, int32_t* d_res,
                           cudaStream_t st);
// mean_ws: device workspace of chan_end floats.
void launch_zero_dm_callsite(void* data, int nbits, size_t chan_start, size_t chan_end,
                             size_t down_ndata, float* mean_ws, cudaStream_t st);
// Per-sample float mean of the non-zero (after the IQRM segment masks) values of
// channels [cs, ce), in the arithmetic of the reference's range kernels.
void launch_zdm_range_mean(const void* x, int nbits, int64_t nsamp, int64_t nchans, int64_t cs,
                           int64_t ce, const uint8_t* d_segmask, const uint32_t* d_seg_t0,
                           int nseg, float* d_mean, cudaStream_t st);

// ---- RFI and layout (dd_rfi.cu) ----
// Time binning (dedispered.cu:337-376).  lut: the plan's table of full-bin values
// (launch_binning_lut; nullptr evaluates every bin directly).
void launch_time_binning(const void* in, void* out, int nbits, int64_t ndata, int64_t nchans,
                         int ds, const void* lut, cudaStream_t st);
// Entries of the full-bin table for these samples and bin width (0: no table).
int64_t binning_lut_entries(int nbits, int ds);
// Fills the full-bin table: lut[sum] for every sum of ds samples.
void launch_binning_lut(void* lut, int nbits, int ds, cudaStream_t st);
// d_win: [nwin][2] (t0, t1); d_sums: [nwin][2][csub] (sum, sum of squares).
void launch_iqrm_stats(const void* x, int nbits, int64_t nsamp, int64_t nchans, int64_t cs,
                       int64_t csub, const uint32_t* d_win, int nwin,
                       unsigned long long* d_sums, cudaStream_t st);
size_t iqrm_scratch_bytes(int nwin, int64_t csub, int nlags);
// Throws DD_ERR_INVALID when csub channels exceed what k_iqrm_decide's
// shared-memory sort holds on the current device.
void check_iqrm_channels(int64_t csub);
void launch_iqrm_decide(const unsigned long long* d_sums, int nwin, const uint32_t* d_win,
                        int64_t nchans, int64_t cs, int64_t csub, int mode, float nsigma,
                        const int32_t* d_lags, int nlags, int variant, void* scratch,
                        uint8_t* d_masks, cudaStream_t st);
void launch_segment_masks(const uint8_t* d_masks, int nwin, const uint32_t* d_win,
                          const uint32_t* d_seg_t0, int nseg, int64_t nchans,
                          uint8_t* d_segmask, cudaStream_t st);
void launch_apply_masks_inplace(void* x, int nbits, int64_t nsamp, int64_t nchans,
                                const uint8_t* d_segmask, const uint32_t* d_seg_t0, int nseg,
                                cudaStream_t st);
void launch_zdm_offsets(const void* x, int nbits, int64_t nsamp, int64_t nchans, int64_t cs,
                        int64_t ce_excl, const uint8_t* d_segmask, const uint32_t* d_seg_t0,
                        int nseg, uint32_t* d_off, cudaStream_t st);
struct PrepArgs {
  const void* x;           // [nsamp][nchans] input (binned)
  int nbits;
  int64_t nsamp, nchans;
  const uint8_t* segmask;  // nullptr: no IQRM masking in this pass
  const uint32_t* seg_t0;
  int nseg;
  const uint32_t* zdm_off; // nullptr: no zero-DM subtraction in this pass
  const float* zdm_mean;   // per-sample float mean (DD_ZDM_RANGE_REF), or nullptr
  int64_t zdm_cs, zdm_ce;  // channel range the zero-DM offset applies to
  const uint8_t* keep;     // nullptr: no static mask
  // channel-major output: out[(c - c0) * rows_per_chan + phase][q] with
  // q = t / ds, phase = t % ds (ds = 1 for the subband layout)
  void* out;
  int64_t c0, c1;          // channels [c0, c1)
  int ds;
  int64_t pitch;           // elements per output row
  void* full_out;          // optional [nsamp][nchans] copy after all stages
};
void launch_prep(const PrepArgs& a, cudaStream_t st);

// ---- dedispersion sums (dd_dedisp.cu) ----
struct Stage1Args {
  const void* x;           // channel-major input, row pitch xpitch (elements)
  int64_t xpitch;
  int nbits;
  const int32_t* delay1;   // [ndm_nom][dch]
  int64_t dch, nsb, ndm_nom;
  int sbw;
  int64_t t0;              // absolute start sample of the tile
  int64_t ncols;           // columns of inter to compute
  void* inter;             // [ndm_nom][nsb][tile_pitch]
  int64_t tile_pitch;
  int inter16;
};
void launch_stage1(const Stage1Args& a, cudaStream_t st);
struct Stage2Args {
  const void* inter;
  int64_t tile_pitch;
  int inter16;
  const int32_t* res;      // [dm_steps][nsb]
  int64_t nsb, dm_steps;
  int ndm0;
  int64_t ncols;           // output columns of this tile
  void* out;               // row m at out + m*out_pitch + col0
  int64_t out_pitch, col0;
  int out64;
  int sbw;
  int src_max;             // largest value one inter element can hold
};
void launch_stage2(const Stage2Args& a, cudaStream_t st);
struct BruteArgs {
  const void* x;           // phase layout [nc][ds][phase_len]
  int64_t phase_len;
  int ds;
  int nbits;
  const int32_t* delay;    // [dm_steps][nc]
  int64_t nc, dm_steps;
  int64_t start;           // first input sample of the slice
  int64_t ncols;           // columns of this slice
  void* out;
  int64_t out_pitch, col0;
  int out64;
};
void launch_brute(const BruteArgs& a, cudaStream_t st);

// Allows `kernel` `dynamic_smem` bytes of dynamic shared memory: above 48 KB per
// block, counting the kernel's static shared memory, a launch needs the opt-in.
template <typename K>
inline void allow_dynamic_smem(K kernel, size_t dynamic_smem) {
  if (dynamic_smem == 0) return;
  cudaFuncAttributes fa{};
  DD_CUDA_TRY(cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(kernel)));
  if (dynamic_smem + fa.sharedSizeBytes > 48 * 1024)
    DD_CUDA_TRY(cudaFuncSetAttribute(reinterpret_cast<const void*>(kernel),
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(dynamic_smem)));
}

// ---- shared-memory staged sums (dd_sumsmem.cu) ----
constexpr int kSumRows = 8;  // output rows per block
// Groups of warps the block's rows are split over: each group covers the whole
// tile for kSumRows/ROWSPLIT rows (fewer accumulators per thread, more words per
// lane).  Measured at the headline size (ms, stage 1 / stage 2): one group, 5
// words per lane 77.0 / 53.9; two groups, 5 words 80.0 / 51.4; two groups, 9
// words 77.6 / 50.9; two groups, 7 words 82.1 / 52.1.  The quad kernel (stage 2)
// takes two groups of 9 words, the 8-bit kernels one group of 5.
#ifndef DD_SUM_ROWSPLIT
#define DD_SUM_ROWSPLIT 1
#endif
#ifndef DD_SUM16Q_ROWSPLIT
#define DD_SUM16Q_ROWSPLIT 2
#endif
constexpr int kSumRowsPT = kSumRows / DD_SUM_ROWSPLIT;
constexpr int kSumRowsPTQ = kSumRows / DD_SUM16Q_ROWSPLIT;
// Staging descriptor of one (row group, source) pair of a staged sum: the
// smallest offset of the group's rows for that source, the spread of their
// offsets, and each row's offset relative to the smallest.  Built on the host
// from the plan's tables; the kernels read one per source and row group.
struct SumDesc {
  int32_t lo;
  int32_t span;
  uint16_t rel[kSumRows];
  int32_t pad[2];
};
static_assert(sizeof(SumDesc) == 32, "SumDesc is 32 bytes");
struct SumLaunch {
  enum Mode { kStage1 = 0, kStage2 = 1, kBrute = 2 };
  int mode;
  const char* src;         // byte address of source row 0
  int64_t src_pitch;       // bytes between source rows
  const int32_t* off;      // per-row, per-source offsets (elements)
  int64_t off_pitch;       // entries between consecutive rows of `off`
  int64_t base;            // element index added to every offset
  int64_t nsrc_total;      // stage 1: channels of the band; stage 2: subbands; brute: channels
  int64_t nrows_total;     // stage 1: nominal DMs; stage 2 and brute: DM trials
  int group;               // stage 1: subband width; stage 2: fine DMs per nominal DM
  int rows_per_block;      // kSumRows
  int64_t nsb_out;         // stage 1: subbands (inter rows are (j, sb))
  char* out;               // byte address of output row 0, column 0
  int64_t out_pitch;       // bytes between output rows (stage 1: between (j, sb) rows)
  int64_t out_col0;        // first output column of the launch (elements)
  int out_elem;            // bytes per output element
  int64_t ncols;           // columns of the launch
  int win_bytes;           // bytes of one staged source window
  int src_bytes;           // 1 or 2
  int flush;               // 8-bit sources: add the lanes into the output every 256 sources
  int lane_per;            // 16-bit sources: sources per 16-bit lane before widening
  unsigned grid_y, grid_z;
  const SumDesc* desc;     // [grid_y][desc_pitch] staging descriptors
  int64_t desc_pitch;      // descriptors per row group (= columns of the offset table)
  int stages;              // staged source pairs in flight (2..4)
  int* err;                // device error word: set when a bounded wait gives up
  unsigned one;            // 1 (a multiplier the compiler cannot fold)
  // 16-bit subband sums with a one-sample-shifted twin (0: none): the twin of the
  // element at byte address a sits at a + twin_off and holds the element before
  // it, twin[i] = sums[i - 1].  Stage 1 writes both; stage 2 reads a source whose
  // offset is odd from the twin, so every read is a whole aligned word.
  int64_t twin_off;
};
#ifndef DD_SUM_MAX_STAGES
#define DD_SUM_MAX_STAGES 8
#endif
// Shared memory (KB) the staged sums stay within by default: two blocks per SM.
#ifndef DD_SUM_SMEM_KB
#define DD_SUM_SMEM_KB 100
#endif
constexpr int kSumMaxStages = DD_SUM_MAX_STAGES;  // staged source pairs in flight, at most
void launch_sum(const SumLaunch& L, cudaStream_t st);
int sum_tile_samples(int src_bytes, int nw);
// Shared memory of a staged sum with `stages` pairs in flight.
// qs: source windows per pipeline stage (2, or 4 for the quad kernel).
size_t sum_smem_bytes(int win_bytes, int stages, int qs = 2);
// Pairs in flight that fit the shared memory of two blocks per SM (at least 2),
// next to `extra` bytes the kernel needs besides its ring (cap_kb: the shared
// memory to stay within, 0 for the default).
int sum_stages(int win_bytes, int qs = 2, size_t extra = 0, int cap_kb = 0);
// Stages of a kernel variant for a window size (its windows per stage, staging
// and shared-memory cap).
int sum_kind_stages(int kind, int win_bytes);
// Descriptors of a [nrows][ncols] offset table for row groups of kSumRows rows,
// grouped within blocks of `group` rows (0: one block), in the launch's
// blockIdx.y order.  Fails if a group's spread exceeds 65535.
std::vector<SumDesc> build_sum_desc(const std::vector<int32_t>& tab, int64_t nrows,
                                    int64_t ncols, int64_t group);
// Device error codes of the staged sums.
constexpr int kErrWaitFull = 1;   // a consumer gave up waiting for a staged window
constexpr int kErrWaitEmpty = 2;  // the producer gave up waiting for a free stage
// Tile (samples per block) of the kernel launch_sum picks for these sources.
// Words per lane of the staged sums (tile = 8 warps x 32 lanes x words x samples
// per word): 16-bit sources, 8-bit sources, 8-bit sources widened to 32 bits.
#ifndef DD_SUM16_NW
#define DD_SUM16_NW 4
#endif
#ifndef DD_SUM8_NW
#define DD_SUM8_NW 5
#endif
#ifndef DD_SUM8F_NW
#define DD_SUM8F_NW 5
#endif
// Blocks per SM the staged-sum kernels are compiled for (register budget).
#ifndef DD_SUM16_MINB
#define DD_SUM16_MINB 2
#endif
#ifndef DD_SUM8_MINB
#define DD_SUM8_MINB 2
#endif
#ifndef DD_SUM32_NW
#define DD_SUM32_NW 8
#endif
#ifndef DD_SUM32_MINB
#define DD_SUM32_MINB 2
#endif
constexpr int kSum32NW = DD_SUM32_NW;  // words per lane of the 32-bit staged sum
#ifndef DD_SUM16W_NW
#define DD_SUM16W_NW 5
#endif
// Warp groups the block's rows are split over in the 16-bit-into-32-bit kernel,
// blocks per SM it is built for and the shared memory (KB) it stays within.  Two
// warp groups of four rows at three blocks per SM take stage 1 of the
// 8192-channel 16-bit case on 2^18 samples (DM 0:0.25:500) from 29.5 to 24.5 ms
// but leave the full configuration (2^21 samples, three ranges) unchanged (first
// range 194.8 against 195.6 ms), so one group at two blocks per SM stays the
// default.
#ifndef DD_SUM16W_ROWSPLIT
#define DD_SUM16W_ROWSPLIT 1
#endif
#ifndef DD_SUM16W_MINB
#define DD_SUM16W_MINB 2
#endif
#ifndef DD_SUM16W_SMEM_KB
#define DD_SUM16W_SMEM_KB 100
#endif
constexpr int kSumRowsPTW = kSumRows / DD_SUM16W_ROWSPLIT;
// Words per lane of the 16-bit quad stage-2 kernel (odd: conflict-free consecutive words).
#ifndef DD_SUM16Q_NW
#define DD_SUM16Q_NW 9
#endif
constexpr int kSum16QNW = DD_SUM16Q_NW;
// Stage 2 on 16-bit sums with a shifted twin (k_sum_u16t): words per lane (lanes
// own interleaved words, so any count is conflict-free) and warp groups the
// block's rows are split over.
#ifndef DD_SUM16T_NW
#define DD_SUM16T_NW 6
#endif
#ifndef DD_SUM16T_ROWSPLIT
#define DD_SUM16T_ROWSPLIT 2
#endif
constexpr int kSum16TNW = DD_SUM16T_NW;
constexpr int kSumRowsPTT = kSumRows / DD_SUM16T_ROWSPLIT;
// Stage 2 of 8-bit input reads a twin of the subband sums (1) or aligns odd
// offsets with byte permutes (0, the quad kernel).  Measured at the headline
// size (ms, stage 1 / stage 2 / step): quad 69.3 / 46.8 / 120.6; twin with the
// stage-1 twin stored lane by lane 81.2 / 36.6 / 122.1; twin stored in 16-byte
// chunks through shared memory 71.1 / 36.6 / 112.0.
#ifndef DD_SUM16_TWIN
#define DD_SUM16_TWIN 1
#endif
// flush: 8-bit lanes added into the output every 256 sources; 16-bit sources summed into
// 32-bit lanes (the k_sum_u16w variant).
inline int sum_variant_tile(int src_bytes, bool flush) {
  return src_bytes == 4   ? sum_tile_samples(4, kSum32NW)
         : src_bytes == 2 ? (flush ? sum_tile_samples(2, DD_SUM16W_NW) / DD_SUM16W_ROWSPLIT
                                   : sum_tile_samples(2, DD_SUM16_NW))
                          : sum_tile_samples(1, flush ? DD_SUM8F_NW : DD_SUM8_NW) / DD_SUM_ROWSPLIT;
}
// Tile (samples per block) of a kernel variant (SumKind below).
inline int sum_kind_tile(int kind);
// Kernel variant of a staged sum: 8-bit sources into 16-bit sums, 8-bit sources
// widened to 32 bits (many sources), 8-bit, 16-bit and 32-bit sources.
enum SumKind { kSumKindU8Out16 = 0, kSumKindU8Flush = 1, kSumKindU8 = 2, kSumKindU16 = 3,
               kSumKindU32 = 4, kSumKindU16Wide = 5, kSumKindU16Quad = 6, kSumKindU16Twin = 7 };
constexpr int kSumKinds = 8;
int sum_kind(const SumLaunch& L);
inline int sum_kind_tile(int kind) {
  switch (kind) {
    case kSumKindU8Out16: case kSumKindU8: return sum_tile_samples(1, DD_SUM8_NW) / DD_SUM_ROWSPLIT;
    case kSumKindU8Flush: return sum_tile_samples(1, DD_SUM8F_NW) / DD_SUM_ROWSPLIT;
    case kSumKindU16: return sum_tile_samples(2, DD_SUM16_NW);
    case kSumKindU16Wide: return sum_tile_samples(2, DD_SUM16W_NW) / DD_SUM16W_ROWSPLIT;
    case kSumKindU16Quad: return sum_tile_samples(2, kSum16QNW) / DD_SUM16Q_ROWSPLIT;
    case kSumKindU16Twin: return sum_tile_samples(2, kSum16TNW) / DD_SUM16T_ROWSPLIT;
    default: return sum_tile_samples(4, kSum32NW);
  }
}
// Source windows per pipeline stage of a kernel variant: 4 for kSumKindU16Quad, 8
// for kSumKindU16Twin (four sources, each with its twin), else 2.
inline int sum_kind_qs(int kind) {
  return kind == kSumKindU16Quad ? 4 : kind == kSumKindU16Twin ? 8 : 2;
}
// Shared memory of a launch (its variant's windows per stage, plus the variant's
// staging past the ring, sum_kind_extra_smem).
size_t sum_launch_smem(const SumLaunch& L);
size_t sum_kind_extra_smem(int kind);
// Stage 1 of one tile and stage 2 of another in one launch (false: no paired
// kernel for these variants; nothing launched).
bool launch_sum_pair(const SumLaunch& L1, const SumLaunch& L2, cudaStream_t st);
unsigned sum_grid_x(const SumLaunch& L);
// One group of a batched (persistent) launch: all blocks of one staged sum.
struct SumBatchGroup {
  SumLaunch L;
  int kind;
  unsigned gx;           // blocks along x (time tiles)
  long long first;       // index of the group's first block in the batch
  int wait_ctr;          // counter to wait for (-1: none)
  int wait_need;         // ... until it reaches this value
  int done_ctr;          // counter each finished block increments
  int pad;
};
constexpr int kErrWaitGroup = 3;  // a batched group gave up waiting for its inputs
int sum_batch_blocks_per_sm(size_t smem);
// Persistent launch over groups (dependent stages ordered by counters).
void launch_sum_batch(const SumBatchGroup* d_groups, int ngroups, long long total, int* d_ctrs,
                      unsigned long long* d_next, int* d_err, size_t smem, unsigned grid,
                      cudaStream_t st);
// Grouped launch: one grid over independent groups of one variant (`kind`).
void launch_sum_grouped(const SumBatchGroup* d_groups, int ngroups, long long total, int kind,
                        size_t smem, cudaStream_t st);

// ---- brute-force table in the reference's host arithmetic (dd_hosttable.cpp) ----
void brute_delay_table_fastmath(const double* freq, size_t chan_start, size_t chan_end,
                                float dm_low, float dm_step, size_t dm_steps,
                                float ref_freq_value, double tsamp, int32_t* table);

// ---- probes (dd_probe.cu) ----
double measure_int_add_rate(int device);

}  // namespace dd
