// C ABI of the B200 dedispersion library: plan construction (argument checks,
// frequency table, channel range, DM grid, delay tables, workspace) and the run
// orchestration.  Host arithmetic that decides table entries is compiled with
// -ffp-contract=off and without fast-math, so every float expression below is
// evaluated in IEEE single precision exactly as written.
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <limits>
#include <new>
#include <string>
#include <vector>

#include "dd_internal.h"

namespace dd {

int tile_samples();

namespace {
thread_local std::string g_last_error;

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) DD_CUDA_TRY(cudaSetDevice(dev));
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

Error invalid(const char* fmt, double a = 0, double b = 0, double c = 0, double d = 0) {
  char buf[512];
  std::snprintf(buf, sizeof(buf), fmt, a, b, c, d);
  return Error{DD_ERR_INVALID, buf};
}

int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

// Bytes of one stage-1 sum: uint16 for 8-bit input in narrow subbands, else the
// reference's accumulator type (uint32, or uint64 for 32-bit samples).
int64_t inter_elem(const dd_plan& P) { return P.inter16 ? 2 : (P.nbits == 32 ? 8 : 4); }
// Stage 1 of 8-bit samples into 32-bit sums widens its 16-bit lanes every 256
// sources only when a subband holds more than 257 channels (257 x 255 fits).
// 16-bit samples are always summed into 32-bit lanes (the "wide" variant).
#ifndef DD_SUM16_WIDE
#define DD_SUM16_WIDE 1
#endif
bool stage1_flush(const dd_plan& P) {
  return (P.nbits == 8 && !P.inter16 && P.sbw > 257) || (P.nbits == 16 && DD_SUM16_WIDE);
}

// ---- frequency table and band (dedispered.cu:1003-1031, cpucal.hpp:85-116)
// Kernel variant of stage 2: 16-bit subband sums (8-bit input, subbands of at
// most 64 channels) four per pipeline stage, read from the sums and their
// shifted twin when stage 1 writes one, else 32-bit sums.
int stage2_kind(const dd_plan& P) {
  return P.inter16 ? (P.twin ? kSumKindU16Twin : kSumKindU16Quad) : kSumKindU32;
}
#ifndef DD_PAIR_STAGES
#define DD_PAIR_STAGES 0
#endif
// Byte offset from a subband-sum buffer to its twin (0: no twin).
int64_t twin_offset(const dd_plan& P) {
  return P.twin ? (DD_PAIR_STAGES ? 2 : 1) * P.inter_bytes : 0;
}

void build_freq(dd_plan& P) {
  const int n = P.hdr.nchans;
  P.freq.resize(n);
  if (P.p.freq_mode == DD_FREQ_FIL) {
    if (P.p.freq_table) {
      P.freq.assign(P.p.freq_table, P.p.freq_table + n);
    } else {
      // src/data/filterbank.cpp:445-449, in double; the reference build (-Ofast
      // with FMA) contracts fch1 + i*foff into a fused multiply-add.
      const double f1 = P.hdr.fch1, fo = P.hdr.foff;
      for (int i = 0; i < n; ++i) P.freq[i] = std::fma(static_cast<double>(i), fo, f1);
    }
  } else {
    // dedispered.cu:1004-1005: header.fch1 + i*header.foff in float, contracted into a
    // fused multiply-add by the reference build (-ffast-math with FMA); with separate
    // roundings about one channel in ten lands one float step away, which moves
    // delays that sit at a rounding tie.
    const float f1 = static_cast<float>(P.hdr.fch1), fo = static_cast<float>(P.hdr.foff);
    for (int i = 0; i < n; ++i)
      P.freq[i] = static_cast<double>(std::fmaf(static_cast<float>(static_cast<size_t>(i)), fo, f1));
  }
  for (int i = 1; i < n; ++i)
    if (!(P.freq[i] > P.freq[i - 1]))
      throw Error{DD_ERR_INVALID, "channel frequencies must be ascending (flip foff < 0 data first)"};
}

void build_band(dd_plan& P) {
  const int n = P.hdr.nchans;
  const float fmin = static_cast<float>(P.freq.front());
  const float fmax = static_cast<float>(P.freq.back());
  if (P.p.freq_start < fmin || P.p.freq_end > fmax)
    // the Filterbank entry points (dedispered.cu:509-516, cpucal.hpp:86-93) name the
    // file's range, the spectrum call (dedispered.cu:1009-1015) the spectrum's
    throw invalid(P.p.algorithm == DD_ALGO_BRUTE || P.p.freq_mode == DD_FREQ_FIL
                      ? "Frequency range [%.3f-%.3f MHz] out of filterbank range [%.3f-%.3f MHz]"
                      : "Frequency range [%.3f-%.3f MHz] out of spectrum range [%.3f-%.3f MHz]",
                  P.p.freq_start, P.p.freq_end, fmin, fmax);
  const float n1 = static_cast<float>(static_cast<size_t>(n - 1));
  volatile float span = fmax - fmin;
  volatile float qa = (P.p.freq_start - fmin) / span;
  volatile float qb = (P.p.freq_end - fmin) / span;
  size_t cs = static_cast<size_t>(qa * n1);
  size_t ce = static_cast<size_t>(qb * n1);
  ce = std::min<size_t>(static_cast<size_t>(n - 1), ce);
  if (cs >= static_cast<size_t>(n) || ce >= static_cast<size_t>(n))
    throw invalid("Invalid channel range [%.0f-%.0f] for %.0f channels", double(cs), double(ce), n);
  P.cs = static_cast<int64_t>(cs);
  P.ce = static_cast<int64_t>(ce);
  volatile float q = (P.p.dm_high - P.p.dm_low) / P.p.dm_step;
  P.dm_steps = static_cast<int64_t>(static_cast<size_t>(q)) + 1;
  P.ref_freq = static_cast<float>(P.freq[ce]);  // REF_FREQ_END
}

// ---- brute-force delay table (cpucal.hpp:119-132)
// table[m][c - cs] for c in [cs, ce); freq[ref_ch]: the reference frequency.
// Returns the number of entries that differ from the FP64 evaluation.
int64_t brute_table(const double* freq, int64_t cs, int64_t ce, int64_t ref_ch, float dm_low,
                    float dm_step, int64_t dm_steps, double tsamp, int mode, int32_t* table) {
  const int64_t nc = ce - cs;
  const float ref = static_cast<float>(freq[ref_ch]);
  if (mode == DD_TABLE_REFERENCE)
    brute_delay_table_fastmath(freq, static_cast<size_t>(cs), static_cast<size_t>(ce), dm_low,
                               dm_step, static_cast<size_t>(dm_steps), ref, tsamp, table);
  volatile float ref2 = ref * ref;
  const float inv_ref2 = 1.0f / ref2;
  int64_t mism = 0;
  for (int64_t s = 0; s < dm_steps; ++s) {
    volatile float idx = static_cast<float>(static_cast<size_t>(s));
    volatile float prod = idx * dm_step;
    volatile float dm = dm_low + prod;
    for (int64_t c = 0; c < nc; ++c) {
      const double dm64 = static_cast<double>(dm_low) + static_cast<double>(s) * dm_step;
      const double f = freq[cs + c], r = freq[ref_ch];
      const double e = 4148.808 * dm64 * (1.0 / (f * f) - 1.0 / (r * r)) / tsamp;
      const int v64 = static_cast<int>(std::floor(e + 0.5));
      int32_t& out = table[s * nc + c];
      if (mode == DD_TABLE_IEEE) {
        const float fr = static_cast<float>(freq[cs + c]);
        volatile float f2 = fr * fr;
        volatile float a = 1.0f / f2;
        volatile float diff = a - inv_ref2;
        volatile float kd = 4148.808f * dm;
        volatile float delay = kd * diff;
        out = static_cast<int>(std::round(static_cast<double>(delay) / tsamp));
      } else if (mode == DD_TABLE_FP64) {
        out = v64;
      }
      mism += (out != v64);
    }
  }
  return mism;
}

void build_brute_table(dd_plan& P) {
  P.h_delay.assign(static_cast<size_t>(P.dm_steps * P.nc), 0);
  P.table_mismatch_fp64 = brute_table(P.freq.data(), P.cs, P.cs + P.nc, P.ce, P.p.dm_low,
                                      P.p.dm_step, P.dm_steps, P.tsamp, P.p.table_mode,
                                      P.h_delay.data());
}

// ---- IQRM window plan (iqrm.cu:348-397) and lags (iqrm.cu:188-200)
void build_iqrm(dd_plan& P) {
  const dd_iqrm_config& q = P.rfi.iqrm;
  const double win_sec = std::max(0.0, q.win_sec), hop_sec = std::max(0.0, q.hop_sec);
  // header.tsamp * time_downsample in float (dedispered.cu:1088), or
  // fil.tsamp * time_downsample in double (dedispered.cu:580).
  double tsamp;
  if (P.p.freq_mode == DD_FREQ_FIL) {
    tsamp = P.tsamp * P.p.time_downsample;
  } else {
    volatile float ts = static_cast<float>(P.tsamp) * static_cast<float>(P.p.time_downsample);
    tsamp = static_cast<double>(ts);
  }
  const uint32_t ns = static_cast<uint32_t>(P.nbin);
  const uint32_t W = win_sec > 0.0 ? static_cast<uint32_t>(std::floor(win_sec / tsamp)) : 0u;
  const uint32_t H = hop_sec > 0.0 ? static_cast<uint32_t>(std::floor(hop_sec / tsamp)) : W;
  P.win_t0.clear();
  P.win_t1.clear();
  if (W == 0 || W >= ns) {
    P.win_t0.push_back(0);
    P.win_t1.push_back(ns);
  } else {
    uint32_t t0 = 0;
    while (t0 + W <= ns) {
      P.win_t0.push_back(t0);
      P.win_t1.push_back(t0 + W);
      t0 += (H ? H : W);
    }
    if (q.include_tail && t0 < ns && ns > t0 + 4) {
      P.win_t0.push_back(t0);
      P.win_t1.push_back(ns);
    }
  }
  const int64_t csub = P.ce - P.cs;  // IQRM's chan_end is exclusive (iqrm.cu:219)
  const float rf = std::max(0.0f, q.radius_frac);
  volatile float rprod = rf * static_cast<float>(csub);
  int radius = std::max(1, static_cast<int>(std::floor(static_cast<float>(rprod))));
  const double g = q.geofactor > 1.0 ? q.geofactor : 1.5;
  P.lags.clear();
  int lag = 1;
  while (lag <= radius) {
    // |lag| >= csub would index outside the statistic vector (the reference
    // reads past its end there); such lags are left out.
    if (lag < csub) {
      P.lags.push_back(+lag);
      P.lags.push_back(-lag);
    }
    int nxt = static_cast<int>(g * lag);
    lag = std::max(nxt, lag + 1);
  }
  // Segments: maximal runs of samples covered by the same set of windows.
  std::vector<uint32_t> cuts{0u, ns};
  for (size_t w = 0; w < P.win_t0.size(); ++w) {
    cuts.push_back(std::min(P.win_t0[w], ns));
    cuts.push_back(std::min(P.win_t1[w], ns));
  }
  std::sort(cuts.begin(), cuts.end());
  cuts.erase(std::unique(cuts.begin(), cuts.end()), cuts.end());
  P.segs.clear();
  for (size_t k = 0; k + 1 < cuts.size(); ++k) P.segs.push_back(IqrmSeg{cuts[k], cuts[k + 1]});
  if (P.segs.empty()) P.segs.push_back(IqrmSeg{0u, ns});
}

// Event recorder for dd_run_profiled: a plan-owned pool of events, recorded in
// pairs around the stages on the run's stream.
struct Prof {
  dd_plan& P;
  cudaStream_t st;
  size_t used = 0;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prep, s1, s2, total;
  cudaEvent_t take() {
    if (used == P.events.size()) {
      cudaEvent_t e;
      DD_CUDA_TRY(cudaEventCreate(&e));
      P.events.push_back(e);
    }
    return P.events[used++];
  }
  cudaEvent_t mark() {
    cudaEvent_t e = take();
    DD_CUDA_TRY(cudaEventRecord(e, st));
    return e;
  }
  static float sum(const std::vector<std::pair<cudaEvent_t, cudaEvent_t>>& v) {
    float t = 0.f;
    for (auto& pr : v) {
      float ms = 0.f;
      DD_CUDA_TRY(cudaEventElapsedTime(&ms, pr.first, pr.second));
      t += ms;
    }
    return t;
  }
};

// Largest spread (max - min) of a table's offsets over groups of `rows` consecutive
// rows, per column; rows are grouped within blocks of `group` rows (0: no blocks).
int table_spread(const std::vector<int32_t>& tab, int64_t nrows, int64_t ncols, int rows,
                 int64_t group) {
  int spread = 0;
  const int64_t blk = group > 0 ? group : nrows;
  for (int64_t b0 = 0; b0 < nrows; b0 += blk) {
    const int64_t b1 = std::min(nrows, b0 + blk);
    for (int64_t r0 = b0; r0 < b1; r0 += rows) {
      const int64_t r1 = std::min(b1, r0 + rows);
      for (int64_t c = 0; c < ncols; ++c) {
        int lo = tab[r0 * ncols + c], hi = lo;
        for (int64_t r = r0 + 1; r < r1; ++r) {
          lo = std::min(lo, tab[r * ncols + c]);
          hi = std::max(hi, tab[r * ncols + c]);
        }
        spread = std::max(spread, hi - lo);
      }
    }
  }
  return spread;
}

// Bytes of one staged window: the tile plus the rows' spread, 16-byte alignment
// slack and the funnel shift's extra word; 0 when the four windows of a block
// would not fit comfortably in shared memory.
int window_bytes(int spread, int tile, int elem, int qs = 2) {
  const int64_t w = round_up(static_cast<int64_t>(spread + tile) * elem + 40, 16);
  return sum_smem_bytes(static_cast<int>(w), 2, qs) <= 200 * 1024 ? static_cast<int>(w) : 0;
}

void upload_desc(DevBuf& b, const std::vector<SumDesc>& d) {
  b.alloc(sizeof(SumDesc) * d.size());
  DD_CUDA_TRY(cudaMemcpy(b.p, d.data(), sizeof(SumDesc) * d.size(), cudaMemcpyHostToDevice));
}

bool callsite_zdm_active(const dd_plan& P) {
  return P.rfi.use_zero_dm && P.p.zero_dm_mode == DD_ZDM_CALLSITE && P.cs > 0;
}

void upload(DevBuf& b, const void* h, size_t bytes) {
  b.alloc(bytes);
  if (bytes) DD_CUDA_TRY(cudaMemcpy(b.p, h, bytes, cudaMemcpyHostToDevice));
}


#ifndef DD_INTER_MB
#define DD_INTER_MB 2048
#endif
// Time tiling of the subband path for a subband-sum budget (bytes per tile): the
// tile length, the pitches, and the prepared-input and subband-sum buffers
// (reallocated, zeroed).  Results do not depend on the tiling.
void set_tiling(dd_plan& P, int64_t budget) {
  const int64_t kT = tile_samples();
  // Subband sums: 32-bit words (uint64 for 32-bit samples; uint16 in builds with
  // DD_INTER32=0).  Tile length L plus the stage-2 halo (max_res) should fill
  // whole stage-1 block tiles T1: L = n*T1 - R with R the halo rounded to the
  // base tile; n grows while one tile of subband sums stays within the budget and
  // the tile is not longer than the chunk.
  const int64_t per_col = P.ndm_nom * P.nsb * inter_elem(P) * (P.twin ? 2 : 1);
  const int64_t T1 = P.win1 ? sum_variant_tile(P.elem, stage1_flush(P)) : kT;
  const int64_t R = round_up(std::max<int64_t>(P.max_res, 1), kT);
  int64_t n = 1;
  while (n * T1 - R < kT) ++n;
  while (((n + 1) * T1 - R) * per_col <= budget && (n * T1 - R) < P.nout) ++n;
  const int64_t L = std::max<int64_t>(kT, n * T1 - R);
  P.tile = L;
  P.inter_budget = budget;
  // Stage-2 blocks past the tile's last column read up to one block tile beyond it
  // (their columns are not stored).
  const int64_t T2 = P.win2 ? sum_kind_tile(stage2_kind(P)) : kT;
  P.tile_pitch = round_up(round_up(L + P.max_res, kT) + T2 + 64, 64);
  const int64_t ntiles = (P.nbin + L - 1) / L;
  P.xpitch = round_up(ntiles * L + round_up(L + P.max_res, 8192) + P.max_delay + 8192, 64);
  P.d_x.alloc(static_cast<size_t>(P.dch * P.xpitch) * P.elem);
  DD_CUDA_TRY(cudaMemsetAsync(P.d_x.p, 0, P.d_x.bytes, cudaStreamLegacy));
  P.inter_bytes = P.ndm_nom * P.nsb * P.tile_pitch * inter_elem(P);
  // (+256: the twin's staged windows may start one 16-byte block past the sums')
  P.d_inter.alloc(static_cast<size_t>((DD_PAIR_STAGES ? 2 : 1) * (P.twin ? 2 : 1) * P.inter_bytes) + 256);
  DD_CUDA_TRY(cudaMemsetAsync(P.d_inter.p, 0, P.d_inter.bytes, cudaStreamLegacy));
  DD_CUDA_TRY(cudaStreamSynchronize(cudaStreamLegacy));
}

void create_subband(dd_plan& P) {
  P.sbw = P.p.subband_width > 0 ? P.p.subband_width : 32;
  P.ndm0 = P.p.ndm0 > 0 ? P.p.ndm0 : 32;
  const int ds = P.p.time_downsample;
  P.nbin = (P.nin + ds - 1) / ds;
  if (P.nout <= 0 || P.nout > P.nbin) P.nout = P.nbin;
  P.dch = P.ce - P.cs + 1;
  P.nsb = (P.dch + P.sbw - 1) / P.sbw;
  P.ndm_nom = (P.dm_steps + P.ndm0 - 1) / P.ndm0;
  P.h_delay.assign(static_cast<size_t>(P.ndm_nom * P.dch), 0);
  P.h_res.assign(static_cast<size_t>(P.dm_steps * P.nsb), 0);
  DevBuf d_freq;
  upload(d_freq, P.freq.data(), sizeof(double) * P.freq.size());
  P.d_delay.alloc(sizeof(int32_t) * P.h_delay.size());
  P.d_res.alloc(sizeof(int32_t) * P.h_res.size());
  launch_subband_tables(d_freq.as<double>(), P.cs, P.ce, P.p.dm_low, P.p.dm_step, P.dm_steps,
                        P.sbw, P.ndm0, P.ref_freq, P.tsamp, ds,
                        P.d_delay.as<int32_t>(), P.d_res.as<int32_t>(), 0);
  DD_CUDA_TRY(cudaMemcpy(P.h_delay.data(), P.d_delay.p, sizeof(int32_t) * P.h_delay.size(),
                         cudaMemcpyDeviceToHost));
  DD_CUDA_TRY(cudaMemcpy(P.h_res.data(), P.d_res.p, sizeof(int32_t) * P.h_res.size(),
                         cudaMemcpyDeviceToHost));
  // FP64 comparison table for the coarse delays (and replacement in FP64 mode).
  int64_t mism = 0;
  const double tsamp = P.tsamp, r = P.freq[P.ce];
  for (int64_t j = 0; j < P.ndm_nom; ++j) {
    const double dm = static_cast<double>(P.p.dm_low) + static_cast<double>(j) * P.ndm0 * P.p.dm_step;
    for (int64_t c = 0; c < P.dch; ++c) {
      const double f = P.freq[P.cs + c];
      const int v = static_cast<int>(std::floor(4148.808 * dm * (1.0 / (f * f) - 1.0 / (r * r)) / tsamp + 0.5)) / ds;
      mism += (v != P.h_delay[j * P.dch + c]);
      if (P.p.table_mode == DD_TABLE_FP64) P.h_delay[j * P.dch + c] = v;
    }
  }
  if (P.p.table_mode == DD_TABLE_FP64) {
    for (int64_t m = 0; m < P.dm_steps; ++m) {
      const int64_t j = m / P.ndm0;
      const double dd = (static_cast<double>(m) - static_cast<double>(j * P.ndm0)) * P.p.dm_step;
      for (int64_t sb = 0; sb < P.nsb; ++sb) {
        const int64_t ch0 = P.cs + sb * P.sbw;
        const int64_t ch1 = std::min<int64_t>(ch0 + P.sbw, P.ce + 1);
        const double f = P.freq[(ch0 + ch1 - 1) / 2];
        P.h_res[m * P.nsb + sb] = static_cast<int>(std::floor(4148.808 * dd * (1.0 / (f * f) - 1.0 / (r * r)) / (tsamp * ds) + 0.5));
      }
    }
    DD_CUDA_TRY(cudaMemcpy(P.d_delay.p, P.h_delay.data(), sizeof(int32_t) * P.h_delay.size(), cudaMemcpyHostToDevice));
    DD_CUDA_TRY(cudaMemcpy(P.d_res.p, P.h_res.data(), sizeof(int32_t) * P.h_res.size(), cudaMemcpyHostToDevice));
  }
  P.table_mismatch_fp64 = mism;
  int mind = 0, minr = 0;
  P.max_delay = 0;
  P.max_res = 0;
  for (int v : P.h_delay) { P.max_delay = std::max(P.max_delay, v); mind = std::min(mind, v); }
  for (int v : P.h_res) { P.max_res = std::max(P.max_res, v); minr = std::min(minr, v); }
  if (mind < 0 || minr < 0)
    throw invalid("negative dispersion delays (DM below zero or band order) are not supported");
#ifndef DD_INTER32
#define DD_INTER32 0
#endif
  P.inter16 = (P.nbits == 8 && P.sbw <= 64 && !DD_INTER32) ? 1 : 0;
  if (P.nbits <= 16) {
    const int T1 = sum_variant_tile(P.elem, stage1_flush(P));
    P.win1 = window_bytes(table_spread(P.h_delay, P.ndm_nom, P.dch, kSumRows, 0), T1, P.elem);
  }
  // the twin needs the staged stage 1 (which writes it) and the staged stage 2
  P.twin = (P.inter16 && P.win1 && DD_SUM16_TWIN) ? 1 : 0;
  if (P.nbits <= 16) {
    // stage-2 sources: the stage-1 sums (uint16 or uint32)
    const int e2 = static_cast<int>(inter_elem(P));
    const int T2 = sum_kind_tile(stage2_kind(P));
    P.win2 = window_bytes(table_spread(P.h_res, P.dm_steps, P.nsb, kSumRows, P.ndm0), T2, e2,
                          sum_kind_qs(stage2_kind(P)));
  }
  if (!P.win2) P.twin = 0;
  if (P.win1) upload_desc(P.d_desc1, build_sum_desc(P.h_delay, P.ndm_nom, P.dch, 0));
  if (P.win2) upload_desc(P.d_desc2, build_sum_desc(P.h_res, P.dm_steps, P.nsb, P.ndm0));
  set_tiling(P, int64_t(DD_INTER_MB) << 20);
  if (ds > 1 || callsite_zdm_active(P))
    P.d_binned.alloc(static_cast<size_t>(P.nbin * P.hdr.nchans) * P.elem);
  if (ds > 1 && binning_lut_entries(P.nbits, ds)) {
    P.d_bin_lut.alloc(static_cast<size_t>(binning_lut_entries(P.nbits, ds)) * P.elem);
    launch_binning_lut(P.d_bin_lut.p, P.nbits, ds, cudaStreamLegacy);
    DD_CUDA_TRY(cudaStreamSynchronize(cudaStreamLegacy));
  }
  P.adds = static_cast<double>(P.ndm_nom) * P.dch * P.nout +
           static_cast<double>(P.dm_steps) * P.nsb * P.nout;
}

// The staged-window sums serve 8- and 16-bit samples without downsampling (one
// source row per channel); other cases use the direct kernels.
void set_brute_window(dd_plan& P) {
  P.winb = 0;
  if (P.p.time_downsample == 1 && P.nbits <= 16) {
    const int T = sum_variant_tile(P.elem, P.nbits == 8 || P.nbits == 16);
    P.winb = window_bytes(table_spread(P.h_delay, P.dm_steps, P.nc, kSumRows, 0), T, P.elem);
  }
  if (P.winb) upload_desc(P.d_descb, build_sum_desc(P.h_delay, P.dm_steps, P.nc, 0));
}

void create_brute(dd_plan& P) {
  const int ds = P.p.time_downsample;
  if (P.cs >= P.ce) throw invalid("Invalid chan parameters");
  if (ds < 1) throw invalid("time_downsample must be >= 1");
  if (P.p.dm_low > P.p.dm_high || P.p.dm_low < 0 || P.p.dm_step <= 0)
    throw invalid("Invalid DM parameters");
  if (P.p.t_sample > P.nin * P.tsamp)
    throw invalid("t_sample exceeds total observation time");
  P.nbin = P.nin;
  P.nc = P.ce - P.cs;
  build_brute_table(P);
  P.sps = static_cast<int64_t>(std::round(static_cast<double>(P.p.t_sample) / P.tsamp));
  if (P.sps <= 0) throw invalid("t_sample shorter than one sample");
  P.nslices = (P.nin + P.sps - 1) / P.sps;
  P.slice_cols.clear();
  P.out_cols = 0;
  for (int64_t s = 0; s < P.nslices; ++s) {
    const int64_t start = s * P.sps, end = std::min(start + P.sps, P.nin);
    const int64_t cols = (end - start + ds - 1) / ds;
    P.slice_cols.push_back(cols);
    P.out_cols += cols;
  }
  P.cols0 = P.slice_cols.front();
  P.phases_merge = (P.sps % ds) == 0;
  P.max_delay = 0;
  int mind = 0;
  for (int v : P.h_delay) { P.max_delay = std::max(P.max_delay, v); mind = std::min(mind, v); }
  if (mind < 0) throw invalid("negative dispersion delays are not supported");
  const int64_t kT = tile_samples();
  P.phase_len = round_up((P.nin + ds - 1) / ds + P.max_delay / ds + round_up(P.cols0, kT) + kT + 64, 64);
  P.d_x.alloc(static_cast<size_t>(P.nc * ds * P.phase_len) * P.elem);
  DD_CUDA_TRY(cudaMemset(P.d_x.p, 0, P.d_x.bytes));
  P.d_delay.alloc(sizeof(int32_t) * P.h_delay.size());
  DD_CUDA_TRY(cudaMemcpy(P.d_delay.p, P.h_delay.data(), sizeof(int32_t) * P.h_delay.size(),
                         cudaMemcpyHostToDevice));
  set_brute_window(P);
  P.adds = static_cast<double>(P.dm_steps) * P.nc * P.out_cols;
}

void create_rfi(dd_plan& P) {
  const int64_t n = P.hdr.nchans;
  std::vector<uint8_t> keep(static_cast<size_t>(n), 1);
  bool any_bad = false;
  for (int32_t c : P.bad)
    if (c >= 0 && c < n) { keep[c] = 0; any_bad = true; }
  if (P.rfi.use_mask && any_bad) upload(P.d_bad_keep, keep.data(), keep.size());
  if (P.rfi.use_iqrm) {
    build_iqrm(P);
    const int nwin = static_cast<int>(P.win_t0.size());
    std::vector<uint32_t> win(2 * nwin);
    for (int w = 0; w < nwin; ++w) { win[2 * w] = P.win_t0[w]; win[2 * w + 1] = P.win_t1[w]; }
    upload(P.d_win, win.data(), sizeof(uint32_t) * win.size());
    std::vector<uint32_t> st0(P.segs.size());
    for (size_t k = 0; k < P.segs.size(); ++k) st0[k] = P.segs[k].t0;
    upload(P.d_seg_t0, st0.data(), sizeof(uint32_t) * st0.size());
    if (!P.lags.empty()) upload(P.d_lags, P.lags.data(), sizeof(int32_t) * P.lags.size());
    const int64_t csub = std::max<int64_t>(P.ce - P.cs, 1);
    if (!P.lags.empty()) check_iqrm_channels(csub);
    P.d_stats.alloc(sizeof(unsigned long long) * 2 * csub * nwin);
    P.d_iqrm_scratch.alloc(iqrm_scratch_bytes(nwin, csub, static_cast<int>(P.lags.size())));
    P.d_masks.alloc(static_cast<size_t>(nwin) * n);
    P.d_segmask.alloc(P.segs.size() * n);
  }
  if (callsite_zdm_active(P) && P.cs * P.ce > P.nbin * n)
    throw invalid("zero-DM at the reference call site would read past the chunk (%.0f x %.0f elements)",
                  double(P.ce), double(P.cs));
  if (P.rfi.use_zero_dm) {
    if (P.p.zero_dm_mode == DD_ZDM_RANGE) P.d_zdm.alloc(sizeof(uint32_t) * P.nbin);
    else if (P.p.zero_dm_mode == DD_ZDM_RANGE_REF) P.d_zdm.alloc(sizeof(float) * P.nbin);
    else if (callsite_zdm_active(P)) P.d_zdm.alloc(sizeof(float) * (P.ce + 1));
  }
}

void run_rfi_and_prep(dd_plan& P, const void* input, uint8_t* masks_out, uint32_t* bounds_out,
                      void* prepped, cudaStream_t st) {
  const int64_t n = P.hdr.nchans;
  const void* src = input;
  const int ds = P.p.time_downsample;
  if (ds > 1) {
    launch_time_binning(input, P.d_binned.p, P.nbits, P.nin, n, ds,
                        P.d_bin_lut.bytes ? P.d_bin_lut.p : nullptr, st);
    src = P.d_binned.p;
  }
  const bool callsite = callsite_zdm_active(P);
  if (callsite && src == input) {
    DD_CUDA_TRY(cudaMemcpyAsync(P.d_binned.p, input, static_cast<size_t>(P.nbin * n) * P.elem,
                                cudaMemcpyDeviceToDevice, st));
    src = P.d_binned.p;
  }
  const uint8_t* segmask = nullptr;
  const int nseg = static_cast<int>(P.segs.size());
  if (P.rfi.use_iqrm) {
    const int nwin = static_cast<int>(P.win_t0.size());
    const int64_t csub = P.ce - P.cs;
    if (csub > 0 && !P.lags.empty()) {
      launch_iqrm_stats(src, P.nbits, P.nbin, n, P.cs, csub, P.d_win.as<uint32_t>(), nwin,
                        P.d_stats.as<unsigned long long>(), st);
      launch_iqrm_decide(P.d_stats.as<unsigned long long>(), nwin, P.d_win.as<uint32_t>(), n,
                         P.cs, csub, P.rfi.iqrm.mode, std::max(0.0f, P.rfi.iqrm.nsigma),
                         P.d_lags.as<int32_t>(), static_cast<int>(P.lags.size()), P.iqrm_variant,
                         P.d_iqrm_scratch.p, P.d_masks.as<uint8_t>(), st);
    } else {
      DD_CUDA_TRY(cudaMemsetAsync(P.d_masks.p, 0, P.d_masks.bytes, st));
    }
    launch_segment_masks(P.d_masks.as<uint8_t>(), nwin, P.d_win.as<uint32_t>(),
                         P.d_seg_t0.as<uint32_t>(), nseg, n, P.d_segmask.as<uint8_t>(), st);
    segmask = P.d_segmask.as<uint8_t>();
    if (masks_out)
      DD_CUDA_TRY(cudaMemcpyAsync(masks_out, P.d_masks.p, static_cast<size_t>(nwin) * n,
                                  cudaMemcpyDeviceToDevice, st));
    if (bounds_out)
      DD_CUDA_TRY(cudaMemcpyAsync(bounds_out, P.d_win.p, sizeof(uint32_t) * 2 * nwin,
                                  cudaMemcpyDeviceToDevice, st));
  }
  PrepArgs a{};
  a.nbits = P.nbits;
  a.nsamp = P.nbin;
  a.nchans = n;
  a.keep = P.d_bad_keep.as<uint8_t>();
  a.nseg = nseg;
  a.seg_t0 = P.d_seg_t0.as<uint32_t>();
  if (callsite) {
    // Reference order on the flat buffer: IQRM mask, zero-DM as called, mask file.
    if (segmask) launch_apply_masks_inplace(const_cast<void*>(src), P.nbits, P.nbin, n, segmask,
                                            P.d_seg_t0.as<uint32_t>(), nseg, st);
    launch_zero_dm_callsite(const_cast<void*>(src), P.nbits, static_cast<size_t>(P.cs),
                            static_cast<size_t>(P.ce), static_cast<size_t>(P.nbin),
                            P.d_zdm.as<float>(), st);
    a.segmask = nullptr;
  } else {
    a.segmask = segmask;
    if (P.rfi.use_zero_dm && P.p.zero_dm_mode == DD_ZDM_RANGE) {
      launch_zdm_offsets(src, P.nbits, P.nbin, n, P.cs, P.ce, segmask, P.d_seg_t0.as<uint32_t>(),
                         nseg, P.d_zdm.as<uint32_t>(), st);
      a.zdm_off = P.d_zdm.as<uint32_t>();
      a.zdm_cs = P.cs;
      a.zdm_ce = P.ce;
    } else if (P.rfi.use_zero_dm && P.p.zero_dm_mode == DD_ZDM_RANGE_REF) {
      launch_zdm_range_mean(src, P.nbits, P.nbin, n, P.cs, P.ce, segmask,
                            P.d_seg_t0.as<uint32_t>(), nseg, P.d_zdm.as<float>(), st);
      a.zdm_mean = P.d_zdm.as<float>();
      a.zdm_cs = P.cs;
      a.zdm_ce = P.ce;
    }
  }
  a.x = src;
  a.out = P.d_x.p;
  a.c0 = P.cs;
  a.c1 = P.ce + 1;
  a.ds = 1;
  a.pitch = P.xpitch;
  a.full_out = prepped;
  launch_prep(a, st);
}

// Staged-sum launches of one subband time tile starting at t0 (stage 1: the
// prepared input into the tile of subband sums; stage 2: the tile into the output).
SumLaunch stage1_launch(const dd_plan& P, int64_t t0, int buf = 0) {
  SumLaunch L{};
  L.mode = SumLaunch::kStage1;
  L.src = static_cast<const char*>(P.d_x.p);
  L.src_pitch = P.xpitch * P.elem;
  L.off = P.d_delay.as<int32_t>();
  L.off_pitch = P.dch;
  L.base = t0;
  L.nsrc_total = P.dch;
  L.nrows_total = P.ndm_nom;
  L.group = P.sbw;
  L.rows_per_block = kSumRows;
  L.nsb_out = P.nsb;
  L.out = static_cast<char*>(P.d_inter.p) + buf * P.inter_bytes;
  L.out_pitch = P.tile_pitch * inter_elem(P);
  L.out_col0 = 0;
  L.out_elem = static_cast<int>(inter_elem(P));
  L.ncols = P.tile + P.max_res;
  L.win_bytes = P.win1;
  L.src_bytes = P.elem;
  L.flush = stage1_flush(P) ? 1 : 0;
  L.lane_per = 1;
  L.grid_y = static_cast<unsigned>((P.ndm_nom + kSumRows - 1) / kSumRows);
  L.grid_z = static_cast<unsigned>(P.nsb);
  L.desc = P.d_desc1.as<SumDesc>();
  L.desc_pitch = P.dch;
  L.stages = P.stages_override ? P.stages_override : sum_kind_stages(sum_kind(L), P.win1);
  L.err = P.d_err.as<int>();
  L.one = 1;
  L.twin_off = twin_offset(P);
  return L;
}

SumLaunch stage2_launch(const dd_plan& P, int64_t t0, void* output, int buf = 0) {
  SumLaunch L{};
  L.mode = SumLaunch::kStage2;
  L.src = static_cast<const char*>(P.d_inter.p) + buf * P.inter_bytes;
  L.src_pitch = P.tile_pitch * inter_elem(P);
  L.off = P.d_res.as<int32_t>();
  L.off_pitch = P.nsb;
  L.base = 0;
  L.nsrc_total = P.nsb;
  L.nrows_total = P.dm_steps;
  L.group = P.ndm0;
  L.rows_per_block = kSumRows;
  L.out = static_cast<char*>(output);
  L.out_pitch = P.nout * 4;
  L.out_col0 = t0;
  L.out_elem = 4;
  L.ncols = std::min<int64_t>(P.tile, P.nout - t0);
  L.win_bytes = P.win2;
  L.src_bytes = static_cast<int>(inter_elem(P));
  L.flush = 0;
  L.lane_per = P.inter16 ? 65535 / (255 * P.sbw) : 1;  // >= 4 for subbands of <= 64 channels
  L.grid_y = static_cast<unsigned>(P.ndm_nom * ((P.ndm0 + kSumRows - 1) / kSumRows));
  L.grid_z = 1;
  L.desc = P.d_desc2.as<SumDesc>();
  L.desc_pitch = P.nsb;
  L.stages = P.stages_override ? P.stages_override : sum_kind_stages(stage2_kind(P), P.win2);
  L.err = P.d_err.as<int>();
  L.one = 1;
  L.twin_off = twin_offset(P);
  return L;
}

// after_tile(t0, cols): called once the work producing output columns
// [t0, t0 + cols) of every DM row has been queued on the stream.
using TileHook = std::function<void(int64_t, int64_t)>;

// before_sums: called once the RFI stages and the layout are queued, before the
// first sum that writes `output`.
// before_out(t0, cols): called before the first launch that writes output
// columns [t0, t0 + cols) of the DM rows.
void run_subband(dd_plan& P, const void* input, void* output, uint8_t* masks_out,
                 uint32_t* bounds_out, void* prepped, cudaStream_t st, Prof* pf = nullptr,
                 const TileHook& after_tile = TileHook(),
                 const std::function<void()>& before_sums = std::function<void()>(),
                 const TileHook& before_out = TileHook()) {
  cudaEvent_t a = pf ? pf->mark() : nullptr;
  run_rfi_and_prep(P, input, masks_out, bounds_out, prepped, st);
  if (pf) pf->prep.emplace_back(a, pf->mark());
  if (before_sums) before_sums();
  // With DD_PAIR_STAGES, stage 1 of tile k+1 shares a launch with stage 2 of tile
  // k (alternating subband-sum buffers).  Measured on B200 at the headline size it
  // is no faster than running the stages one after another (148.6 vs 145.8 ms per
  // step), so the default build keeps them apart.
  if (DD_PAIR_STAGES && !pf && P.win1 && P.win2 && P.nout > P.tile) {
    const int64_t ntiles = (P.nout + P.tile - 1) / P.tile;
    launch_sum(stage1_launch(P, 0, 0), st);
    bool paired = true;
    for (int64_t k = 1; k <= ntiles; ++k) {
      const int64_t tprev = (k - 1) * P.tile;
      if (before_out) before_out(tprev, std::min<int64_t>(P.tile, P.nout - tprev));
      const SumLaunch s2 = stage2_launch(P, tprev, output, static_cast<int>((k - 1) & 1));
      if (k < ntiles) {
        const SumLaunch s1 = stage1_launch(P, k * P.tile, static_cast<int>(k & 1));
        if (!(paired = launch_sum_pair(s1, s2, st))) {
          launch_sum(s2, st);
          launch_sum(s1, st);
        }
      } else {
        launch_sum(s2, st);
      }
      if (after_tile) after_tile(tprev, std::min<int64_t>(P.tile, P.nout - tprev));
    }
    (void)paired;
    return;
  }
  for (int64_t t0 = 0; t0 < P.nout; t0 += P.tile) {
    cudaEvent_t b1 = pf ? pf->mark() : nullptr;
    if (P.win1) {
      launch_sum(stage1_launch(P, t0), st);
    } else {
      Stage1Args s1{};
      s1.x = P.d_x.p;
      s1.xpitch = P.xpitch;
      s1.nbits = P.nbits;
      s1.delay1 = P.d_delay.as<int32_t>();
      s1.dch = P.dch;
      s1.nsb = P.nsb;
      s1.ndm_nom = P.ndm_nom;
      s1.sbw = P.sbw;
      s1.t0 = t0;
      s1.ncols = P.tile + P.max_res;
      s1.inter = P.d_inter.p;
      s1.tile_pitch = P.tile_pitch;
      s1.inter16 = P.inter16;
      launch_stage1(s1, st);
    }
    if (pf) pf->s1.emplace_back(b1, pf->mark());
    if (before_out) before_out(t0, std::min<int64_t>(P.tile, P.nout - t0));
    cudaEvent_t b2 = pf ? pf->mark() : nullptr;
    if (P.win2) {
      launch_sum(stage2_launch(P, t0, output), st);
    } else {
      Stage2Args s2{};
      s2.inter = P.d_inter.p;
      s2.tile_pitch = P.tile_pitch;
      s2.inter16 = P.inter16;
      s2.res = P.d_res.as<int32_t>();
      s2.nsb = P.nsb;
      s2.dm_steps = P.dm_steps;
      s2.ndm0 = P.ndm0;
      s2.ncols = std::min<int64_t>(P.tile, P.nout - t0);
      s2.out = output;
      s2.out_pitch = P.nout;
      s2.col0 = t0;
      s2.out64 = P.nbits == 32 ? 1 : 0;
      s2.sbw = P.sbw;
      s2.src_max = P.sbw * 255;
      launch_stage2(s2, st);
    }
    if (pf) pf->s2.emplace_back(b2, pf->mark());
    if (after_tile) after_tile(t0, std::min<int64_t>(P.tile, P.nout - t0));
  }
}

// Staged-sum launch of the brute-force sums (all DMs, all slices at once).
SumLaunch brute_launch(const dd_plan& P, void* output) {
  SumLaunch L{};
  L.mode = SumLaunch::kBrute;
  L.src = static_cast<const char*>(P.d_x.p);
  L.src_pitch = P.phase_len * P.elem;
  L.off = P.d_delay.as<int32_t>();
  L.off_pitch = P.nc;
  L.base = 0;
  L.nsrc_total = P.nc;
  L.nrows_total = P.dm_steps;
  L.rows_per_block = kSumRows;
  L.out = static_cast<char*>(output);
  L.out_pitch = P.out_cols * 4;
  L.out_col0 = 0;
  L.out_elem = 4;
  L.ncols = P.out_cols;
  L.win_bytes = P.winb;
  L.src_bytes = P.elem;
  L.flush = (P.nbits == 8 || P.nbits == 16) ? 1 : 0;  // 8-bit: widened lanes; 16-bit: 32-bit sums
  L.lane_per = 1;
  L.grid_y = static_cast<unsigned>((P.dm_steps + kSumRows - 1) / kSumRows);
  L.grid_z = 1;
  L.desc = P.d_descb.as<SumDesc>();
  L.desc_pitch = P.nc;
  L.stages = sum_kind_stages(sum_kind(L), P.winb);
  L.err = P.d_err.as<int>();
  L.one = 1;
  return L;
}

void run_brute_prep(dd_plan& P, const void* input, void* prepped, cudaStream_t st) {
  PrepArgs a{};
  a.x = input;
  a.nbits = P.nbits;
  a.nsamp = P.nin;
  a.nchans = P.hdr.nchans;
  a.out = P.d_x.p;
  a.c0 = P.cs;
  a.c1 = P.ce;
  a.ds = P.p.time_downsample;
  a.pitch = P.phase_len;
  a.full_out = prepped;
  launch_prep(a, st);
}

void run_brute(dd_plan& P, const void* input, void* output, void* prepped, cudaStream_t st,
               Prof* pf = nullptr) {
  cudaEvent_t e0 = pf ? pf->mark() : nullptr;
  run_brute_prep(P, input, prepped, st);
  if (pf) pf->prep.emplace_back(e0, pf->mark());
  cudaEvent_t e1 = pf ? pf->mark() : nullptr;
  BruteArgs b{};
  b.x = P.d_x.p;
  b.phase_len = P.phase_len;
  b.ds = P.p.time_downsample;
  b.nbits = P.nbits;
  b.delay = P.d_delay.as<int32_t>();
  b.nc = P.nc;
  b.dm_steps = P.dm_steps;
  b.out = output;
  b.out_pitch = P.out_cols;
  b.out64 = P.nbits == 32;
  if (P.winb) {
    launch_sum(brute_launch(P, output), st);
  } else if (P.phases_merge) {
    b.start = 0;
    b.ncols = P.out_cols;
    b.col0 = 0;
    launch_brute(b, st);
  } else {
    for (int64_t s = 0; s < P.nslices; ++s) {
      b.start = s * P.sps;
      b.ncols = P.slice_cols[s];
      b.col0 = s * P.cols0;
      launch_brute(b, st);
    }
  }
  if (pf) pf->s2.emplace_back(e1, pf->mark());
}


// After a synchronising call: report (and clear) a bounded wait that gave up
// inside a staged-sum kernel.
void check_device_error(dd_plan& P, cudaStream_t st) {
  int e = 0;
  DD_CUDA_TRY(cudaMemcpyAsync(&e, P.d_err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  DD_CUDA_TRY(cudaStreamSynchronize(st));
  if (e) {
    DD_CUDA_TRY(cudaMemsetAsync(P.d_err.p, 0, sizeof(int), st));
    DD_CUDA_TRY(cudaStreamSynchronize(st));
    throw Error{DD_ERR_RUNTIME, e == kErrWaitFull
                                    ? "a staged-sum block timed out waiting for its input window"
                                    : "a staged-sum block timed out waiting for a free stage"};
  }
}

int64_t workspace_of(const dd_plan& P) {
  const DevBuf* bufs[] = {&P.d_delay, &P.d_res, &P.d_lags, &P.d_bad_keep, &P.d_win, &P.d_seg_t0,
                          &P.d_binned, &P.d_bin_lut, &P.d_x, &P.d_inter, &P.d_stats, &P.d_iqrm_scratch,
                          &P.d_masks, &P.d_segmask, &P.d_zdm, &P.d_desc1, &P.d_desc2,
                          &P.d_descb, &P.d_err};
  int64_t t = 0;
  for (auto* b : bufs) t += static_cast<int64_t>(b->bytes);
  return t;
}

template <typename F>
int guarded(F&& f) {
  try {
    g_last_error.clear();
    f();
    return DD_OK;
  } catch (const Error& e) {
    g_last_error = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    g_last_error = "host allocation failed";
    return DD_ERR_NOMEM;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return DD_ERR_RUNTIME;
  }
}

}  // namespace

void set_error(const std::string& msg) { g_last_error = msg; }

long long& launch_count() {
  thread_local long long n = 0;
  return n;
}

// Device memory comes from the stream-ordered allocator (the device's default
// pool), allocated on the legacy stream; callers synchronise the legacy stream
// before other streams use it (plan creation does).  It is released either
// after a device-wide synchronisation (dd_plan_destroy and every other path), or
// stream-ordered on a caller's stream without stalling the device
// (dd_plan_destroy_async sets g_free_stream for the duration of the call).
thread_local cudaStream_t g_free_stream = nullptr;
thread_local bool g_free_async = false;

void DevBuf::alloc(size_t n) {
  release();
  if (n == 0) return;
  cudaError_t e = cudaMallocAsync(&p, n, cudaStreamLegacy);
  if (e != cudaSuccess) {
    p = nullptr;
    cudaGetLastError();
    throw Error{e == cudaErrorMemoryAllocation ? DD_ERR_NOMEM : DD_ERR_CUDA,
                std::string("device allocation of ") + std::to_string(n) + " bytes failed: " +
                    cudaGetErrorString(e)};
  }
  bytes = n;
}

void DevBuf::release() {
  if (p) {
    if (g_free_async) {
      cudaFreeAsync(p, g_free_stream);
    } else {
      cudaDeviceSynchronize();
      cudaFreeAsync(p, cudaStreamLegacy);
    }
  }
  p = nullptr;
  bytes = 0;
}

}  // namespace dd

using namespace dd;

extern "C" {

int dd_abi_version(void) { return DD_ABI_VERSION; }

const char* dd_last_error(void) { return g_last_error.c_str(); }

}  // extern "C"

namespace dd {
namespace {
// Builds a plan (throws on error).  nout > 0 limits a subband plan's output to
// the first nout binned columns (the plan of a stream).
dd_plan* make_plan(const dd_header* header, const dd_plan_params* params, const dd_rfi_config* rfi,
                   const int32_t* bad_channels, int32_t n_bad, int32_t device, int64_t nout) {
  if (!header || !params) throw Error{DD_ERR_INVALID, "header and params are required"};
  if (header->nbits != 8 && header->nbits != 16 && header->nbits != 32)
    throw Error{DD_ERR_INVALID, "nbits must be 8, 16 or 32"};
  if (header->nchans < 2 || header->ndata < 1 || !(header->tsamp > 0))
    throw Error{DD_ERR_INVALID, "header needs nchans >= 2, ndata >= 1 and tsamp > 0"};
  if (params->time_downsample < 1) throw Error{DD_ERR_INVALID, "time_downsample must be >= 1"};
  if (params->zero_dm_mode != DD_ZDM_CALLSITE && params->zero_dm_mode != DD_ZDM_RANGE &&
      params->zero_dm_mode != DD_ZDM_RANGE_REF)
    throw Error{DD_ERR_INVALID, "unknown zero-DM mode"};
  if (!(params->dm_step > 0) || params->dm_high < params->dm_low)
    throw Error{DD_ERR_INVALID, "Invalid DM parameters"};
  int ndev = 0;
  DD_CUDA_TRY(cudaGetDeviceCount(&ndev));
  if (ndev == 0) throw Error{DD_ERR_RUNTIME, "No CUDA devices found"};
  if (device < 0 || device >= ndev) throw Error{DD_ERR_INVALID, "invalid target device"};
  DeviceGuard g(device);
  std::unique_ptr<dd_plan> P(new dd_plan());
  P->hdr = *header;
  P->p = *params;
  if (rfi) P->rfi = *rfi;
  if (P->p.algorithm == DD_ALGO_BRUTE) {
    // The CPU path the brute-force mode follows has no RFI stages.
    P->rfi.use_iqrm = P->rfi.use_mask = P->rfi.use_zero_dm = 0;
  }
  if (bad_channels && n_bad > 0) P->bad.assign(bad_channels, bad_channels + n_bad);
  P->device = device;
  P->nbits = header->nbits;
  P->elem = header->nbits / 8;
  P->nin = header->ndata;
  P->nout = nout;
  // The reference's GPU path casts sample counts to unsigned int in its RFI
  // kernels (rfimarker.cu, iqrm.cu).
  if (P->nin >= (int64_t(1) << 32)) throw Error{DD_ERR_INVALID, "ndata too large"};
  // Floating-point forms of the reference's IQRM arithmetic (bit 8: std from a
  // fused multiply-add; bit 4: threshold through the reciprocal of 1.349).
  P->iqrm_variant = 8 | 4;
  if (const char* v = std::getenv("ASTROFLOW_DD_IQRM_VARIANT")) P->iqrm_variant = std::atoi(v);
  // The _dedisperse_spec path's Header carries tsamp as float.
  P->tsamp = P->p.freq_mode == DD_FREQ_FIL ? header->tsamp
                                            : static_cast<double>(static_cast<float>(header->tsamp));
  P->d_err.alloc(sizeof(int));
  DD_CUDA_TRY(cudaMemset(P->d_err.p, 0, sizeof(int)));
  build_freq(*P);
  build_band(*P);
  if (P->p.algorithm == DD_ALGO_BRUTE) {
    create_brute(*P);
  } else if (P->p.algorithm == DD_ALGO_SUBBAND) {
    create_subband(*P);
    create_rfi(*P);
  } else {
    throw Error{DD_ERR_INVALID, "unknown algorithm"};
  }
  // plan set-up work ran on the legacy stream; other streams keep running
  DD_CUDA_TRY(cudaStreamSynchronize(cudaStreamLegacy));
  return P.release();
}
}  // namespace
}  // namespace dd

extern "C" {

int dd_plan_create(const dd_header* header, const dd_plan_params* params,
                   const dd_rfi_config* rfi, const int32_t* bad_channels, int32_t n_bad,
                   int32_t device, dd_plan** plan) {
  if (!plan) { set_error("plan pointer is NULL"); return DD_ERR_INVALID; }
  *plan = nullptr;
  return guarded([&] { *plan = make_plan(header, params, rfi, bad_channels, n_bad, device, 0); });
}

int dd_plan_destroy(dd_plan* plan) {
  if (!plan) return DD_OK;
  return guarded([&] {
    DeviceGuard g(plan->device);
    delete plan;
  });
}

int dd_plan_destroy_async(dd_plan* plan, void* stream) {
  if (!plan) return DD_OK;
  return guarded([&] {
    DeviceGuard g(plan->device);
    g_free_stream = static_cast<cudaStream_t>(stream);
    g_free_async = true;
    delete plan;
    g_free_async = false;
    g_free_stream = nullptr;
  });
}

int dd_plan_get_info(const dd_plan* P, dd_plan_info* info) {
  if (!P || !info) { set_error("NULL argument"); return DD_ERR_INVALID; }
  return guarded([&] {
    dd_plan_info o{};
    o.chan_start = P->cs;
    o.chan_end = P->ce;
    o.dm_steps = P->dm_steps;
    o.nsamp_in = P->nin;
    o.nsamp_binned = P->nbin;
    o.out_cols = P->p.algorithm == DD_ALGO_BRUTE ? P->out_cols : P->nout;
    o.out_elem_bytes = P->nbits == 32 ? 8 : 4;
    o.nsb = P->nsb;
    o.ndm_nom = P->ndm_nom;
    o.max_delay = P->max_delay;
    o.max_residual = P->max_res;
    o.nslices = P->nslices;
    o.n_iqrm_windows = P->rfi.use_iqrm ? static_cast<int64_t>(P->win_t0.size()) : 0;
    o.workspace_bytes = workspace_of(*P);
    o.delay_rows = P->p.algorithm == DD_ALGO_BRUTE ? P->dm_steps : P->ndm_nom;
    o.delay_cols = P->p.algorithm == DD_ALGO_BRUTE ? P->nc : P->dch;
    o.table_mismatch_fp64 = P->table_mismatch_fp64;
    o.tile_samples = P->tile;
    o.subband_sum_copies = P->p.algorithm == DD_ALGO_SUBBAND ? (P->twin ? 2 : 1) : 0;
    o.adds_per_run = P->adds;
    *info = o;
  });
}

int dd_plan_get_tables(const dd_plan* P, int32_t* delay, int32_t* residual) {
  if (!P) { set_error("NULL plan"); return DD_ERR_INVALID; }
  return guarded([&] {
    if (delay) std::memcpy(delay, P->h_delay.data(), sizeof(int32_t) * P->h_delay.size());
    if (residual && !P->h_res.empty())
      std::memcpy(residual, P->h_res.data(), sizeof(int32_t) * P->h_res.size());
  });
}

int dd_brute_delay_table(const double* freq, int64_t chan_start, int64_t chan_end,
                         int64_t ref_channel, float dm_low, float dm_step, int64_t dm_steps,
                         double tsamp, int32_t mode, int32_t* table, int64_t* mismatch_fp64) {
  if (!freq || !table) { set_error("NULL argument"); return DD_ERR_INVALID; }
  return guarded([&] {
    if (chan_start < 0 || chan_end <= chan_start || ref_channel < 0 || dm_steps < 1 ||
        !(tsamp > 0) || !(dm_step > 0))
      throw Error{DD_ERR_INVALID, "need 0 <= chan_start < chan_end, ref_channel >= 0, "
                                  "dm_steps >= 1, tsamp > 0 and dm_step > 0"};
    if (mode != DD_TABLE_REFERENCE && mode != DD_TABLE_IEEE && mode != DD_TABLE_FP64)
      throw Error{DD_ERR_INVALID, "unknown table mode"};
    const int64_t m = brute_table(freq, chan_start, chan_end, ref_channel, dm_low, dm_step,
                                  dm_steps, tsamp, mode, table);
    if (mismatch_fp64) *mismatch_fp64 = m;
  });
}

int dd_plan_set_delay_table(dd_plan* P, const int32_t* delay) {
  if (!P || !delay) { set_error("NULL argument"); return DD_ERR_INVALID; }
  return guarded([&] {
    if (P->p.algorithm != DD_ALGO_BRUTE)
      throw Error{DD_ERR_UNSUPPORTED, "delay table injection is for the brute-force algorithm"};
    DeviceGuard g(P->device);
    int mx = 0;
    for (size_t i = 0; i < P->h_delay.size(); ++i) {
      if (delay[i] < 0) throw Error{DD_ERR_INVALID, "negative delay in table"};
      mx = std::max(mx, delay[i]);
    }
    const int ds = P->p.time_downsample;
    const int64_t need = (P->nin + ds - 1) / ds + mx / ds + 96;
    if (need + tile_samples() > P->phase_len) throw Error{DD_ERR_INVALID, "delay larger than the plan's padding"};
    std::memcpy(P->h_delay.data(), delay, sizeof(int32_t) * P->h_delay.size());
    P->max_delay = mx;
    ++P->generation;
    set_brute_window(*P);
    DD_CUDA_TRY(cudaMemcpy(P->d_delay.p, delay, sizeof(int32_t) * P->h_delay.size(), cudaMemcpyHostToDevice));
  });
}

int dd_run_ex(dd_plan* P, const void* input, void* output, uint8_t* iqrm_masks,
              uint32_t* iqrm_bounds, void* prepped, void* stream) {
  if (!P || !input || !output) { set_error("NULL argument"); return DD_ERR_INVALID; }
  return guarded([&] {
    DeviceGuard g(P->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (P->p.algorithm == DD_ALGO_BRUTE) run_brute(*P, input, output, prepped, st);
    else run_subband(*P, input, output, iqrm_masks, iqrm_bounds, prepped, st);
    DD_CUDA_TRY(cudaGetLastError());
  });
}

int dd_run(dd_plan* P, const void* input, void* output, void* stream) {
  return dd_run_ex(P, input, output, nullptr, nullptr, nullptr, stream);
}

int dd_plan_autotune(dd_plan* P, const void* input, void* output, int32_t reps, void* stream,
                     dd_tune_report* report) {
  if (!P || !input || !output || !report) { set_error("NULL argument"); return DD_ERR_INVALID; }
  return guarded([&] {
    DeviceGuard g(P->device);
    if (P->p.algorithm != DD_ALGO_SUBBAND || !P->win1 || !P->win2)
      throw Error{DD_ERR_UNSUPPORTED, "autotuning covers the staged subband path"};
    if (reps < 1) throw Error{DD_ERR_INVALID, "reps must be >= 1"};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaEvent_t e0, e1;
    DD_CUDA_TRY(cudaEventCreate(&e0));
    DD_CUDA_TRY(cudaEventCreate(&e1));
    auto time_shape = [&]() -> double {
      run_subband(*P, input, output, nullptr, nullptr, nullptr, st);  // warm-up
      DD_CUDA_TRY(cudaEventRecord(e0, st));
      for (int i = 0; i < reps; ++i) run_subband(*P, input, output, nullptr, nullptr, nullptr, st);
      DD_CUDA_TRY(cudaEventRecord(e1, st));
      DD_CUDA_TRY(cudaEventSynchronize(e1));
      float ms = 0;
      DD_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
      check_device_error(*P, st);
      return static_cast<double>(ms) / reps;
    };
    // stage counts that keep two blocks per SM for both stages
    auto fits = [&](int S) {
      if (S < 2 || S > kSumMaxStages) return false;
      SumLaunch l1 = stage1_launch(*P, 0), l2 = stage2_launch(*P, 0, output);
      l1.stages = l2.stages = S;
      return sum_launch_smem(l1) <= 113 * 1024 && sum_launch_smem(l2) <= 113 * 1024;
    };
    const int64_t budget0 = P->inter_budget;
    const int stages0 = P->stages_override;
    dd_tune_report rep{};
    rep.default_ms = time_shape();
    rep.best_ms = rep.default_ms;
    rep.best_budget_bytes = budget0;
    rep.best_tile_samples = P->tile;
    rep.best_stages = stages0;
    rep.candidates = 1;
    std::vector<int64_t> tiles_seen;
    for (int64_t budget : {int64_t(512) << 20, int64_t(1) << 30, int64_t(2) << 30, int64_t(4) << 30}) {
      try {
        set_tiling(*P, budget);
      } catch (const Error& e) {
        if (e.code != DD_ERR_NOMEM) throw;
        continue;  // does not fit: skip
      }
      if (std::find(tiles_seen.begin(), tiles_seen.end(), P->tile) != tiles_seen.end()) continue;
      tiles_seen.push_back(P->tile);
      for (int S : {0, 4, 6, 8}) {
        if (S && !fits(S)) continue;
        if (budget == budget0 && S == stages0) continue;  // the default, timed already
        P->stages_override = S;
        const double ms = time_shape();
        ++rep.candidates;
        if (ms < rep.best_ms) {
          rep.best_ms = ms;
          rep.best_budget_bytes = budget;
          rep.best_tile_samples = P->tile;
          rep.best_stages = S;
        }
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // keep the fastest shape
    P->stages_override = rep.best_stages;
    set_tiling(*P, rep.best_budget_bytes);
    ++P->generation;
    *report = rep;
  });
}

int dd_launch_count(int64_t* count) {
  if (!count) { set_error("NULL argument"); return DD_ERR_INVALID; }
  *count = launch_count();
  return DD_OK;
}

int dd_run_profiled(dd_plan* P, const void* input, void* output, void* stream,
                    dd_run_stats* stats) {
  if (!P || !input || !output || !stats) { set_error("NULL argument"); return DD_ERR_INVALID; }
  return guarded([&] {
    DeviceGuard g(P->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Prof pf{*P, st};
    const long long l0 = launch_count();
    cudaEvent_t t0 = pf.mark();
    if (P->p.algorithm == DD_ALGO_BRUTE) run_brute(*P, input, output, nullptr, st, &pf);
    else run_subband(*P, input, output, nullptr, nullptr, nullptr, st, &pf);
    cudaEvent_t t1 = pf.mark();
    DD_CUDA_TRY(cudaEventSynchronize(t1));
    dd_run_stats o{};
    DD_CUDA_TRY(cudaEventElapsedTime(&o.total_ms, t0, t1));
    o.prep_ms = Prof::sum(pf.prep);
    o.stage1_ms = Prof::sum(pf.s1);
    o.stage2_ms = Prof::sum(pf.s2);
    o.launches = static_cast<int32_t>(launch_count() - l0);
    o.stage1_launches = static_cast<int32_t>(pf.s1.size());
    o.stage2_launches = P->p.algorithm == DD_ALGO_BRUTE
                            ? static_cast<int32_t>((P->winb || P->phases_merge) ? 1 : P->nslices)
                            : static_cast<int32_t>(pf.s2.size());
    check_device_error(*P, st);
    *stats = o;
  });
}

int dd_measure_int_add_rate(int32_t device, double* adds_per_second) {
  if (!adds_per_second) { set_error("NULL argument"); return DD_ERR_INVALID; }
  return guarded([&] {
    DeviceGuard g(device);
    *adds_per_second = measure_int_add_rate(device);
  });
}

namespace {
// Queues one host-path run on `st`: input copy, run, output copies (each time
// tile's columns on the plan's copy stream while the next tile is summed).  Each
// time tile's sums wait for the earlier queued run's copy of the same output
// columns (they write the same device output), the input copy and RFI stages do
// not: consecutive runs overlap one run's output copy with the next one's input
// copy, and the output copies run back to back.  P.host_done marks this run's
// last output copy.
void enqueue_host_run(dd_plan& P, const void* h_input, void* h_output, cudaStream_t st) {
  const size_t in_bytes = static_cast<size_t>(P.nin * P.hdr.nchans) * P.elem;
  const int64_t cols = P.p.algorithm == DD_ALGO_BRUTE ? P.out_cols : P.nout;
  const size_t oelem = P.nbits == 32 ? 8 : 4;
  const size_t out_bytes = static_cast<size_t>(P.dm_steps) * cols * oelem;
  // device buffers of the host path, kept by the plan across calls
  if (P.d_host_in.bytes < in_bytes || P.d_host_out.bytes < out_bytes) {
    // earlier queued runs may still use the old buffers
    if (P.copy_stream) DD_CUDA_TRY(cudaStreamSynchronize(P.copy_stream));
    DD_CUDA_TRY(cudaStreamSynchronize(st));
    P.host_pending = false;
  }
  if (P.d_host_in.bytes < in_bytes) P.d_host_in.alloc(in_bytes);
  if (P.d_host_out.bytes < out_bytes) {
    P.d_host_out.release();
    try {
      P.d_host_out.alloc(out_bytes);
    } catch (const Error& er) {
      throw Error{DD_ERR_NOMEM, "output allocation failed: " + er.msg};
    }
  }
  // buffers are allocated stream-ordered on the legacy stream: make them visible to `st`
  DD_CUDA_TRY(cudaStreamSynchronize(cudaStreamLegacy));
  char* d_out = P.d_host_out.as<char>();
  if (!P.copy_stream) DD_CUDA_TRY(cudaStreamCreateWithFlags(&P.copy_stream, cudaStreamNonBlocking));
  if (!P.host_done) DD_CUDA_TRY(cudaEventCreateWithFlags(&P.host_done, cudaEventDisableTiming));
  auto wait_output_free = [&]() {
    if (P.host_pending) DD_CUDA_TRY(cudaStreamWaitEvent(st, P.host_done, 0));
  };
  DD_CUDA_TRY(cudaMemcpyAsync(P.d_host_in.p, h_input, in_bytes, cudaMemcpyHostToDevice, st));
  if (P.p.algorithm == DD_ALGO_BRUTE) {
    wait_output_free();
    run_brute(P, P.d_host_in.p, d_out, nullptr, st);
    cudaEvent_t ev;
    DD_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    DD_CUDA_TRY(cudaEventRecord(ev, st));
    DD_CUDA_TRY(cudaStreamWaitEvent(P.copy_stream, ev, 0));
    cudaEventDestroy(ev);
    DD_CUDA_TRY(cudaMemcpyAsync(h_output, d_out, out_bytes, cudaMemcpyDeviceToHost, P.copy_stream));
  } else {
    // each tile's sums wait only for the earlier run's copy of the same columns
    // (events kept per tile; any other tiling waits for the earlier run's last copy)
    std::vector<cudaEvent_t> evs, copied;
    auto cleanup = [&]() {
      for (cudaEvent_t ev : evs) cudaEventDestroy(ev);
      for (cudaEvent_t ev : copied) cudaEventDestroy(ev);
    };
    const bool same_tiling = P.host_pending && P.host_tile == P.tile &&
                             P.host_tile_copied.size() == static_cast<size_t>((P.nout + P.tile - 1) / P.tile);
    try {
      run_subband(P, P.d_host_in.p, d_out, nullptr, nullptr, nullptr, st, nullptr,
                  [&](int64_t t0, int64_t n) {
                    cudaEvent_t ev, done;
                    DD_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
                    evs.push_back(ev);
                    DD_CUDA_TRY(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
                    copied.push_back(done);
                    DD_CUDA_TRY(cudaEventRecord(ev, st));
                    DD_CUDA_TRY(cudaStreamWaitEvent(P.copy_stream, ev, 0));
                    const size_t pitch = static_cast<size_t>(cols) * oelem;
                    DD_CUDA_TRY(cudaMemcpy2DAsync(static_cast<char*>(h_output) + t0 * oelem, pitch,
                                                  d_out + t0 * oelem, pitch, n * oelem,
                                                  static_cast<size_t>(P.dm_steps),
                                                  cudaMemcpyDeviceToHost, P.copy_stream));
                    DD_CUDA_TRY(cudaEventRecord(done, P.copy_stream));
                  },
                  [&]() {
                    if (!same_tiling) wait_output_free();
                  },
                  [&](int64_t t0, int64_t) {
                    if (same_tiling)
                      DD_CUDA_TRY(cudaStreamWaitEvent(st, P.host_tile_copied[t0 / P.tile], 0));
                  });
    } catch (...) {
      cudaStreamSynchronize(P.copy_stream);
      cleanup();
      P.host_pending = false;
      throw;
    }
    for (cudaEvent_t ev : evs) cudaEventDestroy(ev);
    for (cudaEvent_t ev : P.host_tile_copied) cudaEventDestroy(ev);
    P.host_tile_copied.swap(copied);
    P.host_tile = P.tile;
  }
  DD_CUDA_TRY(cudaEventRecord(P.host_done, P.copy_stream));
  P.host_pending = true;
}

// Makes `st` wait for every host-path output copy queued so far.
void join_host_runs(dd_plan& P, cudaStream_t st) {
  if (P.host_pending) DD_CUDA_TRY(cudaStreamWaitEvent(st, P.host_done, 0));
}
}  // namespace

int dd_run_host(dd_plan* P, const void* h_input, void* h_output, void* stream) {
  if (!P || !h_input || !h_output) { set_error("NULL argument"); return DD_ERR_INVALID; }
  return guarded([&] {
    DeviceGuard g(P->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    enqueue_host_run(*P, h_input, h_output, st);
    join_host_runs(*P, st);
    DD_CUDA_TRY(cudaStreamSynchronize(st));
    P->host_pending = false;
    check_device_error(*P, st);
  });
}

int dd_run_host_async(dd_plan* P, const void* h_input, void* h_output, void* stream) {
  if (!P || !h_input || !h_output) { set_error("NULL argument"); return DD_ERR_INVALID; }
  return guarded([&] {
    DeviceGuard g(P->device);
    enqueue_host_run(*P, h_input, h_output, static_cast<cudaStream_t>(stream));
  });
}

int dd_run_host_join(dd_plan* P, void* stream, int32_t sync) {
  if (!P) { set_error("NULL argument"); return DD_ERR_INVALID; }
  return guarded([&] {
    DeviceGuard g(P->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    join_host_runs(*P, st);
    if (sync) {
      DD_CUDA_TRY(cudaStreamSynchronize(st));
      P->host_pending = false;
      check_device_error(*P, st);
    }
  });
}

}  // extern "C"

// ---------------------------------------------------------------- batches
// A batch runs one chunk through each of its plans.  Every plan's RFI and layout
// kernels run first; then the dedispersion sums of all plans run batched:
//  * grouped (default): one launch per (time tile, stage, kernel variant) over
//    that stage of every plan, stage 1 of the first tiles, stage 2 of the first
//    tiles, stage 1 of the second tiles, ... (stream order keeps each plan's
//    stages in sequence);
//  * persistent (DD_BATCH_PERSISTENT): a single launch (k_sum_batch) over all
//    of them, a plan's dependent stages ordered by completion counters.
// Plans whose sums cannot be batched (32-bit samples, windows wider than the
// staged kernels take, or in persistent mode wider than two resident blocks per
// SM allow) run their own kernels in the same run.  With DD_BATCH_GRAPH the
// whole sequence is captured into a CUDA graph on the batch's own stream and
// replayed while the caller passes the same buffers.
struct dd_batch {
  int device = 0;
  std::vector<dd_plan*> plans;
  std::vector<int64_t> generations;
  bool use_graph = true;
  bool persistent = false;
  cudaStream_t st = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  cudaGraphExec_t exec = nullptr;
  int captures = 0;
  std::vector<const void*> cur_in;
  std::vector<void*> cur_out;
  bool table_ready = false;
  std::vector<dd::SumBatchGroup> groups;
  struct Launch {  // one batched sum launch over groups [begin, end)
    int begin = 0, end = 0;
    long long blocks = 0;
    size_t smem = 0;
    int kind = 0;
    unsigned grid = 0;  // persistent launch: resident blocks
  };
  std::vector<Launch> sums;
  std::vector<char> own;  // per plan: runs its own kernels
  int nctrs = 0;
  long long blocks = 0;
  int64_t launches = 0;
  dd::DevBuf d_groups, d_ctrs, d_next, d_err;
  ~dd_batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (ev_in) cudaEventDestroy(ev_in);
    if (ev_out) cudaEventDestroy(ev_out);
    if (st) cudaStreamDestroy(st);
  }
};

namespace dd {
namespace {

// Shared memory of a staged sum that leaves two persistent blocks per SM.
constexpr size_t kBatchSmemCap = 100 * 1024;


// Whether plan P's sums run in the batched launches.
bool batched_plan(const dd_plan& P, bool persistent) {
  if (P.nbits > 16) return false;
  const bool brute = P.p.algorithm == DD_ALGO_BRUTE;
  if (brute ? !P.winb : (!P.win1 || !P.win2)) return false;
  if (!persistent) return true;
  return brute ? sum_launch_smem(brute_launch(P, nullptr)) <= kBatchSmemCap
               : sum_launch_smem(stage1_launch(P, 0)) <= kBatchSmemCap &&
                     sum_launch_smem(stage2_launch(P, 0, nullptr)) <= kBatchSmemCap;
}

long long group_blocks(const SumBatchGroup& g) {
  return static_cast<long long>(g.gx) * g.L.grid_y * g.L.grid_z;
}

SumBatchGroup make_group(const SumLaunch& L) {
  SumBatchGroup g{};
  g.L = L;
  g.kind = sum_kind(L);
  g.gx = sum_grid_x(L);
  g.wait_ctr = -1;
  return g;
}

// The batched sums for the given outputs (stage-2 / brute-force sums write there).
void build_groups(dd_batch& B, void* const* outputs) {
  B.groups.clear();
  B.sums.clear();
  const int n = static_cast<int>(B.plans.size());
  B.own.assign(n, 0);
  for (int p = 0; p < n; ++p) B.own[p] = batched_plan(*B.plans[p], B.persistent) ? 0 : 1;
  int64_t max_tiles = 1;
  for (int p = 0; p < n; ++p)
    if (!B.own[p] && B.plans[p]->p.algorithm == DD_ALGO_SUBBAND)
      max_tiles = std::max<int64_t>(max_tiles, (B.plans[p]->nout + B.plans[p]->tile - 1) / B.plans[p]->tile);
  // The sums of one stage of every plan, tile by tile: stage[k][0] = stage 1 of tile
  // k, stage[k][1] = stage 2 of tile k (and the brute-force sums at k = 0).
  std::vector<std::vector<std::pair<int, SumLaunch>>> stage(2 * max_tiles);
  for (int64_t k = 0; k < max_tiles; ++k)
    for (int p = 0; p < n; ++p) {
      const dd_plan& P = *B.plans[p];
      if (B.own[p]) continue;
      if (P.p.algorithm == DD_ALGO_BRUTE) {
        if (k == 0) stage[1].emplace_back(p, brute_launch(P, outputs[p]));
        continue;
      }
      if (k * P.tile >= P.nout) continue;
      stage[2 * k].emplace_back(p, stage1_launch(P, k * P.tile));
      stage[2 * k + 1].emplace_back(p, stage2_launch(P, k * P.tile, outputs[p]));
    }
  int dev = 0, sms = 0;
  DD_CUDA_TRY(cudaGetDevice(&dev));
  DD_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  B.nctrs = 0;
  if (B.persistent) {
    dd_batch::Launch la;
    la.begin = 0;
    std::vector<int> prev_ctr(n, -1), prev_need(n, 0), s1_ctr(n, -1), s1_need(n, 0);
    for (size_t st = 0; st < stage.size(); ++st)
      for (auto& [p, L] : stage[st]) {
        SumBatchGroup g = make_group(L);
        const bool s1 = (st % 2) == 0;
        const bool brute = B.plans[p]->p.algorithm == DD_ALGO_BRUTE;
        // stage 1 of tile k overwrites the sums stage 2 of tile k-1 reads;
        // stage 2 of tile k reads what stage 1 of tile k wrote
        if (!brute) {
          g.wait_ctr = s1 ? prev_ctr[p] : s1_ctr[p];
          g.wait_need = s1 ? prev_need[p] : s1_need[p];
        }
        g.first = la.blocks;
        g.done_ctr = B.nctrs++;
        la.blocks += group_blocks(g);
        la.smem = std::max(la.smem, sum_launch_smem(L));
        if (!brute) {
          (s1 ? s1_ctr[p] : prev_ctr[p]) = g.done_ctr;
          (s1 ? s1_need[p] : prev_need[p]) = static_cast<int>(group_blocks(g));
        }
        B.groups.push_back(g);
      }
    la.end = static_cast<int>(B.groups.size());
    if (la.end > 0) {
      const int per_sm = std::max(1, sum_batch_blocks_per_sm(la.smem));
      la.grid = static_cast<unsigned>(std::min<long long>(static_cast<long long>(sms) * per_sm, la.blocks));
      B.sums.push_back(la);
    }
  } else {
    for (auto& list : stage) {
      // one launch per kernel variant; windows too wide for two blocks per SM get
      // their own launch so they do not lower the others' occupancy
      for (int kind = 0; kind < kSumKinds; ++kind)
        for (int wide = 0; wide < 2; ++wide) {
          dd_batch::Launch la;
          la.begin = static_cast<int>(B.groups.size());
          la.kind = kind;
          for (auto& [p, L] : list) {
            SumBatchGroup g = make_group(L);
            const size_t sm = sum_launch_smem(L);
            if (g.kind != kind || (sm > kBatchSmemCap) != (wide != 0)) continue;
            g.first = la.blocks;
            la.blocks += group_blocks(g);
            la.smem = std::max(la.smem, sm);
            B.groups.push_back(g);
          }
          la.end = static_cast<int>(B.groups.size());
          if (la.end > la.begin) B.sums.push_back(la);
        }
    }
  }
  B.blocks = 0;
  for (const auto& la : B.sums) B.blocks += la.blocks;
  if (B.groups.empty()) return;
  B.d_groups.alloc(sizeof(SumBatchGroup) * B.groups.size());
  DD_CUDA_TRY(cudaMemcpy(B.d_groups.p, B.groups.data(), sizeof(SumBatchGroup) * B.groups.size(),
                         cudaMemcpyHostToDevice));
  if (B.persistent) {
    B.d_ctrs.alloc(sizeof(int) * std::max(B.nctrs, 1));
    B.d_next.alloc(sizeof(unsigned long long));
  }
  DD_CUDA_TRY(cudaStreamSynchronize(cudaStreamLegacy));
}

// Everything one run launches, on stream s.
void enqueue_batch(dd_batch& B, const void* const* inputs, void* const* outputs,
                   cudaStream_t s) {
  const long long l0 = launch_count();
  for (size_t p = 0; p < B.plans.size(); ++p) {
    dd_plan& P = *B.plans[p];
    const bool brute = P.p.algorithm == DD_ALGO_BRUTE;
    if (B.own[p]) {
      if (brute) run_brute(P, inputs[p], outputs[p], nullptr, s);
      else run_subband(P, inputs[p], outputs[p], nullptr, nullptr, nullptr, s);
    } else if (brute) {
      run_brute_prep(P, inputs[p], nullptr, s);
    } else {
      run_rfi_and_prep(P, inputs[p], nullptr, nullptr, nullptr, s);
    }
  }
  const SumBatchGroup* dg = B.d_groups.as<SumBatchGroup>();
  for (const auto& la : B.sums) {
    if (B.persistent) {
      DD_CUDA_TRY(cudaMemsetAsync(B.d_ctrs.p, 0, B.d_ctrs.bytes, s));
      DD_CUDA_TRY(cudaMemsetAsync(B.d_next.p, 0, B.d_next.bytes, s));
      launch_sum_batch(dg + la.begin, la.end - la.begin, la.blocks, B.d_ctrs.as<int>(),
                       B.d_next.as<unsigned long long>(), B.d_err.as<int>(), la.smem, la.grid, s);
    } else {
      launch_sum_grouped(dg + la.begin, la.end - la.begin, la.blocks, la.kind, la.smem, s);
    }
  }
  B.launches = launch_count() - l0;
}

}  // namespace
}  // namespace dd

extern "C" {

int dd_batch_create(dd_plan* const* plans, int32_t nplans, int32_t flags, dd_batch** batch) {
  if (!plans || nplans < 1 || !batch) { set_error("NULL argument"); return DD_ERR_INVALID; }
  dd_batch* B = nullptr;
  const int rc = guarded([&] {
    if (flags & ~(DD_BATCH_GRAPH | DD_BATCH_PERSISTENT)) throw Error{DD_ERR_INVALID, "unknown batch flags"};
    for (int i = 0; i < nplans; ++i) {
      if (!plans[i]) throw Error{DD_ERR_INVALID, "NULL plan"};
      if (plans[i]->device != plans[0]->device)
        throw Error{DD_ERR_INVALID, "all plans of a batch must be on one device"};
      for (int j = 0; j < i; ++j)
        if (plans[j] == plans[i]) throw Error{DD_ERR_INVALID, "a plan appears twice in the batch"};
    }
    DeviceGuard g(plans[0]->device);
    B = new dd_batch();
    B->device = plans[0]->device;
    B->plans.assign(plans, plans + nplans);
    B->use_graph = (flags & DD_BATCH_GRAPH) != 0;
    B->persistent = (flags & DD_BATCH_PERSISTENT) != 0;
    DD_CUDA_TRY(cudaStreamCreateWithFlags(&B->st, cudaStreamNonBlocking));
    DD_CUDA_TRY(cudaEventCreateWithFlags(&B->ev_in, cudaEventDisableTiming));
    DD_CUDA_TRY(cudaEventCreateWithFlags(&B->ev_out, cudaEventDisableTiming));
    B->d_err.alloc(sizeof(int));
    DD_CUDA_TRY(cudaMemsetAsync(B->d_err.p, 0, sizeof(int), cudaStreamLegacy));
    DD_CUDA_TRY(cudaStreamSynchronize(cudaStreamLegacy));
  });
  if (rc != DD_OK) {
    delete B;
    return rc;
  }
  *batch = B;
  return DD_OK;
}

int dd_batch_destroy(dd_batch* batch) {
  if (!batch) return DD_OK;
  return guarded([&] {
    DeviceGuard g(batch->device);
    delete batch;
  });
}

int dd_batch_run(dd_batch* B, const void* const* inputs, void* const* outputs, void* stream) {
  if (!B || !inputs || !outputs) { set_error("NULL argument"); return DD_ERR_INVALID; }
  return guarded([&] {
    DeviceGuard g(B->device);
    const size_t n = B->plans.size();
    for (size_t p = 0; p < n; ++p)
      if (!inputs[p] || !outputs[p]) throw Error{DD_ERR_INVALID, "NULL input or output buffer"};
    std::vector<int64_t> gens(n);
    for (size_t p = 0; p < n; ++p) gens[p] = B->plans[p]->generation;
    const bool same = B->table_ready && gens == B->generations &&
                      std::equal(B->cur_in.begin(), B->cur_in.end(), inputs) &&
                      std::equal(B->cur_out.begin(), B->cur_out.end(), outputs);
    cudaStream_t user = static_cast<cudaStream_t>(stream);
    if (!same) {
      // the previous run may still read the old table
      DD_CUDA_TRY(cudaStreamSynchronize(B->st));
      build_groups(*B, outputs);
      B->cur_in.assign(inputs, inputs + n);
      B->cur_out.assign(outputs, outputs + n);
      B->generations = gens;
      B->table_ready = true;
      if (B->exec) {
        DD_CUDA_TRY(cudaGraphExecDestroy(B->exec));
        B->exec = nullptr;
      }
    }
    DD_CUDA_TRY(cudaEventRecord(B->ev_in, user));
    DD_CUDA_TRY(cudaStreamWaitEvent(B->st, B->ev_in, 0));
    if (B->use_graph) {
      if (!B->exec) {
        cudaGraph_t graph = nullptr;
        DD_CUDA_TRY(cudaStreamBeginCapture(B->st, cudaStreamCaptureModeThreadLocal));
        try {
          enqueue_batch(*B, inputs, outputs, B->st);
        } catch (...) {
          cudaStreamEndCapture(B->st, &graph);
          if (graph) cudaGraphDestroy(graph);
          throw;
        }
        DD_CUDA_TRY(cudaStreamEndCapture(B->st, &graph));
        const cudaError_t e = cudaGraphInstantiate(&B->exec, graph, 0);
        cudaGraphDestroy(graph);
        DD_CUDA_TRY(e);
        ++B->captures;
      }
      DD_CUDA_TRY(cudaGraphLaunch(B->exec, B->st));
    } else {
      enqueue_batch(*B, inputs, outputs, B->st);
    }
    DD_CUDA_TRY(cudaEventRecord(B->ev_out, B->st));
    DD_CUDA_TRY(cudaStreamWaitEvent(user, B->ev_out, 0));
  });
}

int dd_batch_status(dd_batch* B) {
  if (!B) { set_error("NULL argument"); return DD_ERR_INVALID; }
  return guarded([&] {
    DeviceGuard g(B->device);
    DD_CUDA_TRY(cudaStreamSynchronize(B->st));
    int e = 0;
    DD_CUDA_TRY(cudaMemcpy(&e, B->d_err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
      DD_CUDA_TRY(cudaMemset(B->d_err.p, 0, sizeof(int)));
      throw Error{DD_ERR_RUNTIME, "a batched group timed out waiting for its inputs"};
    }
    for (dd_plan* P : B->plans) check_device_error(*P, B->st);
  });
}

int dd_batch_get_info(const dd_batch* B, dd_batch_info* info) {
  if (!B || !info) { set_error("NULL argument"); return DD_ERR_INVALID; }
  dd_batch_info o{};
  o.nplans = static_cast<int64_t>(B->plans.size());
  o.groups = static_cast<int64_t>(B->groups.size());
  o.blocks = B->blocks;
  o.sum_launches = static_cast<int64_t>(B->sums.size());
  o.launches = B->launches;
  int64_t own = 0;
  for (char c : B->own) own += c;
  o.own_plans = own;
  o.graph = B->use_graph ? 1 : 0;
  o.persistent = B->persistent ? 1 : 0;
  o.graph_captures = B->captures;
  *info = o;
  return DD_OK;
}

}  // extern "C"


// ---------------------------------------------------------------- streams
// A stream dedisperses a beam chunk by chunk.  It keeps the last `tail` input
// samples of the beam on the device (tail = the plan's largest total delay,
// stage-1 delay plus stage-2 shift, in input samples) and runs each push as the
// plain call on [tail | chunk], keeping the first chunk/ds output columns: those
// are the columns whose every delayed sample lies inside the buffer.  Push k's
// column t is the beam's binned time (samples pushed before push k - tail)/ds + t,
// so the first tail/ds columns of the beam come from a zero-filled tail.
struct dd_stream {
  dd_plan* plan = nullptr;
  int device = 0;
  int64_t chunk = 0, tail = 0, buf_len = 0;  // input samples
  int64_t row_bytes = 0;                     // bytes per input sample (all channels)
  dd::DevBuf buf[2];
  int cur = 0;
  int64_t pushed = 0;
};

extern "C" {

int dd_stream_open(const dd_header* header, const dd_plan_params* params, const dd_rfi_config* rfi,
                   const int32_t* bad_channels, int32_t n_bad, int32_t device, dd_stream** out) {
  if (!out || !header || !params) { set_error("NULL argument"); return DD_ERR_INVALID; }
  *out = nullptr;
  dd_stream* S = nullptr;
  const int rc = guarded([&] {
    if (params->algorithm != DD_ALGO_SUBBAND)
      throw Error{DD_ERR_UNSUPPORTED, "streams run the subband algorithm"};
    const int ds = params->time_downsample;
    if (ds < 1 || header->ndata < 1 || header->ndata % ds != 0)
      throw Error{DD_ERR_INVALID, "the chunk length (header ndata) must be a positive multiple "
                                  "of time_downsample"};
    DeviceGuard g(device);
    // the delays set the tail: learn them from a plan over one chunk
    std::unique_ptr<dd_plan> probe(make_plan(header, params, rfi, bad_channels, n_bad, device, 0));
    const int64_t tail_bin = static_cast<int64_t>(probe->max_delay) + probe->max_res;
    probe.reset();
    S = new dd_stream();
    S->device = device;
    S->chunk = header->ndata;
    S->tail = tail_bin * ds;
    S->buf_len = S->tail + S->chunk;
    S->row_bytes = static_cast<int64_t>(header->nchans) * (header->nbits / 8);
    dd_header h = *header;
    h.ndata = S->buf_len;
    S->plan = make_plan(&h, params, rfi, bad_channels, n_bad, device, S->chunk / ds);
    for (int b = 0; b < 2; ++b) {
      S->buf[b].alloc(static_cast<size_t>(S->buf_len * S->row_bytes));
      DD_CUDA_TRY(cudaMemsetAsync(S->buf[b].p, 0, S->buf[b].bytes, cudaStreamLegacy));
    }
    DD_CUDA_TRY(cudaStreamSynchronize(cudaStreamLegacy));
  });
  if (rc != DD_OK) {
    if (S) {
      DeviceGuard g(device);
      delete S->plan;
      delete S;
    }
    return rc;
  }
  *out = S;
  return DD_OK;
}

int dd_stream_push(dd_stream* S, const void* chunk, void* output, void* stream) {
  if (!S || !chunk || !output) { set_error("NULL argument"); return DD_ERR_INVALID; }
  return guarded([&] {
    DeviceGuard g(S->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    char* cur = static_cast<char*>(S->buf[S->cur].p);
    char* nxt = static_cast<char*>(S->buf[S->cur ^ 1].p);
    DD_CUDA_TRY(cudaMemcpyAsync(cur + S->tail * S->row_bytes, chunk,
                                static_cast<size_t>(S->chunk * S->row_bytes),
                                cudaMemcpyDeviceToDevice, st));
    run_subband(*S->plan, cur, output, nullptr, nullptr, nullptr, st);
    // the next buffer starts with this buffer's last `tail` samples
    if (S->tail)
      DD_CUDA_TRY(cudaMemcpyAsync(nxt, cur + S->chunk * S->row_bytes,
                                  static_cast<size_t>(S->tail * S->row_bytes),
                                  cudaMemcpyDeviceToDevice, st));
    S->cur ^= 1;
    S->pushed += S->chunk;
  });
}

int dd_stream_get_info(const dd_stream* S, dd_stream_info* info) {
  if (!S || !info) { set_error("NULL argument"); return DD_ERR_INVALID; }
  dd_stream_info o{};
  o.dm_steps = S->plan->dm_steps;
  o.out_cols = S->plan->nout;
  o.chunk_samples = S->chunk;
  o.tail_samples = S->tail;
  o.pushed_samples = S->pushed;
  o.workspace_bytes = workspace_of(*S->plan) + static_cast<int64_t>(S->buf[0].bytes + S->buf[1].bytes);
  o.adds_per_push = S->plan->adds;
  *info = o;
  return DD_OK;
}

int dd_stream_plan(const dd_stream* S, dd_plan** plan) {
  if (!S || !plan) { set_error("NULL argument"); return DD_ERR_INVALID; }
  *plan = S->plan;
  return DD_OK;
}

int dd_stream_close(dd_stream* S) {
  if (!S) return DD_OK;
  return guarded([&] {
    DeviceGuard g(S->device);
    delete S->plan;
    S->plan = nullptr;
    delete S;
  });
}

}  // extern "C"
