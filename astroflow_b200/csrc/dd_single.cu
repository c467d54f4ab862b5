// Single-DM dedispersed spectrum of a time window, for candidate plots:
// cpucal::dedisperse_spec_with_dm (include/cpucal.hpp:341-483, Header input) and
// cpucal::dedispered_fil_with_dm (include/cpucal.hpp:203-339, Filterbank input).
//
// Per selected channel c the spectrum is the channel shifted by its delay at
// one DM: out[ti][c - chan_start] = x[t_start + ti + delay(c)][c].  Before the
// gather the reference runs IQRM and the mask file on an extended slice of the
// input, [t_start - max_delay, ... + 2 max_delay), zeroing those samples in the
// caller's array; here the slice is copied to device scratch, processed there
// (the same IQRM kernels as the plan path), optionally copied to `masked_rows`
// (what the reference leaves in the caller's array), and gathered from.
//
// Geometry and delays are host code in the reference's arithmetic: float
// frequencies, the linear frequency-to-channel map with its 1e-9 guard, and
// delay = lround(4148.808f * dm * (1/f^2 - 1/f_high^2) / tsamp) with f_high the
// highest selected frequency, evaluated as IEEE float operations.  The two
// multiply-adds the reference build (-ffast-math with FMA) contracts are FMAs
// here too: the Header frequency table fch1 + i*foff and tend = tstart +
// ntimes*tsamp.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "dd_internal.h"

namespace dd {
namespace {

template <typename T>
__global__ void k_gather_single(const T* __restrict__ x, int64_t nchans, int64_t row0,
                                int64_t cs, int64_t nsel, const int32_t* __restrict__ delay,
                                int64_t ntimes, T* __restrict__ out) {
  const int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (j >= nsel) return;
  const int64_t d = delay[j];
  for (int64_t ti = blockIdx.y; ti < ntimes; ti += gridDim.y)
    out[ti * nsel + j] = x[(row0 + ti + d) * nchans + cs + j];
}

struct Geometry {
  int64_t t_start, ntimes, cs, nsel, rfi_t0, rfi_len;
  float tend, fs, fe;
  std::vector<int32_t> delay;
};

int64_t freq_to_index(float f, float f0, float fN, int64_t nchans) {
  volatile float df = f - f0, dn = fN - f0;
  const double pos = static_cast<double>(df) / static_cast<double>(dn);
  double raw = pos * static_cast<double>(nchans - 1);
  if (raw < 0.0) raw = 0.0;
  if (raw > static_cast<double>(nchans - 1)) raw = static_cast<double>(nchans - 1);
  return static_cast<int64_t>(std::floor(raw + 1e-9));
}

Geometry geometry(const dd_header& h, const dd_single_dm_params& q) {
  const bool fil = q.freq_mode == DD_FREQ_FIL;
  const int64_t n = h.nchans;
  if (n < 1 || h.ndata < 1 || !(h.tsamp > 0)) throw Error{DD_ERR_INVALID, "bad header"};
  if (!(q.tend > q.tstart)) throw Error{DD_ERR_INVALID, "tend must be > tstart"};
  // frequency table: float fch1 + i*foff (Header), or the file's double table
  std::vector<float> freq(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i) {
    if (fil && q.freq_table) {
      freq[i] = static_cast<float>(q.freq_table[i]);
    } else if (fil) {
      freq[i] = static_cast<float>(std::fma(static_cast<double>(i), h.foff, h.fch1));
    } else {
      freq[i] = std::fmaf(static_cast<float>(i), static_cast<float>(h.foff), static_cast<float>(h.fch1));
    }
  }
  // sample indices: float / float (Header) or float / double (Filterbank)
  int64_t t0, t1;
  if (fil) {
    t0 = static_cast<int64_t>(static_cast<double>(q.tstart) / h.tsamp);
    t1 = static_cast<int64_t>(static_cast<double>(q.tend) / h.tsamp);
  } else {
    volatile float a = q.tstart / static_cast<float>(h.tsamp), b = q.tend / static_cast<float>(h.tsamp);
    t0 = static_cast<int64_t>(a);
    t1 = static_cast<int64_t>(b);
  }
  const int64_t t_len_req = t1 > t0 ? t1 - t0 : 0;
  if (t_len_req == 0 || t0 >= h.ndata) throw Error{DD_ERR_INVALID, "Invalid time window for this file."};
  if (!fil) {
    if (q.freq_start >= q.freq_end) throw Error{DD_ERR_INVALID, "freq_end must be > freq_start"};
    if (q.dm < 0.0f) throw Error{DD_ERR_INVALID, "dm must be >= 0"};
    if (h.foff < 0)
      throw Error{DD_ERR_INVALID,
                  "frequency channels are in descending order, which is not supported yet."};
  }
  const float f0 = freq.front(), fN = freq.back();
  const float fmin = std::min(f0, fN), fmax = std::max(f0, fN);
  if (q.freq_start < fmin || q.freq_end > fmax || q.freq_end <= q.freq_start) {
    char buf[256];
    std::snprintf(buf, sizeof(buf), fil ? "Frequency range [%.3f, %.3f] MHz is out of file range [%.3f, %.3f] MHz"
                                        : "Frequency range [%.3f, %.3f] MHz out of file range [%.3f, %.3f] MHz",
                  q.freq_start, q.freq_end, fmin, fmax);
    throw Error{DD_ERR_INVALID, buf};
  }
  int64_t cs = freq_to_index(q.freq_start, f0, fN, n);
  int64_t ce_incl = freq_to_index(q.freq_end, f0, fN, n);
  if (ce_incl < cs) std::swap(cs, ce_incl);
  const int64_t ce = std::min(ce_incl + 1, n);
  const int64_t nsel = ce > cs ? ce - cs : 0;
  if (nsel == 0) throw Error{DD_ERR_INVALID, "Empty channel selection."};
  const float f_high = std::max(freq[cs], freq[ce - 1]);
  Geometry g;
  g.delay.resize(static_cast<size_t>(nsel));
  int dmax = 0;
  for (int64_t c = cs; c < ce; ++c) {
    volatile float fc2 = freq[c] * freq[c], fh2 = f_high * f_high;
    volatile float inv_c = 1.0f / fc2, inv_h = 1.0f / fh2;
    volatile float diff = inv_c - inv_h;
    volatile float k = 4148.808f * q.dm;
    volatile float delay = k * diff;  // seconds
    long d;
    if (fil) {
      d = std::lround(static_cast<double>(delay) / h.tsamp);
    } else {
      volatile float ds = delay / static_cast<float>(h.tsamp);
      d = std::lround(static_cast<float>(ds));
    }
    g.delay[c - cs] = static_cast<int32_t>(d);
    dmax = std::max(dmax, static_cast<int>(d));
    // A negative delay (dm < 0 on a Filterbank, which the reference does not
    // reject) would read before the window's RFI slice, or before the file.
    if (d < 0) throw Error{DD_ERR_INVALID, "dm must be >= 0"};
  }
  const int64_t cap = h.ndata > t0 ? h.ndata - t0 : 0;
  const int64_t t_len = cap > dmax ? std::min(t_len_req, cap - dmax) : 0;
  if (t_len == 0)
    throw Error{DD_ERR_INVALID, fil ? "Time window too short for this DM and band (no valid "
                                      "samples after dedispersion)."
                                    : "Time window too short for this DM and band."};
  g.t_start = t0;
  g.ntimes = t_len;
  g.cs = cs;
  g.nsel = nsel;
  g.rfi_t0 = t0 > dmax ? t0 - dmax : 0;
  g.rfi_len = std::min(t_len + (t0 - g.rfi_t0) + 2 * static_cast<int64_t>(dmax), h.ndata - g.rfi_t0);
  if (fil) {
    g.tend = static_cast<float>(std::fma(static_cast<double>(static_cast<float>(t_len)), h.tsamp,
                                         static_cast<double>(q.tstart)));
  } else {
    g.tend = std::fmaf(static_cast<float>(t_len), static_cast<float>(h.tsamp), q.tstart);
  }
  g.fs = std::min(freq[cs], freq[ce - 1]);
  g.fe = std::max(freq[cs], freq[ce - 1]);
  return g;
}

dd_single_dm_info info_of(const Geometry& g) {
  dd_single_dm_info o{};
  o.t_start = g.t_start;
  o.ntimes = g.ntimes;
  o.chan_start = g.cs;
  o.nchans = g.nsel;
  o.rfi_t0 = g.rfi_t0;
  o.rfi_len = g.rfi_len;
  o.tend = g.tend;
  o.freq_start = g.fs;
  o.freq_end = g.fe;
  return o;
}

// IQRM windows over n samples (src/core/iqrm.cu:348-397) and lags (:188-200).
void iqrm_plan(const dd_iqrm_config& q, double tsamp, uint32_t ns, int64_t csub,
               std::vector<uint32_t>& win, std::vector<int32_t>& lags,
               std::vector<uint32_t>& seg_t0) {
  const double win_sec = std::max(0.0, q.win_sec), hop_sec = std::max(0.0, q.hop_sec);
  const uint32_t W = win_sec > 0.0 ? static_cast<uint32_t>(std::floor(win_sec / tsamp)) : 0u;
  const uint32_t H = hop_sec > 0.0 ? static_cast<uint32_t>(std::floor(hop_sec / tsamp)) : W;
  win.clear();
  if (W == 0 || W >= ns) {
    win = {0u, ns};
  } else {
    uint32_t t0 = 0;
    while (t0 + W <= ns) {
      win.push_back(t0);
      win.push_back(t0 + W);
      t0 += (H ? H : W);
    }
    if (q.include_tail && t0 < ns && ns > t0 + 4) {
      win.push_back(t0);
      win.push_back(ns);
    }
  }
  const float rf = std::max(0.0f, q.radius_frac);
  volatile float rprod = rf * static_cast<float>(csub);
  const int radius = std::max(1, static_cast<int>(std::floor(static_cast<float>(rprod))));
  const double gf = q.geofactor > 1.0 ? q.geofactor : 1.5;
  lags.clear();
  for (int lag = 1; lag <= radius;) {
    if (lag < csub) {
      lags.push_back(+lag);
      lags.push_back(-lag);
    }
    lag = std::max(static_cast<int>(gf * lag), lag + 1);
  }
  std::vector<uint32_t> cuts{0u, ns};
  for (uint32_t v : win) cuts.push_back(std::min(v, ns));
  std::sort(cuts.begin(), cuts.end());
  cuts.erase(std::unique(cuts.begin(), cuts.end()), cuts.end());
  seg_t0.assign(cuts.begin(), cuts.end() - 1);
  if (seg_t0.empty()) seg_t0.push_back(0);
}

}  // namespace
}  // namespace dd

using namespace dd;

extern "C" int dd_single_dm_geometry(const dd_header* header, const dd_single_dm_params* params,
                                     dd_single_dm_info* info) {
  if (!header || !params || !info) { set_error("NULL argument"); return DD_ERR_INVALID; }
  try {
    set_error("");
    *info = info_of(geometry(*header, *params));
    return DD_OK;
  } catch (const Error& e) {
    set_error(e.msg);
    return e.code;
  }
}

extern "C" int dd_single_dm_run(const dd_header* header, const dd_single_dm_params* params,
                                const dd_rfi_config* rfi, const int32_t* bad_channels,
                                int32_t n_bad, const void* input, void* output,
                                void* masked_rows, void* stream) {
  if (!header || !params || !input || !output) { set_error("NULL argument"); return DD_ERR_INVALID; }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::vector<void*> scratch;
  auto salloc = [&](size_t bytes) {
    void* p = nullptr;
    DD_CUDA_TRY(cudaMallocAsync(&p, std::max<size_t>(bytes, 16), st));
    scratch.push_back(p);
    return p;
  };
  int rc = DD_OK;
  try {
    set_error("");
    if (header->nbits != 8 && header->nbits != 16 && header->nbits != 32)
      throw Error{DD_ERR_INVALID, "nbits must be 8, 16 or 32"};
    const Geometry g = geometry(*header, *params);
    const int64_t n = header->nchans;
    const int elem = header->nbits / 8;
    const size_t row = static_cast<size_t>(n) * elem;
    // the extended slice, processed in device scratch
    char* ws = static_cast<char*>(salloc(static_cast<size_t>(g.rfi_len) * row));
    DD_CUDA_TRY(cudaMemcpyAsync(ws, static_cast<const char*>(input) + g.rfi_t0 * row,
                                static_cast<size_t>(g.rfi_len) * row, cudaMemcpyDeviceToDevice, st));
    const dd_rfi_config r = rfi ? *rfi : dd_rfi_config{};
    std::vector<uint32_t> win, seg_t0;
    std::vector<int32_t> lags;
    if (r.use_iqrm) {
      // the reference passes header.tsamp (float) or fil.tsamp (double) as double
      const double tsamp = params->freq_mode == DD_FREQ_FIL
                               ? header->tsamp
                               : static_cast<double>(static_cast<float>(header->tsamp));
      const int64_t csub = g.nsel;
      iqrm_plan(r.iqrm, tsamp, static_cast<uint32_t>(g.rfi_len), csub, win, lags, seg_t0);
      const int nwin = static_cast<int>(win.size() / 2);
      uint32_t* d_win = static_cast<uint32_t*>(salloc(sizeof(uint32_t) * win.size()));
      DD_CUDA_TRY(cudaMemcpyAsync(d_win, win.data(), sizeof(uint32_t) * win.size(),
                                  cudaMemcpyHostToDevice, st));
      uint8_t* d_masks = static_cast<uint8_t*>(salloc(static_cast<size_t>(nwin) * n));
      if (!lags.empty()) {
        int32_t* d_lags = static_cast<int32_t*>(salloc(sizeof(int32_t) * lags.size()));
        DD_CUDA_TRY(cudaMemcpyAsync(d_lags, lags.data(), sizeof(int32_t) * lags.size(),
                                    cudaMemcpyHostToDevice, st));
        auto* d_sums = static_cast<unsigned long long*>(
            salloc(sizeof(unsigned long long) * 2 * csub * nwin));
        void* d_scr = salloc(iqrm_scratch_bytes(nwin, csub, static_cast<int>(lags.size())));
        launch_iqrm_stats(ws, header->nbits, g.rfi_len, n, g.cs, csub, d_win, nwin, d_sums, st);
        launch_iqrm_decide(d_sums, nwin, d_win, n, g.cs, csub, r.iqrm.mode,
                           std::max(0.0f, r.iqrm.nsigma), d_lags, static_cast<int>(lags.size()),
                           8 | 4, d_scr, d_masks, st);
      } else {
        DD_CUDA_TRY(cudaMemsetAsync(d_masks, 0, static_cast<size_t>(nwin) * n, st));
      }
      uint32_t* d_seg = static_cast<uint32_t*>(salloc(sizeof(uint32_t) * seg_t0.size()));
      DD_CUDA_TRY(cudaMemcpyAsync(d_seg, seg_t0.data(), sizeof(uint32_t) * seg_t0.size(),
                                  cudaMemcpyHostToDevice, st));
      uint8_t* d_segmask = static_cast<uint8_t*>(salloc(seg_t0.size() * n));
      launch_segment_masks(d_masks, nwin, d_win, d_seg, static_cast<int>(seg_t0.size()), n,
                           d_segmask, st);
      launch_apply_masks_inplace(ws, header->nbits, g.rfi_len, n, d_segmask, d_seg,
                                 static_cast<int>(seg_t0.size()), st);
    }
    if (r.use_mask && bad_channels && n_bad > 0) {
      std::vector<uint8_t> keep(static_cast<size_t>(n), 1);
      bool any = false;
      for (int32_t i = 0; i < n_bad; ++i)
        if (bad_channels[i] >= 0 && bad_channels[i] < n) { keep[bad_channels[i]] = 0; any = true; }
      if (any) {
        uint8_t* d_keep = static_cast<uint8_t*>(salloc(keep.size()));
        DD_CUDA_TRY(cudaMemcpyAsync(d_keep, keep.data(), keep.size(), cudaMemcpyHostToDevice, st));
        PrepArgs a{};
        a.x = ws;
        a.nbits = header->nbits;
        a.nsamp = g.rfi_len;
        a.nchans = n;
        a.keep = d_keep;
        a.full_out = ws;  // in place: every thread rewrites the element it read
        launch_prep(a, st);
      }
    }
    if (masked_rows)
      DD_CUDA_TRY(cudaMemcpyAsync(masked_rows, ws, static_cast<size_t>(g.rfi_len) * row,
                                  cudaMemcpyDeviceToDevice, st));
    int32_t* d_delay = static_cast<int32_t*>(salloc(sizeof(int32_t) * g.delay.size()));
    DD_CUDA_TRY(cudaMemcpyAsync(d_delay, g.delay.data(), sizeof(int32_t) * g.delay.size(),
                                cudaMemcpyHostToDevice, st));
    const int64_t row0 = g.t_start - g.rfi_t0;
    dim3 grid(static_cast<unsigned>((g.nsel + 255) / 256),
              static_cast<unsigned>(std::min<int64_t>(g.ntimes, 4096)));
    switch (header->nbits) {
      case 8: k_gather_single<uint8_t><<<grid, 256, 0, st>>>(reinterpret_cast<const uint8_t*>(ws), n, row0, g.cs, g.nsel, d_delay, g.ntimes, static_cast<uint8_t*>(output)); break;
      case 16: k_gather_single<uint16_t><<<grid, 256, 0, st>>>(reinterpret_cast<const uint16_t*>(ws), n, row0, g.cs, g.nsel, d_delay, g.ntimes, static_cast<uint16_t*>(output)); break;
      default: k_gather_single<uint32_t><<<grid, 256, 0, st>>>(reinterpret_cast<const uint32_t*>(ws), n, row0, g.cs, g.nsel, d_delay, g.ntimes, static_cast<uint32_t*>(output)); break;
    }
    DD_LAUNCHED();
  } catch (const Error& e) {
    set_error(e.msg);
    rc = e.code;
  }
  for (void* p : scratch) cudaFreeAsync(p, st);
  return rc;
}
