// Checker harness ("tap") around the reference's GPU dedispersion path.
// Test infrastructure only: compiled from the reference's own sources by
// oracle/Makefile into oracle/_ref/libref_gpu_sb<W>.so (one build per
// compile-time subband width AF_SUBBAND_SIZE_CH = W) and run on a GPU as the
// ground truth for
//   * the whole call gpucal::dedisperse_spec<T> (src/core/dedispered.cu:988-1304),
//     whose raw [dm_steps, down_ndata] sums are captured before the image step
//     by the stand-in data.h (oracle/ref_stub/data.h);
//   * the fast-math device delay tables (dedispered.cu:318-335, 379-413),
//     launched with the same arguments the reference's host code passes
//     (dedispered.cu:1124-1182);
//   * the IQRM window masks (src/core/iqrm.cu:400-467) and the RFI-processed
//     input (binning -> IQRM mask -> zero-DM -> mask file, dedispered.cu:1057-1122).
#include "dedispered.cu"

#include <cstdio>
#include <exception>
#include <string>

namespace {

#define TAP_CUDA(call)                                                          \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      std::snprintf(err, errlen, "CUDA %s at line %d", cudaGetErrorString(e_),   \
                    __LINE__);                                                  \
      return 90;                                                                \
    }                                                                           \
  } while (0)

struct TapRfi {
  int use_mask, use_zero_dm, use_iqrm;
  int iq_mode;
  float iq_radius_frac, iq_nsigma;
  double iq_geofactor, iq_win_sec, iq_hop_sec;
  int iq_include_tail;
};

rficonfig make_rfi(const TapRfi* r) {
  iqrmconfig iq(r->iq_mode, r->iq_radius_frac, r->iq_nsigma, r->iq_geofactor, r->iq_win_sec,
                r->iq_hop_sec, r->iq_include_tail != 0);
  return rficonfig(r->use_mask != 0, r->use_zero_dm != 0, r->use_iqrm != 0, iq);
}

template <typename T>
int run_spec(const void* data, const Header& hdr, float dm_low, float dm_high, float freq_start,
             float freq_end, float dm_step, int ds, float t_sample, int device,
             const char* mask_file, const TapRfi* rfi, uint64_t* out, long out_cap, long* rows,
             long* cols, char* err, int errlen) {
  try {
    gpucal::dedisperse_spec<T>(static_cast<T*>(const_cast<void*>(data)), hdr, dm_low, dm_high,
                               freq_start, freq_end, dm_step, REF_FREQ_END, ds, t_sample, device,
                               std::string(mask_file), make_rfi(rfi));
  } catch (const std::exception& e) {
    std::snprintf(err, errlen, "%s", e.what());
    return 2;
  }
  const RefCapture& cap = ref_capture();
  *rows = static_cast<long>(cap.rows);
  *cols = static_cast<long>(cap.cols);
  if (cap.typed.empty()) return 0;  // timing build: dimensions only
  if (static_cast<long>(cap.rows * cap.cols) > out_cap) {
    std::snprintf(err, errlen, "output capacity too small");
    return 3;
  }
  std::memcpy(out, cap.typed.data(), cap.rows * cap.cols * sizeof(uint64_t));
  return 0;
}

// Host side of the table build, stated after dedispered.cu:1003-1031 and
// 1124-1193, launching the reference's own table kernels.
int run_tables(float tsamp, float fch1, float foff, int nchans, long ndata, float dm_low,
               float dm_high, float freq_start, float freq_end, float dm_step, int ds,
               int* delay1, long delay1_cap, int* residual2, long residual2_cap, long* info,
               char* err, int errlen) {
  std::vector<double> h_freq(nchans);
  for (size_t i = 0; i < static_cast<size_t>(nchans); ++i) h_freq[i] = fch1 + i * foff;
  float freq_min = h_freq.front();
  float freq_max = h_freq.back();
  if (freq_start < freq_min || freq_end > freq_max) {
    std::snprintf(err, errlen, "frequency range out of spectrum range");
    return 2;
  }
  size_t chan_start =
      static_cast<size_t>((freq_start - freq_min) / (freq_max - freq_min) * (nchans - 1));
  size_t chan_end =
      static_cast<size_t>((freq_end - freq_min) / (freq_max - freq_min) * (nchans - 1));
  chan_start = std::max<size_t>(0, chan_start);
  chan_end = std::min<size_t>(nchans - 1, chan_end);
  const size_t dm_steps = static_cast<size_t>((dm_high - dm_low) / dm_step) + 1;
  const float ref_freq_value = h_freq[chan_end];
  const size_t down_ndata = (ndata + ds - 1) / ds;
  const size_t Dch = chan_end - chan_start + 1;
  const size_t NSB = (Dch + AF_SUBBAND_SIZE_CH - 1) / AF_SUBBAND_SIZE_CH;
  const size_t NDM0 = AF_SUBBAND_NDM0;
  const size_t NDM_nom = (dm_steps + NDM0 - 1) / NDM0;
  info[0] = (long)chan_start; info[1] = (long)chan_end; info[2] = (long)dm_steps;
  info[3] = (long)down_ndata; info[4] = (long)NSB; info[5] = (long)NDM_nom;
  info[6] = (long)AF_SUBBAND_SIZE_CH; info[7] = (long)NDM0;
  if ((long)(NDM_nom * Dch) > delay1_cap || (long)(dm_steps * NSB) > residual2_cap) {
    std::snprintf(err, errlen, "table capacity too small");
    return 3;
  }
  double* d_freq = nullptr;
  TAP_CUDA(cudaMalloc(&d_freq, nchans * sizeof(double)));
  TAP_CUDA(cudaMemcpy(d_freq, h_freq.data(), nchans * sizeof(double), cudaMemcpyHostToDevice));
  int* d_delay1 = nullptr;
  // Managed memory, as the reference allocates it; entries the kernel skips
  // (its `dm > dm_high` early return) keep the allocation's initial contents.
  TAP_CUDA(cudaMallocManaged(&d_delay1, NDM_nom * Dch * sizeof(int)));
  {
    float dm_step_coarse = dm_step * static_cast<float>(NDM0);
    float dm_high_coarse = dm_low + (NDM_nom - 1) * dm_step_coarse;
    dim3 bs(64, 16);
    dim3 gs((NDM_nom + bs.x - 1) / bs.x, (Dch + bs.y - 1) / bs.y);
    gpucal::pre_calculate_dedispersion_kernel<<<gs, bs>>>(d_delay1, dm_low, dm_high_coarse,
                                                         dm_step_coarse, chan_start, chan_end,
                                                         d_freq, ref_freq_value, static_cast<double>(tsamp));
    TAP_CUDA(cudaGetLastError());
    TAP_CUDA(cudaDeviceSynchronize());
    size_t tot = NDM_nom * Dch;
    gpucal::divide_delay_inplace_kernel<<<(tot + 255) / 256, 256>>>(d_delay1, tot, ds);
    TAP_CUDA(cudaGetLastError());
    TAP_CUDA(cudaDeviceSynchronize());
  }
  std::vector<double> h_sbfreq(NSB, 0.0);
  for (size_t sb = 0; sb < NSB; ++sb) {
    size_t ch0 = chan_start + sb * AF_SUBBAND_SIZE_CH;
    size_t ch1 = std::min(ch0 + AF_SUBBAND_SIZE_CH, chan_end + 1);
    h_sbfreq[sb] = h_freq[(ch0 + ch1 - 1) / 2];
  }
  double* d_sbfreq = nullptr;
  TAP_CUDA(cudaMalloc(&d_sbfreq, NSB * sizeof(double)));
  TAP_CUDA(cudaMemcpy(d_sbfreq, h_sbfreq.data(), NSB * sizeof(double), cudaMemcpyHostToDevice));
  int* d_res = nullptr;
  TAP_CUDA(cudaMalloc(&d_res, dm_steps * NSB * sizeof(int)));
  gpucal::compute_residual2_kernel<<<(dm_steps * NSB + 255) / 256, 256>>>(
      d_res, d_sbfreq, dm_steps, NSB, NDM0, dm_low, dm_step, ref_freq_value,
      static_cast<double>(tsamp), ds);
  TAP_CUDA(cudaGetLastError());
  TAP_CUDA(cudaDeviceSynchronize());
  TAP_CUDA(cudaMemcpy(delay1, d_delay1, NDM_nom * Dch * sizeof(int), cudaMemcpyDefault));
  TAP_CUDA(cudaMemcpy(residual2, d_res, dm_steps * NSB * sizeof(int), cudaMemcpyDeviceToHost));
  cudaFree(d_freq);
  cudaFree(d_delay1);
  cudaFree(d_sbfreq);
  cudaFree(d_res);
  return 0;
}

// Replay of the RFI stages of dedispered.cu:1046-1122 on a device copy of the
// input, using the reference's own kernels and classes; returns the processed
// (binned) input and the IQRM window masks.
template <typename T>
int run_rfi(const void* data, float tsamp, float fch1, float foff, int nchans, long ndata,
            float freq_start, float freq_end, int ds, const char* mask_file, const TapRfi* rfi,
            void* out_data, long out_cap, unsigned* win_t0, unsigned* win_t1, uint8_t* win_mask,
            long win_cap, long* nwin, long* info, char* err, int errlen) {
  std::vector<double> h_freq(nchans);
  for (size_t i = 0; i < static_cast<size_t>(nchans); ++i) h_freq[i] = fch1 + i * foff;
  float freq_min = h_freq.front();
  float freq_max = h_freq.back();
  if (freq_start < freq_min || freq_end > freq_max) {
    std::snprintf(err, errlen, "frequency range out of spectrum range");
    return 2;
  }
  size_t chan_start =
      static_cast<size_t>((freq_start - freq_min) / (freq_max - freq_min) * (nchans - 1));
  size_t chan_end =
      static_cast<size_t>((freq_end - freq_min) / (freq_max - freq_min) * (nchans - 1));
  chan_start = std::max<size_t>(0, chan_start);
  chan_end = std::min<size_t>(nchans - 1, chan_end);
  const size_t down_ndata = (ndata + ds - 1) / ds;
  info[0] = (long)chan_start; info[1] = (long)chan_end; info[2] = (long)down_ndata;
  if ((long)(down_ndata * nchans) > out_cap) {
    std::snprintf(err, errlen, "output capacity too small");
    return 3;
  }
  T* d_input = nullptr;
  TAP_CUDA(cudaMalloc(&d_input, ndata * nchans * sizeof(T)));
  TAP_CUDA(cudaMemcpy(d_input, data, ndata * nchans * sizeof(T), cudaMemcpyHostToDevice));
  T* d_binned = d_input;
  if (ds > 1) {
    TAP_CUDA(cudaMalloc(&d_binned, down_ndata * nchans * sizeof(T)));
    const size_t total = nchans * down_ndata;
    gpucal::time_binning_kernel<T><<<(total + 255) / 256, 256>>>(d_binned, d_input, nchans,
                                                                ndata, ds, down_ndata);
    TAP_CUDA(cudaGetLastError());
    TAP_CUDA(cudaDeviceSynchronize());
    TAP_CUDA(cudaFree(d_input));
  }
  rficonfig rficfg = make_rfi(rfi);
  RfiMarker<T> rfi_marker{std::string(mask_file)};
  *nwin = 0;
  if (rficfg.use_iqrm) {
    auto win_masks = iqrm_cuda::rfi_iqrm_gpu<T>(d_binned, chan_start, chan_end, down_ndata,
                                                nchans, tsamp * ds, rficfg);
    if ((long)win_masks.size() > win_cap) {
      std::snprintf(err, errlen, "window capacity too small");
      return 4;
    }
    for (size_t w = 0; w < win_masks.size(); ++w) {
      win_t0[w] = win_masks[w].t0;
      win_t1[w] = win_masks[w].t1;
      std::memcpy(win_mask + w * nchans, win_masks[w].mask.data(), nchans);
    }
    *nwin = (long)win_masks.size();
    rfi_marker.mask(d_binned, nchans, down_ndata, win_masks);
  }
  if (rficfg.use_zero_dm) rfi_marker.zero_dm_filter(d_binned, chan_start, chan_end, down_ndata);
  if (rficfg.use_mask) rfi_marker.mark_rfi(d_binned, nchans, down_ndata);
  TAP_CUDA(cudaDeviceSynchronize());
  TAP_CUDA(cudaMemcpy(out_data, d_binned, down_ndata * nchans * sizeof(T),
                      cudaMemcpyDeviceToHost));
  TAP_CUDA(cudaFree(d_binned));
  return 0;
}

}  // namespace

extern "C" int ref_gpu_subband_width(void) { return AF_SUBBAND_SIZE_CH; }

// Direct capture of the next calls' raw sums (see RefCapture::sink): rows
// `rows[0..nrows)` (all rows when nrows is 0) into `sink` in the output's own
// element type; NULL sink turns it off.  Returns nothing; ref_capture_elem()
// reports the element size the last captured call wrote.
extern "C" void ref_set_capture_sink(void* sink, const long* rows, long nrows) {
  RefCapture& cap = ref_capture();
  cap.sink = sink;
  cap.sink_rows = rows;
  cap.sink_nrows = nrows;
  cap.sink_elem = 0;
}
extern "C" long ref_capture_elem(void) { return static_cast<long>(ref_capture().sink_elem); }

// The reference's range zero-DM filter, RfiMarker<T>::zero_dm_filter(d, num_channels,
// num_samples, chan_start, chan_end, alpha, clip_to_zero) (src/rfi/rfimarker.cu:257-305),
// which no reference call site reaches, run on a device copy of `data`
// ([nsamp][nchans], host) with the default alpha 1 and clipping; the filtered
// samples are copied back into `out`.
template <typename T>
int run_zdm_range(const void* data, int nchans, long nsamp, int chan_start, int chan_end,
                  void* out, char* err, int errlen) {
  T* d = nullptr;
  const size_t bytes = static_cast<size_t>(nsamp) * nchans * sizeof(T);
  TAP_CUDA(cudaMalloc(&d, bytes));
  TAP_CUDA(cudaMemcpy(d, data, bytes, cudaMemcpyHostToDevice));
  RfiMarker<T> marker{std::string("")};
  marker.zero_dm_filter(d, static_cast<unsigned int>(nchans), static_cast<unsigned int>(nsamp),
                        static_cast<unsigned int>(chan_start), static_cast<unsigned int>(chan_end));
  TAP_CUDA(cudaDeviceSynchronize());
  TAP_CUDA(cudaMemcpy(out, d, bytes, cudaMemcpyDeviceToHost));
  TAP_CUDA(cudaFree(d));
  return 0;
}

extern "C" int ref_gpu_zero_dm_range(int nbits, const void* data, int nchans, long nsamp,
                                     int chan_start, int chan_end, void* out, char* err,
                                     int errlen) {
  switch (nbits) {
    case 8: return run_zdm_range<uint8_t>(data, nchans, nsamp, chan_start, chan_end, out, err, errlen);
    case 16: return run_zdm_range<uint16_t>(data, nchans, nsamp, chan_start, chan_end, out, err, errlen);
    case 32: return run_zdm_range<uint32_t>(data, nchans, nsamp, chan_start, chan_end, out, err, errlen);
  }
  std::snprintf(err, errlen, "unsupported nbits");
  return 5;
}

extern "C" int ref_gpu_dedisperse_spec(int nbits, const void* data, float mjd, float tsamp,
                                       float fch1, float foff, int nchans, long ndata,
                                       float dm_low, float dm_high, float freq_start,
                                       float freq_end, float dm_step, int ds, float t_sample,
                                       int device, const char* mask_file, const void* rfi,
                                       uint64_t* out, long out_cap, long* rows, long* cols,
                                       char* err, int errlen) {
  Header hdr(mjd, tsamp, fch1, foff, nbits, nchans, ndata, "tap");
  const TapRfi* r = static_cast<const TapRfi*>(rfi);
  switch (nbits) {
    case 8:
      return run_spec<uint8_t>(data, hdr, dm_low, dm_high, freq_start, freq_end, dm_step, ds,
                               t_sample, device, mask_file, r, out, out_cap, rows, cols, err,
                               errlen);
    case 16:
      return run_spec<uint16_t>(data, hdr, dm_low, dm_high, freq_start, freq_end, dm_step, ds,
                                t_sample, device, mask_file, r, out, out_cap, rows, cols, err,
                                errlen);
    case 32:
      return run_spec<uint32_t>(data, hdr, dm_low, dm_high, freq_start, freq_end, dm_step, ds,
                                t_sample, device, mask_file, r, out, out_cap, rows, cols, err,
                                errlen);
  }
  std::snprintf(err, errlen, "unsupported nbits");
  return 5;
}

extern "C" int ref_gpu_tables(float tsamp, float fch1, float foff, int nchans, long ndata,
                              float dm_low, float dm_high, float freq_start, float freq_end,
                              float dm_step, int ds, int* delay1, long delay1_cap,
                              int* residual2, long residual2_cap, long* info, char* err,
                              int errlen) {
  return run_tables(tsamp, fch1, foff, nchans, ndata, dm_low, dm_high, freq_start, freq_end,
                    dm_step, ds, delay1, delay1_cap, residual2, residual2_cap, info, err,
                    errlen);
}

extern "C" int ref_gpu_rfi(int nbits, const void* data, float tsamp, float fch1, float foff,
                           int nchans, long ndata, float freq_start, float freq_end, int ds,
                           const char* mask_file, const void* rfi, void* out_data,
                           long out_cap, unsigned* win_t0, unsigned* win_t1,
                           uint8_t* win_mask, long win_cap, long* nwin, long* info, char* err,
                           int errlen) {
  const TapRfi* r = static_cast<const TapRfi*>(rfi);
  switch (nbits) {
    case 8:
      return run_rfi<uint8_t>(data, tsamp, fch1, foff, nchans, ndata, freq_start, freq_end, ds,
                              mask_file, r, out_data, out_cap, win_t0, win_t1, win_mask,
                              win_cap, nwin, info, err, errlen);
    case 16:
      return run_rfi<uint16_t>(data, tsamp, fch1, foff, nchans, ndata, freq_start, freq_end,
                               ds, mask_file, r, out_data, out_cap, win_t0, win_t1, win_mask,
                               win_cap, nwin, info, err, errlen);
  }
  std::snprintf(err, errlen, "unsupported nbits");
  return 5;
}

// The file entry point: Filterbank(filename) (src/data/filterbank.cpp:64-116, header,
// data and channel flip) then gpucal::dedispered_fil_cuda<T>
// (src/core/dedispered.cu:483-986), as _dedispered_fil calls them for target 1
// (src/bindpy/pyapi.cpp:6-51).  Raw sums captured before the image step.
extern "C" int ref_gpu_dedispered_fil(const char* filename, float dm_low, float dm_high,
                                      float freq_start, float freq_end, float dm_step, int ds,
                                      float t_sample, int device, const char* mask_file,
                                      const void* rfi, uint64_t* out, long out_cap, long* rows,
                                      long* cols, char* err, int errlen) {
  const TapRfi* r = static_cast<const TapRfi*>(rfi);
  try {
    Filterbank fil{std::string(filename)};
    switch (fil.nbits) {
      case 8:
        gpucal::dedispered_fil_cuda<uint8_t>(fil, dm_low, dm_high, freq_start, freq_end, dm_step,
                                             REF_FREQ_END, ds, t_sample, device,
                                             std::string(mask_file), make_rfi(r));
        break;
      case 16:
        gpucal::dedispered_fil_cuda<uint16_t>(fil, dm_low, dm_high, freq_start, freq_end,
                                              dm_step, REF_FREQ_END, ds, t_sample, device,
                                              std::string(mask_file), make_rfi(r));
        break;
      case 32:
        gpucal::dedispered_fil_cuda<uint32_t>(fil, dm_low, dm_high, freq_start, freq_end,
                                              dm_step, REF_FREQ_END, ds, t_sample, device,
                                              std::string(mask_file), make_rfi(r));
        break;
      default:
        std::snprintf(err, errlen, "unsupported nbits %d", fil.nbits);
        return 5;
    }
  } catch (const std::exception& e) {
    std::snprintf(err, errlen, "%s", e.what());
    return 2;
  }
  const RefCapture& cap = ref_capture();
  if (static_cast<long>(cap.rows * cap.cols) > out_cap) {
    std::snprintf(err, errlen, "output capacity too small");
    return 3;
  }
  std::memcpy(out, cap.typed.data(), cap.rows * cap.cols * sizeof(uint64_t));
  *rows = static_cast<long>(cap.rows);
  *cols = static_cast<long>(cap.cols);
  return 0;
}

// ---- single-DM spectra: cpucal::dedisperse_spec_with_dm (include/cpucal.hpp:341-483)
// and cpucal::dedispered_fil_with_dm (:203-339).  Both zero the RFI-masked samples of
// their input in place, so `data` (a copy owned by the caller) shows that mutation.
#include "cpucal.hpp"

namespace {
template <typename T>
int copy_spectrum(const Spectrum<T>& s, void* out, long out_cap, long* ntimes, long* nsel,
                  float* meta, char* err, int errlen) {
  if (static_cast<long>(s.ntimes * s.nchans) > out_cap) {
    std::snprintf(err, errlen, "output capacity too small");
    return 3;
  }
  std::memcpy(out, s.data.get(), s.ntimes * s.nchans * sizeof(T));
  *ntimes = static_cast<long>(s.ntimes);
  *nsel = static_cast<long>(s.nchans);
  meta[0] = s.tstart;
  meta[1] = s.tend;
  meta[2] = s.freq_start;
  meta[3] = s.freq_end;
  return 0;
}

template <typename T>
int spec_with_dm(void* data, const Header& hdr, float tstart, float tend, float dm, float fs,
                 float fe, const char* mask_file, const TapRfi* r, void* out, long out_cap,
                 long* ntimes, long* nsel, float* meta, char* err, int errlen) {
  try {
    Spectrum<T> s = cpucal::dedisperse_spec_with_dm<T>(static_cast<T*>(data), hdr, dm, tstart,
                                                       tend, fs, fe, std::string(mask_file),
                                                       make_rfi(r));
    return copy_spectrum(s, out, out_cap, ntimes, nsel, meta, err, errlen);
  } catch (const std::exception& e) {
    std::snprintf(err, errlen, "%s", e.what());
    return 2;
  }
}
}  // namespace

extern "C" int ref_gpu_spec_with_dm(int nbits, void* data, float tsamp, float fch1, float foff,
                                    int nchans, long ndata, float tstart, float tend, float dm,
                                    float fs, float fe, const char* mask_file, const void* rfi,
                                    void* out, long out_cap, long* ntimes, long* nsel,
                                    float* meta, char* err, int errlen) {
  Header hdr(0.0f, tsamp, fch1, foff, nbits, nchans, ndata, "tap");
  const TapRfi* r = static_cast<const TapRfi*>(rfi);
  switch (nbits) {
    case 8: return spec_with_dm<uint8_t>(data, hdr, tstart, tend, dm, fs, fe, mask_file, r, out, out_cap, ntimes, nsel, meta, err, errlen);
    case 16: return spec_with_dm<uint16_t>(data, hdr, tstart, tend, dm, fs, fe, mask_file, r, out, out_cap, ntimes, nsel, meta, err, errlen);
    case 32: return spec_with_dm<uint32_t>(data, hdr, tstart, tend, dm, fs, fe, mask_file, r, out, out_cap, ntimes, nsel, meta, err, errlen);
  }
  std::snprintf(err, errlen, "unsupported nbits");
  return 5;
}

extern "C" int ref_gpu_fil_with_dm(const char* filename, float tstart, float tend, float dm,
                                   float fs, float fe, const char* mask_file, const void* rfi,
                                   void* out, long out_cap, long* ntimes, long* nsel, float* meta,
                                   char* err, int errlen) {
  const TapRfi* r = static_cast<const TapRfi*>(rfi);
  try {
    Filterbank fil{std::string(filename)};
    switch (fil.nbits) {
      case 8: return copy_spectrum(cpucal::dedispered_fil_with_dm<uint8_t>(&fil, tstart, tend, dm, fs, fe, std::string(mask_file), make_rfi(r)), out, out_cap, ntimes, nsel, meta, err, errlen);
      case 16: return copy_spectrum(cpucal::dedispered_fil_with_dm<uint16_t>(&fil, tstart, tend, dm, fs, fe, std::string(mask_file), make_rfi(r)), out, out_cap, ntimes, nsel, meta, err, errlen);
      case 32: return copy_spectrum(cpucal::dedispered_fil_with_dm<uint32_t>(&fil, tstart, tend, dm, fs, fe, std::string(mask_file), make_rfi(r)), out, out_cap, ntimes, nsel, meta, err, errlen);
    }
  } catch (const std::exception& e) {
    std::snprintf(err, errlen, "%s", e.what());
    return 2;
  }
  std::snprintf(err, errlen, "unsupported nbits");
  return 5;
}
