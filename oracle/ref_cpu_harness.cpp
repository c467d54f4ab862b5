// Checker harness: exposes the reference's CPU brute-force dedispersion
// (include/cpucal.hpp:75-201, cpucal::dedispered_fil_omp) through a plain C
// entry point so the tests can compare against it.  Test infrastructure only;
// compiled from the reference's own sources by oracle/Makefile into
// oracle/_ref/libref_cpu.so.  The image post-process is bypassed by the
// stand-in data.h (oracle/ref_stub/data.h), which captures the raw uint64
// DM x time slices.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>

#include "cpucal.hpp"
#include "filterbank.h"

namespace {

template <typename T>
int run_bruteforce(const void* data, long ndata, int nchans, double fch1, double foff,
                   double tsamp, float dm_low, float dm_high, float freq_start,
                   float freq_end, float dm_step, int time_downsample, float t_sample,
                   uint64_t* out, long out_cap, long* nslices, long* slice_cols,
                   long slice_cap, long* ndm, char* err, int errlen) {
  if (nchans <= 0 || nchans > 16320) {
    std::snprintf(err, errlen, "nchans out of range for the reference Filterbank");
    return 1;
  }
  Filterbank fil;  // default constructor owns a 16320-entry frequency table
  fil.nchans = nchans;
  fil.nbits = 8 * static_cast<int>(sizeof(T));
  fil.nifs = 1;
  fil.tsamp = tsamp;
  fil.fch1 = fch1;
  fil.foff = foff;
  fil.ndata = ndata;
  fil.nsamples = ndata;
  fil.data = const_cast<void*>(data);
  // Same table the SIGPROC reader builds (src/data/filterbank.cpp:445-449).
  for (long i = 0; i < nchans; ++i) fil.frequency_table[i] = fch1 + i * foff;
  int rc = 0;
  try {
    cpucal::dedispered_fil_omp<T>(fil, dm_low, dm_high, freq_start, freq_end, dm_step,
                                  REF_FREQ_END, time_downsample, t_sample);
  } catch (const std::exception& e) {
    std::snprintf(err, errlen, "%s", e.what());
    rc = 2;
  }
  fil.data = nullptr;  // borrowed buffer: the Filterbank must not own it
  if (rc) return rc;

  const RefCapture& cap = ref_capture();
  const size_t rows = cap.rows;
  // Slice plan of cpucal.hpp:141-152: slices of round(t_sample/tsamp) input
  // samples, each strided by time_downsample.
  const size_t sps = static_cast<size_t>(std::round(t_sample / tsamp));
  const size_t ns = cap.u64.size();
  if (static_cast<long>(ns) > slice_cap) {
    std::snprintf(err, errlen, "too many slices (%zu)", ns);
    return 3;
  }
  size_t off = 0;
  for (size_t s = 0; s < ns; ++s) {
    const size_t start = s * sps;
    const size_t end = std::min(start + sps, static_cast<size_t>(ndata));
    const size_t cols = (end - start + time_downsample - 1) / time_downsample;
    if (static_cast<long>(off + rows * cols) > out_cap) {
      std::snprintf(err, errlen, "output capacity too small");
      return 4;
    }
    std::memcpy(out + off, cap.u64[s].get(), rows * cols * sizeof(uint64_t));
    off += rows * cols;
    slice_cols[s] = static_cast<long>(cols);
  }
  *nslices = static_cast<long>(ns);
  *ndm = static_cast<long>(rows);
  return 0;
}

}  // namespace

extern "C" int ref_cpu_dedispered_fil_omp(int nbits, const void* data, long ndata,
                                          int nchans, double fch1, double foff,
                                          double tsamp, float dm_low, float dm_high,
                                          float freq_start, float freq_end, float dm_step,
                                          int time_downsample, float t_sample, uint64_t* out,
                                          long out_cap, long* nslices, long* slice_cols,
                                          long slice_cap, long* ndm, char* err, int errlen) {
  switch (nbits) {
    case 8:
      return run_bruteforce<uint8_t>(data, ndata, nchans, fch1, foff, tsamp, dm_low, dm_high,
                                     freq_start, freq_end, dm_step, time_downsample, t_sample,
                                     out, out_cap, nslices, slice_cols, slice_cap, ndm, err,
                                     errlen);
    case 16:
      return run_bruteforce<uint16_t>(data, ndata, nchans, fch1, foff, tsamp, dm_low, dm_high,
                                      freq_start, freq_end, dm_step, time_downsample, t_sample,
                                      out, out_cap, nslices, slice_cols, slice_cap, ndm, err,
                                      errlen);
    case 32:
      return run_bruteforce<uint32_t>(data, ndata, nchans, fch1, foff, tsamp, dm_low, dm_high,
                                      freq_start, freq_end, dm_step, time_downsample, t_sample,
                                      out, out_cap, nslices, slice_cols, slice_cap, ndm, err,
                                      errlen);
    default:
      std::snprintf(err, errlen, "unsupported nbits %d", nbits);
      return 5;
  }
}

extern "C" int ref_cpu_threads(void) { return omp_get_max_threads(); }
