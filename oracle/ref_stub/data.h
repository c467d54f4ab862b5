// Stand-in for the reference's include/data.h, used ONLY when the reference's
// own dedispersion sources are compiled as a parity reference (oracle/_ref).  It is test
// infrastructure, never part of the product.
//
// It declares the same container types as include/data.h:24-163 (Header,
// dedisperseddata[_uint8], Spectrum<T>, DedispersionOutputType,
// DedispersedDataTyped) so that src/core/dedispered.cu and include/cpucal.hpp
// compile unchanged.  The image post-process of include/data.h:299-727
// (OpenCV slice -> resize -> normalize -> viridis) is replaced by a capture of
// the raw integer DM-time arrays, which is what the parity tests compare.
// AF_DEBUG (include/data.h:22) is left undefined, so the reference's debug
// timers and the synchronisations they add are off in the parity build; the
// timing build (oracle/Makefile, libref_gpu_timed_*) defines it to print the
// reference's own per-stage timers, and REF_CAPTURE_DIMS_ONLY to skip the
// host copy of the sums.
#ifndef _DATA_H
#define _DATA_H

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <memory>
#include <omp.h>
#include <stdexcept>
#include <string>
#include <vector>

struct Header {
  float mjd;
  float tsamp;
  float fch1;
  float foff;
  int nbits;
  int nchans;
  long int ndata;
  std::string filename;
  Header() : mjd(0), tsamp(0), fch1(0), foff(0), nbits(0), nchans(0), ndata(0) {}
  Header(float mjd_, float tsamp_, float fch1_, float foff_, int nbits_, int nchans_,
         long int ndata_, std::string filename_)
      : mjd(mjd_), tsamp(tsamp_), fch1(fch1_), foff(foff_), nbits(nbits_),
        nchans(nchans_), ndata(ndata_), filename(filename_) {}
};

struct dedisperseddata_uint8 {
  std::vector<std::shared_ptr<uint8_t[]>> dm_times;
  std::vector<size_t> shape;
  int dm_ndata = 0;
  int downtsample_ndata = 0;
  float dm_low = 0, dm_high = 0, dm_step = 0, tsample = 0;
  std::string filname;
};

struct dedisperseddata {
  std::vector<std::shared_ptr<uint64_t[]>> dm_times;
  std::vector<size_t> shape;
  int dm_ndata = 0;
  int downtsample_ndata = 0;
  float dm_low = 0, dm_high = 0, dm_step = 0, tsample = 0;
  std::string filname;
};

template <typename T> struct Spectrum {
  std::shared_ptr<T[]> data;
  size_t nchans;
  size_t ntimes;
  float tstart;
  float tend;
  float dm;
  int nbits;
  float freq_start;
  float freq_end;
};

template <typename InputType> struct DedispersionOutputType {};
template <> struct DedispersionOutputType<uint8_t> { using type = uint32_t; };
template <> struct DedispersionOutputType<uint16_t> { using type = uint32_t; };
template <> struct DedispersionOutputType<uint32_t> { using type = uint64_t; };
template <typename T>
using dedispersion_output_t = typename DedispersionOutputType<T>::type;

template <typename OutputType> struct DedispersedDataTyped {
  std::vector<std::shared_ptr<OutputType[]>> dm_times;
  std::vector<size_t> shape;
  int dm_ndata = 0;
  int downtsample_ndata = 0;
  float dm_low = 0, dm_high = 0, dm_step = 0, tsample = 0;
  std::string filname;
};

// ---- capture sink (parity builds only) ------------------------------------
// Each raw array handed to the post-process is kept alive here, widened to
// uint64, together with its number of rows and columns.
struct RefCapture {
  std::vector<std::shared_ptr<uint64_t[]>> u64;   // CPU path arrays (per slice)
  std::vector<uint64_t> typed;                    // GPU path array, widened
  size_t rows = 0;
  size_t cols = 0;
  void clear() { u64.clear(); typed.clear(); rows = cols = 0; }
  // Optional direct sink for the GPU path's array, set by the harness before a
  // call and kept across clear(): rows sink_rows[0..sink_nrows) (all rows when
  // sink_nrows is 0) are copied into `sink` as [n][cols] in the array's own
  // element type (sink_elem bytes), and the widened copy is skipped.  Large
  // chunks need this: the widened copy of a full chunk would not fit in host memory.
  void* sink = nullptr;
  const long* sink_rows = nullptr;
  long sink_nrows = 0;
  size_t sink_elem = 0;
};
inline RefCapture& ref_capture() { static RefCapture c; return c; }

// Replaces include/data.h:299-369 (called by cpucal::dedispered_fil_omp).
// The per-slice widths are not stored by the reference (only the first
// slice's width is in `shape`), so the harness derives them from the slice plan.
inline dedisperseddata_uint8 preprocess_dedisperseddata(const dedisperseddata& in,
                                                        int target_size = 512) {
  (void)target_size;
  auto& cap = ref_capture();
  cap.clear();
  cap.u64 = in.dm_times;
  cap.rows = in.shape.size() > 0 ? in.shape[0] : 0;
  cap.cols = in.shape.size() > 1 ? in.shape[1] : 0;
  return dedisperseddata_uint8{};
}

// Replaces include/data.h:620-727 (called by gpucal::dedisperse_spec and
// gpucal::dedispered_fil_cuda): keeps the single [dm_steps, down_ndata] array.
template <typename InputType>
inline dedisperseddata_uint8 preprocess_typed_dedisperseddata_with_slicing(
    const DedispersedDataTyped<dedispersion_output_t<InputType>>& in, Header header,
    int time_downsample, float slice_duration = 0.5, int target_size = 512) {
  (void)header; (void)time_downsample; (void)slice_duration; (void)target_size;
  auto& cap = ref_capture();
  cap.clear();
  cap.rows = in.shape.at(0);
  cap.cols = in.shape.at(1);
  if (cap.sink) {
    using Out = dedispersion_output_t<InputType>;
    const Out* src = in.dm_times.at(0).get();
    cap.sink_elem = sizeof(Out);
    const size_t n = cap.sink_nrows > 0 ? static_cast<size_t>(cap.sink_nrows) : cap.rows;
    for (size_t i = 0; i < n; ++i) {
      const size_t r = cap.sink_nrows > 0 ? static_cast<size_t>(cap.sink_rows[i]) : i;
      if (r >= cap.rows) continue;
      std::memcpy(static_cast<char*>(cap.sink) + i * cap.cols * sizeof(Out), src + r * cap.cols,
                  cap.cols * sizeof(Out));
    }
    return dedisperseddata_uint8{};
  }
#ifdef REF_CAPTURE_DIMS_ONLY
  // timing build: keep the dimensions only (no host copy of the sums)
  return dedisperseddata_uint8{};
#endif
  cap.typed.resize(cap.rows * cap.cols);
  const auto* p = in.dm_times.at(0).get();
  for (size_t i = 0; i < cap.rows * cap.cols; ++i) cap.typed[i] = static_cast<uint64_t>(p[i]);
  return dedisperseddata_uint8{};
}
#endif
