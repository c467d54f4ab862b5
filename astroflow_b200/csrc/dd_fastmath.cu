// Kernels whose results must equal the reference's fast-math device arithmetic.
//
// This translation unit is compiled with the reference's device flags
// (--use_fast_math --ftz=true --prec-div=false --prec-sqrt=false --fmad=true,
// CMakeLists.txt:79-91).  The float expressions below are written with the same
// operand types and order as the reference kernels they replace, so the
// compiler evaluates them with the same approximate reciprocal/division and
// the same multiply-add contractions; nothing here restates those operations.
//
//  * subband delay tables: coarse delays of pre_calculate_dedispersion_kernel
//    (src/core/dedispered.cu:318-335) with the downsample division of
//    divide_delay_inplace_kernel (:379-382) fused, and the residual shifts of
//    compute_residual2_kernel (:385-413);
//  * the zero-DM filter as the reference's call site invokes it
//    (dedispered.cu:1107 -> RfiMarker::zero_dm_filter, src/rfi/rfimarker.cu:130-169);
//  * the per-sample mean of the range zero-DM filter (rfimarker.cu:172-216),
//    whose subtraction the layout kernels apply (DD_ZDM_RANGE_REF).
#include <algorithm>
#include <cstdint>
#include <limits>

#include "dd_internal.h"

namespace dd {
namespace {

__global__ void k_delay1(int32_t* __restrict__ delay1, float dm_low, float dm_high,
                         float dm_step, size_t chan_start, size_t chan_end,
                         const double* __restrict__ freq_table, float ref_freq_value,
                         double tsamp, size_t ndm_nom, int ds) {
  // Same index arithmetic as the reference launch: x = coarse DM, y = channel.
  size_t dmidx = blockDim.x * blockIdx.x + threadIdx.x;
  size_t chan = blockDim.y * blockIdx.y + threadIdx.y + chan_start;
  if (dmidx >= ndm_nom || chan > chan_end) return;
  float dm = dm_low + (blockDim.x * blockIdx.x + threadIdx.x) * dm_step;
  size_t slot = dmidx * (chan_end - chan_start + 1) + chan - chan_start;
  // A coarse DM above dm_high is skipped by the reference kernel, whose
  // zero-initialised managed table then keeps 0 for that row.
  if (dm > dm_high) {
    delay1[slot] = 0;
    return;
  }
  double f = freq_table[chan];
  float ref2 = ref_freq_value * ref_freq_value;
  float f2 = static_cast<float>(f * f);
  float delay = 4148.808f * dm * (1.0f / f2 - 1.0f / ref2);
  int v = static_cast<int>(roundf(delay / tsamp));
  delay1[slot] = v / ds;
}

__global__ void k_residual2(int32_t* __restrict__ residual2, const double* __restrict__ sbfreq,
                            size_t dm_steps, size_t NSB, size_t NDM0, float dm_low,
                            float dm_step, float ref_freq_value, double tsamp,
                            int time_downsample) {
  size_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  size_t total = dm_steps * NSB;
  if (idx >= total) return;
  size_t m = idx / NSB;
  size_t sb = idx % NSB;
  size_t j = m / NDM0;
  float dmj = dm_low + static_cast<float>(j * NDM0) * dm_step;
  float dmm = dm_low + static_cast<float>(m) * dm_step;
  float dmdelta = dmm - dmj;
  double f = sbfreq[sb];
  float ref2 = ref_freq_value * ref_freq_value;
  float f2 = static_cast<float>(f * f);
  float delay = 4148.808f * dmdelta * (1.0f / f2 - 1.0f / ref2);
  float bins_f = delay / static_cast<float>(tsamp * time_downsample);
  int bins = static_cast<int>(floorf(bins_f + 0.5f));
  residual2[idx] = bins;
}

// Per-row mean of the non-zero values: one block of 256 threads per row,
// thread-strided float partial sums reduced by a power-of-two tree.
template <typename T>
__global__ void k_zdm_mean(const T* __restrict__ data, unsigned int num_channels,
                           unsigned int num_samples, float* __restrict__ mean) {
  unsigned int t = blockIdx.x;
  if (t >= num_samples) return;
  float sum = 0.0f;
  unsigned int cnt = 0u;
  for (unsigned int ch = threadIdx.x; ch < num_channels; ch += blockDim.x) {
    T v = data[static_cast<size_t>(t) * num_channels + ch];
    if (v != T(0)) {
      sum += static_cast<float>(v);
      cnt += 1u;
    }
  }
  __shared__ float ssum[256];
  __shared__ unsigned int scnt[256];
  ssum[threadIdx.x] = sum;
  scnt[threadIdx.x] = cnt;
  __syncthreads();
  for (unsigned int s = blockDim.x >> 1; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      ssum[threadIdx.x] += ssum[threadIdx.x + s];
      scnt[threadIdx.x] += scnt[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    unsigned int nz = scnt[0];
    mean[t] = (nz > 0u) ? (ssum[0] / static_cast<float>(nz)) : 0.0f;
  }
}

template <typename T>
__device__ __forceinline__ T zdm_clip_sub(T v, float delta) {
  float r = static_cast<float>(v) - delta;
  if (r < 0.0f) r = 0.0f;
  const float vmax = static_cast<float>(std::numeric_limits<T>::max());
  if (r > vmax) r = vmax;
  return static_cast<T>(r);
}

template <typename T>
__global__ void k_zdm_subtract(T* __restrict__ data, unsigned int num_channels,
                               unsigned int num_samples, const float* __restrict__ mean,
                               float alpha) {
  unsigned int t = blockIdx.x;
  unsigned int ch = blockIdx.y * blockDim.x + threadIdx.x;
  if (t >= num_samples || ch >= num_channels) return;
  size_t idx = static_cast<size_t>(t) * num_channels + ch;
  float delta = alpha * mean[t];
  data[idx] = zdm_clip_sub<T>(data[idx], delta);
}

// Range zero-DM mean (rfimarker.cu:172-216 arithmetic): one block of 256
// threads per sample; thread i sums, in channel order, the float values of the
// non-zero samples of channels cs+i, cs+i+256, ... below ce (samples that the
// IQRM segment mask drops count as zero); the 256 partial sums are combined
// pairwise, i += i+s for s = 128, 64, ..., 1 (the last five steps as warp
// shuffles, which pair the same lanes), and the mean is the float quotient of
// this translation unit's fast-math divide.
template <typename T>
__global__ void __launch_bounds__(256) k_zdm_range_mean(
    const T* __restrict__ x, int64_t nsamp, int64_t nchans, int64_t cs, int64_t ce,
    const uint8_t* __restrict__ segmask, const uint32_t* __restrict__ seg_t0, int nseg,
    float* __restrict__ mean) {
  __shared__ float ssum[256];
  __shared__ unsigned int scnt[256];
  const int tid = threadIdx.x;
  for (int64_t t = blockIdx.x; t < nsamp; t += gridDim.x) {
    const uint8_t* sm = nullptr;
    if (segmask) {
      int lo = 0, hi = nseg - 1;  // last segment whose first sample is <= t
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (static_cast<int64_t>(seg_t0[mid]) <= t) lo = mid; else hi = mid - 1;
      }
      sm = segmask + static_cast<int64_t>(lo) * nchans;
    }
    const T* row = x + t * nchans;
    float sum = 0.0f;
    unsigned int cnt = 0u;
    for (int64_t c = cs + tid; c < ce; c += 256) {
      const T v = (sm && sm[c]) ? T(0) : row[c];
      if (v != T(0)) {
        sum += static_cast<float>(v);
        cnt += 1u;
      }
    }
    ssum[tid] = sum;
    scnt[tid] = cnt;
    __syncthreads();
    for (int s = 128; s >= 32; s >>= 1) {
      if (tid < s) {
        ssum[tid] += ssum[tid + s];
        scnt[tid] += scnt[tid + s];
      }
      __syncthreads();
    }
    if (tid < 32) {
      sum = ssum[tid];
      cnt = scnt[tid];
      for (int s = 16; s > 0; s >>= 1) {
        sum += __shfl_down_sync(0xffffffffu, sum, s);
        cnt += __shfl_down_sync(0xffffffffu, cnt, s);
      }
      if (tid == 0) mean[t] = cnt > 0u ? sum / static_cast<float>(cnt) : 0.0f;
    }
    __syncthreads();
  }
}

template <typename T>
void zero_dm_callsite_t(T* data, size_t chan_start, size_t chan_end, size_t down_ndata,
                        float* mean, cudaStream_t st) {
  // The call zero_dm_filter(d, chan_start, chan_end, down_ndata) binds
  // num_channels = chan_start, num_samples = chan_end, alpha = down_ndata.
  const unsigned int num_channels = static_cast<unsigned int>(chan_start);
  const unsigned int num_samples = static_cast<unsigned int>(chan_end);
  const float alpha = static_cast<float>(down_ndata);
  if (num_channels == 0 || num_samples == 0) return;
  k_zdm_mean<T><<<num_samples, 256, 0, st>>>(data, num_channels, num_samples, mean);
  dim3 grid(num_samples, (num_channels + 255) / 256);
  k_zdm_subtract<T><<<grid, 256, 0, st>>>(data, num_channels, num_samples, mean, alpha);
  DD_COUNT_LAUNCH();
  DD_LAUNCHED();
}

}  // namespace

void launch_subband_tables(const double* d_freq, int64_t cs, int64_t ce, float dm_low,
                           float dm_step, int64_t dm_steps, int sbw, int ndm0, float ref_freq,
                           double tsamp, int ds, int32_t* d_delay1, int32_t* d_res,
                           cudaStream_t st) {
  const size_t dch = static_cast<size_t>(ce - cs + 1);
  const size_t ndm_nom = static_cast<size_t>((dm_steps + ndm0 - 1) / ndm0);
  const size_t nsb = (dch + sbw - 1) / sbw;
  // Nominal DM grid of dedispered.cu:1131-1132.
  float dm_step_coarse = dm_step * static_cast<float>(ndm0);
  float dm_high_coarse = dm_low + (ndm_nom - 1) * dm_step_coarse;
  dim3 bs(64, 16);
  dim3 gs(static_cast<unsigned>((ndm_nom + bs.x - 1) / bs.x),
          static_cast<unsigned>((dch + bs.y - 1) / bs.y));
  k_delay1<<<gs, bs, 0, st>>>(d_delay1, dm_low, dm_high_coarse, dm_step_coarse,
                              static_cast<size_t>(cs), static_cast<size_t>(ce), d_freq, ref_freq,
                              tsamp, ndm_nom, ds);
  DD_LAUNCHED();
  // Subband centre frequencies, dedispered.cu:1151-1157.
  std::vector<double> h_sbfreq(nsb);
  std::vector<double> h_freq(static_cast<size_t>(ce + 1));
  DD_CUDA_TRY(cudaMemcpyAsync(h_freq.data(), d_freq, sizeof(double) * (ce + 1),
                              cudaMemcpyDeviceToHost, st));
  DD_CUDA_TRY(cudaStreamSynchronize(st));
  for (size_t sb = 0; sb < nsb; ++sb) {
    size_t ch0 = cs + sb * sbw;
    size_t ch1 = ch0 + sbw < static_cast<size_t>(ce) + 1 ? ch0 + sbw : static_cast<size_t>(ce) + 1;
    h_sbfreq[sb] = h_freq[(ch0 + ch1 - 1) / 2];
  }
  double* d_sbfreq = nullptr;
  DD_CUDA_TRY(cudaMallocAsync(&d_sbfreq, sizeof(double) * nsb, st));
  DD_CUDA_TRY(cudaMemcpyAsync(d_sbfreq, h_sbfreq.data(), sizeof(double) * nsb,
                              cudaMemcpyHostToDevice, st));
  const size_t total = static_cast<size_t>(dm_steps) * nsb;
  k_residual2<<<static_cast<unsigned>((total + 255) / 256), 256, 0, st>>>(
      d_res, d_sbfreq, static_cast<size_t>(dm_steps), nsb, static_cast<size_t>(ndm0), dm_low,
      dm_step, ref_freq, tsamp, ds);
  DD_LAUNCHED();
  DD_CUDA_TRY(cudaFreeAsync(d_sbfreq, st));
  DD_CUDA_TRY(cudaStreamSynchronize(st));
}

void launch_zdm_range_mean(const void* x, int nbits, int64_t nsamp, int64_t nchans, int64_t cs,
                           int64_t ce, const uint8_t* d_segmask, const uint32_t* d_seg_t0,
                           int nseg, float* d_mean, cudaStream_t st) {
  if (nsamp <= 0) return;
  const unsigned grid = static_cast<unsigned>(std::min<int64_t>(nsamp, 148 * 16));
  switch (nbits) {
    case 8: k_zdm_range_mean<uint8_t><<<grid, 256, 0, st>>>(static_cast<const uint8_t*>(x), nsamp, nchans, cs, ce, d_segmask, d_seg_t0, nseg, d_mean); break;
    case 16: k_zdm_range_mean<uint16_t><<<grid, 256, 0, st>>>(static_cast<const uint16_t*>(x), nsamp, nchans, cs, ce, d_segmask, d_seg_t0, nseg, d_mean); break;
    default: k_zdm_range_mean<uint32_t><<<grid, 256, 0, st>>>(static_cast<const uint32_t*>(x), nsamp, nchans, cs, ce, d_segmask, d_seg_t0, nseg, d_mean); break;
  }
  DD_LAUNCHED();
}

void launch_zero_dm_callsite(void* data, int nbits, size_t chan_start, size_t chan_end,
                             size_t down_ndata, float* mean_ws, cudaStream_t st) {
  switch (nbits) {
    case 8: zero_dm_callsite_t(static_cast<uint8_t*>(data), chan_start, chan_end, down_ndata, mean_ws, st); break;
    case 16: zero_dm_callsite_t(static_cast<uint16_t*>(data), chan_start, chan_end, down_ndata, mean_ws, st); break;
    default: zero_dm_callsite_t(static_cast<uint32_t*>(data), chan_start, chan_end, down_ndata, mean_ws, st); break;
  }
}

}  // namespace dd
