// RFI stages and input layout for the B200 dedispersion path.
//
//  * time binning with sqrt compression (src/core/dedispered.cu:337-376);
//  * IQRM channel masks (src/core/iqrm.cu:21-185, 203-345), computed entirely on
//    the device: per-channel sums are exact 64-bit integers (the reference's
//    double sums of integer samples are exact, so the statistics agree), and
//    the per-lag sort, percentiles, threshold and votes run in one block per
//    window instead of the reference's two host round trips per lag;
//  * window-mask application (src/rfi/rfimarker.cu:309-390), zero-DM over a
//    channel range with an exact integer mean, and the static channel mask
//    (rfimarker.cu:469-488), fused into the pass that writes the channel-major
//    layout the dedispersion kernels read.
// Host-side arithmetic of the reference (its percentile and threshold code runs
// on the CPU) is reproduced with explicitly rounded intrinsics so that no
// multiply-add contraction changes it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>

#include "dd_internal.h"

namespace dd {
namespace {

template <typename T> struct Lim;
template <> struct Lim<uint8_t> { static constexpr uint64_t vmax = 255u; };
template <> struct Lim<uint16_t> { static constexpr uint64_t vmax = 65535u; };
template <> struct Lim<uint32_t> { static constexpr uint64_t vmax = 4294967295u; };

// ---------------------------------------------------------------- binning
// One thread per channel and output sample (grid: channel blocks x output rows,
// rows strided by gridDim.y); smax_full = sqrt(vmax * ds) of the full bins,
// evaluated on the host with the same IEEE square root.
template <typename T>
__global__ void k_time_binning(const T* __restrict__ in, T* __restrict__ out, int64_t nchans,
                               int64_t ndata, int ds, int64_t nout, double smax_full) {
  const int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= nchans) return;
  const uint64_t vmax = Lim<T>::vmax;
  for (int64_t k = blockIdx.y; k < nout; k += gridDim.y) {
    const int64_t t0 = k * ds;
    const int64_t t1 = t0 + ds < ndata ? t0 + ds : ndata;
    uint64_t sum = 0;
    for (int64_t t = t0; t < t1; ++t) sum += static_cast<uint64_t>(in[c + t * nchans]);
    const uint64_t cnt = static_cast<uint64_t>(t1 - t0);
    const double s = sqrt(static_cast<double>(sum));
    const double smax = cnt == static_cast<uint64_t>(ds)
                            ? smax_full
                            : sqrt(static_cast<double>(vmax * (cnt ? cnt : 1)));
    const double v = __dmul_rn(__ddiv_rn(s, smax > 0.0 ? smax : 1.0), static_cast<double>(vmax));
    out[c + k * nchans] = static_cast<T>(v < static_cast<double>(vmax) ? v : static_cast<double>(vmax));
  }
}

// The value of a full bin depends only on the integer sum of its ds samples, so
// for 8- and 16-bit samples every value is tabulated once per plan (lut[sum],
// sum in [0, ds * vmax]) by the same expression as k_time_binning, and the
// binning becomes a gather: V channels per thread (V * sizeof(T) = 4 bytes, one
// word per load and store).  A last, partial bin uses the expression directly.
template <typename T>
__global__ void k_binning_lut(T* __restrict__ lut, int64_t n, double smax_full) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t vmax = Lim<T>::vmax;
  const double s = sqrt(static_cast<double>(i));
  const double v = __dmul_rn(__ddiv_rn(s, smax_full > 0.0 ? smax_full : 1.0), static_cast<double>(vmax));
  lut[i] = static_cast<T>(v < static_cast<double>(vmax) ? v : static_cast<double>(vmax));
}

template <typename T>
__device__ __forceinline__ T binned_value(uint64_t sum, uint64_t cnt) {
  const uint64_t vmax = Lim<T>::vmax;
  const double s = sqrt(static_cast<double>(sum));
  const double smax = sqrt(static_cast<double>(vmax * (cnt ? cnt : 1)));
  const double v = __dmul_rn(__ddiv_rn(s, smax > 0.0 ? smax : 1.0), static_cast<double>(vmax));
  return static_cast<T>(v < static_cast<double>(vmax) ? v : static_cast<double>(vmax));
}

template <typename T>
__global__ void k_time_binning_lut(const T* __restrict__ in, T* __restrict__ out, int64_t nchans,
                                   int64_t ndata, int ds, int64_t nout, const T* __restrict__ lut) {
  constexpr int V = 4 / sizeof(T);
  const int64_t c = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) * V;
  if (c >= nchans) return;
  for (int64_t k = blockIdx.y; k < nout; k += gridDim.y) {
    const int64_t t0 = k * ds;
    const int64_t t1 = t0 + ds < ndata ? t0 + ds : ndata;
    uint32_t sum[V];
#pragma unroll
    for (int v = 0; v < V; ++v) sum[v] = 0;
    for (int64_t t = t0; t < t1; ++t) {
      const uint32_t w = __ldg(reinterpret_cast<const uint32_t*>(in + t * nchans + c));
#pragma unroll
      for (int v = 0; v < V; ++v) sum[v] += (w >> (8 * sizeof(T) * v)) & static_cast<uint32_t>(Lim<T>::vmax);
    }
    const bool full = t1 - t0 == ds;
    uint32_t o = 0;
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const T b = full ? __ldg(lut + sum[v]) : binned_value<T>(sum[v], static_cast<uint64_t>(t1 - t0));
      o |= static_cast<uint32_t>(b) << (8 * sizeof(T) * v);
    }
    *reinterpret_cast<uint32_t*>(out + k * nchans + c) = o;
  }
}

// ---------------------------------------------------------------- IQRM sums
// Block: 256 consecutive channels of [cs, cs+csub); grid.y: time chunks.
template <typename T>
__global__ void k_iqrm_stats(const T* __restrict__ x, int64_t nsamp, int64_t nchans, int64_t cs,
                             int64_t csub, const uint32_t* __restrict__ win, int nwin,
                             int64_t chunk, unsigned long long* __restrict__ sums) {
  int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= csub) return;
  const int64_t c = cs + i;
  const int64_t lo = static_cast<int64_t>(blockIdx.y) * chunk;
  const int64_t hi = lo + chunk < nsamp ? lo + chunk : nsamp;
  for (int w = 0; w < nwin; ++w) {
    int64_t a = win[2 * w] > lo ? win[2 * w] : lo;
    int64_t b = win[2 * w + 1] < hi ? win[2 * w + 1] : hi;
    if (a >= b) continue;
    unsigned long long s = 0, s2 = 0;
    for (int64_t t = a; t < b; ++t) {
      unsigned long long v = x[t * nchans + c];
      s += v;
      s2 += v * v;
    }
    atomicAdd(&sums[(static_cast<int64_t>(w) * 2) * csub + i], s);
    atomicAdd(&sums[(static_cast<int64_t>(w) * 2 + 1) * csub + i], s2);
  }
}

// 8-bit samples, four channels per thread (one aligned 32-bit load per row, a
// warp reading 128 contiguous bytes): thread k covers channels (cs & ~3) + 4k ..
// + 3; per window and time chunk it keeps 32-bit partial sums (a chunk of at
// most 1024 rows: 1024 x 255^2 < 2^32) and adds them to the 64-bit sums of the
// channels inside [cs, cs+csub).  Needs nchans % 4 == 0 and an aligned input.
__global__ void k_iqrm_stats_u8w(const uint8_t* __restrict__ x, int64_t nsamp, int64_t nchans,
                                 int64_t cs, int64_t csub, const uint32_t* __restrict__ win,
                                 int nwin, int64_t chunk, unsigned long long* __restrict__ sums) {
  const int64_t c4 = (cs & ~int64_t(3)) + 4 * (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x);
  if (c4 >= cs + csub) return;
  const int64_t lo = static_cast<int64_t>(blockIdx.y) * chunk;
  const int64_t hi = lo + chunk < nsamp ? lo + chunk : nsamp;
  for (int w = 0; w < nwin; ++w) {
    const int64_t a = win[2 * w] > lo ? win[2 * w] : lo;
    const int64_t b = win[2 * w + 1] < hi ? win[2 * w + 1] : hi;
    if (a >= b) continue;
    uint32_t s[4] = {0u, 0u, 0u, 0u}, q[4] = {0u, 0u, 0u, 0u};
#pragma unroll 8
    for (int64_t t = a; t < b; ++t) {  // unrolled: eight rows' loads in flight
      const uint32_t v = __ldg(reinterpret_cast<const uint32_t*>(x + t * nchans + c4));
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const uint32_t e = (v >> (8 * k)) & 0xffu;
        s[k] += e;
        q[k] += e * e;
      }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int64_t ch = c4 + k;
      if (ch < cs || ch >= cs + csub) continue;
      const int64_t i = ch - cs;
      atomicAdd(&sums[(static_cast<int64_t>(w) * 2) * csub + i], static_cast<unsigned long long>(s[k]));
      atomicAdd(&sums[(static_cast<int64_t>(w) * 2 + 1) * csub + i], static_cast<unsigned long long>(q[k]));
    }
  }
}

__device__ __forceinline__ int iqrm_target(int lag, int i, int csub) {
  if (lag < 0) return i < csub + lag ? i - lag : csub - 1;
  return i < lag ? 0 : i - lag;
}

// Percentile of iqrm.cu:299-306 (host code there): pos = q*(n-1) in double,
// linear interpolation with the float difference promoted to double.
__device__ __forceinline__ float pct_sorted(const float* v, int n, float q) {
  if (n == 1) return v[0];
  double pos = __dmul_rn(static_cast<double>(q), static_cast<double>(n - 1));
  int lo = static_cast<int>(floor(pos));
  int hi = static_cast<int>(ceil(pos));
  double w = __dsub_rn(pos, static_cast<double>(lo));
  float dlt = __fsub_rn(v[hi], v[lo]);
  return static_cast<float>(__dadd_rn(static_cast<double>(v[lo]), __dmul_rn(static_cast<double>(dlt), w)));
}

// One block per window.  Scratch per window: x, d (float), recv, cast (int),
// flags (nlags x csub bytes).  Dynamic shared memory: the sort buffer.
__global__ void k_iqrm_decide(const unsigned long long* __restrict__ sums,
                              const uint32_t* __restrict__ win, int64_t nchans, int64_t cs,
                              int csub, int mode, float nsigma, const int32_t* __restrict__ lags,
                              int nlags, int variant, float* __restrict__ xs,
                              float* __restrict__ ds_, int* __restrict__ recv,
                              int* __restrict__ cast_, uint8_t* __restrict__ flags,
                              int sort_n, uint8_t* __restrict__ masks) {
  extern __shared__ float srt[];
  __shared__ float s_med, s_thr;
  __shared__ int s_skip;
  const int w = blockIdx.x;
  const unsigned W = win[2 * w + 1] - win[2 * w];
  float* x = xs + static_cast<int64_t>(w) * csub;
  float* d = ds_ + static_cast<int64_t>(w) * csub;
  int* rc = recv + static_cast<int64_t>(w) * csub;
  int* cc = cast_ + static_cast<int64_t>(w) * csub;
  uint8_t* fl = flags + static_cast<int64_t>(w) * nlags * csub;
  uint8_t* mask = masks + static_cast<int64_t>(w) * nchans;
  const unsigned long long* s1 = sums + (static_cast<int64_t>(w) * 2) * csub;
  const unsigned long long* s2 = s1 + csub;
  for (int c = threadIdx.x; c < nchans; c += blockDim.x) mask[c] = 0;
  if (W == 0 || csub == 0) return;
  // Statistic per channel, make_stat_from_sums (iqrm.cu:72-91).
  for (int i = threadIdx.x; i < csub; i += blockDim.x) {
    double mean = __ddiv_rn(static_cast<double>(s1[i]), static_cast<double>(W));
    if (mode == 0) {
      x[i] = static_cast<float>(mean);
    } else {
      double e2 = __ddiv_rn(static_cast<double>(s2[i]), static_cast<double>(W));
      double var = (variant & 8) ? __fma_rn(-mean, mean, e2) : __dsub_rn(e2, __dmul_rn(mean, mean));
      if (var < 0.0) var = 0.0;
      x[i] = static_cast<float>(sqrt(var));
    }
    rc[i] = 0;
    cc[i] = 0;
  }
  __syncthreads();
  for (int l = 0; l < nlags; ++l) {
    const int lag = lags[l];
    // Lagged difference with edge clipping, make_diff_with_clipping (iqrm.cu:94-117).
    for (int k = threadIdx.x; k < sort_n; k += blockDim.x) {
      float v = FLT_MAX;
      if (k < csub) {
        if (lag < 0) {
          int cut = csub + lag;
          v = k < cut ? __fsub_rn(x[k], x[k - lag]) : __fsub_rn(x[cut], x[csub - 1]);
        } else {
          v = k < lag ? __fsub_rn(x[lag], x[0]) : __fsub_rn(x[k], x[k - lag]);
        }
        d[k] = v;
        fl[static_cast<int64_t>(l) * csub + k] = 0;
      }
      srt[k] = k < csub ? v : __int_as_float(0x7f800000);  // +inf pads past the end
    }
    __syncthreads();
    // Bitonic sort of sort_n (power of two) floats, ascending.
    for (int size = 2; size <= sort_n; size <<= 1) {
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        for (int k = threadIdx.x; k < sort_n; k += blockDim.x) {
          int p = k ^ stride;
          if (p > k) {
            float a = srt[k], b = srt[p];
            bool up = (k & size) == 0;
            if ((a > b) == up) { srt[k] = b; srt[p] = a; }
          }
        }
        __syncthreads();
      }
    }
    if (threadIdx.x == 0) {
      float q1 = pct_sorted(srt, csub, 0.25f);
      float med = pct_sorted(srt, csub, 0.50f);
      float q3 = pct_sorted(srt, csub, 0.75f);
      float s;
      if (variant & 4) s = fabsf(__fmul_rn(__fsub_rn(q3, q1), __frcp_rn(1.349f)));
      else s = fabsf(__fdiv_rn(__fsub_rn(q3, q1), 1.349f));
      bool skip = !(s > 0.f) || !isfinite(s);
      s_skip = skip;
      s_med = med;
      s_thr = __fmul_rn(nsigma, s);
    }
    __syncthreads();
    if (!s_skip) {
      // flag_and_count_kernel (iqrm.cu:120-151).
      const float med = s_med, thr = s_thr;
      for (int i = threadIdx.x; i < csub; i += blockDim.x) {
        float val = __fsub_rn(d[i], med);
        if (val > thr) {
          fl[static_cast<int64_t>(l) * csub + i] = 1;
          atomicAdd(&rc[i], 1);
          atomicAdd(&cc[iqrm_target(lag, i, csub)], 1);
        }
      }
    }
    __syncthreads();
  }
  // merge_lags_to_mask_kernel (iqrm.cu:154-185).
  for (int i = threadIdx.x; i < csub; i += blockDim.x) {
    int ri = rc[i];
    uint8_t m = 0;
    if (ri > 0) {
      for (int l = 0; l < nlags; ++l) {
        if (!fl[static_cast<int64_t>(l) * csub + i]) continue;
        if (cc[iqrm_target(lags[l], i, csub)] < ri) { m = 1; break; }
      }
    }
    mask[cs + i] = m;
  }
}

// OR of the masks of all windows covering each segment of samples.
__global__ void k_segment_masks(const uint8_t* __restrict__ masks, int nwin,
                                const uint32_t* __restrict__ win, const uint32_t* __restrict__ seg_t0,
                                int nseg, int64_t nchans, uint8_t* __restrict__ segmask) {
  const int s = blockIdx.y;
  const int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= nchans || s >= nseg) return;
  const uint32_t a = seg_t0[s];
  uint8_t m = 0;
  for (int w = 0; w < nwin; ++w)
    if (win[2 * w] <= a && a < win[2 * w + 1]) m |= masks[static_cast<int64_t>(w) * nchans + c];
  segmask[static_cast<int64_t>(s) * nchans + c] = m;
}

__device__ __forceinline__ int find_seg(const uint32_t* seg_t0, int nseg, int64_t t) {
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (static_cast<int64_t>(seg_t0[mid]) <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

template <typename T>
__global__ void k_apply_masks(T* __restrict__ x, int64_t nsamp, int64_t nchans,
                              const uint8_t* __restrict__ segmask, const uint32_t* __restrict__ seg_t0,
                              int nseg) {
  const int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= nchans) return;
  for (int64_t t = blockIdx.y; t < nsamp; t += gridDim.y) {
    const int s = find_seg(seg_t0, nseg, t);
    if (segmask[static_cast<int64_t>(s) * nchans + c]) x[t * nchans + c] = 0;
  }
}

// Zero-DM offset per sample: one warp per sample row, warp-shuffle reduction of
// the sum and count of the non-zero (post-IQRM) values of [cs, ce).
template <typename T>
__global__ void k_zdm_offsets(const T* __restrict__ x, int64_t nsamp, int64_t nchans, int64_t cs,
                              int64_t ce, const uint8_t* __restrict__ segmask,
                              const uint32_t* __restrict__ seg_t0, int nseg,
                              uint32_t* __restrict__ off) {
  const int lane = threadIdx.x & 31;
  const int64_t t = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (t >= nsamp) return;
  const uint8_t* sm = nullptr;
  if (segmask) sm = segmask + static_cast<int64_t>(find_seg(seg_t0, nseg, t)) * nchans;
  unsigned long long s = 0;
  unsigned int n = 0;
  const T* row = x + t * nchans;
  for (int64_t c = cs + lane; c < ce; c += 32) {
    uint64_t v = row[c];
    if (sm && sm[c]) v = 0;
    if (v) { s += v; n += 1; }
  }
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_xor_sync(0xffffffffu, s, o);
    n += __shfl_xor_sync(0xffffffffu, n, o);
  }
  if (lane == 0) off[t] = n ? static_cast<uint32_t>((s + n - 1) / n) : 0u;
}

// Range zero-DM subtraction with a float mean (zdm_sat_sub of
// rfimarker.cu:218-225 with alpha 1 and clipping): float(v) - mean, clipped to
// [0, max of T], truncated.
template <typename T>
__device__ __forceinline__ T zdm_float_sub(T v, float mean) {
  float r = __fsub_rn(static_cast<float>(v), mean);
  if (r < 0.0f) r = 0.0f;
  const float vmax = static_cast<float>(Lim<T>::vmax);
  if (r > vmax) r = vmax;
  return static_cast<T>(r);
}

// Fused RFI application and transpose to the channel-major layout.
// Tile: 64 samples x 64 channels, 256 threads.
template <typename T>
__global__ void k_prep(PrepArgs a) {
  __shared__ T tile[64][65];
  const T* x = static_cast<const T*>(a.x);
  const int64_t tb = static_cast<int64_t>(blockIdx.x) * 64;
  const int64_t cb = a.c0 + static_cast<int64_t>(blockIdx.y) * 64;
  const int tx = threadIdx.x & 63;   // channel within tile (read phase)
  const int ty = threadIdx.x >> 6;   // 0..3
  const int64_t c = cb + tx;
  for (int r = ty; r < 64; r += 4) {
    const int64_t t = tb + r;
    T v = 0;
    if (t < a.nsamp && c < a.c1) {
      v = x[t * a.nchans + c];
      if (a.segmask) {
        const int s = find_seg(a.seg_t0, a.nseg, t);
        if (a.segmask[static_cast<int64_t>(s) * a.nchans + c]) v = 0;
      }
      if (a.zdm_off && c >= a.zdm_cs && c < a.zdm_ce) {
        const uint32_t m = a.zdm_off[t];
        v = static_cast<T>(static_cast<uint32_t>(v) > m ? static_cast<uint32_t>(v) - m : 0u);
      }
      if (a.zdm_mean && c >= a.zdm_cs && c < a.zdm_ce) v = zdm_float_sub<T>(v, a.zdm_mean[t]);
      if (a.keep && !a.keep[c]) v = 0;
    }
    tile[r][tx] = v;
  }
  __syncthreads();
  if (a.out) {
    T* out = static_cast<T*>(a.out);
    // write phase: thread -> (channel row, sample)
    for (int r = ty; r < 64; r += 4) {
      const int64_t cc = cb + r;
      const int64_t t = tb + tx;
      if (cc < a.c1 && t < a.nsamp) {
        const int64_t row = (cc - a.c0) * a.ds + (t % a.ds);
        out[row * a.pitch + t / a.ds] = tile[tx][r];
      }
    }
  }
}

// 8-bit samples without downsampling (the subband layout), as k_prep but four
// channels per load and four samples per store: a block takes kPrepU8Subtiles
// consecutive tiles of 64 samples x 64 channels, one after another; for each it
// applies the masks and the zero-DM offset to whole words with byte-wise SIMD
// operations and transposes 4x4 byte blocks in registers.  Needs
// nchans % 4 == 0 (aligned word loads); channel words are read from c0 & ~3 and
// channels outside [c0, c1) are not stored.
constexpr int kPrepU8Subtiles = 4;
__global__ void __launch_bounds__(256) k_prep_u8(PrepArgs a) {
  __shared__ uint32_t tile[64][17];  // [sample][channel word], padded
  const uint8_t* x = static_cast<const uint8_t*>(a.x);
  const int64_t cb = (a.c0 & ~int64_t(3)) + static_cast<int64_t>(blockIdx.y) * 64;
  const int w = threadIdx.x & 15;  // channel word of the tile (load phase)
  const int64_t c = cb + 4 * w;
  const bool cvalid = c < a.nchans;
  uint32_t drop = 0, inrange = 0;  // per byte: bad channel / zero-DM applies
  if (cvalid) {
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int64_t ch = c + b;
      if (a.keep && !a.keep[ch]) drop |= 0xffu << (8 * b);
      if (a.zdm_off && ch >= a.zdm_cs && ch < a.zdm_ce) inrange |= 0xffu << (8 * b);
    }
  }
  const int i = threadIdx.x & 15;  // store phase: samples 4i .. 4i+3
  const int j = threadIdx.x >> 4;  // channel word j: channels 4j .. 4j+3
  const int r0 = threadIdx.x >> 4;  // load phase: rows r0, r0 + 16, r0 + 32, r0 + 48
  uint8_t* out = static_cast<uint8_t*>(a.out);
  const int64_t tile0 = static_cast<int64_t>(blockIdx.x) * kPrepU8Subtiles * 64;
  // this thread's source word in row tile0 + r0, and the stride of 16 rows
  const uint8_t* src = x + (tile0 + r0) * a.nchans + c;
  const int64_t step16 = 16 * a.nchans;
  // this thread's four output rows (channels 4j .. 4j+3) at sample tile0 + 4i
  uint8_t* dst[4];
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int64_t cc = cb + 4 * j + b;
    dst[b] = (out && cc >= a.c0 && cc < a.c1) ? out + (cc - a.c0) * a.pitch + tile0 + 4 * i : nullptr;
  }
  // the raw words of sub-tile `sub` (loads only; masks applied when staged)
  auto fetch = [&](int sub, uint32_t (&v)[4]) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int64_t t = tile0 + sub * 64 + r0 + 16 * k;
      v[k] = (cvalid && t < a.nsamp)
                 ? __ldg(reinterpret_cast<const uint32_t*>(src + (4 * sub + k) * step16))
                 : 0u;
    }
  };
  uint32_t cur[4], nxt[4];
  fetch(0, cur);
  int seg = -1;          // IQRM segment whose mask word is cached in seg_keep
  uint32_t seg_keep = ~0u;
  for (int sub = 0; sub < kPrepU8Subtiles; ++sub) {
    const int64_t tb = tile0 + sub * 64;
    if (tb >= a.nsamp) break;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int r = r0 + 16 * k;
      const int64_t t = tb + r;
      uint32_t v = cur[k];
      if (cvalid && t < a.nsamp) {
        if (a.segmask) {
          const int sg = find_seg(a.seg_t0, a.nseg, t);
          if (sg != seg) {  // segments span many rows: the mask word changes rarely
            seg = sg;
            seg_keep = ~__vcmpne4(*reinterpret_cast<const uint32_t*>(
                                      a.segmask + static_cast<int64_t>(sg) * a.nchans + c),
                                  0u);
          }
          v &= seg_keep;
        }
        if (a.zdm_off) {
          const uint32_t m = min(a.zdm_off[t], 255u) * 0x01010101u;
          v = (__vsubus4(v, m) & inrange) | (v & ~inrange);
        }
        v &= ~drop;
      }
      tile[r][w] = v;
    }
    __syncthreads();
    if (sub + 1 < kPrepU8Subtiles) fetch(sub + 1, nxt);  // in flight during the stores
    if (out) {
      const uint32_t q0 = tile[4 * i][j], q1 = tile[4 * i + 1][j];
      const uint32_t q2 = tile[4 * i + 2][j], q3 = tile[4 * i + 3][j];
      const uint32_t lo01 = __byte_perm(q0, q1, 0x5140), hi01 = __byte_perm(q0, q1, 0x7362);
      const uint32_t lo23 = __byte_perm(q2, q3, 0x5140), hi23 = __byte_perm(q2, q3, 0x7362);
      const uint32_t o[4] = {__byte_perm(lo01, lo23, 0x5410), __byte_perm(lo01, lo23, 0x7632),
                             __byte_perm(hi01, hi23, 0x5410), __byte_perm(hi01, hi23, 0x7632)};
#pragma unroll
      for (int b = 0; b < 4; ++b)
        if (dst[b]) *reinterpret_cast<uint32_t*>(dst[b] + sub * 64) = o[b];
    }
    __syncthreads();  // the tile is refilled by the next sub-tile
#pragma unroll
    for (int k = 0; k < 4; ++k) cur[k] = nxt[k];
  }
}

// 16-bit samples without downsampling, as k_prep_u8 with 16-bit lanes: a block
// takes 64 samples x 64 channels, loads four channels per 8-byte word pair,
// applies the masks and the zero-DM offset lane-wise, and transposes 4x4 blocks
// of 16-bit samples in registers into 8-byte stores of four samples per
// channel.  Needs nchans % 4 == 0; channel words are read from c0 & ~3 and
// channels outside [c0, c1) are not stored.
__global__ void __launch_bounds__(256) k_prep_u16(PrepArgs a) {
  __shared__ uint2 tile[64][17];  // [sample][four-channel group], padded
  const uint16_t* x = static_cast<const uint16_t*>(a.x);
  const int64_t tb = static_cast<int64_t>(blockIdx.x) * 64;
  const int64_t cb = (a.c0 & ~int64_t(3)) + static_cast<int64_t>(blockIdx.y) * 64;
  {
    const int w = threadIdx.x & 15;  // four-channel group of the tile
    const int64_t c = cb + 4 * w;
    const bool cvalid = c < a.nchans;
    uint2 drop = make_uint2(0, 0), inrange = make_uint2(0, 0);  // per 16-bit lane
    if (cvalid) {
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int64_t ch = c + b;
        const uint32_t lane = 0xffffu << (16 * (b & 1));
        if (a.keep && !a.keep[ch]) (b < 2 ? drop.x : drop.y) |= lane;
        if (a.zdm_off && ch >= a.zdm_cs && ch < a.zdm_ce) (b < 2 ? inrange.x : inrange.y) |= lane;
      }
    }
    for (int r = threadIdx.x >> 4; r < 64; r += 16) {
      const int64_t t = tb + r;
      uint2 v = make_uint2(0, 0);
      if (cvalid && t < a.nsamp) {
        v = *reinterpret_cast<const uint2*>(x + t * a.nchans + c);
        if (a.segmask) {
          const int sg = find_seg(a.seg_t0, a.nseg, t);
          const uint32_t k = __vcmpne4(*reinterpret_cast<const uint32_t*>(
                                           a.segmask + static_cast<int64_t>(sg) * a.nchans + c),
                                       0u);
          v.x &= ~__byte_perm(k, 0u, 0x1100);
          v.y &= ~__byte_perm(k, 0u, 0x3322);
        }
        if (a.zdm_off) {
          const uint32_t m = min(a.zdm_off[t], 65535u) * 0x00010001u;
          v.x = (__vsubus2(v.x, m) & inrange.x) | (v.x & ~inrange.x);
          v.y = (__vsubus2(v.y, m) & inrange.y) | (v.y & ~inrange.y);
        }
        v.x &= ~drop.x;
        v.y &= ~drop.y;
      }
      tile[r][w] = v;
    }
  }
  __syncthreads();
  if (!a.out) return;
  const int i = threadIdx.x & 15;  // samples 4i .. 4i+3
  const int j = threadIdx.x >> 4;  // channels 4j .. 4j+3
  const uint2 q0 = tile[4 * i][j], q1 = tile[4 * i + 1][j];
  const uint2 q2 = tile[4 * i + 2][j], q3 = tile[4 * i + 3][j];
  const uint2 o[4] = {
      make_uint2(__byte_perm(q0.x, q1.x, 0x5410), __byte_perm(q2.x, q3.x, 0x5410)),
      make_uint2(__byte_perm(q0.x, q1.x, 0x7632), __byte_perm(q2.x, q3.x, 0x7632)),
      make_uint2(__byte_perm(q0.y, q1.y, 0x5410), __byte_perm(q2.y, q3.y, 0x5410)),
      make_uint2(__byte_perm(q0.y, q1.y, 0x7632), __byte_perm(q2.y, q3.y, 0x7632))};
  uint16_t* out = static_cast<uint16_t*>(a.out);
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int64_t cc = cb + 4 * j + b;
    if (cc >= a.c0 && cc < a.c1)
      *reinterpret_cast<uint2*>(out + (cc - a.c0) * a.pitch + tb + 4 * i) = o[b];
  }
}

// Full-layout copy of the prepared input (parity checks only): all channels.
template <typename T>
__global__ void k_prep_full(PrepArgs a) {
  const T* x = static_cast<const T*>(a.x);
  T* out = static_cast<T*>(a.full_out);
  const int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= a.nchans) return;
  for (int64_t t = blockIdx.y; t < a.nsamp; t += gridDim.y) {
  T v = x[t * a.nchans + c];
  if (a.segmask) {
    const int s = find_seg(a.seg_t0, a.nseg, t);
    if (a.segmask[static_cast<int64_t>(s) * a.nchans + c]) v = 0;
  }
  if (a.zdm_off && c >= a.zdm_cs && c < a.zdm_ce) {
    const uint32_t m = a.zdm_off[t];
    v = static_cast<T>(static_cast<uint32_t>(v) > m ? static_cast<uint32_t>(v) - m : 0u);
  }
  if (a.zdm_mean && c >= a.zdm_cs && c < a.zdm_ce) v = zdm_float_sub<T>(v, a.zdm_mean[t]);
  if (a.keep && !a.keep[c]) v = 0;
  out[t * a.nchans + c] = v;
  }
}

}  // namespace

int64_t binning_lut_entries(int nbits, int ds) {
  if (nbits != 8 && nbits != 16) return 0;
  const int64_t n = static_cast<int64_t>(ds) * (nbits == 8 ? 255 : 65535) + 1;
  return n <= (int64_t(1) << 24) ? n : 0;
}

void launch_binning_lut(void* lut, int nbits, int ds, cudaStream_t st) {
  const int64_t n = binning_lut_entries(nbits, ds);
  if (!n) throw Error{DD_ERR_RUNTIME, "no binning table for these samples"};
  const uint64_t vmax = nbits == 8 ? 255u : 65535u;
  const double smax_full = std::sqrt(static_cast<double>(vmax * static_cast<uint64_t>(ds)));
  const unsigned grid = static_cast<unsigned>((n + 255) / 256);
  if (nbits == 8) k_binning_lut<uint8_t><<<grid, 256, 0, st>>>(static_cast<uint8_t*>(lut), n, smax_full);
  else k_binning_lut<uint16_t><<<grid, 256, 0, st>>>(static_cast<uint16_t*>(lut), n, smax_full);
  DD_LAUNCHED();
}

void launch_time_binning(const void* in, void* out, int nbits, int64_t ndata, int64_t nchans,
                         int ds, const void* lut, cudaStream_t st) {
  const int64_t nout = (ndata + ds - 1) / ds;
  if (lut && (nbits == 8 || nbits == 16) && nchans % (32 / nbits) == 0 &&
      reinterpret_cast<uintptr_t>(in) % 4 == 0 && reinterpret_cast<uintptr_t>(out) % 4 == 0) {
    const int64_t nthreads = nchans / (32 / nbits);
    const dim3 g(static_cast<unsigned>((nthreads + 255) / 256),
                 static_cast<unsigned>(std::min<int64_t>(nout, 65535)));
    if (nbits == 8)
      k_time_binning_lut<uint8_t><<<g, 256, 0, st>>>(static_cast<const uint8_t*>(in), static_cast<uint8_t*>(out),
                                                     nchans, ndata, ds, nout, static_cast<const uint8_t*>(lut));
    else
      k_time_binning_lut<uint16_t><<<g, 256, 0, st>>>(static_cast<const uint16_t*>(in), static_cast<uint16_t*>(out),
                                                      nchans, ndata, ds, nout, static_cast<const uint16_t*>(lut));
    DD_LAUNCHED();
    return;
  }
  const dim3 grid(static_cast<unsigned>((nchans + 255) / 256),
                  static_cast<unsigned>(std::min<int64_t>(nout, 65535)));
  const uint64_t vmax = nbits == 8 ? 255u : nbits == 16 ? 65535u : 4294967295u;
  const double smax_full = std::sqrt(static_cast<double>(vmax * static_cast<uint64_t>(ds)));
  switch (nbits) {
    case 8: k_time_binning<uint8_t><<<grid, 256, 0, st>>>(static_cast<const uint8_t*>(in), static_cast<uint8_t*>(out), nchans, ndata, ds, nout, smax_full); break;
    case 16: k_time_binning<uint16_t><<<grid, 256, 0, st>>>(static_cast<const uint16_t*>(in), static_cast<uint16_t*>(out), nchans, ndata, ds, nout, smax_full); break;
    default: k_time_binning<uint32_t><<<grid, 256, 0, st>>>(static_cast<const uint32_t*>(in), static_cast<uint32_t*>(out), nchans, ndata, ds, nout, smax_full); break;
  }
  DD_LAUNCHED();
}

void launch_iqrm_stats(const void* x, int nbits, int64_t nsamp, int64_t nchans, int64_t cs,
                       int64_t csub, const uint32_t* d_win, int nwin, unsigned long long* d_sums,
                       cudaStream_t st) {
  DD_CUDA_TRY(cudaMemsetAsync(d_sums, 0, sizeof(unsigned long long) * 2 * csub * nwin, st));
  const int64_t chunk = 1024;
  dim3 grid(static_cast<unsigned>((csub + 255) / 256), static_cast<unsigned>((nsamp + chunk - 1) / chunk));
  if (nbits == 8 && nchans % 4 == 0 && reinterpret_cast<uintptr_t>(x) % 4 == 0) {
    const int64_t words = (csub + (cs & 3) + 3) / 4;
    dim3 g4(static_cast<unsigned>((words + 255) / 256), grid.y);
    k_iqrm_stats_u8w<<<g4, 256, 0, st>>>(static_cast<const uint8_t*>(x), nsamp, nchans, cs, csub,
                                         d_win, nwin, chunk, d_sums);
    DD_LAUNCHED();
    return;
  }
  switch (nbits) {
    case 8: k_iqrm_stats<uint8_t><<<grid, 256, 0, st>>>(static_cast<const uint8_t*>(x), nsamp, nchans, cs, csub, d_win, nwin, chunk, d_sums); break;
    case 16: k_iqrm_stats<uint16_t><<<grid, 256, 0, st>>>(static_cast<const uint16_t*>(x), nsamp, nchans, cs, csub, d_win, nwin, chunk, d_sums); break;
    default: k_iqrm_stats<uint32_t><<<grid, 256, 0, st>>>(static_cast<const uint32_t*>(x), nsamp, nchans, cs, csub, d_win, nwin, chunk, d_sums); break;
  }
  DD_LAUNCHED();
}

size_t iqrm_scratch_bytes(int nwin, int64_t csub, int nlags) {
  return static_cast<size_t>(nwin) * csub * (4 + 4 + 4 + 4 + nlags) + 256;
}

// k_iqrm_decide sorts one window's csub statistics in shared memory (the next
// power of two of csub floats); reject band widths whose sort buffer exceeds the
// current device's opt-in shared memory per block.
void check_iqrm_channels(int64_t csub) {
  int64_t sort_n = 1;
  while (sort_n < csub) sort_n <<= 1;
  int dev = 0, optin = 0;
  DD_CUDA_TRY(cudaGetDevice(&dev));
  DD_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const int64_t need = static_cast<int64_t>(sizeof(float)) * sort_n;
  if (need > optin) {
    char msg[200];
    std::snprintf(msg, sizeof(msg),
                  "IQRM over %lld channels needs a %lld-byte sort buffer, more than the %d bytes "
                  "of shared memory a block can have (at most %d channels)",
                  static_cast<long long>(csub), static_cast<long long>(need), optin,
                  optin / static_cast<int>(sizeof(float)));
    throw Error{DD_ERR_INVALID, msg};
  }
}

void launch_iqrm_decide(const unsigned long long* d_sums, int nwin, const uint32_t* d_win,
                        int64_t nchans, int64_t cs, int64_t csub, int mode, float nsigma,
                        const int32_t* d_lags, int nlags, int variant, void* scratch,
                        uint8_t* d_masks, cudaStream_t st) {
  char* p = static_cast<char*>(scratch);
  float* xs = reinterpret_cast<float*>(p); p += sizeof(float) * nwin * csub;
  float* ds_ = reinterpret_cast<float*>(p); p += sizeof(float) * nwin * csub;
  int* recv = reinterpret_cast<int*>(p); p += sizeof(int) * nwin * csub;
  int* cast_ = reinterpret_cast<int*>(p); p += sizeof(int) * nwin * csub;
  uint8_t* flags = reinterpret_cast<uint8_t*>(p);
  check_iqrm_channels(csub);
  int sort_n = 1;
  while (sort_n < csub) sort_n <<= 1;
  const size_t smem = sizeof(float) * sort_n;
  allow_dynamic_smem(k_iqrm_decide, smem);
  k_iqrm_decide<<<nwin, 1024, smem, st>>>(d_sums, d_win, nchans, cs, static_cast<int>(csub), mode,
                                          nsigma, d_lags, nlags, variant, xs, ds_, recv, cast_,
                                          flags, sort_n, d_masks);
  DD_LAUNCHED();
}

void launch_segment_masks(const uint8_t* d_masks, int nwin, const uint32_t* d_win,
                          const uint32_t* d_seg_t0, int nseg, int64_t nchans, uint8_t* d_segmask,
                          cudaStream_t st) {
  dim3 grid(static_cast<unsigned>((nchans + 255) / 256), static_cast<unsigned>(nseg));
  k_segment_masks<<<grid, 256, 0, st>>>(d_masks, nwin, d_win, d_seg_t0, nseg, nchans, d_segmask);
  DD_LAUNCHED();
}

void launch_apply_masks_inplace(void* x, int nbits, int64_t nsamp, int64_t nchans,
                                const uint8_t* d_segmask, const uint32_t* d_seg_t0, int nseg,
                                cudaStream_t st) {
  dim3 grid(static_cast<unsigned>((nchans + 255) / 256), static_cast<unsigned>(nsamp < 8192 ? nsamp : 8192));
  switch (nbits) {
    case 8: k_apply_masks<uint8_t><<<grid, 256, 0, st>>>(static_cast<uint8_t*>(x), nsamp, nchans, d_segmask, d_seg_t0, nseg); break;
    case 16: k_apply_masks<uint16_t><<<grid, 256, 0, st>>>(static_cast<uint16_t*>(x), nsamp, nchans, d_segmask, d_seg_t0, nseg); break;
    default: k_apply_masks<uint32_t><<<grid, 256, 0, st>>>(static_cast<uint32_t*>(x), nsamp, nchans, d_segmask, d_seg_t0, nseg); break;
  }
  DD_LAUNCHED();
}

void launch_zdm_offsets(const void* x, int nbits, int64_t nsamp, int64_t nchans, int64_t cs,
                        int64_t ce_excl, const uint8_t* d_segmask, const uint32_t* d_seg_t0,
                        int nseg, uint32_t* d_off, cudaStream_t st) {
  const unsigned blocks = static_cast<unsigned>((nsamp + 7) / 8);
  switch (nbits) {
    case 8: k_zdm_offsets<uint8_t><<<blocks, 256, 0, st>>>(static_cast<const uint8_t*>(x), nsamp, nchans, cs, ce_excl, d_segmask, d_seg_t0, nseg, d_off); break;
    case 16: k_zdm_offsets<uint16_t><<<blocks, 256, 0, st>>>(static_cast<const uint16_t*>(x), nsamp, nchans, cs, ce_excl, d_segmask, d_seg_t0, nseg, d_off); break;
    default: k_zdm_offsets<uint32_t><<<blocks, 256, 0, st>>>(static_cast<const uint32_t*>(x), nsamp, nchans, cs, ce_excl, d_segmask, d_seg_t0, nseg, d_off); break;
  }
  DD_LAUNCHED();
}

void launch_prep(const PrepArgs& a, cudaStream_t st) {
  // the word-wise kernels apply integer zero-DM offsets only
  if (a.out && !a.zdm_mean && a.nbits == 8 && a.ds == 1 && a.nchans % 4 == 0 && a.pitch % 4 == 0 &&
      reinterpret_cast<uintptr_t>(a.x) % 4 == 0 && reinterpret_cast<uintptr_t>(a.out) % 4 == 0) {
    const int64_t cw0 = a.c0 & ~int64_t(3);
    const int64_t span = 64 * kPrepU8Subtiles;
    dim3 grid(static_cast<unsigned>((a.nsamp + span - 1) / span), static_cast<unsigned>((a.c1 - cw0 + 63) / 64));
    k_prep_u8<<<grid, 256, 0, st>>>(a);
    DD_LAUNCHED();
  } else if (a.out && !a.zdm_mean && a.nbits == 16 && a.ds == 1 && a.nchans % 4 == 0 && a.pitch % 4 == 0 &&
             reinterpret_cast<uintptr_t>(a.x) % 8 == 0 && reinterpret_cast<uintptr_t>(a.out) % 8 == 0) {
    const int64_t cw0 = a.c0 & ~int64_t(3);
    dim3 grid(static_cast<unsigned>((a.nsamp + 63) / 64), static_cast<unsigned>((a.c1 - cw0 + 63) / 64));
    k_prep_u16<<<grid, 256, 0, st>>>(a);
    DD_LAUNCHED();
  } else if (a.out) {
    dim3 grid(static_cast<unsigned>((a.nsamp + 63) / 64), static_cast<unsigned>((a.c1 - a.c0 + 63) / 64));
    switch (a.nbits) {
      case 8: k_prep<uint8_t><<<grid, 256, 0, st>>>(a); break;
      case 16: k_prep<uint16_t><<<grid, 256, 0, st>>>(a); break;
      default: k_prep<uint32_t><<<grid, 256, 0, st>>>(a); break;
    }
    DD_LAUNCHED();
  }
  if (a.full_out) {
    dim3 grid(static_cast<unsigned>((a.nchans + 255) / 256), static_cast<unsigned>(a.nsamp < 8192 ? a.nsamp : 8192));
    switch (a.nbits) {
      case 8: k_prep_full<uint8_t><<<grid, 256, 0, st>>>(a); break;
      case 16: k_prep_full<uint16_t><<<grid, 256, 0, st>>>(a); break;
      default: k_prep_full<uint32_t><<<grid, 256, 0, st>>>(a); break;
    }
    DD_LAUNCHED();
  }
}

}  // namespace dd
