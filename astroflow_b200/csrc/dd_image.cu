// DM-time images on the GPU: the image step the reference runs on the host with
// OpenCV after every GPU call (include/data.h:620-727, preprocess_typed_
// dedisperseddata_with_slicing) and after the CPU path (data.h:299-369):
//
//   slice of columns -> float -> resize to target x target
//   (INTER_AREA when both dimensions exceed the target, else INTER_LANCZOS4)
//   -> min-max normalise to uint8 -> gray to RGB -> COLORMAP_VIRIDIS
//
// Resampling (both separable: a horizontal pass over every source row the
// output row needs, then a vertical combination), with the rounding of OpenCV's
// float path reproduced operation by operation (each product and each sum
// rounded to float, no fused multiply-add):
//   * area, general scale: each output pixel is the overlap-weighted mean of the
//     source pixels its cell covers (weight = overlap / cell width, overlaps
//     below 1e-3 of a pixel dropped, the last cell clipped to the source);
//     horizontal sums in increasing source column, vertical sums in increasing
//     source row;
//   * area, integer scales (both dimensions multiples of the target): the plain
//     block mean, row sums added row by row, times 1/area;
//   * Lanczos-4: taps at floor(f) - 3 .. floor(f) + 4 of f = (d + 0.5) * scale -
//     0.5 (indices clamped to the source), weights sin(pi x) sin(pi x / 4) /
//     (pi^2 x^2 / 4) at the tap distances, evaluated in double through the
//     angle-addition form, rounded to float and normalised by the float
//     reciprocal of their float sum; horizontal taps summed first to last,
//     vertical taps last to first.
// The weight tables are built on the host in double; the GPU only applies them.
// Normalisation: scale = 255 / (max - min) in double (0 when the image is flat),
// shift = -min * scale, u8 = round-half-even(fmaf(x, (float)scale,
// (float)shift)) clamped to [0, 255]; the color map is a 256-entry BGR table
// supplied by the caller.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <vector>

#include "dd_internal.h"

namespace dd {
namespace {

constexpr int kImgThreads = 256;
constexpr int kStageFloats = 12288;  // source row staged in shared memory up to this width
constexpr double kPi = 3.14159265358979323846;

enum AxisMethod { kAreaGeneral = 0, kAreaInteger = 1, kLanczos = 2 };

// One axis (source size -> target size) as CSR lists of (source index, weight)
// per output index.  Lanczos lists have 8 taps; integer area lists hold the
// block's first index only (the block length is the scale).
struct AxisTab {
  std::vector<int32_t> off, idx;
  std::vector<float> w;
};

AxisTab area_table(int64_t ssize, int dsize) {
  AxisTab t;
  const double scale = static_cast<double>(ssize) / dsize;
  t.off.push_back(0);
  for (int d = 0; d < dsize; ++d) {
    const double f1 = d * scale, f2 = f1 + scale;
    const double cell = std::min(scale, static_cast<double>(ssize) - f1);
    int64_t s1 = static_cast<int64_t>(std::ceil(f1)), s2 = static_cast<int64_t>(std::floor(f2));
    s2 = std::min<int64_t>(s2, ssize - 1);
    s1 = std::min<int64_t>(s1, ssize - 1);
    if (static_cast<double>(s1) - f1 > 1e-3) {
      t.idx.push_back(static_cast<int32_t>(s1 - 1));
      t.w.push_back(static_cast<float>((static_cast<double>(s1) - f1) / cell));
    }
    for (int64_t s = s1; s < s2; ++s) {
      t.idx.push_back(static_cast<int32_t>(s));
      t.w.push_back(static_cast<float>(1.0 / cell));
    }
    if (f2 - static_cast<double>(s2) > 1e-3) {
      t.idx.push_back(static_cast<int32_t>(s2));
      t.w.push_back(static_cast<float>(std::min(std::min(f2 - static_cast<double>(s2), 1.0), cell) / cell));
    }
    t.off.push_back(static_cast<int32_t>(t.idx.size()));
  }
  return t;
}

AxisTab integer_area_table(int64_t ssize, int dsize) {
  AxisTab t;
  const int64_t k = ssize / dsize;
  for (int d = 0; d <= dsize; ++d) t.off.push_back(d);
  for (int d = 0; d < dsize; ++d) {
    t.idx.push_back(static_cast<int32_t>(d * k));
    t.w.push_back(0.0f);
  }
  return t;
}

// Lanczos-4 weights of the 8 taps for fractional position x in (0, 1).
void lanczos4_weights(float x, float* out) {
  if (x < FLT_EPSILON) {
    for (int i = 0; i < 8; ++i) out[i] = 0.0f;
    out[3] = 1.0f;
    return;
  }
  // sin(pi x_i / 4) for x_i = x + 3 - i rotates by 45 degrees from tap to tap;
  // sin(pi x_i) alternates in sign and cancels in the normalisation.
  const double r = std::sqrt(0.5);
  const double rot[8][2] = {{1, 0}, {-r, -r}, {0, 1}, {r, -r}, {-1, 0}, {r, r}, {0, -1}, {-r, r}};
  const double a0 = -(static_cast<double>(x) + 3) * kPi * 0.25;
  const double s0 = std::sin(a0), c0 = std::cos(a0);
  volatile float sum = 0.0f;
  for (int i = 0; i < 8; ++i) {
    const double a = -(static_cast<double>(x) + 3 - i) * kPi * 0.25;
    out[i] = static_cast<float>((rot[i][0] * s0 + rot[i][1] * c0) / (a * a));
    sum = sum + out[i];
  }
  volatile float inv = 1.0f / sum;
  for (int i = 0; i < 8; ++i) {
    volatile float v = out[i] * inv;
    out[i] = v;
  }
}

AxisTab lanczos_table(int64_t ssize, int dsize) {
  AxisTab t;
  const double scale = static_cast<double>(ssize) / dsize;
  for (int d = 0; d < dsize; ++d) {
    const float f = static_cast<float>((d + 0.5) * scale - 0.5);
    const int64_t s = static_cast<int64_t>(std::floor(f));
    volatile float frac = f - static_cast<float>(s);
    float w[8];
    lanczos4_weights(frac, w);
    t.off.push_back(8 * d);
    for (int i = 0; i < 8; ++i) {
      t.idx.push_back(static_cast<int32_t>(std::min(std::max<int64_t>(s - 3 + i, 0), ssize - 1)));
      t.w.push_back(w[i]);
    }
  }
  t.off.push_back(8 * dsize);
  return t;
}

struct ImgLaunch {
  const void* src;      // [rows][pitch] uint32 or uint64
  int64_t pitch;        // elements between rows
  int elem;             // 4 or 8
  int64_t rows, cols;   // slice size
  const int64_t* col0;  // per slice of the group: first column
  int method;
  int target;
  const int32_t* hoff; const int32_t* hidx; const float* hw;
  // general area, horizontal: per output column its first source column, source
  // count and weights (first, interior, last); the interior ones are all equal
  const int32_t* ha_i0; const int32_t* ha_n; const float4* ha_w;
  const int32_t* voff; const int32_t* vidx; const float* vw;
  int ky, kx;           // integer area: block size
  float inv_area;
  float* out;           // [slice][target][target]
  const int* out_slot;  // per slice of the group: index into out
};

__device__ __forceinline__ float to_float(const void* src, int elem, int64_t i) {
  if (elem == 8) return __ull2float_rn(static_cast<const unsigned long long*>(src)[i]);
  return __uint2float_rn(static_cast<const uint32_t*>(src)[i]);
}

// One block per (output row, slice).  Each source row the output row needs is
// brought into shared memory as float (when it fits), then every thread
// resamples its output columns from it.
#ifndef DD_IMG_MINB
#define DD_IMG_MINB 3
#endif
__global__ void __launch_bounds__(kImgThreads, DD_IMG_MINB) k_resize(ImgLaunch L) {
  __shared__ __align__(16) float row[kStageFloats];
  const int dy = blockIdx.x;
  const int s = blockIdx.y;
  const int64_t c0 = L.col0[s];
  const bool staged = L.cols <= kStageFloats;
  constexpr int kMaxPer = 4;  // output columns per thread (target <= 1024)
  float acc[kMaxPer];
  float* out = L.out + (static_cast<int64_t>(L.out_slot[s]) * L.target + dy) * L.target;
  const int per = (L.target + kImgThreads - 1) / kImgThreads;
  const int v0 = L.voff[dy], v1 = L.voff[dy + 1];
  const int nv = L.method == kAreaInteger ? L.ky : v1 - v0;
  int a_i0[kMaxPer], a_n[kMaxPer];
  float4 a_w[kMaxPer];
  if (L.method == kAreaGeneral) {
    for (int q = 0; q < per && q < kMaxPer; ++q) {
      const int dx = threadIdx.x + q * kImgThreads;
      if (dx >= L.target) break;
      a_i0[q] = L.ha_i0[dx];
      a_n[q] = L.ha_n[dx];
      a_w[q] = L.ha_w[dx];
    }
  }
  for (int j = 0; j < nv; ++j) {
    // taps in summation order: Lanczos vertical taps last to first
    const int k = L.method == kLanczos ? v1 - 1 - j : v0 + j;
    const int64_t sy = L.method == kAreaInteger ? static_cast<int64_t>(L.vidx[dy]) + j : L.vidx[k];
    const int64_t base = sy * L.pitch + c0;
    if (staged) {
      __syncthreads();
      if (L.elem == 4 && (base & 3) == 0) {  // 16-byte loads of four 32-bit sums
        const uint4* src4 = reinterpret_cast<const uint4*>(static_cast<const uint32_t*>(L.src) + base);
        const int64_t n4 = L.cols >> 2;
        for (int64_t i = threadIdx.x; i < n4; i += kImgThreads) {
          const uint4 v = __ldg(src4 + i);
          reinterpret_cast<float4*>(row)[i] = make_float4(__uint2float_rn(v.x), __uint2float_rn(v.y),
                                                          __uint2float_rn(v.z), __uint2float_rn(v.w));
        }
        for (int64_t i = 4 * n4 + threadIdx.x; i < L.cols; i += kImgThreads)
          row[i] = to_float(L.src, L.elem, base + i);
      } else {
        for (int64_t i = threadIdx.x; i < L.cols; i += kImgThreads) row[i] = to_float(L.src, L.elem, base + i);
      }
      __syncthreads();
    }
    for (int q = 0; q < per && q < kMaxPer; ++q) {
      const int dx = threadIdx.x + q * kImgThreads;
      if (dx >= L.target) break;
      float h;
      if (L.method == kAreaInteger) {
        const int64_t sx = L.hidx[dx];
        h = staged ? row[sx] : to_float(L.src, L.elem, base + sx);
        for (int i = 1; i < L.kx; ++i)
          h = __fadd_rn(h, staged ? row[sx + i] : to_float(L.src, L.elem, base + sx + i));
      } else {
        if (L.method == kLanczos) {
          const int h0 = L.hoff[dx], h1 = L.hoff[dx + 1];
          const int sx = L.hidx[h0];
          h = __fmul_rn(staged ? row[sx] : to_float(L.src, L.elem, base + sx), L.hw[h0]);
          for (int e = h0 + 1; e < h1; ++e) {
            const int x = L.hidx[e];
            h = __fadd_rn(h, __fmul_rn(staged ? row[x] : to_float(L.src, L.elem, base + x), L.hw[e]));
          }
        } else {
          // first, interior and last sources, each product and sum rounded to float
          const int x0 = a_i0[q], n = a_n[q];
          const float4 w = a_w[q];
          h = __fmul_rn(staged ? row[x0] : to_float(L.src, L.elem, base + x0), w.x);
          for (int i = 1; i < n - 1; ++i)
            h = __fadd_rn(h, __fmul_rn(staged ? row[x0 + i] : to_float(L.src, L.elem, base + x0 + i), w.y));
          if (n > 1)
            h = __fadd_rn(h, __fmul_rn(staged ? row[x0 + n - 1] : to_float(L.src, L.elem, base + x0 + n - 1), w.z));
        }
      }
      if (L.method == kAreaInteger) {
        acc[q] = j == 0 ? h : __fadd_rn(acc[q], h);
      } else if (L.method == kLanczos) {
        const float t = __fmul_rn(h, L.vw[k]);
        acc[q] = j == 0 ? t : __fadd_rn(acc[q], t);
      } else {
        acc[q] = __fadd_rn(j == 0 ? 0.0f : acc[q], __fmul_rn(h, L.vw[k]));
      }
    }
  }
  for (int q = 0; q < per && q < kMaxPer; ++q) {
    const int dx = threadIdx.x + q * kImgThreads;
    if (dx >= L.target) break;
    out[dx] = L.method == kAreaInteger ? __fmul_rn(acc[q], L.inv_area) : acc[q];
  }
}

// Per image: min and max of the resized floats, then the scale and shift of the
// min-max normalisation.
__global__ void __launch_bounds__(1024) k_minmax(const float* img, int64_t npix, float2* ab) {
  __shared__ float smin[32], smax[32];
  const float* p = img + static_cast<int64_t>(blockIdx.x) * npix;
  float mn = FLT_MAX, mx = -FLT_MAX;
  for (int64_t i = threadIdx.x; i < npix; i += blockDim.x) {
    const float v = p[i];
    mn = fminf(mn, v);
    mx = fmaxf(mx, v);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { smin[w] = mn; smax[w] = mx; }
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    mn = l < nw ? smin[l] : FLT_MAX;
    mx = l < nw ? smax[l] : -FLT_MAX;
    for (int o = 16; o > 0; o >>= 1) {
      mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
      mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if (l == 0) {
      const double d = static_cast<double>(mx) - static_cast<double>(mn);
      const double scale = d > DBL_EPSILON ? __ddiv_rn(255.0, d) : 0.0;
      const double shift = 0.0 - static_cast<double>(mn) * scale;
      ab[blockIdx.x] = make_float2(__double2float_rn(scale), __double2float_rn(shift));
    }
  }
}

struct Lut {
  uint8_t bgr[768];
};

// Normalise, then color: one thread per pixel, 3 bytes (B, G, R) out.
__global__ void k_colorize(const float* img, int64_t npix, const float2* ab, Lut lut,
                           uint8_t* out) {
  __shared__ uint8_t s_lut[768];
  for (int i = threadIdx.x; i < 768; i += blockDim.x) s_lut[i] = lut.bgr[i];
  __syncthreads();
  const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int img_i = blockIdx.y;
  if (p >= npix) return;
  const float2 k = ab[img_i];
  const float v = __fmaf_rn(img[static_cast<int64_t>(img_i) * npix + p], k.x, k.y);
  const int u = min(max(__float2int_rn(v), 0), 255);
  uint8_t* o = out + (static_cast<int64_t>(img_i) * npix + p) * 3;
  o[0] = s_lut[3 * u];
  o[1] = s_lut[3 * u + 1];
  o[2] = s_lut[3 * u + 2];
}

template <typename T>
T* upload(const std::vector<T>& v, cudaStream_t st, std::vector<void*>& scratch) {
  void* p = nullptr;
  DD_CUDA_TRY(cudaMallocAsync(&p, std::max<size_t>(v.size() * sizeof(T), 16), st));
  scratch.push_back(p);
  if (!v.empty())
    DD_CUDA_TRY(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  return static_cast<T*>(p);
}

}  // namespace
}  // namespace dd

using namespace dd;

extern "C" int dd_images(const void* dm_time, int32_t elem_bytes, int64_t nrows, int64_t row_pitch,
                         int32_t nslices, const int64_t* col_start, const int64_t* col_count,
                         int32_t target, const uint8_t* lut_bgr, uint8_t* images, float* resized,
                         void* stream) {
  if (!dm_time || !col_start || !col_count || (!images && !resized) || (images && !lut_bgr)) {
    set_error("NULL argument");
    return DD_ERR_INVALID;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::vector<void*> scratch;
  int rc = DD_OK;
  try {
    set_error("");
    if (elem_bytes != 4 && elem_bytes != 8) throw Error{DD_ERR_INVALID, "elem_bytes must be 4 or 8"};
    if (nrows < 1 || nslices < 0 || target < 1 || target > 4 * kImgThreads)
      throw Error{DD_ERR_INVALID, "bad image geometry"};
    if (nslices == 0) return DD_OK;
    for (int32_t i = 0; i < nslices; ++i)
      if (col_count[i] < 1 || col_start[i] < 0 || col_start[i] + col_count[i] > row_pitch)
        throw Error{DD_ERR_INVALID, "slice outside the rows"};
    const int64_t npix = static_cast<int64_t>(target) * target;
    float* img = resized;
    if (!img) {
      void* p = nullptr;
      DD_CUDA_TRY(cudaMallocAsync(&p, sizeof(float) * npix * nslices, st));
      scratch.push_back(p);
      img = static_cast<float*>(p);
    }
    // slices of equal width share one launch and one pair of tables
    std::map<int64_t, std::vector<int32_t>> groups;
    for (int32_t i = 0; i < nslices; ++i) groups[col_count[i]].push_back(i);
    for (const auto& kv : groups) {
      const int64_t cols = kv.first;
      const bool area = nrows > target && cols > target;
      const bool integer = area && nrows % target == 0 && cols % target == 0;
      const int method = integer ? kAreaInteger : area ? kAreaGeneral : kLanczos;
      AxisTab h = integer ? integer_area_table(cols, target)
                  : area  ? area_table(cols, target)
                          : lanczos_table(cols, target);
      AxisTab v = integer ? integer_area_table(nrows, target)
                  : area  ? area_table(nrows, target)
                          : lanczos_table(nrows, target);
      std::vector<int64_t> c0;
      std::vector<int> slot;
      for (int32_t i : kv.second) {
        c0.push_back(col_start[i]);
        slot.push_back(i);
      }
      ImgLaunch L{};
      L.src = dm_time;
      L.pitch = row_pitch;
      L.elem = elem_bytes;
      L.rows = nrows;
      L.cols = cols;
      L.col0 = upload(c0, st, scratch);
      L.out_slot = upload(slot, st, scratch);
      L.method = method;
      L.target = target;
      L.hoff = upload(h.off, st, scratch);
      L.hidx = upload(h.idx, st, scratch);
      L.hw = upload(h.w, st, scratch);
      L.voff = upload(v.off, st, scratch);
      L.vidx = upload(v.idx, st, scratch);
      L.vw = upload(v.w, st, scratch);
      if (method == kAreaGeneral) {
        std::vector<int32_t> i0(static_cast<size_t>(target)), n(static_cast<size_t>(target));
        std::vector<float4> w(static_cast<size_t>(target));
        for (int d = 0; d < target; ++d) {
          const int a = h.off[d], b = h.off[d + 1];
          if (b <= a) throw Error{DD_ERR_RUNTIME, "empty area cell"};
          i0[d] = h.idx[a];
          n[d] = b - a;
          const float mid = b - a > 2 ? h.w[a + 1] : h.w[a];
          for (int e = a; e < b; ++e) {
            if (h.idx[e] != h.idx[a] + (e - a) || (e > a && e < b - 1 && h.w[e] != mid))
              throw Error{DD_ERR_RUNTIME, "area table is not a contiguous run"};
          }
          w[d] = make_float4(h.w[a], mid, h.w[b - 1], 0.0f);
        }
        L.ha_i0 = upload(i0, st, scratch);
        L.ha_n = upload(n, st, scratch);
        L.ha_w = upload(w, st, scratch);
      }
      L.ky = static_cast<int>(nrows / target);
      L.kx = static_cast<int>(cols / target);
      L.inv_area = integer ? static_cast<float>(1.0 / (static_cast<double>(L.kx) * L.ky)) : 1.0f;
      L.out = img;
      const int64_t ng = static_cast<int64_t>(kv.second.size());
      for (int64_t g0 = 0; g0 < ng; g0 += 65535) {
        ImgLaunch Lg = L;
        Lg.col0 = L.col0 + g0;
        Lg.out_slot = L.out_slot + g0;
        dim3 grid(static_cast<unsigned>(target), static_cast<unsigned>(std::min<int64_t>(ng - g0, 65535)));
        k_resize<<<grid, kImgThreads, 0, st>>>(Lg);
        DD_LAUNCHED();
      }
    }
    if (images) {
      void* p = nullptr;
      DD_CUDA_TRY(cudaMallocAsync(&p, sizeof(float2) * nslices, st));
      scratch.push_back(p);
      float2* ab = static_cast<float2*>(p);
      k_minmax<<<nslices, 1024, 0, st>>>(img, npix, ab);
      DD_LAUNCHED();
      Lut lut;
      std::memcpy(lut.bgr, lut_bgr, sizeof(lut.bgr));
      for (int32_t i0 = 0; i0 < nslices; i0 += 65535) {
        const int32_t n = std::min<int32_t>(nslices - i0, 65535);
        dim3 grid(static_cast<unsigned>((npix + 255) / 256), static_cast<unsigned>(n));
        k_colorize<<<grid, 256, 0, st>>>(img + static_cast<int64_t>(i0) * npix, npix, ab + i0, lut,
                                          images + static_cast<int64_t>(i0) * npix * 3);
        DD_LAUNCHED();
      }
    }
  } catch (const Error& e) {
    set_error(e.msg);
    rc = e.code;
  }
  for (void* p : scratch) cudaFreeAsync(p, st);
  return rc;
}
