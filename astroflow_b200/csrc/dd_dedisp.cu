// Dedispersion sums for the B200 path: one "shift-and-add" kernel family,
//
//   out[r][t] = sum_i src_i(r)[t + off(r, i)]
//
// instantiated for the three sums of astroflow's path:
//   * subband stage 1 (src/core/dedispered.cu:416-447): rows = nominal DMs of one
//     subband, sources = the subband's channels, offsets = coarse delays;
//   * subband stage 2 (dedispered.cu:449-476): rows = the fine DMs of one
//     nominal DM, sources = that nominal DM's subband sums, offsets = residuals;
//   * brute force with the CPU path's semantics (include/cpucal.hpp:154-190):
//     rows = DMs, sources = channels, offsets = per-DM channel delays.
// Sources are channel-major rows, zero-padded past their valid length so the
// reference's bound tests (t + delay < N) become reads of zeros.
//
// Work decomposition: a block of 256 threads covers 2048 consecutive output
// samples (8 per thread) for RB output rows; every thread keeps RB x 8 sums in
// registers.  Source samples are fetched as aligned 32-bit words through the
// read-only path and funnel-shifted to the row's offset.  8-bit samples are
// accumulated two per 32-bit register (16-bit lanes, split with one byte
// permute per word), so one integer add performs two sample additions; lanes
// are widened into 32-bit sums before they can overflow.
#include <cuda_runtime.h>

#include <cstdint>

#include "dd_internal.h"

namespace dd {
namespace {

constexpr int kThreads = 256;
constexpr int kRun = 8;                       // samples per thread
constexpr int kTile = kThreads * kRun;        // samples per block
constexpr int kRows = 8;                      // output rows per block

__device__ __forceinline__ uint32_t ldg32(const void* p) {
  return __ldg(static_cast<const uint32_t*>(p));
}

// Adds the 8 bytes row[pos .. pos+8) into acc as 16-bit lane pairs:
// acc[0] += (b0, b2), acc[1] += (b1, b3), acc[2] += (b4, b6), acc[3] += (b5, b7).
__device__ __forceinline__ void add8_u8(const uint8_t* row, int64_t pos, uint32_t (&acc)[4]) {
  const uint8_t* base = row + (pos & ~int64_t(3));
  const uint32_t w0 = ldg32(base), w1 = ldg32(base + 4), w2 = ldg32(base + 8);
  const uint32_t sh = static_cast<uint32_t>(pos & 3) * 8u;
  const uint32_t a = __funnelshift_r(w0, w1, sh);
  const uint32_t b = __funnelshift_r(w1, w2, sh);
  acc[0] += __byte_perm(a, 0u, 0x4240);
  acc[1] += __byte_perm(a, 0u, 0x4341);
  acc[2] += __byte_perm(b, 0u, 0x4240);
  acc[3] += __byte_perm(b, 0u, 0x4341);
}

// Loads 8 consecutive 16-bit samples row[pos .. pos+8) as 4 lane pairs.
__device__ __forceinline__ void load8_u16(const uint16_t* row, int64_t pos, uint32_t (&v)[4]) {
  const uint16_t* base = row + (pos & ~int64_t(1));
  const uint32_t w0 = ldg32(base), w1 = ldg32(base + 2), w2 = ldg32(base + 4), w3 = ldg32(base + 6);
  if (pos & 1) {
    const uint32_t w4 = ldg32(base + 8);
    v[0] = __funnelshift_r(w0, w1, 16);
    v[1] = __funnelshift_r(w1, w2, 16);
    v[2] = __funnelshift_r(w2, w3, 16);
    v[3] = __funnelshift_r(w3, w4, 16);
  } else {
    v[0] = w0; v[1] = w1; v[2] = w2; v[3] = w3;
  }
}

// 32-bit sums of the 16-bit-lane accumulator words into acc32[8] (sample order).
__device__ __forceinline__ void widen_u8pairs(uint32_t (&a16)[4], uint32_t (&a32)[8]) {
  a32[0] += a16[0] & 0xffffu; a32[2] += a16[0] >> 16;
  a32[1] += a16[1] & 0xffffu; a32[3] += a16[1] >> 16;
  a32[4] += a16[2] & 0xffffu; a32[6] += a16[2] >> 16;
  a32[5] += a16[3] & 0xffffu; a32[7] += a16[3] >> 16;
  a16[0] = a16[1] = a16[2] = a16[3] = 0;
}
__device__ __forceinline__ void widen_u16pairs(uint32_t (&a16)[4], uint32_t (&a32)[8]) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    a32[2 * k] += a16[k] & 0xffffu;
    a32[2 * k + 1] += a16[k] >> 16;
    a16[k] = 0;
  }
}

template <typename O>
__device__ __forceinline__ void store_run(O* dst, int64_t valid, const O (&v)[8]) {
  if (valid >= 8 && (reinterpret_cast<uintptr_t>(dst) % 16) == 0) {
    if constexpr (sizeof(O) == 4) {
      reinterpret_cast<uint4*>(dst)[0] = make_uint4(v[0], v[1], v[2], v[3]);
      reinterpret_cast<uint4*>(dst)[1] = make_uint4(v[4], v[5], v[6], v[7]);
    } else {
#pragma unroll
      for (int k = 0; k < 8; ++k) dst[k] = v[k];
    }
  } else {
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (k < valid) dst[k] = v[k];
  }
}

// ---------------------------------------------------------------- stage 1
// grid: x = time tile, y = block of kRows nominal DMs, z = subband.
__global__ void __launch_bounds__(kThreads) k_stage1_u8(Stage1Args a) {
  const int64_t t_local = static_cast<int64_t>(blockIdx.x) * kTile + threadIdx.x * kRun;
  const int64_t j0 = static_cast<int64_t>(blockIdx.y) * kRows;
  const int64_t sb = blockIdx.z;
  const int64_t c0 = sb * a.sbw;
  const int64_t c1 = c0 + a.sbw < a.dch ? c0 + a.sbw : a.dch;
  const uint8_t* x = static_cast<const uint8_t*>(a.x);
  uint32_t acc[kRows][4];
  uint32_t wide[kRows][8];
#pragma unroll
  for (int r = 0; r < kRows; ++r) {
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[r][k] = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) wide[r][k] = 0;
  }
  const int64_t nrows = a.ndm_nom - j0 < kRows ? a.ndm_nom - j0 : kRows;
  int since = 0;
  for (int64_t c = c0; c < c1; ++c) {
    const uint8_t* row = x + c * a.xpitch;
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      if (r < nrows) {
        const int64_t d = __ldg(a.delay1 + (j0 + r) * a.dch + c);
        add8_u8(row, a.t0 + t_local + d, acc[r]);
      }
    }
    if (++since == 257) {  // 257 x 255 still fits a 16-bit lane
#pragma unroll
      for (int r = 0; r < kRows; ++r) widen_u8pairs(acc[r], wide[r]);
      since = 0;
    }
  }
  const int64_t valid = a.ncols - t_local;
  if (valid <= 0) return;
  for (int r = 0; r < nrows; ++r) {
    const int64_t orow = ((j0 + r) * a.nsb + sb) * a.tile_pitch + t_local;
    if (a.inter16) {
      uint16_t v[8];
      v[0] = acc[r][0] & 0xffffu; v[2] = acc[r][0] >> 16;
      v[1] = acc[r][1] & 0xffffu; v[3] = acc[r][1] >> 16;
      v[4] = acc[r][2] & 0xffffu; v[6] = acc[r][2] >> 16;
      v[5] = acc[r][3] & 0xffffu; v[7] = acc[r][3] >> 16;
      uint16_t* dst = static_cast<uint16_t*>(a.inter) + orow;
      if (valid >= 8) {
        uint4 pk;
        pk.x = v[0] | (uint32_t(v[1]) << 16); pk.y = v[2] | (uint32_t(v[3]) << 16);
        pk.z = v[4] | (uint32_t(v[5]) << 16); pk.w = v[6] | (uint32_t(v[7]) << 16);
        *reinterpret_cast<uint4*>(dst) = pk;
      } else {
        for (int k = 0; k < valid; ++k) dst[k] = v[k];
      }
    } else {
      widen_u8pairs(acc[r], wide[r]);
      uint32_t v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) v[k] = wide[r][k];
      store_run(static_cast<uint32_t*>(a.inter) + orow, valid, v);
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_stage1_wide(Stage1Args a) {
  const int64_t t_local = static_cast<int64_t>(blockIdx.x) * kTile + threadIdx.x * kRun;
  const int64_t j0 = static_cast<int64_t>(blockIdx.y) * kRows;
  const int64_t sb = blockIdx.z;
  const int64_t c0 = sb * a.sbw;
  const int64_t c1 = c0 + a.sbw < a.dch ? c0 + a.sbw : a.dch;
  const T* x = static_cast<const T*>(a.x);
  uint32_t acc[kRows][8];
#pragma unroll
  for (int r = 0; r < kRows; ++r)
#pragma unroll
    for (int k = 0; k < 8; ++k) acc[r][k] = 0;
  const int64_t nrows = a.ndm_nom - j0 < kRows ? a.ndm_nom - j0 : kRows;
  for (int64_t c = c0; c < c1; ++c) {
    const T* row = x + c * a.xpitch;
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      if (r < nrows) {
        const int64_t pos = a.t0 + t_local + __ldg(a.delay1 + (j0 + r) * a.dch + c);
        if constexpr (sizeof(T) == 2) {
          uint32_t v[4];
          load8_u16(row, pos, v);
#pragma unroll
          for (int k = 0; k < 4; ++k) { acc[r][2 * k] += v[k] & 0xffffu; acc[r][2 * k + 1] += v[k] >> 16; }
        } else {
#pragma unroll
          for (int k = 0; k < 8; ++k) acc[r][k] += __ldg(row + pos + k);
        }
      }
    }
  }
  const int64_t valid = a.ncols - t_local;
  if (valid <= 0) return;
  for (int r = 0; r < nrows; ++r) {
    const int64_t orow = ((j0 + r) * a.nsb + sb) * a.tile_pitch + t_local;
    uint32_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = acc[r][k];
    store_run(static_cast<uint32_t*>(a.inter) + orow, valid, v);
  }
}

// ---------------------------------------------------------------- stage 2
// grid: x = time tile, y = block of kRows fine DMs inside one nominal DM.
__global__ void __launch_bounds__(kThreads) k_stage2(Stage2Args a) {
  const int64_t t_local = static_cast<int64_t>(blockIdx.x) * kTile + threadIdx.x * kRun;
  const int blocks_per_nom = (a.ndm0 + kRows - 1) / kRows;
  const int64_t j = blockIdx.y / blocks_per_nom;
  const int64_t m0 = j * a.ndm0 + static_cast<int64_t>(blockIdx.y % blocks_per_nom) * kRows;
  const int64_t mend_nom = (j + 1) * a.ndm0 < a.dm_steps ? (j + 1) * a.ndm0 : a.dm_steps;
  const int64_t nrows = mend_nom - m0 < kRows ? mend_nom - m0 : kRows;
  if (nrows <= 0) return;
  uint32_t wide[kRows][8];
#pragma unroll
  for (int r = 0; r < kRows; ++r)
#pragma unroll
    for (int k = 0; k < 8; ++k) wide[r][k] = 0;
  const int64_t inter_base = j * a.nsb * a.tile_pitch;
  if (a.inter16) {
    const uint16_t* inter = static_cast<const uint16_t*>(a.inter) + inter_base;
    // Lanes hold sums of up to `per` subband values before they are widened.
    const int per = a.src_max > 0 ? (65535 / a.src_max < 1 ? 1 : 65535 / a.src_max) : 1;
    uint32_t acc[kRows][4];
#pragma unroll
    for (int r = 0; r < kRows; ++r)
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[r][k] = 0;
    int since = 0;
    for (int64_t sb = 0; sb < a.nsb; ++sb) {
      const uint16_t* row = inter + sb * a.tile_pitch;
#pragma unroll
      for (int r = 0; r < kRows; ++r) {
        if (r < nrows) {
          const int64_t pos = t_local + __ldg(a.res + (m0 + r) * a.nsb + sb);
          uint32_t v[4];
          load8_u16(row, pos, v);
#pragma unroll
          for (int k = 0; k < 4; ++k) acc[r][k] += v[k];
        }
      }
      if (++since == per) {
#pragma unroll
        for (int r = 0; r < kRows; ++r) widen_u16pairs(acc[r], wide[r]);
        since = 0;
      }
    }
#pragma unroll
    for (int r = 0; r < kRows; ++r) widen_u16pairs(acc[r], wide[r]);
  } else {
    const uint32_t* inter = static_cast<const uint32_t*>(a.inter) + inter_base;
    for (int64_t sb = 0; sb < a.nsb; ++sb) {
      const uint32_t* row = inter + sb * a.tile_pitch;
#pragma unroll
      for (int r = 0; r < kRows; ++r) {
        if (r < nrows) {
          const int64_t pos = t_local + __ldg(a.res + (m0 + r) * a.nsb + sb);
#pragma unroll
          for (int k = 0; k < 8; ++k) wide[r][k] += __ldg(row + pos + k);
        }
      }
    }
  }
  const int64_t valid = a.ncols - t_local;
  if (valid <= 0) return;
  for (int r = 0; r < nrows; ++r) {
    uint32_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = wide[r][k];
    store_run(static_cast<uint32_t*>(a.out) + (m0 + r) * a.out_pitch + a.col0 + t_local, valid, v);
  }
}

// ---------------------------------------------------------------- 32-bit samples
// For 32-bit samples the subband sums and the output are 64-bit
// (dedispersion_output_t<uint32_t> is uint64_t, include/data.h:98-118).  Four
// rows per block keep the 64-bit accumulators in registers.
constexpr int kRows64 = 4;

__global__ void __launch_bounds__(kThreads) k_stage1_u32(Stage1Args a) {
  const int64_t t_local = static_cast<int64_t>(blockIdx.x) * kTile + threadIdx.x * kRun;
  const int64_t j0 = static_cast<int64_t>(blockIdx.y) * kRows64;
  const int64_t sb = blockIdx.z;
  const int64_t c0 = sb * a.sbw;
  const int64_t c1 = c0 + a.sbw < a.dch ? c0 + a.sbw : a.dch;
  const uint32_t* x = static_cast<const uint32_t*>(a.x);
  unsigned long long acc[kRows64][kRun];
#pragma unroll
  for (int r = 0; r < kRows64; ++r)
#pragma unroll
    for (int k = 0; k < kRun; ++k) acc[r][k] = 0;
  const int64_t nrows = a.ndm_nom - j0 < kRows64 ? a.ndm_nom - j0 : kRows64;
  for (int64_t c = c0; c < c1; ++c) {
    const uint32_t* row = x + c * a.xpitch;
#pragma unroll
    for (int r = 0; r < kRows64; ++r) {
      if (r < nrows) {
        const int64_t pos = a.t0 + t_local + __ldg(a.delay1 + (j0 + r) * a.dch + c);
#pragma unroll
        for (int k = 0; k < kRun; ++k) acc[r][k] += __ldg(row + pos + k);
      }
    }
  }
  const int64_t valid = a.ncols - t_local;
  if (valid <= 0) return;
  for (int r = 0; r < nrows; ++r) {
    unsigned long long* dst = static_cast<unsigned long long*>(a.inter) +
                              ((j0 + r) * a.nsb + sb) * a.tile_pitch + t_local;
#pragma unroll
    for (int k = 0; k < kRun; ++k)
      if (k < valid) dst[k] = acc[r][k];
  }
}

__global__ void __launch_bounds__(kThreads) k_stage2_u64(Stage2Args a) {
  const int64_t t_local = static_cast<int64_t>(blockIdx.x) * kTile + threadIdx.x * kRun;
  const int blocks_per_nom = (a.ndm0 + kRows64 - 1) / kRows64;
  const int64_t j = blockIdx.y / blocks_per_nom;
  const int64_t m0 = j * a.ndm0 + static_cast<int64_t>(blockIdx.y % blocks_per_nom) * kRows64;
  const int64_t mend_nom = (j + 1) * a.ndm0 < a.dm_steps ? (j + 1) * a.ndm0 : a.dm_steps;
  const int64_t nrows = mend_nom - m0 < kRows64 ? mend_nom - m0 : kRows64;
  if (nrows <= 0) return;
  unsigned long long acc[kRows64][kRun];
#pragma unroll
  for (int r = 0; r < kRows64; ++r)
#pragma unroll
    for (int k = 0; k < kRun; ++k) acc[r][k] = 0;
  const unsigned long long* inter =
      static_cast<const unsigned long long*>(a.inter) + j * a.nsb * a.tile_pitch;
  for (int64_t sb = 0; sb < a.nsb; ++sb) {
    const unsigned long long* row = inter + sb * a.tile_pitch;
#pragma unroll
    for (int r = 0; r < kRows64; ++r) {
      if (r < nrows) {
        const int64_t pos = t_local + __ldg(a.res + (m0 + r) * a.nsb + sb);
#pragma unroll
        for (int k = 0; k < kRun; ++k) acc[r][k] += __ldg(row + pos + k);
      }
    }
  }
  const int64_t valid = a.ncols - t_local;
  if (valid <= 0) return;
  for (int r = 0; r < nrows; ++r) {
    unsigned long long* dst =
        static_cast<unsigned long long*>(a.out) + (m0 + r) * a.out_pitch + a.col0 + t_local;
#pragma unroll
    for (int k = 0; k < kRun; ++k)
      if (k < valid) dst[k] = acc[r][k];
  }
}

// ---------------------------------------------------------------- brute force
// grid: x = time tile of the slice, y = block of kRows DMs.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_brute(BruteArgs a) {
  const int64_t t_local = static_cast<int64_t>(blockIdx.x) * kTile + threadIdx.x * kRun;
  const int64_t m0 = static_cast<int64_t>(blockIdx.y) * kRows;
  const int64_t nrows = a.dm_steps - m0 < kRows ? a.dm_steps - m0 : kRows;
  const T* x = static_cast<const T*>(a.x);
  uint32_t wide[kRows][8];
#pragma unroll
  for (int r = 0; r < kRows; ++r)
#pragma unroll
    for (int k = 0; k < 8; ++k) wide[r][k] = 0;
  uint32_t acc[kRows][4];
#pragma unroll
  for (int r = 0; r < kRows; ++r)
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[r][k] = 0;
  int since = 0;
  for (int64_t c = 0; c < a.nc; ++c) {
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      if (r < nrows) {
        // Input sample start + (t)*ds + delay lives in phase (start+delay) % ds
        // at index (start+delay)/ds + t of that phase row.
        const int64_t s = a.start + __ldg(a.delay + (m0 + r) * a.nc + c);
        const int64_t ph = s % a.ds;
        const T* row = x + (c * a.ds + ph) * a.phase_len;
        const int64_t pos = s / a.ds + t_local;
        if constexpr (sizeof(T) == 1) {
          add8_u8(row, pos, acc[r]);
        } else if constexpr (sizeof(T) == 2) {
          uint32_t v[4];
          load8_u16(row, pos, v);
#pragma unroll
          for (int k = 0; k < 4; ++k) { wide[r][2 * k] += v[k] & 0xffffu; wide[r][2 * k + 1] += v[k] >> 16; }
        }
      }
    }
    if constexpr (sizeof(T) == 1) {
      if (++since == 257) {
#pragma unroll
        for (int r = 0; r < kRows; ++r) widen_u8pairs(acc[r], wide[r]);
        since = 0;
      }
    }
  }
  if constexpr (sizeof(T) == 1) {
#pragma unroll
    for (int r = 0; r < kRows; ++r) widen_u8pairs(acc[r], wide[r]);
  }
  const int64_t valid = a.ncols - t_local;
  if (valid <= 0) return;
  for (int r = 0; r < nrows; ++r) {
    uint32_t v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = wide[r][k];
    store_run(static_cast<uint32_t*>(a.out) + (m0 + r) * a.out_pitch + a.col0 + t_local, valid, v);
  }
}

// 32-bit input samples accumulate into 64-bit sums (include/data.h:113-116).
__global__ void __launch_bounds__(kThreads) k_brute_u32(BruteArgs a) {
  const int64_t t_local = static_cast<int64_t>(blockIdx.x) * kTile + threadIdx.x * kRun;
  const int64_t m0 = static_cast<int64_t>(blockIdx.y) * kRows;
  const int64_t nrows = a.dm_steps - m0 < kRows ? a.dm_steps - m0 : kRows;
  const uint32_t* x = static_cast<const uint32_t*>(a.x);
  unsigned long long acc[kRows][8];
#pragma unroll
  for (int r = 0; r < kRows; ++r)
#pragma unroll
    for (int k = 0; k < 8; ++k) acc[r][k] = 0;
  for (int64_t c = 0; c < a.nc; ++c) {
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      if (r < nrows) {
        const int64_t s = a.start + __ldg(a.delay + (m0 + r) * a.nc + c);
        const uint32_t* row = x + (c * a.ds + s % a.ds) * a.phase_len;
        const int64_t pos = s / a.ds + t_local;
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[r][k] += __ldg(row + pos + k);
      }
    }
  }
  const int64_t valid = a.ncols - t_local;
  if (valid <= 0) return;
  for (int r = 0; r < nrows; ++r) {
    unsigned long long* dst = static_cast<unsigned long long*>(a.out) + (m0 + r) * a.out_pitch + a.col0 + t_local;
    for (int k = 0; k < 8; ++k)
      if (k < valid) dst[k] = acc[r][k];
  }
}

}  // namespace

void launch_stage1(const Stage1Args& a, cudaStream_t st) {
  dim3 grid(static_cast<unsigned>((a.ncols + kTile - 1) / kTile),
            static_cast<unsigned>((a.ndm_nom + kRows - 1) / kRows), static_cast<unsigned>(a.nsb));
  if (a.nbits == 8) {
    k_stage1_u8<<<grid, kThreads, 0, st>>>(a);
  } else if (a.nbits == 16) {
    k_stage1_wide<uint16_t><<<grid, kThreads, 0, st>>>(a);
  } else {
    grid.y = static_cast<unsigned>((a.ndm_nom + kRows64 - 1) / kRows64);
    k_stage1_u32<<<grid, kThreads, 0, st>>>(a);
  }
  DD_LAUNCHED();
}

void launch_stage2(const Stage2Args& a, cudaStream_t st) {
  const int64_t nnom = (a.dm_steps + a.ndm0 - 1) / a.ndm0;
  const int rows = a.out64 ? kRows64 : kRows;
  const int64_t per_nom = (a.ndm0 + rows - 1) / rows;
  dim3 grid(static_cast<unsigned>((a.ncols + kTile - 1) / kTile), static_cast<unsigned>(nnom * per_nom));
  if (a.out64) k_stage2_u64<<<grid, kThreads, 0, st>>>(a);
  else k_stage2<<<grid, kThreads, 0, st>>>(a);
  DD_LAUNCHED();
}

void launch_brute(const BruteArgs& a, cudaStream_t st) {
  dim3 grid(static_cast<unsigned>((a.ncols + kTile - 1) / kTile),
            static_cast<unsigned>((a.dm_steps + kRows - 1) / kRows));
  if (a.nbits == 8) k_brute<uint8_t><<<grid, kThreads, 0, st>>>(a);
  else if (a.nbits == 16) k_brute<uint16_t><<<grid, kThreads, 0, st>>>(a);
  else k_brute_u32<<<grid, kThreads, 0, st>>>(a);
  DD_LAUNCHED();
}

int tile_samples() { return kTile; }

}  // namespace dd
