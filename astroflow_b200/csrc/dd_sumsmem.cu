// Shared-memory staged shift-and-add kernels: the dedispersion sums of
// src/core/dedispered.cu:416-476 (subband stages 1 and 2) and
// include/cpucal.hpp:154-190 (brute force), all of the form
//
//   out[r][t] = sum_i src_i[base + off(r, i) + t],   t in [0, T) of the block's tile.
//
// A block owns RB output rows and T consecutive samples.  Sources are processed
// two at a time: the time window of each source that the block's rows need,
// [base + min_r off, base + max_r off + T), is copied once into shared memory with
// cp.async (16-byte chunks, double-buffered: the next pair streams in while the
// current pair is summed), and every row then reads its shifted samples from
// there.  Lanes own interleaved 32-bit output words (lane l: words l, l+32, ...),
// so each shared load touches 32 consecutive words, free of bank conflicts; a shift
// that is not a multiple of 4 bytes costs one funnel shift of two words.
//
// 8-bit samples: each word is split into two 16-bit-lane words by byte permutes
// and two sources are added by one three-input add, i.e. four sample additions
// per add instruction; lanes are widened to 32 bits every 256 sources.  16-bit
// samples are added as lane pairs and widened before they can overflow.
#include <cuda_runtime.h>

#include <cstdint>

#include "dd_internal.h"

namespace dd {
namespace {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Per-block view of the sum.
struct Geo {
  const char* src;     // source 0 (byte address)
  int64_t src_pitch;   // bytes between consecutive sources
  const int32_t* off;  // off[r * off_pitch + i]
  int64_t off_pitch;
  int64_t base;        // element index added to every offset
  int nsrc, nrows;
  char* out;           // row 0, first column of the block (byte address)
  int64_t out_pitch;   // bytes between output rows
  int64_t valid;       // columns of this block to store (<= T)
};

__device__ __forceinline__ Geo make_geo(const SumLaunch& L, int T) {
  Geo g;
  const int64_t tile = blockIdx.x;
  const int64_t col = tile * T;  // launch-local column of the block
  g.valid = L.ncols - col;
  switch (L.mode) {
    case SumLaunch::kStage1: {
      // rows: nominal DMs j0.. of subband sb; sources: the subband's channels
      const int64_t j0 = static_cast<int64_t>(blockIdx.y) * L.rows_per_block;
      const int64_t sb = blockIdx.z;
      const int64_t c0 = sb * L.group;
      g.src = L.src + c0 * L.src_pitch;
      g.src_pitch = L.src_pitch;
      g.off = L.off + j0 * L.off_pitch + c0;
      g.off_pitch = L.off_pitch;
      g.nsrc = static_cast<int>(min(static_cast<int64_t>(L.group), L.nsrc_total - c0));
      g.nrows = static_cast<int>(min(static_cast<int64_t>(L.rows_per_block), L.nrows_total - j0));
      g.out = L.out + (j0 * L.nsb_out + sb) * L.out_pitch + (L.out_col0 + col) * L.out_elem;
      g.out_pitch = L.nsb_out * L.out_pitch;
      break;
    }
    case SumLaunch::kStage2: {
      // rows: fine DMs of nominal DM j; sources: the subband sums of j
      const int per_nom = (L.group + L.rows_per_block - 1) / L.rows_per_block;
      const int64_t j = blockIdx.y / per_nom;
      const int64_t m0 = j * L.group + static_cast<int64_t>(blockIdx.y % per_nom) * L.rows_per_block;
      const int64_t mend = min((j + 1) * L.group, L.nrows_total);
      g.src = L.src + j * L.nsrc_total * L.src_pitch;
      g.src_pitch = L.src_pitch;
      g.off = L.off + m0 * L.off_pitch;
      g.off_pitch = L.off_pitch;
      g.nsrc = static_cast<int>(L.nsrc_total);
      g.nrows = static_cast<int>(max(static_cast<int64_t>(0), min(static_cast<int64_t>(L.rows_per_block), mend - m0)));
      g.out = L.out + m0 * L.out_pitch + (L.out_col0 + col) * L.out_elem;
      g.out_pitch = L.out_pitch;
      break;
    }
    default: {  // brute force: rows = DMs, sources = channels
      const int64_t m0 = static_cast<int64_t>(blockIdx.y) * L.rows_per_block;
      g.src = L.src;
      g.src_pitch = L.src_pitch;
      g.off = L.off + m0 * L.off_pitch;
      g.off_pitch = L.off_pitch;
      g.nsrc = static_cast<int>(L.nsrc_total);
      g.nrows = static_cast<int>(min(static_cast<int64_t>(L.rows_per_block), L.nrows_total - m0));
      g.out = L.out + m0 * L.out_pitch + (L.out_col0 + col) * L.out_elem;
      g.out_pitch = L.out_pitch;
      break;
    }
  }
  g.base = L.base + col;
  return g;
}

// Stage the windows of sources i, i+1 into words [wbase_s, wbase_s + win_words) of
// the shared array (one window per source), and publish, for every row, the
// word index and byte shift of its sample 0 inside the window.
template <int SB, int RB>
__device__ __forceinline__ void stage_pair(const Geo& g, int i, uint32_t* sw, int win_words,
                                           int tile_bytes, int* rowq, int* rowsh) {
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const int src = i + s;
    if (src >= g.nsrc) {
      if (threadIdx.x < RB) { rowq[s * RB + threadIdx.x] = 0; rowsh[s * RB + threadIdx.x] = 0; }
      continue;
    }
    int lo = 0x7fffffff, hi = -0x7fffffff;
#pragma unroll
    for (int r = 0; r < RB; ++r) {
      if (r < g.nrows) {
        const int o = __ldg(g.off + r * g.off_pitch + src);
        lo = min(lo, o);
        hi = max(hi, o);
      }
    }
    const int64_t first = (g.base + lo) * SB;
    const int64_t a0 = first & ~int64_t(15);
    const int64_t last = (g.base + hi) * SB + tile_bytes + 8;  // + the funnel's second word
    const int nbytes = static_cast<int>((last - a0 + 15) & ~int64_t(15));
    const char* gsrc = g.src + static_cast<int64_t>(src) * g.src_pitch + a0;
    uint32_t* dst = sw + s * win_words;
    for (int b = threadIdx.x * 16; b < nbytes; b += kThreads * 16)
      cp_async16(reinterpret_cast<char*>(dst) + b, gsrc + b);
    if (threadIdx.x < RB) {
      // Rows past nrows are summed too (their results are never stored); they
      // take the window's first offset so their reads stay inside the window.
      const int r = threadIdx.x;
      const int o = r < g.nrows ? __ldg(g.off + r * g.off_pitch + src) : lo;
      const int ob = static_cast<int>(first - a0) + (o - lo) * SB;  // byte offset of sample 0
      rowq[s * RB + r] = s * win_words + (ob >> 2);
      rowsh[s * RB + r] = (ob & 3) * 8;
    }
  }
}

// ------------------------------------------------------------------ 8-bit samples
template <int RB, int NW, bool OUT16, bool FLUSH>
__global__ void __launch_bounds__(kThreads) k_sum_u8(SumLaunch L) {
  extern __shared__ __align__(16) uint32_t sw[];
  __shared__ int rowq[2][2 * RB], rowsh[2][2 * RB];
  constexpr int T = kWarps * 32 * NW * 4;
  const Geo g = make_geo(L, T);
  if (g.nrows <= 0) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wbase = warp * 32 * NW + lane;
  uint32_t ev[RB][NW], od[RB][NW];  // 16-bit lanes: samples (4w, 4w+2) and (4w+1, 4w+3)
  uint32_t w32[FLUSH ? RB : 1][FLUSH ? NW * 4 : 1];
#pragma unroll
  for (int r = 0; r < RB; ++r)
#pragma unroll
    for (int k = 0; k < NW; ++k) ev[r][k] = od[r][k] = 0;
  if constexpr (FLUSH) {
#pragma unroll
    for (int r = 0; r < RB; ++r)
#pragma unroll
      for (int k = 0; k < NW * 4; ++k) w32[r][k] = 0;
  }
  const int ww = L.win_bytes >> 2;  // words per window
  const int npairs = (g.nsrc + 1) / 2;
  int since = 0;
  stage_pair<1, RB>(g, 0, sw, ww, T, rowq[0], rowsh[0]);
  cp_async_commit();
  for (int p = 0; p < npairs; ++p) {
    const int cur = p & 1;
    if (p + 1 < npairs)
      stage_pair<1, RB>(g, 2 * (p + 1), sw + (cur ^ 1) * 2 * ww, ww, T, rowq[cur ^ 1], rowsh[cur ^ 1]);
    cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    const uint32_t* win = sw + cur * 2 * ww;
    const bool two = 2 * p + 1 < g.nsrc;
#pragma unroll
    for (int r = 0; r < RB; ++r) {
      const int q0 = rowq[cur][r] + wbase, q1 = rowq[cur][RB + r] + wbase;
      const uint32_t s0 = rowsh[cur][r], s1 = rowsh[cur][RB + r];
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        const uint32_t a = __funnelshift_r(win[q0 + 32 * k], win[q0 + 32 * k + 1], s0);
        uint32_t b = __funnelshift_r(win[q1 + 32 * k], win[q1 + 32 * k + 1], s1);
        b = two ? b : 0u;
        ev[r][k] += __byte_perm(a, 0u, 0x4240) + __byte_perm(b, 0u, 0x4240);
        od[r][k] += __byte_perm(a, 0u, 0x4341) + __byte_perm(b, 0u, 0x4341);
      }
    }
    if constexpr (FLUSH) {
      since += 2;
      if (since >= 256) {  // 256 x 255 fits a 16-bit lane
#pragma unroll
        for (int r = 0; r < RB; ++r)
#pragma unroll
          for (int k = 0; k < NW; ++k) {
            w32[r][4 * k + 0] += ev[r][k] & 0xffffu; w32[r][4 * k + 2] += ev[r][k] >> 16;
            w32[r][4 * k + 1] += od[r][k] & 0xffffu; w32[r][4 * k + 3] += od[r][k] >> 16;
            ev[r][k] = od[r][k] = 0;
          }
        since = 0;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < RB; ++r) {
    if (r >= g.nrows) break;
#pragma unroll
    for (int k = 0; k < NW; ++k) {
      const int64_t t = static_cast<int64_t>(wbase + 32 * k) * 4;  // block-local sample
      if (t >= g.valid) continue;
      uint32_t s0, s1, s2, s3;
      if constexpr (FLUSH) {
        s0 = w32[r][4 * k + 0] + (ev[r][k] & 0xffffu);
        s1 = w32[r][4 * k + 1] + (od[r][k] & 0xffffu);
        s2 = w32[r][4 * k + 2] + (ev[r][k] >> 16);
        s3 = w32[r][4 * k + 3] + (od[r][k] >> 16);
      } else {
        s0 = ev[r][k] & 0xffffu; s1 = od[r][k] & 0xffffu;
        s2 = ev[r][k] >> 16;     s3 = od[r][k] >> 16;
      }
      char* row = g.out + r * g.out_pitch;
      if constexpr (OUT16) {
        uint16_t* dst = reinterpret_cast<uint16_t*>(row) + t;
        if (t + 4 <= g.valid && (reinterpret_cast<uintptr_t>(dst) & 7) == 0) {
          *reinterpret_cast<uint2*>(dst) = make_uint2(__byte_perm(ev[r][k], od[r][k], 0x5410),
                                                      __byte_perm(ev[r][k], od[r][k], 0x7632));
        } else {
          const uint32_t v[4] = {s0, s1, s2, s3};
          for (int q = 0; q < 4 && t + q < g.valid; ++q) dst[q] = static_cast<uint16_t>(v[q]);
        }
      } else {
        uint32_t* dst = reinterpret_cast<uint32_t*>(row) + t;
        if (t + 4 <= g.valid && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
          *reinterpret_cast<uint4*>(dst) = make_uint4(s0, s1, s2, s3);
        } else {
          const uint32_t v[4] = {s0, s1, s2, s3};
          for (int q = 0; q < 4 && t + q < g.valid; ++q) dst[q] = v[q];
        }
      }
    }
  }
}

// ------------------------------------------------------------------ 16-bit samples
// L.lane_per: sources summed in 16-bit lanes before widening (< 2: 32-bit sums).
template <int RB, int NW>
__global__ void __launch_bounds__(kThreads) k_sum_u16(SumLaunch L) {
  extern __shared__ __align__(16) uint32_t sw[];
  __shared__ int rowq[2][2 * RB], rowsh[2][2 * RB];
  constexpr int T = kWarps * 32 * NW * 2;
  const Geo g = make_geo(L, T);
  if (g.nrows <= 0) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wbase = warp * 32 * NW + lane;
  uint32_t a16[RB][NW], lo32[RB][NW], hi32[RB][NW];
#pragma unroll
  for (int r = 0; r < RB; ++r)
#pragma unroll
    for (int k = 0; k < NW; ++k) a16[r][k] = lo32[r][k] = hi32[r][k] = 0;
  const int ww = L.win_bytes >> 2;
  const int npairs = (g.nsrc + 1) / 2;
  const int per = L.lane_per;
  int since = 0;
  stage_pair<2, RB>(g, 0, sw, ww, 2 * T, rowq[0], rowsh[0]);
  cp_async_commit();
  for (int p = 0; p < npairs; ++p) {
    const int cur = p & 1;
    if (p + 1 < npairs)
      stage_pair<2, RB>(g, 2 * (p + 1), sw + (cur ^ 1) * 2 * ww, ww, 2 * T, rowq[cur ^ 1], rowsh[cur ^ 1]);
    cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    const uint32_t* win = sw + cur * 2 * ww;
    const bool two = 2 * p + 1 < g.nsrc;
    if (per >= 2) {
#pragma unroll
      for (int r = 0; r < RB; ++r) {
        const int q0 = rowq[cur][r] + wbase, q1 = rowq[cur][RB + r] + wbase;
        const uint32_t s0 = rowsh[cur][r], s1 = rowsh[cur][RB + r];
#pragma unroll
        for (int k = 0; k < NW; ++k) {
          const uint32_t a = __funnelshift_r(win[q0 + 32 * k], win[q0 + 32 * k + 1], s0);
          const uint32_t b = __funnelshift_r(win[q1 + 32 * k], win[q1 + 32 * k + 1], s1);
          a16[r][k] += a + (two ? b : 0u);
        }
      }
      since += 2;
      if (since + 2 > per || p + 1 == npairs) {
#pragma unroll
        for (int r = 0; r < RB; ++r)
#pragma unroll
          for (int k = 0; k < NW; ++k) {
            lo32[r][k] += a16[r][k] & 0xffffu;
            hi32[r][k] += a16[r][k] >> 16;
            a16[r][k] = 0;
          }
        since = 0;
      }
    } else {
#pragma unroll
      for (int r = 0; r < RB; ++r) {
        const int q0 = rowq[cur][r] + wbase, q1 = rowq[cur][RB + r] + wbase;
        const uint32_t s0 = rowsh[cur][r], s1 = rowsh[cur][RB + r];
#pragma unroll
        for (int k = 0; k < NW; ++k) {
          const uint32_t a = __funnelshift_r(win[q0 + 32 * k], win[q0 + 32 * k + 1], s0);
          uint32_t b = __funnelshift_r(win[q1 + 32 * k], win[q1 + 32 * k + 1], s1);
          b = two ? b : 0u;
          lo32[r][k] += (a & 0xffffu) + (b & 0xffffu);
          hi32[r][k] += (a >> 16) + (b >> 16);
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < RB; ++r) {
    if (r >= g.nrows) break;
#pragma unroll
    for (int k = 0; k < NW; ++k) {
      const int64_t t = static_cast<int64_t>(wbase + 32 * k) * 2;
      if (t >= g.valid) continue;
      uint32_t* dst = reinterpret_cast<uint32_t*>(g.out + r * g.out_pitch) + t;
      if (t + 2 <= g.valid && (reinterpret_cast<uintptr_t>(dst) & 7) == 0) {
        *reinterpret_cast<uint2*>(dst) = make_uint2(lo32[r][k], hi32[r][k]);
      } else {
        dst[0] = lo32[r][k];
        if (t + 1 < g.valid) dst[1] = hi32[r][k];
      }
    }
  }
}

template <typename K>
void launch_k(K kernel, dim3 grid, size_t smem, const SumLaunch& L, cudaStream_t st) {
  if (smem > 48 * 1024)
    DD_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(smem)));
  kernel<<<grid, kThreads, smem, st>>>(L);
  DD_LAUNCHED();
}

}  // namespace

int sum_tile_samples(int src_bytes, int nw) { return kWarps * 32 * nw * (4 / src_bytes); }

size_t sum_smem_bytes(int win_bytes) { return static_cast<size_t>(4) * win_bytes; }

void launch_sum(const SumLaunch& L, cudaStream_t st) {
  const int T = sum_variant_tile(L.src_bytes, L.flush && L.out_elem != 2);
  dim3 grid(static_cast<unsigned>((L.ncols + T - 1) / T), L.grid_y, L.grid_z);
  const size_t smem = sum_smem_bytes(L.win_bytes);
  if (L.rows_per_block != kSumRows) throw Error{DD_ERR_RUNTIME, "unsupported rows per block"};
  if (L.src_bytes == 1) {
    if (L.out_elem == 2) {
      launch_k(k_sum_u8<kSumRows, 4, true, false>, grid, smem, L, st);
    } else if (L.flush) {
      launch_k(k_sum_u8<kSumRows, 2, false, true>, grid, smem, L, st);
    } else {
      launch_k(k_sum_u8<kSumRows, 4, false, false>, grid, smem, L, st);
    }
  } else {
    launch_k(k_sum_u16<kSumRows, 2>, grid, smem, L, st);
  }
}

}  // namespace dd
