// Shared-memory staged shift-and-add kernels: the dedispersion sums of
// src/core/dedispered.cu:416-476 (subband stages 1 and 2) and
// include/cpucal.hpp:154-190 (brute force), all of the form
//
//   out[r][t] = sum_i src_i[base + off(r, i) + t],   t in [0, T) of the block's tile.
//
// A block owns RB output rows and T consecutive samples.  Sources are processed
// two at a time.  The time window of each source that the block's rows need,
// [base + min_r off, base + max_r off + T), is brought into shared memory by one
// bulk asynchronous copy (cp.async.bulk, completion counted in bytes on an
// mbarrier); up to `stages` source pairs are in flight in a ring of buffers.
// Warp 0 acts as the producer: before summing pair p it refills the buffer pair
// p-1 used with pair p+stages-1, once every warp has released it (an "empty"
// mbarrier with one arrival per warp).  The window bounds and each row's offset
// inside its window come from descriptors precomputed on the host (SumDesc),
// which reach shared memory by bulk copies of 32 sources, a chunk ahead, so the
// producer only unpacks them (one lane per source and row).
//
// Summing: lanes own 32-bit output words (an odd number of consecutive words, or
// interleaved words l, l+32, ...), so a warp's shared loads are free of bank
// conflicts; a shift that is not a multiple of 4 bytes costs one funnel shift of
// two words.  8-bit samples are split into two 16-bit-lane words by byte
// permutes; 16-bit stage-1 sums come with a twin shifted by one sample so that
// stage 2 reads aligned words only (sum_u16_twin), four sources at a time in
// packed 16-bit lanes; 16-bit samples are aligned pairwise and summed whole
// beside their high halves (sum_u16_wide).  Outputs leave through shared memory
// as 16-byte chunks where a lane's words are scattered (16-bit stage-1 sums and
// their twin; the 32-bit flushes of 8-bit sums of more than 256 sources, which
// read back the block's own partial sums).  A missing source (source count not
// a multiple of the group) reads a zeroed window.
//
// Every wait on an mbarrier is bounded (about two seconds of SM clock); a wait
// that gives up records an error code in L.err and the block stops summing, and
// the other blocks of the launch stop at their next wait.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <vector>

#include "dd_internal.h"

namespace dd {
namespace {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
#ifndef DD_SUM_MAX_STAGES
#define DD_SUM_MAX_STAGES 8
#endif
constexpr int kMaxStages = DD_SUM_MAX_STAGES;  // staged source pairs in flight, at most
constexpr long long kWaitCycles = 4000000000LL;

// ------------------------------------------------------------------ mbarrier helpers
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the phase with the given parity to complete; false after ~2 s, or
// as soon as this block (*failed) or any block of the launch (*gerr) has failed.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* failed,
                                          volatile int* gerr) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  for (uint32_t i = 1;; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 255u) == 0) {  // the failure checks read memory: keep them off the wake-up path
      if (*failed || *gerr) return false;
      if (clock64() - t0 > kWaitCycles) return false;
    }
  }
}
// One bulk copy global -> shared, completing `bytes` on `bar`.
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

#ifndef DD_SUM_IMAD
#define DD_SUM_IMAD 1
#endif
// 8-bit sums without periodic widening accumulate with integer multiply-adds
// (by a runtime 1) on the FMA pipe instead of adds on the integer pipe, which
// the shifts and byte permutes keep busy (stage 1: 78.0 -> 74.8 ms at the
// headline size; the widening variant is faster with plain adds).
constexpr bool kSumImad = DD_SUM_IMAD != 0;
// High word of a*b plus c on the FMA pipe (b a runtime value, e.g. 2^k built
// from L.one, so the compiler cannot turn it into a shift on the integer pipe).
__device__ __forceinline__ uint32_t madhi_u32(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t d;
  asm("mad.hi.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}
// How 8-bit samples are split into 16-bit lanes (DD_SUM8_SPLIT):
//  0: two byte permutes per word (integer pipe), lanes added by multiply-adds;
//  1: even lanes = word & 0x00ff00ff (integer pipe), odd lanes accumulated as the
//     high word of (word - even) * 2^24 (FMA pipe), even lanes added by
//     multiply-adds: one integer-pipe operation per word fewer than 0;
//  2: as 1, with two sources' even lanes added by one three-input add.
//  3: even lanes by mask (as 1), whole words summed as they are, top bytes summed
//     by a multiply-high; the odd lanes are recovered once per output word.
// Measured at the headline size (stage 1, ms): 0 -> 76.5, 1 -> 107, 2 -> 92; the
// multiply-high chains cost more than the integer-pipe operations they save.
// 16-bit stage-1 sums leave through shared memory as 16-byte chunks (1) or as
// each lane's words (0).
#ifndef DD_SUM8_STAGED_OUT
#define DD_SUM8_STAGED_OUT 1
#endif
// The 32-bit flushes of 8-bit sums go through shared memory as 16-byte chunks
// (1) or as each lane's words (0); the staging takes flush_smem_bytes() past the ring.
#ifndef DD_SUM8_STAGED_FLUSH
#define DD_SUM8_STAGED_FLUSH 1
#endif
#ifndef DD_SUM16Q_MINB
#define DD_SUM16Q_MINB 2
#endif
#ifndef DD_SUM8_SPLIT
#define DD_SUM8_SPLIT 0
#endif
__device__ __forceinline__ uint32_t mad_u32(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t d;
  asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}

// Per-block view of the sum.
struct Geo {
  const char* src;     // source 0 (byte address)
  int64_t src_pitch;   // bytes between consecutive sources
  const SumDesc* desc; // descriptor of source 0 for this block's row group
  int64_t base;        // element index added to every offset
  int nsrc, nrows;
  char* out;           // row 0, first column of the block (byte address)
  int64_t out_pitch;   // bytes between output rows
  int64_t valid;       // columns of this block to store (<= T)
};

__device__ __forceinline__ Geo make_geo(const SumLaunch& L, int T, uint3 blk) {
  Geo g;
  const int64_t tile = blk.x;
  const int64_t col = tile * T;  // launch-local column of the block
  g.valid = L.ncols - col;
  const SumDesc* drow = L.desc + static_cast<int64_t>(blk.y) * L.desc_pitch;
  switch (L.mode) {
    case SumLaunch::kStage1: {
      // rows: nominal DMs j0.. of subband sb; sources: the subband's channels
      const int64_t j0 = static_cast<int64_t>(blk.y) * L.rows_per_block;
      const int64_t sb = blk.z;
      const int64_t c0 = sb * L.group;
      g.src = L.src + c0 * L.src_pitch;
      g.desc = drow + c0;
      g.nsrc = static_cast<int>(min(static_cast<int64_t>(L.group), L.nsrc_total - c0));
      g.nrows = static_cast<int>(min(static_cast<int64_t>(L.rows_per_block), L.nrows_total - j0));
      g.out = L.out + (j0 * L.nsb_out + sb) * L.out_pitch + (L.out_col0 + col) * L.out_elem;
      g.out_pitch = L.nsb_out * L.out_pitch;
      break;
    }
    case SumLaunch::kStage2: {
      // rows: fine DMs of nominal DM j; sources: the subband sums of j
      const int per_nom = (L.group + L.rows_per_block - 1) / L.rows_per_block;
      const int64_t j = blk.y / per_nom;
      const int64_t m0 = j * L.group + static_cast<int64_t>(blk.y % per_nom) * L.rows_per_block;
      const int64_t mend = min((j + 1) * L.group, L.nrows_total);
      g.src = L.src + j * L.nsrc_total * L.src_pitch;
      g.desc = drow;
      g.nsrc = static_cast<int>(L.nsrc_total);
      g.nrows = static_cast<int>(max(static_cast<int64_t>(0), min(static_cast<int64_t>(L.rows_per_block), mend - m0)));
      g.out = L.out + m0 * L.out_pitch + (L.out_col0 + col) * L.out_elem;
      g.out_pitch = L.out_pitch;
      break;
    }
    default: {  // brute force: rows = DMs, sources = channels
      const int64_t m0 = static_cast<int64_t>(blk.y) * L.rows_per_block;
      g.src = L.src;
      g.desc = drow;
      g.nsrc = static_cast<int>(L.nsrc_total);
      g.nrows = static_cast<int>(min(static_cast<int64_t>(L.rows_per_block), L.nrows_total - m0));
      g.out = L.out + m0 * L.out_pitch + (L.out_col0 + col) * L.out_elem;
      g.out_pitch = L.out_pitch;
      break;
    }
  }
  g.src_pitch = L.src_pitch;
  g.base = L.base + col;
  return g;
}

// Source descriptors come into shared memory in chunks of kDescChunk sources by
// bulk copies, two chunks in flight, so that the producer never waits on a
// global load between two stages.
constexpr int kDescChunk = 32;

// Shared state of the pipeline.  A stage holds QS (2 or 4) source windows.
struct __align__(16) Pipe {
  uint64_t full[kMaxStages];   // completes when a stage's windows have landed
  uint64_t empty[kMaxStages];  // completes when all warps released a stage
  SumDesc desc[2][kDescChunk]; // descriptors of chunks k (half k & 1)
  uint64_t dfull[2];           // completes when a half's chunk has landed
  // per row: word index and shift (bits) of sample 0 in the window of source
  // i of the stage at [2i], [2i+1]
  int row[kMaxStages][kSumRows][8];
  int failed;
};
static_assert(offsetof(Pipe, desc) % 16 == 0, "bulk copies land on 16-byte boundaries");

// Bulk copy of descriptor chunk k of the block's sources into half k & 1.
__device__ __forceinline__ void fetch_desc(const Geo& g, Pipe& P, int k) {
  const int n = min(kDescChunk, g.nsrc - k * kDescChunk);
  const uint32_t bytes = static_cast<uint32_t>(n * sizeof(SumDesc));
  mbar_arrive_expect_tx(&P.dfull[k & 1], bytes);
  bulk_copy(&P.desc[k & 1][0], g.desc + static_cast<int64_t>(k) * kDescChunk, bytes,
            &P.dfull[k & 1]);
}
__device__ __forceinline__ int4 row_pair(const Pipe& P, int s, int r, int half) {
  return *reinterpret_cast<const int4*>(&P.row[s][r][4 * half]);
}

// Producer step for source group q in stage s, by all lanes of warp 0: lane
// 8i + r writes row r's offsets into the window of source QS*q + i, and lane 8i
// issues that window's copy.  The caller has made sure stage s is free.  False
// when the wait for the group's descriptors gave up.
template <int SB, int QS>
__device__ __forceinline__ bool produce(const Geo& g, Pipe& P, uint32_t* sw, int ww, int zero_q,
                                        int tile_bytes, int q, int s, int lane,
                                        volatile int* failed, volatile int* gerr) {
  static_assert(kSumRows == 8 && kDescChunk % QS == 0, "lane = 8 * source + row");
  const int first = QS * q;
  const int chunk = first / kDescChunk;
  if (first % kDescChunk == 0) {
    // the group opens a chunk: wait for its descriptors, then refill the other
    // half (the previous chunk, read by this warp only) with the next chunk
    const bool ok = __all_sync(0xffffffffu, mbar_wait(&P.dfull[chunk & 1], (chunk >> 1) & 1,
                                                      failed, gerr));
    if (!ok) return false;
    if (lane == 0 && chunk >= 1 && (chunk + 1) * kDescChunk < g.nsrc) {
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      fetch_desc(g, P, chunk + 1);
    }
  }
  const int i = lane >> 3, r = lane & 7;
  const int src = first + i;
  uint32_t nbytes = 0;
  const char* gsrc = nullptr;
  if (i < QS) {
    int* rw = &P.row[s][r][2 * i];
    if (src < g.nsrc) {
      const SumDesc& d = P.desc[chunk & 1][src % kDescChunk];
      const int64_t firstb = (g.base + d.lo) * SB;
      const int64_t a0 = firstb & ~int64_t(15);
      // rows past nrows take offset lo (rel 0): their reads stay in the window
      const int ob = static_cast<int>(firstb - a0) + (r < g.nrows ? static_cast<int>(d.rel[r]) : 0) * SB;
      rw[0] = (QS * s + i) * ww + (ob >> 2);
      rw[1] = (ob & 3) * 8;
      if (r == 0) {
        const int64_t last = (g.base + d.lo + d.span) * SB + tile_bytes + 8;  // + funnel word
        nbytes = static_cast<uint32_t>((last - a0 + 15) & ~int64_t(15));
        gsrc = g.src + static_cast<int64_t>(src) * g.src_pitch + a0;
      }
    } else {
      rw[0] = zero_q;
      rw[1] = 0;
    }
  }
  uint32_t total = nbytes + __shfl_xor_sync(0xffffffffu, nbytes, 8);
  if (QS == 4) total += __shfl_xor_sync(0xffffffffu, total, 16);
  __syncwarp();
  if (lane == 0) mbar_arrive_expect_tx(&P.full[s], total);
  __syncwarp();
  if (nbytes) bulk_copy(sw + (QS * s + i) * ww, gsrc, nbytes, &P.full[s]);
  return true;
}

// Producer step of the twin-window sums (16-bit sources with a one-sample-shifted
// twin, twin[i] = sums[i - 1], four sources per stage): each source is staged
// twice, the sums and the twin, each from the 16-byte boundary at or below the
// first element the block's rows read there, and lane 8i + r points row r of
// source 4q + i into the copy in which its first element starts a 32-bit word:
// an even element index e at byte 2e of the sums, an odd one at byte 2(e + 1)
// of the twin.  Lane 8i issues both copies.
__device__ __forceinline__ bool produce_twin(const Geo& g, Pipe& P, uint32_t* sw, int ww, int zero_q,
                                             int tile_bytes, int64_t twin_off, int q, int s,
                                             int lane, volatile int* failed, volatile int* gerr) {
  constexpr int QS = 4;
  static_assert(kSumRows == 8 && kDescChunk % QS == 0, "lane = 8 * source + row");
  const int first = QS * q;
  const int chunk = first / kDescChunk;
  if (first % kDescChunk == 0) {
    const bool ok = __all_sync(0xffffffffu, mbar_wait(&P.dfull[chunk & 1], (chunk >> 1) & 1,
                                                      failed, gerr));
    if (!ok) return false;
    if (lane == 0 && chunk >= 1 && (chunk + 1) * kDescChunk < g.nsrc) {
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      fetch_desc(g, P, chunk + 1);
    }
  }
  const int i = lane >> 3, r = lane & 7;
  const int src = first + i;
  const int win0 = 2 * (QS * s + i) * ww;  // the sums; the twin follows at win0 + ww
  uint32_t n0 = 0, n1 = 0;
  const char *c0 = nullptr, *c1 = nullptr;
  int* rw = &P.row[s][r][2 * i];
  if (src < g.nsrc) {
    const SumDesc& d = P.desc[chunk & 1][src % kDescChunk];
    const int64_t e0 = g.base + d.lo;  // first element any row of the block reads
    // element e sits at byte 2e of the sums and at byte 2(e + 1) of the twin
    const int64_t a0 = (2 * e0) & ~int64_t(15);
    const int64_t a1 = (2 * (e0 + 1)) & ~int64_t(15);
    // rows past nrows take offset lo (rel 0): their reads stay in the windows
    const int64_t o = e0 + (r < g.nrows ? static_cast<int64_t>(d.rel[r]) : 0);
    rw[0] = (o & 1) ? win0 + ww + static_cast<int>((2 * (o + 1) - a1) >> 2)
                    : win0 + static_cast<int>((2 * o - a0) >> 2);
    rw[1] = 0;
    if (r == 0) {
      const int64_t last = 2 * (e0 + d.span) + tile_bytes;  // past the last byte any row reads
      n0 = static_cast<uint32_t>((last - a0 + 15) & ~int64_t(15));
      n1 = static_cast<uint32_t>((last + 2 - a1 + 15) & ~int64_t(15));
      c0 = g.src + static_cast<int64_t>(src) * g.src_pitch + a0;
      c1 = g.src + static_cast<int64_t>(src) * g.src_pitch + twin_off + a1;
    }
  } else {
    rw[0] = zero_q;
    rw[1] = 0;
  }
  uint32_t total = n0 + n1;
  total += __shfl_xor_sync(0xffffffffu, total, 8);
  total += __shfl_xor_sync(0xffffffffu, total, 16);
  __syncwarp();
  if (lane == 0) mbar_arrive_expect_tx(&P.full[s], total);
  __syncwarp();
  if (n0) {
    bulk_copy(sw + win0, c0, n0, &P.full[s]);
    bulk_copy(sw + win0 + ww, c1, n1, &P.full[s]);
  }
  return true;
}

// Pipeline driver shared by the kernels: calls body(stage, cur) for every
// group of QS sources once their windows are in shared memory (TWIN: each
// source is staged with its shifted twin, see produce_twin; QS is 4).
// Window modes of the pipeline: one window per source, or a source and its twin
// (four sources per stage).
constexpr int kModePlain = 0, kModeTwin = 1;
template <int SB, int QS = 2, int MODE = kModePlain, typename Body>
__device__ __forceinline__ void run_pipeline(const SumLaunch& L, const Geo& g, Pipe& P,
                                             uint32_t* sw, int tile_bytes, Body&& body) {
  static_assert(MODE != kModeTwin || QS == 4, "twin windows come four sources per stage");
  constexpr int kWinPerSrc = MODE == kModeTwin ? 2 : 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ww = L.win_bytes >> 2;
  const int S = L.stages;
  const int zero_q = kWinPerSrc * QS * S * ww;
  const int npairs = (g.nsrc + QS - 1) / QS;
  const int nchunks = (g.nsrc + kDescChunk - 1) / kDescChunk;
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&P.full[s], 1);
      mbar_init(&P.empty[s], kWarps);
    }
    mbar_init(&P.dfull[0], 1);
    mbar_init(&P.dfull[1], 1);
    P.failed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    // order earlier generic accesses to the windows (a previous task of a
    // persistent block) before the bulk copies that refill them
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    fetch_desc(g, P, 0);
    if (nchunks > 1) fetch_desc(g, P, 1);
  }
  for (int i = threadIdx.x; i < ww; i += kThreads) sw[zero_q + i] = 0u;
  __syncthreads();
  volatile int* failed = &P.failed;
  int issued = 0;  // pairs whose copies warp 0 has issued
  bool prod_ok = true;
  auto produce_group = [&](int q, int s) -> bool {
    if constexpr (MODE == kModeTwin)
      return produce_twin(g, P, sw, ww, zero_q, tile_bytes, L.twin_off, q, s, lane, failed, L.err);
    else
      return produce<SB, QS>(g, P, sw, ww, zero_q, tile_bytes, q, s, lane, failed, L.err);
  };
  if (warp == 0)
    for (; issued < min(S - 1, npairs); ++issued)
      if (!(prod_ok = produce_group(issued, issued))) break;
  if (!prod_ok && lane == 0) {
    if (!*failed) atomicCAS(L.err, 0, kErrWaitFull);
    *failed = 1;
  }
  int s_cur = 0, p = 0;
  uint32_t ph_cur = 0;
  for (; prod_ok && p < npairs; ++p) {
    if (warp == 0 && issued < npairs) {
      const int q = issued;  // == p + S - 1: refills the stage pair p-1 used
      const int s = q % S;
      bool ok = true;
      int code = kErrWaitEmpty;
      if (q >= S) {
        if (lane == 0) ok = mbar_wait(&P.empty[s], ((q / S) - 1) & 1, failed, L.err);
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      }
      if (ok) {
        ok = produce_group(q, s);
        code = kErrWaitFull;
      }
      if (!ok) {
        if (lane == 0) {
          if (!*failed) atomicCAS(L.err, 0, code);
          *failed = 1;
        }
        break;
      }
      ++issued;
    }
    const bool ok = mbar_wait(&P.full[s_cur], ph_cur, failed, L.err);
    if (!ok) {
      if (lane == 0) {
        if (!*failed) atomicCAS(L.err, 0, kErrWaitFull);
        *failed = 1;
      }
      break;
    }
    body(s_cur, sw);
    __syncwarp();
    if (lane == 0) mbar_arrive(&P.empty[s_cur]);
    if (++s_cur == S) {
      s_cur = 0;
      ph_cur ^= 1u;
    }
  }
  if (warp == 0 && lane == 0 && *failed) {
    // let the copies already issued land before the block's shared memory goes away
    for (int q = p; q < issued; ++q) {
      const long long t0 = clock64();
      while (!mbar_try_wait(&P.full[q % S], (q / S) & 1) && clock64() - t0 < kWaitCycles) {
      }
    }
    // descriptor chunks: 0 and 1 at the start, k + 1 once chunk k >= 1 was
    // waited for; the chunks up to that of the last issued group were waited for
    const int opened = issued > 0 ? (QS * (issued - 1)) / kDescChunk : -1;
    const int last = min(nchunks - 1, max(1, opened + 1));
    for (int k = opened + 1; k <= last; ++k) {
      const long long t0 = clock64();
      while (!mbar_try_wait(&P.dfull[k & 1], (k >> 1) & 1) && clock64() - t0 < kWaitCycles) {
      }
    }
  }
  // every phase has completed: retire the barriers so the next task of a
  // persistent block can initialise them again
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int st = 0; st < S; ++st) {
      asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_addr(&P.full[st])) : "memory");
      asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_addr(&P.empty[st])) : "memory");
    }
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_addr(&P.dfull[0])) : "memory");
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_addr(&P.dfull[1])) : "memory");
  }
}

// ------------------------------------------------------------------ 8-bit samples
template <int RB, int NW, bool OUT16, bool FLUSH>
__device__ __forceinline__ void sum_u8(const SumLaunch& L, uint3 blk, uint32_t* sw, Pipe& P) {
  static_assert(!(OUT16 && FLUSH), "16-bit outputs hold at most 257 sources: no flushes");
  // RB rows per thread: the block's kSumRows rows are split over kSumRows/RB
  // groups of warps, each group covering the whole tile for its RB rows
  constexpr int kGroups = kSumRows / RB;
  constexpr int kWarpsPerTile = kWarps / kGroups;
  constexpr int T = kWarpsPerTile * 32 * NW * 4;
  const Geo g = make_geo(L, T, blk);
  if (g.nrows <= 0) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int rbase = (warp / kWarpsPerTile) * RB, wt = warp % kWarpsPerTile;
  // odd NW: lane owns NW consecutive words (NW+1 conflict-free loads per row and
  // source); even NW: lane owns words lane, lane+32, ... (2 loads per word)
  constexpr bool kConsec = (NW & 1) != 0;
  constexpr int kStride = kConsec ? 1 : 32;
  const int wbase = kConsec ? wt * 32 * NW + lane * NW : wt * 32 * NW + lane;
  const uint32_t one = L.one;
  const uint32_t neg1 = 0u - one, sh24 = one << 24;  // runtime -1 and 2^24
  uint32_t ev[RB][NW], od[RB][NW];  // 16-bit lanes: samples (4w, 4w+2) and (4w+1, 4w+3)
  // DD_SUM8_SPLIT 3: od holds the wrapping sum of whole words and hd the sum of
  // their top bytes; the odd lanes are recovered at the end (see emit)
  constexpr bool kWord = DD_SUM8_SPLIT == 3;
  uint32_t hd[kWord ? RB : 1][kWord ? NW : 1];
  const uint32_t sh8 = L.one << 8;  // 256, a runtime value: the multiply-high stays an IMAD
#pragma unroll
  for (int r = 0; r < RB; ++r)
#pragma unroll
    for (int k = 0; k < NW; ++k) {
      ev[r][k] = od[r][k] = 0;
      if constexpr (kWord) hd[r][k] = 0;
    }
  // Writes the lane sums of rows [0, nrows) to the output, adding them to the
  // partial sums an earlier flush stored there when `add`, and clears the lanes.
  auto emit = [&](bool add) {
    if constexpr (kWord) {
      // whole-word sum = E0 + 2^8 O1 + 2^16 E2 + 2^24 O3 (mod 2^32), with ev = E0 + 2^16 E2
      // exact and hd = O3: O1 = (sum - ev - 2^24 O3) / 2^8 (O1 < 2^16, no wrap)
#pragma unroll
      for (int r = 0; r < RB; ++r)
#pragma unroll
        for (int k = 0; k < NW; ++k) {
          const uint32_t o1 = (od[r][k] - ev[r][k] - (hd[r][k] << 24)) >> 8;
          od[r][k] = o1 | (hd[r][k] << 16);
          hd[r][k] = 0;
        }
    }
#pragma unroll
    for (int r = 0; r < RB; ++r) {
      if (rbase + r >= g.nrows) break;
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        const int64_t t = static_cast<int64_t>(wbase + kStride * k) * 4;  // block-local sample
        if (t < g.valid) {
          const uint32_t s0 = ev[r][k] & 0xffffu, s1 = od[r][k] & 0xffffu;
          const uint32_t s2 = ev[r][k] >> 16, s3 = od[r][k] >> 16;
          char* row = g.out + (rbase + r) * g.out_pitch;
          if constexpr (OUT16) {
            uint16_t* dst = reinterpret_cast<uint16_t*>(row) + t;
            if (t + 4 <= g.valid && (reinterpret_cast<uintptr_t>(dst) & 7) == 0) {
              *reinterpret_cast<uint2*>(dst) = make_uint2(__byte_perm(ev[r][k], od[r][k], 0x5410),
                                                          __byte_perm(ev[r][k], od[r][k], 0x7632));
            } else {
              const uint32_t v[4] = {s0, s1, s2, s3};
              for (int q = 0; q < 4 && t + q < g.valid; ++q) dst[q] = static_cast<uint16_t>(v[q]);
            }
            if (L.twin_off) {  // the twin, twin[i] = sums[i - 1], element by element
              uint16_t* tw = reinterpret_cast<uint16_t*>(row + L.twin_off) + t;
              const uint32_t v[4] = {s0, s1, s2, s3};
              for (int q = 0; q < 4 && t + q < g.valid; ++q) tw[q + 1] = static_cast<uint16_t>(v[q]);
            }
          } else {
            uint32_t* dst = reinterpret_cast<uint32_t*>(row) + t;
            if (t + 4 <= g.valid && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
              uint4 v = make_uint4(s0, s1, s2, s3);
              if (add) {
                const uint4 o = *reinterpret_cast<const uint4*>(dst);
                v.x += o.x; v.y += o.y; v.z += o.z; v.w += o.w;
              }
              *reinterpret_cast<uint4*>(dst) = v;
            } else {
              const uint32_t v[4] = {s0, s1, s2, s3};
              for (int q = 0; q < 4 && t + q < g.valid; ++q) dst[q] = add ? dst[q] + v[q] : v[q];
            }
          }
        }
        ev[r][k] = od[r][k] = 0;
      }
    }
  };
  // 32-bit outputs of many 8-bit sources: every 256 sources each warp adds its
  // lanes into the output through a slice of shared memory past the ring (one row
  // at a time, ordered by __syncwarp), as whole 16-byte chunks: a read-add-write
  // of the partial sums an earlier flush stored when `add`.  Clears the lanes.
  auto flush_staged = [&](bool add) {
    constexpr int kSeg = 32 * NW * 4;  // samples of a warp's segment
    uint32_t* st = sw + (2 * L.stages + 1) * (L.win_bytes >> 2) + warp * kSeg;
    const int64_t seg0 = static_cast<int64_t>(wt) * kSeg;
    const int64_t nv = g.valid - seg0;  // samples of the segment to store (may be <= 0)
#pragma unroll
    for (int r = 0; r < RB; ++r) {
      if (rbase + r >= g.nrows) break;
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        *reinterpret_cast<uint4*>(st + 4 * (lane * NW + k)) =
            make_uint4(ev[r][k] & 0xffffu, od[r][k] & 0xffffu, ev[r][k] >> 16, od[r][k] >> 16);
        ev[r][k] = od[r][k] = 0;
      }
      __syncwarp();
      uint32_t* out = reinterpret_cast<uint32_t*>(g.out + (rbase + r) * g.out_pitch) + seg0;
      for (int c = lane; c < kSeg / 4; c += 32) {
        const int e = 4 * c;
        uint4 v = *reinterpret_cast<const uint4*>(st + e);
        if (e + 4 <= nv && (reinterpret_cast<uintptr_t>(out + e) & 15) == 0) {
          if (add) {
            const uint4 o = *reinterpret_cast<const uint4*>(out + e);
            v.x += o.x; v.y += o.y; v.z += o.z; v.w += o.w;
          }
          *reinterpret_cast<uint4*>(out + e) = v;
        } else {
          const uint32_t a[4] = {v.x, v.y, v.z, v.w};
          for (int q = 0; q < 4; ++q)
            if (e + q < nv) out[e + q] = add ? out[e + q] + a[q] : a[q];
        }
      }
      __syncwarp();
    }
  };
  constexpr bool kStagedFlush = FLUSH && kConsec && DD_SUM8_STAGED_FLUSH;
  int since = 0;       // sources summed in the 16-bit lanes since the last flush
  bool stored = false; // the output holds partial sums of an earlier flush
  run_pipeline<1>(L, g, P, sw, T, [&](int s, const uint32_t* win) {
#pragma unroll
    for (int r = 0; r < RB; ++r) {
      const int4 rw = row_pair(P, s, rbase + r, 0);
      const uint32_t* w0 = win + rw.x + wbase;
      const uint32_t* w1 = win + rw.z + wbase;
      uint32_t va[NW + 1], vb[NW + 1];
      if constexpr (kConsec) {
#pragma unroll
        for (int i = 0; i <= NW; ++i) { va[i] = w0[i]; vb[i] = w1[i]; }
      }
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        const uint32_t a = kConsec ? __funnelshift_r(va[k], va[k + 1], rw.y)
                                   : __funnelshift_r(w0[32 * k], w0[32 * k + 1], rw.y);
        const uint32_t b = kConsec ? __funnelshift_r(vb[k], vb[k + 1], rw.w)
                                   : __funnelshift_r(w1[32 * k], w1[32 * k + 1], rw.w);
        if constexpr (kWord) {
          ev[r][k] += (a & 0x00ff00ffu) + (b & 0x00ff00ffu);
          od[r][k] += a + b;
          hd[r][k] = madhi_u32(a, sh8, hd[r][k]);
          hd[r][k] = madhi_u32(b, sh8, hd[r][k]);
        } else if constexpr (DD_SUM8_SPLIT == 1) {
          const uint32_t ea = a & 0x00ff00ffu, eb = b & 0x00ff00ffu;
          ev[r][k] = mad_u32(ea, one, ev[r][k]);
          ev[r][k] = mad_u32(eb, one, ev[r][k]);
          od[r][k] = madhi_u32(mad_u32(ea, neg1, a), sh24, od[r][k]);
          od[r][k] = madhi_u32(mad_u32(eb, neg1, b), sh24, od[r][k]);
        } else if constexpr (DD_SUM8_SPLIT == 2) {
          const uint32_t ea = a & 0x00ff00ffu, eb = b & 0x00ff00ffu;
          ev[r][k] += ea + eb;
          od[r][k] = madhi_u32(mad_u32(ea, neg1, a), sh24, od[r][k]);
          od[r][k] = madhi_u32(mad_u32(eb, neg1, b), sh24, od[r][k]);
        } else if constexpr (kSumImad) {
          ev[r][k] = mad_u32(__byte_perm(a, 0u, 0x4240), one, ev[r][k]);
          ev[r][k] = mad_u32(__byte_perm(b, 0u, 0x4240), one, ev[r][k]);
          od[r][k] = mad_u32(__byte_perm(a, 0u, 0x4341), one, od[r][k]);
          od[r][k] = mad_u32(__byte_perm(b, 0u, 0x4341), one, od[r][k]);
        } else {
          ev[r][k] += __byte_perm(a, 0u, 0x4240) + __byte_perm(b, 0u, 0x4240);
          od[r][k] += __byte_perm(a, 0u, 0x4341) + __byte_perm(b, 0u, 0x4341);
        }
      }
    }
    if constexpr (FLUSH) {
      since += 2;
      if (since >= 256) {  // 256 x 255 fits a 16-bit lane: move the lanes to the output
        if constexpr (kStagedFlush) flush_staged(stored);
        else emit(stored);
        stored = true;
        since = 0;
      }
    }
  });
  if (P.failed) return;
  if constexpr (OUT16 && kConsec && DD_SUM8_STAGED_OUT) {
    // 16-bit sums leave through shared memory as whole 16-byte chunks: the ring is
    // free once the pipeline has ended (every warp passed its final barrier), and
    // each warp stages one row of its segment at a time in a slice of its own, so
    // only __syncwarp orders the staging.  With a twin (twin[i] = sums[i - 1]) a
    // warp writes twin[1 .. seg] of its segment; twin[0] is the element before
    // the segment, written by the warp (or block) that holds it.
    constexpr int kSeg = 32 * NW * 4;  // samples of a warp's segment
    uint16_t* st = reinterpret_cast<uint16_t*>(sw) + warp * kSeg;
    const int64_t seg0 = static_cast<int64_t>(wt) * kSeg;
    const int64_t nv = g.valid - seg0;  // samples of the segment to store (may be <= 0)
#pragma unroll
    for (int r = 0; r < RB; ++r) {
      if (rbase + r >= g.nrows) break;
#pragma unroll
      for (int k = 0; k < NW; ++k)
        *reinterpret_cast<uint2*>(st + 4 * (lane * NW + k)) =
            make_uint2(__byte_perm(ev[r][k], od[r][k], 0x5410), __byte_perm(ev[r][k], od[r][k], 0x7632));
      __syncwarp();
      char* row = g.out + (rbase + r) * g.out_pitch;
      uint16_t* out = reinterpret_cast<uint16_t*>(row) + seg0;
      uint16_t* tw = L.twin_off ? reinterpret_cast<uint16_t*>(row + L.twin_off) + seg0 : nullptr;
      for (int c = lane; c < kSeg / 8; c += 32) {
        const int e = 8 * c;
        const uint4 v = *reinterpret_cast<const uint4*>(st + e);
        if (e + 8 <= nv && (reinterpret_cast<uintptr_t>(out + e) & 15) == 0) {
          *reinterpret_cast<uint4*>(out + e) = v;
        } else {
          for (int q = 0; q < 8; ++q)
            if (e + q < nv) out[e + q] = st[e + q];
        }
        if (tw) {
          if (c > 0 && e + 7 <= nv && (reinterpret_cast<uintptr_t>(tw + e) & 15) == 0) {
            const uint32_t p = st[e - 1];
            *reinterpret_cast<uint4*>(tw + e) =
                make_uint4(__byte_perm(p, v.x, 0x5410), __byte_perm(v.x, v.y, 0x5432),
                           __byte_perm(v.y, v.z, 0x5432), __byte_perm(v.z, v.w, 0x5432));
          } else {
            for (int q = c == 0 ? 1 : 0; q < 8; ++q)
              if (e + q <= nv) tw[e + q] = st[e + q - 1];
          }
        }
      }
      // the first twin element of the next segment (its warp skips it)
      if (tw && lane == 31 && kSeg <= nv) tw[kSeg] = st[kSeg - 1];
      __syncwarp();
    }
    return;
  }
  if constexpr (kStagedFlush) flush_staged(stored);
  else emit(FLUSH && stored);
}

// ------------------------------------------------------------------ 16-bit samples
// L.lane_per: sources summed in 16-bit lanes before widening (< 2: 32-bit sums).
template <int RB, int NW>
__device__ __forceinline__ void sum_u16(const SumLaunch& L, uint3 blk, uint32_t* sw, Pipe& P) {
  constexpr int T = kWarps * 32 * NW * 2;
  const Geo g = make_geo(L, T, blk);
  if (g.nrows <= 0) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr bool kConsec = (NW & 1) != 0;  // lane layout as in k_sum_u8
  constexpr int kStride = kConsec ? 1 : 32;
  const int wbase = kConsec ? warp * 32 * NW + lane * NW : warp * 32 * NW + lane;
  uint32_t a16[RB][NW], lo32[RB][NW], hi32[RB][NW];
#pragma unroll
  for (int r = 0; r < RB; ++r)
#pragma unroll
    for (int k = 0; k < NW; ++k) a16[r][k] = lo32[r][k] = hi32[r][k] = 0;
  const int npairs = (g.nsrc + 1) / 2;
  const int per = L.lane_per;
  int since = 0, done = 0;
  run_pipeline<2>(L, g, P, sw, 2 * T, [&](int s, const uint32_t* win) {
    ++done;
    if (per >= 2) {
#pragma unroll
      for (int r = 0; r < RB; ++r) {
        const int4 rw = row_pair(P, s, r, 0);
        const uint32_t* w0 = win + rw.x + wbase;
        const uint32_t* w1 = win + rw.z + wbase;
        if ((rw.y | rw.w) == 0) {  // both sources word-aligned (uniform over the block)
#pragma unroll
          for (int k = 0; k < NW; ++k) a16[r][k] += w0[kStride * k] + w1[kStride * k];
        } else if constexpr (kConsec) {
          uint32_t va[NW + 1], vb[NW + 1];
#pragma unroll
          for (int i = 0; i <= NW; ++i) { va[i] = w0[i]; vb[i] = w1[i]; }
#pragma unroll
          for (int k = 0; k < NW; ++k)
            a16[r][k] += __funnelshift_r(va[k], va[k + 1], rw.y) +
                         __funnelshift_r(vb[k], vb[k + 1], rw.w);
        } else {
#pragma unroll
          for (int k = 0; k < NW; ++k) {
            const uint32_t a = __funnelshift_r(w0[32 * k], w0[32 * k + 1], rw.y);
            const uint32_t b = __funnelshift_r(w1[32 * k], w1[32 * k + 1], rw.w);
            a16[r][k] += a + b;
          }
        }
      }
      since += 2;
      if (since + 2 > per || done == npairs) {
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
        const int4 rw = row_pair(P, s, r, 0);
        const uint32_t* w0 = win + rw.x + wbase;
        const uint32_t* w1 = win + rw.z + wbase;
#pragma unroll
        for (int k = 0; k < NW; ++k) {
          const uint32_t a = __funnelshift_r(w0[kStride * k], w0[kStride * k + 1], rw.y);
          const uint32_t b = __funnelshift_r(w1[kStride * k], w1[kStride * k + 1], rw.w);
          lo32[r][k] += (a & 0xffffu) + (b & 0xffffu);
          hi32[r][k] += (a >> 16) + (b >> 16);
        }
      }
    }
  });
  if (P.failed) return;
#pragma unroll
  for (int r = 0; r < RB; ++r) {
    if (r >= g.nrows) break;
#pragma unroll
    for (int k = 0; k < NW; ++k) {
      const int64_t t = static_cast<int64_t>(wbase + kStride * k) * 2;
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

// DD_SUM16W_WHOLE 1: each 32-bit pair of samples is aligned by one byte permute and
// summed whole (wrapping) beside the sum of its high halves; 0: low and high
// halves are taken apart per word by masks and shifts chosen by the offset.
#ifndef DD_SUM16W_WHOLE
#define DD_SUM16W_WHOLE 1
#endif
// 16-bit samples into 32-bit sums (stage 1 and brute force of 16-bit input).
// For output word k (samples 2k, 2k+1 of the block) a source whose offset is
// word-aligned gives the pair w[k] and one offset by a sample the pair
// (w[k] >> 16, w[k+1] & 0xffff), one byte permute of two words (selector 0x3210
// or 0x5432, so no branch separates a row's sources).  The aligned pairs are
// summed whole into a wrapping 32-bit word and their high halves into another
// (two sources per three-input add); the low samples' sums come out at the end
// as whole - (high << 16).  Three integer-pipe operations per word and source,
// where taking the halves apart by masks and offset-dependent selects took five.
template <int RB, int NW>
__device__ __forceinline__ void sum_u16_wide(const SumLaunch& L, uint3 blk, uint32_t* sw, Pipe& P) {
  // RB rows per thread: the block's rows are split over kSumRows/RB warp groups,
  // each covering the whole tile for its RB rows (as in sum_u8)
  constexpr int kGroups = kSumRows / RB;
  constexpr int kWarpsPerTile = kWarps / kGroups;
  constexpr int T = kWarpsPerTile * 32 * NW * 2;
  const Geo g = make_geo(L, T, blk);
  if (g.nrows <= 0) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int rbase = (warp / kWarpsPerTile) * RB, wt = warp % kWarpsPerTile;
  constexpr bool kConsec = (NW & 1) != 0;  // lane layout as in k_sum_u8
  constexpr int kStride = kConsec ? 1 : 32;
  const int wbase = kConsec ? wt * 32 * NW + lane * NW : wt * 32 * NW + lane;
  uint32_t lo32[RB][NW], hi32[RB][NW];
#pragma unroll
  for (int r = 0; r < RB; ++r)
#pragma unroll
    for (int k = 0; k < NW; ++k) lo32[r][k] = hi32[r][k] = 0;
  run_pipeline<2>(L, g, P, sw, 2 * T, [&](int s, const uint32_t* win) {
#pragma unroll
    for (int r = 0; r < RB; ++r) {
      const int4 rw = row_pair(P, s, rbase + r, 0);
      const uint32_t* w0 = win + rw.x + wbase;
      const uint32_t* w1 = win + rw.z + wbase;
      uint32_t va[NW + 1], vb[NW + 1];
#pragma unroll
      for (int i = 0; i <= NW; ++i) {
        if (kConsec || i < NW) {
          va[i] = w0[kStride * i];
          vb[i] = w1[kStride * i];
        } else {  // interleaved lanes: the word after the last one
          va[i] = w0[kStride * (NW - 1) + 1];
          vb[i] = w1[kStride * (NW - 1) + 1];
        }
      }
      if constexpr (DD_SUM16W_WHOLE) {
        // rw.y / rw.w: 0 (word-aligned) or 16 (one sample in): one byte permute
        // aligns the pair; whole words are summed (wrapping) and high halves apart
        const uint32_t sa = rw.y ? 0x5432u : 0x3210u, sb = rw.w ? 0x5432u : 0x3210u;
#pragma unroll
        for (int k = 0; k < NW; ++k) {
          const uint32_t an = kConsec ? va[k + 1] : w0[kStride * k + 1];
          const uint32_t bn = kConsec ? vb[k + 1] : w1[kStride * k + 1];
          const uint32_t a = __byte_perm(va[k], an, sa), b = __byte_perm(vb[k], bn, sb);
          lo32[r][k] += a + b;
          hi32[r][k] += (a >> 16) + (b >> 16);
        }
      } else {
#pragma unroll
        for (int k = 0; k < NW; ++k) {
          const uint32_t an = kConsec ? va[k + 1] : w0[kStride * k + 1];
          const uint32_t bn = kConsec ? vb[k + 1] : w1[kStride * k + 1];
          // rw.y / rw.w: 0 (word-aligned) or 16 (one sample in)
          const uint32_t alo = rw.y ? __umulhi(va[k], 0x10000u) : (va[k] & 0xffffu);
          const uint32_t ahi = rw.y ? (an & 0xffffu) : __umulhi(va[k], 0x10000u);
          const uint32_t blo = rw.w ? __umulhi(vb[k], 0x10000u) : (vb[k] & 0xffffu);
          const uint32_t bhi = rw.w ? (bn & 0xffffu) : __umulhi(vb[k], 0x10000u);
          lo32[r][k] += alo + blo;
          hi32[r][k] += ahi + bhi;
        }
      }
    }
  });
  if constexpr (DD_SUM16W_WHOLE) {
    // lo32 holds sum(low) + 2^16 sum(high) mod 2^32 and sum(low) < 2^32 (at most
    // 65537 sources of 65535), so the low sums are lo32 - (hi32 << 16)
#pragma unroll
    for (int r = 0; r < RB; ++r)
#pragma unroll
      for (int k = 0; k < NW; ++k) lo32[r][k] -= hi32[r][k] << 16;
  }
  if (P.failed) return;
#pragma unroll
  for (int r = 0; r < RB; ++r) {
    if (rbase + r >= g.nrows) break;
#pragma unroll
    for (int k = 0; k < NW; ++k) {
      const int64_t t = static_cast<int64_t>(wbase + kStride * k) * 2;
      if (t >= g.valid) continue;
      uint32_t* dst = reinterpret_cast<uint32_t*>(g.out + (rbase + r) * g.out_pitch) + t;
      if (t + 2 <= g.valid && (reinterpret_cast<uintptr_t>(dst) & 7) == 0) {
        *reinterpret_cast<uint2*>(dst) = make_uint2(lo32[r][k], hi32[r][k]);
      } else {
        dst[0] = lo32[r][k];
        if (t + 1 < g.valid) dst[1] = hi32[r][k];
      }
    }
  }
}

// ------------------------------------------------------------------ 32-bit samples
// Sources of 32-bit words (stage-1 sums stored as uint32): every sample is a whole
// word, so no shifts; sums wrap modulo 2^32 like the reference's uint32 accumulators.
template <int RB, int NW>
__device__ __forceinline__ void sum_u32(const SumLaunch& L, uint3 blk, uint32_t* sw, Pipe& P) {
  constexpr int T = kWarps * 32 * NW;
  const Geo g = make_geo(L, T, blk);
  if (g.nrows <= 0) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wbase = warp * 32 * NW + lane;
  uint32_t acc[RB][NW];
#pragma unroll
  for (int r = 0; r < RB; ++r)
#pragma unroll
    for (int k = 0; k < NW; ++k) acc[r][k] = 0;
  run_pipeline<4>(L, g, P, sw, 4 * T, [&](int s, const uint32_t* win) {
#pragma unroll
    for (int r = 0; r < RB; ++r) {
      const int4 rw = row_pair(P, s, r, 0);
      const uint32_t* w0 = win + rw.x + wbase;
      const uint32_t* w1 = win + rw.z + wbase;
#pragma unroll
      for (int k = 0; k < NW; ++k) acc[r][k] += w0[32 * k] + w1[32 * k];
    }
  });
  if (P.failed) return;
#pragma unroll
  for (int r = 0; r < RB; ++r) {
    if (r >= g.nrows) break;
    uint32_t* row = reinterpret_cast<uint32_t*>(g.out + r * g.out_pitch);
#pragma unroll
    for (int k = 0; k < NW; ++k) {
      const int64_t t = wbase + 32 * k;
      if (t < g.valid) row[t] = acc[r][k];
    }
  }
}

// ------------------------------------------------------------------ 16-bit sums, four sources per stage
// Stage 2 of 8-bit input: sources are 16-bit subband sums of at most 64 channels
// (each <= 64 x 255 = 16320), so the sum of four of them still fits a 16-bit lane
// (<= 65280).  A lane owns NW consecutive 32-bit words of the block's tile (two
// samples each); per row and group of four sources it adds the four aligned
// words in packed 16-bit lanes (a source offset by one sample is aligned with a
// byte permute of two neighbouring words), then folds the packed sum q into two
// 32-bit accumulators: lo += q (wrapping) and hi += q >> 16 (a multiply-high on
// the FMA pipe).  Since no group's low lane carries, the low samples' sum is
// lo - (hi << 16) at the end.  Shared-memory bytes per sample addition are
// about half those of 32-bit subband sums.
// Adds one source's NW aligned words to q: always NW + 1 loads and one byte
// permute per word, whose selector is 0x3210 (even offset) or 0x5432 (offset by
// one sample), so that no branch separates the loads of a row's four sources
// (the form that skipped the extra load and the permutes of even offsets was
// 3 ms slower per headline step).
template <int NW>
__device__ __forceinline__ void add_u16_src(uint32_t (&q)[NW], const uint32_t* w, int shift) {
  const uint32_t sel = shift ? 0x5432u : 0x3210u;
  uint32_t v[NW + 1];
#pragma unroll
  for (int i = 0; i <= NW; ++i) v[i] = w[i];
#pragma unroll
  for (int k = 0; k < NW; ++k) q[k] += __byte_perm(v[k], v[k + 1], sel);
}

template <int RB, int NW>
__device__ __forceinline__ void sum_u16_quad(const SumLaunch& L, uint3 blk, uint32_t* sw, Pipe& P) {
  static_assert(NW & 1, "an odd number of consecutive words per lane keeps the loads conflict-free");
  constexpr int kGroups = kSumRows / RB;  // warp groups sharing the rows, as in sum_u8
  constexpr int kWarpsPerTile = kWarps / kGroups;
  constexpr int T = kWarpsPerTile * 32 * NW * 2;
  const Geo g = make_geo(L, T, blk);
  if (g.nrows <= 0) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int rbase = (warp / kWarpsPerTile) * RB;
  const int wbase = (warp % kWarpsPerTile) * 32 * NW + lane * NW;
  uint32_t lo[RB][NW], hi[RB][NW];
#pragma unroll
  for (int r = 0; r < RB; ++r)
#pragma unroll
    for (int k = 0; k < NW; ++k) lo[r][k] = hi[r][k] = 0;
  run_pipeline<2, 4>(L, g, P, sw, 2 * T, [&](int s, const uint32_t* win) {
#pragma unroll
    for (int r = 0; r < RB; ++r) {
      const int4 a = row_pair(P, s, rbase + r, 0), b = row_pair(P, s, rbase + r, 1);
      uint32_t q[NW];
#pragma unroll
      for (int k = 0; k < NW; ++k) q[k] = 0;
      add_u16_src<NW>(q, win + a.x + wbase, a.y);
      add_u16_src<NW>(q, win + a.z + wbase, a.w);
      add_u16_src<NW>(q, win + b.x + wbase, b.y);
      add_u16_src<NW>(q, win + b.z + wbase, b.w);
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        lo[r][k] += q[k];
        hi[r][k] = __umulhi(q[k], 0x10000u) + hi[r][k];
      }
    }
  });
  if (P.failed) return;
#pragma unroll
  for (int r = 0; r < RB; ++r) {
    if (rbase + r >= g.nrows) break;
#pragma unroll
    for (int k = 0; k < NW; ++k) {
      const int64_t t = static_cast<int64_t>(wbase + k) * 2;
      if (t >= g.valid) continue;
      const uint32_t s0 = lo[r][k] - (hi[r][k] << 16), s1 = hi[r][k];
      uint32_t* dst = reinterpret_cast<uint32_t*>(g.out + (rbase + r) * g.out_pitch) + t;
      if (t + 2 <= g.valid && (reinterpret_cast<uintptr_t>(dst) & 7) == 0) {
        *reinterpret_cast<uint2*>(dst) = make_uint2(s0, s1);
      } else {
        dst[0] = s0;
        if (t + 1 < g.valid) dst[1] = s1;
      }
    }
  }
}

// ------------------------------------------------------------------ 16-bit sums with a shifted twin
// Stage 2 of 8-bit input when stage 1 also wrote the one-sample-shifted twin of
// its sums (SumLaunch::twin_off): a row whose offset for a source is odd reads
// that source's twin, so every source word a row needs is one aligned shared
// load, with no permute.  Four sources per stage are added in packed 16-bit
// lanes (each <= 64 x 255, four <= 65280) and folded into two 32-bit sums as in
// sum_u16_quad; lanes own interleaved words (lane l: l, l + 32, ...), so the
// loads of a warp are 32 consecutive words for any words per lane.  With half
// the instructions of the quad kernel it waits on its shared loads instead
// (long-scoreboard stalls 3.3 per issue at two blocks per SM), so it is built for
// three blocks per SM: 36.7 ms per headline step against 43.2 at two blocks and
// 46.8 for the quad kernel.
#ifndef DD_SUM16T_MINB
#define DD_SUM16T_MINB 3
#endif
template <int RB, int NW>
__device__ __forceinline__ void sum_u16_twin(const SumLaunch& L, uint3 blk, uint32_t* sw, Pipe& P) {
  constexpr int kGroups = kSumRows / RB;  // warp groups sharing the rows, as in sum_u8
  constexpr int kWarpsPerTile = kWarps / kGroups;
  constexpr int T = kWarpsPerTile * 32 * NW * 2;
  const Geo g = make_geo(L, T, blk);
  if (g.nrows <= 0) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int rbase = (warp / kWarpsPerTile) * RB;
  const int wbase = (warp % kWarpsPerTile) * 32 * NW + lane;
  uint32_t lo[RB][NW], hi[RB][NW];
#pragma unroll
  for (int r = 0; r < RB; ++r)
#pragma unroll
    for (int k = 0; k < NW; ++k) lo[r][k] = hi[r][k] = 0;
  run_pipeline<2, 4, kModeTwin>(L, g, P, sw, 2 * T, [&](int s, const uint32_t* win) {
#pragma unroll
    for (int r = 0; r < RB; ++r) {
      const int4 a = row_pair(P, s, rbase + r, 0), b = row_pair(P, s, rbase + r, 1);
      const uint32_t* w0 = win + a.x + wbase;
      const uint32_t* w1 = win + a.z + wbase;
      const uint32_t* w2 = win + b.x + wbase;
      const uint32_t* w3 = win + b.z + wbase;
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        const uint32_t q = (w0[32 * k] + w1[32 * k] + w2[32 * k]) + w3[32 * k];
        lo[r][k] += q;
        hi[r][k] = __umulhi(q, 0x10000u) + hi[r][k];
      }
    }
  });
  if (P.failed) return;
#pragma unroll
  for (int r = 0; r < RB; ++r) {
    if (rbase + r >= g.nrows) break;
#pragma unroll
    for (int k = 0; k < NW; ++k) {
      const int64_t t = static_cast<int64_t>(wbase + 32 * k) * 2;
      if (t >= g.valid) continue;
      const uint32_t s0 = lo[r][k] - (hi[r][k] << 16), s1 = hi[r][k];
      uint32_t* dst = reinterpret_cast<uint32_t*>(g.out + (rbase + r) * g.out_pitch) + t;
      if (t + 2 <= g.valid && (reinterpret_cast<uintptr_t>(dst) & 7) == 0) {
        *reinterpret_cast<uint2*>(dst) = make_uint2(s0, s1);
      } else {
        dst[0] = s0;
        if (t + 1 < g.valid) dst[1] = s1;
      }
    }
  }
}

template <int RB, int NW, bool OUT16, bool FLUSH>
__global__ void __launch_bounds__(kThreads, DD_SUM8_MINB) k_sum_u8(SumLaunch L) {
  extern __shared__ __align__(128) uint32_t sw[];
  __shared__ Pipe P;
  sum_u8<RB, NW, OUT16, FLUSH>(L, blockIdx, sw, P);
}
template <int RB, int NW>
__global__ void __launch_bounds__(kThreads, DD_SUM16_MINB) k_sum_u16(SumLaunch L) {
  extern __shared__ __align__(128) uint32_t sw[];
  __shared__ Pipe P;
  sum_u16<RB, NW>(L, blockIdx, sw, P);
}
template <int RB, int NW>
__global__ void __launch_bounds__(kThreads, DD_SUM16W_MINB) k_sum_u16w(SumLaunch L) {
  extern __shared__ __align__(128) uint32_t sw[];
  __shared__ Pipe P;
  sum_u16_wide<RB, NW>(L, blockIdx, sw, P);
}
template <int RB, int NW>
__global__ void __launch_bounds__(kThreads, DD_SUM16Q_MINB) k_sum_u16q(SumLaunch L) {
  extern __shared__ __align__(128) uint32_t sw[];
  __shared__ Pipe P;
  sum_u16_quad<RB, NW>(L, blockIdx, sw, P);
}
template <int RB, int NW>
__global__ void __launch_bounds__(kThreads, DD_SUM16T_MINB) k_sum_u16t(SumLaunch L) {
  extern __shared__ __align__(128) uint32_t sw[];
  __shared__ Pipe P;
  sum_u16_twin<RB, NW>(L, blockIdx, sw, P);
}
template <int RB, int NW>
__global__ void __launch_bounds__(kThreads, DD_SUM32_MINB) k_sum_u32(SumLaunch L) {
  extern __shared__ __align__(128) uint32_t sw[];
  __shared__ Pipe P;
  sum_u32<RB, NW>(L, blockIdx, sw, P);
}

// ------------------------------------------------------------------ batched launches
// Block-to-group search: the last group whose first block is <= b.
__device__ __forceinline__ int find_group(const SumBatchGroup* groups, int ngroups, long long b) {
  int lo = 0, hi = ngroups - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(&groups[mid].first) <= b) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// The group's launch description, once per block, into shared memory.
__device__ __forceinline__ void load_launch(const SumBatchGroup* g, SumLaunch& s_L) {
  const uint32_t* src = reinterpret_cast<const uint32_t*>(&g->L);
  uint32_t* dst = reinterpret_cast<uint32_t*>(&s_L);
  for (int i = threadIdx.x; i < static_cast<int>(sizeof(SumLaunch) / 4); i += kThreads)
    dst[i] = __ldg(src + i);
}

__device__ __forceinline__ uint3 group_block(long long local, unsigned gx, unsigned gy) {
  uint3 blk;
  blk.x = static_cast<unsigned>(local % gx);
  local /= gx;
  blk.y = static_cast<unsigned>(local % gy);
  blk.z = static_cast<unsigned>(local / gy);
  return blk;
}

template <int KIND>
__device__ __forceinline__ void run_one(const SumLaunch& L, uint3 blk, uint32_t* sw, Pipe& P) {
  if constexpr (KIND == kSumKindU8Out16) sum_u8<kSumRowsPT, DD_SUM8_NW, true, false>(L, blk, sw, P);
  else if constexpr (KIND == kSumKindU8Flush) sum_u8<kSumRowsPT, DD_SUM8F_NW, false, true>(L, blk, sw, P);
  else if constexpr (KIND == kSumKindU8) sum_u8<kSumRowsPT, DD_SUM8_NW, false, false>(L, blk, sw, P);
  else if constexpr (KIND == kSumKindU16) sum_u16<kSumRows, DD_SUM16_NW>(L, blk, sw, P);
  else if constexpr (KIND == kSumKindU16Wide) sum_u16_wide<kSumRowsPTW, DD_SUM16W_NW>(L, blk, sw, P);
  else if constexpr (KIND == kSumKindU16Quad) sum_u16_quad<kSumRowsPTQ, kSum16QNW>(L, blk, sw, P);
  else if constexpr (KIND == kSumKindU16Twin) sum_u16_twin<kSumRowsPTT, kSum16TNW>(L, blk, sw, P);
  else sum_u32<kSumRows, kSum32NW>(L, blk, sw, P);
}

// Grouped launch: one grid over the blocks of several staged sums of the same
// variant (the same stage of many plans), none of which reads another's output.
template <int KIND>
__global__ void __launch_bounds__(kThreads, 2) k_sum_grouped(const SumBatchGroup* groups,
                                                            int ngroups) {
  extern __shared__ __align__(128) uint32_t sw[];
  __shared__ Pipe P;
  __shared__ SumLaunch s_L;
  __shared__ int s_group;
  const long long b = blockIdx.x;
  if (threadIdx.x == 0) s_group = find_group(groups, ngroups, b);
  __syncthreads();
  const SumBatchGroup* G = groups + s_group;
  load_launch(G, s_L);
  __syncthreads();
  run_one<KIND>(s_L, group_block(b - __ldg(&G->first), __ldg(&G->gx), s_L.grid_y), sw, P);
}

// Persistent launch over the blocks of many staged sums, dependent stages
// included.  Blocks are handed out in order by an atomic counter; a group whose
// input is produced by an earlier group waits (bounded) until that group's
// blocks have all signalled completion.  Every block of an earlier group has
// already been handed to a running block, so the waits always end.
__device__ __forceinline__ void run_kind(int kind, const SumLaunch& L, uint3 blk, uint32_t* sw,
                                         Pipe& P) {
  switch (kind) {
    case kSumKindU8Out16: run_one<kSumKindU8Out16>(L, blk, sw, P); break;
    case kSumKindU8Flush: run_one<kSumKindU8Flush>(L, blk, sw, P); break;
    case kSumKindU8: run_one<kSumKindU8>(L, blk, sw, P); break;
    case kSumKindU16: run_one<kSumKindU16>(L, blk, sw, P); break;
    case kSumKindU16Wide: run_one<kSumKindU16Wide>(L, blk, sw, P); break;
    case kSumKindU16Quad: run_one<kSumKindU16Quad>(L, blk, sw, P); break;
    case kSumKindU16Twin: run_one<kSumKindU16Twin>(L, blk, sw, P); break;
    default: run_one<kSumKindU32>(L, blk, sw, P); break;
  }
}

__global__ void __launch_bounds__(kThreads, 2) k_sum_batch(const SumBatchGroup* groups,
                                                          int ngroups, long long total,
                                                          int* ctrs, unsigned long long* next,
                                                          int* err) {
  extern __shared__ __align__(128) uint32_t sw[];
  __shared__ Pipe P;
  __shared__ SumLaunch s_L;
  __shared__ long long s_blk;
  __shared__ int s_group, s_ok;
  // the next block is taken while the current one runs, so the atomic's latency
  // overlaps work (the hand-out order is unchanged)
  long long b_next = 0;
  if (threadIdx.x == 0) b_next = static_cast<long long>(atomicAdd(next, 1ull));
  for (;;) {
    if (threadIdx.x == 0) {
      const long long b = b_next;
      s_blk = b;
      s_ok = 1;
      if (b < total) {
        b_next = static_cast<long long>(atomicAdd(next, 1ull));
        const int g = find_group(groups, ngroups, b);
        s_group = g;
        const int wc = groups[g].wait_ctr;
        if (wc >= 0) {
          const int need = groups[g].wait_need;
          const long long t0 = clock64();
          for (;;) {
            int v;
            asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(ctrs + wc) : "memory");
            if (v >= need) break;
            if (*reinterpret_cast<volatile int*>(err) || clock64() - t0 > kWaitCycles) {
              atomicCAS(err, 0, kErrWaitGroup);
              s_ok = 0;
              break;
            }
            __nanosleep(128);
          }
          // the bulk copies that follow read what the other blocks wrote
          asm volatile("fence.proxy.async.global;\n" ::: "memory");
        }
      }
    }
    __syncthreads();
    const long long b = s_blk;
    if (b >= total) break;
    const SumBatchGroup* G = groups + s_group;
    load_launch(G, s_L);
    __syncthreads();
    if (s_ok) run_kind(G->kind, s_L, group_block(b - G->first, G->gx, s_L.grid_y), sw, P);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(ctrs + G->done_ctr, 1);
  }
}

template <typename K>
void launch_k(K kernel, dim3 grid, size_t smem, const SumLaunch& L, cudaStream_t st) {
  allow_dynamic_smem(kernel, smem);
  kernel<<<grid, kThreads, smem, st>>>(L);
  DD_LAUNCHED();
}

}  // namespace

int sum_tile_samples(int src_bytes, int nw) { return kWarps * 32 * nw * (4 / src_bytes); }

// Ring of `stages` groups of qs windows plus one zeroed window.
size_t sum_smem_bytes(int win_bytes, int stages, int qs) {
  return static_cast<size_t>(qs * stages + 1) * win_bytes;
}

size_t sum_kind_extra_smem(int kind) {
  // the flush staging of the 8-bit kernel with 32-bit outputs: one segment of
  // 32-bit sums per warp
  return (kind == kSumKindU8Flush && DD_SUM8_STAGED_FLUSH && (DD_SUM8F_NW & 1))
             ? static_cast<size_t>(kWarps) * 32 * DD_SUM8F_NW * 4 * sizeof(uint32_t)
             : 0;
}

size_t sum_launch_smem(const SumLaunch& L) {
  const int kind = sum_kind(L);
  return sum_smem_bytes(L.win_bytes, L.stages, sum_kind_qs(kind)) + sum_kind_extra_smem(kind);
}

// Staged source pairs for a window size: as many as fit DD_SUM_SMEM_KB of shared
// memory (two blocks per SM at the default), at least two.
// The twin-window stage-2 kernel (eight windows per stage) is limited by the
// latency of its shared loads rather than by issue: it takes at most
// DD_SUM16T_SMEM_KB so that three blocks fit an SM.
#ifndef DD_SUM16T_SMEM_KB
#define DD_SUM16T_SMEM_KB 68
#endif
int sum_stages(int win_bytes, int qs, size_t extra, int cap_kb) {
  const size_t cap = static_cast<size_t>(cap_kb > 0 ? cap_kb : DD_SUM_SMEM_KB) * 1024;
  int s = kMaxStages;
  while (s > 2 && sum_smem_bytes(win_bytes, s, qs) + extra > cap) --s;
  return s;
}

int sum_kind_stages(int kind, int win_bytes) {
  return sum_stages(win_bytes, sum_kind_qs(kind), sum_kind_extra_smem(kind),
                    kind == kSumKindU16Twin   ? DD_SUM16T_SMEM_KB
                    : kind == kSumKindU16Wide ? DD_SUM16W_SMEM_KB
                                              : DD_SUM_SMEM_KB);
}

std::vector<SumDesc> build_sum_desc(const std::vector<int32_t>& tab, int64_t nrows,
                                    int64_t ncols, int64_t group) {
  const int64_t blk = group > 0 ? group : nrows;
  const int64_t per = (blk + kSumRows - 1) / kSumRows;  // row groups per block of rows
  const int64_t nblk = (nrows + blk - 1) / blk;
  std::vector<SumDesc> d(static_cast<size_t>(nblk * per * ncols));
  for (int64_t b = 0; b < nblk; ++b) {
    const int64_t b0 = b * blk, b1 = std::min(nrows, b0 + blk);
    for (int64_t gi = 0; gi < per; ++gi) {
      const int64_t r0 = b0 + gi * kSumRows;
      const int64_t r1 = std::min(b1, r0 + kSumRows);
      SumDesc* row = d.data() + (b * per + gi) * ncols;
      if (r0 >= r1) continue;
      for (int64_t c = 0; c < ncols; ++c) {
        int lo = tab[r0 * ncols + c], hi = lo;
        for (int64_t r = r0 + 1; r < r1; ++r) {
          lo = std::min(lo, tab[r * ncols + c]);
          hi = std::max(hi, tab[r * ncols + c]);
        }
        if (hi - lo > 65535) throw Error{DD_ERR_RUNTIME, "staged-sum offsets spread too far"};
        SumDesc& e = row[c];
        e.lo = lo;
        e.span = hi - lo;
        for (int r = 0; r < kSumRows; ++r)
          e.rel[r] = static_cast<uint16_t>(r0 + r < r1 ? tab[(r0 + r) * ncols + c] - lo : 0);
      }
    }
  }
  return d;
}

void launch_sum(const SumLaunch& L, cudaStream_t st) {
  dim3 grid(sum_grid_x(L), L.grid_y, L.grid_z);
  if (L.stages < 2 || L.stages > kMaxStages) throw Error{DD_ERR_RUNTIME, "bad stage count"};
  if (!L.desc || !L.err) throw Error{DD_ERR_RUNTIME, "staged sum without descriptors"};
  const size_t smem = sum_launch_smem(L);
  if (L.rows_per_block != kSumRows) throw Error{DD_ERR_RUNTIME, "unsupported rows per block"};
  switch (sum_kind(L)) {
    case kSumKindU8Out16: launch_k(k_sum_u8<kSumRowsPT, DD_SUM8_NW, true, false>, grid, smem, L, st); break;
    case kSumKindU8Flush: launch_k(k_sum_u8<kSumRowsPT, DD_SUM8F_NW, false, true>, grid, smem, L, st); break;
    case kSumKindU8: launch_k(k_sum_u8<kSumRowsPT, DD_SUM8_NW, false, false>, grid, smem, L, st); break;
    case kSumKindU16: launch_k(k_sum_u16<kSumRows, DD_SUM16_NW>, grid, smem, L, st); break;
    case kSumKindU16Wide: launch_k(k_sum_u16w<kSumRowsPTW, DD_SUM16W_NW>, grid, smem, L, st); break;
    case kSumKindU16Quad: launch_k(k_sum_u16q<kSumRowsPTQ, kSum16QNW>, grid, smem, L, st); break;
    case kSumKindU16Twin: launch_k(k_sum_u16t<kSumRowsPTT, kSum16TNW>, grid, smem, L, st); break;
    default: launch_k(k_sum_u32<kSumRows, kSum32NW>, grid, smem, L, st); break;
  }
}

int sum_kind(const SumLaunch& L) {
  if (L.src_bytes == 1) {
    if (L.out_elem == 2) return kSumKindU8Out16;
    return L.flush ? kSumKindU8Flush : kSumKindU8;
  }
  if (L.src_bytes == 2)
    return L.flush              ? kSumKindU16Wide
           : L.lane_per < 4     ? kSumKindU16
           : L.twin_off != 0   ? kSumKindU16Twin
                                : kSumKindU16Quad;
  return kSumKindU32;
}

unsigned sum_grid_x(const SumLaunch& L) {
  const int T = sum_kind_tile(sum_kind(L));
  return static_cast<unsigned>((L.ncols + T - 1) / T);
}

int sum_batch_blocks_per_sm(size_t smem) {
  int n = 0;
  DD_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_sum_batch, kThreads, smem));
  return n;
}

void launch_sum_batch(const SumBatchGroup* d_groups, int ngroups, long long total, int* d_ctrs,
                      unsigned long long* d_next, int* d_err, size_t smem, unsigned grid,
                      cudaStream_t st) {
  allow_dynamic_smem(k_sum_batch, smem);
  k_sum_batch<<<grid, kThreads, smem, st>>>(d_groups, ngroups, total, d_ctrs, d_next, d_err);
  DD_LAUNCHED();
}

template <int KIND>
void launch_grouped_k(const SumBatchGroup* d_groups, int ngroups, long long total, size_t smem,
                      cudaStream_t st) {
  allow_dynamic_smem(k_sum_grouped<KIND>, smem);
  k_sum_grouped<KIND><<<static_cast<unsigned>(total), kThreads, smem, st>>>(d_groups, ngroups);
  DD_LAUNCHED();
}

// Two independent staged sums in one launch: stage 1 of time tile k+1 and
// stage 2 of tile k (different subband-sum buffers).  Stage 1 of 8-bit input is
// bound by the integer pipe and stage 2 by shared-memory loads; with the blocks
// of the two interleaved, each SM runs one of each and both units stay busy.
// Blocks 0, 2, 4, ... take the first sum's blocks in order, 1, 3, 5, ... the
// second's, and the tail of the longer one follows.
template <int K1, int K2>
__global__ void __launch_bounds__(kThreads, 2) k_sum_pair(SumLaunch L1, SumLaunch L2,
                                                          long long n1, long long n2, unsigned gx1,
                                                          unsigned gx2) {
  extern __shared__ __align__(128) uint32_t sw[];
  __shared__ Pipe P;
  const long long b = blockIdx.x;
  const long long m = n1 < n2 ? n1 : n2;
  int role;
  long long local;
  if (b < 2 * m) {
    role = static_cast<int>(b & 1);
    local = b >> 1;
  } else {
    role = n1 > n2 ? 0 : 1;
    local = m + (b - 2 * m);
  }
  if (role == 0) run_one<K1>(L1, group_block(local, gx1, L1.grid_y), sw, P);
  else run_one<K2>(L2, group_block(local, gx2, L2.grid_y), sw, P);
}

template <int K1, int K2>
void launch_pair_k(const SumLaunch& L1, const SumLaunch& L2, cudaStream_t st) {
  const unsigned gx1 = sum_grid_x(L1), gx2 = sum_grid_x(L2);
  const long long n1 = static_cast<long long>(gx1) * L1.grid_y * L1.grid_z;
  const long long n2 = static_cast<long long>(gx2) * L2.grid_y * L2.grid_z;
  const size_t smem = std::max(sum_launch_smem(L1), sum_launch_smem(L2));
  if (n1 + n2 >= (1LL << 31)) throw Error{DD_ERR_RUNTIME, "paired launch too large"};
  allow_dynamic_smem(k_sum_pair<K1, K2>, smem);
  k_sum_pair<K1, K2><<<static_cast<unsigned>(n1 + n2), kThreads, smem, st>>>(L1, L2, n1, n2, gx1, gx2);
  DD_LAUNCHED();
}

bool launch_sum_pair(const SumLaunch& L1, const SumLaunch& L2, cudaStream_t st) {
  for (const SumLaunch* L : {&L1, &L2}) {
    if (L->stages < 2 || L->stages > kMaxStages || !L->desc || !L->err ||
        L->rows_per_block != kSumRows)
      throw Error{DD_ERR_RUNTIME, "bad staged-sum launch"};
  }
  const int k1 = sum_kind(L1), k2 = sum_kind(L2);
  if (k1 == kSumKindU8 && k2 == kSumKindU32) launch_pair_k<kSumKindU8, kSumKindU32>(L1, L2, st);
  else if (k1 == kSumKindU8Out16 && k2 == kSumKindU16Quad) launch_pair_k<kSumKindU8Out16, kSumKindU16Quad>(L1, L2, st);
  else if (k1 == kSumKindU8Out16 && k2 == kSumKindU16Twin) launch_pair_k<kSumKindU8Out16, kSumKindU16Twin>(L1, L2, st);
  else if (k1 == kSumKindU16Wide && k2 == kSumKindU32) launch_pair_k<kSumKindU16Wide, kSumKindU32>(L1, L2, st);
  else if (k1 == kSumKindU8Flush && k2 == kSumKindU32) launch_pair_k<kSumKindU8Flush, kSumKindU32>(L1, L2, st);
  else return false;
  return true;
}

void launch_sum_grouped(const SumBatchGroup* d_groups, int ngroups, long long total, int kind,
                        size_t smem, cudaStream_t st) {
  if (total <= 0) return;
  if (total >= (1LL << 31)) throw Error{DD_ERR_RUNTIME, "grouped launch too large"};
  switch (kind) {
    case kSumKindU8Out16: launch_grouped_k<kSumKindU8Out16>(d_groups, ngroups, total, smem, st); break;
    case kSumKindU8Flush: launch_grouped_k<kSumKindU8Flush>(d_groups, ngroups, total, smem, st); break;
    case kSumKindU8: launch_grouped_k<kSumKindU8>(d_groups, ngroups, total, smem, st); break;
    case kSumKindU16: launch_grouped_k<kSumKindU16>(d_groups, ngroups, total, smem, st); break;
    case kSumKindU16Wide: launch_grouped_k<kSumKindU16Wide>(d_groups, ngroups, total, smem, st); break;
    case kSumKindU16Quad: launch_grouped_k<kSumKindU16Quad>(d_groups, ngroups, total, smem, st); break;
    case kSumKindU16Twin: launch_grouped_k<kSumKindU16Twin>(d_groups, ngroups, total, smem, st); break;
    default: launch_grouped_k<kSumKindU32>(d_groups, ngroups, total, smem, st); break;
  }
}

}  // namespace dd
