// IQRM channel masks without any device allocation (dd_iqrm_masks_noalloc).
//
// Some callers cannot allocate device memory while they run: a real-time beam
// pipeline whose deadline forbids cudaMalloc/cudaFree (both can synchronise
// the whole device and take unbounded time), or a host framework that has
// already reserved the GPU's memory for its own pools and ring buffers, where
// an extra cudaMalloc would fail or fragment that reservation.  For them this
// entry point computes the same IQRM window masks as the plan path
// (dd_run_ex's iqrm_masks output) with all of its working memory taken from
// g_iqrm_scratch below, a fixed array every GPU that loads this library holds
// until the process exits.  Only the input and the two outputs belong to the
// caller.
//
// Limits: the working set of one call (per-window column sums, statistics,
// lagged differences, votes and per-lag flags, plus the window and lag lists)
// must fit in kScratchBytes; larger requests are rejected with DD_ERR_INVALID
// and a message giving the size needed.
//
// Every call uses the same array, and the array keeps the previous call's
// contents: each call clears the sums it accumulates into before using them.
// Calls whose GPU work overlaps (on different streams, or from different host
// threads without ordering) race on the array and corrupt each other's results;
// callers must serialise them.
//
// The first call on a device looks up the array's device address for that
// device (cudaGetSymbolAddress) with the device current; make that first call
// before any stream capture.  The library's device code is loaded lazily, so
// that first call is also when the 8 MiB array is placed in the device's
// memory: a host that reserves most of the GPU's memory for its own pools
// should make one call (any valid small request) before reserving it.  After
// cudaDeviceReset the cached address is stale and the process must not call
// this entry point on that device again.
//
// The window list and the lags are written into the array by a kernel that
// takes their few defining numbers by value, so the GPU work of a call never
// reads host memory after the call has returned.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>

#include "dd_internal.h"

namespace dd {
namespace {

constexpr size_t kScratchBytes = size_t(8) << 20;  // 8 MiB per device
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_iqrm_scratch[kScratchBytes];

std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of g_iqrm_scratch on the current device (looked up once per device).
void* scratch_on_current_device() {
  int dev = -1;
  DD_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) throw Error{DD_ERR_RUNTIME, "device index out of range"};
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_iqrm_scratch);
    if (e != cudaSuccess || p == nullptr)
      throw Error{DD_ERR_CUDA, std::string("cudaGetSymbolAddress(g_iqrm_scratch): ") +
                                   cudaGetErrorString(e)};
    g_scratch_addr[dev] = p;
  }
  return g_scratch_addr[dev];
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// IQRM windows and lags of one call, written into the scratch array.
// Windows (the reference's plan, src/core/iqrm.cu:348-397): a single window
// [0, ns) when single != 0; else window k < nfull is [k*hop, k*hop + W) and, when
// tail != 0, window nfull is [nfull*hop, ns).  Lags (src/core/iqrm.cu:188-200):
// +lag, -lag for lag = 1, max(floor(g*lag), lag+1), ... while lag <= radius,
// leaving out lags of magnitude >= csub; the host sized the list with the same
// double arithmetic.
__global__ void k_noalloc_tables(uint32_t* win, int nwin, int single, uint32_t ns, uint32_t W,
                                 uint32_t hop, int nfull, int32_t* lags, int radius, double g,
                                 int64_t csub) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nwin; k += gridDim.x * blockDim.x) {
    uint32_t t0, t1;
    if (single) {
      t0 = 0u;
      t1 = ns;
    } else if (k < nfull) {
      t0 = static_cast<uint32_t>(static_cast<uint64_t>(k) * hop);
      t1 = t0 + W;
    } else {
      t0 = static_cast<uint32_t>(static_cast<uint64_t>(nfull) * hop);
      t1 = ns;
    }
    win[2 * k] = t0;
    win[2 * k + 1] = t1;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    int n = 0;
    for (int lag = 1; lag <= radius;) {
      if (lag < csub) {
        lags[n++] = +lag;
        lags[n++] = -lag;
      }
      const int nxt = static_cast<int>(g * lag);
      lag = nxt > lag + 1 ? nxt : lag + 1;
    }
  }
}

}  // namespace
}  // namespace dd

using namespace dd;

extern "C" int dd_iqrm_masks_noalloc(const void* input, int32_t nbits, int64_t nsamp,
                                     int32_t nchans, int32_t chan_start, int32_t chan_end,
                                     double tsamp, const dd_iqrm_config* cfg, uint8_t* masks,
                                     uint32_t* bounds, int32_t max_windows, int32_t* n_windows,
                                     void* stream) {
  try {
    set_error("");
    if (!input || !cfg || !masks || !bounds || !n_windows)
      throw Error{DD_ERR_INVALID, "NULL argument"};
    if (nbits != 8 && nbits != 16 && nbits != 32) throw Error{DD_ERR_INVALID, "nbits must be 8, 16 or 32"};
    if (nsamp < 1 || nsamp >= (int64_t(1) << 32) || nchans < 1 || !(tsamp > 0))
      throw Error{DD_ERR_INVALID, "need 1 <= nsamp < 2^32, nchans >= 1 and tsamp > 0"};
    if (chan_start < 0 || chan_end > nchans || chan_start >= chan_end)
      throw Error{DD_ERR_INVALID, "channel range must satisfy 0 <= chan_start < chan_end <= nchans"};
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // Window plan (src/core/iqrm.cu:348-397 with the clamps of include/iqrm.hpp:30-41).
    const double win_sec = std::max(0.0, cfg->win_sec), hop_sec = std::max(0.0, cfg->hop_sec);
    const uint32_t ns = static_cast<uint32_t>(nsamp);
    const uint32_t W = win_sec > 0.0 ? static_cast<uint32_t>(std::floor(win_sec / tsamp)) : 0u;
    const uint32_t H = hop_sec > 0.0 ? static_cast<uint32_t>(std::floor(hop_sec / tsamp)) : W;
    const bool single = (W == 0 || W >= ns);
    const uint32_t hop = H ? H : W;
    int nfull = 0, tail = 0;
    if (!single) {
      uint64_t t0 = 0;
      while (t0 + W <= ns) {
        ++nfull;
        t0 += hop;
      }
      tail = (cfg->include_tail && t0 < ns && ns > t0 + 4) ? 1 : 0;
    }
    const int nwin = single ? 1 : nfull + tail;
    *n_windows = nwin;
    if (nwin > max_windows)
      throw Error{DD_ERR_INVALID, "max_windows (" + std::to_string(max_windows) +
                                      ") is smaller than the " + std::to_string(nwin) +
                                      " IQRM windows of this chunk"};
    // Lags (src/core/iqrm.cu:188-200); lags of magnitude >= csub are left out.
    const int64_t csub = chan_end - chan_start;
    const float rf = std::max(0.0f, cfg->radius_frac);
    volatile float rprod = rf * static_cast<float>(csub);
    const int radius = std::max(1, static_cast<int>(std::floor(static_cast<float>(rprod))));
    const double g = cfg->geofactor > 1.0 ? cfg->geofactor : 1.5;
    int nlags = 0;
    for (int lag = 1; lag <= radius;) {
      if (lag < csub) nlags += 2;
      lag = std::max(static_cast<int>(g * lag), lag + 1);
    }
    if (nlags) check_iqrm_channels(csub);  // the per-window sort fits shared memory

    // Scratch layout inside g_iqrm_scratch.
    const size_t b_win = align256(sizeof(uint32_t) * 2 * nwin);
    const size_t b_lags = align256(sizeof(int32_t) * std::max(1, nlags));
    const size_t b_sums = align256(sizeof(unsigned long long) * 2 * csub * nwin);
    const size_t b_work = align256(iqrm_scratch_bytes(nwin, csub, nlags));
    const size_t need = b_win + b_lags + b_sums + b_work;
    if (need > kScratchBytes) {
      char msg[256];
      std::snprintf(msg, sizeof(msg),
                    "IQRM working set of %zu bytes exceeds the %zu-byte static scratch "
                    "(%d windows x %lld channels x %d lags)",
                    need, kScratchBytes, nwin, static_cast<long long>(csub), nlags);
      throw Error{DD_ERR_INVALID, msg};
    }
    char* base = static_cast<char*>(scratch_on_current_device());
    uint32_t* d_win = reinterpret_cast<uint32_t*>(base);
    int32_t* d_lags = reinterpret_cast<int32_t*>(base + b_win);
    unsigned long long* d_sums = reinterpret_cast<unsigned long long*>(base + b_win + b_lags);
    void* d_work = base + b_win + b_lags + b_sums;

    const int tb = 256;
    const int tg = static_cast<int>(std::min<int64_t>((nwin + tb - 1) / tb, 1024));
    k_noalloc_tables<<<tg, tb, 0, st>>>(d_win, nwin, single ? 1 : 0, ns, W, hop, nfull, d_lags,
                                        radius, g, csub);
    DD_LAUNCHED();
    if (nlags) {
      // launch_iqrm_stats clears the sums before accumulating into them.
      launch_iqrm_stats(input, nbits, nsamp, nchans, chan_start, csub, d_win, nwin, d_sums, st);
      launch_iqrm_decide(d_sums, nwin, d_win, nchans, chan_start, csub, cfg->mode,
                         std::max(0.0f, cfg->nsigma), d_lags, nlags, 8 | 4, d_work, masks, st);
    } else {
      DD_CUDA_TRY(cudaMemsetAsync(masks, 0, static_cast<size_t>(nwin) * nchans, st));
    }
    DD_CUDA_TRY(cudaMemcpyAsync(bounds, d_win, sizeof(uint32_t) * 2 * nwin,
                                cudaMemcpyDeviceToDevice, st));
    return DD_OK;
  } catch (const Error& e) {
    set_error(e.msg);
    return e.code;
  } catch (const std::exception& e) {
    set_error(e.what());
    return DD_ERR_RUNTIME;
  }
}
