// Ingest: chunks from SIGPROC filterbank files or host arrays into device memory
// in the layout the plans read ([time][channel], ascending frequency).
//
// The reference reads a whole file with one fread into host memory
// (src/data/filterbank.cpp:454-473), reverses the channel order of every
// sample on the host when foff < 0 (filterbank.cpp:793-842), and later copies
// the array to the device from pageable memory; its PSRFITS reader averages the
// first two polarisations and flips the band in numpy
// (python/astroflow/io/psrfits.py:31-80).  Here the data travel in fixed-size
// blocks: worker threads read (pread) or copy blocks into pinned staging
// buffers, each block is copied to the device on the worker's stream, and the
// channel flip and polarisation average run on the device on that block, so
// disk or host-memory reads, PCIe/C2C copies and the transforms overlap.
#include <cuda_runtime.h>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <mutex>
#include <type_traits>
#include <string>
#include <thread>
#include <vector>

#include "dd_internal.h"

namespace dd {
namespace {

// ------------------------------------------------------------------ SIGPROC header
struct FileReader {
  int fd = -1;
  int64_t pos = 0;
  ~FileReader() {
    if (fd >= 0) close(fd);
  }
  void read(void* dst, size_t n) {
    size_t got = 0;
    while (got < n) {
      const ssize_t r = pread(fd, static_cast<char*>(dst) + got, n - got, pos + static_cast<int64_t>(got));
      if (r <= 0) throw Error{DD_ERR_INVALID, "unexpected end of file in the header"};
      got += static_cast<size_t>(r);
    }
    pos += static_cast<int64_t>(n);
  }
  std::string string() {
    int32_t n = 0;
    read(&n, 4);
    if (n < 0 || n > 4096) throw Error{DD_ERR_INVALID, "Non-Standard file format."};
    std::string s(static_cast<size_t>(n), '\0');
    if (n) read(&s[0], static_cast<size_t>(n));
    return s;
  }
};

// Keywords of src/data/filterbank.cpp:319-452 with their value types.
const char* const kIntKeys[] = {"telescope_id", "machine_id", "data_type", "barycentric",
                                "pulsarcentric", "nbits", "nchans", "nifs", "nbins", "ibeam",
                                "nbeams", "npuls", "nsamples"};
const char* const kDoubleKeys[] = {"az_start", "za_start", "src_raj", "src_dej", "tstart",
                                   "tsamp", "period", "fch1", "foff", "refdm"};

struct ParsedHeader {
  dd_fil_header h{};
  std::vector<double> table;  // as stored in the file
};

ParsedHeader parse_header(const char* path) {
  FileReader f;
  f.fd = open(path, O_RDONLY | O_CLOEXEC);
  if (f.fd < 0) throw Error{DD_ERR_INVALID, std::string("cannot open ") + path};
  ParsedHeader P;
  dd_fil_header& h = P.h;
  if (f.string() != "HEADER_START") throw Error{DD_ERR_INVALID, "Non-Standard file format."};
  bool table_mode = false;
  int32_t nbits = 0, nchans = 0, nifs = 0;
  double tsamp = 0, fch1 = 0, foff = 0, tstart = 0;
  for (;;) {
    const std::string key = f.string();
    if (key == "HEADER_END") break;
    if (key == "rawdatafile" || key == "source_name") {
      f.string();
    } else if (key == "FREQUENCY_START") {
      table_mode = true;
      P.table.clear();
    } else if (key == "FREQUENCY_END") {
      nchans = static_cast<int32_t>(P.table.size());
    } else if (key == "fchannel") {
      double v;
      f.read(&v, 8);
      P.table.push_back(v);
      table_mode = true;
    } else if (std::find_if(std::begin(kDoubleKeys), std::end(kDoubleKeys),
                            [&](const char* k) { return key == k; }) != std::end(kDoubleKeys)) {
      double v;
      f.read(&v, 8);
      if (key == "tsamp") tsamp = v;
      else if (key == "fch1") fch1 = v;
      else if (key == "foff") foff = v;
      else if (key == "tstart") tstart = v;
    } else if (std::find_if(std::begin(kIntKeys), std::end(kIntKeys),
                            [&](const char* k) { return key == k; }) != std::end(kIntKeys)) {
      int32_t v;
      f.read(&v, 4);
      if (key == "nbits") nbits = v;
      else if (key == "nchans") nchans = v;
      else if (key == "nifs") nifs = v;
    } else {
      throw Error{DD_ERR_INVALID, "read_header - unknown parameter : " + key};
    }
  }
  if (nifs == 0) nifs = 1;
  if (nbits != 8 && nbits != 16 && nbits != 32)
    throw Error{DD_ERR_INVALID, "Unsupported nbits value: " + std::to_string(nbits)};
  if (nchans < 1) throw Error{DD_ERR_INVALID, "nchans must be positive"};
  const bool use_table = table_mode && !P.table.empty();
  if (use_table) fch1 = foff = 0.0;  // the reader keeps only the table
  struct stat st {};
  if (fstat(f.fd, &st) != 0) throw Error{DD_ERR_INVALID, "cannot stat the file"};
  const int64_t per = static_cast<int64_t>(nifs) * nchans * (nbits / 8);
  h.header_bytes = f.pos;
  h.ndata = (static_cast<int64_t>(st.st_size) - f.pos) / per;
  h.nbits = nbits;
  h.nchans = nchans;
  h.nifs = nifs;
  h.tsamp = tsamp;
  h.tstart = tstart;
  h.has_freq_table = use_table ? 1 : 0;
  h.flipped = foff < 0 ? 1 : 0;
  if (h.flipped && nifs != 1)
    throw Error{DD_ERR_INVALID, "Only supports nifs == 1 in reverse_channanl_data"};
  if (!use_table) {
    P.table.resize(static_cast<size_t>(nchans));
    // fch1 + i*foff, which the reference build contracts into a fused multiply-add
    for (int32_t i = 0; i < nchans; ++i) P.table[i] = std::fma(static_cast<double>(i), foff, fch1);
  }
  if (h.flipped) {
    std::reverse(P.table.begin(), P.table.end());
    if (!use_table) {
      fch1 = P.table[0];
      foff = std::fabs(foff);
    }
  }
  h.fch1 = fch1;
  h.foff = foff;
  return P;
}

// ------------------------------------------------------------------ device transforms
// Reverse the channel order of `rows` rows of n elements, in place.
template <typename T>
__global__ void k_flip_rows(T* x, int64_t rows, int64_t n) {
  const int64_t half = n / 2;
  const int64_t total = rows * half;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / half, c = i - r * half;
    T* row = x + r * n;
    const T a = row[c], b = row[n - 1 - c];
    row[c] = b;
    row[n - 1 - c] = a;
  }
}

// Average of polarisations 0 and 1 of [rows][npol][n] as the reference's numpy
// expression ((a + b) / 2).astype(dtype): the sum wraps in the sample type, the
// halving truncates toward zero; optionally with the channel order reversed.
template <typename T>
__global__ void k_pol_average(const T* in, int64_t rows, int npol, int64_t n, int flip, T* out) {
  const int64_t total = rows * n;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / n, c = i - r * n;
    using U = typename std::make_unsigned<T>::type;
    const T* row = in + r * npol * n;
    const T s = static_cast<T>(static_cast<U>(row[c]) + static_cast<U>(row[n + c]));  // wraps like numpy
    const T v = static_cast<T>(s / 2);                // integer halving truncates toward 0
    out[r * n + (flip ? n - 1 - c : c)] = v;
  }
}

template <typename T>
__global__ void k_select_pol0(const T* in, int64_t rows, int npol, int64_t n, int flip, T* out) {
  const int64_t total = rows * n;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / n, c = i - r * n;
    out[r * n + (flip ? n - 1 - c : c)] = in[r * npol * n + c];
  }
}

unsigned grid_for(int64_t work) {
  return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, 148 * 16)));
}

void launch_flip(void* x, int elem, int64_t rows, int64_t n, cudaStream_t st) {
  if (n < 2 || rows < 1) return;
  const unsigned g = grid_for(rows * (n / 2));
  switch (elem) {
    case 1: k_flip_rows<uint8_t><<<g, 256, 0, st>>>(static_cast<uint8_t*>(x), rows, n); break;
    case 2: k_flip_rows<uint16_t><<<g, 256, 0, st>>>(static_cast<uint16_t*>(x), rows, n); break;
    default: k_flip_rows<uint32_t><<<g, 256, 0, st>>>(static_cast<uint32_t*>(x), rows, n); break;
  }
  DD_LAUNCHED();
}

void launch_pol(const void* in, int elem, bool is_signed, int64_t rows, int npol, int64_t n,
                bool flip, void* out, cudaStream_t st) {
  const unsigned g = grid_for(rows * n);
  const int f = flip ? 1 : 0;
  if (npol >= 2) {
    switch (elem * (is_signed ? -1 : 1)) {
      case 1: k_pol_average<uint8_t><<<g, 256, 0, st>>>(static_cast<const uint8_t*>(in), rows, npol, n, f, static_cast<uint8_t*>(out)); break;
      case -1: k_pol_average<int8_t><<<g, 256, 0, st>>>(static_cast<const int8_t*>(in), rows, npol, n, f, static_cast<int8_t*>(out)); break;
      case 2: k_pol_average<uint16_t><<<g, 256, 0, st>>>(static_cast<const uint16_t*>(in), rows, npol, n, f, static_cast<uint16_t*>(out)); break;
      case -2: k_pol_average<int16_t><<<g, 256, 0, st>>>(static_cast<const int16_t*>(in), rows, npol, n, f, static_cast<int16_t*>(out)); break;
      case 4: k_pol_average<uint32_t><<<g, 256, 0, st>>>(static_cast<const uint32_t*>(in), rows, npol, n, f, static_cast<uint32_t*>(out)); break;
      default: k_pol_average<int32_t><<<g, 256, 0, st>>>(static_cast<const int32_t*>(in), rows, npol, n, f, static_cast<int32_t*>(out)); break;
    }
  } else {
    switch (elem) {
      case 1: k_select_pol0<uint8_t><<<g, 256, 0, st>>>(static_cast<const uint8_t*>(in), rows, npol, n, f, static_cast<uint8_t*>(out)); break;
      case 2: k_select_pol0<uint16_t><<<g, 256, 0, st>>>(static_cast<const uint16_t*>(in), rows, npol, n, f, static_cast<uint16_t*>(out)); break;
      default: k_select_pol0<uint32_t><<<g, 256, 0, st>>>(static_cast<const uint32_t*>(in), rows, npol, n, f, static_cast<uint32_t*>(out)); break;
    }
  }
  DD_LAUNCHED();
}

// ------------------------------------------------------------------ staged transfer
// Pinned staging buffers kept for the life of the process (pinning is slow);
// one transfer at a time uses them.
constexpr size_t kBlockBytes = size_t(16) << 20;
constexpr int kWorkers = 8;
constexpr int kBuffersPerWorker = 2;

struct Staging {
  std::mutex mu;
  std::vector<void*> pinned;
  int device = -1;
};
Staging& staging() {
  static Staging s;
  return s;
}

// One transfer: `nblocks` blocks of whole rows.  fill(block, dst) puts block b's
// source bytes into pinned memory dst and returns its size; then the block is
// copied to device_dst + offset(b) (or to a device staging buffer when a
// transform reads it) and transformed on the worker's stream.
struct Transfer {
  int64_t rows;            // rows in total
  int64_t rows_per_block;
  size_t src_row_bytes;    // bytes per row in the source
  size_t dst_row_bytes;    // bytes per row in the destination
  char* device_dst;
  // transform of a block already in device memory at `src` (device), writing
  // `rows` rows to `dst` (device); nullptr: none (the copy lands in place)
  std::function<void(const void* src, int64_t rows, void* dst, cudaStream_t)> transform;
  bool in_place = true;    // transform runs on the destination rows themselves
  std::function<void(int64_t row0, int64_t rows, void* pinned)> fill;
};

void run_transfer(const Transfer& T, cudaStream_t caller) {
  if (T.rows <= 0) return;
  Staging& S = staging();
  std::lock_guard<std::mutex> lock(S.mu);
  int dev = 0;
  DD_CUDA_TRY(cudaGetDevice(&dev));
  if (S.pinned.empty()) {
    for (int i = 0; i < kWorkers * kBuffersPerWorker; ++i) {
      void* p = nullptr;
      DD_CUDA_TRY(cudaHostAlloc(&p, kBlockBytes, cudaHostAllocPortable));
      S.pinned.push_back(p);
    }
  }
  const int64_t nblocks = (T.rows + T.rows_per_block - 1) / T.rows_per_block;
  const int nw = static_cast<int>(std::min<int64_t>(kWorkers, nblocks));
  cudaEvent_t start;
  DD_CUDA_TRY(cudaEventCreateWithFlags(&start, cudaEventDisableTiming));
  DD_CUDA_TRY(cudaEventRecord(start, caller));
  std::vector<cudaStream_t> streams(static_cast<size_t>(nw), nullptr);
  std::vector<cudaEvent_t> done(static_cast<size_t>(nw * kBuffersPerWorker), nullptr);
  std::vector<void*> dstage(static_cast<size_t>(nw * kBuffersPerWorker), nullptr);
  std::atomic<int> failed{0};
  std::string first_error;
  std::mutex err_mu;
  auto fail = [&](const std::string& m) {
    std::lock_guard<std::mutex> g(err_mu);
    if (!failed.exchange(1)) first_error = m;
  };
  std::vector<std::thread> threads;
  try {
    for (int w = 0; w < nw; ++w) {
      DD_CUDA_TRY(cudaStreamCreateWithFlags(&streams[w], cudaStreamNonBlocking));
      DD_CUDA_TRY(cudaStreamWaitEvent(streams[w], start, 0));
      for (int k = 0; k < kBuffersPerWorker; ++k) {
        DD_CUDA_TRY(cudaEventCreateWithFlags(&done[w * kBuffersPerWorker + k], cudaEventDisableTiming));
        if (!T.in_place)
          DD_CUDA_TRY(cudaMallocAsync(&dstage[w * kBuffersPerWorker + k], kBlockBytes, streams[w]));
      }
    }
    for (int w = 0; w < nw; ++w) {
      threads.emplace_back([&, w]() {
        cudaSetDevice(dev);
        int use = 0;
        for (int64_t b = w; b < nblocks && !failed.load(); b += nw, ++use) {
          const int slot = w * kBuffersPerWorker + (use % kBuffersPerWorker);
          void* pin = S.pinned[static_cast<size_t>(slot)];
          if (use >= kBuffersPerWorker && cudaEventSynchronize(done[slot]) != cudaSuccess) {
            fail("staged copy failed");
            return;
          }
          const int64_t row0 = b * T.rows_per_block;
          const int64_t rows = std::min(T.rows_per_block, T.rows - row0);
          try {
            T.fill(row0, rows, pin);
          } catch (const Error& e) {
            fail(e.msg);
            return;
          }
          const size_t bytes = static_cast<size_t>(rows) * T.src_row_bytes;
          char* dst = T.device_dst + row0 * static_cast<int64_t>(T.dst_row_bytes);
          void* land = T.in_place ? static_cast<void*>(dst) : dstage[slot];
          cudaError_t e = cudaMemcpyAsync(land, pin, bytes, cudaMemcpyHostToDevice, streams[w]);
          if (e == cudaSuccess && T.transform) {
            try {
              T.transform(land, rows, dst, streams[w]);
            } catch (const Error& er) {
              fail(er.msg);
              return;
            }
          }
          if (e == cudaSuccess) e = cudaEventRecord(done[slot], streams[w]);
          if (e != cudaSuccess) {
            fail(std::string("staged copy: ") + cudaGetErrorString(e));
            return;
          }
        }
      });
    }
  } catch (const Error& e) {
    fail(e.msg);
  } catch (const std::exception& e) {  // e.g. a worker thread that could not start
    fail(e.what());
  }
  for (auto& t : threads)
    if (t.joinable()) t.join();
  // order the caller's stream after every block, then release the workers' resources
  for (int w = 0; w < nw; ++w) {
    if (!streams[w]) continue;
    cudaEvent_t end;
    if (cudaEventCreateWithFlags(&end, cudaEventDisableTiming) == cudaSuccess) {
      cudaEventRecord(end, streams[w]);
      cudaStreamWaitEvent(caller, end, 0);
      cudaEventDestroy(end);
    }
    for (int k = 0; k < kBuffersPerWorker; ++k)
      if (dstage[w * kBuffersPerWorker + k]) cudaFreeAsync(dstage[w * kBuffersPerWorker + k], streams[w]);
  }
  // the pinned buffers are reused by the next transfer: wait for this one's copies
  for (cudaStream_t s : streams)
    if (s) cudaStreamSynchronize(s);
  for (cudaEvent_t e : done)
    if (e) cudaEventDestroy(e);
  for (cudaStream_t s : streams)
    if (s) cudaStreamDestroy(s);
  cudaEventDestroy(start);
  if (failed.load()) throw Error{DD_ERR_INVALID, first_error};
}

}  // namespace
}  // namespace dd

using namespace dd;

extern "C" int dd_fil_read_header(const char* path, dd_fil_header* out, double* freq_table,
                                  int32_t cap) {
  if (!path || !out) { set_error("NULL argument"); return DD_ERR_INVALID; }
  try {
    set_error("");
    ParsedHeader P = parse_header(path);
    *out = P.h;
    if (freq_table)
      for (int32_t i = 0; i < std::min<int32_t>(cap, P.h.nchans); ++i) freq_table[i] = P.table[static_cast<size_t>(i)];
    return DD_OK;
  } catch (const Error& e) {
    set_error(e.msg);
    return e.code;
  }
}

extern "C" int dd_fil_read(const char* path, int64_t t0, int64_t nsamp, void* device_out,
                           void* stream) {
  if (!path || !device_out) { set_error("NULL argument"); return DD_ERR_INVALID; }
  try {
    set_error("");
    const ParsedHeader P = parse_header(path);
    const dd_fil_header& h = P.h;
    if (h.nifs != 1) throw Error{DD_ERR_INVALID, "only single-IF files can be read to the device"};
    if (t0 < 0 || nsamp < 0 || t0 + nsamp > h.ndata)
      throw Error{DD_ERR_INVALID, "samples outside the file"};
    const int elem = h.nbits / 8;
    const size_t row = static_cast<size_t>(h.nchans) * elem;
    if (row > kBlockBytes) throw Error{DD_ERR_INVALID, "a sample does not fit a staging block"};
    const int fd = open(path, O_RDONLY | O_CLOEXEC);
    if (fd < 0) throw Error{DD_ERR_INVALID, std::string("cannot open ") + path};
    struct Closer { int fd; ~Closer() { close(fd); } } closer{fd};
    Transfer T;
    T.rows = nsamp;
    T.rows_per_block = static_cast<int64_t>(kBlockBytes / row);
    T.src_row_bytes = T.dst_row_bytes = row;
    T.device_dst = static_cast<char*>(device_out);
    T.in_place = true;
    const int64_t data0 = h.header_bytes + t0 * static_cast<int64_t>(row);
    T.fill = [&](int64_t r0, int64_t rows, void* pin) {
      const size_t n = static_cast<size_t>(rows) * row;
      size_t got = 0;
      while (got < n) {
        const ssize_t r = pread(fd, static_cast<char*>(pin) + got, n - got,
                                data0 + r0 * static_cast<int64_t>(row) + static_cast<int64_t>(got));
        if (r <= 0) throw Error{DD_ERR_INVALID, "Data ends unexpected read to EOF"};
        got += static_cast<size_t>(r);
      }
    };
    if (h.flipped) {
      const int64_t n = h.nchans;
      T.transform = [elem, n](const void*, int64_t rows, void* dst, cudaStream_t s) {
        launch_flip(dst, elem, rows, n, s);
      };
    }
    run_transfer(T, static_cast<cudaStream_t>(stream));
    return DD_OK;
  } catch (const Error& e) {
    set_error(e.msg);
    return e.code;
  }
}

extern "C" int dd_ingest_host(const void* host, int64_t nsamp, int32_t npol, int32_t nchans,
                              int32_t elem_bytes, int32_t flags, void* device_out, void* stream) {
  if (!host || !device_out) { set_error("NULL argument"); return DD_ERR_INVALID; }
  try {
    set_error("");
    if (elem_bytes != 1 && elem_bytes != 2 && elem_bytes != 4)
      throw Error{DD_ERR_INVALID, "elem_bytes must be 1, 2 or 4"};
    if (nsamp < 0 || npol < 1 || nchans < 1) throw Error{DD_ERR_INVALID, "bad array shape"};
    const bool flip = (flags & DD_INGEST_FLIP) != 0;
    const bool is_signed = (flags & DD_INGEST_SIGNED) != 0;
    const size_t src_row = static_cast<size_t>(npol) * nchans * elem_bytes;
    const size_t dst_row = static_cast<size_t>(nchans) * elem_bytes;
    if (src_row > kBlockBytes) throw Error{DD_ERR_INVALID, "a sample does not fit a staging block"};
    Transfer T;
    T.rows = nsamp;
    T.rows_per_block = static_cast<int64_t>(kBlockBytes / src_row);
    T.src_row_bytes = src_row;
    T.dst_row_bytes = dst_row;
    T.device_dst = static_cast<char*>(device_out);
    const char* src = static_cast<const char*>(host);
    T.fill = [src, src_row](int64_t r0, int64_t rows, void* pin) {
      std::memcpy(pin, src + r0 * static_cast<int64_t>(src_row), static_cast<size_t>(rows) * src_row);
    };
    const int64_t n = nchans;
    const int elem = elem_bytes;
    if (npol > 1) {
      T.in_place = false;
      const int np = npol;
      T.transform = [=](const void* in, int64_t rows, void* dst, cudaStream_t s) {
        launch_pol(in, elem, is_signed, rows, np, n, flip, dst, s);
      };
    } else if (flip) {
      T.transform = [=](const void*, int64_t rows, void* dst, cudaStream_t s) {
        launch_flip(dst, elem, rows, n, s);
      };
    }
    run_transfer(T, static_cast<cudaStream_t>(stream));
    return DD_OK;
  } catch (const Error& e) {
    set_error(e.msg);
    return e.code;
  }
}
