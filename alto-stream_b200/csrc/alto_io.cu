// Tensor files (the reference's ImportSparseTensor / ExportSparseTensor,
// src/sptensor.cpp:22-249), with the parse on the device.
//
// Text (.tns) import.  The file is streamed into HBM by reader threads (one
// per host hardware thread, 4 to 16) through pinned staging buffers; then,
// all on the device:
//   1. per 16 KiB tile, the line starts that getline's rule keeps (more
//      than one byte read, no leading '#'), counted from 16-byte loads
//      (tns_count_kernel); an exclusive scan over the tiles gives each kept
//      line its nonzero slot, and the same tiles again write every kept
//      line's start at its slot (tns_starts_kernel);
//   2. per kept line, the reference's own parse (tns_parse_kernel, a
//      block's 256 lines staged in shared memory): nmodes
//      strtoull calls (exact, including sign, overflow and no-digit cases)
//      and one strtod.  Decimal values whose significand fits 19 digits and
//      whose value is exact in Clinger's fast path (significand <= 2^53,
//      power of ten <= 10^22, so one correctly rounded IEEE multiply or
//      divide) are converted on the device; any other value text
//      (hexadecimal, inf/nan, long significands, large exponents) is
//      listed; its text is copied back in bulk and converted with the C
//      library's strtod on all host cores, so every value equals the
//      reference's bit for bit.
// The mode count comes from the first valid line, split on space and tab as
// the reference's strtok does (the newline stays in the last token).
//
// Binary import streams the file's index and value arrays straight into one
// device buffer.  Export formats on the host with all cores ("%llu " of index
// + 1, "%g\n" of the value; integral values below 1e6 are written digit by
// digit, which is what %g prints for them) and writes in order.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <mutex>
#include <new>
#include <string>
#include <thread>

#include "alto_internal.cuh"

namespace alto {
alto_status check_coo_shape(const alto_coo* coo);
}

using namespace alto;

struct alto_dcoo {
  int nmodes = 0;
  uint64_t nnz = 0;
  uint64_t dims[ALTO_MAX_MODES] = {};
  DevBuf raw;  // [nmodes][nnz] uint64 indices, then [nnz] float64 values
  const void* ptrs[ALTO_MAX_MODES] = {};
  double read_ms = 0, parse_ms = 0;
  uint64_t file_bytes = 0, host_lines = 0;
};

namespace {

constexpr int kIoThreads = 256;
constexpr int kIoBytesPerThread = 64;
constexpr uint64_t kIoTile = (uint64_t)kIoThreads * kIoBytesPerThread;  // 16 KiB
constexpr size_t kStage = 16ull << 20;                                   // pinned staging buffer

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* total) {
  __shared__ uint32_t ws[kIoThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[warp] = x;
  __syncthreads();
  uint32_t pre = 0, tot = 0;
#pragma unroll
  for (int w = 0; w < kIoThreads / 32; ++w) {
    if (w < warp) pre += ws[w];
    tot += ws[w];
  }
  __syncthreads();
  *total = tot;
  return pre + x - v;
}

// The valid line starts in this thread's 64 bytes [base, base + 64): a
// position q starts a line when q == 0 or byte q - 1 is a newline, and the
// line is one getline reads with more than one byte and without a leading
// '#' exactly when q + 1 < size and byte q is neither '\n' nor '#'.  The
// bytes come from four 16-byte loads (the buffer is zero-padded to a whole
// tile, so they stay inside it).  Calls f(q) for each, in order.
template <typename F>
__device__ __forceinline__ void valid_starts(const uint4* __restrict__ buf, uint64_t base, uint64_t size, F f) {
  const unsigned char* b8 = reinterpret_cast<const unsigned char*>(buf);
  unsigned prev = base ? b8[base - 1] : (unsigned)'\n';
#pragma unroll
  for (int k = 0; k < kIoBytesPerThread / 16; ++k) {
    const uint4 w = buf[base / 16 + k];
    const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const unsigned c = (ws[j] >> (8 * b)) & 0xffu;
        const uint64_t q = base + k * 16 + j * 4 + b;
        if (prev == '\n' && q + 1 < size && c != '\n' && c != '#') f(q);
        prev = c;
      }
  }
}

__global__ void __launch_bounds__(kIoThreads)
    tns_count_kernel(const uint4* __restrict__ buf, uint64_t size, uint32_t* __restrict__ tile_lines) {
  const uint64_t base = blockIdx.x * kIoTile + threadIdx.x * (uint64_t)kIoBytesPerThread;
  uint32_t c = 0, tot;
  valid_starts(buf, base, size, [&](uint64_t) { ++c; });
  block_excl_scan(c, &tot);
  if (threadIdx.x == 0) tile_lines[blockIdx.x] = tot;
}

// starts[k] = the start of the k-th valid line (its nonzero slot is k).
__global__ void __launch_bounds__(kIoThreads)
    tns_starts_kernel(const uint4* __restrict__ buf, uint64_t size, const uint32_t* __restrict__ tile_base,
                      uint64_t* __restrict__ starts) {
  const uint64_t base = blockIdx.x * kIoTile + threadIdx.x * (uint64_t)kIoBytesPerThread;
  uint32_t c = 0, tot;
  valid_starts(buf, base, size, [&](uint64_t) { ++c; });
  uint32_t r = tile_base[blockIdx.x] + block_excl_scan(c, &tot);
  valid_starts(buf, base, size, [&](uint64_t q) { starts[r++] = q; });
}

// 10^0 .. 10^22, every one exact in float64.
__constant__ double c_p10[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,  1e8,  1e9,  1e10, 1e11,
                                 1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};

__device__ __forceinline__ bool is_space(unsigned c) {
  return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
}

// Byte sources for the parse: at(q) is byte q of the line's buffer, 0 (the
// C string's terminator) at or past the end.  Shared memory with 32-bit
// offsets for staged lines, global memory otherwise.
struct SmemBytes {
  const unsigned char* b;
  uint32_t e;
  __device__ __forceinline__ unsigned at(uint32_t q) const { return q < e ? (unsigned)b[q] : 0u; }
};
struct GlobalBytes {
  const unsigned char* b;
  uint64_t e;
  __device__ __forceinline__ unsigned at(uint64_t q) const { return q < e ? (unsigned)__ldg(b + q) : 0u; }
};

// strtoull(p, &end, 10) on the line at p: the line ends at its newline, a
// NUL or the buffer's end (the reference parses one getline buffer, so
// nothing after the newline is reached: skipping whitespace stops there as
// it stops at the buffer's terminating NUL).
template <typename Src, typename Pos>
__device__ __forceinline__ uint64_t dev_strtoull(const Src& s, Pos& p) {
  Pos q = p;
  unsigned c = s.at(q);
  while (c != 0u && c != '\n' && is_space(c)) c = s.at(++q);
  bool neg = false;
  if (c == '+' || c == '-') {
    neg = c == '-';
    c = s.at(++q);
  }
  uint64_t v = 0;
  bool any = false, over = false;
  constexpr uint64_t kMax10 = 1844674407370955161ull;  // (2^64 - 1) / 10, remainder 5
  while (c - '0' < 10u) {
    const unsigned d = c - '0';
    if (v > kMax10 || (v == kMax10 && d > 5)) over = true;
    v = v * 10 + d;
    any = true;
    c = s.at(++q);
  }
  if (!any) return 0;  // no conversion: the end pointer stays at p
  p = q;
  if (over) return ~0ull;
  return neg ? (uint64_t)(0 - v) : v;
}

// strtod's decimal fast path; false when the host must convert the text.
template <typename Src, typename Pos>
__device__ __forceinline__ bool dev_strtod(const Src& s, Pos p, double& out) {
  Pos q = p;
  unsigned c = s.at(q);
  while (c != 0u && c != '\n' && is_space(c)) c = s.at(++q);
  bool neg = false;
  if (c == '+' || c == '-') {
    neg = c == '-';
    c = s.at(++q);
  }
  {  // hexadecimal, inf, nan: the host converts
    const unsigned lc = c | 0x20u;
    if (lc == 'i' || lc == 'n') return false;
    if (c == '0' && (s.at(q + 1) | 0x20u) == 'x') return false;
  }
  uint64_t w = 0;
  int nd = 0, ex = 0;
  bool any = false;
  while (c - '0' < 10u) {
    const unsigned d = c - '0';
    any = true;
    if (w != 0 || d != 0) {  // (leading zeros carry no digit)
      if (nd == 19) return false;
      w = w * 10 + d;
      ++nd;
    }
    c = s.at(++q);
  }
  if (c == '.') {
    c = s.at(++q);
    while (c - '0' < 10u) {
      const unsigned d = c - '0';
      any = true;
      if (w != 0 || d != 0) {
        if (nd == 19) return false;
        w = w * 10 + d;
        ++nd;
      }
      --ex;
      c = s.at(++q);
    }
  }
  if (!any) {  // no conversion
    out = 0.0;
    return true;
  }
  if ((c | 0x20u) == 'e') {
    Pos r = q + 1;
    unsigned ce = s.at(r);
    bool eneg = false;
    if (ce == '+' || ce == '-') {
      eneg = ce == '-';
      ce = s.at(++r);
    }
    if (ce - '0' < 10u) {
      int x = 0;
      while (ce - '0' < 10u) {
        if (x < 100000) x = x * 10 + (int)(ce - '0');
        ce = s.at(++r);
      }
      ex += eneg ? -x : x;
    }
  }
  if (w == 0) {
    out = neg ? -0.0 : 0.0;
    return true;
  }
  constexpr uint64_t k2p53 = 1ull << 53;
  if (w > k2p53) return false;
  double v;
  if (ex >= 0 && ex <= 22) {
    v = __dmul_rn((double)w, c_p10[ex]);
  } else if (ex < 0 && ex >= -22) {
    v = __ddiv_rn((double)w, c_p10[-ex]);
  } else if (ex > 22 && ex <= 22 + 16) {  // move powers into the significand while it stays exact
    uint64_t ww = w;
    for (int k = 22; k < ex; ++k) {
      if (ww > k2p53 / 10) return false;
      ww *= 10;
    }
    v = __dmul_rn((double)ww, c_p10[22]);
  } else {
    return false;
  }
  out = neg ? -v : v;
  return true;
}

// One line: nmodes indices and the value (its slot k, the line's start s).
// NM > 0: the mode count at compile time (the loop unrolls and dmax stays in
// registers); NM = 0: nmodes at run time.
template <int NM, typename Src, typename Pos>
__device__ __forceinline__ void parse_line(const Src& src, Pos s, uint64_t k, int nmodes, uint64_t zero_based,
                                           uint64_t nnz, uint64_t* __restrict__ idx, double* __restrict__ vals,
                                           uint64_t (&dmax)[ALTO_MAX_MODES], uint64_t* __restrict__ host_list,
                                           uint32_t host_cap, uint32_t* __restrict__ host_count) {
  const uint64_t one_based = zero_based ? 0 : 1;
  Pos p = s;
#pragma unroll
  for (int m = 0; m < (NM ? NM : nmodes); ++m) {
    const uint64_t x = dev_strtoull(src, p);
    dmax[m] = max(dmax[m], x + zero_based);
    idx[(uint64_t)m * nnz + k] = x - one_based;
  }
  double v = 0.0;
  if (!dev_strtod(src, p, v)) {  // the host converts this value (line start + value offset)
    const uint32_t h = atomicAdd(host_count, 1u);
    if (h < host_cap) {  // (past the capacity the count still grows; the host then reruns)
      host_list[2 * (uint64_t)h] = k;
      host_list[2 * (uint64_t)h + 1] = (uint64_t)(p - s);
    }
  }
  vals[k] = v;
}

constexpr int kStageBytes = 24 << 10;  // a block's lines staged in shared memory

// One thread per valid line.  A block takes 256 consecutive lines; when
// their bytes fit kStageBytes they are staged in shared memory with 16-byte
// loads and parsed from there, else parsed from global memory.
template <int NM>
__global__ void __launch_bounds__(kIoThreads)
    tns_parse_kernel(const unsigned char* __restrict__ buf, uint64_t size, const uint64_t* __restrict__ starts,
                     uint64_t nnz, int nmodes, uint64_t zero_based, uint64_t* __restrict__ idx,
                     double* __restrict__ vals, unsigned long long* __restrict__ dims,
                     uint64_t* __restrict__ host_list, uint32_t host_cap, uint32_t* __restrict__ host_count) {
  __shared__ __align__(16) unsigned char sm[kStageBytes];
  uint64_t dmax[ALTO_MAX_MODES];
  for (int m = 0; m < ALTO_MAX_MODES; ++m) dmax[m] = 0;
  for (uint64_t k0 = (uint64_t)blockIdx.x * kIoThreads; k0 < nnz; k0 += (uint64_t)gridDim.x * kIoThreads) {
    const uint64_t k1 = min(k0 + kIoThreads, nnz);
    const uint64_t lo = starts[k0], hi = k1 < nnz ? starts[k1] : size;
    const uint64_t alo = lo & ~15ull, span = hi - alo;
    const bool staged = span <= (uint64_t)kStageBytes;
    if (staged) {
      const uint4* src = reinterpret_cast<const uint4*>(buf + alo);
      for (uint64_t o = threadIdx.x; o * 16 < span; o += kIoThreads) reinterpret_cast<uint4*>(sm)[o] = src[o];
    }
    __syncthreads();
    const uint64_t k = k0 + threadIdx.x;
    if (k < k1) {
      if (staged)
        parse_line<NM>(SmemBytes{sm, (uint32_t)span}, (uint32_t)(starts[k] - alo), k, nmodes, zero_based, nnz,
                       idx, vals, dmax, host_list, host_cap, host_count);
      else
        parse_line<NM>(GlobalBytes{buf, hi}, starts[k], k, nmodes, zero_based, nnz, idx, vals, dmax, host_list,
                       host_cap, host_count);
    }
    __syncthreads();
  }
#pragma unroll
  for (int m = 0; m < (NM ? NM : nmodes); ++m) atomicMax(dims + m, (unsigned long long)dmax[m]);
}

// The parse for nmodes modes (3, 4 and 5, the reference's specialised mode
// counts, compiled for their count).
alto_status launch_parse(unsigned grid, cudaStream_t st, const unsigned char* buf, uint64_t size,
                         const uint64_t* starts, uint64_t nnz, int nmodes, uint64_t zero_based, uint64_t* idx,
                         double* vals, unsigned long long* dims, uint64_t* host_list, uint32_t host_cap,
                         uint32_t* host_count) {
  if (nmodes == 3)
    tns_parse_kernel<3><<<grid, kIoThreads, 0, st>>>(buf, size, starts, nnz, nmodes, zero_based, idx, vals, dims,
                                                     host_list, host_cap, host_count);
  else if (nmodes == 4)
    tns_parse_kernel<4><<<grid, kIoThreads, 0, st>>>(buf, size, starts, nnz, nmodes, zero_based, idx, vals, dims,
                                                     host_list, host_cap, host_count);
  else if (nmodes == 5)
    tns_parse_kernel<5><<<grid, kIoThreads, 0, st>>>(buf, size, starts, nnz, nmodes, zero_based, idx, vals, dims,
                                                     host_list, host_cap, host_count);
  else
    tns_parse_kernel<0><<<grid, kIoThreads, 0, st>>>(buf, size, starts, nnz, nmodes, zero_based, idx, vals, dims,
                                                     host_list, host_cap, host_count);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

// Listed entries [i0, i0 + n): each value's text, from its offset to the
// line's newline, a NUL or the file's end, NUL-terminated in a kValText-byte
// slot; a text that does not fit ends with byte 1 in the slot's last byte
// (the host then re-reads that line from the file).
constexpr int kValText = 64;
__global__ void value_text_kernel(const uint64_t* __restrict__ list, uint64_t i0, uint32_t n,
                                  const uint64_t* __restrict__ starts, const unsigned char* __restrict__ buf,
                                  uint64_t size, char* __restrict__ out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint64_t k = list[2 * (i0 + i)], off = list[2 * (i0 + i) + 1];
    uint64_t q = starts[k] + off;
    char* o = out + (uint64_t)i * kValText;
    int c = 0;
    while (c < kValText - 1 && q < size && buf[q] != '\n' && buf[q] != 0) o[c++] = (char)buf[q++];
    o[c] = 0;
    o[kValText - 1] = (c == kValText - 1 && q < size && buf[q] != '\n' && buf[q] != 0) ? 1 : 0;
  }
}

__global__ void scatter_vals_kernel(const uint32_t* __restrict__ at, const double* __restrict__ v, uint32_t n,
                                    double* __restrict__ vals) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) vals[at[i]] = v[i];
}

unsigned grid_io(uint64_t n, int threads) {
  uint64_t b = (n + threads - 1) / threads;
  if (b > 148ull * 16) b = 148ull * 16;
  return (unsigned)(b ? b : 1);
}

double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Pinned staging for file reads, kept per device for the life of the
// process (pinning is slow; a read should not pay for it): up to kReaders
// reader
// threads, each with two buffers and its own non-blocking stream.
constexpr int kReaders = 16;  // (used: the host's hardware threads, 4 .. 16)

int reader_count() {
  static const int n = (int)std::min(16u, std::max(4u, std::thread::hardware_concurrency()));
  return n;
}

struct Staging {
  std::mutex mu;  // one read at a time per device
  void* buf[kReaders][2] = {};
  cudaEvent_t ev[kReaders][2] = {};
  cudaStream_t st[kReaders] = {};
  bool ready = false;
  alto_status init() {
    if (ready) return ALTO_OK;
    for (int r = 0; r < reader_count(); ++r) {
      ALTO_TRY_CUDA(cudaStreamCreateWithFlags(&st[r], cudaStreamNonBlocking));
      for (int i = 0; i < 2; ++i) {
        ALTO_TRY_CUDA(cudaHostAlloc(&buf[r][i], kStage, cudaHostAllocDefault));
        ALTO_TRY_CUDA(cudaEventCreateWithFlags(&ev[r][i], cudaEventDisableTiming));
      }
    }
    ready = true;
    return ALTO_OK;
  }
};

Staging* staging_for_device() {
  static std::mutex mu;
  static Staging* per[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> g(mu);
  if (!per[dev]) per[dev] = new Staging();
  return per[dev];
}

// Read bytes [off, off + n) of fd into device memory dst: chunk c goes to
// reader c % (reader count), which reads it into one of its pinned buffers and
// copies it on its own stream, so file reads and copies overlap.  Every copy
// is complete on return (work that follows on any stream sees the bytes).
alto_status stream_file(int fd, uint64_t off, uint64_t n, char* dst) {
  Staging* sg = staging_for_device();
  if (!sg) {
    set_error("no current CUDA device");
    return ALTO_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lock(sg->mu);
  ALTO_TRY(sg->init());
  const uint64_t nchunks = (n + kStage - 1) / kStage;
  const int nr = (int)std::min<uint64_t>(reader_count(), std::max<uint64_t>(nchunks, 1));
  std::atomic<int> failed{0};
  std::vector<std::string> errs(nr);
  auto reader = [&](int r) {
    int slot = 0;
    bool used[2] = {false, false};
    for (uint64_t c = r; c < nchunks && !failed.load(); c += nr) {
      const uint64_t at = c * kStage;
      const size_t want = (size_t)std::min<uint64_t>(kStage, n - at);
      if (used[slot] && cudaEventSynchronize(sg->ev[r][slot]) != cudaSuccess) {
        errs[r] = "staging copy failed";
        failed = 1;
        break;
      }
      size_t got = 0;
      while (got < want) {
        const ssize_t k = pread(fd, static_cast<char*>(sg->buf[r][slot]) + got, want - got, (off_t)(off + at + got));
        if (k <= 0) break;
        got += (size_t)k;
      }
      if (got < want) {
        errs[r] = "file ended early or could not be read";
        failed = 1;
        break;
      }
      if (cudaMemcpyAsync(dst + at, sg->buf[r][slot], want, cudaMemcpyHostToDevice, sg->st[r]) != cudaSuccess ||
          cudaEventRecord(sg->ev[r][slot], sg->st[r]) != cudaSuccess) {
        errs[r] = "staging copy failed";
        failed = 1;
        break;
      }
      used[slot] = true;
      slot ^= 1;
    }
    if (cudaStreamSynchronize(sg->st[r]) != cudaSuccess && errs[r].empty()) {
      errs[r] = "staging copy failed";
      failed = 1;
    }
  };
  std::vector<std::thread> th;
  for (int r = 1; r < nr; ++r) th.emplace_back(reader, r);
  reader(0);
  for (auto& x : th) x.join();
  if (failed) {
    for (auto& e : errs)
      if (!e.empty()) {
        set_error("%s", e.c_str());
        break;
      }
    return ALTO_ERR_INVALID;
  }
  return ALTO_OK;
}

// The line of the file starting at `start`, up to and including its newline
// (or to the end of the file), as getline returns it.
alto_status read_line(int fd, uint64_t start, uint64_t size, std::string* out) {
  out->clear();
  char chunk[4096];
  for (uint64_t at = start; at < size;) {
    const size_t want = (size_t)std::min<uint64_t>(sizeof(chunk), size - at);
    const ssize_t r = pread(fd, chunk, want, (off_t)at);
    if (r <= 0) {
      set_error("could not re-read a line of the file");
      return ALTO_ERR_INVALID;
    }
    const char* nl = static_cast<const char*>(memchr(chunk, '\n', (size_t)r));
    if (nl) {
      out->append(chunk, (size_t)(nl - chunk) + 1);
      return ALTO_OK;
    }
    out->append(chunk, (size_t)r);
    at += (uint64_t)r;
  }
  return ALTO_OK;
}

// The reference's strtok count on the first valid line, minus one.
int count_modes(std::string line) {
  line = line.substr(0, strnlen(line.c_str(), line.size()));
  int n = 0;
  bool in = false;
  for (char c : line) {
    const bool delim = c == ' ' || c == '\t';
    if (!delim && !in) ++n;
    in = !delim;
  }
  return n - 1;
}

alto_status read_text(int fd, uint64_t size, uint64_t zero_based, cudaStream_t st, alto_dcoo* d) {
  if (size >= (1ull << 33)) {  // (line slots are counted in 32 bits: a valid line has two bytes or more)
    set_error("text files of 8 GiB or more are not supported");
    return ALTO_ERR_UNSUPPORTED;
  }
  const uint64_t ntiles = (size + kIoTile - 1) / kIoTile;
  PoolBuf file, starts;  // (transient: the library pool keeps them for the next read)
  DevBuf tiles, scan_scratch, misc;
  ALTO_TRY(file.ensure(ntiles * kIoTile + 16, st));
  const double t0 = now_ms();
  ALTO_TRY_CUDA(cudaMemsetAsync(file.as<char>() + size, 0, ntiles * kIoTile + 16 - size, st));
  ALTO_TRY_CUDA(cudaStreamSynchronize(st));  // the padding is cleared before the readers copy
  ALTO_TRY(stream_file(fd, 0, size, file.as<char>()));
  d->read_ms = now_ms() - t0;

  // device time of the parse: the kernels' spans, without the host work and
  // allocations between them
  cudaEvent_t ev[6] = {};
  struct EvGuard {
    cudaEvent_t* e;
    ~EvGuard() {
      for (int i = 0; i < 6; ++i)
        if (e[i]) cudaEventDestroy(e[i]);
    }
  } evg{ev};
  for (int i = 0; i < 6; ++i) ALTO_TRY_CUDA(cudaEventCreate(&ev[i]));
  ALTO_TRY_CUDA(cudaEventRecord(ev[0], st));
  ALTO_TRY(tiles.ensure((ntiles + 1) * 4));
  tns_count_kernel<<<(unsigned)ntiles, kIoThreads, 0, st>>>(file.as<uint4>(), size, tiles.as<uint32_t>());
  ALTO_LAUNCHED();
  ALTO_TRY_CUDA(cudaMemsetAsync(tiles.as<uint32_t>() + ntiles, 0, 4, st));
  ALTO_TRY(exclusive_scan_u32(tiles.as<uint32_t>(), ntiles + 1, scan_scratch, st));
  ALTO_TRY_CUDA(cudaEventRecord(ev[1], st));
  uint32_t nl = 0;
  ALTO_TRY_CUDA(cudaMemcpyAsync(&nl, tiles.as<uint32_t>() + ntiles, 4, cudaMemcpyDeviceToHost, st));
  ALTO_TRY_CUDA(cudaStreamSynchronize(st));
  const uint64_t nnz = nl;
  if (nnz == 0) {
    set_error("no nonzero lines in the file (the reference asserts)");
    return ALTO_ERR_INVALID;
  }
  ALTO_TRY(starts.ensure(nnz * 8, st));
  ALTO_TRY_CUDA(cudaEventRecord(ev[2], st));
  tns_starts_kernel<<<(unsigned)ntiles, kIoThreads, 0, st>>>(file.as<uint4>(), size, tiles.as<uint32_t>(),
                                                              starts.as<uint64_t>());
  ALTO_LAUNCHED();
  ALTO_TRY_CUDA(cudaEventRecord(ev[3], st));
  // the first valid line, on the host, for the mode count
  uint64_t s0 = 0;
  ALTO_TRY_CUDA(cudaMemcpyAsync(&s0, starts.p, 8, cudaMemcpyDeviceToHost, st));
  ALTO_TRY_CUDA(cudaStreamSynchronize(st));
  std::string first;
  ALTO_TRY(read_line(fd, s0, size, &first));
  const int N = count_modes(first);
  if (N < 1 || N > ALTO_MAX_MODES) {
    set_error("the first line gives %d modes (1..%d supported)", N, ALTO_MAX_MODES);
    return N < 1 ? ALTO_ERR_INVALID : ALTO_ERR_UNSUPPORTED;
  }
  ALTO_TRY(misc.ensure(64 + 8 * ALTO_MAX_MODES));
  uint32_t* host_count = misc.as<uint32_t>();
  unsigned long long* ddims = reinterpret_cast<unsigned long long*>(misc.as<char>() + 64);
  ALTO_TRY_CUDA(cudaMemsetAsync(misc.p, 0, 64 + 8 * ALTO_MAX_MODES, st));
  ALTO_TRY(d->raw.ensure((uint64_t)(N + 1) * nnz * 8));
  uint64_t* idx = d->raw.as<uint64_t>();
  double* vals = reinterpret_cast<double*>(idx + (uint64_t)N * nnz);
  // lines whose value the host converts: room for 2^20, a rerun with room
  // for every line when more turn up
  uint32_t cap = (uint32_t)std::min<uint64_t>(nnz, 1u << 20);
  PoolBuf hl;
  ALTO_TRY(hl.ensure((uint64_t)cap * 16, st));
  ALTO_TRY_CUDA(cudaEventRecord(ev[4], st));
  ALTO_TRY(launch_parse(grid_io(nnz, kIoThreads), st, file.as<unsigned char>(), size, starts.as<uint64_t>(), nnz, N,
                        zero_based, idx, vals, ddims, hl.as<uint64_t>(), cap, host_count));
  ALTO_TRY_CUDA(cudaEventRecord(ev[5], st));
  uint32_t nhost = 0;
  ALTO_TRY_CUDA(cudaMemcpyAsync(d->dims, ddims, 8 * N, cudaMemcpyDeviceToHost, st));
  ALTO_TRY_CUDA(cudaMemcpyAsync(&nhost, host_count, 4, cudaMemcpyDeviceToHost, st));
  ALTO_TRY_CUDA(cudaStreamSynchronize(st));
  float pm[3] = {0, 0, 0};
  for (int i = 0; i < 3; ++i) cudaEventElapsedTime(&pm[i], ev[2 * i], ev[2 * i + 1]);
  d->parse_ms = (double)pm[0] + pm[1] + pm[2];
  if (nhost > cap) {  // every listed line again, with room for all
    cap = (uint32_t)nnz;
    ALTO_TRY(hl.ensure((uint64_t)cap * 16, st));
    ALTO_TRY_CUDA(cudaMemsetAsync(misc.p, 0, 64 + 8 * ALTO_MAX_MODES, st));
    ALTO_TRY(launch_parse(grid_io(nnz, kIoThreads), st, file.as<unsigned char>(), size, starts.as<uint64_t>(), nnz,
                          N, zero_based, idx, vals, ddims, hl.as<uint64_t>(), cap, host_count));
    ALTO_TRY_CUDA(cudaMemcpyAsync(&nhost, host_count, 4, cudaMemcpyDeviceToHost, st));
    ALTO_TRY_CUDA(cudaStreamSynchronize(st));
  }
  d->host_lines = nhost;
  if (nhost) {  // values the device left to the C library, in chunks of up to 4M
    const uint32_t chunk = std::min<uint32_t>(nhost, 1u << 22);
    PoolBuf txt, hb;
    ALTO_TRY(txt.ensure((size_t)chunk * kValText, st));
    ALTO_TRY(hb.ensure((size_t)chunk * 12, st));
    std::vector<char> htxt((size_t)chunk * kValText);
    std::vector<uint64_t> list(2 * (size_t)chunk);
    std::vector<uint32_t> at(chunk);
    std::vector<double> v(chunk);
    const unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    for (uint32_t i0 = 0; i0 < nhost; i0 += chunk) {
      const uint32_t n = std::min(chunk, nhost - i0);
      value_text_kernel<<<grid_io(n, 256), 256, 0, st>>>(hl.as<uint64_t>(), i0, n, starts.as<uint64_t>(),
                                                         file.as<unsigned char>(), size, txt.as<char>());
      ALTO_LAUNCHED();
      ALTO_TRY_CUDA(cudaMemcpyAsync(htxt.data(), txt.p, (size_t)n * kValText, cudaMemcpyDeviceToHost, st));
      ALTO_TRY_CUDA(cudaMemcpyAsync(list.data(), hl.as<uint64_t>() + 2 * (size_t)i0, (size_t)n * 16,
                                    cudaMemcpyDeviceToHost, st));
      ALTO_TRY_CUDA(cudaStreamSynchronize(st));
      // the C library's strtod on every listed text, on all host cores
      std::vector<std::thread> th;
      for (unsigned r = 0; r < nt; ++r)
        th.emplace_back([&, r] {
          for (uint32_t i = r; i < n; i += nt) {
            at[i] = (uint32_t)list[2 * (size_t)i];
            const char* tx = htxt.data() + (size_t)i * kValText;
            v[i] = tx[kValText - 1] ? 0.0 : strtod(tx, nullptr);
          }
        });
      for (auto& x : th) x.join();
      // texts longer than a slot: the whole line again from the file
      std::string line;
      for (uint32_t i = 0; i < n; ++i) {
        if (!htxt[(size_t)i * kValText + kValText - 1]) continue;
        uint64_t ls = 0;
        ALTO_TRY_CUDA(cudaMemcpyAsync(&ls, starts.as<uint64_t>() + at[i], 8, cudaMemcpyDeviceToHost, st));
        ALTO_TRY_CUDA(cudaStreamSynchronize(st));
        ALTO_TRY(read_line(fd, ls, size, &line));
        const size_t o = (size_t)list[2 * (size_t)i + 1];
        v[i] = o <= line.size() ? strtod(line.c_str() + o, nullptr) : 0.0;
      }
      ALTO_TRY_CUDA(cudaMemcpyAsync(hb.p, v.data(), (size_t)n * 8, cudaMemcpyHostToDevice, st));
      ALTO_TRY_CUDA(cudaMemcpyAsync(hb.as<char>() + (size_t)chunk * 8, at.data(), (size_t)n * 4,
                                    cudaMemcpyHostToDevice, st));
      scatter_vals_kernel<<<grid_io(n, 256), 256, 0, st>>>(
          reinterpret_cast<const uint32_t*>(hb.as<char>() + (size_t)chunk * 8), hb.as<double>(), n, vals);
      ALTO_LAUNCHED();
      ALTO_TRY_CUDA(cudaStreamSynchronize(st));  // (v and at are refilled by the next chunk)
    }
  }
  d->nmodes = N;
  d->nnz = nnz;
  return ALTO_OK;
}

alto_status read_binary(int fd, uint64_t size, cudaStream_t st, alto_dcoo* d) {
  uint64_t nm = 0;
  if (size >= 8 && pread(fd, &nm, 8, 0) == 8 && (nm >> 32) && (nm & 0xffffffffull) <= ALTO_MAX_MODES)
    nm &= 0xffffffffull;  // the reference writes its int nmodes as 8 bytes (src/sptensor.cpp:59): the
                          // upper half is whatever followed the int in memory
  if (size < 8 || nm < 1 || nm > ALTO_MAX_MODES) {
    set_error("binary header: bad mode count");
    return ALTO_ERR_INVALID;
  }
  uint64_t head[ALTO_MAX_MODES + 1];
  if (pread(fd, head, 8 * (nm + 1), 8) != (ssize_t)(8 * (nm + 1))) {
    set_error("binary header is short");
    return ALTO_ERR_INVALID;
  }
  const uint64_t nnz = head[nm];
  const uint64_t body = 8 * (nm + 2);
  if (nnz == 0 || nnz >= (1ull << 32) || size < body + (nm + 1) * nnz * 8) {
    set_error("binary file: nnz %llu does not match the file size", (unsigned long long)nnz);
    return nnz >= (1ull << 32) ? ALTO_ERR_UNSUPPORTED : ALTO_ERR_INVALID;
  }
  ALTO_TRY(d->raw.ensure((nm + 1) * nnz * 8));
  const double t0 = now_ms();
  ALTO_TRY(stream_file(fd, body, (nm + 1) * nnz * 8, d->raw.as<char>()));
  d->read_ms = now_ms() - t0;
  d->nmodes = (int)nm;
  d->nnz = nnz;
  for (uint64_t m = 0; m < nm; ++m) d->dims[m] = head[m];
  return ALTO_OK;
}

// "%g" of v as glibc prints it.
void put_g(std::string& out, double v) {
  if (std::isfinite(v) && v == std::floor(v) && std::fabs(v) < 1e6) {
    if (v == 0) {
      out += std::signbit(v) ? "-0" : "0";
      return;
    }
    long long i = (long long)v;
    char b[24];
    int n = 0;
    const bool neg = i < 0;
    unsigned long long u = neg ? (unsigned long long)(-i) : (unsigned long long)i;
    while (u) {
      b[n++] = (char)('0' + u % 10);
      u /= 10;
    }
    if (neg) out += '-';
    while (n) out += b[--n];
    return;
  }
  char b[64];
  snprintf(b, sizeof(b), "%g", v);
  out += b;
}

void put_u64(std::string& out, uint64_t u) {
  char b[24];
  int n = 0;
  do {
    b[n++] = (char)('0' + u % 10);
    u /= 10;
  } while (u);
  while (n) out += b[--n];
}

}  // namespace

extern "C" {

alto_status alto_read_tensor(const char* path, alto_file_format format, int zero_based, alto_cuda_stream stream,
                             alto_dcoo** out) {
  if (!path || !out || (format != ALTO_FILE_TEXT && format != ALTO_FILE_BINARY)) {
    set_error("bad path, format or out");
    return ALTO_ERR_INVALID;
  }
  *out = nullptr;
  const int fd = open(path, O_RDONLY);
  if (fd < 0) {
    set_error("cannot open %s", path);
    return ALTO_ERR_INVALID;
  }
  struct stat sb;
  if (fstat(fd, &sb) != 0 || sb.st_size == 0) {
    close(fd);
    set_error("%s is empty or cannot be read", path);
    return ALTO_ERR_INVALID;
  }
  alto_dcoo* d = new (std::nothrow) alto_dcoo();
  if (!d) {
    close(fd);
    set_error("host allocation failed");
    return ALTO_ERR_NOMEM;
  }
  d->file_bytes = (uint64_t)sb.st_size;
  cudaStream_t st = (cudaStream_t)stream;
  alto_status r = format == ALTO_FILE_TEXT ? read_text(fd, (uint64_t)sb.st_size, zero_based ? 1 : 0, st, d)
                                           : read_binary(fd, (uint64_t)sb.st_size, st, d);
  close(fd);
  if (r != ALTO_OK) {
    cudaStreamSynchronize(st);
    delete d;
    return r;
  }
  for (int m = 0; m < d->nmodes; ++m) d->ptrs[m] = d->raw.as<uint64_t>() + (uint64_t)m * d->nnz;
  *out = d;
  return ALTO_OK;
}

alto_status alto_dcoo_view(const alto_dcoo* d, alto_coo* view) {
  if (!d || !view) {
    set_error("tensor or view is NULL");
    return ALTO_ERR_INVALID;
  }
  view->nmodes = d->nmodes;
  view->dims = d->dims;
  view->nnz = d->nnz;
  view->cidx = d->ptrs;
  view->index_bytes = 8;
  view->vals = d->raw.as<uint64_t>() + (uint64_t)d->nmodes * d->nnz;
  view->val_dtype = ALTO_F64;
  view->on_device = 1;
  return ALTO_OK;
}

alto_status alto_dcoo_stats(const alto_dcoo* d, double* read_ms, double* parse_ms, uint64_t* file_bytes,
                            uint64_t* host_values) {
  if (!d) {
    set_error("tensor is NULL");
    return ALTO_ERR_INVALID;
  }
  if (read_ms) *read_ms = d->read_ms;
  if (parse_ms) *parse_ms = d->parse_ms;
  if (file_bytes) *file_bytes = d->file_bytes;
  if (host_values) *host_values = d->host_lines;
  return ALTO_OK;
}

alto_status alto_dcoo_to_host(const alto_dcoo* d, uint64_t* cidx, double* vals) {
  if (!d) {
    set_error("tensor is NULL");
    return ALTO_ERR_INVALID;
  }
  const uint64_t n = d->nnz, N = (uint64_t)d->nmodes;
  if (cidx) ALTO_TRY_CUDA(cudaMemcpy(cidx, d->raw.p, N * n * 8, cudaMemcpyDeviceToHost));
  if (vals) ALTO_TRY_CUDA(cudaMemcpy(vals, d->raw.as<uint64_t>() + N * n, n * 8, cudaMemcpyDeviceToHost));
  return ALTO_OK;
}

alto_status alto_dcoo_destroy(alto_dcoo* d) {
  delete d;
  return ALTO_OK;
}

alto_status alto_write_tensor(const char* path, alto_file_format format, const alto_coo* coo) {
  if (!path || (format != ALTO_FILE_TEXT && format != ALTO_FILE_BINARY)) {
    set_error("bad path or format");
    return ALTO_ERR_INVALID;
  }
  ALTO_TRY(check_coo_shape(coo));
  if (coo->nnz == 0) {
    set_error("empty tensor (the reference asserts nnz > 0)");
    return ALTO_ERR_INVALID;
  }
  const int N = coo->nmodes;
  const uint64_t nnz = coo->nnz;
  // host copies: uint64 indices, float64 values
  std::vector<std::vector<uint64_t>> ci(N, std::vector<uint64_t>(nnz));
  std::vector<double> v(nnz);
  for (int m = 0; m < N; ++m) {
    if (coo->index_bytes == 8 && coo->on_device) {
      ALTO_TRY_CUDA(cudaMemcpy(ci[m].data(), coo->cidx[m], nnz * 8, cudaMemcpyDeviceToHost));
    } else if (coo->index_bytes == 8) {
      memcpy(ci[m].data(), coo->cidx[m], nnz * 8);
    } else {
      std::vector<uint32_t> t(nnz);
      if (coo->on_device)
        ALTO_TRY_CUDA(cudaMemcpy(t.data(), coo->cidx[m], nnz * 4, cudaMemcpyDeviceToHost));
      else
        memcpy(t.data(), coo->cidx[m], nnz * 4);
      for (uint64_t i = 0; i < nnz; ++i) ci[m][i] = t[i];
    }
  }
  if (coo->val_dtype == ALTO_F64) {
    if (coo->on_device)
      ALTO_TRY_CUDA(cudaMemcpy(v.data(), coo->vals, nnz * 8, cudaMemcpyDeviceToHost));
    else
      memcpy(v.data(), coo->vals, nnz * 8);
  } else {
    std::vector<float> t(nnz);
    if (coo->on_device)
      ALTO_TRY_CUDA(cudaMemcpy(t.data(), coo->vals, nnz * 4, cudaMemcpyDeviceToHost));
    else
      memcpy(t.data(), coo->vals, nnz * 4);
    for (uint64_t i = 0; i < nnz; ++i) v[i] = t[i];
  }
  FILE* f = fopen(path, "wb");
  if (!f) {
    set_error("cannot create %s", path);
    return ALTO_ERR_INVALID;
  }
  bool ok = true;
  if (format == ALTO_FILE_BINARY) {
    const uint64_t nm = (uint64_t)N;
    ok = fwrite(&nm, 8, 1, f) == 1 && fwrite(coo->dims, 8, N, f) == (size_t)N && fwrite(&nnz, 8, 1, f) == 1;
    for (int m = 0; m < N && ok; ++m) ok = fwrite(ci[m].data(), 8, nnz, f) == nnz;
    ok = ok && fwrite(v.data(), 8, nnz, f) == nnz;
  } else {
    // format blocks of lines on all cores, write them in order
    const unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    const uint64_t block = 1 << 20;
    for (uint64_t b0 = 0; b0 < nnz && ok; b0 += block * nt) {
      std::vector<std::string> parts(nt);
      std::vector<std::thread> th;
      for (unsigned k = 0; k < nt; ++k) {
        const uint64_t lo = b0 + k * block, hi = std::min(nnz, lo + block);
        if (lo >= hi) break;
        th.emplace_back([&, k, lo, hi] {
          std::string& s = parts[k];
          s.reserve((hi - lo) * (8 * N + 12));
          for (uint64_t i = lo; i < hi; ++i) {
            for (int m = 0; m < N; ++m) {
              put_u64(s, ci[m][i] + 1);
              s += ' ';
            }
            put_g(s, v[i]);
            s += '\n';
          }
        });
      }
      for (auto& t : th) t.join();
      for (auto& s : parts) ok = ok && fwrite(s.data(), 1, s.size(), f) == s.size();
    }
  }
  ok = (fclose(f) == 0) && ok;
  if (!ok) {
    set_error("writing %s failed", path);
    return ALTO_ERR_INVALID;
  }
  return ALTO_OK;
}

}  // extern "C"
