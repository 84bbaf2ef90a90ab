// Internal declarations shared by the CUDA translation units of libalto_b200.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/alto_b200.h"

namespace alto {

// ------------------------------------------------------------------ errors

void set_error(const char* fmt, ...);
extern std::atomic<uint64_t> g_kernel_launches;

inline alto_status cuda_status(cudaError_t e, const char* what, const char* file, int line) {
  if (e == cudaSuccess) return ALTO_OK;
  set_error("%s: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
  return e == cudaErrorMemoryAllocation ? ALTO_ERR_NOMEM : ALTO_ERR_CUDA;
}

#define ALTO_TRY_CUDA(call)                                                   \
  do {                                                                        \
    alto_status s_ = ::alto::cuda_status((call), #call, __FILE__, __LINE__);  \
    if (s_ != ALTO_OK) return s_;                                             \
  } while (0)

#define ALTO_TRY(call)               \
  do {                               \
    alto_status s_ = (call);         \
    if (s_ != ALTO_OK) return s_;    \
  } while (0)

// Count and check a kernel launch.
#define ALTO_LAUNCHED()                                                        \
  do {                                                                         \
    ::alto::g_kernel_launches.fetch_add(1, std::memory_order_relaxed);         \
    ALTO_TRY_CUDA(cudaGetLastError());                                         \
  } while (0)

// ------------------------------------------------------------ device memory

// The stream on which this host thread allocates and frees device memory.
// Null (the default) means cudaMalloc / cudaFree; a stream means the
// stream-ordered allocator (cudaMallocAsync / cudaFreeAsync), which does not
// synchronise the device, so threads that work on their own streams (the
// serving workers) do not stall one another when buffers grow.
extern thread_local cudaStream_t tls_alloc_stream;

// A growable device allocation owned by a handle.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) {
      if (tls_alloc_stream)
        cudaFreeAsync(p, tls_alloc_stream);
      else
        cudaFree(p);
    }
    p = nullptr;
    bytes = 0;
  }
  // Ensure at least n bytes; contents are not preserved on growth.
  alto_status ensure(size_t n) {
    if (n <= bytes && p) return ALTO_OK;
    release();
    size_t want = n < 256 ? 256 : n;
    cudaError_t e = tls_alloc_stream ? cudaMallocAsync(&p, want, tls_alloc_stream) : cudaMalloc(&p, want);
    if (e != cudaSuccess) {
      p = nullptr;
      return cuda_status(e, "cudaMalloc", __FILE__, __LINE__);
    }
    bytes = want;
    return ALTO_OK;
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

// Transient device memory from a stream-ordered pool the library owns, one
// per device, which keeps what is freed for the next allocation (its memory
// stays reserved until the process exits).  For buffers that live within
// one call and are several GB: cudaMalloc / cudaFree of such sizes cost
// milliseconds each and cudaFree synchronises the device.  Freed in stream
// order on the stream given to ensure(); any other stream that used the
// buffer must be complete before release.
cudaMemPool_t transient_pool();
struct PoolBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaStream_t st = nullptr;
  PoolBuf() = default;
  PoolBuf(const PoolBuf&) = delete;
  PoolBuf& operator=(const PoolBuf&) = delete;
  ~PoolBuf() { release(); }
  void release() {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    bytes = 0;
  }
  // At least n bytes on stream s; contents are not preserved on growth.
  alto_status ensure(size_t n, cudaStream_t s) {
    if (n <= bytes && p && s == st) return ALTO_OK;
    release();
    cudaMemPool_t pool = transient_pool();
    if (!pool) return cuda_status(cudaErrorInvalidDevice, "transient pool", __FILE__, __LINE__);
    st = s;
    const size_t want = n < 256 ? 256 : n;
    cudaError_t e = cudaMallocFromPoolAsync(&p, want, pool, s);
    if (e != cudaSuccess) {
      p = nullptr;
      return cuda_status(e, "cudaMallocFromPoolAsync", __FILE__, __LINE__);
    }
    bytes = want;
    return ALTO_OK;
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

// ------------------------------------------------------------- ALTO keys

struct Key2 {
  uint64_t lo, hi;
};

// Per-mode bit fields of the mode-contiguous ("line") key: mode m occupies
// bits [pos[m], pos[m] + bits[m]) of a 128-bit word stored as a 64-bit low
// part plus, when the fields need more than 64 bits, a 32- or 64-bit high
// part.  This is the reference's ALT_PEXT layout (include/alto.hpp:541-573,
// mode_pos at :982-988) split into separately streamed words.
struct LineDecode {
  int nmodes;
  int hi_words;    // 0: no high part; 1: uint32 high part; 2: uint64 high part
  int pos[ALTO_MAX_MODES];
  uint64_t mask[ALTO_MAX_MODES];  // (1 << bits) - 1
};

// Entries of padding after every line array, so that bulk copies rounded
// up to 16 bytes stay inside the allocation.
constexpr uint64_t kLinePad = 16;

// One line record per nonzero: the mode-contiguous key and the value, read
// with one 16-byte load when the key fits 96 bits (hi_words <= 1):
//   {key bits 0..63, key bits 64..95, value}
// and with two when it needs up to 128 bits (hi_words == 2):
//   {key bits 0..63, key bits 64..127, value, 12 bytes of padding}.
struct __align__(16) LineRec16 {
  uint64_t lo;
  uint32_t hi;
  float v;
};
struct __align__(16) LineRec32 {
  uint64_t lo;
  uint64_t hi;
  float v;
  uint32_t pad[3];
};

// Record format code 3: a 3-mode record with the rows stored decoded,
// {row of mode 0, row of mode 1, row of mode 2, value} (16 bytes); used for
// the row-sorted copies of 3-mode lines, where the kernels then skip the
// bit-field decode.
constexpr int kDecoded3 = 3;

__host__ __device__ __forceinline__ int rec_bytes(int hi_words) { return hi_words == 2 ? 32 : 16; }

// Read record i of a line with any key width.
__device__ __forceinline__ void rec_read(const void* line, int hi_words, uint64_t i, uint64_t& lo,
                                         uint64_t& hi, float& v) {
  if (hi_words == 2) {
    const LineRec32 r = static_cast<const LineRec32*>(line)[i];
    lo = r.lo;
    hi = r.hi;
    v = r.v;
  } else {
    const uint4 q = static_cast<const uint4*>(line)[i];
    lo = (uint64_t)q.x | ((uint64_t)q.y << 32);
    hi = q.z;
    v = __uint_as_float(q.w);
  }
}

__device__ __forceinline__ void rec_write(void* line, int hi_words, uint64_t i, uint64_t lo, uint64_t hi,
                                          float v) {
  if (hi_words == 2) {
    LineRec32 r;
    r.lo = lo;
    r.hi = hi;
    r.v = v;
    r.pad[0] = r.pad[1] = r.pad[2] = 0;
    static_cast<LineRec32*>(line)[i] = r;
  } else {
    static_cast<uint4*>(line)[i] =
        make_uint4((uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi, __float_as_uint(v));
  }
}

// Field of mode-contiguous key (lo, hi) at bit pos with the given mask; hi is
// 0 when the key has no high part.
__device__ __forceinline__ uint64_t line_field(uint64_t lo, uint64_t hi, int pos, uint64_t mask) {
  if (pos >= 64) return (hi >> (pos - 64)) & mask;
  uint64_t v = lo >> pos;
  if (pos > 0) v |= hi << (64 - pos);
  return v & mask;
}

// --------------------------------------------------------------- scans

// Exclusive prefix sum of n uint32 counts in place (device), stream-ordered.
alto_status exclusive_scan_u32(uint32_t* data, size_t n, DevBuf& scratch, cudaStream_t st);

}  // namespace alto

// ------------------------------------------------------------- the handle

namespace alto {
// A copy of the line ordered by one mode's row (see build_sorted_line).
struct SortedLine {
  DevBuf line, tile_iv;
  int hw = 0;  // record format: the line's hi_words, or kDecoded3
  uint32_t ntiles = 0;
  uint64_t for_nnz = 0;
  bool ready = false;
};

// Tuned MTTKRP choice per (mode, rank, factor dtype).
struct TuneEntry {
  int mode, rank, fdtype;
  alto_mttkrp_variant variant;
  int feed;  // 0 direct, 1 line streamed through shared memory by bulk copy, 2 direct at five blocks per SM,
             // 3 as 2 with the target mode fixed at compile time
};
}  // namespace alto

struct alto_tensor {
  int nmodes = 0;
  int nprtn = 1;
  int stream_mode = -1;
  int key_bits = 64;   // width of the reference key type (64 or 128)
  int alto_bits = 0;   // bits the masks use
  uint64_t nnz = 0;
  uint64_t cap = 0;    // capacity of the per-nonzero device arrays
  uint64_t dims[ALTO_MAX_MODES] = {0};
  alto::Key2 masks[ALTO_MAX_MODES] = {};
  alto::Key2 alto_mask = {0, 0};
  int mode_bits[ALTO_MAX_MODES] = {0};
  alto::LineDecode dec = {};

  // The line: per nonzero, one record (mode-contiguous key and value, see
  // LineRec16 / LineRec32) in ALTO (bit-interleaved key) order.
  alto::DevBuf line;   // records [cap + kLinePad]
  alto::DevBuf perm;   // uint32  [cap]: input position of each line entry

  // Tiles of the line used by the MTTKRP kernels: tile t covers
  // [t * tile_nnz, min((t+1) * tile_nnz, nnz)); tile_iv holds, per tile and
  // mode, the first row and the row count of its interval.
  uint32_t tile_nnz = 4096;
  uint32_t ntiles = 0;
  alto::DevBuf tile_iv;  // uint32 [ntiles * nmodes * 2]

  // The reference's partitions (prtn_ptr / prtn_intervals).
  std::vector<uint64_t> prtn_ptr;
  alto::DevBuf prtn_iv;  // uint64 [nprtn * nmodes * 2]

  // Row-sorted copies of the line, built on first use per mode.
  alto::SortedLine sorted[ALTO_MAX_MODES];
  // Per mode, the tiles' interval lengths in ascending order (host copy),
  // used to decide whether per-tile shared-memory staging can pay off.
  std::vector<uint32_t> tile_len_sorted[ALTO_MAX_MODES];
  // Variants chosen by alto_mttkrp_autotune, per (mode, rank, dtype).
  std::vector<alto::TuneEntry> tuned;
  // Whether encoding collects tile_len_sorted (a host copy and a
  // synchronisation; only ALTO_MTTKRP_AUTO's rule reads it -- CP-stream
  // sessions, which always run the deterministic variant, skip it).
  bool tile_stats = true;
  // Whether the per-nonzero buffers grow by half again past a request (a
  // session's tensor, re-encoded slice after slice: slices of varying
  // sizes then reallocate rarely).
  bool grow = false;

  // Device error word of the kernels' bounded waits (0 = none).
  alto::DevBuf err;

  // Deterministic MTTKRP: sub-range boundary slots (rows, partial sums) and
  // the list of long chains with its count.
  alto::DevBuf det_rows, det_vals, det_long;

  // Construction scratch (sort buffers, scan partials).
  alto::DevBuf scratch;
  alto::DevBuf scan_scratch;
  cudaStream_t stream = nullptr;
};

namespace alto {
// At least n bytes in b, with t->grow's headroom.
inline alto_status tensor_ensure(const alto_tensor* t, DevBuf& b, size_t n) {
  if (n <= b.bytes && b.p) return ALTO_OK;
  return b.ensure(t->grow ? std::max(n, b.bytes + b.bytes / 2) : n);
}

// Encode (linearise, sort, lay out, partition) a COO tensor into t.
alto_status encode_tensor(alto_tensor* t, const alto_coo* coo, int nprtn, cudaStream_t st);
// Stable one-sweep LSD radix sort of (key, uint32 payload) pairs
// (alto_encode.cu); scratch of radix_scratch_bytes(n) bytes; *err (device)
// is set if a look-back gave up.
alto_status radix_sort_pairs(uint64_t* klo[2], uint64_t* khi[2], uint32_t* pm[2], uint32_t n, int bits,
                             void* scratch, int* err, cudaStream_t st, int* cur_out);
size_t radix_scratch_bytes(uint64_t n);
// Device error words of a tensor (t->err, four ints): [0] a bulk-feed
// MTTKRP wait gave up, [kSortErrorWord] a radix-sort look-back gave up.
constexpr int kSortErrorWord = 3;
alto_status ensure_error_words(alto_tensor* t, cudaStream_t st);
// ALTO_ERR_TIMEOUT (and the word cleared) if words[kSortErrorWord] is set.
alto_status sort_error_status(alto_tensor* t, const int* words, cudaStream_t st);
// Keep line entries [begin, end) and rebuild tiles, intervals, partitions.
alto_status restrict_line(alto_tensor* t, uint64_t begin, uint64_t end, cudaStream_t st);
// Host-side mask setup (setup_packed_alto).
int setup_masks(int nmodes, const uint64_t* dims, int max_bits, Key2* masks, Key2* alto_mask,
                int* bits);
// MTTKRP dispatcher.
alto_status run_mttkrp(alto_tensor* t, int mode, const void* const* factors, alto_dtype fdtype,
                       int rank, float* out, int accumulate, alto_mttkrp_variant variant,
                       cudaStream_t st);
alto_status run_mttkrp_feed(alto_tensor* t, int mode, const void* const* factors, alto_dtype fdtype,
                            int rank, float* out, int accumulate, alto_mttkrp_variant variant, int feed,
                            cudaStream_t st);
alto_mttkrp_variant choose_variant(const alto_tensor* t, int mode, int rank, alto_dtype fdtype);
// Whether ALTO_MTTKRP_DETERMINISTIC runs for this rank and factor type.
bool deterministic_supported(int rank, alto_dtype fdtype);
// Build the per-mode row-sorted copy of the line.
alto_status build_sorted_line(alto_tensor* t, int mode, cudaStream_t st);
// Measure the variants per mode and record the fastest (synchronous).
alto_status autotune(alto_tensor* t, const void* const* factors, alto_dtype fdtype, int rank,
                     cudaStream_t st, alto_mttkrp_variant* chosen);
}  // namespace alto
