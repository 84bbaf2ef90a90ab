// ALTO encoding on the device: linearisation, radix sort, line layout and
// partition intervals.
//
// Reference behaviour (jeewhanchoi/ALTO-stream):
//   setup_packed_alto(LSB_FIRST, SHORT_FIRST)  include/alto.hpp:955-1057
//   linearisation (PDEP per mode)              include/alto.hpp:513-533, 239-252
//   sort_alto (std::sort by key)               include/alto.hpp:1066-1090
//   ALT_PEXT re-encoding                       include/alto.hpp:541-573
//   prtn_alto (partitions, intervals)          include/alto.hpp:1128-1226
//
// The device pipeline: (1) every nonzero's bit-interleaved key is built by
// depositing each mode index into its mask bits; (2) an LSD radix sort
// (8-bit digits, stable, over only the bits the masks use) orders keys with
// the input position as payload -- keys are unique for unique coordinates,
// so the order equals std::sort's; (3) one pass extracts each mode's index
// from the sorted key, packs it into the mode-contiguous line key and
// gathers the value; (4) per-tile and per-partition interval reductions.
#include <algorithm>
#include <cstring>

#include "alto_internal.cuh"

namespace alto {

// ------------------------------------------------------- host mask setup

static int bits_for(uint64_t dim) {
  if (dim <= 1) return 0;  // clz(0) = 64 on LZCNT hardware: a length-1 mode takes no bits
  return 64 - __builtin_clzll(dim - 1);
}

// setup_packed_alto, include/alto.hpp:955-1057: modes ordered by bit count
// (stable), bits dealt LSB first round-robin over the modes still active at
// each level.  Returns the total bits or -1 when they exceed max_bits.
int setup_masks(int nmodes, const uint64_t* dims, int max_bits, Key2* masks, Key2* alto_mask,
                int* bits) {
  int order[ALTO_MAX_MODES];
  int total = 0;
  for (int n = 0; n < nmodes; ++n) {
    bits[n] = bits_for(dims[n]);
    order[n] = n;
    total += bits[n];
    masks[n] = {0, 0};
  }
  if (total > max_bits) return -1;
  std::stable_sort(order, order + nmodes, [&](int a, int b) { return bits[a] < bits[b]; });
  int shift = 0;
  for (int level = 0;; ++level) {
    bool any = false;
    for (int k = 0; k < nmodes; ++k) {
      int n = order[k];
      if (level < bits[n]) {
        if (shift < 64)
          masks[n].lo |= 1ull << shift;
        else
          masks[n].hi |= 1ull << (shift - 64);
        ++shift;
        any = true;
      }
    }
    if (!any) break;
  }
  *alto_mask = {0, 0};
  for (int n = 0; n < nmodes; ++n) {
    alto_mask->lo |= masks[n].lo;
    alto_mask->hi |= masks[n].hi;
  }
  return total;
}

// ------------------------------------------------------------- kernels

struct MaskSet {
  int nmodes;
  uint64_t lo[ALTO_MAX_MODES];
  uint64_t hi[ALTO_MAX_MODES];
};

// PDEP: scatter the low bits of x into the set bits of (mlo, mhi).
__device__ __forceinline__ void deposit(uint64_t x, uint64_t mlo, uint64_t mhi, uint64_t& klo,
                                        uint64_t& khi) {
  while (mlo) {
    int b = __ffsll((long long)mlo) - 1;
    klo |= (x & 1ull) << b;
    x >>= 1;
    mlo &= mlo - 1;
  }
  while (mhi) {
    int b = __ffsll((long long)mhi) - 1;
    khi |= (x & 1ull) << b;
    x >>= 1;
    mhi &= mhi - 1;
  }
}

// PEXT: gather the bits of (klo, khi) selected by (mlo, mhi) into the low bits.
__device__ __forceinline__ uint64_t extract(uint64_t klo, uint64_t khi, uint64_t mlo,
                                            uint64_t mhi) {
  uint64_t r = 0;
  int k = 0;
  while (mlo) {
    int b = __ffsll((long long)mlo) - 1;
    r |= ((klo >> b) & 1ull) << k;
    ++k;
    mlo &= mlo - 1;
  }
  while (mhi) {
    int b = __ffsll((long long)mhi) - 1;
    r |= ((khi >> b) & 1ull) << k;
    ++k;
    mhi &= mhi - 1;
  }
  return r;
}

struct CooPtrs {
  const void* cidx[ALTO_MAX_MODES];
};

// Key of nonzero i = OR over modes of PDEP(cidx[m][i], mask[m]).
template <int IB>
__global__ void linearize_kernel(CooPtrs coo, MaskSet ms, uint32_t nnz, uint64_t* __restrict__ klo,
                                 uint64_t* __restrict__ khi, uint32_t* __restrict__ perm) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += gridDim.x * blockDim.x) {
    uint64_t lo = 0, hi = 0;
#pragma unroll
    for (int m = 0; m < ALTO_MAX_MODES; ++m) {
      if (m < ms.nmodes) {
        uint64_t x = IB == 8 ? ((const uint64_t*)coo.cidx[m])[i]
                             : (uint64_t)((const uint32_t*)coo.cidx[m])[i];
        deposit(x, ms.lo[m], ms.hi[m], lo, hi);
      }
    }
    klo[i] = lo;
    if (khi) khi[i] = hi;
    perm[i] = i;
  }
}

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;

__device__ __forceinline__ uint32_t digit_of(const uint64_t* klo, const uint64_t* khi, uint32_t i,
                                             int shift) {
  uint64_t w = shift >= 64 ? khi[i] : klo[i];
  return (uint32_t)(w >> (shift & 63)) & (kRadix - 1);
}

// One-sweep LSD radix sort.  The digit counts of every pass come from one
// read of the keys (radix_all_hist_kernel; radix_offsets_kernel turns them
// into each digit's start in the array).  A pass is then one kernel: a block
// takes the next tile in order (a ticket), ranks its pairs by digit,
// publishes its per-digit counts, and finds each digit's start among the
// preceding tiles by looking back over their published words (decoupled
// look-back): an aggregate (that tile's count) or an inclusive prefix (the
// count of all tiles up to it), so the walk stops at the first prefix.  Each
// pass reads and writes the pairs once.
constexpr int kMaxSortPasses = 16;  // 128-bit keys in 8-bit digits
constexpr unsigned long long kLbAggregate = 1ull << 62;
constexpr unsigned long long kLbPrefix = 2ull << 62;
constexpr uint32_t kLookbackSpins = 1u << 22;  // polls of an unpublished word before giving up
constexpr int kLookbackBatch = 8;               // look-back words loaded together

// Digit counts of every pass, ghist[pass * kRadix + digit] (atomically
// accumulated; zeroed by the caller), in shared memory first.  A warp whose
// lanes all hold one digit (the high digits of keys take few values) adds
// it once.
__global__ void __launch_bounds__(kSortThreads)
    radix_all_hist_kernel(const uint64_t* __restrict__ klo, const uint64_t* __restrict__ khi, uint32_t n,
                          int npass, uint32_t* __restrict__ ghist) {
  __shared__ uint32_t h[kMaxSortPasses * kRadix];
  for (int q = threadIdx.x; q < npass * kRadix; q += kSortThreads) h[q] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  for (uint32_t base = blockIdx.x * kSortThreads; base < n; base += gridDim.x * kSortThreads) {
    const uint32_t i = base + threadIdx.x;
    const bool valid = i < n;
    const unsigned vmask = __ballot_sync(0xffffffffu, valid);
    const uint64_t lo = valid ? klo[i] : 0, hi = (valid && khi) ? khi[i] : 0;
    if (valid) {
      const int leader = __ffs(vmask) - 1;
      for (int p = 0; p < npass; ++p) {
        const int shift = p * kRadixBits;
        const uint32_t d = (uint32_t)((shift >= 64 ? hi : lo) >> (shift & 63)) & (kRadix - 1);
        const uint32_t d0 = __shfl_sync(vmask, d, leader);
        if (__all_sync(vmask, d == d0)) {
          if (lane == leader) atomicAdd(&h[p * kRadix + d], (uint32_t)__popc(vmask));
        } else {
          atomicAdd(&h[p * kRadix + d], 1u);
        }
      }
    }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < npass * kRadix; q += kSortThreads)
    if (h[q]) atomicAdd(&ghist[q], h[q]);
}

// ghist -> exclusive start of each digit within the array, per pass (one
// block, a thread per digit).
static_assert(kRadix == kSortThreads, "one digit per thread");
__global__ void __launch_bounds__(kSortThreads) radix_offsets_kernel(uint32_t* __restrict__ ghist, int npass) {
  __shared__ uint32_t wsum[kSortThreads / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int p = 0; p < npass; ++p) {
    const uint32_t c = ghist[p * kRadix + tid];
    uint32_t x = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    uint32_t pre = 0;
    for (int w = 0; w < warp; ++w) pre += wsum[w];
    ghist[p * kRadix + tid] = pre + x - c;
    __syncthreads();
  }
}

// One pass over the digit at `shift`.  Warp w of the block owns the tile's
// elements [w*256, w*256 + 256) and ranks them in index order, 32 at a time,
// with its own per-digit counters (the lanes of one digit found with
// match_any; no block barrier while ranking).  The tile's digit counts are
// published and looked back on (thread d for digit d), the tile is
// reordered by digit in shared memory and written out in that order, so
// consecutive threads write consecutive addresses of a digit's run.
// status holds one word per (tile, digit): kind (aggregate / prefix) in bits
// 62-63, the pass tag in bits 32-61 (words of other passes read as not yet
// published), the count in bits 0-31.  A look-back that polls one word
// kLookbackSpins times sets *err and takes the count so far (a lower start,
// so every write stays inside the array).
// Dynamic shared memory: the tile's keys (one or two words) and payloads.
static_assert(kSortTile / (kSortThreads / 32) == kSortItems * 32, "each warp ranks kSortItems rounds of 32");
__global__ void __launch_bounds__(kSortThreads)
    radix_onesweep_kernel(const uint64_t* __restrict__ klo, const uint64_t* __restrict__ khi,
                          const uint32_t* __restrict__ pin, uint32_t n, int shift, uint32_t tag,
                          const uint32_t* __restrict__ goff, uint32_t* __restrict__ ticket,
                          unsigned long long* __restrict__ status, int* __restrict__ err,
                          uint64_t* __restrict__ olo, uint64_t* __restrict__ ohi, uint32_t* __restrict__ pout) {
  constexpr int kWarps = kSortThreads / 32;
  constexpr int kPerWarp = kSortTile / kWarps;  // 256 elements, kPerWarp / 32 = kSortItems rounds
  __shared__ uint32_t wrun[kWarps][kRadix];      // per warp: digit counts, then the warp's start in the digit
  __shared__ uint32_t gbase[kRadix];
  __shared__ uint32_t lstart[kRadix];
  __shared__ uint32_t wsum[kWarps];
  __shared__ uint32_t s_tile;
  extern __shared__ __align__(16) unsigned char dsm[];
  uint64_t* s_lo = reinterpret_cast<uint64_t*>(dsm);
  uint64_t* s_hi = s_lo + kSortTile;
  uint32_t* s_p = reinterpret_cast<uint32_t*>(khi ? s_hi + kSortTile : s_lo + kSortTile);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) wrun[w][tid] = 0;
  if (tid == 0) s_tile = atomicAdd(ticket, 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint32_t base = tile * kSortTile;
  uint64_t vlo[kSortItems], vhi[kSortItems];
  uint32_t vp[kSortItems], dg[kSortItems], rk[kSortItems];
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {  // every round's loads first, all in flight together
    const uint32_t i = base + warp * kPerWarp + r * 32 + lane;
    vlo[r] = 0;
    vhi[r] = 0;
    vp[r] = 0;
    if (i < n) {
      vlo[r] = klo[i];
      if (khi) vhi[r] = khi[i];
      vp[r] = pin[i];
    }
  }
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    const uint32_t i = base + warp * kPerWarp + r * 32 + lane;
    const bool valid = i < n;
    dg[r] = 0;
    rk[r] = 0;
    const unsigned vmask = __ballot_sync(0xffffffffu, valid);
    if (valid) {
      dg[r] = (uint32_t)((shift >= 64 ? vhi[r] : vlo[r]) >> (shift & 63)) & (kRadix - 1);
      const unsigned peers = __match_any_sync(vmask, dg[r]);
      const int leader = __ffs(peers) - 1;
      uint32_t before = 0;
      if (lane == leader) {
        before = wrun[warp][dg[r]];
        wrun[warp][dg[r]] = before + __popc(peers);
      }
      before = __shfl_sync(peers, before, leader);
      rk[r] = before + __popc(peers & ((1u << lane) - 1));  // rank among the warp's digit-d elements
    }
    __syncwarp();
  }
  __syncthreads();
  uint32_t cnt;
  {  // digit tid: each warp's start within the digit, in warp order; the tile's count
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      const uint32_t c = wrun[w][tid];
      wrun[w][tid] = run;
      run += c;
    }
    cnt = run;
  }
  // the tile's count of digit tid, published for the tiles after it
  const unsigned long long tg = (unsigned long long)tag << 32;
  volatile unsigned long long* mine = status + (size_t)tile * kRadix + tid;
  *mine = (tile == 0 ? kLbPrefix : kLbAggregate) | tg | cnt;
  {  // the tile's digit starts: exclusive scan of its digit counts
    uint32_t x = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    uint32_t pre = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w)
      if (w < warp) pre += wsum[w];
    lstart[tid] = pre + x - cnt;
  }
  __syncthreads();
  // the tile reordered by digit in shared memory (frees the registers
  // before the look-back)
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    if (base + warp * kPerWarp + r * 32 + lane < n) {
      const uint32_t at = lstart[dg[r]] + wrun[warp][dg[r]] + rk[r];
      s_lo[at] = vlo[r];
      if (khi) s_hi[at] = vhi[r];
      s_p[at] = vp[r];
    }
  }
  {  // digit tid's start among the preceding tiles (decoupled look-back)
    uint32_t excl = 0;
    if (tile > 0) {
      // the preceding tiles' words, kLookbackBatch at a time (independent
      // loads in flight together), summed nearest first up to the first
      // inclusive prefix; an unpublished word is waited on alone
      uint32_t j = tile;  // tiles [0, j) are still to be looked at
      uint32_t spins = 0;
      while (j > 0) {
        const uint32_t nb = min(j, (uint32_t)kLookbackBatch);
        unsigned long long w[kLookbackBatch];
#pragma unroll
        for (int k = 0; k < kLookbackBatch; ++k)
          w[k] = (uint32_t)k < nb ? *(volatile unsigned long long*)(status + (size_t)(j - 1 - k) * kRadix + tid)
                                  : 0ull;
        bool found = false;
        uint32_t used = 0;
#pragma unroll
        for (int k = 0; k < kLookbackBatch; ++k) {
          if (found || (uint32_t)k >= nb || used < (uint32_t)k) continue;
          if ((uint32_t)((w[k] >> 32) & 0x3fffffffu) != tag) continue;  // not yet published in this pass
          excl += (uint32_t)w[k];
          used = k + 1;
          if (w[k] & kLbPrefix) found = true;
        }
        if (found) break;
        j -= used;
        if (used < nb) {  // word j - 1 is not yet published: wait for it
          if (++spins > kLookbackSpins) {
            atomicOr(err, 1);
            break;
          }
          __nanosleep(32);
        }
      }
      *mine = kLbPrefix | tg | (excl + cnt);
    }
    gbase[tid] = goff[tid] + excl;
  }
  __syncthreads();
  const uint32_t tile_n = min((uint32_t)kSortTile, n - base);
  for (uint32_t j = tid; j < tile_n; j += kSortThreads) {
    const uint64_t lo = s_lo[j], hi = khi ? s_hi[j] : 0;
    const uint32_t d = (uint32_t)((shift >= 64 ? hi : lo) >> (shift & 63)) & (kRadix - 1);
    const uint32_t dst = gbase[d] + (j - lstart[d]);
    olo[dst] = lo;
    if (ohi) ohi[dst] = hi;
    pout[dst] = s_p[j];
  }
}

// Dynamic shared memory of radix_onesweep_kernel for one- or two-word keys.
size_t scatter_smem(bool two_words) { return (size_t)kSortTile * ((two_words ? 16 : 8) + 4); }

// Sorted interleaved keys -> line records (mode-contiguous key + value), the
// value gathered by input position (float64 or float32 input, stored float32).
template <typename VT>
__global__ void layout_kernel(const uint64_t* __restrict__ slo, const uint64_t* __restrict__ shi,
                              const uint32_t* __restrict__ sperm, const VT* __restrict__ vin,
                              MaskSet ms, LineDecode dec, uint32_t nnz, void* __restrict__ line,
                              uint32_t* __restrict__ perm_out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += gridDim.x * blockDim.x) {
    uint64_t klo = slo[i], khi = shi ? shi[i] : 0;
    uint64_t lo = 0, hi = 0;
#pragma unroll
    for (int m = 0; m < ALTO_MAX_MODES; ++m) {
      if (m < ms.nmodes) {
        uint64_t x = extract(klo, khi, ms.lo[m], ms.hi[m]);
        int p = dec.pos[m];
        if (p >= 64) {
          hi |= x << (p - 64);
        } else {
          lo |= x << p;
          if (p > 0) hi |= x >> (64 - p);
        }
      }
    }
    const uint32_t p = sperm[i];
    rec_write(line, dec.hi_words, i, lo, hi, (float)vin[p]);
    perm_out[i] = p;
  }
}

// Per tile and mode: [min, max] row of the tile's nonzeros, stored as
// (first row, row count).
__global__ void __launch_bounds__(256)
    tile_interval_kernel(const void* __restrict__ line, LineDecode dec, uint32_t nnz,
                         uint32_t tile_nnz, uint32_t* __restrict__ tile_iv) {
  __shared__ uint32_t smin[ALTO_MAX_MODES][8], smax[ALTO_MAX_MODES][8];
  uint32_t lo_r[ALTO_MAX_MODES], hi_r[ALTO_MAX_MODES];
#pragma unroll
  for (int m = 0; m < ALTO_MAX_MODES; ++m) {
    lo_r[m] = 0xffffffffu;
    hi_r[m] = 0;
  }
  uint32_t s = blockIdx.x * tile_nnz;
  uint32_t e = min(s + tile_nnz, nnz);
  for (uint32_t i = s + threadIdx.x; i < e; i += blockDim.x) {
    uint64_t lo, hi;
    float val;
    rec_read(line, dec.hi_words, i, lo, hi, val);
#pragma unroll
    for (int m = 0; m < ALTO_MAX_MODES; ++m) {
      if (m < dec.nmodes) {
        uint32_t v = (uint32_t)line_field(lo, hi, dec.pos[m], dec.mask[m]);
        lo_r[m] = min(lo_r[m], v);
        hi_r[m] = max(hi_r[m], v);
      }
    }
  }
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int m = 0; m < ALTO_MAX_MODES; ++m) {
    if (m >= dec.nmodes) continue;
    uint32_t a = lo_r[m], b = hi_r[m];
    for (int o = 16; o; o >>= 1) {
      a = min(a, __shfl_xor_sync(0xffffffffu, a, o));
      b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
    if (lane == 0) {
      smin[m][warp] = a;
      smax[m][warp] = b;
    }
  }
  __syncthreads();
  if (threadIdx.x < (unsigned)dec.nmodes) {
    int m = threadIdx.x;
    uint32_t a = 0xffffffffu, b = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      a = min(a, smin[m][w]);
      b = max(b, smax[m][w]);
    }
    if (a > b) a = b;  // empty tile
    tile_iv[((size_t)blockIdx.x * dec.nmodes + m) * 2] = a;
    tile_iv[((size_t)blockIdx.x * dec.nmodes + m) * 2 + 1] = b - a + 1;
  }
}

// prtn_alto's intervals (include/alto.hpp:1199-1226), computed over the
// whole grid: block b reduces its chunk of the line separately for every
// partition the chunk overlaps and merges the result with 64-bit atomic
// min / max.  iv starts at the reference's sentinels (start = dims, stop = 0);
// prtn_interval_fix_kernel clamps start to stop for empty partitions.
constexpr uint32_t kPrtnChunk = 4096;

__global__ void prtn_interval_init_kernel(const uint64_t* __restrict__ dims, int nmodes, int nprtn,
                                          unsigned long long* __restrict__ iv) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nprtn * nmodes; q += gridDim.x * blockDim.x) {
    iv[2 * q] = dims[q % nmodes];
    iv[2 * q + 1] = 0;
  }
}

__global__ void prtn_interval_fix_kernel(int n, unsigned long long* __restrict__ iv) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
    if (iv[2 * q] > iv[2 * q + 1]) iv[2 * q] = iv[2 * q + 1];
}

__global__ void __launch_bounds__(256)
    prtn_interval_kernel(const void* __restrict__ line, LineDecode dec, uint64_t nnz, uint64_t per,
                         unsigned long long* __restrict__ iv) {
  __shared__ unsigned long long smin[ALTO_MAX_MODES][8], smax[ALTO_MAX_MODES][8];
  const uint64_t cs = (uint64_t)blockIdx.x * kPrtnChunk;
  const uint64_t ce = min(cs + kPrtnChunk, nnz);
  if (cs >= ce) return;
  const uint64_t p0 = cs / per, p1 = (ce - 1) / per;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint64_t p = p0; p <= p1; ++p) {
    const uint64_t s = max(cs, p * per), e = min(ce, (p + 1) * per);
    unsigned long long lo_r[ALTO_MAX_MODES], hi_r[ALTO_MAX_MODES];
#pragma unroll
    for (int m = 0; m < ALTO_MAX_MODES; ++m) {
      lo_r[m] = ~0ull;
      hi_r[m] = 0;
    }
    for (uint64_t i = s + threadIdx.x; i < e; i += blockDim.x) {
      uint64_t lo, hi;
      float val;
      rec_read(line, dec.hi_words, i, lo, hi, val);
#pragma unroll
      for (int m = 0; m < ALTO_MAX_MODES; ++m) {
        if (m < dec.nmodes) {
          const unsigned long long v = line_field(lo, hi, dec.pos[m], dec.mask[m]);
          lo_r[m] = v < lo_r[m] ? v : lo_r[m];
          hi_r[m] = v > hi_r[m] ? v : hi_r[m];
        }
      }
    }
#pragma unroll
    for (int m = 0; m < ALTO_MAX_MODES; ++m) {
      if (m >= dec.nmodes) continue;
      unsigned long long a = lo_r[m], b = hi_r[m];
      for (int o = 16; o; o >>= 1) {
        const unsigned long long x = __shfl_xor_sync(0xffffffffu, a, o);
        const unsigned long long y = __shfl_xor_sync(0xffffffffu, b, o);
        a = x < a ? x : a;
        b = y > b ? y : b;
      }
      if (lane == 0) {
        smin[m][warp] = a;
        smax[m][warp] = b;
      }
    }
    __syncthreads();
    if (threadIdx.x < (unsigned)dec.nmodes) {
      const int m = threadIdx.x;
      unsigned long long a = ~0ull, b = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
        a = smin[m][w] < a ? smin[m][w] : a;
        b = smax[m][w] > b ? smax[m][w] : b;
      }
      atomicMin(&iv[(p * dec.nmodes + m) * 2], a);
      atomicMax(&iv[(p * dec.nmodes + m) * 2 + 1], b);
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------ scan utility

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total) {
  __shared__ uint32_t wsum[kScanThreads / 32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  uint32_t wpre = 0, tot = 0;
#pragma unroll
  for (int w = 0; w < kScanThreads / 32; ++w) {
    uint32_t c = wsum[w];
    if (w < warp) wpre += c;
    tot += c;
  }
  __syncthreads();
  if (total) *total = tot;
  return wpre + x - v;
}

__global__ void __launch_bounds__(kScanThreads)
    scan_reduce_kernel(const uint32_t* __restrict__ data, size_t n, uint32_t* __restrict__ part) {
  size_t base = (size_t)blockIdx.x * kScanTile;
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    size_t i = base + (size_t)k * kScanThreads + threadIdx.x;
    if (i < n) s += data[i];
  }
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ uint32_t ws[kScanThreads / 32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < kScanThreads / 32; ++w) t += ws[w];
    part[blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(kScanThreads)
    scan_apply_kernel(uint32_t* __restrict__ data, size_t n, const uint32_t* __restrict__ part) {
  size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = base + k < n ? data[base + k] : 0;
    s += v[k];
  }
  uint32_t pre = block_exclusive_scan(s, nullptr) + (part ? part[blockIdx.x] : 0);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) data[base + k] = pre;
    pre += v[k];
  }
}

static alto_status scan_level(uint32_t* data, size_t n, uint32_t* scratch, cudaStream_t st) {
  if (n <= (size_t)kScanTile) {
    scan_apply_kernel<<<1, kScanThreads, 0, st>>>(data, n, nullptr);
    ALTO_LAUNCHED();
    return ALTO_OK;
  }
  size_t nb = (n + kScanTile - 1) / kScanTile;
  uint32_t* part = scratch;
  scan_reduce_kernel<<<(unsigned)nb, kScanThreads, 0, st>>>(data, n, part);
  ALTO_LAUNCHED();
  ALTO_TRY(scan_level(part, nb, scratch + nb, st));
  scan_apply_kernel<<<(unsigned)nb, kScanThreads, 0, st>>>(data, n, part);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

alto_status exclusive_scan_u32(uint32_t* data, size_t n, DevBuf& scratch, cudaStream_t st) {
  if (n == 0) return ALTO_OK;
  size_t need = 0, m = n;
  while (m > (size_t)kScanTile) {
    m = (m + kScanTile - 1) / kScanTile;
    need += m;
  }
  ALTO_TRY(scratch.ensure((need + 1) * sizeof(uint32_t)));
  return scan_level(data, n, scratch.as<uint32_t>(), st);
}

// -------------------------------------------------------------- pipeline

static unsigned grid_for(uint64_t n, int threads) {
  uint64_t b = (n + threads - 1) / threads;
  if (b > 148ull * 64) b = 148ull * 64;
  return (unsigned)(b ? b : 1);
}

static size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Tiles, their intervals and the reference's partitions of the line (the
// part of encoding after the sort), for t->nnz line entries.
alto_status ensure_error_words(alto_tensor* t, cudaStream_t st) {
  if (t->err.p) return ALTO_OK;
  ALTO_TRY(t->err.ensure(16));
  ALTO_TRY_CUDA(cudaMemsetAsync(t->err.p, 0, 16, st));
  return ALTO_OK;
}

alto_status sort_error_status(alto_tensor* t, const int* words, cudaStream_t st) {
  if (!words[kSortErrorWord]) return ALTO_OK;
  ALTO_TRY_CUDA(cudaMemsetAsync(t->err.as<int>() + kSortErrorWord, 0, 4, st));
  set_error("a device radix sort gave up waiting on a preceding tile");
  return ALTO_ERR_TIMEOUT;
}

static alto_status finish_layout(alto_tensor* t, int nprtn, cudaStream_t st) {
  const int N = t->nmodes;
  const uint64_t nnz = t->nnz;
  const uint32_t n32 = (uint32_t)nnz;
  const LineDecode dec = t->dec;
  // MTTKRP tiles and their intervals.  Tiles hold 4096 nonzeros, fewer for
  // small tensors (down to 256) so the grid still has two tiles per SM: a
  // lane group walks tile/64 nonzeros in order, so the tile size is also the
  // length of the kernel's latency chain.
  {
    static int sm_count = 0;
    if (!sm_count) {
      int dev = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev);
      if (sm_count <= 0) sm_count = 148;
    }
    uint32_t tile = 4096;
    while (tile > 256 && (nnz + tile - 1) / tile < 2ull * (uint64_t)sm_count) tile >>= 1;
    t->tile_nnz = tile;
  }
  t->ntiles = (uint32_t)((nnz + t->tile_nnz - 1) / t->tile_nnz);
  ALTO_TRY(tensor_ensure(t, t->tile_iv, (size_t)std::max<uint32_t>(t->ntiles, 1) * N * 2 * 4));
  for (int m = 0; m < ALTO_MAX_MODES; ++m) {
    t->sorted[m].ready = false;
    t->tile_len_sorted[m].clear();
  }
  t->tuned.clear();
  if (t->ntiles) {
    tile_interval_kernel<<<t->ntiles, 256, 0, st>>>(t->line.p, dec, n32, t->tile_nnz,
                                                    t->tile_iv.as<uint32_t>());
    ALTO_LAUNCHED();
  }
  if (t->ntiles && t->tile_stats) {
    std::vector<uint32_t> iv((size_t)t->ntiles * N * 2);
    ALTO_TRY_CUDA(cudaMemcpyAsync(iv.data(), t->tile_iv.p, iv.size() * 4, cudaMemcpyDeviceToHost, st));
    int ew[4] = {0, 0, 0, 0};
    if (t->err.p) ALTO_TRY_CUDA(cudaMemcpyAsync(ew, t->err.p, sizeof(ew), cudaMemcpyDeviceToHost, st));
    ALTO_TRY_CUDA(cudaStreamSynchronize(st));
    ALTO_TRY(sort_error_status(t, ew, st));
    for (int m = 0; m < N; ++m) {
      auto& v = t->tile_len_sorted[m];
      v.resize(t->ntiles);
      for (uint32_t k = 0; k < t->ntiles; ++k) v[k] = iv[((size_t)k * N + m) * 2 + 1];
      std::sort(v.begin(), v.end());
    }
  }

  // the reference's partitions
  t->prtn_ptr.assign(nprtn + 1, 0);
  uint64_t per = (nnz + nprtn - 1) / nprtn;
  for (int p = 0; p < nprtn; ++p) {
    uint64_t e = std::min<uint64_t>((uint64_t)(p + 1) * per, nnz);
    t->prtn_ptr[p + 1] = e;
  }
  ALTO_TRY(t->prtn_iv.ensure((size_t)nprtn * N * 2 * 8 + (size_t)(nprtn + 1) * 8 + N * 8));
  uint64_t* d_iv = t->prtn_iv.as<uint64_t>();
  uint64_t* d_ptr = d_iv + (size_t)nprtn * N * 2;
  uint64_t* d_dims = d_ptr + nprtn + 1;
  ALTO_TRY_CUDA(cudaMemcpyAsync(d_ptr, t->prtn_ptr.data(), (nprtn + 1) * 8, cudaMemcpyHostToDevice, st));
  ALTO_TRY_CUDA(cudaMemcpyAsync(d_dims, t->dims, N * 8, cudaMemcpyHostToDevice, st));
  unsigned long long* d_ivu = reinterpret_cast<unsigned long long*>(d_iv);
  prtn_interval_init_kernel<<<(nprtn * N + 255) / 256, 256, 0, st>>>(d_dims, N, nprtn, d_ivu);
  ALTO_LAUNCHED();
  if (nnz) {
    prtn_interval_kernel<<<(unsigned)((nnz + kPrtnChunk - 1) / kPrtnChunk), 256, 0, st>>>(
        t->line.p, dec, nnz, per, d_ivu);
    ALTO_LAUNCHED();
  }
  prtn_interval_fix_kernel<<<(nprtn * N + 255) / 256, 256, 0, st>>>(nprtn * N, d_ivu);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

alto_status encode_tensor(alto_tensor* t, const alto_coo* coo, int nprtn, cudaStream_t st) {
  const int N = coo->nmodes;
  const uint64_t nnz = coo->nnz;
  t->nmodes = N;
  t->nnz = nnz;
  t->nprtn = nprtn;
  for (int m = 0; m < N; ++m) t->dims[m] = coo->dims[m];
  int total = setup_masks(N, t->dims, t->key_bits, t->masks, &t->alto_mask, t->mode_bits);
  if (total < 0) {
    set_error("index bits of the modes exceed the %d-bit key", t->key_bits);
    return ALTO_ERR_UNSUPPORTED;
  }
  t->alto_bits = total;

  // line layout: fields in natural mode order (ALT_PEXT mode_pos)
  LineDecode& dec = t->dec;
  dec.nmodes = N;
  int pos = 0;
  for (int m = 0; m < ALTO_MAX_MODES; ++m) {
    dec.pos[m] = 0;
    dec.mask[m] = 0;
  }
  for (int m = 0; m < N; ++m) {
    dec.pos[m] = pos;
    dec.mask[m] = t->mode_bits[m] >= 64 ? ~0ull : ((1ull << t->mode_bits[m]) - 1);
    pos += t->mode_bits[m];
  }
  dec.hi_words = total <= 64 ? 0 : (total <= 96 ? 1 : 2);

  // capacity of the per-nonzero arrays
  uint64_t cap = std::max<uint64_t>(nnz, 1);
  ALTO_TRY(tensor_ensure(t, t->line, (cap + kLinePad) * rec_bytes(dec.hi_words)));
  if (cap > t->cap || !t->perm.p) {
    ALTO_TRY(tensor_ensure(t, t->perm, cap * 4));
    t->cap = cap;
  }

  // construction scratch: two key/payload buffers, staged COO, counts
  const bool two_words = total > 64;
  const int vbytes = coo->val_dtype == ALTO_F64 ? 8 : 4;
  size_t off = 0;
  size_t o_lo0 = off; off = align_up(off + cap * 8, 256);
  size_t o_lo1 = off; off = align_up(off + cap * 8, 256);
  size_t o_hi0 = off; off = align_up(off + (two_words ? cap * 8 : 0), 256);
  size_t o_hi1 = off; off = align_up(off + (two_words ? cap * 8 : 0), 256);
  size_t o_p0 = off; off = align_up(off + cap * 4, 256);
  size_t o_p1 = off; off = align_up(off + cap * 4, 256);
  size_t o_cnt = off; off = align_up(off + radix_scratch_bytes(nnz), 256);
  size_t o_vals = off; off = align_up(off + (coo->on_device ? 0 : cap * vbytes), 256);
  size_t o_cidx = off; off = align_up(off + (coo->on_device ? 0 : cap * coo->index_bytes * N), 256);
  ALTO_TRY(tensor_ensure(t, t->scratch, off));
  char* sb = t->scratch.as<char>();
  uint64_t* klo[2] = {(uint64_t*)(sb + o_lo0), (uint64_t*)(sb + o_lo1)};
  uint64_t* khi[2] = {two_words ? (uint64_t*)(sb + o_hi0) : nullptr,
                      two_words ? (uint64_t*)(sb + o_hi1) : nullptr};
  uint32_t* pm[2] = {(uint32_t*)(sb + o_p0), (uint32_t*)(sb + o_p1)};
  void* sort_scratch = sb + o_cnt;

  CooPtrs cp{};
  const void* vin = coo->vals;
  if (coo->on_device) {
    for (int m = 0; m < N; ++m) cp.cidx[m] = coo->cidx[m];
  } else {
    for (int m = 0; m < N; ++m) {
      void* dst = sb + o_cidx + (size_t)m * cap * coo->index_bytes;
      if (nnz)
        ALTO_TRY_CUDA(cudaMemcpyAsync(dst, coo->cidx[m], nnz * coo->index_bytes,
                                      cudaMemcpyHostToDevice, st));
      cp.cidx[m] = dst;
    }
    if (nnz)
      ALTO_TRY_CUDA(cudaMemcpyAsync(sb + o_vals, coo->vals, nnz * vbytes, cudaMemcpyHostToDevice, st));
    vin = sb + o_vals;
  }

  MaskSet ms{};
  ms.nmodes = N;
  for (int m = 0; m < N; ++m) {
    ms.lo[m] = t->masks[m].lo;
    ms.hi[m] = t->masks[m].hi;
  }

  const uint32_t n32 = (uint32_t)nnz;
  if (nnz) {
    if (coo->index_bytes == 8)
      linearize_kernel<8><<<grid_for(nnz, 256), 256, 0, st>>>(cp, ms, n32, klo[0], khi[0], pm[0]);
    else
      linearize_kernel<4><<<grid_for(nnz, 256), 256, 0, st>>>(cp, ms, n32, klo[0], khi[0], pm[0]);
    ALTO_LAUNCHED();

    // LSD radix sort over the used bits
    int cur = 0;
    ALTO_TRY(ensure_error_words(t, st));
    ALTO_TRY(radix_sort_pairs(klo, khi, pm, n32, total, sort_scratch, t->err.as<int>() + kSortErrorWord, st, &cur));

    if (coo->val_dtype == ALTO_F64)
      layout_kernel<double><<<grid_for(nnz, 256), 256, 0, st>>>(
          klo[cur], khi[cur], pm[cur], (const double*)vin, ms, dec, n32, t->line.p, t->perm.as<uint32_t>());
    else
      layout_kernel<float><<<grid_for(nnz, 256), 256, 0, st>>>(
          klo[cur], khi[cur], pm[cur], (const float*)vin, ms, dec, n32, t->line.p, t->perm.as<uint32_t>());
    ALTO_LAUNCHED();
  }

  ALTO_TRY(finish_layout(t, nprtn, st));
  if (!coo->on_device) ALTO_TRY_CUDA(cudaStreamSynchronize(st));  // host COO must outlive the copies
  return ALTO_OK;
}

// Keep line entries [begin, end) (a shard of the nonzeros in ALTO order),
// then rebuild tiles, intervals and partitions for them.
alto_status restrict_line(alto_tensor* t, uint64_t begin, uint64_t end, cudaStream_t st) {
  const uint64_t n = end - begin;
  const size_t rb = rec_bytes(t->dec.hi_words);
  if (begin > 0 && n > 0) {
    ALTO_TRY(t->scratch.ensure(n * (rb + 4)));
    char* tmp = t->scratch.as<char>();
    ALTO_TRY_CUDA(cudaMemcpyAsync(tmp, t->line.as<char>() + begin * rb, n * rb, cudaMemcpyDeviceToDevice, st));
    ALTO_TRY_CUDA(cudaMemcpyAsync(tmp + n * rb, t->perm.as<uint32_t>() + begin, n * 4, cudaMemcpyDeviceToDevice, st));
    ALTO_TRY_CUDA(cudaMemcpyAsync(t->line.p, tmp, n * rb, cudaMemcpyDeviceToDevice, st));
    ALTO_TRY_CUDA(cudaMemcpyAsync(t->perm.p, tmp + n * rb, n * 4, cudaMemcpyDeviceToDevice, st));
  }
  t->nnz = n;
  return finish_layout(t, t->nprtn, st);
}

// ------------------------------------------------ per-mode row-sorted lines

// Row index of every line entry for one mode, and the identity payload.
__global__ void mode_rows_kernel(const void* __restrict__ line, LineDecode dec, int mode, uint32_t nnz,
                                 uint64_t* __restrict__ rows, uint32_t* __restrict__ pos) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += gridDim.x * blockDim.x) {
    uint64_t lo, hi;
    float v;
    rec_read(line, dec.hi_words, i, lo, hi, v);
    rows[i] = line_field(lo, hi, dec.pos[mode], dec.mask[mode]);
    pos[i] = i;
  }
}

// Gather line records (`words` 16-byte words each) in the given order.
__global__ void gather_line_kernel(const uint4* __restrict__ line, int words,
                                   const uint32_t* __restrict__ order, uint32_t nnz,
                                   uint4* __restrict__ out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += gridDim.x * blockDim.x) {
    const uint32_t p = order[i];
    for (int w = 0; w < words; ++w) out[(size_t)i * words + w] = line[(size_t)p * words + w];
  }
}

// Gather line records in the given order, writing them with the rows
// decoded (3-mode lines): {row 0, row 1, row 2, value}.
__global__ void gather_decode3_kernel(const void* __restrict__ line, LineDecode dec,
                                      const uint32_t* __restrict__ order, uint32_t nnz,
                                      uint4* __restrict__ out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += gridDim.x * blockDim.x) {
    uint64_t lo, hi;
    float v;
    rec_read(line, dec.hi_words, order[i], lo, hi, v);
    out[i] = make_uint4((uint32_t)line_field(lo, hi, dec.pos[0], dec.mask[0]),
                        (uint32_t)line_field(lo, hi, dec.pos[1], dec.mask[1]),
                        (uint32_t)line_field(lo, hi, dec.pos[2], dec.mask[2]), __float_as_uint(v));
  }
}

// Scratch of radix_sort_pairs for n pairs: the look-back words (one per
// tile and digit), the digit counts / starts of every pass, the per-pass
// tile tickets.
static size_t lookback_bytes(uint64_t n) {
  const size_t tiles = std::max<uint64_t>((n + kSortTile - 1) / kSortTile, 1);
  return align_up(tiles * kRadix * sizeof(unsigned long long), 256);
}
size_t radix_scratch_bytes(uint64_t n) {
  return lookback_bytes(n) + align_up((size_t)kMaxSortPasses * kRadix * 4 + kMaxSortPasses * 4, 256);
}

// Stable LSD radix sort of (key, payload) pairs over the low `bits` bits of a
// 64- or 128-bit key (khi[0] NULL for 64-bit keys), ping-ponging between
// the two buffers of each array; *cur receives the buffer holding the
// result.  scratch: radix_scratch_bytes(n) bytes; *err (device) is set if a
// look-back gave up.
alto_status radix_sort_pairs(uint64_t* klo[2], uint64_t* khi[2], uint32_t* pm[2], uint32_t n, int bits,
                             void* scratch, int* err, cudaStream_t st, int* cur_out) {
  int cur = 0;
  *cur_out = 0;
  const int npass = (bits + kRadixBits - 1) / kRadixBits;
  if (!n || npass <= 0) return ALTO_OK;
  if (npass > kMaxSortPasses) {
    set_error("sort key of %d bits (at most %d)", bits, kMaxSortPasses * kRadixBits);
    return ALTO_ERR_UNSUPPORTED;
  }
  const uint32_t ntiles = (n + kSortTile - 1) / kSortTile;
  static std::atomic<bool> raised[64];  // per device
  int dev = 0;
  ALTO_TRY_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64 || !raised[dev].load()) {
    ALTO_TRY_CUDA(cudaFuncSetAttribute(radix_onesweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)scatter_smem(true)));
    if (dev >= 0 && dev < 64) raised[dev] = true;
  }
  char* sb = static_cast<char*>(scratch);
  auto* status = reinterpret_cast<unsigned long long*>(sb);
  auto* ghist = reinterpret_cast<uint32_t*>(sb + lookback_bytes(n));
  uint32_t* tickets = ghist + kMaxSortPasses * kRadix;
  ALTO_TRY_CUDA(cudaMemsetAsync(scratch, 0, radix_scratch_bytes(n), st));
  int sms = 0;
  ALTO_TRY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const unsigned hist_grid =
      std::min<unsigned>((n + kSortThreads - 1) / kSortThreads, (unsigned)std::max(sms, 1) * 4);
  radix_all_hist_kernel<<<hist_grid, kSortThreads, 0, st>>>(klo[0], khi[0], n, npass, ghist);
  ALTO_LAUNCHED();
  radix_offsets_kernel<<<1, kSortThreads, 0, st>>>(ghist, npass);
  ALTO_LAUNCHED();
  for (int p = 0; p < npass; ++p) {
    radix_onesweep_kernel<<<ntiles, kSortThreads, scatter_smem(khi[cur] != nullptr), st>>>(
        klo[cur], khi[cur], pm[cur], n, p * kRadixBits, (uint32_t)p + 1, ghist + p * kRadix, tickets + p, status,
        err, klo[cur ^ 1], khi[cur ^ 1], pm[cur ^ 1]);
    ALTO_LAUNCHED();
    cur ^= 1;
  }
  *cur_out = cur;
  return ALTO_OK;
}


// A copy of the line ordered by the row of `mode`, ALTO order kept among
// equal rows (stable LSD sort over the mode's bits).  This is the device
// form of the reference's op_sched traversal (include/alto.hpp:1708-1801,
// oidx from sort_alto_rowsparse :1100-1126): runs of one output row become
// contiguous, so they reduce in registers and need one update per run.
alto_status build_sorted_line(alto_tensor* t, int mode, cudaStream_t st) {
  SortedLine& s = t->sorted[mode];
  const uint64_t nnz = t->nnz;
  const int hw = t->dec.hi_words;
  // 3-mode copies store the rows decoded (same 16 bytes per record)
  s.hw = t->nmodes == 3 ? kDecoded3 : hw;
  ALTO_TRY(tensor_ensure(t, s.line, (nnz + kLinePad) * rec_bytes(s.hw)));
  const size_t cap = std::max<uint64_t>(nnz, 1);
  size_t off = 0;
  size_t o_r0 = off; off = align_up(off + cap * 8, 256);
  size_t o_r1 = off; off = align_up(off + cap * 8, 256);
  size_t o_p0 = off; off = align_up(off + cap * 4, 256);
  size_t o_p1 = off; off = align_up(off + cap * 4, 256);
  size_t o_cnt = off; off = align_up(off + radix_scratch_bytes(nnz), 256);
  ALTO_TRY(tensor_ensure(t, t->scratch, off));
  char* sb = t->scratch.as<char>();
  uint64_t* rk[2] = {(uint64_t*)(sb + o_r0), (uint64_t*)(sb + o_r1)};
  uint32_t* pm[2] = {(uint32_t*)(sb + o_p0), (uint32_t*)(sb + o_p1)};
  void* sort_scratch = sb + o_cnt;
  const uint32_t n32 = (uint32_t)nnz;
  if (nnz) {
    ALTO_TRY(ensure_error_words(t, st));
    mode_rows_kernel<<<grid_for(nnz, 256), 256, 0, st>>>(t->line.p, t->dec, mode, n32, rk[0], pm[0]);
    ALTO_LAUNCHED();
    int cur = 0;
    uint64_t* nohi[2] = {nullptr, nullptr};
    ALTO_TRY(radix_sort_pairs(rk, nohi, pm, n32, t->mode_bits[mode], sort_scratch,
                              t->err.as<int>() + kSortErrorWord, st, &cur));
    if (s.hw == kDecoded3)
      gather_decode3_kernel<<<grid_for(nnz, 256), 256, 0, st>>>(t->line.p, t->dec, pm[cur], n32,
                                                                 s.line.as<uint4>());
    else
      gather_line_kernel<<<grid_for(nnz, 256), 256, 0, st>>>(t->line.as<uint4>(), rec_bytes(hw) / 16,
                                                             pm[cur], n32, s.line.as<uint4>());
    ALTO_LAUNCHED();
  }
  s.ntiles = t->ntiles;
  ALTO_TRY(tensor_ensure(t, s.tile_iv, (size_t)std::max<uint32_t>(t->ntiles, 1) * t->nmodes * 2 * 4));
  // (tile intervals are read only by shared-memory staging, which never
  // walks a sorted copy; the decoded copies carry none)
  if (t->ntiles && s.hw != kDecoded3) {
    tile_interval_kernel<<<t->ntiles, 256, 0, st>>>(s.line.p, t->dec, n32, t->tile_nnz,
                                                    s.tile_iv.as<uint32_t>());
    ALTO_LAUNCHED();
  }
  s.ready = true;
  s.for_nnz = nnz;
  return ALTO_OK;
}

// Re-derive the reference's interleaved key from the line key (export).
__global__ void export_key_kernel(const void* __restrict__ line, LineDecode dec, MaskSet ms, uint32_t nnz,
                                  uint64_t* __restrict__ out, float* __restrict__ vals) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += gridDim.x * blockDim.x) {
    uint64_t lo, hi;
    float v;
    rec_read(line, dec.hi_words, i, lo, hi, v);
    if (vals) vals[i] = v;
    if (!out) continue;
    uint64_t klo = 0, khi = 0;
#pragma unroll
    for (int m = 0; m < ALTO_MAX_MODES; ++m)
      if (m < dec.nmodes) deposit(line_field(lo, hi, dec.pos[m], dec.mask[m]), ms.lo[m], ms.hi[m], klo, khi);
    out[2 * (size_t)i] = klo;
    out[2 * (size_t)i + 1] = khi;
  }
}

// Re-derive the interleaved keys (d_out, 2 words per nonzero, may be NULL)
// and the values (d_vals, may be NULL) of the line.
alto_status export_keys(const alto_tensor* t, uint64_t* d_out, float* d_vals, cudaStream_t st) {
  MaskSet ms{};
  ms.nmodes = t->nmodes;
  for (int m = 0; m < t->nmodes; ++m) {
    ms.lo[m] = t->masks[m].lo;
    ms.hi[m] = t->masks[m].hi;
  }
  if (!t->nnz) return ALTO_OK;
  export_key_kernel<<<grid_for(t->nnz, 256), 256, 0, st>>>(t->line.p, t->dec, ms, (uint32_t)t->nnz, d_out,
                                                           d_vals);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

}  // namespace alto
