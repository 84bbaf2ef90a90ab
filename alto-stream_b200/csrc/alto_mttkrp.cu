// ALTO MTTKRP on the device.
//
// Reference: mttkrp_alto_par and its variants (jeewhanchoi/ALTO-stream
// include/alto.hpp:826-908 dispatch, :1349-1407 atomic, :1544-1634
// da_mem_pull, :1636-1706 stream, :1708-1801 op_sched).  For every nonzero
// x = (i_0..i_{N-1}, v) of the line:  out[i_n, :] += v * prod_{m != n} U_m[i_m, :].
//
// Device design.  The line is cut into tiles of tile_nnz nonzeros (the
// reference's partitions, sized for the GPU); a persistent grid, sized by
// occupancy, walks the tiles, and each warp takes an equal chunk of a tile.
// Inside a warp, G = R/8 lanes own one nonzero (each lane 8 consecutive rank
// elements, two 16-byte loads per factor row), and the warp's chunk is split
// into 32/G contiguous sub-ranges, one per lane group.  A group walks its
// sub-range in line order, two nonzeros per iteration with all their keys,
// values and factor rows loaded before any product is formed, and keeps the
// running sum of the current output row in registers: each run of equal
// rows costs one update, with no cross-lane traffic.  Updates go
//   * to shared memory, when the tile's output interval (rows between its
//     smallest and largest target index, the reference's prtn_intervals)
//     fits the staging buffer -- the reference's da_mem, on chip -- and the
//     staged rows are flushed once per tile with vector atomics (STAGED;
//     the single-row output of the stream mode is its degenerate case); or
//   * to global memory with 16-byte vector atomics (red.global.add.v4.f32),
//     the reference's atomic variant (ATOMIC); or
//   * (SORTED) the same kernel walks a per-mode copy of the line ordered by
//     the output row (ALTO order among equal rows), so every run of a row is
//     contiguous, reduces in registers, and is written once per warp chunk --
//     the reference's op_sched traversal, materialised.
// ALTO_MTTKRP_AUTO uses the autotuned choice when alto_mttkrp_autotune has
// measured one, else a rule on the tile intervals and the mode's reuse.
#include <algorithm>

#include "alto_group.cuh"

namespace alto {

constexpr uint32_t kNoRow = 0xffffffffu;
constexpr int kMttkrpThreads = 256;
constexpr int kMttkrpWarps = kMttkrpThreads / 32;
constexpr int kStageBytes = 96 * 1024;

template <typename FT>
__device__ __forceinline__ float4 load4(const void* base, size_t off);

template <>
__device__ __forceinline__ float4 load4<float>(const void* base, size_t off) {
  return __ldg(reinterpret_cast<const float4*>(static_cast<const float*>(base) + off));
}

template <>
__device__ __forceinline__ float4 load4<__nv_bfloat16>(const void* base, size_t off) {
  uint2 u = __ldg(reinterpret_cast<const uint2*>(static_cast<const __nv_bfloat16*>(base) + off));
  float4 r;
  r.x = __uint_as_float(u.x << 16);
  r.y = __uint_as_float(u.x & 0xffff0000u);
  r.z = __uint_as_float(u.y << 16);
  r.w = __uint_as_float(u.y & 0xffff0000u);
  return r;
}


// Decode one mode's field from the line key held as 32-bit words
// w0..w3 (w0 lowest): a funnel shift of the two words the field starts in.
// Fields are at most 32 bits wide (mode lengths below 2^32).
__device__ __forceinline__ uint32_t field32(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3, int pos,
                                            uint32_t mask) {
  const int s = pos & 31;
  uint32_t v;
  switch (pos >> 5) {
    case 0: v = __funnelshift_r(w0, w1, s); break;
    case 1: v = __funnelshift_r(w1, w2, s); break;
    case 2: v = __funnelshift_r(w2, w3, s); break;
    default: v = w3 >> s; break;
  }
  return v & mask;
}

// Row of mode m of a record held as words w (HW = kDecoded3: stored
// decoded; else the field of the mode-contiguous key).
template <int HW>
__device__ __forceinline__ uint32_t rec_row(const uint32_t (&w)[4], const LineDecode& dec, int m) {
  // (selects, not w[m]: a runtime index would move w to local memory)
  if (HW == kDecoded3) return m == 0 ? w[0] : (m == 1 ? w[1] : w[2]);
  return field32(w[0], w[1], w[2], w[3], dec.pos[m], (uint32_t)dec.mask[m]);
}

// This lane's V floats of a factor row: V/4 float4 pieces at columns
// q*4G + 4*sub (q = 0..V/4-1), so that one load instruction of the G lanes of
// a group reads 4G contiguous floats (whole 32-byte sectors).
template <typename FT, int V, int G>
__device__ __forceinline__ void load_row(const void* base, size_t row_off, int sub, float (&x)[V]) {
#pragma unroll
  for (int q = 0; q < V / 4; ++q) {
    const float4 f = load4<FT>(base, row_off + q * 4 * G + sub * 4);
    x[q * 4 + 0] = f.x;
    x[q * 4 + 1] = f.y;
    x[q * 4 + 2] = f.z;
    x[q * 4 + 3] = f.w;
  }
}

// One update of output row `row` with this lane's V floats.
template <int R, int V, int G>
__device__ __forceinline__ void flush_row(bool staged, float* smem, uint32_t iv_start, float* out,
                                          uint32_t row, int sub, const float (&acc)[V]) {
  if (staged) {
    float* s = smem + (size_t)(row - iv_start) * R + sub * 4;
#pragma unroll
    for (int q = 0; q < V / 4; ++q)
#pragma unroll
      for (int k = 0; k < 4; ++k) atomicAdd(s + q * 4 * G + k, acc[q * 4 + k]);
  } else {
    float* o = out + (size_t)row * R + sub * 4;
#pragma unroll
    for (int q = 0; q < V / 4; ++q)
      atomicAdd(reinterpret_cast<float4*>(o + q * 4 * G),
                make_float4(acc[q * 4], acc[q * 4 + 1], acc[q * 4 + 2], acc[q * 4 + 3]));
  }
}

// Floats per lane for rank R: 4, so the G = R/4 lanes of a group read one
// factor row with one 16-byte load each -- whole 128-byte lines at R = 32,
// which keeps the L1 data pipe at one wavefront per row.
template <int R>
struct LaneWidth {
  static constexpr int V = 4;
  static constexpr int G = R / V;     // lanes per nonzero
  static constexpr int NPW = 32 / G;  // groups (nonzeros in flight) per warp
};

// Keys and values of U consecutive line records, from global memory or
// from the line tile staged in shared memory (SMEM): one 16-byte load per
// record (two when the key needs more than 96 bits, HW == 2).
template <int HW, int U, bool SMEM>
__device__ __forceinline__ void load_keys(const void* line, uint32_t i0, uint32_t ge,
                                          uint32_t (&w)[U][4], float (&v)[U], bool (&valid)[U]) {
  const uint4* q = static_cast<const uint4*>(line);
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const uint32_t i = i0 + u;
    valid[u] = i < ge;
    uint4 a = make_uint4(0, 0, 0, 0), b = make_uint4(0, 0, 0, 0);
    if (valid[u]) {
      if (HW == 2) {
        a = SMEM ? q[2 * i] : __ldg(q + 2 * i);
        b = SMEM ? q[2 * i + 1] : __ldg(q + 2 * i + 1);
      } else {
        a = SMEM ? q[i] : __ldg(q + i);
      }
    }
    w[u][0] = a.x;
    w[u][1] = a.y;
    if (HW == 2) {
      w[u][2] = a.z;
      w[u][3] = a.w;
      v[u] = __uint_as_float(b.x);
    } else {
      w[u][2] = a.z;
      w[u][3] = 0;
      v[u] = __uint_as_float(a.w);
    }
  }
}

// Walk line range [ws, we) with one warp: the range is split into NPW
// contiguous sub-ranges, one per lane group; a group walks its sub-range in
// order, U nonzeros per iteration (two for 3 modes, one for more, to stay in
// registers), with the next iteration's keys loaded while this iteration's
// factor rows are in flight; it keeps the running sum of the current output
// row in registers and updates the output once per run of equal rows.  NM is
// the mode count (3, 4, 5 specialised as in the reference's
// ALTO_MODES_SPECIALIZED, 8 for the rest).
// Deterministic mode (DET): the line is ordered by the target row, so a run
// that is neither the first nor the last of its sub-range holds every
// nonzero of its row and is added to the output without atomics; the first
// and last runs go to the sub-range's two slots (sub-range `sr`) and are
// summed in slot order by det_fix_*.
template <int R, int V, int G>
__device__ __forceinline__ void det_slot(const MttkrpArgs& a, uint32_t slot, uint32_t row, int sub,
                                         const float (&acc)[V], bool zero) {
  if (sub == 0) a.det_rows[slot] = row;
#pragma unroll
  for (int q = 0; q < V / 4; ++q)
    *reinterpret_cast<float4*>(a.det_vals + (size_t)slot * R + q * 4 * G + sub * 4) =
        zero ? make_float4(0.f, 0.f, 0.f, 0.f)
             : make_float4(acc[q * 4], acc[q * 4 + 1], acc[q * 4 + 2], acc[q * 4 + 3]);
}

template <int R, int V, int G>
__device__ __forceinline__ void det_plain(float* out, uint32_t row, int sub, const float (&acc)[V]) {
#pragma unroll
  for (int q = 0; q < V / 4; ++q) {
    float4* o = reinterpret_cast<float4*>(out + (size_t)row * R + q * 4 * G + sub * 4);
    float4 x = *o;
    x.x += acc[q * 4];
    x.y += acc[q * 4 + 1];
    x.z += acc[q * 4 + 2];
    x.w += acc[q * 4 + 3];
    *o = x;
  }
}

// The open run of a lane group (CARRY walks take it in and hand it back
// instead of updating the output at the end of their sub-range).
template <int V>
struct OpenRun {
  uint32_t row;
  float acc[V];
};

// TGT >= 0 (decoded 3-mode records only) fixes the target mode at compile
// time: the target and input rows are then fixed words of the record and the
// input factors fixed arguments, with no per-nonzero selects or mode checks.
template <int R, typename FT, int HW, int NM, bool SMEM, bool DET = false, bool CARRY = false, int TGT = -1>
__device__ __forceinline__ void warp_range(const MttkrpArgs& a, const void* line, uint32_t ws, uint32_t we,
                                           bool staged, float* smem, uint32_t iv_start, uint32_t sr_base = 0,
                                           OpenRun<LaneWidth<R>::V>* carry = nullptr) {
  static_assert(TGT < 0 || (HW == kDecoded3 && NM == 3), "a compile-time target needs decoded 3-mode records");
  using LW = LaneWidth<R>;
  const int target = TGT >= 0 ? TGT : a.target;
  constexpr int V = LW::V, G = LW::G, NPW = LW::NPW;
  // nonzeros per step: 2 for 3 modes (4 measured faster for DET only), 1
  // beyond (two measured 30% slower on the rank-64 5-mode tensor: its four
  // gathered rows per nonzero already fill the registers); the accumulation
  // order is the line order whatever U is
  constexpr int U = NM <= 3 ? (DET ? 4 : 2) : 1;
  const int lane = threadIdx.x & 31;
  const int grp = lane / G, sub = lane % G;
  // groups' sub-ranges; odd lengths when reading shared memory, so the
  // groups' records fall in different banks
  uint32_t sublen = (we - ws + NPW - 1) / NPW;
  if (SMEM) sublen |= 1u;
  const uint32_t gs = min(ws + grp * sublen, we);
  const uint32_t ge = min(gs + sublen, we);
  float acc[V];
  uint32_t cur = kNoRow;
  if constexpr (CARRY) {
    cur = carry->row;
#pragma unroll
    for (int q = 0; q < V; ++q) acc[q] = carry->acc[q];
  } else {
#pragma unroll
    for (int q = 0; q < V; ++q) acc[q] = 0.f;
  }
  uint32_t nrun = 0;  // runs emitted (DET)
  const uint32_t slot0 = 2 * (sr_base + grp);

  uint32_t w[U][4];
  float v[U];
  bool valid[U];
  load_keys<HW, U, SMEM>(line, gs, ge, w, v, valid);
  for (uint32_t k = 0; k < sublen; k += U) {
    // factor rows of the NM-1 input modes (j-th input mode m = j, or j+1
    // past the target)
    float f[U][NM - 1][V];
#pragma unroll
    for (int u = 0; u < U; ++u) {
#pragma unroll
      for (int j = 0; j < NM - 1; ++j) {
        const int m = j < target ? j : j + 1;
        if ((TGT >= 0 || m < a.dec.nmodes) && valid[u]) {
          const uint32_t r = rec_row<HW>(w[u], a.dec, m);
          load_row<FT, V, G>(a.fac.f[m], (size_t)r * R, sub, f[u][j]);
        }
      }
    }
    uint32_t rows[U];
    float vals[U];
    bool ok[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      rows[u] = rec_row<HW>(w[u], a.dec, target);
      vals[u] = v[u];
      ok[u] = valid[u];
    }
    load_keys<HW, U, SMEM>(line, gs + k + U, ge, w, v, valid);  // next iteration's keys
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (!ok[u]) continue;
      if constexpr (NM <= 5) {
        // exact mode count: packed FP32x2 products, the last factor fused
        // into the running sum (acc = p f_last, or acc += p f_last)
        float2 p2[V / 2];
#pragma unroll
        for (int h = 0; h < V / 2; ++h) {
          p2[h] = __fmul2_rn(make_float2(vals[u], vals[u]), make_float2(f[u][0][2 * h], f[u][0][2 * h + 1]));
#pragma unroll
          for (int j = 1; j < NM - 2; ++j)
            p2[h] = __fmul2_rn(p2[h], make_float2(f[u][j][2 * h], f[u][j][2 * h + 1]));
        }
        if (rows[u] != cur) {
          if (cur != kNoRow) {
            if (!DET)
              flush_row<R, V, G>(staged, smem, iv_start, a.out, cur, sub, acc);
            else if (nrun++ == 0)
              det_slot<R, V, G>(a, slot0, cur, sub, acc, false);
            else
              det_plain<R, V, G>(a.out, cur, sub, acc);
          }
          cur = rows[u];
#pragma unroll
          for (int h = 0; h < V / 2; ++h) {
            const float2 r2 = __fmul2_rn(p2[h], make_float2(f[u][NM - 2][2 * h], f[u][NM - 2][2 * h + 1]));
            acc[2 * h] = r2.x;
            acc[2 * h + 1] = r2.y;
          }
        } else {
#pragma unroll
          for (int h = 0; h < V / 2; ++h) {
            const float2 r2 = __ffma2_rn(p2[h], make_float2(f[u][NM - 2][2 * h], f[u][NM - 2][2 * h + 1]),
                                         make_float2(acc[2 * h], acc[2 * h + 1]));
            acc[2 * h] = r2.x;
            acc[2 * h + 1] = r2.y;
          }
        }
      } else {
        float p[V];
#pragma unroll
        for (int q = 0; q < V; ++q) p[q] = vals[u];
#pragma unroll
        for (int j = 0; j < NM - 1; ++j)
          if ((j < a.target ? j : j + 1) < a.dec.nmodes)
#pragma unroll
            for (int q = 0; q < V; ++q) p[q] *= f[u][j][q];
        if (rows[u] != cur) {
          if (cur != kNoRow) {
            if (!DET)
              flush_row<R, V, G>(staged, smem, iv_start, a.out, cur, sub, acc);
            else if (nrun++ == 0)
              det_slot<R, V, G>(a, slot0, cur, sub, acc, false);
            else
              det_plain<R, V, G>(a.out, cur, sub, acc);
          }
          cur = rows[u];
#pragma unroll
          for (int q = 0; q < V; ++q) acc[q] = p[q];
        } else {
#pragma unroll
          for (int q = 0; q < V; ++q) acc[q] += p[q];
        }
      }
    }
  }
  if (!DET) {
    if constexpr (CARRY) {
      carry->row = cur;
#pragma unroll
      for (int q = 0; q < V; ++q) carry->acc[q] = acc[q];
    } else if (cur != kNoRow) {
      flush_row<R, V, G>(staged, smem, iv_start, a.out, cur, sub, acc);
    }
  } else if (cur == kNoRow) {
    // empty sub-range: both slots carry the row of the entry before it (the
    // last run of an earlier sub-range) with zeros, keeping slot rows sorted
    uint32_t w0[1][4];
    float v0[1];
    bool ok0[1];
    const uint32_t at = gs > 0 ? gs - 1 : 0;
    load_keys<HW, 1, SMEM>(line, at, at + 1, w0, v0, ok0);
    const uint32_t r0 = rec_row<HW>(w0[0], a.dec, a.target);
    det_slot<R, V, G>(a, slot0, r0, sub, acc, true);
    det_slot<R, V, G>(a, slot0 + 1, r0, sub, acc, true);
  } else if (nrun == 0) {
    det_slot<R, V, G>(a, slot0, cur, sub, acc, false);
    det_slot<R, V, G>(a, slot0 + 1, cur, sub, acc, true);
  } else {
    det_slot<R, V, G>(a, slot0 + 1, cur, sub, acc, false);
  }
}

template <int R, typename FT, int HW, bool STAGE, int NM, bool DET = false, int MINB = 3, int TGT = -1>
__global__ void __launch_bounds__(kMttkrpThreads, MINB)
    mttkrp_tile_kernel(const MttkrpArgs a) {
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  const int warp = threadIdx.x >> 5;
  const int N = a.dec.nmodes;
  if constexpr (!STAGE && !DET) {
    // chunks of chunk_tiles consecutive tiles, round robin over the blocks;
    // within a chunk each lane group walks its sub-range of every tile with
    // its open run carried along, so a row running through the chunk (a hot
    // row) is updated once per group and chunk rather than once per tile:
    // fewer float32 additions in the output, and fewer atomics
    using LW = LaneWidth<R>;
    const uint32_t ct = a.chunk_tiles ? a.chunk_tiles : 1;
    const uint32_t nchunks = (a.ntiles + ct - 1) / ct;
    for (uint32_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
      OpenRun<LW::V> run;
      run.row = kNoRow;
#pragma unroll
      for (int q = 0; q < LW::V; ++q) run.acc[q] = 0.f;
      const uint32_t t_end = min(c * ct + ct, a.ntiles);
      for (uint32_t tile = c * ct; tile < t_end; ++tile) {
        const uint32_t ts = tile * a.tile_nnz;
        const uint32_t te = min(ts + a.tile_nnz, a.nnz);
        const uint32_t chunk = (te - ts + kMttkrpWarps - 1) / kMttkrpWarps;
        const uint32_t ws = min(ts + warp * chunk, te);
        const uint32_t we = min(ws + chunk, te);
        warp_range<R, FT, HW, NM, false, false, true, TGT>(a, a.line, ws, we, false, smem, 0, 0, &run);
      }
      if (run.row != kNoRow)
        flush_row<R, LW::V, LW::G>(false, smem, 0, a.out, run.row, (threadIdx.x & 31) % LW::G, run.acc);
    }
    return;
  }
  for (uint32_t tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
    const uint32_t ts = tile * a.tile_nnz;
    const uint32_t te = min(ts + a.tile_nnz, a.nnz);
    uint32_t iv_start = 0;
    bool staged = false;
    if (STAGE) {
      iv_start = a.tile_iv[((size_t)tile * N + a.target) * 2];
      const uint32_t iv_len = a.tile_iv[((size_t)tile * N + a.target) * 2 + 1];
      staged = iv_len <= (uint32_t)a.stage_rows && iv_len * 2 <= (te - ts);
      if (staged) {
        for (uint32_t q = threadIdx.x; q < iv_len * (R / 4); q += blockDim.x)
          smem4[q] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
      __syncthreads();
    }
    const uint32_t chunk = (te - ts + kMttkrpWarps - 1) / kMttkrpWarps;
    const uint32_t ws = min(ts + warp * chunk, te);
    const uint32_t we = min(ws + chunk, te);
    warp_range<R, FT, HW, NM, false, DET>(a, a.line, ws, we, staged, smem, iv_start,
                                          (tile * kMttkrpWarps + warp) * LaneWidth<R>::NPW);
    if (STAGE && staged) {
      __syncthreads();
      const uint32_t iv_len = a.tile_iv[((size_t)tile * N + a.target) * 2 + 1];
      for (uint32_t q = threadIdx.x; q < iv_len * (R / 4); q += blockDim.x) {
        const float4 v = smem4[q];
        if (v.x != 0.f || v.y != 0.f || v.z != 0.f || v.w != 0.f) {
          const uint32_t r = q / (R / 4), s = q % (R / 4);
          atomicAdd(reinterpret_cast<float4*>(a.out + (size_t)(iv_start + r) * R + s * 4), v);
        }
      }
      __syncthreads();
    }
  }
}

// ------------------------------------------------ deterministic fix-up
//
// The slots of DET hold, in line order, the first and last run of every
// sub-range; their rows are non-decreasing, and a row appears in the slots
// only if it is in none of the interior runs.  A chain (maximal stretch of
// slots with one row) is summed in slot order, by one warp when it is short
// and by one block with a fixed split and a fixed tree when it is long (a
// hot row, or the single row of the stream mode).  The summation order is a
// function of nnz, the rank and the line alone, so results repeat bit for
// bit from run to run and whatever else runs on the device.

constexpr uint32_t kShortChain = 64;
constexpr uint32_t kChainSeg = 256;  // slots per segment of a long chain

// Chain starting at slot i (one warp; lanes cooperate): a short chain is
// summed in slot order into its row; a long one registers itself and its
// segments for det_fix_seg / det_fix_final.
__device__ __forceinline__ void det_short_chain(const uint32_t* __restrict__ rows, const float* __restrict__ vals,
                                                uint32_t nslots, int R, float* __restrict__ out, const DetLong& dl,
                                                uint32_t i, int lane) {
  const uint32_t row = rows[i];
  if (i > 0 && rows[i - 1] == row) return;  // not the head of its chain
  // chain end: first slot with a larger row -- the next 32 slots in one
  // coalesced probe, a binary search beyond them
  const uint32_t pi = i + 1 + lane;
  const unsigned differ = __ballot_sync(0xffffffffu, pi < nslots && rows[pi] != row);
  uint32_t lo;
  if (differ) {
    lo = i + 1 + __ffs(differ) - 1;
  } else if (i + 33 >= nslots) {
    lo = nslots;
  } else {
    lo = i + 33;
    uint32_t hi = nslots;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (rows[mid] == row)
        lo = mid + 1;
      else
        hi = mid;
    }
  }
  if (lo - i > kShortChain) {
    // long chain: register it and its segments (the order of the lists
    // varies from run to run; what each entry sums does not)
    const uint32_t nseg = (lo - i + kChainSeg - 1) / kChainSeg;
    uint32_t c = 0, base = 0;
    if (lane == 0) {
      c = atomicAdd(&dl.counters[0], 1u);
      base = atomicAdd(&dl.counters[1], nseg);
      dl.chains[c] = make_uint4(i, lo, base, nseg);
    }
    c = __shfl_sync(0xffffffffu, c, 0);
    base = __shfl_sync(0xffffffffu, base, 0);
    for (uint32_t k = lane; k < nseg; k += 32) dl.segs[base + k] = make_uint2(c, k);
    return;
  }
  for (int r = lane; r < R; r += 32) {
    float x = 0.f;
    for (uint32_t k = i; k < lo; ++k) x += vals[(size_t)k * R + r];
    out[(size_t)row * R + r] += x;
  }
}

__global__ void __launch_bounds__(256)
    det_fix_short_kernel(const uint32_t* __restrict__ rows, const float* __restrict__ vals, uint32_t nslots,
                         int R, float* __restrict__ out, DetLong dl) {
  const int lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = gw; i < nslots; i += nw) det_short_chain(rows, vals, nslots, R, out, dl, i, lane);
}

// One segment g of a long chain (one block): thread (s, q) sums slots
// start+s, start+s+S, ... of rank quad q (S = 256 / (R/4)), then a fixed tree
// over s; the segment's R sums go to segpart.
__device__ __forceinline__ void det_segment(const float* __restrict__ vals, int R, const DetLong& dl, uint32_t g,
                                            float4* part) {
  const int Q = R / 4, S = 256 / Q;
  const int sidx = threadIdx.x / Q, q = threadIdx.x % Q;
  const uint2 sg = dl.segs[g];
  const uint4 ch = dl.chains[sg.x];
  const uint32_t s0 = ch.x + sg.y * kChainSeg;
  const uint32_t s1 = min(s0 + kChainSeg, ch.y);
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  if (sidx < S)
    for (uint32_t k = s0 + sidx; k < s1; k += S) {
      const float4 v = *reinterpret_cast<const float4*>(vals + (size_t)k * R + q * 4);
      acc.x += v.x;
      acc.y += v.y;
      acc.z += v.z;
      acc.w += v.w;
    }
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int stride = S / 2; stride >= 1; stride >>= 1) {
    if (sidx < stride) {
      const float4 o = part[(sidx + stride) * Q + q];
      float4& m = part[sidx * Q + q];
      m.x += o.x;
      m.y += o.y;
      m.z += o.z;
      m.w += o.w;
    }
    __syncthreads();
  }
  if (sidx == 0) *reinterpret_cast<float4*>(dl.segpart + (size_t)(ch.z + sg.y) * R + q * 4) = part[q];
  __syncthreads();
}

__global__ void __launch_bounds__(256)
    det_fix_seg_kernel(const float* __restrict__ vals, int R, DetLong dl) {
  __shared__ float4 part[256];
  const uint32_t nseg = dl.counters[1];
  for (uint32_t g = blockIdx.x; g < nseg; g += gridDim.x) det_segment(vals, R, dl, g, part);
}

// One long chain c (one block): thread (s, q) sums segments s, s+S, ... of
// rank quad q, then a fixed tree over s; the result is added to the chain's
// row.
__device__ __forceinline__ void det_chain_final(const uint32_t* __restrict__ rows, int R, float* __restrict__ out,
                                                const DetLong& dl, uint32_t c, float4* part) {
  const int Q = R / 4, S = 256 / Q;
  const int sidx = threadIdx.x / Q, q = threadIdx.x % Q;
  const uint4 ch = dl.chains[c];
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  if (sidx < S)
    for (uint32_t k = sidx; k < ch.w; k += S) {
      const float4 v = *reinterpret_cast<const float4*>(dl.segpart + (size_t)(ch.z + k) * R + q * 4);
      acc.x += v.x;
      acc.y += v.y;
      acc.z += v.z;
      acc.w += v.w;
    }
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int stride = S / 2; stride >= 1; stride >>= 1) {
    if (sidx < stride) {
      const float4 o = part[(sidx + stride) * Q + q];
      float4& m = part[sidx * Q + q];
      m.x += o.x;
      m.y += o.y;
      m.z += o.z;
      m.w += o.w;
    }
    __syncthreads();
  }
  if (sidx == 0) {
    float4* o = reinterpret_cast<float4*>(out + (size_t)rows[ch.x] * R + q * 4);
    float4 x = *o;
    const float4 p = part[q];
    x.x += p.x;
    x.y += p.y;
    x.z += p.z;
    x.w += p.w;
    *o = x;
  }
  __syncthreads();
}

// The long-chain count of dl (every thread of the block gets it); the last
// block to have read it clears the counters for the next call (they start
// at zero when the workspace is allocated).
__device__ __forceinline__ uint32_t det_take_chains(const DetLong& dl, uint32_t* s_nlong) {
  if (threadIdx.x == 0) *s_nlong = dl.counters[0];
  __syncthreads();
  const uint32_t nlong = *s_nlong;
  if (threadIdx.x == 0 && atomicAdd(&dl.counters[2], 1u) == gridDim.x - 1) {
    dl.counters[0] = 0;
    dl.counters[1] = 0;
    dl.counters[2] = 0;
  }
  __syncthreads();
  return nlong;
}

__global__ void __launch_bounds__(256)
    det_fix_final_kernel(const uint32_t* __restrict__ rows, int R, float* __restrict__ out, DetLong dl) {
  __shared__ float4 part[256];
  __shared__ uint32_t s_nlong;
  const uint32_t nlong = det_take_chains(dl, &s_nlong);
  for (uint32_t c = blockIdx.x; c < nlong; c += gridDim.x) det_chain_final(rows, R, out, dl, c, part);
}

// ------------------------------------------------ grouped deterministic MTTKRP
//
// The same kernels over a table of items (sessions' MTTKRPs, one mode each):
// a global tile index runs over the items' tiles (prefix sums tile_off), and
// the fix-ups walk every item's slots, segments and chains in turn.  An
// item's sums, and their order, are those of its own launch.

__device__ __forceinline__ bool item_live(const int* active) { return !active || *active; }

// The last s in [0, K) with off[s] <= v (items with no blocks are skipped).
__device__ __forceinline__ int item_of(const uint32_t* __restrict__ off, int K, uint32_t v) {
  int lo = 0, hi = K;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= v)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(256) det_zero_group_kernel(Strided<DetItem> items) {
  const int K = *items.count;
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
  for (int s = 0; s < K; ++s) {
    const DetItem& it = items[s];
    if (!item_live(it.active)) continue;
    float4* o = reinterpret_cast<float4*>(it.a.out);
    const uint64_t n4 = it.out_floats / 4;
    for (uint64_t q = tid; q < n4; q += nth) o[q] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

template <int R, int HW, int NM>
__global__ void __launch_bounds__(kMttkrpThreads, 3)
    det_tile_group_kernel(Strided<DetItem> items, const uint32_t* __restrict__ tile_off) {
  // the item's arguments staged in shared memory: the walk reads them per
  // nonzero (as a launch of its own reads them from the parameter bank)
  __shared__ MttkrpArgs sa;
  __shared__ int s_item;
  const int K = *items.count;
  const uint32_t total = K > 0 ? tile_off[K] : 0;
  const int warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_item = -1;
  for (uint32_t v = blockIdx.x; v < total; v += gridDim.x) {
    const int s = item_of(tile_off, K, v);
    const DetItem& it = items[s];
    if (!item_live(it.active)) continue;
    __syncthreads();  // (everyone is done with the previous item's copy)
    if (s != s_item) {
      constexpr int kWords = (int)(sizeof(MttkrpArgs) / 4);
      const uint32_t* src = reinterpret_cast<const uint32_t*>(&it.a);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&sa);
      for (int q = threadIdx.x; q < kWords; q += blockDim.x) dst[q] = src[q];
      __syncthreads();
      if (threadIdx.x == 0) s_item = s;
    }
    __syncthreads();
    const MttkrpArgs& a = sa;
    const uint32_t tile = v - tile_off[s];
    const uint32_t ts = tile * a.tile_nnz;
    const uint32_t te = min(ts + a.tile_nnz, a.nnz);
    const uint32_t chunk = (te - ts + kMttkrpWarps - 1) / kMttkrpWarps;
    const uint32_t ws = min(ts + warp * chunk, te);
    const uint32_t we = min(ws + chunk, te);
    warp_range<R, float, HW, NM, false, true>(a, a.line, ws, we, false, nullptr, 0,
                                              (tile * kMttkrpWarps + warp) * LaneWidth<R>::NPW);
  }
}

__global__ void __launch_bounds__(256) det_short_group_kernel(Strided<DetItem> items, int R) {
  const int K = *items.count;
  const int lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (int s = 0; s < K; ++s) {
    const DetItem& it = items[s];
    if (!item_live(it.active)) continue;
    for (uint32_t i = gw; i < it.nslots; i += nw)
      det_short_chain(it.a.det_rows, it.a.det_vals, it.nslots, R, it.a.out, it.dl, i, lane);
  }
}

__global__ void __launch_bounds__(256) det_seg_group_kernel(Strided<DetItem> items, int R) {
  __shared__ float4 part[256];
  const int K = *items.count;
  for (int s = 0; s < K; ++s) {
    const DetItem& it = items[s];
    if (!item_live(it.active)) continue;
    const uint32_t nseg = it.dl.counters[1];
    for (uint32_t g = blockIdx.x; g < nseg; g += gridDim.x) det_segment(it.a.det_vals, R, it.dl, g, part);
  }
}

__global__ void __launch_bounds__(256) det_final_group_kernel(Strided<DetItem> items, int R) {
  __shared__ float4 part[256];
  __shared__ uint32_t s_nlong;
  const int K = *items.count;
  for (int s = 0; s < K; ++s) {
    const DetItem& it = items[s];
    if (!item_live(it.active)) continue;
    const uint32_t nlong = det_take_chains(it.dl, &s_nlong);
    for (uint32_t c = blockIdx.x; c < nlong; c += gridDim.x) det_chain_final(it.a.det_rows, R, it.a.out, it.dl, c, part);
  }
}

// ------------------------------------------- line tiles staged by bulk copy
//
// The non-staged variants (ATOMIC, SORTED) stream the line through shared
// memory: per CTA, tiles of kLineTile entries are copied global -> shared by
// the bulk-copy engine (cp.async.bulk, completion on an mbarrier), double
// buffered, so the next tile is in flight while this one is walked.  The
// keys then come from shared memory (broadcast reads) and the LSU pipe
// carries only the factor-row gathers.  Waits are bounded: a wait that runs
// out sets *err and the whole block leaves after a second bounded wait for
// its copies in flight.

constexpr uint32_t kLineTile = 1024;
constexpr uint32_t kSpinLimit = 1u << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase) {
  for (uint32_t spin = 0; spin < kSpinLimit; ++spin)
    if (mbar_try_wait(bar, phase)) return true;
  return false;
}

template <int R, typename FT, int HW, int NM>
__global__ void __launch_bounds__(kMttkrpThreads, 3)
    mttkrp_tma_kernel(const MttkrpArgs a, int* __restrict__ err) {
  constexpr uint32_t kRec = HW == 2 ? 32 : 16;  // record bytes
  constexpr uint32_t kBuf = kLineTile * kRec;
  extern __shared__ __align__(128) unsigned char sline[];
  __shared__ __align__(8) uint64_t bars[2];
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t ntiles = (a.nnz + kLineTile - 1) / kLineTile;

  auto buf = [&](int b) { return static_cast<void*>(sline + b * kBuf); };
  auto issue = [&](uint32_t tile, int b) {
    const uint32_t s0 = tile * kLineTile;
    const uint32_t n = min(kLineTile, a.nnz - s0);
    mbar_expect_tx(&bars[b], n * kRec);
    bulk_g2s(buf(b), static_cast<const unsigned char*>(a.line) + (size_t)s0 * kRec, n * kRec, &bars[b]);
  };

  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    if (blockIdx.x < ntiles) issue(blockIdx.x, 0);
    if (blockIdx.x + gridDim.x < ntiles) issue(blockIdx.x + gridDim.x, 1);
  }
  uint32_t it = 0;
  for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
    const int b = it & 1;
    const uint32_t phase = (it >> 1) & 1;
    const bool ok = mbar_wait_bounded(&bars[b], phase);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(err, 1);
        // the other buffer may still have a copy in flight: give it a bounded wait
        mbar_wait_bounded(&bars[b ^ 1], ((it + 1) >> 1) & 1);
      }
      return;
    }
    const uint32_t s0 = tile * kLineTile;
    const uint32_t n = min(kLineTile, a.nnz - s0);
    const uint32_t chunk = (n + kMttkrpWarps - 1) / kMttkrpWarps;
    const uint32_t ws = min(warp * chunk, n);
    const uint32_t we = min(ws + chunk, n);
    warp_range<R, FT, HW, NM, true>(a, buf(b), ws, we, false, nullptr, 0);
    __syncthreads();  // every warp is done with buffer b
    if (tid == 0) {
      const uint32_t nt = tile + 2 * gridDim.x;
      if (nt < ntiles) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue(nt, b);
      }
    }
  }
}

// Any rank: one warp per nonzero, lanes stride the rank, scalar atomics.
template <typename FT, int HW>
__global__ void __launch_bounds__(kMttkrpThreads)
    mttkrp_generic_kernel(const MttkrpArgs a, int rank) {
  const int lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = gw; i < a.nnz; i += nw) {
    uint32_t rows[ALTO_MAX_MODES];
    float v;
    if (HW == kDecoded3) {
      const uint4 q = static_cast<const uint4*>(a.line)[i];
      rows[0] = q.x;
      rows[1] = q.y;
      rows[2] = q.z;
#pragma unroll
      for (int m = 3; m < ALTO_MAX_MODES; ++m) rows[m] = 0;
      v = __uint_as_float(q.w);
    } else {
      uint64_t lo, hi;
      rec_read(a.line, HW, i, lo, hi, v);
#pragma unroll
      for (int m = 0; m < ALTO_MAX_MODES; ++m)
        rows[m] = m < a.dec.nmodes ? (uint32_t)line_field(lo, hi, a.dec.pos[m], a.dec.mask[m]) : 0;
    }
    for (int r = lane; r < rank; r += 32) {
      float x = v;
#pragma unroll
      for (int m = 0; m < ALTO_MAX_MODES; ++m) {
        if (m < a.dec.nmodes && m != a.target) {
          const size_t off = (size_t)rows[m] * rank + r;
          if (sizeof(FT) == 4)
            x *= __ldg(static_cast<const float*>(a.fac.f[m]) + off);
          else
            x *= __bfloat162float(static_cast<const __nv_bfloat16*>(a.fac.f[m])[off]);
        }
      }
      atomicAdd(a.out + (size_t)rows[a.target] * rank + r, x);
    }
  }
}

static int g_num_sms = 0;

static int num_sms() {
  if (!g_num_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_num_sms <= 0) g_num_sms = 148;
  }
  return g_num_sms;
}

// Tiles per chunk of the direct walks: up to kChunkTilesMax, keeping at
// least kChunksPerBlock chunks per block so the round robin still balances
// the blocks.
constexpr uint32_t kChunkTilesMax = 8;
constexpr uint32_t kChunksPerBlock = 8;
static uint32_t chunk_tiles_for(uint32_t ntiles, unsigned grid) {
  uint32_t c = kChunkTilesMax;
  while (c > 1 && (uint64_t)ntiles < (uint64_t)c * grid * kChunksPerBlock) c >>= 1;
  return c;
}

template <int R, typename FT, int HW, bool STAGE, int NM, int MINB = 3, int TGT = -1>
static alto_status launch_tile(const MttkrpArgs& a, cudaStream_t st) {
  MttkrpArgs b = a;
  b.stage_rows = STAGE ? kStageBytes / (R * 4) : 0;
  const size_t smem = STAGE ? (size_t)kStageBytes : 0;
  static int blocks_per_sm = 0;
  if (!blocks_per_sm) {
    if (STAGE)
      ALTO_TRY_CUDA(cudaFuncSetAttribute(mttkrp_tile_kernel<R, FT, HW, STAGE, NM, false, MINB, TGT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, kStageBytes));
    else  // no shared memory: all of the unified L1 / shared storage as L1 (factor rows hit it)
      ALTO_TRY_CUDA(cudaFuncSetAttribute(mttkrp_tile_kernel<R, FT, HW, STAGE, NM, false, MINB, TGT>,
                                         cudaFuncAttributePreferredSharedMemoryCarveout, 0));
    ALTO_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &blocks_per_sm, mttkrp_tile_kernel<R, FT, HW, STAGE, NM, false, MINB, TGT>, kMttkrpThreads, smem));
    if (blocks_per_sm < 1) blocks_per_sm = 1;
  }
  unsigned grid = std::min<unsigned>(a.ntiles, (unsigned)(num_sms() * blocks_per_sm));
  if (!grid) return ALTO_OK;
  b.chunk_tiles = chunk_tiles_for(a.ntiles, grid);
  mttkrp_tile_kernel<R, FT, HW, STAGE, NM, false, MINB, TGT><<<grid, kMttkrpThreads, smem, st>>>(b);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

template <int R, typename FT, int HW, int NM>
static alto_status launch_tma(const MttkrpArgs& a, int* err, cudaStream_t st) {
  const size_t smem = 2 * (size_t)kLineTile * (HW == 2 ? 32 : 16);
  static int blocks_per_sm = 0;
  if (!blocks_per_sm) {
    ALTO_TRY_CUDA(cudaFuncSetAttribute(mttkrp_tma_kernel<R, FT, HW, NM>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    ALTO_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &blocks_per_sm, mttkrp_tma_kernel<R, FT, HW, NM>, kMttkrpThreads, smem));
    if (blocks_per_sm < 1) blocks_per_sm = 1;
  }
  const unsigned ntiles = (a.nnz + kLineTile - 1) / kLineTile;
  const unsigned grid = std::min<unsigned>(ntiles, (unsigned)(num_sms() * blocks_per_sm));
  if (!grid) return ALTO_OK;
  mttkrp_tma_kernel<R, FT, HW, NM><<<grid, kMttkrpThreads, smem, st>>>(a, err);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

// Deterministic MTTKRP: the tile kernel in DET mode (float32 factors, the
// specialised ranks) followed by the two fix-up kernels.
template <int R, int HW, int NM>
static alto_status launch_det_nm(const MttkrpArgs& a, const DetLong& dl, cudaStream_t st) {
  static int blocks_per_sm = 0;
  if (!blocks_per_sm) {
    ALTO_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &blocks_per_sm, mttkrp_tile_kernel<R, float, HW, false, NM, true>, kMttkrpThreads, 0));
    if (blocks_per_sm < 1) blocks_per_sm = 1;
  }
  const unsigned grid = std::min<unsigned>(a.ntiles, (unsigned)(num_sms() * blocks_per_sm));
  if (!grid) return ALTO_OK;
  mttkrp_tile_kernel<R, float, HW, false, NM, true><<<grid, kMttkrpThreads, 0, st>>>(a);
  ALTO_LAUNCHED();
  const uint32_t nslots = a.ntiles * kMttkrpWarps * LaneWidth<R>::NPW * 2;
  const unsigned g1 = std::min<unsigned>((nslots + 7) / 8, (unsigned)num_sms() * 16);
  det_fix_short_kernel<<<g1, 256, 0, st>>>(a.det_rows, a.det_vals, nslots, R, a.out, dl);
  ALTO_LAUNCHED();
  det_fix_seg_kernel<<<(unsigned)num_sms() * 4, 256, 0, st>>>(a.det_vals, R, dl);
  ALTO_LAUNCHED();
  det_fix_final_kernel<<<(unsigned)num_sms(), 256, 0, st>>>(a.det_rows, R, a.out, dl);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

template <int R, int HW>
static alto_status launch_det(const MttkrpArgs& a, const DetLong& dl, cudaStream_t st) {
  if constexpr (HW == kDecoded3) return launch_det_nm<R, HW, 3>(a, dl, st);
  switch (a.dec.nmodes) {
    case 3: return launch_det_nm<R, HW, 3>(a, dl, st);
    case 4: return launch_det_nm<R, HW, 4>(a, dl, st);
    case 5: return launch_det_nm<R, HW, 5>(a, dl, st);
    default: return launch_det_nm<R, HW, ALTO_MAX_MODES>(a, dl, st);
  }
}

template <int HW>
static alto_status launch_det_rank(const MttkrpArgs& a, int rank, const DetLong& dl,
                                   cudaStream_t st) {
  switch (rank) {
    case 8: return launch_det<8, HW>(a, dl, st);
    case 16: return launch_det<16, HW>(a, dl, st);
    case 32: return launch_det<32, HW>(a, dl, st);
    case 64: return launch_det<64, HW>(a, dl, st);
    case 128: return launch_det<128, HW>(a, dl, st);
    default: break;
  }
  set_error("the deterministic MTTKRP takes rank 8, 16, 32, 64 or 128 (got %d)", rank);
  return ALTO_ERR_UNSUPPORTED;
}

// Lane groups per warp of the specialised kernels at this rank.
static uint32_t groups_per_warp(int rank) {
  switch (rank) {
    case 8: return LaneWidth<8>::NPW;
    case 16: return LaneWidth<16>::NPW;
    case 32: return LaneWidth<32>::NPW;
    case 64: return LaneWidth<64>::NPW;
    default: return LaneWidth<128>::NPW;
  }
}

bool deterministic_supported(int rank, alto_dtype fdtype) {
  return fdtype == ALTO_F32 && (rank == 8 || rank == 16 || rank == 32 || rank == 64 || rank == 128);
}

template <int R, typename FT, int HW>
static alto_status launch_modes(const MttkrpArgs& a, bool stage, bool bulk_feed, int dense, int* err,
                                cudaStream_t st) {
  if constexpr (HW == kDecoded3) {  // sorted 3-mode copies: no staging
    if (dense == 2 && !bulk_feed) {  // the target mode fixed at compile time
      switch (a.target) {
        case 0: return launch_tile<R, FT, HW, false, 3, 5, 0>(a, st);
        case 1: return launch_tile<R, FT, HW, false, 3, 5, 1>(a, st);
        default: return launch_tile<R, FT, HW, false, 3, 5, 2>(a, st);
      }
    }
    if (dense && !bulk_feed) return launch_tile<R, FT, HW, false, 3, 5>(a, st);
    return bulk_feed ? launch_tma<R, FT, HW, 3>(a, err, st) : launch_tile<R, FT, HW, false, 3>(a, st);
  } else {
#define NM_CASE(NN)                                                                   \
  case NN:                                                                            \
    if (stage) return launch_tile<R, FT, HW, true, NN>(a, st);                        \
    return bulk_feed ? launch_tma<R, FT, HW, NN>(a, err, st) : launch_tile<R, FT, HW, false, NN>(a, st);
  switch (a.dec.nmodes) {
    NM_CASE(3)
    NM_CASE(4)
    NM_CASE(5)
    default:
      return stage ? launch_tile<R, FT, HW, true, ALTO_MAX_MODES>(a, st)
                   : launch_tile<R, FT, HW, false, ALTO_MAX_MODES>(a, st);
  }
#undef NM_CASE
  }
}

template <typename FT, int HW>
static alto_status launch_rank(const MttkrpArgs& a, int rank, bool stage, bool bulk_feed, int dense,
                               bool aligned, int* err, cudaStream_t st) {
  if (aligned) {
#define RANK_CASE(RR) \
  case RR:            \
    return launch_modes<RR, FT, HW>(a, stage, bulk_feed, dense, err, st);
    switch (rank) {
      RANK_CASE(8)
      RANK_CASE(16)
      RANK_CASE(32)
      RANK_CASE(64)
      RANK_CASE(128)
      default: break;
    }
#undef RANK_CASE
  }
  unsigned grid = (unsigned)std::min<uint64_t>((a.nnz + 7) / 8, (uint64_t)num_sms() * 16);
  if (!grid) return ALTO_OK;
  mttkrp_generic_kernel<FT, HW><<<grid, kMttkrpThreads, 0, st>>>(a, rank);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

// Fraction of the mode's tiles whose output interval fits the staging buffer
// at this rank and is at most half the tile (so staging saves updates).
static double stageable_fraction(const alto_tensor* t, int mode, int rank) {
  const auto& v = t->tile_len_sorted[mode];
  if (v.empty()) return 0.0;
  const uint32_t cap = std::min<uint32_t>(kStageBytes / (rank * 4), t->tile_nnz / 2);
  const size_t n = std::upper_bound(v.begin(), v.end(), cap) - v.begin();
  return (double)n / (double)v.size();
}

static const TuneEntry* tuned_entry(const alto_tensor* t, int mode, int rank, alto_dtype fdtype) {
  for (const auto& e : t->tuned)
    if (e.mode == mode && e.rank == rank && e.fdtype == (int)fdtype) return &e;
  return nullptr;
}

alto_mttkrp_variant choose_variant(const alto_tensor* t, int mode, int rank, alto_dtype fdtype) {
  if (const TuneEntry* e = tuned_entry(t, mode, rank, fdtype)) return e->variant;
  // The reference's rule (include/alto.hpp:835-846) picks atomics for long
  // low-reuse modes, the stream kernel for the stream mode and da_mem
  // otherwise.  On the device: stage where the tiles' intervals fit, walk a
  // row-sorted copy where rows are reused but the intervals are too wide,
  // else plain vector atomics.
  const uint64_t dim = t->dims[mode];
  const uint64_t reuse = dim ? t->nnz / dim : 0;
  if (mode == t->stream_mode && dim * rank * 4 <= (uint64_t)kStageBytes) return ALTO_MTTKRP_STREAM;
  if (stageable_fraction(t, mode, rank) >= 0.5) return ALTO_MTTKRP_STAGED;
  if (reuse > 4) return ALTO_MTTKRP_SORTED;
  return ALTO_MTTKRP_ATOMIC;
}

alto_status run_mttkrp(alto_tensor* t, int mode, const void* const* factors, alto_dtype fdtype,
                       int rank, float* out, int accumulate, alto_mttkrp_variant variant,
                       cudaStream_t st) {
  return run_mttkrp_feed(t, mode, factors, fdtype, rank, out, accumulate, variant, -1, st);
}

// feed: 1 streams the line through shared memory by bulk copy, 0 loads it
// directly, 2 loads it directly with five blocks per SM (decoded 3-mode
// copies: at most 48 registers a thread; six, at 40, measured slower), 3 as
// 2 with the target mode fixed at compile time, -1 uses the autotuned choice
// (direct when untuned).
alto_status run_mttkrp_feed(alto_tensor* t, int mode, const void* const* factors, alto_dtype fdtype,
                            int rank, float* out, int accumulate, alto_mttkrp_variant variant, int feed,
                            cudaStream_t st) {
  if (feed < 0) {
    const TuneEntry* e = variant == ALTO_MTTKRP_AUTO ? tuned_entry(t, mode, rank, fdtype) : nullptr;
    feed = e ? e->feed : 0;
  }
  if (variant == ALTO_MTTKRP_AUTO) variant = choose_variant(t, mode, rank, fdtype);
  const bool det = variant == ALTO_MTTKRP_DETERMINISTIC;
  if (det && !deterministic_supported(rank, fdtype)) {
    set_error("the deterministic MTTKRP takes float32 factors at rank 8, 16, 32, 64 or 128");
    return ALTO_ERR_UNSUPPORTED;
  }
  if (!accumulate)
    ALTO_TRY_CUDA(cudaMemsetAsync(out, 0, (size_t)t->dims[mode] * rank * sizeof(float), st));
  if (!t->nnz) return ALTO_OK;
  if (det) {
    DetItem it;
    ALTO_TRY(det_prepare(t, mode, factors, rank, out, &it, st));
    if (it.hw == 0) return launch_det_rank<0>(it.a, rank, it.dl, st);
    if (it.hw == 1) return launch_det_rank<1>(it.a, rank, it.dl, st);
    if (it.hw == kDecoded3) return launch_det_rank<kDecoded3>(it.a, rank, it.dl, st);
    return launch_det_rank<2>(it.a, rank, it.dl, st);
  }
  MttkrpArgs a{};
  a.line = t->line.p;
  a.tile_iv = t->tile_iv.as<uint32_t>();
  a.ntiles = t->ntiles;
  int hw = t->dec.hi_words;  // record format of the line walked
  if (variant == ALTO_MTTKRP_SORTED) {
    if (!t->sorted[mode].ready || t->sorted[mode].for_nnz != t->nnz)
      ALTO_TRY(build_sorted_line(t, mode, st));
    const SortedLine& s = t->sorted[mode];
    a.line = s.line.p;
    a.tile_iv = s.tile_iv.as<uint32_t>();
    a.ntiles = s.ntiles;
    hw = s.hw;
  }
  a.nnz = (uint32_t)t->nnz;
  a.tile_nnz = t->tile_nnz;
  a.target = mode;
  a.dec = t->dec;
  a.out = out;
  bool aligned = (reinterpret_cast<uintptr_t>(out) % 16) == 0;
  const int esz = fdtype == ALTO_BF16 ? 2 : 4;
  for (int m = 0; m < t->nmodes; ++m) {
    a.fac.f[m] = factors[m];
    if (m != mode && (reinterpret_cast<uintptr_t>(factors[m]) % (4 * esz)) != 0) aligned = false;
  }
  const bool stage = variant == ALTO_MTTKRP_STAGED || variant == ALTO_MTTKRP_STREAM;
  ALTO_TRY(ensure_error_words(t, st));
  int* err = t->err.as<int>();
  const bool bulk = feed == 1;
  const int dense = feed == 2 ? 1 : feed == 3 ? 2 : 0;
  if (fdtype == ALTO_BF16) {
    if (hw == 0) return launch_rank<__nv_bfloat16, 0>(a, rank, stage, bulk, 0, aligned, err, st);
    if (hw == 1) return launch_rank<__nv_bfloat16, 1>(a, rank, stage, bulk, 0, aligned, err, st);
    if (hw == kDecoded3)
      return launch_rank<__nv_bfloat16, kDecoded3>(a, rank, false, bulk, dense, aligned, err, st);
    return launch_rank<__nv_bfloat16, 2>(a, rank, stage, bulk, 0, aligned, err, st);
  }
  if (hw == 0) return launch_rank<float, 0>(a, rank, stage, bulk, 0, aligned, err, st);
  if (hw == 1) return launch_rank<float, 1>(a, rank, stage, bulk, 0, aligned, err, st);
  if (hw == kDecoded3) return launch_rank<float, kDecoded3>(a, rank, false, bulk, dense, aligned, err, st);
  return launch_rank<float, 2>(a, rank, stage, bulk, 0, aligned, err, st);
}

alto_status det_prepare(alto_tensor* t, int mode, const void* const* factors, int rank, float* out, DetItem* item,
                        cudaStream_t st) {
  if (!deterministic_supported(rank, ALTO_F32)) {
    set_error("the deterministic MTTKRP takes float32 factors at rank 8, 16, 32, 64 or 128");
    return ALTO_ERR_UNSUPPORTED;
  }
  MttkrpArgs a{};
  a.line = t->line.p;
  a.tile_iv = t->tile_iv.as<uint32_t>();
  a.ntiles = t->nnz ? t->ntiles : 0;
  int hw = t->dec.hi_words;
  // (a mode of length 1 is already in row order in the ALTO line)
  if (t->dims[mode] > 1 && t->nnz) {
    if (!t->sorted[mode].ready || t->sorted[mode].for_nnz != t->nnz) ALTO_TRY(build_sorted_line(t, mode, st));
    const SortedLine& s = t->sorted[mode];
    a.line = s.line.p;
    a.tile_iv = s.tile_iv.as<uint32_t>();
    a.ntiles = s.ntiles;
    hw = s.hw;
  }
  a.nnz = (uint32_t)t->nnz;
  a.tile_nnz = t->tile_nnz;
  a.target = mode;
  a.dec = t->dec;
  a.out = out;
  bool aligned = (reinterpret_cast<uintptr_t>(out) % 16) == 0;
  for (int m = 0; m < t->nmodes; ++m) {
    a.fac.f[m] = factors[m];
    if (m != mode && (reinterpret_cast<uintptr_t>(factors[m]) % 16) != 0) aligned = false;
  }
  if (!aligned) {
    set_error("the deterministic MTTKRP needs 16-byte aligned factors and output");
    return ALTO_ERR_UNSUPPORTED;
  }
  const uint64_t nslots = (uint64_t)a.ntiles * kMttkrpWarps * groups_per_warp(rank) * 2;
  ALTO_TRY(tensor_ensure(t, t->det_rows, std::max<uint64_t>(nslots, 1) * 4));
  ALTO_TRY(tensor_ensure(t, t->det_vals, std::max<uint64_t>(nslots, 1) * rank * 4));
  // long chains: each has more than kShortChain slots; segments:
  // sum over chains of ceil(len / kChainSeg)
  const uint64_t max_chains = nslots / (kShortChain + 1) + 1;
  const uint64_t max_segs = nslots / kChainSeg + max_chains;
  auto up = [](uint64_t x) { return (x + 255) & ~uint64_t(255); };
  const uint64_t o_chains = 256, o_segs = o_chains + up(max_chains * sizeof(uint4)),
                 o_part = o_segs + up(max_segs * sizeof(uint2)), bytes = o_part + max_segs * rank * 4;
  const size_t before = t->det_long.bytes;  // a new allocation starts with zero counters
  ALTO_TRY(tensor_ensure(t, t->det_long, bytes));
  if (t->det_long.bytes != before) ALTO_TRY_CUDA(cudaMemsetAsync(t->det_long.p, 0, 16, st));
  a.det_rows = t->det_rows.as<uint32_t>();
  a.det_vals = t->det_vals.as<float>();
  char* base = t->det_long.as<char>();
  item->a = a;
  item->dl = DetLong{reinterpret_cast<uint32_t*>(base), reinterpret_cast<uint4*>(base + o_chains),
                     reinterpret_cast<uint2*>(base + o_segs), reinterpret_cast<float*>(base + o_part)};
  item->nslots = (uint32_t)nslots;
  item->hw = hw;
  item->out_floats = t->dims[mode] * (uint64_t)rank;
  item->active = nullptr;
  return ALTO_OK;
}

template <int R, int HW, int NM>
static alto_status det_group_nm(Strided<DetItem> items, const uint32_t* tile_off, cudaStream_t st) {
  static int blocks_per_sm = 0;
  if (!blocks_per_sm) {
    ALTO_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, det_tile_group_kernel<R, HW, NM>,
                                                                kMttkrpThreads, 0));
    if (blocks_per_sm < 1) blocks_per_sm = 1;
  }
  const unsigned sm = (unsigned)num_sms();
  det_zero_group_kernel<<<sm * 4, 256, 0, st>>>(items);
  ALTO_LAUNCHED();
  det_tile_group_kernel<R, HW, NM><<<sm * blocks_per_sm, kMttkrpThreads, 0, st>>>(items, tile_off);
  ALTO_LAUNCHED();
  det_short_group_kernel<<<sm * 16, 256, 0, st>>>(items, R);
  ALTO_LAUNCHED();
  det_seg_group_kernel<<<sm * 4, 256, 0, st>>>(items, R);
  ALTO_LAUNCHED();
  det_final_group_kernel<<<sm, 256, 0, st>>>(items, R);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

template <int R>
static alto_status det_group_rank(Strided<DetItem> items, const uint32_t* tile_off, int hw, int nmodes,
                                  cudaStream_t st) {
  if (hw == kDecoded3 && nmodes == 3) return det_group_nm<R, kDecoded3, 3>(items, tile_off, st);
#define DG_CASE(H, NN) \
  if (hw == H && nmodes == NN) return det_group_nm<R, H, NN>(items, tile_off, st);
  DG_CASE(0, 3) DG_CASE(0, 4) DG_CASE(0, 5)
  DG_CASE(1, 3) DG_CASE(1, 4) DG_CASE(1, 5)
  DG_CASE(2, 3) DG_CASE(2, 4) DG_CASE(2, 5)
#undef DG_CASE
  set_error("grouped MTTKRP: record format %d with %d modes is not supported", hw, nmodes);
  return ALTO_ERR_UNSUPPORTED;
}

alto_status det_group_launch(Strided<DetItem> items, const uint32_t* tile_off, int rank, int hw, int nmodes,
                             cudaStream_t st) {
  switch (rank) {
    case 8: return det_group_rank<8>(items, tile_off, hw, nmodes, st);
    case 16: return det_group_rank<16>(items, tile_off, hw, nmodes, st);
    case 32: return det_group_rank<32>(items, tile_off, hw, nmodes, st);
    case 64: return det_group_rank<64>(items, tile_off, hw, nmodes, st);
    default: break;
  }
  set_error("grouped MTTKRP: rank %d is not supported (8, 16, 32 or 64)", rank);
  return ALTO_ERR_UNSUPPORTED;
}

// Time every applicable variant once per mode (after one warm run) into a
// scratch output and record the fastest for ALTO_MTTKRP_AUTO.  Synchronous;
// not for use inside stream capture.
alto_status autotune(alto_tensor* t, const void* const* factors, alto_dtype fdtype, int rank,
                     cudaStream_t st, alto_mttkrp_variant* chosen) {
  uint64_t max_dim = 0;
  for (int m = 0; m < t->nmodes; ++m) max_dim = std::max<uint64_t>(max_dim, t->dims[m]);
  DevBuf out;
  ALTO_TRY(out.ensure(max_dim * rank * 4));
  cudaEvent_t e0, e1;
  ALTO_TRY_CUDA(cudaEventCreate(&e0));
  ALTO_TRY_CUDA(cudaEventCreate(&e1));
  std::vector<TuneEntry> keep;
  for (const auto& e : t->tuned)
    if (!(e.rank == rank && e.fdtype == (int)fdtype)) keep.push_back(e);
  t->tuned = keep;
  alto_status status = ALTO_OK;
  for (int m = 0; m < t->nmodes && status == ALTO_OK; ++m) {
    struct Cand {
      alto_mttkrp_variant v;
      int feed;
    };
    const Cand cands[] = {{ALTO_MTTKRP_ATOMIC, 0}, {ALTO_MTTKRP_ATOMIC, 1}, {ALTO_MTTKRP_STAGED, 0},
                          {ALTO_MTTKRP_SORTED, 0}, {ALTO_MTTKRP_SORTED, 1}, {ALTO_MTTKRP_SORTED, 2},
                          {ALTO_MTTKRP_SORTED, 3}};
    alto_mttkrp_variant best = ALTO_MTTKRP_ATOMIC;
    int best_feed = 0;
    float best_ms = 1e30f;
    for (const Cand& c : cands) {
      const alto_mttkrp_variant v = c.v;
      if (v == ALTO_MTTKRP_STAGED && stageable_fraction(t, m, rank) == 0.0) continue;
      if (v == ALTO_MTTKRP_SORTED && t->nnz / std::max<uint64_t>(t->dims[m], 1) < 2) continue;
      if (c.feed >= 2 && t->nmodes != 3) continue;  // (decoded 3-mode copies only)
      status = run_mttkrp_feed(t, m, factors, fdtype, rank, out.as<float>(), 0, v, c.feed, st);  // warm / build
      if (status != ALTO_OK) break;
      cudaEventRecord(e0, st);
      status = run_mttkrp_feed(t, m, factors, fdtype, rank, out.as<float>(), 0, v, c.feed, st);
      cudaEventRecord(e1, st);
      if (status != ALTO_OK) break;
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        status = cuda_status(cudaGetLastError(), "autotune", __FILE__, __LINE__);
        break;
      }
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < best_ms) {
        best_ms = ms;
        best = v;
        best_feed = c.feed;
      }
    }
    t->tuned.push_back({m, rank, (int)fdtype, best, best_feed});
    if (chosen) chosen[m] = best;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return status;
}

}  // namespace alto
