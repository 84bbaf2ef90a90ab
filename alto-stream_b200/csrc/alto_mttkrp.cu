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

#include "alto_internal.cuh"

namespace alto {

constexpr uint32_t kNoRow = 0xffffffffu;
constexpr int kMttkrpThreads = 256;
constexpr int kMttkrpWarps = kMttkrpThreads / 32;
constexpr int kStageBytes = 96 * 1024;

struct FactorSet {
  const void* f[ALTO_MAX_MODES];
};

struct MttkrpArgs {
  const uint64_t* klo;
  const void* khi;
  const float* vals;
  const uint32_t* tile_iv;
  uint32_t nnz;
  uint32_t tile_nnz;
  uint32_t ntiles;
  int target;
  int stage_rows;  // rows of the shared staging buffer (0: never stage)
  LineDecode dec;
  FactorSet fac;
  float* out;
};

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

template <int HW>
__device__ __forceinline__ uint64_t hi_word(const void* khi, uint32_t i) {
  if (HW == 1) return __ldg(static_cast<const uint32_t*>(khi) + i);
  if (HW == 2) return __ldg(static_cast<const uint64_t*>(khi) + i);
  return 0;
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

// V consecutive floats of a factor row (V = 4 or 8 or 16).
template <typename FT, int V>
__device__ __forceinline__ void load_row(const void* base, size_t off, float (&x)[V]) {
#pragma unroll
  for (int q = 0; q < V / 4; ++q) {
    const float4 f = load4<FT>(base, off + q * 4);
    x[q * 4 + 0] = f.x;
    x[q * 4 + 1] = f.y;
    x[q * 4 + 2] = f.z;
    x[q * 4 + 3] = f.w;
  }
}

// One update of output row `row` with this lane's V floats (at column c0).
template <int R, int V>
__device__ __forceinline__ void flush_row(bool staged, float* smem, uint32_t iv_start, float* out,
                                          uint32_t row, int c0, const float (&acc)[V]) {
  if (staged) {
    float* s = smem + (size_t)(row - iv_start) * R + c0;
#pragma unroll
    for (int q = 0; q < V; ++q) atomicAdd(s + q, acc[q]);
  } else {
    float* o = out + (size_t)row * R + c0;
#pragma unroll
    for (int q = 0; q < V / 4; ++q)
      atomicAdd(reinterpret_cast<float4*>(o + q * 4),
                make_float4(acc[q * 4], acc[q * 4 + 1], acc[q * 4 + 2], acc[q * 4 + 3]));
  }
}

// Floats per lane for rank R: 8 where the rank allows (R >= 8), else R.
template <int R>
struct LaneWidth {
  static constexpr int V = R >= 8 ? 8 : R;
  static constexpr int G = R / V;     // lanes per nonzero
  static constexpr int NPW = 32 / G;  // groups (nonzeros in flight) per warp
};

// Walk line range [ws, we) with one warp: the range is split into NPW
// contiguous sub-ranges, one per lane group; a group walks its sub-range in
// order, two nonzeros per iteration (loads of both issued first), keeps the
// running sum of the current output row in registers and updates the output
// once per run of equal rows.  NM is the mode count (3, 4, 5 specialised as
// in the reference's ALTO_MODES_SPECIALIZED, 8 for the rest).
template <int R, typename FT, int HW, int NM>
__device__ __forceinline__ void warp_range(const MttkrpArgs& a, uint32_t ws, uint32_t we,
                                           bool staged, float* smem, uint32_t iv_start) {
  using LW = LaneWidth<R>;
  constexpr int V = LW::V, G = LW::G, NPW = LW::NPW;
  constexpr int U = NM <= 3 ? 2 : 1;  // nonzeros per group per iteration
  const int lane = threadIdx.x & 31;
  const int grp = lane / G, sub = lane % G;
  const int c0 = sub * V;
  const uint32_t sublen = (we - ws + NPW - 1) / NPW;
  const uint32_t gs = min(ws + grp * sublen, we);
  const uint32_t ge = min(gs + sublen, we);
  float acc[V];
#pragma unroll
  for (int q = 0; q < V; ++q) acc[q] = 0.f;
  uint32_t cur = kNoRow;

  for (uint32_t k = 0; k < sublen; k += U) {
    uint32_t w[U][4];
    float v[U];
    bool valid[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint32_t i = gs + k + u;
      valid[u] = i < ge;
      const uint64_t lo = valid[u] ? __ldg(a.klo + i) : 0;
      const uint64_t hi = valid[u] ? hi_word<HW>(a.khi, i) : 0;
      v[u] = valid[u] ? __ldg(a.vals + i) : 0.f;
      w[u][0] = (uint32_t)lo;
      w[u][1] = (uint32_t)(lo >> 32);
      w[u][2] = (uint32_t)hi;
      w[u][3] = (uint32_t)(hi >> 32);
    }
    // factor rows of the NM-1 input modes (j-th input mode m = j, or j+1
    // past the target)
    float f[U][NM - 1][V];
#pragma unroll
    for (int u = 0; u < U; ++u) {
#pragma unroll
      for (int j = 0; j < NM - 1; ++j) {
        const int m = j < a.target ? j : j + 1;
        if (m < a.dec.nmodes && valid[u]) {
          const uint32_t r = field32(w[u][0], w[u][1], w[u][2], w[u][3], a.dec.pos[m], (uint32_t)a.dec.mask[m]);
          load_row<FT, V>(a.fac.f[m], (size_t)r * R + c0, f[u][j]);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (!valid[u]) continue;
      float p[V];
#pragma unroll
      for (int q = 0; q < V; ++q) p[q] = v[u];
#pragma unroll
      for (int j = 0; j < NM - 1; ++j)
        if ((j < a.target ? j : j + 1) < a.dec.nmodes)
#pragma unroll
          for (int q = 0; q < V; ++q) p[q] *= f[u][j][q];
      const uint32_t row =
          field32(w[u][0], w[u][1], w[u][2], w[u][3], a.dec.pos[a.target], (uint32_t)a.dec.mask[a.target]);
      if (row != cur) {
        if (cur != kNoRow) flush_row<R, V>(staged, smem, iv_start, a.out, cur, c0, acc);
        cur = row;
#pragma unroll
        for (int q = 0; q < V; ++q) acc[q] = p[q];
      } else {
#pragma unroll
        for (int q = 0; q < V; ++q) acc[q] += p[q];
      }
    }
  }
  if (cur != kNoRow) flush_row<R, V>(staged, smem, iv_start, a.out, cur, c0, acc);
}

template <int R, typename FT, int HW, bool STAGE, int NM>
__global__ void __launch_bounds__(kMttkrpThreads, 3)
    mttkrp_tile_kernel(const MttkrpArgs a) {
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  const int warp = threadIdx.x >> 5;
  const int N = a.dec.nmodes;
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
    warp_range<R, FT, HW, NM>(a, ws, we, staged, smem, iv_start);
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

// Any rank: one warp per nonzero, lanes stride the rank, scalar atomics.
template <typename FT, int HW>
__global__ void __launch_bounds__(kMttkrpThreads)
    mttkrp_generic_kernel(const MttkrpArgs a, int rank) {
  const int lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = gw; i < a.nnz; i += nw) {
    const uint64_t lo = __ldg(a.klo + i);
    const uint64_t hi = hi_word<HW>(a.khi, i);
    const float v = __ldg(a.vals + i);
    uint32_t rows[ALTO_MAX_MODES];
#pragma unroll
    for (int m = 0; m < ALTO_MAX_MODES; ++m)
      rows[m] = m < a.dec.nmodes ? (uint32_t)line_field(lo, hi, a.dec.pos[m], a.dec.mask[m]) : 0;
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

template <int R, typename FT, int HW, bool STAGE, int NM>
static alto_status launch_tile(const MttkrpArgs& a, cudaStream_t st) {
  MttkrpArgs b = a;
  b.stage_rows = STAGE ? kStageBytes / (R * 4) : 0;
  const size_t smem = STAGE ? (size_t)kStageBytes : 0;
  static int blocks_per_sm = 0;
  if (!blocks_per_sm) {
    if (STAGE)
      ALTO_TRY_CUDA(cudaFuncSetAttribute(mttkrp_tile_kernel<R, FT, HW, STAGE, NM>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, kStageBytes));
    ALTO_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &blocks_per_sm, mttkrp_tile_kernel<R, FT, HW, STAGE, NM>, kMttkrpThreads, smem));
    if (blocks_per_sm < 1) blocks_per_sm = 1;
  }
  unsigned grid = std::min<unsigned>(a.ntiles, (unsigned)(num_sms() * blocks_per_sm));
  if (!grid) return ALTO_OK;
  mttkrp_tile_kernel<R, FT, HW, STAGE, NM><<<grid, kMttkrpThreads, smem, st>>>(b);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

template <int R, typename FT, int HW>
static alto_status launch_modes(const MttkrpArgs& a, bool stage, cudaStream_t st) {
#define NM_CASE(NN)                                                                        \
  case NN:                                                                                 \
    return stage ? launch_tile<R, FT, HW, true, NN>(a, st) : launch_tile<R, FT, HW, false, NN>(a, st);
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

template <typename FT, int HW>
static alto_status launch_rank(const MttkrpArgs& a, int rank, bool stage, bool aligned,
                               cudaStream_t st) {
  if (aligned) {
#define RANK_CASE(RR) \
  case RR:            \
    return launch_modes<RR, FT, HW>(a, stage, st);
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

alto_mttkrp_variant choose_variant(const alto_tensor* t, int mode, int rank, alto_dtype fdtype) {
  for (const auto& e : t->tuned)
    if (e.mode == mode && e.rank == rank && e.fdtype == (int)fdtype) return e.variant;
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
  if (variant == ALTO_MTTKRP_AUTO) variant = choose_variant(t, mode, rank, fdtype);
  if (!accumulate)
    ALTO_TRY_CUDA(cudaMemsetAsync(out, 0, (size_t)t->dims[mode] * rank * sizeof(float), st));
  if (!t->nnz) return ALTO_OK;
  MttkrpArgs a{};
  a.klo = t->klo.as<uint64_t>();
  a.khi = t->khi.p;
  a.vals = t->vals.as<float>();
  a.tile_iv = t->tile_iv.as<uint32_t>();
  a.ntiles = t->ntiles;
  if (variant == ALTO_MTTKRP_SORTED) {
    if (!t->sorted[mode].ready || t->sorted[mode].for_nnz != t->nnz)
      ALTO_TRY(build_sorted_line(t, mode, st));
    const SortedLine& s = t->sorted[mode];
    a.klo = s.klo.as<uint64_t>();
    a.khi = s.khi.p;
    a.vals = s.vals.as<float>();
    a.tile_iv = s.tile_iv.as<uint32_t>();
    a.ntiles = s.ntiles;
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
  const int hw = t->dec.hi_words;
  if (fdtype == ALTO_BF16) {
    if (hw == 0) return launch_rank<__nv_bfloat16, 0>(a, rank, stage, aligned, st);
    if (hw == 1) return launch_rank<__nv_bfloat16, 1>(a, rank, stage, aligned, st);
    return launch_rank<__nv_bfloat16, 2>(a, rank, stage, aligned, st);
  }
  if (hw == 0) return launch_rank<float, 0>(a, rank, stage, aligned, st);
  if (hw == 1) return launch_rank<float, 1>(a, rank, stage, aligned, st);
  return launch_rank<float, 2>(a, rank, stage, aligned, st);
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
    const alto_mttkrp_variant cands[] = {ALTO_MTTKRP_ATOMIC, ALTO_MTTKRP_STAGED, ALTO_MTTKRP_SORTED};
    alto_mttkrp_variant best = ALTO_MTTKRP_ATOMIC;
    float best_ms = 1e30f;
    for (auto v : cands) {
      if (v == ALTO_MTTKRP_STAGED && stageable_fraction(t, m, rank) == 0.0) continue;
      if (v == ALTO_MTTKRP_SORTED && t->nnz / std::max<uint64_t>(t->dims[m], 1) < 2) continue;
      status = run_mttkrp(t, m, factors, fdtype, rank, out.as<float>(), 0, v, st);  // warm / build
      if (status != ALTO_OK) break;
      cudaEventRecord(e0, st);
      status = run_mttkrp(t, m, factors, fdtype, rank, out.as<float>(), 0, v, st);
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
      }
    }
    t->tuned.push_back({m, rank, (int)fdtype, best});
    if (chosen) chosen[m] = best;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return status;
}

}  // namespace alto
