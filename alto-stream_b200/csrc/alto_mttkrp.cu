// ALTO MTTKRP on the device.
//
// Reference: mttkrp_alto_par and its variants (jeewhanchoi/ALTO-stream
// include/alto.hpp:826-908 dispatch, :1349-1407 atomic, :1544-1634
// da_mem_pull, :1636-1706 stream, :1708-1801 op_sched).  For every nonzero
// x = (i_0..i_{N-1}, v) of the line:  out[i_n, :] += v * prod_{m != n} U_m[i_m, :].
//
// Device design.  The line is cut into tiles of tile_nnz nonzeros (the
// reference's partitions, sized for the GPU); a persistent grid walks the
// tiles.  Inside a warp, G = R/4 lanes own one nonzero (each lane a float4
// slice of the rank), so a warp step covers 32/G consecutive nonzeros and
// every factor-row gather is a fully used 16-byte-per-lane load.  Products of
// consecutive nonzeros with the same output row are merged by a segmented
// suffix sum over the warp's groups, and a run that continues into the next
// step is carried in registers, so each run of equal rows issues one update.
// Updates go either to
//   * shared memory, when the tile's output interval (rows between its
//     smallest and largest target index, the reference's prtn_intervals)
//     fits the staging buffer -- the reference's da_mem, on chip -- and the
//     staged rows are flushed once per tile with vector atomics; or
//   * global memory with 16-byte vector atomics (red.global.add.v4.f32),
//     the reference's atomic variant.
// The single-row output of the stream mode is the degenerate staged case.
#include <algorithm>

#include "alto_internal.cuh"

namespace alto {

constexpr uint32_t kNoRow = 0xffffffffu;
constexpr int kMttkrpThreads = 256;
constexpr int kMttkrpWarps = kMttkrpThreads / 32;

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

__device__ __forceinline__ float4 shfl4(float4 v, int src) {
  float4 r;
  r.x = __shfl_sync(0xffffffffu, v.x, src);
  r.y = __shfl_sync(0xffffffffu, v.y, src);
  r.z = __shfl_sync(0xffffffffu, v.z, src);
  r.w = __shfl_sync(0xffffffffu, v.w, src);
  return r;
}

__device__ __forceinline__ float4 shfl4_down(float4 v, int d) {
  float4 r;
  r.x = __shfl_down_sync(0xffffffffu, v.x, d);
  r.y = __shfl_down_sync(0xffffffffu, v.y, d);
  r.z = __shfl_down_sync(0xffffffffu, v.z, d);
  r.w = __shfl_down_sync(0xffffffffu, v.w, d);
  return r;
}

__device__ __forceinline__ void add4(float4& a, const float4& b) {
  a.x += b.x;
  a.y += b.y;
  a.z += b.z;
  a.w += b.w;
}

template <int HW>
__device__ __forceinline__ uint64_t hi_word(const void* khi, uint32_t i) {
  if (HW == 1) return __ldg(static_cast<const uint32_t*>(khi) + i);
  if (HW == 2) return __ldg(static_cast<const uint64_t*>(khi) + i);
  return 0;
}

// One update of output row `row` with this lane's float4 slice.
template <int R>
__device__ __forceinline__ void flush_row(bool staged, float* smem, uint32_t iv_start,
                                          float* out, uint32_t row, int sub, const float4& acc) {
  if (staged) {
    float* s = smem + (size_t)(row - iv_start) * R + sub * 4;
    atomicAdd(s + 0, acc.x);
    atomicAdd(s + 1, acc.y);
    atomicAdd(s + 2, acc.z);
    atomicAdd(s + 3, acc.w);
  } else {
    atomicAdd(reinterpret_cast<float4*>(out + (size_t)row * R + sub * 4), acc);
  }
}

// Process line range [ws, we) with one warp (see the file comment).
template <int R, typename FT, int HW>
__device__ __forceinline__ void warp_range(const MttkrpArgs& a, uint32_t ws, uint32_t we,
                                           bool staged, float* smem, uint32_t iv_start) {
  constexpr int G = R / 4;
  constexpr int NPW = 32 / G;
  const int lane = threadIdx.x & 31;
  const int grp = lane / G, sub = lane % G;
  float4 carry = make_float4(0.f, 0.f, 0.f, 0.f);
  uint32_t carry_row = kNoRow;

  for (uint32_t base = ws; base < we; base += NPW) {
    const uint32_t i = base + grp;
    const bool valid = i < we;
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    uint32_t row = kNoRow;
    if (valid) {
      const uint64_t lo = __ldg(a.klo + i);
      const uint64_t hi = hi_word<HW>(a.khi, i);
      const float v = __ldg(a.vals + i);
      acc = make_float4(v, v, v, v);
#pragma unroll
      for (int m = 0; m < ALTO_MAX_MODES; ++m) {
        if (m < a.dec.nmodes && m != a.target) {
          const uint32_t r = (uint32_t)line_field(lo, hi, a.dec.pos[m], a.dec.mask[m]);
          const float4 f = load4<FT>(a.fac.f[m], (size_t)r * R + sub * 4);
          acc.x *= f.x;
          acc.y *= f.y;
          acc.z *= f.z;
          acc.w *= f.w;
        }
      }
      row = (uint32_t)line_field(lo, hi, a.dec.pos[a.target], a.dec.mask[a.target]);
    }
    if (NPW > 1) {
      // segmented suffix sum over groups with equal consecutive rows
      const uint32_t next_row = __shfl_down_sync(0xffffffffu, row, G);
      const bool tail = (grp == NPW - 1) || (next_row != row);
      const unsigned tails = __ballot_sync(0xffffffffu, tail && sub == 0);
      const unsigned geq = tails & ~((1u << (grp * G)) - 1u);
      const int run_end = (__ffs(geq) - 1) / G;
#pragma unroll
      for (int d = 1; d < NPW; d <<= 1) {
        const float4 o = shfl4_down(acc, d * G);
        if (grp + d <= run_end) add4(acc, o);
      }
    }
    const uint32_t prev_row = __shfl_up_sync(0xffffffffu, row, G);
    const bool head = (grp == 0) || (prev_row != row);
    if (grp == 0) {
      if (carry_row == row) {
        add4(acc, carry);
      } else if (carry_row != kNoRow) {
        flush_row<R>(staged, smem, iv_start, a.out, carry_row, sub, carry);
      }
      carry_row = kNoRow;
    }
    const bool last_step = base + NPW >= we;
    const int last_grp = last_step ? (int)(we - 1 - base) : NPW - 1;
    const unsigned heads = __ballot_sync(0xffffffffu, head && sub == 0 && row != kNoRow);
    const int last_lane = last_grp * G;
    const unsigned upto = last_lane >= 31 ? heads : (heads & ((2u << last_lane) - 1u));
    const int h_last = (31 - __clz(upto)) / G;
    if (head && row != kNoRow && (grp != h_last || last_step))
      flush_row<R>(staged, smem, iv_start, a.out, row, sub, acc);
    if (!last_step) {
      const float4 c = shfl4(acc, h_last * G + sub);
      const uint32_t cr = __shfl_sync(0xffffffffu, row, h_last * G);
      if (grp == 0) {
        carry = c;
        carry_row = cr;
      }
    }
  }
}

template <int R, typename FT, int HW>
__global__ void __launch_bounds__(kMttkrpThreads)
    mttkrp_tile_kernel(const MttkrpArgs a) {
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  const int warp = threadIdx.x >> 5;
  const int N = a.dec.nmodes;
  for (uint32_t tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
    const uint32_t ts = tile * a.tile_nnz;
    const uint32_t te = min(ts + a.tile_nnz, a.nnz);
    const uint32_t iv_start = a.tile_iv[((size_t)tile * N + a.target) * 2];
    const uint32_t iv_len = a.tile_iv[((size_t)tile * N + a.target) * 2 + 1];
    const bool staged = a.stage_rows > 0 && iv_len <= (uint32_t)a.stage_rows &&
                        iv_len * 2 <= (te - ts);
    if (staged) {
      for (uint32_t q = threadIdx.x; q < iv_len * (R / 4); q += blockDim.x)
        smem4[q] = make_float4(0.f, 0.f, 0.f, 0.f);
      __syncthreads();
    }
    const uint32_t chunk = (te - ts + kMttkrpWarps - 1) / kMttkrpWarps;
    const uint32_t ws = min(ts + warp * chunk, te);
    const uint32_t we = min(ws + chunk, te);
    warp_range<R, FT, HW>(a, ws, we, staged, smem, iv_start);
    if (staged) {
      __syncthreads();
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

constexpr int kStageBytes = 96 * 1024;

template <int R, typename FT, int HW>
static alto_status launch_tile(const MttkrpArgs& a, bool allow_stage, cudaStream_t st) {
  MttkrpArgs b = a;
  b.stage_rows = allow_stage ? kStageBytes / (R * 4) : 0;
  const size_t smem = allow_stage ? (size_t)kStageBytes : 0;
  static bool attr_set = false;
  if (!attr_set) {
    ALTO_TRY_CUDA(cudaFuncSetAttribute(mttkrp_tile_kernel<R, FT, HW>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, kStageBytes));
    attr_set = true;
  }
  unsigned grid = std::min<unsigned>(a.ntiles, (unsigned)num_sms() * 2);
  if (!grid) return ALTO_OK;
  mttkrp_tile_kernel<R, FT, HW><<<grid, kMttkrpThreads, smem, st>>>(b);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

template <typename FT, int HW>
static alto_status launch_rank(const MttkrpArgs& a, int rank, bool allow_stage, bool aligned,
                               cudaStream_t st) {
  if (aligned) {
    switch (rank) {
      case 4: return launch_tile<4, FT, HW>(a, allow_stage, st);
      case 8: return launch_tile<8, FT, HW>(a, allow_stage, st);
      case 16: return launch_tile<16, FT, HW>(a, allow_stage, st);
      case 32: return launch_tile<32, FT, HW>(a, allow_stage, st);
      case 64: return launch_tile<64, FT, HW>(a, allow_stage, st);
      case 128: return launch_tile<128, FT, HW>(a, allow_stage, st);
      default: break;
    }
  }
  unsigned grid = (unsigned)std::min<uint64_t>((a.nnz + 7) / 8, (uint64_t)num_sms() * 16);
  if (!grid) return ALTO_OK;
  mttkrp_generic_kernel<FT, HW><<<grid, kMttkrpThreads, 0, st>>>(a, rank);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

alto_mttkrp_variant choose_variant(const alto_tensor* t, int mode, int rank, alto_dtype fdtype) {
  // The reference's rule (include/alto.hpp:835-846): low-reuse long modes use
  // atomics, the stream mode its own kernel, everything else da_mem.  On the
  // device the staged kernel decides per tile and falls back to atomics
  // where the tile's interval does not fit, which covers all three cases.
  (void)rank;
  (void)fdtype;
  const uint64_t dim = t->dims[mode];
  const uint64_t reuse = dim ? t->nnz / dim : 0;
  if (dim > 512 && reuse <= 4) return ALTO_MTTKRP_ATOMIC;
  if (mode == t->stream_mode) return ALTO_MTTKRP_STREAM;
  return ALTO_MTTKRP_STAGED;
}

alto_status run_mttkrp(alto_tensor* t, int mode, const void* const* factors, alto_dtype fdtype,
                       int rank, float* out, int accumulate, alto_mttkrp_variant variant,
                       cudaStream_t st) {
  if (variant == ALTO_MTTKRP_AUTO) variant = choose_variant(t, mode, rank, fdtype);
  if (variant == ALTO_MTTKRP_SORTED) {
    set_error("the SORTED MTTKRP variant needs a row-sparse tensor (is_oidx)");
    return ALTO_ERR_UNSUPPORTED;
  }
  if (!accumulate)
    ALTO_TRY_CUDA(cudaMemsetAsync(out, 0, (size_t)t->dims[mode] * rank * sizeof(float), st));
  if (!t->nnz) return ALTO_OK;
  MttkrpArgs a{};
  a.klo = t->klo.as<uint64_t>();
  a.khi = t->khi.p;
  a.vals = t->vals.as<float>();
  a.tile_iv = t->tile_iv.as<uint32_t>();
  a.nnz = (uint32_t)t->nnz;
  a.tile_nnz = t->tile_nnz;
  a.ntiles = t->ntiles;
  a.target = mode;
  a.dec = t->dec;
  a.out = out;
  bool aligned = (reinterpret_cast<uintptr_t>(out) % 16) == 0;
  const int esz = fdtype == ALTO_BF16 ? 2 : 4;
  for (int m = 0; m < t->nmodes; ++m) {
    a.fac.f[m] = factors[m];
    if (m != mode && (reinterpret_cast<uintptr_t>(factors[m]) % (4 * esz)) != 0) aligned = false;
  }
  const bool stage = variant != ALTO_MTTKRP_ATOMIC;
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

}  // namespace alto
