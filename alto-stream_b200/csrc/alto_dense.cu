// Dense R x R and I x R kernels of CP-ALS and CP-stream, all in float64
// arithmetic over float32-stored factors.
//
// Reference operations (jeewhanchoi/ALTO-stream):
//   update_gram / mat_aTa (cblas_dsyrk)      src/gram.cpp:29-41, src/matrix.cpp:252-267
//   historical cross-Gram (cblas_dgemm)      src/streaming_cpd.cpp:1391-1400
//   hadamard_product / pseudo_inverse Hadamard src/matrix.cpp:269-294, include/cpd.hpp:383-397
//   Cholesky + solve (dpotrf/dpotrs)         include/cpd.hpp:409-476, src/matrix.cpp:226-250, 333-372
//   KruskalModelNorm                         src/kruskal_model.cpp:227-353
//   cpd_fit_alto                             include/cpd.hpp:193-275
//
// Reductions are deterministic: every kernel that reduces over rows writes
// per-block partials and a second, single-block kernel sums them in block
// order.  The normal-equation solve forms the inverse of the Cholesky-
// factored R x R matrix once (one CTA) and applies it to all I rows as a
// float64 row-times-matrix product; the reference runs dpotrs over the rows.
#include <algorithm>
#include <cmath>
#include <mutex>

#include "alto_dense.cuh"
#include "alto_group.cuh"

namespace alto {

constexpr int kGramThreads = 256;
constexpr int kGramRows = 32;

static int g_sms = 0;
static int sms() {
  if (!g_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_sms <= 0) g_sms = 148;
  }
  return g_sms;
}

template <typename T>
__device__ __forceinline__ double ld(const T* p, size_t i) {
  return (double)p[i];
}
template <>
__device__ __forceinline__ double ld<__nv_bfloat16>(const __nv_bfloat16* p, size_t i) {
  return (double)__bfloat162float(p[i]);
}

// Partial A^T B over a block's row range; PPT (a, b) pairs per thread.
template <int PPT, typename TA, typename TB>
__global__ void __launch_bounds__(kGramThreads)
    gram_partial_kernel(const TA* __restrict__ A, const TB* __restrict__ B, uint64_t I, int R,
                        uint64_t rows_per_block, double* __restrict__ partials) {
  extern __shared__ double sm[];
  double* sa = sm;
  double* sb = sm + kGramRows * R;
  double acc[PPT];
#pragma unroll
  for (int k = 0; k < PPT; ++k) acc[k] = 0.0;
  const uint64_t r0 = (uint64_t)blockIdx.x * rows_per_block;
  const uint64_t r1 = min(r0 + rows_per_block, I);
  const int RR = R * R;
  for (uint64_t t0 = r0; t0 < r1; t0 += kGramRows) {
    const int nr = (int)min((uint64_t)kGramRows, r1 - t0);
    for (int q = threadIdx.x; q < nr * R; q += kGramThreads) {
      sa[q] = ld(A, t0 * R + q);
      sb[q] = ld(B, t0 * R + q);
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
      const int p = threadIdx.x + k * kGramThreads;
      if (p < RR) {
        const int a = p / R, b = p % R;
        double s = 0.0;
        for (int r = 0; r < nr; ++r) s += sa[r * R + a] * sb[r * R + b];
        acc[k] += s;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    const int p = threadIdx.x + k * kGramThreads;
    if (p < RR) partials[(size_t)blockIdx.x * RR + p] = acc[k];
  }
}

// out[p] = sum over blocks b of partials[b][p] in a fixed order: block x
// takes 32 consecutive p (one per lane, coalesced), warp w sums blocks
// w, w+8, w+16, ... and the 8 warp sums are added in warp order.  Launch with
// reduce_grid(n) blocks of kReduceThreads threads.
constexpr int kReduceThreads = 256;
__host__ __device__ inline unsigned reduce_grid(int n) { return (unsigned)((n + 31) / 32); }

__global__ void __launch_bounds__(kReduceThreads)
    reduce_partials_kernel(const double* __restrict__ partials, int nblocks, int n, double* __restrict__ out) {
  __shared__ double s[kReduceThreads / 32][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int p = blockIdx.x * 32 + lane;
  double acc = 0.0;
  if (p < n)
    for (int b = w; b < nblocks; b += kReduceThreads / 32) acc += partials[(size_t)b * n + p];
  s[w][lane] = acc;
  __syncthreads();
  if (w == 0 && p < n) {
    double t = s[0][lane];
    for (int k = 1; k < kReduceThreads / 32; ++k) t += s[k][lane];
    out[p] = t;
  }
}

template <typename TA, typename TB>
static alto_status gram_launch(const TA* A, const TB* B, uint64_t I, int R, double* out,
                               DevBuf& scratch, cudaStream_t st) {
  const int RR = R * R;
  const int ppt = (RR + kGramThreads - 1) / kGramThreads;
  uint64_t nb = std::min<uint64_t>((I + 255) / 256, (uint64_t)sms() * 2);
  if (nb < 1) nb = 1;
  const uint64_t rpb = (I + nb - 1) / nb;
  nb = I ? (I + rpb - 1) / rpb : 1;
  ALTO_TRY(scratch.ensure(nb * RR * sizeof(double)));
  const size_t smem = 2 * kGramRows * R * sizeof(double);
  double* part = scratch.as<double>();
  if (I == 0) {
    ALTO_TRY_CUDA(cudaMemsetAsync(out, 0, RR * sizeof(double), st));
    return ALTO_OK;
  }
  // (the shared-memory limit is raised once per kernel, outside any capture)
#define GRAM_CASE(P)                                                                             \
  case P:                                                                                        \
    if (smem > 48 * 1024) {                                                                      \
      static size_t raised = 0;                                                                  \
      if (smem > raised) {                                                                       \
        ALTO_TRY_CUDA(cudaFuncSetAttribute(gram_partial_kernel<P, TA, TB>,                      \
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
        raised = smem;                                                                           \
      }                                                                                          \
    }                                                                                            \
    gram_partial_kernel<P, TA, TB><<<(unsigned)nb, kGramThreads, smem, st>>>(A, B, I, R, rpb, part); \
    break;
  switch (ppt <= 1 ? 1 : ppt <= 2 ? 2 : ppt <= 4 ? 4 : ppt <= 8 ? 8 : ppt <= 16 ? 16 : 64) {
    GRAM_CASE(1)
    GRAM_CASE(2)
    GRAM_CASE(4)
    GRAM_CASE(8)
    GRAM_CASE(16)
    GRAM_CASE(64)
  }
#undef GRAM_CASE
  ALTO_LAUNCHED();
  reduce_partials_kernel<<<reduce_grid(RR), kReduceThreads, 0, st>>>(part, (int)nb, RR, out);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

// One pass over P and U (float32, I x R): per-block partials of U^T U,
// P^T U and {sum p u, sum (p - u)^2, sum u^2} (the CP-stream Gram, cross
// Gram and change statistics of a freshly updated factor), layout
// [block][2 R^2 + 3].  The rows are staged kGramRows at a time in two
// alternating shared-memory buffers (one barrier per chunk).  For ranks 23
// to 32 the next chunk's loads are issued into registers before the
// current chunk's products, so their latency overlaps the arithmetic
// (measured 17% faster at rank 32; at ranks up to 16 the extra registers
// cost more occupancy than the overlap gains, and larger ranks' accumulators
// fill the registers).  Dynamic shared memory: 4 kGramRows R doubles.
template <int PPT>
constexpr int gram_stage_regs() {  // ceil(kGramRows R / threads) for the largest R of PPT
  return PPT <= 1 ? 2 : PPT <= 2 ? 3 : PPT <= 4 ? 4 : PPT <= 16 ? 8 : 16;
}

template <int PPT>
__device__ __forceinline__ void gram_cross_partial_body(const float* __restrict__ P, const float* __restrict__ U,
                                                        uint64_t I, int R, uint64_t rows_per_block,
                                                        double* __restrict__ partials, uint32_t block) {
  constexpr int L = gram_stage_regs<PPT>();
  constexpr bool kPipe = PPT == 4;
  extern __shared__ double sm[];
  double g[PPT], c[PPT];
#pragma unroll
  for (int k = 0; k < PPT; ++k) g[k] = c[k] = 0.0;
  double q0 = 0.0, q1 = 0.0, q2 = 0.0;
  const uint64_t r0 = (uint64_t)block * rows_per_block;
  const uint64_t r1 = min(r0 + rows_per_block, I);
  const int RR = R * R;
  float pre_p[kPipe ? L : 1], pre_u[kPipe ? L : 1];
  auto fetch = [&](uint64_t t0) {  // chunk at row t0 into registers
    const int n = (int)min((uint64_t)kGramRows, r1 - t0) * R;
#pragma unroll
    for (int l = 0; l < (kPipe ? L : 1); ++l) {
      const int q = threadIdx.x + l * kGramThreads;
      pre_p[l] = q < n ? P[t0 * R + q] : 0.f;
      pre_u[l] = q < n ? U[t0 * R + q] : 0.f;
    }
  };
  if (kPipe && r0 < r1) fetch(r0);
  int buf = 0;
  for (uint64_t t0 = r0; t0 < r1; t0 += kGramRows) {
    const int nr = (int)min((uint64_t)kGramRows, r1 - t0);
    double* sp = sm + (size_t)buf * 2 * kGramRows * R;
    double* su = sp + kGramRows * R;
    if constexpr (kPipe) {
#pragma unroll
      for (int l = 0; l < L; ++l) {
        const int q = threadIdx.x + l * kGramThreads;
        if (q < nr * R) {
          const double pv = (double)pre_p[l], uv = (double)pre_u[l];
          sp[q] = pv;
          su[q] = uv;
          q0 += pv * uv;
          q1 += (pv - uv) * (pv - uv);
          q2 += uv * uv;
        }
      }
    } else {
      for (int q = threadIdx.x; q < nr * R; q += kGramThreads) {
        const double pv = (double)P[t0 * R + q], uv = (double)U[t0 * R + q];
        sp[q] = pv;
        su[q] = uv;
        q0 += pv * uv;
        q1 += (pv - uv) * (pv - uv);
        q2 += uv * uv;
      }
    }
    __syncthreads();
    if (kPipe && t0 + kGramRows < r1) fetch(t0 + kGramRows);
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
      const int p = threadIdx.x + k * kGramThreads;
      if (p < RR) {
        const int a = p / R, b = p % R;
        double sg = 0.0, sc = 0.0;
        for (int r = 0; r < nr; ++r) {
          const double ub = su[r * R + b];
          sg += su[r * R + a] * ub;
          sc += sp[r * R + a] * ub;
        }
        g[k] += sg;
        c[k] += sc;
      }
    }
    buf ^= 1;
  }
  double* out = partials + (size_t)block * (2 * RR + 3);
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    const int p = threadIdx.x + k * kGramThreads;
    if (p < RR) {
      out[p] = g[k];
      out[RR + p] = c[k];
    }
  }
  // the three statistics: warp butterflies, then warps in order
  __shared__ double wq[3][kGramThreads / 32];
  for (int o = 16; o; o >>= 1) {
    q0 += __shfl_xor_sync(0xffffffffu, q0, o);
    q1 += __shfl_xor_sync(0xffffffffu, q1, o);
    q2 += __shfl_xor_sync(0xffffffffu, q2, o);
  }
  if ((threadIdx.x & 31) == 0) {
    wq[0][threadIdx.x >> 5] = q0;
    wq[1][threadIdx.x >> 5] = q1;
    wq[2][threadIdx.x >> 5] = q2;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0.0;
    for (int w = 0; w < kGramThreads / 32; ++w) t += wq[threadIdx.x][w];
    out[2 * RR + threadIdx.x] = t;
  }
  __syncthreads();
}

template <int PPT>
__global__ void __launch_bounds__(kGramThreads)
    gram_cross_partial_kernel(const float* __restrict__ P, const float* __restrict__ U, uint64_t I, int R,
                              uint64_t rows_per_block, double* __restrict__ partials) {
  gram_cross_partial_body<PPT>(P, U, I, R, rows_per_block, partials, blockIdx.x);
}

// reduce_partials_kernel with the result split over three outputs:
// [0, n1) -> o1, [n1, 2 n1) -> o2, the rest -> o3.
__device__ __forceinline__ void reduce_split_body(const double* __restrict__ partials, int nblocks, int n1, int n,
                                                  double* __restrict__ o1, double* __restrict__ o2,
                                                  double* __restrict__ o3, uint32_t block) {
  __shared__ double s[kReduceThreads / 32][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int p = block * 32 + lane;
  double acc = 0.0;
  if (p < n)
    for (int b = w; b < nblocks; b += kReduceThreads / 32) acc += partials[(size_t)b * n + p];
  s[w][lane] = acc;
  __syncthreads();
  if (w == 0 && p < n) {
    double t = s[0][lane];
    for (int k = 1; k < kReduceThreads / 32; ++k) t += s[k][lane];
    if (p < n1)
      o1[p] = t;
    else if (p < 2 * n1)
      o2[p - n1] = t;
    else if (o3)
      o3[p - 2 * n1] = t;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kReduceThreads)
    reduce_split_kernel(const double* __restrict__ partials, int nblocks, int n1, int n, double* __restrict__ o1,
                        double* __restrict__ o2, double* __restrict__ o3) {
  reduce_split_body(partials, nblocks, n1, n, o1, o2, o3, blockIdx.x);
}

// Grouped gram_cross_stats: partial blocks over all items (block_off
// prefix sums of the items' nb), then reduction blocks (red_off).
template <int PPT>
__global__ void __launch_bounds__(kGramThreads)
    gram_group_partial_kernel(Strided<GramItem> items, const uint32_t* __restrict__ block_off, int R) {
  const int K = *items.count;
  const uint32_t total = K > 0 ? block_off[K] : 0;
  for (uint32_t v = blockIdx.x; v < total; v += gridDim.x) {
    int lo = 0, hi = K;  // the last s with block_off[s] <= v
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (block_off[mid] <= v)
        lo = mid;
      else
        hi = mid;
    }
    const GramItem& it = items[lo];
    if (it.active && !*it.active) continue;
    gram_cross_partial_body<PPT>(it.P, it.U, it.I, R, it.rpb, it.part, v - block_off[lo]);
  }
}

__global__ void __launch_bounds__(kReduceThreads)
    gram_group_reduce_kernel(Strided<GramItem> items, const uint32_t* __restrict__ red_off, int R) {
  const int K = *items.count;
  const uint32_t total = K > 0 ? red_off[K] : 0;
  const int RR = R * R, n = 2 * RR + 3;
  for (uint32_t v = blockIdx.x; v < total; v += gridDim.x) {
    int lo = 0, hi = K;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (red_off[mid] <= v)
        lo = mid;
      else
        hi = mid;
    }
    const GramItem& it = items[lo];
    if (it.active && !*it.active) continue;
    reduce_split_body(it.part, (int)it.nb, RR, n, it.G, it.C, it.stats3, v - red_off[lo]);
  }
}

// At least 64 rows per block, at most 4 blocks per SM.
void gram_split(uint64_t I, uint32_t* nb_out, uint64_t* rpb_out) {
  uint64_t nb = std::min<uint64_t>((I + 63) / 64, (uint64_t)sms() * 4);
  if (nb < 1) nb = 1;
  const uint64_t rpb = (I + nb - 1) / nb;
  nb = I ? (I + rpb - 1) / rpb : 1;
  *nb_out = (uint32_t)nb;
  *rpb_out = rpb;
}

uint32_t gram_reduce_blocks(int R) { return reduce_grid(2 * R * R + 3); }

// The grouped Gram's shared-memory limit for rank R raised ahead of a
// capture (gram_group_launch raises it too; this keeps the call out of the
// captured sequence).
alto_status gram_group_ready(int R) {
  const int ppt = (R * R + kGramThreads - 1) / kGramThreads;
  const int smem = 4 * kGramRows * R * (int)sizeof(double);
  if (smem <= 48 * 1024) return ALTO_OK;
  const void* fn = ppt <= 1 ? (const void*)gram_group_partial_kernel<1>
                   : ppt <= 2 ? (const void*)gram_group_partial_kernel<2>
                   : ppt <= 4 ? (const void*)gram_group_partial_kernel<4>
                   : ppt <= 16 ? (const void*)gram_group_partial_kernel<16>
                               : (const void*)gram_group_partial_kernel<64>;
  ALTO_TRY_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  return ALTO_OK;
}

alto_status gram_group_launch(Strided<GramItem> items, const uint32_t* block_off, const uint32_t* red_off,
                              int max_items, int R, cudaStream_t st) {
  const int RR = R * R;
  const int ppt = (RR + kGramThreads - 1) / kGramThreads;
  const size_t smem = 4 * kGramRows * R * sizeof(double);  // two staged chunks of P and U
  const unsigned grid = (unsigned)sms() * 4;
#define GG_CASE(PP)                                                                                   \
  case PP: {                                                                                          \
    static size_t raised = 0;                                                                         \
    if (smem > 48 * 1024 && smem > raised) {                                                          \
      ALTO_TRY_CUDA(cudaFuncSetAttribute(gram_group_partial_kernel<PP>,                               \
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));   \
      raised = smem;                                                                                  \
    }                                                                                                 \
    gram_group_partial_kernel<PP><<<grid, kGramThreads, smem, st>>>(items, block_off, R);             \
    break;                                                                                            \
  }
  switch (ppt <= 1 ? 1 : ppt <= 2 ? 2 : ppt <= 4 ? 4 : ppt <= 16 ? 16 : 64) {
    GG_CASE(1)
    GG_CASE(2)
    GG_CASE(4)
    GG_CASE(16)
    GG_CASE(64)
  }
#undef GG_CASE
  ALTO_LAUNCHED();
  const unsigned rgrid = (unsigned)std::max(1, std::min(max_items * (int)gram_reduce_blocks(R), (int)sms() * 8));
  gram_group_reduce_kernel<<<rgrid, kReduceThreads, 0, st>>>(items, red_off, R);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

alto_status gram_cross_stats(const float* P, const float* U, uint64_t I, int R, double* G, double* C,
                             double* stats3, DevBuf& scratch, cudaStream_t st) {
  const int RR = R * R;
  const int n = 2 * RR + 3;
  const int ppt = (RR + kGramThreads - 1) / kGramThreads;
  uint32_t nb32 = 1;
  uint64_t rpb = 1;
  gram_split(I, &nb32, &rpb);
  uint64_t nb = nb32;
  ALTO_TRY(scratch.ensure(nb * n * sizeof(double)));
  double* part = scratch.as<double>();
  const size_t smem = 4 * kGramRows * R * sizeof(double);  // two staged chunks of P and U
  if (I == 0) {
    ALTO_TRY_CUDA(cudaMemsetAsync(part, 0, n * sizeof(double), st));
    nb = 1;
  } else {
#define GC_CASE(PP)                                                                                  \
  case PP: {                                                                                         \
    static size_t raised = 0;                                                                        \
    if (smem > 48 * 1024 && smem > raised) {                                                         \
      ALTO_TRY_CUDA(cudaFuncSetAttribute(gram_cross_partial_kernel<PP>,                             \
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));  \
      raised = smem;                                                                                 \
    }                                                                                                \
    gram_cross_partial_kernel<PP><<<(unsigned)nb, kGramThreads, smem, st>>>(P, U, I, R, rpb, part); \
    break;                                                                                           \
  }
    switch (ppt <= 1 ? 1 : ppt <= 2 ? 2 : ppt <= 4 ? 4 : ppt <= 16 ? 16 : 64) {
      GC_CASE(1)
      GC_CASE(2)
      GC_CASE(4)
      GC_CASE(16)
      GC_CASE(64)
    }
#undef GC_CASE
    ALTO_LAUNCHED();
  }
  reduce_split_kernel<<<reduce_grid(n), kReduceThreads, 0, st>>>(part, (int)nb, RR, n, G, C, stats3);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

alto_status gram(const float* A, uint64_t I, int R, double* out, DevBuf& scratch, cudaStream_t st) {
  return gram_launch<float, float>(A, A, I, R, out, scratch, st);
}

alto_status cross_gram(const float* A, const float* B, uint64_t I, int R, double* out,
                       DevBuf& scratch, cudaStream_t st) {
  return gram_launch<float, float>(A, B, I, R, out, scratch, st);
}

// ------------------------------------------------------- R x R solve setup

// One CTA: V = prod_{m in mask} G_m (elementwise), then per `kind`:
//   SOLVE_RIDGE: V += ridge * I;  ADMM: rho = tr(V)/R, V += rho * I.
// Cholesky of V (upper triangle read, as dpotrf 'L' on the column-major
// view); on success W = V^{-1}.  On failure: kind SOLVE_RIDGE_DIAG_FALLBACK
// writes the reference's dgelsy fallback for CP-ALS, W = diag(1/V_rr) of V
// without the ridge (include/cpd.hpp:436-476: its restored V has zero
// lower triangles mirrored over the upper one); kind kSolveRidgeKeep writes
// W = I (the right-hand side is left as it is); otherwise W = 0.
// status[0] = LAPACK-style info (0 = success), rho_out[0] = rho.
__global__ void solve_setup_kernel(const double* __restrict__ grams, int nmodes, unsigned mask,
                                   int R, int kind, double ridge, double* __restrict__ W,
                                   int* __restrict__ status, double* __restrict__ rho_out) {
  extern __shared__ double A[];  // R x R
  const int RR = R * R;
  for (int p = threadIdx.x; p < RR; p += blockDim.x) {
    double v = 1.0;
    for (int m = 0; m < nmodes; ++m)
      if (mask & (1u << m)) v *= grams[(size_t)m * RR + p];
    A[p] = v;
  }
  __syncthreads();
  __shared__ double s_rho;
  __shared__ int s_info;
  if (threadIdx.x == 0) {
    double add = ridge;
    if (kind == kSolveAdmm) {
      double tr = 0.0;
      for (int r = 0; r < R; ++r) tr += A[r * R + r];
      add = tr / (double)R;
    }
    s_rho = add;
    s_info = 0;
  }
  __syncthreads();
  // keep the unridged diagonal for the fallback in W's diagonal slots
  if (kind == kSolveRidgeDiagFallback)
    for (int r = threadIdx.x; r < R; r += blockDim.x) W[r * R + r] = A[r * R + r];
  for (int r = threadIdx.x; r < R; r += blockDim.x) A[r * R + r] += s_rho;
  __syncthreads();
  // right-looking Cholesky, lower factor in A's lower triangle (reads upper)
  for (int j = 0; j < R; ++j) {
    if (threadIdx.x == 0) {
      double d = A[j * R + j];
      for (int k = 0; k < j; ++k) d -= A[j * R + k] * A[j * R + k];
      if (!(d > 0.0)) {
        if (!s_info) s_info = j + 1;
        d = 1.0;
      }
      A[j * R + j] = sqrt(d);
    }
    __syncthreads();
    const double djj = A[j * R + j];
    for (int i = j + 1 + threadIdx.x; i < R; i += blockDim.x) {
      double s = A[j * R + i];
      for (int k = 0; k < j; ++k) s -= A[i * R + k] * A[j * R + k];
      A[i * R + j] = s / djj;
    }
    __syncthreads();
  }
  const int info = s_info;
  if (info) {
    for (int p = threadIdx.x; p < RR; p += blockDim.x) {
      const int a = p / R, b = p % R;
      if (kind == kSolveRidgeDiagFallback) {
        if (a != b) W[p] = 0.0;
      } else {
        W[p] = (kind == kSolveRidgeKeep && a == b) ? 1.0 : 0.0;
      }
    }
    __syncthreads();
    if (kind == kSolveRidgeDiagFallback)
      for (int r = threadIdx.x; r < R; r += blockDim.x) {
        const double d = W[r * R + r];
        W[r * R + r] = d != 0.0 ? 1.0 / d : 0.0;
      }
  } else {
    // L^{-1} by forward substitution, one column per thread:
    // x_i = (delta_ic - sum_{k=c}^{i-1} L[i][k] x_k) / L[i][i], kept in row c of W.
    for (int c = threadIdx.x; c < R; c += blockDim.x) {
      double* x = W + (size_t)c * R;
      for (int i = 0; i < c; ++i) x[i] = 0.0;
      for (int i = c; i < R; ++i) {
        double s = (i == c) ? 1.0 : 0.0;
        for (int k = c; k < i; ++k) s -= A[i * R + k] * x[k];
        x[i] = s / A[i * R + i];
      }
    }
    __syncthreads();
    // W currently holds rows c = columns of L^{-1}: Linv[i][c] = W[c*R + i].
    // Copy L^{-1} into A (lower) then W[a][b] = sum_{k >= max(a,b)} Linv[k][a] Linv[k][b].
    for (int p = threadIdx.x; p < RR; p += blockDim.x) {
      const int c = p / R, i = p % R;
      if (i >= c) A[i * R + c] = W[(size_t)c * R + i];
    }
    __syncthreads();
    for (int p = threadIdx.x; p < RR; p += blockDim.x) {
      const int a = p / R, b = p % R;
      const int k0 = a > b ? a : b;
      double s = 0.0;
      for (int k = k0; k < R; ++k) s += A[k * R + a] * A[k * R + b];
      W[p] = s;
    }
  }
  if (threadIdx.x == 0) {
    status[0] = info;
    if (rho_out) rho_out[0] = s_rho;
  }
}

// The same set-up with one thread per element of the R x R matrix (R <= 32,
// blockDim = R * R): a right-looking Cholesky (column j scaled by its
// diagonal, then the trailing lower triangle updated by the rank-one term),
// the inverse of L by a right-looking forward substitution of all columns
// at once, and W = L^-T L^-1.  Every element sees the operations of the
// column-by-column form in the same order (its subtractions in k order,
// then its division), as fused multiply-adds; R barriers per phase instead
// of R^2 dependent steps in one warp.
template <int RMAX>
__device__ __forceinline__ void solve_setup_block_body(const double* __restrict__ grams, int nmodes, unsigned mask,
                                                       int R, int kind, double ridge, double* __restrict__ W,
                                                       int* __restrict__ status, double* __restrict__ rho_out) {
  __shared__ double A[RMAX * RMAX];
  __shared__ double X[RMAX * RMAX];
  __shared__ double s_rho;
  __shared__ int s_info;
  const int RR = R * R;
  const int tid = threadIdx.x;
  const bool mine = tid < RR;
  const int a = mine ? tid / R : 0, b = mine ? tid % R : 0;  // row, column
  if (mine) {
    double v = 1.0;
    for (int m = 0; m < nmodes; ++m)
      if (mask & (1u << m)) v *= grams[(size_t)m * RR + tid];
    A[tid] = v;
    X[tid] = a == b ? 1.0 : 0.0;
  }
  __syncthreads();
  if (tid == 0) {
    double add = ridge;
    if (kind == kSolveAdmm) {
      double tr = 0.0;
      for (int r = 0; r < R; ++r) tr += A[r * R + r];
      add = tr / (double)R;
    }
    s_rho = add;
    s_info = 0;
  }
  __syncthreads();
  if (kind == kSolveRidgeDiagFallback && mine && a == b) W[tid] = A[tid];
  if (mine && a == b) A[tid] += s_rho;
  __syncthreads();
  for (int j = 0; j < R; ++j) {
    if (tid == 0) {
      double d = A[j * R + j];
      if (!(d > 0.0)) {
        if (!s_info) s_info = j + 1;
        d = 1.0;
      }
      A[j * R + j] = sqrt(d);
    }
    __syncthreads();
    if (mine && b == j && a > j) A[tid] = A[tid] / A[j * R + j];
    __syncthreads();
    if (mine && b > j && a >= b) A[tid] = __fma_rn(-A[a * R + j], A[b * R + j], A[tid]);
    __syncthreads();
  }
  const int info = s_info;
  if (info) {
    if (mine) {
      if (kind == kSolveRidgeDiagFallback) {
        if (a != b) W[tid] = 0.0;
      } else {
        W[tid] = (kind == kSolveRidgeKeep && a == b) ? 1.0 : 0.0;
      }
    }
    __syncthreads();
    if (kind == kSolveRidgeDiagFallback && mine && a == b) {
      const double d = W[tid];
      W[tid] = d != 0.0 ? 1.0 / d : 0.0;
    }
  } else {
    // X = L^-1 (lower): row k divided by L_kk once every earlier row has
    // been subtracted from it, then subtracted from the rows below
    for (int k = 0; k < R; ++k) {
      if (mine && a == k && b <= k) X[tid] = X[tid] / A[k * R + k];
      __syncthreads();
      if (mine && a > k && b <= k) X[tid] = __fma_rn(-A[a * R + k], X[k * R + b], X[tid]);
      __syncthreads();
    }
    if (mine) {
      const int k0 = a > b ? a : b;
      double sv = 0.0;
      for (int k = k0; k < R; ++k) sv = __fma_rn(X[k * R + a], X[k * R + b], sv);
      W[tid] = sv;
    }
  }
  if (tid == 0) {
    status[0] = info;
    if (rho_out) rho_out[0] = s_rho;
  }
  __syncthreads();
}

template <int RMAX>
__global__ void __launch_bounds__(RMAX * RMAX)
    solve_setup_block_kernel(const double* __restrict__ grams, int nmodes, unsigned mask, int R, int kind,
                             double ridge, double* __restrict__ W, int* __restrict__ status,
                             double* __restrict__ rho_out) {
  solve_setup_block_body<RMAX>(grams, nmodes, mask, R, kind, ridge, W, status, rho_out);
}

// One CTA of R * R threads per item in turn (R <= 32).
template <int RMAX>
__global__ void __launch_bounds__(RMAX * RMAX) setup_group_kernel(Strided<SetupItem> items, int R) {
  const int K = *items.count;
  for (int s = blockIdx.x; s < K; s += gridDim.x) {
    const SetupItem& it = items[s];
    if (it.active && !*it.active) continue;
    solve_setup_block_body<RMAX>(it.grams, it.nmodes, it.mask, R, it.kind, it.ridge, it.W, it.status, it.rho);
  }
}

alto_status setup_group_launch(Strided<SetupItem> items, int max_items, int R, cudaStream_t st) {
  const unsigned grid = (unsigned)std::max(1, std::min(max_items, 1024));
  if (R <= 8)
    setup_group_kernel<8><<<grid, R * R, 0, st>>>(items, R);
  else if (R <= 16)
    setup_group_kernel<16><<<grid, R * R, 0, st>>>(items, R);
  else if (R <= 32)
    setup_group_kernel<32><<<grid, R * R, 0, st>>>(items, R);
  else {
    set_error("grouped solve set-up takes rank <= 32 (got %d)", R);
    return ALTO_ERR_UNSUPPORTED;
  }
  ALTO_LAUNCHED();
  return ALTO_OK;
}

alto_status solve_setup(const double* grams, int nmodes, unsigned mask, int R, int kind,
                        double ridge, double* W, int* status, double* rho, cudaStream_t st) {
  if (R <= 32) {
    if (R <= 8)
      solve_setup_block_kernel<8><<<1, R * R, 0, st>>>(grams, nmodes, mask, R, kind, ridge, W, status, rho);
    else if (R <= 16)
      solve_setup_block_kernel<16><<<1, R * R, 0, st>>>(grams, nmodes, mask, R, kind, ridge, W, status, rho);
    else
      solve_setup_block_kernel<32><<<1, R * R, 0, st>>>(grams, nmodes, mask, R, kind, ridge, W, status, rho);
    ALTO_LAUNCHED();
    return ALTO_OK;
  }
  const size_t smem = (size_t)R * R * sizeof(double);
  static size_t raised = 0;
  if (smem > 48 * 1024 && smem > raised) {
    ALTO_TRY_CUDA(cudaFuncSetAttribute(solve_setup_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    raised = smem;
  }
  solve_setup_kernel<<<1, 256, smem, st>>>(grams, nmodes, mask, R, kind, ridge, W, status, rho);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

// ------------------------------------------------------------ row apply

// X[i, :] = B[i, :] W (+ C[i, :] when C is given), float64 arithmetic.
// Column statistics of the result go to per-block partials:
// stats[b][0][r] = sum x^2, stats[b][1][r] = max x.
template <typename TB, typename TC, typename TX>
__global__ void __launch_bounds__(256)
    apply_kernel(const TB* __restrict__ B, const TC* __restrict__ C,
                 const double* __restrict__ W, uint64_t I, int R, TX* __restrict__ X,
                 double* __restrict__ stats, uint64_t rows_per_block) {
  extern __shared__ double sw[];  // W (R x R), then column stats (2 x R per warp)
  const int RR = R * R;
  for (int p = threadIdx.x; p < RR; p += blockDim.x) sw[p] = W[p];
  const int nwarps = blockDim.x >> 5;
  double* wsq = sw + RR;            // [nwarps][R]
  double* wmx = wsq + nwarps * R;   // [nwarps][R]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int r = lane; r < R; r += 32) {
    wsq[warp * R + r] = 0.0;
    wmx[warp * R + r] = -INFINITY;
  }
  __syncthreads();
  const uint64_t r0 = (uint64_t)blockIdx.x * rows_per_block;
  const uint64_t r1 = min(r0 + rows_per_block, I);
  for (uint64_t i = r0 + warp; i < r1; i += nwarps) {
    for (int c0 = 0; c0 < R; c0 += 32) {
      const int c = c0 + lane;
      double x = 0.0;
      for (int k0 = 0; k0 < R; k0 += 32) {
        const int kk = k0 + lane;
        const double bk = kk < R ? ld(B, i * R + kk) : 0.0;
        const int kmax = min(32, R - k0);
        for (int k = 0; k < kmax; ++k) {
          const double b = __shfl_sync(0xffffffffu, bk, k);
          if (c < R) x += b * sw[(k0 + k) * R + c];
        }
      }
      if (c < R) {
        if (C) x += (double)C[i * R + c];
        const TX xs = (TX)x;
        X[i * R + c] = xs;
        const double xv = (double)xs;
        wsq[warp * R + c] += xv * xv;
        wmx[warp * R + c] = fmax(wmx[warp * R + c], xv);
      }
    }
  }
  __syncthreads();
  if (stats) {
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
      double s = 0.0, m = -INFINITY;
      for (int w = 0; w < nwarps; ++w) {
        s += wsq[w * R + r];
        m = fmax(m, wmx[w * R + r]);
      }
      stats[((size_t)blockIdx.x * 2 + 0) * R + r] = s;
      stats[((size_t)blockIdx.x * 2 + 1) * R + r] = m;
    }
  }
}

template <typename TB, typename TC, typename TX>
static alto_status apply_launch(const TB* B, const TC* C, const double* W, uint64_t I, int R,
                                TX* X, DevBuf* stats, int* nblocks_out, cudaStream_t st) {
  uint64_t nb = std::min<uint64_t>((I + 63) / 64, (uint64_t)sms() * 4);
  if (nb < 1) nb = 1;
  const uint64_t rpb = (I + nb - 1) / nb;
  nb = I ? (I + rpb - 1) / rpb : 1;
  double* sp = nullptr;
  if (stats) {
    ALTO_TRY(stats->ensure(nb * 2 * R * sizeof(double)));
    sp = stats->as<double>();
  }
  if (nblocks_out) *nblocks_out = (int)nb;
  const size_t smem = ((size_t)R * R + 2 * 8 * R) * sizeof(double);
  static size_t raised = 0;  // raised once per kernel, outside any capture
  if (smem > 48 * 1024 && smem > raised) {
    ALTO_TRY_CUDA(cudaFuncSetAttribute(apply_kernel<TB, TC, TX>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    raised = smem;
  }
  apply_kernel<TB, TC, TX><<<(unsigned)nb, 256, smem, st>>>(B, C, W, I, R, X, sp, rpb);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

alto_status apply_f32(const float* B, const double* W, uint64_t I, int R, float* X,
                      DevBuf* stats, int* nblocks, cudaStream_t st) {
  return apply_launch<float, double, float>(B, nullptr, W, I, R, X, stats, nblocks, st);
}

alto_status apply_f64_to_f32(const double* B, const double* W, uint64_t I, int R, float* X,
                             cudaStream_t st) {
  return apply_launch<double, double, float>(B, nullptr, W, I, R, X, nullptr, nullptr, st);
}

alto_status apply_f32_to_f64(const float* B, const float* C, const double* W, uint64_t I, int R,
                             double* X, cudaStream_t st) {
  return apply_launch<float, float, double>(B, C, W, I, R, X, nullptr, nullptr, st);
}

// ----------------------------------------------------------- normalisation

// lambda from per-block column statistics (block order): which 0 ->
// sqrt(max(sum x^2, 1e-12)); which 1 -> max(1, max x).
__global__ void lambda_kernel(const double* __restrict__ stats, int nblocks, int R, int which,
                              double* __restrict__ lambda) {
  for (int r = threadIdx.x; r < R; r += blockDim.x) {
    double s = 0.0, m = 1.0;
    for (int b = 0; b < nblocks; ++b) {
      s += stats[((size_t)b * 2 + 0) * R + r];
      m = fmax(m, stats[((size_t)b * 2 + 1) * R + r]);
    }
    lambda[r] = which == 0 ? sqrt(s > 1e-12 ? s : 1e-12) : m;
  }
}

alto_status column_lambda(const double* stats, int nblocks, int R, int which, double* lambda,
                          cudaStream_t st) {
  lambda_kernel<<<1, 128, 0, st>>>(stats, nblocks, R, which, lambda);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

// X[i][r] /= lambda[r]; optional bfloat16 shadow copy.
__global__ void scale_kernel(float* __restrict__ X, uint64_t n, int R,
                             const double* __restrict__ lambda, __nv_bfloat16* __restrict__ shadow) {
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < n;
       q += (uint64_t)gridDim.x * blockDim.x) {
    const float v = (float)((double)X[q] / lambda[q % R]);
    X[q] = v;
    if (shadow) shadow[q] = __float2bfloat16(v);
  }
}

alto_status scale_columns(float* X, uint64_t I, int R, const double* lambda, __nv_bfloat16* shadow,
                          cudaStream_t st) {
  const uint64_t n = I * R;
  if (!n) return ALTO_OK;
  const unsigned grid = (unsigned)std::min<uint64_t>((n + 255) / 256, (uint64_t)sms() * 8);
  scale_kernel<<<grid, 256, 0, st>>>(X, n, R, lambda, shadow);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

__global__ void to_bf16_kernel(const float* __restrict__ X, uint64_t n, __nv_bfloat16* __restrict__ Y) {
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < n;
       q += (uint64_t)gridDim.x * blockDim.x)
    Y[q] = __float2bfloat16(X[q]);
}

alto_status to_bf16(const float* X, uint64_t n, __nv_bfloat16* Y, cudaStream_t st) {
  if (!n) return ALTO_OK;
  const unsigned grid = (unsigned)std::min<uint64_t>((n + 255) / 256, (uint64_t)sms() * 8);
  to_bf16_kernel<<<grid, 256, 0, st>>>(X, n, Y);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

// ------------------------------------------------------------ reductions

// Per-block partial sums of up to 4 quantities over n elements:
//   q0 = sum a*b (dot), q1 = sum (a-b)^2, q2 = sum b^2.
template <typename TA, typename TB>
__global__ void __launch_bounds__(256)
    dot_partial_kernel(const TA* __restrict__ a, const TB* __restrict__ b, uint64_t n,
                       const double* __restrict__ colw, int R, double* __restrict__ partials) {
  double q0 = 0, q1 = 0, q2 = 0;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < n;
       q += (uint64_t)gridDim.x * blockDim.x) {
    const double x = (double)a[q], y = (double)b[q];
    const double w = colw ? colw[q % R] : 1.0;
    q0 += x * y * w;
    q1 += (x - y) * (x - y);
    q2 += y * y;
  }
  __shared__ double s[3][8];
  for (int o = 16; o; o >>= 1) {
    q0 += __shfl_xor_sync(0xffffffffu, q0, o);
    q1 += __shfl_xor_sync(0xffffffffu, q1, o);
    q2 += __shfl_xor_sync(0xffffffffu, q2, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    s[0][warp] = q0;
    s[1][warp] = q1;
    s[2][warp] = q2;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s[threadIdx.x][w];
    partials[(size_t)blockIdx.x * 3 + threadIdx.x] = t;
  }
}

static constexpr int kDotBlocks = 296;

alto_status dot_stats(const float* a, const float* b, uint64_t n, const double* colw, int R,
                      double* out3, DevBuf& scratch, cudaStream_t st) {
  ALTO_TRY(scratch.ensure(kDotBlocks * 3 * sizeof(double)));
  dot_partial_kernel<float, float><<<kDotBlocks, 256, 0, st>>>(a, b, n, colw, R, scratch.as<double>());
  ALTO_LAUNCHED();
  reduce_partials_kernel<<<reduce_grid(3), kReduceThreads, 0, st>>>(scratch.as<double>(), kDotBlocks, 3, out3);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

alto_status dot_stats_f64(const double* a, const float* b, uint64_t n, double* out3, DevBuf& scratch,
                          cudaStream_t st) {
  ALTO_TRY(scratch.ensure(kDotBlocks * 3 * sizeof(double)));
  dot_partial_kernel<double, float><<<kDotBlocks, 256, 0, st>>>(a, b, n, nullptr, 1, scratch.as<double>());
  ALTO_LAUNCHED();
  reduce_partials_kernel<<<reduce_grid(3), kReduceThreads, 0, st>>>(scratch.as<double>(), kDotBlocks, 3, out3);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

// Sum of squares of n float values (||X||^2 of the tensor values).
__global__ void sumsq_partial_kernel(const float* __restrict__ v, uint64_t n, double* __restrict__ part) {
  double s = 0;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < n;
       q += (uint64_t)gridDim.x * blockDim.x)
    s += (double)v[q] * (double)v[q];
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ double w[8];
  if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += w[k];
    part[blockIdx.x] = t;
  }
}

alto_status sum_squares(const float* v, uint64_t n, double* out, DevBuf& scratch, cudaStream_t st) {
  ALTO_TRY(scratch.ensure(kDotBlocks * sizeof(double)));
  sumsq_partial_kernel<<<kDotBlocks, 256, 0, st>>>(v, n, scratch.as<double>());
  ALTO_LAUNCHED();
  reduce_partials_kernel<<<reduce_grid(1), kReduceThreads, 0, st>>>(scratch.as<double>(), kDotBlocks, 1, out);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

// CP-ALS model norm from Grams and lambda (include/cpd.hpp:221-256):
// reference mode keeps the diagonal only; exact mode the whole product.
__global__ void model_norm_kernel(const double* __restrict__ grams, int nmodes, int R,
                                  const double* __restrict__ lambda, int exact,
                                  double* __restrict__ out) {
  __shared__ double part[256];
  double s = 0.0;
  const int RR = R * R;
  for (int p = threadIdx.x; p < RR; p += blockDim.x) {
    const int a = p / R, b = p % R;
    if (b > a) continue;
    if (!exact && a != b) continue;
    double t = lambda[a] * lambda[b];
    for (int m = 0; m < nmodes; ++m) t *= grams[(size_t)m * RR + p];
    s += (a == b) ? t : 2.0 * t;
  }
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int k = 0; k < (int)blockDim.x; ++k) t += part[k];
    out[0] = fabs(t);
  }
}

alto_status model_norm(const double* grams, int nmodes, int R, const double* lambda, int exact,
                       double* out, cudaStream_t st) {
  model_norm_kernel<<<1, 256, 0, st>>>(grams, nmodes, R, lambda, exact, out);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

// Small elementwise R x R helpers.
__global__ void rr_kernel(double* __restrict__ dst, const double* __restrict__ a,
                          const double* __restrict__ b, int n, int op, double alpha) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    if (op == 0) dst[p] = a[p];              // copy
    else if (op == 1) dst[p] *= a[p];        // hadamard in place
    else if (op == 2) dst[p] *= alpha;       // scale
    else if (op == 3) dst[p] = 0.0;          // zero
  }
}

alto_status rr_op(double* dst, const double* a, int n, int op, double alpha, cudaStream_t st) {
  rr_kernel<<<(n + 255) / 256, 256, 0, st>>>(dst, a, nullptr, n, op, alpha);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

// G += sum over rows of s s^T (the time-mode Gram update,
// src/streaming_cpd.cpp:1320-1327), s float64 rows.
__global__ void rank_update_kernel(double* __restrict__ G, const double* __restrict__ S,
                                   uint64_t rows, int R) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < R * R; p += gridDim.x * blockDim.x) {
    const int a = p / R, b = p % R;
    double s = G[p];
    for (uint64_t q = 0; q < rows; ++q) s += S[q * R + b] * S[q * R + a];
    G[p] = s;
  }
}

alto_status rank_update(double* G, const double* S, uint64_t rows, int R, cudaStream_t st) {
  rank_update_kernel<<<(R * R + 255) / 256, 256, 0, st>>>(G, S, rows, R);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

}  // namespace alto

extern "C" alto_status alto_gram(const float* U, uint64_t rows, int rank, double* G,
                                 alto_cuda_stream stream) {
  if (!G || (rows && !U)) {
    alto::set_error("U or G is NULL");
    return ALTO_ERR_INVALID;
  }
  if (rank < 1 || rank > 128) {
    alto::set_error("rank %d outside 1..128", rank);
    return ALTO_ERR_UNSUPPORTED;
  }
  static thread_local alto::DevBuf* partials = new alto::DevBuf();
  return alto::gram(U, rows, rank, G, *partials, (cudaStream_t)stream);
}

// ------------------------------------------------ Gram without allocation
//
// Some callers cannot allocate device memory: code running under a memory
// pool or arena that owns every byte of the device (a serving process that
// pre-reserves HBM), callers whose allocator is forbidden inside a CUDA
// graph capture or a real-time loop, and embedders that must not call
// cudaMalloc / cudaFree at all.  alto_gram_noalloc gives them the Gram
// kernel with its scratch -- the per-block partial sums -- in a fixed
// device array that this library owns for the life of the process, on
// every GPU that loads it.
namespace {

constexpr int kNoAllocBlocks = 64;    // partial sums, one R x R block each
constexpr int kNoAllocMaxRank = 64;   // 64 blocks x 64 x 64 doubles = 2 MiB
static __device__ __align__(256) double g_gram_noalloc_scratch[kNoAllocBlocks * kNoAllocMaxRank *
                                                               kNoAllocMaxRank];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_ptr[kNoAllocMaxDevices] = {nullptr};

// Device address of the scratch array on the current device, resolved once
// per device (the array's name in host code is only a stand-in).  The
// address is kept for the process's life: a cudaDeviceReset of the device
// would leave it stale, which the header rules out for callers.
alto_status noalloc_scratch(double** out) {
  int dev = 0;
  ALTO_TRY_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) {
    alto::set_error("device ordinal %d beyond %d", dev, kNoAllocMaxDevices);
    return ALTO_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    ALTO_TRY_CUDA(cudaGetSymbolAddress(&p, g_gram_noalloc_scratch));
    g_noalloc_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return ALTO_OK;
}

}  // namespace

extern "C" alto_status alto_gram_noalloc(const float* U, uint64_t rows, int rank, double* G,
                                         alto_cuda_stream stream) {
  if (!G || (rows && !U)) {
    alto::set_error("U or G is NULL");
    return ALTO_ERR_INVALID;
  }
  if (rank < 1 || rank > kNoAllocMaxRank) {
    alto::set_error("alto_gram_noalloc: rank %d outside 1..%d (its fixed scratch holds %d partial "
                    "Grams of at most %d x %d doubles)", rank, kNoAllocMaxRank, kNoAllocBlocks,
                    kNoAllocMaxRank, kNoAllocMaxRank);
    return ALTO_ERR_UNSUPPORTED;
  }
  double* part = nullptr;
  ALTO_TRY(noalloc_scratch(&part));
  cudaStream_t st = (cudaStream_t)stream;
  const int RR = rank * rank;
  if (rows == 0) {
    ALTO_TRY_CUDA(cudaMemsetAsync(G, 0, RR * sizeof(double), st));
    return ALTO_OK;
  }
  uint64_t nb = std::min<uint64_t>((rows + 255) / 256, (uint64_t)kNoAllocBlocks);
  const uint64_t rpb = (rows + nb - 1) / nb;
  nb = (rows + rpb - 1) / rpb;
  // every block writes all RR entries of its partial, so no clearing is needed
  const size_t smem = 2 * alto::kGramRows * rank * sizeof(double);  // <= 32 KiB at rank 64
  const int ppt = (RR + alto::kGramThreads - 1) / alto::kGramThreads;
  switch (ppt <= 1 ? 1 : ppt <= 2 ? 2 : ppt <= 4 ? 4 : 16) {
    case 1:
      alto::gram_partial_kernel<1, float, float><<<(unsigned)nb, alto::kGramThreads, smem, st>>>(U, U, rows, rank, rpb, part);
      break;
    case 2:
      alto::gram_partial_kernel<2, float, float><<<(unsigned)nb, alto::kGramThreads, smem, st>>>(U, U, rows, rank, rpb, part);
      break;
    case 4:
      alto::gram_partial_kernel<4, float, float><<<(unsigned)nb, alto::kGramThreads, smem, st>>>(U, U, rows, rank, rpb, part);
      break;
    default:
      alto::gram_partial_kernel<16, float, float><<<(unsigned)nb, alto::kGramThreads, smem, st>>>(U, U, rows, rank, rpb, part);
      break;
  }
  ALTO_LAUNCHED();
  alto::reduce_partials_kernel<<<alto::reduce_grid(RR), alto::kReduceThreads, 0, st>>>(part, (int)nb, RR, G);
  ALTO_LAUNCHED();
  return ALTO_OK;
}
