// CP-stream on the device: a session keeps the model, the previous model,
// the Grams and the ADMM duals resident between time batches.
//
// Reference (jeewhanchoi/ALTO-stream):
//   cpstream batch loop              src/streaming_cpd.cpp:26-366
//   cpstream_alto_iter               src/streaming_cpd.cpp:1198-1519
//   admm_cf / admm_cf_               src/admm.cpp:46-66, 216-429
//   GrowKruskalModel / CopyKruskalModel src/kruskal_model.cpp:101-145
//
// Per batch: grow the model (new rows from the caller's initial values,
// previous model rows zero), recompute the non-stream Grams, zero the duals,
// encode the batch (update_salto); on the first batch 2-norm normalise the
// non-stream factors and set lambda = 1.  Inner iterations: solve the time
// rows (MTTKRP of the stream mode, Hadamard of the other Grams + 1e-12 I),
// add s s^T to the temporal Gram, then for every other mode j: MTTKRP into a
// buffer, add the historical term prev_U_j (G_t_old * prod_m prev_U_m^T U_m),
// solve (unconstrained: Cholesky; constrained: ADMM with non-negativity
// projection, rho = tr(Phi)/R, at most 25 sweeps, residual test at
// (double)1e-6f), update G_j and the change delta_j; stop when
// |delta - prev_delta| < epsilon.  After the batch: G_t *= forgetting,
// prev_U <- U, time rows appended.
//
// ADMM of a mode runs as three launches: a pass over the rows that runs all
// 25 sweeps in registers and records every sweep's stopping-test sums, a
// one-block kernel that picks the sweep count from them, and a second pass
// that reruns that many sweeps and writes the result (admm_rows_kernel).
//
// Launch structure.  The first inner iteration of a batch is issued
// directly (it sizes every buffer and builds the row-sorted lines); the
// remaining iterations run as one CUDA graph: a while node whose body is one
// inner iteration, ending in a kernel that computes delta and decides on the
// device whether to go on.  A batch costs one eager iteration, one capture
// and one graph launch, with no host synchronisation between inner
// iterations.  alto_stream_set_graph(s, 0) issues every iteration directly
// instead (the same kernels in the same order: identical results).
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "alto_dense.cuh"
#include "alto_group.cuh"

namespace alto {

constexpr int kAdmmThreads = 256;
constexpr int kAdmmMaxIters = 25;

struct AdmmState {
  int iters;         // sweeps done
  int stop;          // the test passed or 25 sweeps are done
  int converged;     // the test passed
  int chunk_start;   // sweeps done before the current chunk
  int chunk_sweeps;  // sweeps of the current chunk that stand
  unsigned ticket;   // blocks of the current pass 1 done
};

// Inner-iteration bookkeeping kept on the device.
struct IterState {
  int done;     // inner iterations executed in this batch
  int stop;     // converged, or a solve failed
  int info;     // Cholesky info of the failed ADMM solve (0 = none)
  int pad;
  double prev_delta;
  double delta;
};

// Sets a conditional node's value from a kernel in its graph (no-op when the
// kernel was launched outside a graph).
__device__ __forceinline__ void set_condition(cudaGraphConditionalHandle h, int in_graph, bool go) {
  if (in_graph) cudaGraphSetConditional(h, go ? 1u : 0u);
}

// Rows are processed by lane segments of SEG lanes (SEG = 8 or 16 for rank
// <= SEG, so 32/SEG rows share a warp; SEG = 32 otherwise, one row per warp
// with SLOTS columns per lane): lane `col` of a segment owns columns col,
// col + 32, ... of its row.
template <int SEG>
struct RowMap {
  static constexpr int kRows = 32 / SEG;  // rows per warp
  __device__ static int base(int lane) { return SEG < 32 ? (lane & ~(SEG - 1)) : 0; }
  __device__ static int col(int lane) { return SEG < 32 ? (lane & (SEG - 1)) : lane; }
  __device__ static int sub(int lane) { return SEG < 32 ? lane / SEG : 0; }
};

// Row solve: x[c] = sum_k a[k] W[k][c] for the row held by the segment
// (a given per lane slot; W in shared memory), fused multiply-adds in k order.
template <int SLOTS, int SEG>
__device__ __forceinline__ void row_solve(const double (&a)[SLOTS], const double* sw, int R,
                                          int lane, double (&x)[SLOTS]) {
  const int base = RowMap<SEG>::base(lane), col = RowMap<SEG>::col(lane);
#pragma unroll
  for (int s = 0; s < SLOTS; ++s) x[s] = 0.0;
#pragma unroll
  for (int ks = 0; ks < SLOTS; ++ks) {
    const int kbase = ks * 32;
    const int kmax = min(SEG, R - kbase);
    for (int k = 0; k < kmax; ++k) {
      const double ak = __shfl_sync(0xffffffffu, a[ks], base + k);
#pragma unroll
      for (int s = 0; s < SLOTS; ++s) {
        const int c = s * 32 + col;
        if (c < R) x[s] = __fma_rn(ak, sw[(kbase + k) * R + c], x[s]);
      }
    }
  }
}

// ADMM of one mode (admm_cf_, src/admm.cpp:288-425) in chunks of up to
// kAdmmChunk sweeps, each chunk two passes over the rows with the rows'
// state in registers.  Rows are independent except for the stopping test,
// which after every sweep compares four sums over all rows (p_res <= tol
// p_norm and d_res <= tol d_norm).  Per chunk:
//   pass 1  runs the chunk's sweeps for every row (the first chunk starts
//           with the first update) without writing the rows back, and
//           records each sweep's four sums (per block: warps in order);
//   decide  adds the blocks' sums in block order and finds the first sweep
//           of the chunk whose sums pass the test -- k sweeps, else the
//           whole chunk (25 sweeps at most in all);
//   pass 2  reruns the same k sweeps and writes primal, aux and dual.
// Both passes run the same per-row code, so the result is that of stopping
// after exactly the sweep the reference stops after.  Most solves stop
// after one or two sweeps, i.e. within the first chunk: each row is then
// read twice and written once.  Chunks repeat (a while node in the batch
// graph, or launches that return at once when issued directly) until the
// test passes or 25 sweeps are done.
//
// Per sweep, with the reference's variables (x = primal, z = aux, u = dual,
// init = x before the sweep, W = (Phi + rho I)^{-1}):
//   y = x - z;  u += y;  z = (rhs + rho (x + u)) W;  x = max(z - u, 0)
//   p_res += y^2, p_norm += x_before^2, d_norm += u^2, d_res += (x - init)^2.
// The reference sets init = x at the end of every sweep, so d_res is zero
// from the second sweep on; only the first sweep's d_res term is formed.
constexpr int kAdmmChunk = 3;
constexpr int kAdmmSums = kAdmmChunk * 4;

template <int SLOTS>
struct AdmmBatch {
  static constexpr int M = SLOTS == 1 ? 4 : (SLOTS == 2 ? 2 : 1);  // row groups per warp in registers
};

// Right-hand side of row i, mode j (src/streaming_cpd.cpp:1375-1415 and
// :1346-1373): rhs = prev_U_j[i] A + mttkrp[i], A the historical Gram
// product (global memory, L1-resident), in float64 from float32 inputs.
template <int SLOTS, int SEG>
__device__ __forceinline__ void row_rhs(const float* __restrict__ P32, const float* __restrict__ B32,
                                        const double* __restrict__ A, uint64_t i, uint64_t I, int R, int lane,
                                        double (&h)[SLOTS]) {
  const int col = RowMap<SEG>::col(lane);
  double p[SLOTS], b[SLOTS];
#pragma unroll
  for (int s = 0; s < SLOTS; ++s) {
    const int c = s * 32 + col;
    const bool ok = i < I && c < R;
    p[s] = ok ? (double)P32[i * R + c] : 0.0;
    b[s] = ok ? (double)B32[i * R + c] : 0.0;
  }
  row_solve<SLOTS, SEG>(p, A, R, lane, h);
#pragma unroll
  for (int s = 0; s < SLOTS; ++s) h[s] = __dadd_rn(h[s], b[s]);
}

// Unconstrained solve of mode j (src/streaming_cpd.cpp:1423-1431):
// U_j[i] = (prev_U_j[i] A + mttkrp[i]) W, W = (Phi + 1e-12 I)^{-1}.
// Block `block` of `nblocks` of the solve (rows in warp-sized strides).
template <int SLOTS, int SEG>
__device__ __forceinline__ void stream_solve_body(const float* __restrict__ P32, const float* __restrict__ B32,
                                                  const double* __restrict__ A, const double* __restrict__ W,
                                                  uint64_t I, int R, float* __restrict__ U32, uint32_t block,
                                                  uint32_t nblocks) {
  extern __shared__ double sw[];
  for (int p = threadIdx.x; p < R * R; p += blockDim.x) sw[p] = W[p];
  __syncthreads();
  const int lane = threadIdx.x & 31, col = RowMap<SEG>::col(lane), sub = RowMap<SEG>::sub(lane);
  const uint64_t gw = (block * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)nblocks * blockDim.x) >> 5;
  for (uint64_t i0 = gw * RowMap<SEG>::kRows; i0 < I; i0 += nw * RowMap<SEG>::kRows) {
    const uint64_t i = i0 + sub;
    double h[SLOTS], x[SLOTS];
    row_rhs<SLOTS, SEG>(P32, B32, A, i, I, R, lane, h);
    row_solve<SLOTS, SEG>(h, sw, R, lane, x);
#pragma unroll
    for (int s = 0; s < SLOTS; ++s) {
      const int c = s * 32 + col;
      if (i < I && c < R) U32[i * R + c] = (float)x[s];
    }
  }
  __syncthreads();
}

template <int SLOTS, int SEG>
__global__ void __launch_bounds__(kAdmmThreads)
    stream_solve_kernel(const float* __restrict__ P32, const float* __restrict__ B32, const double* __restrict__ A,
                        const double* __restrict__ W, uint64_t I, int R, float* __restrict__ U32) {
  stream_solve_body<SLOTS, SEG>(P32, B32, A, W, I, R, U32, blockIdx.x, gridDim.x);
}

// The ADMM rows of mode j: rhs formed on the fly from prev_U_j, the MTTKRP
// and A; the primal starts from U_j (float32) and ends in U_j; between
// chunks it is kept in float64 (prim), with aux.
// Block `block` of `nblocks` of one ADMM pass (see above).
template <int SLOTS, int SEG, bool PASS1>
__device__ __forceinline__ void admm_rows_body(const float* __restrict__ P32, const float* __restrict__ B32,
                                               const double* __restrict__ A, float* __restrict__ U32,
                                               double* __restrict__ primal, double* __restrict__ aux,
                                               double* __restrict__ dual, const double* __restrict__ W,
                                               const double* __restrict__ rho_p, uint64_t I, int R,
                                               double* __restrict__ partials, AdmmState* __restrict__ state,
                                               double tol, cudaGraphConditionalHandle h, int in_graph,
                                               uint32_t block, uint32_t nblocks) {
  constexpr int M = AdmmBatch<SLOTS>::M;
  constexpr int KR = RowMap<SEG>::kRows;
  constexpr int NW = kAdmmThreads / 32;
  if (PASS1 && state->stop) {  // a chunk after the stop (launched directly): nothing stands
    if (block == 0 && threadIdx.x == 0) state->chunk_sweeps = 0;
    return;
  }
  if (!PASS1 && state->chunk_sweeps == 0) return;
  const int start = PASS1 ? state->iters : state->chunk_start;  // sweeps done before this chunk
  const int nsweeps = PASS1 ? min(kAdmmChunk, kAdmmMaxIters - start) : state->chunk_sweeps;
  const bool first = start == 0;
  extern __shared__ double sw[];
  __shared__ double wsum[PASS1 ? NW : 1][PASS1 ? kAdmmSums : 1];
  for (int p = threadIdx.x; p < R * R; p += blockDim.x) sw[p] = W[p];
  if (PASS1)
    for (int p = threadIdx.x; p < NW * kAdmmSums; p += blockDim.x) (&wsum[0][0])[p] = 0.0;
  __syncthreads();
  const double rho = *rho_p;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int col = RowMap<SEG>::col(lane), sub = RowMap<SEG>::sub(lane);
  const uint64_t gw = (block * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)nblocks * blockDim.x) >> 5;
  for (uint64_t b0 = gw * KR * M; b0 < I; b0 += nw * KR * M) {
    double X[M][SLOTS], Z[M][SLOTS], U[M][SLOTS], H[M][SLOTS], X0[M][SLOTS];
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const uint64_t i = b0 + (uint64_t)m * KR + sub;
      double a[SLOTS], z[SLOTS];
      row_rhs<SLOTS, SEG>(P32, B32, A, i, I, R, lane, H[m]);
#pragma unroll
      for (int s = 0; s < SLOTS; ++s) {
        const int c = s * 32 + col;
        const bool ok = i < I && c < R;
        X[m][s] = ok ? (first ? (double)U32[i * R + c] : primal[i * R + c]) : 0.0;
        U[m][s] = ok ? dual[i * R + c] : 0.0;
        Z[m][s] = ok && !first ? aux[i * R + c] : 0.0;
        X0[m][s] = X[m][s];
        // first update (src/admm.cpp:288-327): z = (rhs + rho (x + u)) W
        a[s] = __fma_rn(rho, __dadd_rn(X[m][s], U[m][s]), H[m][s]);
      }
      if (first) {
        row_solve<SLOTS, SEG>(a, sw, R, lane, z);
#pragma unroll
        for (int s = 0; s < SLOTS; ++s) {
          Z[m][s] = z[s];
          const double v = __dsub_rn(z[s], U[m][s]);
          X[m][s] = v < 0.0 ? 0.0 : v;
        }
      }
    }
    for (int k = 0; k < nsweeps; ++k) {
      double p_res = 0, d_res = 0, p_norm = 0, d_norm = 0;
#pragma unroll
      for (int m = 0; m < M; ++m) {
        double a[SLOTS], z[SLOTS];
#pragma unroll
        for (int s = 0; s < SLOTS; ++s) {
          const double xv = X[m][s];
          if (PASS1) {
            if (first && k == 0) {
              const double dd = __dsub_rn(xv, X0[m][s]);
              d_res = __fma_rn(dd, dd, d_res);
            }
            p_norm = __fma_rn(xv, xv, p_norm);
          }
          const double y = __dsub_rn(xv, Z[m][s]);
          const double di = __dadd_rn(U[m][s], y);
          U[m][s] = di;
          if (PASS1) {
            d_norm = __fma_rn(di, di, d_norm);
            p_res = __fma_rn(y, y, p_res);
          }
          a[s] = __fma_rn(rho, __dadd_rn(xv, di), H[m][s]);
        }
        row_solve<SLOTS, SEG>(a, sw, R, lane, z);
#pragma unroll
        for (int s = 0; s < SLOTS; ++s) {
          Z[m][s] = z[s];
          const double v = __dsub_rn(z[s], U[m][s]);
          X[m][s] = v < 0.0 ? 0.0 : v;
        }
      }
      if (PASS1) {
        double v4[4] = {p_res, d_res, p_norm, d_norm};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          for (int o = 16; o; o >>= 1) v4[q] += __shfl_xor_sync(0xffffffffu, v4[q], o);
          if (lane == 0) wsum[warp][k * 4 + q] += v4[q];
        }
      }
    }
    if (!PASS1) {
      const bool final_chunk = state->stop != 0;
#pragma unroll
      for (int m = 0; m < M; ++m) {
        const uint64_t i = b0 + (uint64_t)m * KR + sub;
#pragma unroll
        for (int s = 0; s < SLOTS; ++s) {
          const int c = s * 32 + col;
          if (i < I && c < R) {
            dual[i * R + c] = U[m][s];
            if (final_chunk) {
              U32[i * R + c] = (float)X[m][s];
            } else {
              primal[i * R + c] = X[m][s];
              aux[i * R + c] = Z[m][s];
            }
          }
        }
      }
    }
  }
  if (PASS1) {
    __syncthreads();
    for (int p = threadIdx.x; p < kAdmmSums; p += blockDim.x) {
      double t = 0.0;
      for (int w = 0; w < NW; ++w) t += wsum[w][p];
      partials[(size_t)block * kAdmmSums + p] = t;
    }
    // the last block to finish adds the blocks' sums (warp per sum, lanes
    // over blocks in order, fixed butterfly) and takes the chunk's sweep
    // count: the first sweep whose sums pass the test, else the whole chunk
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&state->ticket, 1u) == nblocks - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    __shared__ double S[kAdmmSums];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int p = warp; p < kAdmmSums; p += NW) {
      double t = 0.0;
      for (unsigned b = lane; b < nblocks; b += 32) t += __ldcg(partials + (size_t)b * kAdmmSums + p);
      for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
      if (lane == 0) S[p] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const int n = min(kAdmmChunk, kAdmmMaxIters - start);
      int k = n, conv = 0;
      for (int j = 0; j < n; ++j)
        if (S[j * 4 + 0] <= tol * S[j * 4 + 2] && S[j * 4 + 1] <= tol * S[j * 4 + 3]) {
          k = j + 1;
          conv = 1;
          break;
        }
      state->ticket = 0;
      state->chunk_start = start;
      state->chunk_sweeps = k;
      state->iters = start + k;
      state->converged = conv;
      state->stop = conv || start + k >= kAdmmMaxIters;
      __threadfence();
      set_condition(h, in_graph, !state->stop);
    }
  }
}

template <int SLOTS, int SEG, bool PASS1>
__global__ void __launch_bounds__(kAdmmThreads)
    admm_rows_kernel(const float* __restrict__ P32, const float* __restrict__ B32, const double* __restrict__ A,
                     float* __restrict__ U32, double* __restrict__ primal, double* __restrict__ aux,
                     double* __restrict__ dual, const double* __restrict__ W, const double* __restrict__ rho_p,
                     uint64_t I, int R, double* __restrict__ partials, AdmmState* __restrict__ state, double tol,
                     cudaGraphConditionalHandle h, int in_graph) {
  admm_rows_body<SLOTS, SEG, PASS1>(P32, B32, A, U32, primal, aux, dual, W, rho_p, I, R, partials, state, tol, h,
                                    in_graph, blockIdx.x, gridDim.x);
}

// ------------------------------------------------ tiled row solves
//
// The row solves of a mode as small matrix products (ranks 8, 16, 32, 64):
// a block takes a tile of T = 2048 / R rows; thread (rg, cg) holds rows
// 2rg, 2rg + 1 and columns 4cg .. 4cg + 3 of every per-row quantity in
// registers, and each row-times-matrix product stages the tile's input rows
// in shared memory (row stride R + 1 doubles: conflict-free) and forms each
// output with fused multiply-adds in k order -- the sequence of row_solve,
// so every row's result is the one row_solve gives, without its shuffles.
template <int R>
struct TileMap {
  static constexpr int CG = R / 4;                 // column groups
  static constexpr int RGS = kAdmmThreads / CG;    // row groups
  static constexpr int T = 2 * RGS;                // rows per tile
  static constexpr int LD = R + 1;                 // padded row stride
  static constexpr size_t smem_bytes() { return (2 * R * R + (size_t)T * LD) * sizeof(double); }
};

template <int R>
uint64_t tile_blocks(uint64_t I, uint64_t cap) {
  const uint64_t b = std::min<uint64_t>((I + TileMap<R>::T - 1) / TileMap<R>::T, cap);
  return std::max<uint64_t>(b, 1);
}

// x[i][j] = sum_k in[r0 + i][k] M[k][c0 + j], k ascending.
template <int R>
__device__ __forceinline__ void tile_product(const double* __restrict__ in, const double* __restrict__ M, int r0,
                                             int c0, double (&x)[2][4]) {
  constexpr int LD = TileMap<R>::LD;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) x[i][j] = 0.0;
#pragma unroll 8
  for (int k = 0; k < R; ++k) {
    const double a0 = in[r0 * LD + k], a1 = in[(r0 + 1) * LD + k];
    const double2 w01 = *reinterpret_cast<const double2*>(M + k * R + c0);
    const double2 w23 = *reinterpret_cast<const double2*>(M + k * R + c0 + 2);
    x[0][0] = __fma_rn(a0, w01.x, x[0][0]);
    x[0][1] = __fma_rn(a0, w01.y, x[0][1]);
    x[0][2] = __fma_rn(a0, w23.x, x[0][2]);
    x[0][3] = __fma_rn(a0, w23.y, x[0][3]);
    x[1][0] = __fma_rn(a1, w01.x, x[1][0]);
    x[1][1] = __fma_rn(a1, w01.y, x[1][1]);
    x[1][2] = __fma_rn(a1, w23.x, x[1][2]);
    x[1][3] = __fma_rn(a1, w23.y, x[1][3]);
  }
}

// Stage v (this thread's 2 x 4 block) into the tile's rows, multiply by M,
// and return the product in x (barriers on both sides).
template <int R>
__device__ __forceinline__ void tile_stage_product(double* in, const double* M, int r0, int c0,
                                                   const double (&v)[2][4], double (&x)[2][4]) {
  constexpr int LD = TileMap<R>::LD;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) in[(r0 + i) * LD + c0 + j] = v[i][j];
  __syncthreads();
  tile_product<R>(in, M, r0, c0, x);
  __syncthreads();
}

// Right-hand sides of a tile's rows: h = prev_U_j[i] A + mttkrp[i] (row_rhs).
template <int R>
__device__ __forceinline__ void tile_rhs(const float* __restrict__ P32, const float* __restrict__ B32, double* in,
                                         const double* sA, uint64_t t0, uint64_t I, int r0, int c0,
                                         double (&h)[2][4]) {
  double p[2][4];
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const uint64_t row = t0 + r0 + i;
#pragma unroll
    for (int j = 0; j < 4; ++j) p[i][j] = row < I ? (double)P32[row * R + c0 + j] : 0.0;
  }
  tile_stage_product<R>(in, sA, r0, c0, p, h);
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const uint64_t row = t0 + r0 + i;
#pragma unroll
    for (int j = 0; j < 4; ++j) h[i][j] = __dadd_rn(h[i][j], row < I ? (double)B32[row * R + c0 + j] : 0.0);
  }
}

template <int R>
__device__ __forceinline__ void tile_load_mats(double* smem, const double* __restrict__ A,
                                               const double* __restrict__ W) {
  for (int p = threadIdx.x; p < R * R; p += blockDim.x) {
    smem[p] = W[p];
    smem[R * R + p] = A[p];
  }
  __syncthreads();
}

// Unconstrained solve of mode j, tiled: U_j[i] = (prev_U_j[i] A + mttkrp[i]) W.
template <int R>
__device__ __forceinline__ void solve_tile_body(const float* __restrict__ P32, const float* __restrict__ B32,
                                                const double* __restrict__ A, const double* __restrict__ W,
                                                uint64_t I, float* __restrict__ U32, uint32_t block,
                                                uint32_t nblocks) {
  using TM = TileMap<R>;
  extern __shared__ double smem[];
  double* sW = smem;
  double* sA = smem + R * R;
  double* in = smem + 2 * R * R;
  tile_load_mats<R>(smem, A, W);
  const int cg = threadIdx.x % TM::CG, rg = threadIdx.x / TM::CG;
  const int r0 = 2 * rg, c0 = 4 * cg;
  for (uint64_t t0 = (uint64_t)block * TM::T; t0 < I; t0 += (uint64_t)nblocks * TM::T) {
    double h[2][4], x[2][4];
    tile_rhs<R>(P32, B32, in, sA, t0, I, r0, c0, h);
    tile_stage_product<R>(in, sW, r0, c0, h, x);
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const uint64_t row = t0 + r0 + i;
      if (row < I)
#pragma unroll
        for (int j = 0; j < 4; ++j) U32[row * R + c0 + j] = (float)x[i][j];
    }
  }
  __syncthreads();
}

template <int R>
__global__ void __launch_bounds__(kAdmmThreads)
    solve_tile_kernel(const float* __restrict__ P32, const float* __restrict__ B32, const double* __restrict__ A,
                      const double* __restrict__ W, uint64_t I, float* __restrict__ U32) {
  solve_tile_body<R>(P32, B32, A, W, I, U32, blockIdx.x, gridDim.x);
}

// One ADMM pass of mode j, tiled (the passes, the decision and the state
// are those of admm_rows_kernel; see there).
template <int R, bool PASS1>
__device__ __forceinline__ void admm_tile_body(const float* __restrict__ P32, const float* __restrict__ B32,
                                               const double* __restrict__ A, float* __restrict__ U32,
                                               double* __restrict__ primal, double* __restrict__ aux,
                                               double* __restrict__ dual, const double* __restrict__ W,
                                               const double* __restrict__ rho_p, uint64_t I,
                                               double* __restrict__ partials, AdmmState* __restrict__ state,
                                               double tol, cudaGraphConditionalHandle h, int in_graph,
                                               uint32_t block, uint32_t nblocks) {
  using TM = TileMap<R>;
  constexpr int NW = kAdmmThreads / 32;
  if (PASS1 && state->stop) {  // a chunk after the stop (launched directly): nothing stands
    if (block == 0 && threadIdx.x == 0) state->chunk_sweeps = 0;
    return;
  }
  if (!PASS1 && state->chunk_sweeps == 0) return;
  const int start = PASS1 ? state->iters : state->chunk_start;
  const int nsweeps = PASS1 ? min(kAdmmChunk, kAdmmMaxIters - start) : state->chunk_sweeps;
  const bool first = start == 0;
  extern __shared__ double smem[];
  double* sW = smem;
  double* sA = smem + R * R;
  double* in = smem + 2 * R * R;
  __shared__ double wsum[kAdmmSums];
  __shared__ double red[NW][4];
  if (PASS1)
    for (int p = threadIdx.x; p < kAdmmSums; p += blockDim.x) wsum[p] = 0.0;
  tile_load_mats<R>(smem, A, W);
  const double rho = *rho_p;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int cg = threadIdx.x % TM::CG, rg = threadIdx.x / TM::CG;
  const int r0 = 2 * rg, c0 = 4 * cg;
  for (uint64_t t0 = (uint64_t)block * TM::T; t0 < I; t0 += (uint64_t)nblocks * TM::T) {
    double H[2][4], X[2][4], Z[2][4], U[2][4], X0[2][4], a[2][4], z[2][4];
    tile_rhs<R>(P32, B32, in, sA, t0, I, r0, c0, H);
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const uint64_t row = t0 + r0 + i;
      const bool ok = row < I;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const uint64_t e = row * R + c0 + j;
        X[i][j] = ok ? (first ? (double)U32[e] : primal[e]) : 0.0;
        U[i][j] = ok ? dual[e] : 0.0;
        Z[i][j] = ok && !first ? aux[e] : 0.0;
        X0[i][j] = X[i][j];
        // first update (src/admm.cpp:288-327): z = (rhs + rho (x + u)) W
        a[i][j] = __fma_rn(rho, __dadd_rn(X[i][j], U[i][j]), H[i][j]);
      }
    }
    if (first) {
      tile_stage_product<R>(in, sW, r0, c0, a, z);
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          Z[i][j] = z[i][j];
          const double v = __dsub_rn(z[i][j], U[i][j]);
          X[i][j] = v < 0.0 ? 0.0 : v;
        }
    }
    for (int k = 0; k < nsweeps; ++k) {
      double p_res = 0, d_res = 0, p_norm = 0, d_norm = 0;
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const double xv = X[i][j];
          if (PASS1) {
            if (first && k == 0) {
              const double dd = __dsub_rn(xv, X0[i][j]);
              d_res = __fma_rn(dd, dd, d_res);
            }
            p_norm = __fma_rn(xv, xv, p_norm);
          }
          const double y = __dsub_rn(xv, Z[i][j]);
          const double di = __dadd_rn(U[i][j], y);
          U[i][j] = di;
          if (PASS1) {
            d_norm = __fma_rn(di, di, d_norm);
            p_res = __fma_rn(y, y, p_res);
          }
          a[i][j] = __fma_rn(rho, __dadd_rn(xv, di), H[i][j]);
        }
      tile_stage_product<R>(in, sW, r0, c0, a, z);
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          Z[i][j] = z[i][j];
          const double v = __dsub_rn(z[i][j], U[i][j]);
          X[i][j] = v < 0.0 ? 0.0 : v;
        }
      if (PASS1) {  // the tile's four sums: lanes, then warps in order, added per tile
        double v4[4] = {p_res, d_res, p_norm, d_norm};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          for (int o = 16; o; o >>= 1) v4[q] += __shfl_xor_sync(0xffffffffu, v4[q], o);
          if (lane == 0) red[warp][q] = v4[q];
        }
        __syncthreads();
        if (threadIdx.x < 4) {
          double t = 0.0;
          for (int w = 0; w < NW; ++w) t += red[w][threadIdx.x];
          wsum[k * 4 + threadIdx.x] += t;
        }
        __syncthreads();
      }
    }
    if (!PASS1) {
      const bool final_chunk = state->stop != 0;
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const uint64_t row = t0 + r0 + i;
        if (row >= I) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const uint64_t e = row * R + c0 + j;
          dual[e] = U[i][j];
          if (final_chunk) {
            U32[e] = (float)X[i][j];
          } else {
            primal[e] = X[i][j];
            aux[e] = Z[i][j];
          }
        }
      }
    }
  }
  if (PASS1) {
    __syncthreads();
    for (int p = threadIdx.x; p < kAdmmSums; p += blockDim.x) partials[(size_t)block * kAdmmSums + p] = wsum[p];
    // the last block to finish adds the blocks' sums (warp per sum, lanes
    // over blocks in order, fixed butterfly) and takes the chunk's sweep
    // count: the first sweep whose sums pass the test, else the whole chunk
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&state->ticket, 1u) == nblocks - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    __shared__ double S[kAdmmSums];
    for (int p = warp; p < kAdmmSums; p += NW) {
      double t = 0.0;
      for (unsigned b = lane; b < nblocks; b += 32) t += __ldcg(partials + (size_t)b * kAdmmSums + p);
      for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
      if (lane == 0) S[p] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const int n = min(kAdmmChunk, kAdmmMaxIters - start);
      int kk = n, conv = 0;
      for (int j = 0; j < n; ++j)
        if (S[j * 4 + 0] <= tol * S[j * 4 + 2] && S[j * 4 + 1] <= tol * S[j * 4 + 3]) {
          kk = j + 1;
          conv = 1;
          break;
        }
      state->ticket = 0;
      state->chunk_start = start;
      state->chunk_sweeps = kk;
      state->iters = start + kk;
      state->converged = conv;
      state->stop = conv || start + kk >= kAdmmMaxIters;
      __threadfence();
      set_condition(h, in_graph, !state->stop);
    }
  }
}

template <int R, bool PASS1>
__global__ void __launch_bounds__(kAdmmThreads)
    admm_tile_kernel(const float* __restrict__ P32, const float* __restrict__ B32, const double* __restrict__ A,
                     float* __restrict__ U32, double* __restrict__ primal, double* __restrict__ aux,
                     double* __restrict__ dual, const double* __restrict__ W, const double* __restrict__ rho_p,
                     uint64_t I, double* __restrict__ partials, AdmmState* __restrict__ state, double tol,
                     cudaGraphConditionalHandle h, int in_graph) {
  admm_tile_body<R, PASS1>(P32, B32, A, U32, primal, aux, dual, W, rho_p, I, partials, state, tol, h, in_graph,
                           blockIdx.x, gridDim.x);
}

// End of an inner iteration (src/streaming_cpd.cpp:1457-1482): delta = sum
// over the non-stream modes of ||U_j - prev_U_j|| / (||U_j|| + 1e-12) from
// the per-mode statistics; stop once |prev_delta - delta| < epsilon after
// the first iteration, when max_inner iterations are done, or when the
// constrained solve's Cholesky failed.
// The decision itself (one thread); returns whether the batch goes on.
__device__ __forceinline__ bool converge_step(const double* __restrict__ dstat, int N, int t,
                                              const int* __restrict__ status, int constrained, double eps,
                                              int max_inner, IterState* __restrict__ it, int sparse) {
  double delta = 0.0;
  for (int j = 0; j < N; ++j)
    if (j != t)
      delta += sparse ? dstat[3 * j] : sqrt(dstat[3 * j + 1]) / (sqrt(dstat[3 * j + 2]) + 1e-12);
  const int k = it->done;
  bool stop = false;
  if (constrained && status[0]) {
    it->info = status[0];
    stop = true;
  } else if (k > 0 && fabs(it->prev_delta - delta) < eps) {
    stop = true;
  } else {
    it->prev_delta = delta;
  }
  it->delta = delta;
  it->done = k + 1;
  if (stop) it->stop = 1;
  return !stop && k + 1 < max_inner;
}

__global__ void converge_kernel(const double* __restrict__ dstat, int N, int t, const int* __restrict__ status,
                                int constrained, double eps, int max_inner, IterState* __restrict__ it,
                                cudaGraphConditionalHandle h, int in_graph, int sparse) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  set_condition(h, in_graph, converge_step(dstat, N, t, status, constrained, eps, max_inner, it, sparse));
}

// The time rows after their solve set-up, one block: s = mttkrp W (float64,
// k order) into time64 and, rounded, into the float32 factor rows; old =
// G_t; G_t += sum_rows s s^T (the operations of apply, convert, copy and
// rank update, in their order).
__device__ __forceinline__ void time_update_body(const float* __restrict__ B32, const double* __restrict__ W,
                                                 uint64_t rows, int R, double* __restrict__ time64,
                                                 float* __restrict__ U32, double* __restrict__ Gt,
                                                 double* __restrict__ old_gram) {
  const int RR = R * R;
  for (uint64_t q = threadIdx.x; q < rows * R; q += blockDim.x) {
    const uint64_t i = q / R;
    const int c = (int)(q % R);
    double x = 0.0;
    for (int k = 0; k < R; ++k) x = __fma_rn((double)B32[i * R + k], W[k * R + c], x);
    time64[q] = x;
    U32[q] = (float)x;
  }
  for (int p = threadIdx.x; p < RR; p += blockDim.x) old_gram[p] = Gt[p];
  __syncthreads();
  for (int p = threadIdx.x; p < RR; p += blockDim.x) {
    const int a = p / R, b = p % R;
    double sv = Gt[p];
    for (uint64_t q = 0; q < rows; ++q) sv += time64[q * R + b] * time64[q * R + a];
    Gt[p] = sv;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(256)
    time_update_kernel(const float* __restrict__ B32, const double* __restrict__ W, uint64_t rows, int R,
                       double* __restrict__ time64, float* __restrict__ U32, double* __restrict__ Gt,
                       double* __restrict__ old_gram) {
  time_update_body(B32, W, rows, R, time64, U32, Gt, old_gram);
}

// Per mode before its solve: the historical product A = base *
// prod_{m in mask} src[m] (base NULL: 1), and, for a constrained mode, the
// ADMM state cleared and its chunk loop opened.
__device__ __forceinline__ void mode_prep_body(const double* __restrict__ base, const double* __restrict__ src,
                                               unsigned mask, int N, int RR, double* __restrict__ A,
                                               AdmmState* __restrict__ admm) {
  for (int p = threadIdx.x; p < RR; p += blockDim.x) {
    double v = base ? base[p] : 1.0;
    for (int m = 0; m < N; ++m)
      if (mask & (1u << m)) v *= src[(size_t)m * RR + p];
    A[p] = v;
  }
  if (admm && threadIdx.x == 0) {
    admm->iters = 0;
    admm->stop = 0;
    admm->converged = 0;
    admm->chunk_start = 0;
    admm->chunk_sweeps = 0;
    admm->ticket = 0;
  }
  __syncthreads();
}

__global__ void mode_prep_kernel(const double* __restrict__ base, const double* __restrict__ src, unsigned mask,
                                 int N, int RR, double* __restrict__ A, AdmmState* __restrict__ admm,
                                 cudaGraphConditionalHandle h, int in_graph) {
  mode_prep_body(base, src, mask, N, RR, A, admm);
  if (admm && threadIdx.x == 0) set_condition(h, in_graph, true);
}

// Head of the iteration graph: run the loop only if the batch goes on.
__global__ void iter_begin_kernel(const IterState* __restrict__ it, int max_inner, cudaGraphConditionalHandle h) {
  if (threadIdx.x == 0 && blockIdx.x == 0) cudaGraphSetConditional(h, (!it->stop && it->done < max_inner) ? 1u : 0u);
}


// ------------------------------------------------------------ spCP-stream
//
// spcpstream_alto_iter (src/streaming_cpd.cpp:466-1085) works on the rows a
// batch touches.  Per batch and mode: a row map (nonzero_slices,
// :1127-1161; here flags, an exclusive scan and a list), the batch with its
// indices renumbered to those rows and encoded (update_salto_rowsparse), the
// touched rows of the model and the previous model gathered into compact
// factors (A_nz, A_nz_prev).  Per inner iteration only the compact rows are
// solved; the untouched rows enter through R x R Grams kept per mode:
// c = U^T U and h = prev_U^T U, split into touched (c_nz, h_nz) and
// untouched parts (c_z, h_z), the latter updated in closed form through
// Q Phi^{-1}.  After the loop the untouched rows become prev_U Q Phi^{-1}.

// R x R float64 state of spCP-stream per mode, [kind][mode][R][R].
enum { kSpCPrev = 0, kSpCNzPrev, kSpCNz, kSpCZ, kSpHNz, kSpHZ, kSpCZPrev, kSpQPi, kSpKinds };

__global__ void mark_rows_kernel(const uint64_t* __restrict__ idx, uint64_t nnz, uint32_t* __restrict__ flags) {
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < nnz; q += (uint64_t)gridDim.x * blockDim.x)
    flags[idx[q]] = 1u;
}

// After the exclusive scan of the flags (dims + 1 entries): row i is touched
// iff ridx[i + 1] != ridx[i], and then its compact index is ridx[i].
__global__ void row_list_kernel(const uint32_t* __restrict__ ridx, uint64_t dims, uint32_t* __restrict__ nz) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dims; i += (uint64_t)gridDim.x * blockDim.x)
    if (ridx[i + 1] != ridx[i]) nz[ridx[i]] = (uint32_t)i;
}

// A device batch in the spCP-stream staging layout: uint64 indices, float64 values.
__global__ void widen_u32_kernel(const uint32_t* __restrict__ in, uint64_t n, uint64_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = in[i];
}
__global__ void widen_f32_kernel(const float* __restrict__ in, uint64_t n, double* __restrict__ out) {
  for (uint64_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = in[i];
}

__global__ void renumber_kernel(uint64_t* __restrict__ idx, uint64_t nnz, const uint32_t* __restrict__ ridx) {
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < nnz; q += (uint64_t)gridDim.x * blockDim.x)
    idx[q] = ridx[idx[q]];
}

__global__ void gather_rows_kernel(const float* __restrict__ src, const uint32_t* __restrict__ nz, uint64_t n, int R,
                                   float* __restrict__ dst) {
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < n * R; q += (uint64_t)gridDim.x * blockDim.x)
    dst[q] = src[(uint64_t)nz[q / R] * R + q % R];
}

__global__ void sub_kernel(const double* __restrict__ a, const double* __restrict__ b, int n, double* __restrict__ out) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) out[p] = a[p] - b[p];
}

// The Gram bookkeeping of mode m after its rows were solved (:903-975):
// QPi = Q W (Q Phi^{-1}); h_z = c_z_prev QPi; c_z = QPi^T h_z; c = c_nz + c_z;
// h = h_nz + h_z; delta_m = sqrt(|(tr c + tr c_prev - 2 tr h) / (tr c + 1e-12)|).
// One block; products in k order.
__global__ void __launch_bounds__(256)
    sp_gram_update_kernel(const double* __restrict__ Q, const double* __restrict__ W, const double* __restrict__ c_z_prev,
                          const double* __restrict__ c_nz, const double* __restrict__ h_nz,
                          const double* __restrict__ c_prev, int R, double* __restrict__ QPi, double* __restrict__ h_z,
                          double* __restrict__ c_z, double* __restrict__ c, double* __restrict__ h,
                          double* __restrict__ delta_out) {
  const int RR = R * R;
  for (int p = threadIdx.x; p < RR; p += blockDim.x) {
    const int a = p / R, b = p % R;
    double x = 0.0;
    for (int k = 0; k < R; ++k) x += Q[a * R + k] * W[k * R + b];
    QPi[p] = x;
  }
  __syncthreads();
  for (int p = threadIdx.x; p < RR; p += blockDim.x) {
    const int a = p / R, b = p % R;
    double x = 0.0;
    for (int k = 0; k < R; ++k) x += c_z_prev[a * R + k] * QPi[k * R + b];
    h_z[p] = x;
  }
  __syncthreads();
  for (int p = threadIdx.x; p < RR; p += blockDim.x) {
    const int a = p / R, b = p % R;
    double x = 0.0;
    for (int k = 0; k < R; ++k) x += QPi[k * R + a] * h_z[k * R + b];
    c_z[p] = x;
    c[p] = c_nz[p] + x;
    h[p] = h_nz[p] + h_z[p];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double trc = 0.0, trh = 0.0, trp = 0.0;
    for (int r = 0; r < R; ++r) {
      trc += c[r * R + r];
      trh += h[r * R + r];
      trp += c_prev[r * R + r];
    }
    *delta_out = sqrt(fabs((trc + trp - 2.0 * trh) / (trc + 1e-12)));
  }
}

// The model after the inner loop (:985-1024): touched rows from A_nz,
// untouched rows prev_U QPi.
template <int SLOTS, int SEG>
__global__ void __launch_bounds__(kAdmmThreads)
    sp_final_rows_kernel(const float* __restrict__ P32, const float* __restrict__ Anz, const uint32_t* __restrict__ ridx,
                         const double* __restrict__ QPi, uint64_t I, int R, float* __restrict__ U32) {
  extern __shared__ double sw[];
  for (int p = threadIdx.x; p < R * R; p += blockDim.x) sw[p] = QPi[p];
  __syncthreads();
  const int lane = threadIdx.x & 31, col = RowMap<SEG>::col(lane), sub = RowMap<SEG>::sub(lane);
  const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t i0 = gw * RowMap<SEG>::kRows; i0 < I; i0 += nw * RowMap<SEG>::kRows) {
    const uint64_t i = i0 + sub;
    const bool ok = i < I;
    double p[SLOTS], x[SLOTS];
#pragma unroll
    for (int s = 0; s < SLOTS; ++s) {
      const int c = s * 32 + col;
      p[s] = ok && c < R ? (double)P32[i * R + c] : 0.0;
    }
    row_solve<SLOTS, SEG>(p, sw, R, lane, x);
    if (!ok) continue;
    const uint32_t r0 = ridx[i], r1 = ridx[i + 1];
#pragma unroll
    for (int s = 0; s < SLOTS; ++s) {
      const int c = s * 32 + col;
      if (c < R) U32[i * R + c] = r1 != r0 ? Anz[(uint64_t)r0 * R + c] : (float)x[s];
    }
  }
}

// ------------------------------------------------ grouped inner iterations
//
// Many sessions' inner iterations in the same launches: a device table holds
// one descriptor per session (its state's pointers, sizes and the items of
// its per-mode MTTKRPs, solve set-ups and Gram passes), and every kernel
// below runs the single-session kernel's per-block code for each session in
// turn, over "virtual blocks": session s gets exactly the blocks its own
// launch would have (the prefix sums in the offset tables map a global block
// index to (session, block)), so each session's arithmetic, and its order,
// are those of its own launches -- a session's result does not depend on
// which other sessions share the launches.  A session whose batch has
// converged (or ran out of iterations) is skipped (act = 0).

constexpr int kGroupOffKinds = 5;  // tiles, Gram blocks, Gram reduction blocks, ADMM blocks, solve blocks
enum { kOffTile = 0, kOffGram, kOffGramRed, kOffAdmm, kOffSolve };

struct SlotDesc {
  DetItem det[ALTO_MAX_MODES];      // MTTKRP of each mode into buf32
  SetupItem setup[ALTO_MAX_MODES];  // solve set-up of each mode (the stream mode: the time rows)
  GramItem gram[ALTO_MAX_MODES];    // Gram, cross Gram and statistics of each non-stream mode
  uint64_t dims[ALTO_MAX_MODES];
  float* U[ALTO_MAX_MODES];
  float* P[ALTO_MAX_MODES];
  double* dual[ALTO_MAX_MODES];
  uint32_t admm_blocks[ALTO_MAX_MODES];
  uint32_t solve_blocks[ALTO_MAX_MODES];
  double *G, *old_gram, *ata, *cross, *W, *rho, *dstat, *aux, *prim, *time64, *admm_part;
  int* status;
  float* buf32;
  AdmmState* admm;
  IterState* iter;
  double eps;
  int con;        // 1: non-negative ADMM solves
  int max_inner;
  int act;        // runs the current step (set on the device)
  int admm_act;   // its ADMM of the current mode still sweeps (set on the device)
};

// Control block of a group (device): live slots, steps allowed and done in
// the current launch, and per slot the state after the last step.
struct GroupCtl {
  int count;
  int limit;
  int steps;
  int any;
  int chunks;  // ADMM chunks of the current mode's loop
  int error;   // 1: an ADMM loop overran its bound and was stopped
};

// ADMM sweeps stop after kAdmmMaxIters, so a mode's chunk loop ends within
// this many chunks; a loop still going past it is stopped with an error
// (a guard: it cannot happen while every live slot's decision runs).
constexpr int kAdmmChunkBound = (kAdmmMaxIters + kAdmmChunk - 1) / kAdmmChunk + 2;
struct SlotState {
  int running;  // takes part in further steps
  int done;     // inner iterations of the batch so far
  int stop;
  int info;
};

__device__ __forceinline__ bool slot_runnable(const SlotDesc& d) {
  return !d.iter->stop && d.iter->done < d.max_inner;
}

__device__ __forceinline__ int slot_of(const uint32_t* __restrict__ off, int K, uint32_t v) {
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

// Before the step loop of a launch: steps = 0; the loop runs if some slot can.
__global__ void group_begin_kernel(SlotDesc* __restrict__ tab, GroupCtl* __restrict__ ctl,
                                   cudaGraphConditionalHandle h) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  bool any = false;
  for (int s = 0; s < ctl->count; ++s) any = any || slot_runnable(tab[s]);
  ctl->steps = 0;
  cudaGraphSetConditional(h, (any && ctl->limit > 0) ? 1u : 0u);
}

__global__ void group_step_begin_kernel(SlotDesc* __restrict__ tab, const GroupCtl* __restrict__ ctl) {
  for (int s = threadIdx.x; s < ctl->count; s += blockDim.x) tab[s].act = slot_runnable(tab[s]) ? 1 : 0;
}

__global__ void __launch_bounds__(256) group_time_update_kernel(const SlotDesc* __restrict__ tab,
                                                                const GroupCtl* __restrict__ ctl, int t, int R) {
  const size_t RR = (size_t)R * R;
  for (int s = blockIdx.x; s < ctl->count; s += gridDim.x) {
    const SlotDesc& d = tab[s];
    if (!d.act) continue;
    time_update_body(d.buf32, d.W, d.dims[t], R, d.time64, d.U[t], d.G + t * RR, d.old_gram);
  }
}

__global__ void __launch_bounds__(256) group_mode_prep_kernel(SlotDesc* __restrict__ tab,
                                                              const GroupCtl* __restrict__ ctl, int j, int t,
                                                              int N, int R) {
  const int RR = R * R;
  const unsigned mask = ((1u << N) - 1) & ~(1u << j) & ~(1u << t);
  for (int s = blockIdx.x; s < ctl->count; s += gridDim.x) {
    SlotDesc& d = tab[s];
    if (!d.act) continue;
    mode_prep_body(d.old_gram, d.cross, mask, N, RR, d.ata, d.con ? d.admm : nullptr);
    if (threadIdx.x == 0) d.admm_act = d.con;
  }
}

template <int R>
__global__ void __launch_bounds__(kAdmmThreads)
    group_solve_kernel(const SlotDesc* __restrict__ tab, const GroupCtl* __restrict__ ctl,
                       const uint32_t* __restrict__ off, int j) {
  const int K = ctl->count;
  const uint32_t total = K > 0 ? off[K] : 0;
  for (uint32_t v = blockIdx.x; v < total; v += gridDim.x) {
    const int s = slot_of(off, K, v);
    const SlotDesc& d = tab[s];
    if (!d.act || d.con) continue;
    solve_tile_body<R>(d.P[j], d.buf32, d.ata, d.W, d.dims[j], d.U[j], v - off[s], d.solve_blocks[j]);
  }
}

// The ADMM chunk loop goes on while some slot's ADMM of mode j sweeps
// (first: before the loop, which resets the chunk count).
__global__ void group_admm_cond_kernel(SlotDesc* __restrict__ tab, GroupCtl* __restrict__ ctl,
                                       cudaGraphConditionalHandle h, int first) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  bool any = false;
  for (int s = 0; s < ctl->count; ++s) {
    SlotDesc& d = tab[s];
    if (d.act && d.admm_act && d.admm->stop) d.admm_act = 0;
    any = any || (d.act && d.admm_act);
  }
  ctl->chunks = first ? 0 : ctl->chunks + 1;
  if (any && ctl->chunks >= kAdmmChunkBound) {
    ctl->error = 1;
    any = false;
  }
  cudaGraphSetConditional(h, any ? 1u : 0u);
}

template <int R, bool PASS1>
__global__ void __launch_bounds__(kAdmmThreads)
    group_admm_kernel(const SlotDesc* __restrict__ tab, const GroupCtl* __restrict__ ctl,
                      const uint32_t* __restrict__ off, int j, double tol) {
  const int K = ctl->count;
  const uint32_t total = K > 0 ? off[K] : 0;
  for (uint32_t v = blockIdx.x; v < total; v += gridDim.x) {
    const int s = slot_of(off, K, v);
    const SlotDesc& d = tab[s];
    if (!d.act || !d.admm_act) continue;
    admm_tile_body<R, PASS1>(d.P[j], d.buf32, d.ata, d.U[j], d.prim, d.aux, d.dual[j], d.W, d.rho, d.dims[j],
                             d.admm_part, d.admm, tol, cudaGraphConditionalHandle{}, 0, v - off[s],
                             d.admm_blocks[j]);
    __syncthreads();
  }
}

// End of a step: each acting slot's convergence decision; the loop goes on
// while a slot can run and the launch's step allowance lasts.
__global__ void group_converge_kernel(SlotDesc* __restrict__ tab, GroupCtl* __restrict__ ctl,
                                      SlotState* __restrict__ out, int N, int t, cudaGraphConditionalHandle h) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  bool any = false;
  for (int s = 0; s < ctl->count; ++s) {
    SlotDesc& d = tab[s];
    if (d.act) converge_step(d.dstat, N, t, d.status, d.con, d.eps, d.max_inner, d.iter, 0);
    const bool run = slot_runnable(d);
    out[s] = SlotState{run ? 1 : 0, d.iter->done, d.iter->stop, d.iter->info};
    any = any || run;
  }
  ctl->steps += 1;
  ctl->any = any ? 1 : 0;
  cudaGraphSetConditional(h, (any && ctl->steps < ctl->limit) ? 1u : 0u);
}

}  // namespace alto

using namespace alto;

struct alto_stream_session {
  int N = 0, t = 0, R = 0;
  alto_constraint con = ALTO_UNCONSTRAINED;
  double forgetting = 0.99;
  int max_inner = 10;
  double eps = 1e-5;
  cudaStream_t st = nullptr;
  int batches = 0;
  uint64_t dims[ALTO_MAX_MODES] = {0};
  uint64_t cap[ALTO_MAX_MODES] = {0};
  DevBuf U[ALTO_MAX_MODES], P[ALTO_MAX_MODES], dual[ALTO_MAX_MODES];
  DevBuf G, old_gram, ata, cross, W, status, rho, lam, dstat, buf32, aux, prim, time64;
  DevBuf gscr, dscr, admm_part, admm_state, grow_stage, copy_tmp, iter;
  std::vector<double> time_rows;  // concatenated time factor (host)
  alto_tensor* at = nullptr;
  bool use_graph = true;              // inner iterations 1.. as one graph per batch
  // spCP-stream (alto_stream_set_model): rows the batch touches, their maps
  // and compact factors, the R x R Gram state, the batch on the device
  bool sparse = false;
  uint64_t nnzr[ALTO_MAX_MODES] = {0};
  DevBuf ridx[ALTO_MAX_MODES], nzl[ALTO_MAX_MODES], Anz[ALTO_MAX_MODES], Aprev[ALTO_MAX_MODES];
  DevBuf spg, coo_idx, coo_val;
  cudaStream_t capst[2] = {nullptr, nullptr};  // capture-only streams (nothing runs on them)
  // grouped inner iterations: this batch's per-mode MTTKRP items, and the
  // private group (of this session alone) that runs them when the session
  // is not served with others
  DetItem det[ALTO_MAX_MODES];
  alto::StreamGroup* own_group = nullptr;
  // alto_stream_stats: host seconds per phase of the pushes, device ms of
  // their inner iterations (between the two events), pushes, iterations
  double t_prepare = 0, t_inner = 0, t_finish = 0, dev_inner_ms = 0;
  double t_grow = 0, t_encode = 0, t_sorted = 0;  // parts of t_prepare
  uint64_t pushes = 0, inner_total = 0;
  cudaEvent_t inner_ev[2] = {nullptr, nullptr};
  // pinned staging of the new model rows (grown geometrically; the
  // previous push's copies out of it are complete when a push starts)
  float* pin_rows = nullptr;
  size_t pin_cap = 0;
  ~alto_stream_session() {
    alto::group_destroy(own_group);
    delete at;
    for (cudaStream_t c : capst)
      if (c) cudaStreamDestroy(c);
    for (cudaEvent_t e : inner_ev)
      if (e) cudaEventDestroy(e);
    if (pin_rows) cudaFreeHost(pin_rows);
  }
};

namespace {

// At least n bytes, growing by half again past the request, so a buffer
// that grows slice by slice is reallocated a logarithmic number of times.
alto_status ensure_headroom(DevBuf& b, size_t n) {
  if (n <= b.bytes && b.p) return ALTO_OK;
  return b.ensure(std::max(n, b.bytes + b.bytes / 2));
}

// b grown to new_cap rows keeping its first old_rows: the new buffer is
// allocated first and the kept rows copied into it directly; the old one is
// freed once the copy is done.
alto_status grow_rows(DevBuf& b, uint64_t old_rows, uint64_t new_cap, size_t row_bytes, cudaStream_t st) {
  if (b.bytes >= new_cap * row_bytes && b.p) return ALTO_OK;
  const size_t keep = std::min<size_t>(old_rows * row_bytes, b.p ? b.bytes : 0);
  DevBuf nb;
  ALTO_TRY(nb.ensure(new_cap * row_bytes));
  if (keep) {
    ALTO_TRY_CUDA(cudaMemcpyAsync(nb.p, b.p, keep, cudaMemcpyDeviceToDevice, st));
    ALTO_TRY_CUDA(cudaStreamSynchronize(st));  // (the old buffer is freed below)
  }
  std::swap(b.p, nb.p);
  std::swap(b.bytes, nb.bytes);
  return ALTO_OK;  // nb, now the old buffer, is released here
}

__global__ void lambda_from_gram_kernel(const double* __restrict__ G, int R, double* __restrict__ lam) {
  for (int r = threadIdx.x; r < R; r += blockDim.x) {
    const double s = G[r * R + r];
    lam[r] = sqrt(s > 1e-12 ? s : 1e-12);
  }
}

__global__ void fill_kernel(double* __restrict__ p, int n, double v) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) p[q] = v;
}

// How an iteration is issued: directly, or captured into the batch graph
// (then with the conditional handle of the inner loop).
struct IterLaunch {
  const void* fac[ALTO_MAX_MODES];
  alto_mttkrp_variant mv;
  int in_graph;
  cudaGraphConditionalHandle outer;
  cudaGraphConditionalHandle admm[ALTO_MAX_MODES];  // chunk loop of each constrained mode
  cudaStream_t body_stream;                         // captures the chunk loop bodies
};

// In a stream being captured: append a while node on handle h after the
// work captured so far, make later captured work depend on it, and return
// its (empty) body graph.
alto_status capture_while(cudaStream_t cs, cudaGraphConditionalHandle h, cudaGraph_t* body) {
  cudaStreamCaptureStatus cst;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  ALTO_TRY_CUDA(cudaStreamGetCaptureInfo(cs, &cst, nullptr, &g, &deps, &nd));
  if (cst != cudaStreamCaptureStatusActive) {
    set_error("stream is not capturing");
    return ALTO_ERR_CUDA;
  }
  cudaGraphNodeParams p = {};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  ALTO_TRY_CUDA(cudaGraphAddNode(&node, g, deps, nd, &p));
  ALTO_TRY_CUDA(cudaStreamUpdateCaptureDependencies(cs, &node, 1, cudaStreamSetCaptureDependencies));
  *body = p.conditional.phGraph_out[0];
  return ALTO_OK;
}

template <int SLOTS, int SEG>
alto_status admm_run(alto_stream_session* s, uint64_t I, int mode, cudaStream_t st, const IterLaunch& L) {
  double* primal = s->prim.as<double>();
  double* dual = s->dual[mode].as<double>();
  const float* P32 = s->P[mode].as<float>();
  const float* B32 = s->buf32.as<float>();
  const double* A = s->ata.as<double>();
  float* U32 = s->U[mode].as<float>();
  const int R = s->R;
  const size_t smem = (size_t)R * R * sizeof(double);
  constexpr uint64_t rows_per_block = (kAdmmThreads / 32) * RowMap<SEG>::kRows * AdmmBatch<SLOTS>::M;
  uint64_t blocks = std::min<uint64_t>((I + rows_per_block - 1) / rows_per_block, 148ull * 4);
  if (blocks < 1) blocks = 1;
  ALTO_TRY(s->admm_part.ensure(blocks * kAdmmSums * sizeof(double)));
  static size_t raised = 0;  // raised once per kernel, outside any capture
  if (smem > 40 * 1024 && smem > raised) {
    ALTO_TRY_CUDA(cudaFuncSetAttribute(admm_rows_kernel<SLOTS, SEG, true>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    ALTO_TRY_CUDA(cudaFuncSetAttribute(admm_rows_kernel<SLOTS, SEG, false>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    raised = smem;
  }
  AdmmState* state = s->admm_state.as<AdmmState>();
  double* part = s->admm_part.as<double>();
  double* aux = s->aux.as<double>();
  const double tol = (double)1e-6f;
  const cudaGraphConditionalHandle h = L.in_graph ? L.admm[mode] : cudaGraphConditionalHandle{};
  // (the state was cleared and the loop opened by mode_prep_kernel)
  auto chunk = [&](cudaStream_t cs) -> alto_status {
    admm_rows_kernel<SLOTS, SEG, true><<<(unsigned)blocks, kAdmmThreads, smem, cs>>>(
        P32, B32, A, U32, primal, aux, dual, s->W.as<double>(), s->rho.as<double>(), I, R, part, state, tol, h,
        L.in_graph);
    ALTO_LAUNCHED();
    admm_rows_kernel<SLOTS, SEG, false><<<(unsigned)blocks, kAdmmThreads, smem, cs>>>(
        P32, B32, A, U32, primal, aux, dual, s->W.as<double>(), s->rho.as<double>(), I, R, part, state, tol, h,
        L.in_graph);
    ALTO_LAUNCHED();
    return ALTO_OK;
  };
  if (!L.in_graph) {
    // every chunk issued; those after the stop return at once
    for (int c = 0; c < (kAdmmMaxIters + kAdmmChunk - 1) / kAdmmChunk; ++c) ALTO_TRY(chunk(st));
    return ALTO_OK;
  }
  // while (not stopped): one chunk
  cudaGraph_t body;
  ALTO_TRY(capture_while(st, h, &body));
  ALTO_TRY_CUDA(cudaStreamBeginCaptureToGraph(L.body_stream, body, nullptr, nullptr, 0,
                                              cudaStreamCaptureModeThreadLocal));
  const alto_status cst = chunk(L.body_stream);
  cudaGraph_t done = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(L.body_stream, &done);
  ALTO_TRY(cst);
  ALTO_TRY_CUDA(ee);
  return ALTO_OK;
}

// The tiled ADMM passes (ranks 8, 16, 32, 64): launched as admm_run.
template <int R>
alto_status admm_tile_run(alto_stream_session* s, uint64_t I, int mode, cudaStream_t st, const IterLaunch& L) {
  const size_t smem = TileMap<R>::smem_bytes();
  const uint64_t blocks = tile_blocks<R>(I, 148ull * 4);
  ALTO_TRY(s->admm_part.ensure(blocks * kAdmmSums * sizeof(double)));
  static bool raised = false;  // raised once per kernel, outside any capture
  if (smem > 48 * 1024 && !raised) {
    ALTO_TRY_CUDA(cudaFuncSetAttribute(admm_tile_kernel<R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    ALTO_TRY_CUDA(cudaFuncSetAttribute(admm_tile_kernel<R, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    raised = true;
  }
  double* primal = s->prim.as<double>();
  double* dual = s->dual[mode].as<double>();
  const float* P32 = s->P[mode].as<float>();
  const float* B32 = s->buf32.as<float>();
  const double* A = s->ata.as<double>();
  float* U32 = s->U[mode].as<float>();
  AdmmState* state = s->admm_state.as<AdmmState>();
  double* part = s->admm_part.as<double>();
  double* aux = s->aux.as<double>();
  const double tol = (double)1e-6f;
  const cudaGraphConditionalHandle h = L.in_graph ? L.admm[mode] : cudaGraphConditionalHandle{};
  auto chunk = [&](cudaStream_t cs) -> alto_status {
    admm_tile_kernel<R, true><<<(unsigned)blocks, kAdmmThreads, smem, cs>>>(
        P32, B32, A, U32, primal, aux, dual, s->W.as<double>(), s->rho.as<double>(), I, part, state, tol, h,
        L.in_graph);
    ALTO_LAUNCHED();
    admm_tile_kernel<R, false><<<(unsigned)blocks, kAdmmThreads, smem, cs>>>(
        P32, B32, A, U32, primal, aux, dual, s->W.as<double>(), s->rho.as<double>(), I, part, state, tol, h,
        L.in_graph);
    ALTO_LAUNCHED();
    return ALTO_OK;
  };
  if (!L.in_graph) {
    for (int c = 0; c < (kAdmmMaxIters + kAdmmChunk - 1) / kAdmmChunk; ++c) ALTO_TRY(chunk(st));
    return ALTO_OK;
  }
  cudaGraph_t body;
  ALTO_TRY(capture_while(st, h, &body));
  ALTO_TRY_CUDA(cudaStreamBeginCaptureToGraph(L.body_stream, body, nullptr, nullptr, 0,
                                              cudaStreamCaptureModeThreadLocal));
  const alto_status cst = chunk(L.body_stream);
  cudaGraph_t done = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(L.body_stream, &done);
  ALTO_TRY(cst);
  ALTO_TRY_CUDA(ee);
  return ALTO_OK;
}

alto_status admm(alto_stream_session* s, uint64_t I, int mode, cudaStream_t st, const IterLaunch& L) {
  switch (s->R) {
    case 8: return admm_tile_run<8>(s, I, mode, st, L);
    case 16: return admm_tile_run<16>(s, I, mode, st, L);
    case 32: return admm_tile_run<32>(s, I, mode, st, L);
    case 64: return admm_tile_run<64>(s, I, mode, st, L);
    default: break;
  }
  if (s->R <= 8) return admm_run<1, 8>(s, I, mode, st, L);
  if (s->R <= 16) return admm_run<1, 16>(s, I, mode, st, L);
  if (s->R <= 32) return admm_run<1, 32>(s, I, mode, st, L);
  if (s->R <= 64) return admm_run<2, 32>(s, I, mode, st, L);
  return admm_run<4, 32>(s, I, mode, st, L);
}

template <int SLOTS, int SEG>
alto_status solve_run(const float* P32, const float* B32, const double* A, const double* W, uint64_t I, int R,
                      float* U32, cudaStream_t st) {
  const size_t smem = (size_t)R * R * sizeof(double);
  static size_t raised = 0;  // raised once per kernel, outside any capture
  if (smem > 40 * 1024 && smem > raised) {
    ALTO_TRY_CUDA(cudaFuncSetAttribute(stream_solve_kernel<SLOTS, SEG>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    raised = smem;
  }
  const uint64_t warps = (I + RowMap<SEG>::kRows - 1) / RowMap<SEG>::kRows;
  uint64_t blocks = std::min<uint64_t>((warps * 32 + kAdmmThreads - 1) / kAdmmThreads, 148ull * 8);
  if (blocks < 1) blocks = 1;
  stream_solve_kernel<SLOTS, SEG><<<(unsigned)blocks, kAdmmThreads, smem, st>>>(P32, B32, A, W, I, R, U32);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

// U32 = (P32 A + B32) W row by row (float64 arithmetic, float32 in and out).
template <int R>
alto_status solve_tile_run(const float* P32, const float* B32, const double* A, const double* W, uint64_t I,
                           float* U32, cudaStream_t st) {
  const size_t smem = TileMap<R>::smem_bytes();
  static bool raised = false;  // raised once per kernel, outside any capture
  if (smem > 48 * 1024 && !raised) {
    ALTO_TRY_CUDA(cudaFuncSetAttribute(solve_tile_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    raised = true;
  }
  solve_tile_kernel<R><<<(unsigned)tile_blocks<R>(I, 148ull * 8), kAdmmThreads, smem, st>>>(P32, B32, A, W, I, U32);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

alto_status rows_solve(const float* P32, const float* B32, const double* A, const double* W, uint64_t I, int R,
                       float* U32, cudaStream_t st) {
  switch (R) {
    case 8: return solve_tile_run<8>(P32, B32, A, W, I, U32, st);
    case 16: return solve_tile_run<16>(P32, B32, A, W, I, U32, st);
    case 32: return solve_tile_run<32>(P32, B32, A, W, I, U32, st);
    case 64: return solve_tile_run<64>(P32, B32, A, W, I, U32, st);
    default: break;
  }
  if (R <= 8) return solve_run<1, 8>(P32, B32, A, W, I, R, U32, st);
  if (R <= 16) return solve_run<1, 16>(P32, B32, A, W, I, R, U32, st);
  if (R <= 32) return solve_run<1, 32>(P32, B32, A, W, I, R, U32, st);
  if (R <= 64) return solve_run<2, 32>(P32, B32, A, W, I, R, U32, st);
  return solve_run<4, 32>(P32, B32, A, W, I, R, U32, st);
}

alto_status stream_solve(alto_stream_session* s, uint64_t I, int mode, cudaStream_t st) {
  return rows_solve(s->P[mode].as<float>(), s->buf32.as<float>(), s->ata.as<double>(), s->W.as<double>(), I, s->R,
                    s->U[mode].as<float>(), st);
}

// One inner iteration of cpstream_alto_iter (src/streaming_cpd.cpp:1240-1482)
// on stream st, ending with the convergence kernel.
alto_status enqueue_iteration_sparse(alto_stream_session* s, const IterLaunch& L, cudaStream_t st);

alto_status enqueue_iteration(alto_stream_session* s, const IterLaunch& L, cudaStream_t st) {
  if (s->sparse) return enqueue_iteration_sparse(s, L, st);
  const int N = s->N, t = s->t, R = s->R;
  const size_t RR = (size_t)R * R;
  const unsigned all = (1u << N) - 1;
  double* G = s->G.as<double>();
  double* dstat = s->dstat.as<double>();  // [N][3]
  // time rows: MTTKRP of the stream mode, solve with the other Grams
  ALTO_TRY(run_mttkrp(s->at, t, L.fac, ALTO_F32, R, s->buf32.as<float>(), 0, L.mv, st));
  ALTO_TRY(solve_setup(G, N, all & ~(1u << t), R, kSolveRidge, 1e-12, s->W.as<double>(),
                       s->status.as<int>(), nullptr, st));
  double* Gt = G + (size_t)t * RR;
  time_update_kernel<<<1, 256, 0, st>>>(s->buf32.as<float>(), s->W.as<double>(), s->dims[t], R,
                                        s->time64.as<double>(), s->U[t].as<float>(), Gt, s->old_gram.as<double>());
  ALTO_LAUNCHED();

  for (int j = 0; j < N; ++j) {
    if (j == t) continue;
    const uint64_t I = s->dims[j];
    ALTO_TRY(run_mttkrp(s->at, j, L.fac, ALTO_F32, R, s->buf32.as<float>(), 0, L.mv, st));
    // historical term: A = G_t(old) * prod_{m != j, t} prev_U_m^T U_m (and,
    // for a constrained mode, the ADMM state cleared and its loop opened)
    const bool admm_mode = s->con != ALTO_UNCONSTRAINED;
    mode_prep_kernel<<<1, 256, 0, st>>>(s->old_gram.as<double>(), s->cross.as<double>(), all & ~(1u << j) & ~(1u << t),
                                        N, (int)RR, s->ata.as<double>(),
                                        admm_mode ? s->admm_state.as<AdmmState>() : nullptr,
                                        admm_mode && L.in_graph ? L.admm[j] : cudaGraphConditionalHandle{},
                                        admm_mode ? L.in_graph : 0);
    ALTO_LAUNCHED();
    if (s->con == ALTO_UNCONSTRAINED) {
      ALTO_TRY(solve_setup(G, N, all & ~(1u << j), R, kSolveRidge, 1e-12, s->W.as<double>(),
                           s->status.as<int>(), nullptr, st));
      ALTO_TRY(stream_solve(s, I, j, st));
    } else {
      ALTO_TRY(solve_setup(G, N, all & ~(1u << j), R, kSolveAdmm, 0.0, s->W.as<double>(), s->status.as<int>(),
                           s->rho.as<double>(), st));
      ALTO_TRY(admm(s, I, j, st, L));
    }
    // G_j, the cross Gram prev_U_j^T U_j and the change statistics, one pass
    ALTO_TRY(gram_cross_stats(s->P[j].as<float>(), s->U[j].as<float>(), I, R, G + (size_t)j * RR,
                              s->cross.as<double>() + (size_t)j * RR, dstat + 3 * j, s->gscr, st));
  }
  converge_kernel<<<1, 32, 0, st>>>(dstat, N, t, s->status.as<int>(), s->con != ALTO_UNCONSTRAINED ? 1 : 0, s->eps,
                                    s->max_inner, s->iter.as<IterState>(), L.outer, L.in_graph, 0);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

// spCP-stream, per batch before the inner loop (:607-709): row maps, the
// renumbered batch encoded, compact factors, c_z_prev.  The session's G
// holds c (G_t the temporal Gram) and its cross Grams hold h.
alto_status sparse_prepare(alto_stream_session* s, const alto_coo* b, bool first) {
  const int N = s->N, R = s->R;
  const size_t RR = (size_t)R * R;
  cudaStream_t st = s->st;
  const uint64_t nnz = b->nnz;
  ALTO_TRY(s->spg.ensure(kSpKinds * N * RR * 8));
  double* spg = s->spg.as<double>();
  auto SG = [&](int kind, int m) { return spg + ((size_t)kind * N + m) * RR; };
  if (first) ALTO_TRY_CUDA(cudaMemsetAsync(spg, 0, kSpKinds * N * RR * 8, st));
  // the batch on the device: uint64 indices, float64 values
  ALTO_TRY(s->coo_idx.ensure((size_t)N * nnz * 8));
  ALTO_TRY(s->coo_val.ensure(nnz * 8));
  uint64_t* ci = s->coo_idx.as<uint64_t>();
  std::vector<uint64_t> h64;
  const unsigned gw = (unsigned)std::min<uint64_t>((nnz + 255) / 256 + 1, 148ull * 8);
  for (int m = 0; m < N && b->on_device; ++m) {
    if (b->index_bytes == 8) {
      ALTO_TRY_CUDA(cudaMemcpyAsync(ci + (size_t)m * nnz, b->cidx[m], nnz * 8, cudaMemcpyDeviceToDevice, st));
    } else {
      widen_u32_kernel<<<gw, 256, 0, st>>>(static_cast<const uint32_t*>(b->cidx[m]), nnz, ci + (size_t)m * nnz);
      ALTO_LAUNCHED();
    }
  }
  if (b->on_device && b->val_dtype == ALTO_F64) {
    ALTO_TRY_CUDA(cudaMemcpyAsync(s->coo_val.p, b->vals, nnz * 8, cudaMemcpyDeviceToDevice, st));
  } else if (b->on_device) {
    widen_f32_kernel<<<gw, 256, 0, st>>>(static_cast<const float*>(b->vals), nnz, s->coo_val.as<double>());
    ALTO_LAUNCHED();
  }
  for (int m = 0; m < N && !b->on_device; ++m) {
    const void* src = b->cidx[m];
    if (b->index_bytes == 4) {
      h64.resize(nnz);
      for (uint64_t q = 0; q < nnz; ++q) h64[q] = static_cast<const uint32_t*>(b->cidx[m])[q];
      src = h64.data();
    }
    ALTO_TRY_CUDA(cudaMemcpyAsync(ci + (size_t)m * nnz, src, nnz * 8, cudaMemcpyHostToDevice, st));
    if (b->index_bytes == 4) ALTO_TRY_CUDA(cudaStreamSynchronize(st));  // h64 is reused
  }
  if (!b->on_device && b->val_dtype == ALTO_F64) {
    ALTO_TRY_CUDA(cudaMemcpyAsync(s->coo_val.p, b->vals, nnz * 8, cudaMemcpyHostToDevice, st));
  } else if (!b->on_device) {
    std::vector<double> v(nnz);
    for (uint64_t q = 0; q < nnz; ++q) v[q] = static_cast<const float*>(b->vals)[q];
    ALTO_TRY_CUDA(cudaMemcpyAsync(s->coo_val.p, v.data(), nnz * 8, cudaMemcpyHostToDevice, st));
    ALTO_TRY_CUDA(cudaStreamSynchronize(st));
  }
  // row maps: flags, exclusive scan (dims + 1 entries), touched-row count
  for (int m = 0; m < N; ++m) {
    const uint64_t d = s->dims[m];
    ALTO_TRY(s->ridx[m].ensure((d + 1) * 4));
    ALTO_TRY_CUDA(cudaMemsetAsync(s->ridx[m].p, 0, (d + 1) * 4, st));
    mark_rows_kernel<<<(unsigned)std::min<uint64_t>((nnz + 255) / 256, 148ull * 8), 256, 0, st>>>(
        ci + (size_t)m * nnz, nnz, s->ridx[m].as<uint32_t>());
    ALTO_LAUNCHED();
    ALTO_TRY(exclusive_scan_u32(s->ridx[m].as<uint32_t>(), d + 1, s->copy_tmp, st));
  }
  uint32_t cnt[ALTO_MAX_MODES];
  for (int m = 0; m < N; ++m)
    ALTO_TRY_CUDA(cudaMemcpyAsync(&cnt[m], s->ridx[m].as<uint32_t>() + s->dims[m], 4, cudaMemcpyDeviceToHost, st));
  ALTO_TRY_CUDA(cudaStreamSynchronize(st));
  uint64_t max_r = 1;
  for (int m = 0; m < N; ++m) {
    s->nnzr[m] = cnt[m];
    max_r = std::max<uint64_t>(max_r, cnt[m]);
    const uint64_t d = s->dims[m];
    ALTO_TRY(s->nzl[m].ensure(std::max<uint64_t>(cnt[m], 1) * 4));
    row_list_kernel<<<(unsigned)std::min<uint64_t>((d + 255) / 256, 148ull * 8), 256, 0, st>>>(
        s->ridx[m].as<uint32_t>(), d, s->nzl[m].as<uint32_t>());
    ALTO_LAUNCHED();
    renumber_kernel<<<(unsigned)std::min<uint64_t>((nnz + 255) / 256, 148ull * 8), 256, 0, st>>>(
        ci + (size_t)m * nnz, nnz, s->ridx[m].as<uint32_t>());
    ALTO_LAUNCHED();
    ALTO_TRY(s->Anz[m].ensure(std::max<uint64_t>(cnt[m], 1) * R * 4));
    ALTO_TRY(s->Aprev[m].ensure(std::max<uint64_t>(cnt[m], 1) * R * 4));
    const unsigned gg = (unsigned)std::min<uint64_t>((cnt[m] * R + 255) / 256 + 1, 148ull * 8);
    gather_rows_kernel<<<gg, 256, 0, st>>>(s->U[m].as<float>(), s->nzl[m].as<uint32_t>(), cnt[m], R,
                                           s->Anz[m].as<float>());
    ALTO_LAUNCHED();
    gather_rows_kernel<<<gg, 256, 0, st>>>(s->P[m].as<float>(), s->nzl[m].as<uint32_t>(), cnt[m], R,
                                           s->Aprev[m].as<float>());
    ALTO_LAUNCHED();
  }
  // the renumbered batch, encoded (update_salto_rowsparse)
  const void* ptrs[ALTO_MAX_MODES];
  for (int m = 0; m < N; ++m) ptrs[m] = ci + (size_t)m * nnz;
  alto_coo c;
  c.nmodes = N;
  c.dims = s->nnzr;
  c.nnz = nnz;
  c.cidx = ptrs;
  c.index_bytes = 8;
  c.vals = s->coo_val.p;
  c.val_dtype = ALTO_F64;
  c.on_device = 1;
  ALTO_TRY(encode_tensor(s->at, &c, 1, st));
  // c_z_prev = c_prev - c_nz_prev over the touched rows (:679-693)
  if (!first)
    for (int m = 0; m < N; ++m) {
      if (m == s->t) continue;
      ALTO_TRY(gram(s->Aprev[m].as<float>(), s->nnzr[m], R, SG(kSpCNzPrev, m), s->gscr, st));
      sub_kernel<<<(unsigned)((RR + 255) / 256), 256, 0, st>>>(SG(kSpCPrev, m), SG(kSpCNzPrev, m), (int)RR,
                                                               SG(kSpCZPrev, m));
      ALTO_LAUNCHED();
    }
  ALTO_TRY(s->buf32.ensure(max_r * R * 4));
  ALTO_TRY(s->time64.ensure(std::max<uint64_t>(s->nnzr[s->t], s->dims[s->t]) * R * 8));
  return ALTO_OK;
}

// One inner iteration of spcpstream_alto_iter (:716-975), ending with the
// convergence kernel.
alto_status enqueue_iteration_sparse(alto_stream_session* s, const IterLaunch& L, cudaStream_t st) {
  const int N = s->N, t = s->t, R = s->R;
  const size_t RR = (size_t)R * R;
  const unsigned all = (1u << N) - 1;
  double* G = s->G.as<double>();        // c (and G_t)
  double* H = s->cross.as<double>();    // h
  double* spg = s->spg.as<double>();
  auto SG = [&](int kind, int m) { return spg + ((size_t)kind * N + m) * RR; };
  double* dstat = s->dstat.as<double>();
  // s_t: MTTKRP of the stream mode over the compact factors, solve with
  // Hadamard(c) but t (+1e-12 I); the rows stay as they are if it fails
  ALTO_TRY(run_mttkrp(s->at, t, L.fac, ALTO_F32, R, s->buf32.as<float>(), 0, L.mv, st));
  ALTO_TRY(solve_setup(G, N, all & ~(1u << t), R, kSolveRidgeKeep, 1e-12, s->W.as<double>(), s->status.as<int>(),
                       nullptr, st));
  // s_t rows; h_t = G_t (old), then G_t += s s^T (= c_t)
  double* Gt = G + (size_t)t * RR;
  time_update_kernel<<<1, 256, 0, st>>>(s->buf32.as<float>(), s->W.as<double>(), s->nnzr[t], R,
                                        s->time64.as<double>(), s->Anz[t].as<float>(), Gt, H + (size_t)t * RR);
  ALTO_LAUNCHED();
  for (int m = 0; m < N; ++m) {
    if (m == t) continue;
    const uint64_t I = s->nnzr[m];
    // Q = Hadamard(h) but m; Phi = Hadamard(c) but m + 1e-12 I
    mode_prep_kernel<<<1, 256, 0, st>>>(nullptr, H, all & ~(1u << m), N, (int)RR, s->ata.as<double>(), nullptr,
                                        cudaGraphConditionalHandle{}, 0);
    ALTO_LAUNCHED();
    ALTO_TRY(solve_setup(G, N, all & ~(1u << m), R, kSolveRidgeKeep, 1e-12, s->W.as<double>(),
                         s->status.as<int>(), nullptr, st));
    // A_nz = (mttkrp + A_nz_prev Q) Phi^{-1}
    ALTO_TRY(run_mttkrp(s->at, m, L.fac, ALTO_F32, R, s->buf32.as<float>(), 0, L.mv, st));
    ALTO_TRY(rows_solve(s->Aprev[m].as<float>(), s->buf32.as<float>(), s->ata.as<double>(), s->W.as<double>(), I, R,
                        s->Anz[m].as<float>(), st));
    // c_nz = A_nz^T A_nz, h_nz = A_nz_prev^T A_nz; then c, h, delta
    ALTO_TRY(gram_cross_stats(s->Aprev[m].as<float>(), s->Anz[m].as<float>(), I, R, SG(kSpCNz, m), SG(kSpHNz, m),
                              nullptr, s->gscr, st));
    sp_gram_update_kernel<<<1, 256, 0, st>>>(s->ata.as<double>(), s->W.as<double>(), SG(kSpCZPrev, m),
                                             SG(kSpCNz, m), SG(kSpHNz, m), SG(kSpCPrev, m), R, SG(kSpQPi, m),
                                             SG(kSpHZ, m), SG(kSpCZ, m), G + (size_t)m * RR, H + (size_t)m * RR,
                                             dstat + 3 * m);
    ALTO_LAUNCHED();
  }
  converge_kernel<<<1, 32, 0, st>>>(dstat, N, t, s->status.as<int>(), 0, s->eps, s->max_inner,
                                    s->iter.as<IterState>(), L.outer, L.in_graph, 1);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

template <int SLOTS, int SEG>
alto_status sp_final_run(alto_stream_session* s, int m, cudaStream_t st) {
  const int R = s->R;
  const uint64_t I = s->dims[m];
  const size_t smem = (size_t)R * R * sizeof(double);
  static size_t raised = 0;  // raised once per kernel, outside any capture
  if (smem > 40 * 1024 && smem > raised) {
    ALTO_TRY_CUDA(cudaFuncSetAttribute(sp_final_rows_kernel<SLOTS, SEG>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    raised = smem;
  }
  const uint64_t warps = (I + RowMap<SEG>::kRows - 1) / RowMap<SEG>::kRows;
  uint64_t blocks = std::min<uint64_t>((warps * 32 + kAdmmThreads - 1) / kAdmmThreads, 148ull * 8);
  if (blocks < 1) blocks = 1;
  const double* QPi = s->spg.as<double>() + ((size_t)kSpQPi * s->N + m) * R * R;
  sp_final_rows_kernel<SLOTS, SEG><<<(unsigned)blocks, kAdmmThreads, smem, st>>>(
      s->P[m].as<float>(), s->Anz[m].as<float>(), s->ridx[m].as<uint32_t>(), QPi, I, R, s->U[m].as<float>());
  ALTO_LAUNCHED();
  return ALTO_OK;
}

// After the inner loop (:985-1047): the model's rows; c_prev <- c,
// c_nz_prev <- c_nz.
alto_status sparse_finish(alto_stream_session* s) {
  const int N = s->N, t = s->t, R = s->R;
  const size_t RR = (size_t)R * R;
  cudaStream_t st = s->st;
  double* spg = s->spg.as<double>();
  auto SG = [&](int kind, int m) { return spg + ((size_t)kind * N + m) * RR; };
  for (int m = 0; m < N; ++m) {
    if (m == t) {
      // the stream mode's rows are the batch's (a batch touches its time rows)
      ALTO_TRY_CUDA(cudaMemsetAsync(SG(kSpQPi, m), 0, RR * 8, st));
    }
    if (R <= 8)
      ALTO_TRY((sp_final_run<1, 8>(s, m, st)));
    else if (R <= 16)
      ALTO_TRY((sp_final_run<1, 16>(s, m, st)));
    else if (R <= 32)
      ALTO_TRY((sp_final_run<1, 32>(s, m, st)));
    else if (R <= 64)
      ALTO_TRY((sp_final_run<2, 32>(s, m, st)));
    else
      ALTO_TRY((sp_final_run<4, 32>(s, m, st)));
    if (m == t) continue;
    ALTO_TRY(rr_op(SG(kSpCPrev, m), s->G.as<double>() + (size_t)m * RR, (int)RR, 0, 0.0, st));
    ALTO_TRY(rr_op(SG(kSpCNzPrev, m), SG(kSpCNz, m), (int)RR, 0, 0.0, st));
  }
  return ALTO_OK;
}

// Inner iterations 1.. of the batch as one graph (see the file comment);
// launched on the session stream, resources released after the launch is
// queued (CUDA keeps an executable graph alive until its launches finish).
alto_status run_graph(alto_stream_session* s, IterLaunch L) {
  cudaStream_t cs = s->capst[0];
  cudaGraph_t g = nullptr;
  cudaGraphExec_t exec = nullptr;
  alto_status st = ALTO_OK;
  auto end_open_captures = [&]() {
    for (cudaStream_t c : s->capst) {
      cudaStreamCaptureStatus cst = cudaStreamCaptureStatusNone;
      if (cudaStreamIsCapturing(c, &cst) == cudaSuccess && cst != cudaStreamCaptureStatusNone) {
        cudaGraph_t junk = nullptr;
        cudaStreamEndCapture(c, &junk);
      }
    }
    cudaGetLastError();
  };
  do {
    if ((st = cuda_status(cudaGraphCreate(&g, 0), "cudaGraphCreate", __FILE__, __LINE__))) break;
    L.in_graph = 1;
    L.body_stream = s->capst[1];
    if ((st = cuda_status(cudaGraphConditionalHandleCreate(&L.outer, g, 0, 0), "conditional handle", __FILE__,
                          __LINE__)))
      break;
    if (s->con != ALTO_UNCONSTRAINED && !s->sparse)  // (spCP-stream has no ADMM loop)
      for (int j = 0; j < s->N && st == ALTO_OK; ++j)
        if (j != s->t)
          st = cuda_status(cudaGraphConditionalHandleCreate(&L.admm[j], g, 0, 0), "conditional handle", __FILE__,
                           __LINE__);
    if (st) break;
    if ((st = cuda_status(cudaStreamBeginCaptureToGraph(cs, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal),
                          "capture", __FILE__, __LINE__)))
      break;
    iter_begin_kernel<<<1, 32, 0, cs>>>(s->iter.as<IterState>(), s->max_inner, L.outer);
    if ((st = cuda_status(cudaGetLastError(), "iter_begin_kernel", __FILE__, __LINE__))) break;
    cudaGraph_t body = nullptr;
    if ((st = capture_while(cs, L.outer, &body))) break;
    cudaGraph_t tmp = nullptr;
    if ((st = cuda_status(cudaStreamEndCapture(cs, &tmp), "end capture", __FILE__, __LINE__))) break;
    if ((st = cuda_status(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal),
                          "capture", __FILE__, __LINE__)))
      break;
    if ((st = enqueue_iteration(s, L, cs))) break;
    if ((st = cuda_status(cudaStreamEndCapture(cs, &tmp), "end capture", __FILE__, __LINE__))) break;
    if ((st = cuda_status(cudaGraphInstantiate(&exec, g, 0), "cudaGraphInstantiate", __FILE__, __LINE__))) break;
    st = cuda_status(cudaGraphLaunch(exec, s->st), "cudaGraphLaunch", __FILE__, __LINE__);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  } while (false);
  if (st) end_open_captures();
  if (exec) cudaGraphExecDestroy(exec);
  if (g) cudaGraphDestroy(g);
  return st;
}

}  // namespace

// ------------------------------------------------ stream groups (host side)

namespace alto {

struct StreamGroup {
  int R = 0, N = 0, t = 0, cap = 0, count = 0;
  int hw[ALTO_MAX_MODES] = {0};
  cudaStream_t st = nullptr;
  cudaStream_t capst[2] = {nullptr, nullptr};
  DevBuf tab, offs, ctl, states;
  SlotDesc* h_tab = nullptr;  // pinned staging of the table and the offsets
  uint32_t* h_offs = nullptr;
  GroupCtl* h_ctl = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace grp {

constexpr uint32_t kSolveGrid = 148 * 8;
constexpr uint32_t kAdmmGrid = 148 * 4;

// (as admm() and rows_solve() launch the tiled kernels, ranks 8, 16, 32)
uint32_t admm_blocks(int R, uint64_t I) {
  return (uint32_t)(R == 8 ? tile_blocks<8>(I, kAdmmGrid) : (R == 16 ? tile_blocks<16>(I, kAdmmGrid)
                                                                     : tile_blocks<32>(I, kAdmmGrid)));
}
uint32_t solve_blocks(int R, uint64_t I) {
  return (uint32_t)(R == 8 ? tile_blocks<8>(I, kSolveGrid) : (R == 16 ? tile_blocks<16>(I, kSolveGrid)
                                                                      : tile_blocks<32>(I, kSolveGrid)));
}

uint32_t* off_of(uint32_t* base, int cap, int kind, int mode) {
  return base + ((size_t)kind * ALTO_MAX_MODES + mode) * (cap + 1);
}

template <typename T>
Strided<T> strided(const StreamGroup* g, size_t field_offset) {
  return Strided<T>{g->tab.as<char>() + field_offset, sizeof(SlotDesc), &g->ctl.as<GroupCtl>()->count};
}

template <int R>
alto_status capture_mode_solves(StreamGroup* g, cudaStream_t cs, int j, cudaGraphConditionalHandle h) {
  const size_t smem = TileMap<R>::smem_bytes();
  SlotDesc* tab = g->tab.as<SlotDesc>();
  GroupCtl* ctl = g->ctl.as<GroupCtl>();
  uint32_t* offs = g->offs.as<uint32_t>();
  group_solve_kernel<R><<<kSolveGrid, kAdmmThreads, smem, cs>>>(tab, ctl, off_of(offs, g->cap, kOffSolve, j), j);
  ALTO_LAUNCHED();
  // while some slot's ADMM of mode j sweeps: one chunk (pass 1, pass 2)
  group_admm_cond_kernel<<<1, 32, 0, cs>>>(tab, ctl, h, 1);
  ALTO_LAUNCHED();
  cudaGraph_t body;
  ALTO_TRY(capture_while(cs, h, &body));
  ALTO_TRY_CUDA(cudaStreamBeginCaptureToGraph(g->capst[1], body, nullptr, nullptr, 0,
                                              cudaStreamCaptureModeThreadLocal));
  const double tol = (double)1e-6f;
  const uint32_t* ao = off_of(offs, g->cap, kOffAdmm, j);
  group_admm_kernel<R, true><<<kAdmmGrid, kAdmmThreads, smem, g->capst[1]>>>(tab, ctl, ao, j, tol);
  group_admm_kernel<R, false><<<kAdmmGrid, kAdmmThreads, smem, g->capst[1]>>>(tab, ctl, ao, j, tol);
  group_admm_cond_kernel<<<1, 32, 0, g->capst[1]>>>(tab, ctl, h, 0);
  const cudaError_t le = cudaGetLastError();
  cudaGraph_t done = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(g->capst[1], &done);
  ALTO_TRY_CUDA(le);
  ALTO_TRY_CUDA(ee);
  return ALTO_OK;
}

alto_status capture_solves(StreamGroup* g, cudaStream_t cs, int j, cudaGraphConditionalHandle h) {
  if (g->R == 8) return capture_mode_solves<8>(g, cs, j, h);
  if (g->R == 16) return capture_mode_solves<16>(g, cs, j, h);
  return capture_mode_solves<32>(g, cs, j, h);
}

// One inner iteration of every acting slot (the body of the step loop).
alto_status capture_step(StreamGroup* g, cudaStream_t cs, cudaGraphConditionalHandle outer,
                         const cudaGraphConditionalHandle* admm_h) {
  const int N = g->N, t = g->t, R = g->R;
  SlotDesc* tab = g->tab.as<SlotDesc>();
  GroupCtl* ctl = g->ctl.as<GroupCtl>();
  uint32_t* offs = g->offs.as<uint32_t>();
  const unsigned per_slot = (unsigned)std::min(g->cap, 148);
  group_step_begin_kernel<<<1, 256, 0, cs>>>(tab, ctl);
  ALTO_LAUNCHED();
  // time rows: MTTKRP of the stream mode, solve with the other Grams
  ALTO_TRY(det_group_launch(strided<DetItem>(g, offsetof(SlotDesc, det) + t * sizeof(DetItem)),
                            off_of(offs, g->cap, kOffTile, t), R, g->hw[t], N, cs));
  ALTO_TRY(setup_group_launch(strided<SetupItem>(g, offsetof(SlotDesc, setup) + t * sizeof(SetupItem)), g->cap, R,
                              cs));
  group_time_update_kernel<<<per_slot, 256, 0, cs>>>(tab, ctl, t, R);
  ALTO_LAUNCHED();
  for (int j = 0; j < N; ++j) {
    if (j == t) continue;
    ALTO_TRY(det_group_launch(strided<DetItem>(g, offsetof(SlotDesc, det) + j * sizeof(DetItem)),
                              off_of(offs, g->cap, kOffTile, j), R, g->hw[j], N, cs));
    group_mode_prep_kernel<<<per_slot, 256, 0, cs>>>(tab, ctl, j, t, N, R);
    ALTO_LAUNCHED();
    ALTO_TRY(setup_group_launch(strided<SetupItem>(g, offsetof(SlotDesc, setup) + j * sizeof(SetupItem)), g->cap,
                                R, cs));
    ALTO_TRY(capture_solves(g, cs, j, admm_h[j]));
    ALTO_TRY(gram_group_launch(strided<GramItem>(g, offsetof(SlotDesc, gram) + j * sizeof(GramItem)),
                               off_of(offs, g->cap, kOffGram, j), off_of(offs, g->cap, kOffGramRed, j), g->cap, R,
                               cs));
  }
  group_converge_kernel<<<1, 32, 0, cs>>>(tab, ctl, g->states.as<SlotState>(), N, t, outer);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

// The group's graph: while (a slot runs and steps < limit) { one step }.
alto_status build_group_graph(StreamGroup* g) {
  cudaGraph_t graph = nullptr;
  alto_status st = ALTO_OK;
  cudaStream_t cs = g->capst[0];
  do {
    if ((st = cuda_status(cudaGraphCreate(&graph, 0), "cudaGraphCreate", __FILE__, __LINE__))) break;
    cudaGraphConditionalHandle outer, admm_h[ALTO_MAX_MODES] = {};
    if ((st = cuda_status(cudaGraphConditionalHandleCreate(&outer, graph, 0, 0), "conditional handle", __FILE__,
                          __LINE__)))
      break;
    for (int j = 0; j < g->N && st == ALTO_OK; ++j)
      if (j != g->t)
        st = cuda_status(cudaGraphConditionalHandleCreate(&admm_h[j], graph, 0, 0), "conditional handle", __FILE__,
                         __LINE__);
    if (st) break;
    if ((st = cuda_status(cudaStreamBeginCaptureToGraph(cs, graph, nullptr, nullptr, 0,
                                                        cudaStreamCaptureModeThreadLocal),
                          "capture", __FILE__, __LINE__)))
      break;
    group_begin_kernel<<<1, 32, 0, cs>>>(g->tab.as<SlotDesc>(), g->ctl.as<GroupCtl>(), outer);
    if ((st = cuda_status(cudaGetLastError(), "group_begin_kernel", __FILE__, __LINE__))) break;
    cudaGraph_t body = nullptr, tmp = nullptr;
    if ((st = capture_while(cs, outer, &body))) break;
    if ((st = cuda_status(cudaStreamEndCapture(cs, &tmp), "end capture", __FILE__, __LINE__))) break;
    if ((st = cuda_status(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0,
                                                        cudaStreamCaptureModeThreadLocal),
                          "capture", __FILE__, __LINE__)))
      break;
    if ((st = capture_step(g, cs, outer, admm_h))) break;
    if ((st = cuda_status(cudaStreamEndCapture(cs, &tmp), "end capture", __FILE__, __LINE__))) break;
    st = cuda_status(cudaGraphInstantiate(&g->exec, graph, 0), "cudaGraphInstantiate", __FILE__, __LINE__);
  } while (false);
  if (st) {
    for (cudaStream_t c : g->capst) {
      cudaStreamCaptureStatus cst = cudaStreamCaptureStatusNone;
      if (cudaStreamIsCapturing(c, &cst) == cudaSuccess && cst != cudaStreamCaptureStatusNone) {
        cudaGraph_t junk = nullptr;
        cudaStreamEndCapture(c, &junk);
      }
    }
    cudaGetLastError();
  }
  if (graph) cudaGraphDestroy(graph);
  return st;
}

}  // namespace grp

using namespace grp;

bool stream_groupable(const alto_stream_session* s) {
  return !s->sparse && (s->R == 8 || s->R == 16 || s->R == 32) && s->N >= 3 && s->N <= 5 && s->at;
}

alto_status group_prepare_session(alto_stream_session* s) {
  const int N = s->N, R = s->R;
  cudaStream_t st = s->st;
  const void* fac[ALTO_MAX_MODES] = {};
  for (int n = 0; n < N; ++n) fac[n] = s->U[n].p;
  uint64_t admm_part = 1, gram_part = 1;
  for (int m = 0; m < N; ++m) {
    ALTO_TRY(det_prepare(s->at, m, fac, R, s->buf32.as<float>(), &s->det[m], st));
    if (m == s->t) continue;
    admm_part = std::max<uint64_t>(admm_part, (uint64_t)admm_blocks(R, s->dims[m]) * kAdmmSums);
    uint32_t nb = 1;
    uint64_t rpb = 1;
    gram_split(s->dims[m], &nb, &rpb);
    gram_part = std::max<uint64_t>(gram_part, (uint64_t)nb * (2 * R * R + 3));
  }
  ALTO_TRY(s->admm_part.ensure(admm_part * sizeof(double)));
  ALTO_TRY(s->gscr.ensure(gram_part * sizeof(double)));
  ALTO_TRY(s->iter.ensure(sizeof(IterState)));
  ALTO_TRY_CUDA(cudaMemsetAsync(s->iter.p, 0, sizeof(IterState), st));
  return ALTO_OK;
}

bool group_fits(const StreamGroup* g, const alto_stream_session* s) {
  if (g->R != s->R || g->N != s->N || g->t != s->t) return false;
  for (int m = 0; m < s->N; ++m)
    if (g->hw[m] != s->det[m].hw) return false;
  return true;
}

alto_status group_create(const alto_stream_session* like, int capacity, cudaStream_t st, StreamGroup** out) {
  if (!stream_groupable(like) || capacity < 1) {
    set_error("the session cannot run in a group");
    return ALTO_ERR_UNSUPPORTED;
  }
  StreamGroup* g = new StreamGroup();
  g->R = like->R;
  g->N = like->N;
  g->t = like->t;
  g->cap = capacity;
  g->st = st;
  for (int m = 0; m < like->N; ++m) g->hw[m] = like->det[m].hw;
  const size_t offs_n = (size_t)kGroupOffKinds * ALTO_MAX_MODES * (capacity + 1);
  alto_status r = ALTO_OK;
  if ((r = g->tab.ensure(sizeof(SlotDesc) * capacity)) || (r = g->offs.ensure(offs_n * 4)) ||
      (r = g->ctl.ensure(sizeof(GroupCtl))) || (r = g->states.ensure(sizeof(SlotState) * capacity))) {
    group_destroy(g);
    return r;
  }
  if (cudaMallocHost((void**)&g->h_tab, sizeof(SlotDesc) * capacity) != cudaSuccess ||
      cudaMallocHost((void**)&g->h_offs, offs_n * 4) != cudaSuccess ||
      cudaMallocHost((void**)&g->h_ctl, sizeof(GroupCtl)) != cudaSuccess ||
      cudaStreamCreateWithFlags(&g->capst[0], cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&g->capst[1], cudaStreamNonBlocking) != cudaSuccess) {
    group_destroy(g);
    set_error("group set-up failed: %s", cudaGetErrorString(cudaGetLastError()));
    return ALTO_ERR_CUDA;
  }
  std::memset(g->h_tab, 0, sizeof(SlotDesc) * capacity);
  std::memset(g->h_offs, 0, offs_n * 4);
  *g->h_ctl = GroupCtl{0, 0, 0, 0, 0, 0};
  ALTO_TRY_CUDA(cudaMemsetAsync(g->tab.p, 0, sizeof(SlotDesc) * capacity, st));
  ALTO_TRY_CUDA(cudaMemsetAsync(g->offs.p, 0, offs_n * 4, st));
  ALTO_TRY_CUDA(cudaMemsetAsync(g->ctl.p, 0, sizeof(GroupCtl), st));
  if ((r = gram_group_ready(g->R)) || (r = build_group_graph(g))) {
    group_destroy(g);
    return r;
  }
  *out = g;
  return ALTO_OK;
}

void group_destroy(StreamGroup* g) {
  if (!g) return;
  if (g->st) cudaStreamSynchronize(g->st);
  if (g->exec) cudaGraphExecDestroy(g->exec);
  for (cudaStream_t c : g->capst)
    if (c) cudaStreamDestroy(c);
  if (g->h_tab) cudaFreeHost(g->h_tab);
  if (g->h_offs) cudaFreeHost(g->h_offs);
  if (g->h_ctl) cudaFreeHost(g->h_ctl);
  delete g;
}

// The members' descriptors and offsets, copied to the device on the group's
// stream (the staging must not be rewritten before the copy has run: the
// callers synchronise with the group's work between calls).
alto_status group_set(StreamGroup* g, alto_stream_session* const* members, int k) {
  if (k < 0 || k > g->cap) {
    set_error("group of %d slots given %d sessions", g->cap, k);
    return ALTO_ERR_INVALID;
  }
  const int N = g->N, R = g->R;
  const size_t RR = (size_t)R * R;
  SlotDesc* dtab = g->tab.as<SlotDesc>();
  const size_t offs_n = (size_t)kGroupOffKinds * ALTO_MAX_MODES * (g->cap + 1);
  std::memset(g->h_offs, 0, offs_n * 4);
  for (int q = 0; q < k; ++q) {
    alto_stream_session* s = members[q];
    if (!group_fits(g, s)) {
      set_error("session does not fit the group (rank, modes or record format)");
      return ALTO_ERR_INVALID;
    }
    SlotDesc& d = g->h_tab[q];
    std::memset(&d, 0, sizeof(d));
    const int* act = reinterpret_cast<const int*>(reinterpret_cast<const char*>(dtab + q) + offsetof(SlotDesc, act));
    double* G = s->G.as<double>();
    const unsigned all = (1u << N) - 1;
    for (int m = 0; m < N; ++m) {
      d.det[m] = s->det[m];
      d.det[m].active = act;
      d.dims[m] = s->dims[m];
      d.U[m] = s->U[m].as<float>();
      d.P[m] = s->P[m].as<float>();
      d.dual[m] = s->dual[m].as<double>();
      const bool admm_mode = m != s->t && s->con != ALTO_UNCONSTRAINED;
      d.setup[m] = SetupItem{G, all & ~(1u << m), N, admm_mode ? kSolveAdmm : kSolveRidge, admm_mode ? 0.0 : 1e-12,
                             s->W.as<double>(), s->status.as<int>(), admm_mode ? s->rho.as<double>() : nullptr, act};
      if (m == s->t) continue;
      uint32_t nb = 1;
      uint64_t rpb = 1;
      gram_split(s->dims[m], &nb, &rpb);
      d.gram[m] = GramItem{s->P[m].as<float>(), s->U[m].as<float>(), s->dims[m], rpb, nb, G + m * RR,
                           s->cross.as<double>() + m * RR, s->dstat.as<double>() + 3 * m, s->gscr.as<double>(), act};
      d.admm_blocks[m] = admm_blocks(R, s->dims[m]);
      d.solve_blocks[m] = solve_blocks(R, s->dims[m]);
    }
    d.G = G;
    d.old_gram = s->old_gram.as<double>();
    d.ata = s->ata.as<double>();
    d.cross = s->cross.as<double>();
    d.W = s->W.as<double>();
    d.rho = s->rho.as<double>();
    d.dstat = s->dstat.as<double>();
    d.aux = s->aux.as<double>();
    d.prim = s->prim.as<double>();
    d.time64 = s->time64.as<double>();
    d.admm_part = s->admm_part.as<double>();
    d.status = s->status.as<int>();
    d.buf32 = s->buf32.as<float>();
    d.admm = s->admm_state.as<AdmmState>();
    d.iter = s->iter.as<IterState>();
    d.eps = s->eps;
    d.con = s->con != ALTO_UNCONSTRAINED ? 1 : 0;
    d.max_inner = s->max_inner;
    for (int m = 0; m < N; ++m) {
      const uint32_t counts[kGroupOffKinds] = {d.det[m].a.ntiles, m == s->t ? 0u : d.gram[m].nb,
                                               m == s->t ? 0u : gram_reduce_blocks(R),
                                               m == s->t ? 0u : d.admm_blocks[m], m == s->t ? 0u : d.solve_blocks[m]};
      for (int kind = 0; kind < kGroupOffKinds; ++kind) {
        uint32_t* o = off_of(g->h_offs, g->cap, kind, m);
        o[q + 1] = o[q] + counts[kind];
      }
    }
  }
  g->count = k;
  ALTO_TRY_CUDA(cudaMemcpyAsync(g->tab.p, g->h_tab, sizeof(SlotDesc) * std::max(k, 1), cudaMemcpyHostToDevice, g->st));
  ALTO_TRY_CUDA(cudaMemcpyAsync(g->offs.p, g->h_offs, offs_n * 4, cudaMemcpyHostToDevice, g->st));
  return ALTO_OK;
}

// Run up to max_steps inner iterations of every member (stopping early
// when none can run), as one launch of the group's graph on its stream.
alto_status group_launch(StreamGroup* g, int max_steps) {
  *g->h_ctl = GroupCtl{g->count, max_steps, 0, 0, 0, 0};
  ALTO_TRY_CUDA(cudaMemcpyAsync(g->ctl.p, g->h_ctl, sizeof(GroupCtl), cudaMemcpyHostToDevice, g->st));
  ALTO_TRY_CUDA(cudaGraphLaunch(g->exec, g->st));
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  return ALTO_OK;
}

alto_status group_states(StreamGroup* g, int* running, int* done, int* stop, int* info) {
  std::vector<SlotState> h(std::max(g->count, 1));
  ALTO_TRY_CUDA(cudaMemcpyAsync(h.data(), g->states.p, sizeof(SlotState) * g->count, cudaMemcpyDeviceToHost, g->st));
  ALTO_TRY_CUDA(cudaMemcpyAsync(g->h_ctl, g->ctl.p, sizeof(GroupCtl), cudaMemcpyDeviceToHost, g->st));
  ALTO_TRY_CUDA(cudaStreamSynchronize(g->st));
  if (g->h_ctl->error) {
    set_error("a grouped ADMM loop overran %d chunks and was stopped", kAdmmChunkBound);
    return ALTO_ERR_CUDA;
  }
  for (int q = 0; q < g->count; ++q) {
    if (running) running[q] = h[q].running;
    if (done) done[q] = h[q].done;
    if (stop) stop[q] = h[q].stop;
    if (info) info[q] = h[q].info;
  }
  return ALTO_OK;
}

}  // namespace alto

namespace {

// Everything of a batch before its inner iterations (src/streaming_cpd.cpp:
// 124-186): grow the model, Grams and cross Grams, duals cleared, the
// batch encoded, the first batch's normalisation, spCP-stream's row maps.
static double host_seconds();

alto_status prepare_batch(alto_stream_session* s, const alto_coo* b, const double* init_vals, uint64_t n_init) {
  const int N = s->N, t = s->t, R = s->R;
  cudaStream_t st = s->st;
  const size_t RR = (size_t)R * R;
  const bool first = s->batches == 0;
  const double t_grow0 = host_seconds();

  // grow the model: new rows of U from init_vals (mode order), prev rows
  // zero; every mode's new rows staged in the session's pinned buffer
  uint64_t old[ALTO_MAX_MODES];
  uint64_t new_vals = 0;
  for (int n = 0; n < N; ++n) new_vals += (std::max<uint64_t>(b->dims[n], s->dims[n]) - s->dims[n]) * R;
  if (new_vals > s->pin_cap) {
    const size_t want = std::max<size_t>(new_vals, s->pin_cap + s->pin_cap / 2);
    if (s->pin_rows) cudaFreeHost(s->pin_rows);
    s->pin_rows = nullptr;
    s->pin_cap = 0;
    ALTO_TRY_CUDA(cudaMallocHost((void**)&s->pin_rows, want * sizeof(float)));
    s->pin_cap = want;
  }
  uint64_t consumed = 0;
  for (int n = 0; n < N; ++n) {
    old[n] = s->dims[n];
    const uint64_t nd = std::max<uint64_t>(b->dims[n], old[n]);
    if (nd > s->cap[n]) {
      const uint64_t nc = std::max<uint64_t>(nd, s->cap[n] + s->cap[n] / 2);
      ALTO_TRY(grow_rows(s->U[n], old[n], nc, R * 4, st));
      ALTO_TRY(grow_rows(s->P[n], old[n], nc, R * 4, st));
      s->dual[n].release();
      ALTO_TRY(s->dual[n].ensure(nc * R * 8));
      s->cap[n] = nc;
    }
    if (nd > old[n]) {
      const uint64_t cnt = (nd - old[n]) * R;
      float* rows = s->pin_rows + consumed;
      for (uint64_t q = 0; q < cnt; ++q)
        rows[q] = consumed + q < n_init ? (float)init_vals[consumed + q] : 0.0f;
      consumed += cnt;
      ALTO_TRY_CUDA(cudaMemcpyAsync(s->U[n].as<float>() + old[n] * R, rows, cnt * 4, cudaMemcpyHostToDevice, st));
      ALTO_TRY_CUDA(cudaMemsetAsync(s->P[n].as<float>() + old[n] * R, 0, cnt * 4, st));
    }
    s->dims[n] = nd;
  }
  uint64_t max_dim = 0;
  for (int n = 0; n < N; ++n) max_dim = std::max(max_dim, s->dims[n]);
  ALTO_TRY(ensure_headroom(s->buf32, max_dim * R * 4));
  if (s->con != ALTO_UNCONSTRAINED) {  // the ADMM primal and aux between chunks
    ALTO_TRY(ensure_headroom(s->aux, max_dim * R * 8));
    ALTO_TRY(ensure_headroom(s->prim, max_dim * R * 8));
  }
  ALTO_TRY(ensure_headroom(s->time64, s->dims[t] * R * 8));
  s->t_grow += host_seconds() - t_grow0;
  double* G = s->G.as<double>();
  if (first) {
    ALTO_TRY(rr_op(s->lam.as<double>(), nullptr, R, 3, 0.0, st));
    fill_kernel<<<1, 128, 0, st>>>(s->lam.as<double>(), R, 1.0);
    ALTO_LAUNCHED();
    ALTO_TRY_CUDA(cudaMemsetAsync(s->U[t].p, 0, s->dims[t] * R * 4, st));
    ALTO_TRY_CUDA(cudaMemsetAsync(G + (size_t)t * RR, 0, RR * 8, st));
  }
  // Grams and cross Grams (prev_U^T U) of the non-stream modes
  double* C = s->cross.as<double>();
  for (int n = 0; n < N; ++n)
    if (n != t)
      ALTO_TRY(gram_cross_stats(s->P[n].as<float>(), s->U[n].as<float>(), s->dims[n], R, G + (size_t)n * RR,
                                C + (size_t)n * RR, nullptr, s->gscr, st));
  if (!s->sparse)
    for (int n = 0; n < N; ++n) ALTO_TRY_CUDA(cudaMemsetAsync(s->dual[n].p, 0, s->dims[n] * R * 8, st));
  if (!s->at) {
    s->at = new alto_tensor();
    s->at->tile_stats = false;
    s->at->grow = true;
    s->at->key_bits = 128;
    s->at->stream_mode = t;
    s->at->stream = st;
  }
  if (!s->sparse) {  // update_salto
    alto_coo c = *b;
    uint64_t bd[ALTO_MAX_MODES];
    for (int n = 0; n < N; ++n) bd[n] = s->dims[n];
    c.dims = bd;
    const double t_enc0 = host_seconds();
    ALTO_TRY(encode_tensor(s->at, &c, 1, st));
    s->t_encode += host_seconds() - t_enc0;
  }

  // first batch: 2-norm normalise the non-stream factors, lambda = 1
  if (first) {
    for (int m = 0; m < N; ++m) {
      if (m == t) continue;
      double* Gm = G + (size_t)m * RR;
      lambda_from_gram_kernel<<<1, 128, 0, st>>>(Gm, R, s->lam.as<double>());
      ALTO_LAUNCHED();
      ALTO_TRY(scale_columns(s->U[m].as<float>(), s->dims[m], R, s->lam.as<double>(), nullptr, st));
      ALTO_TRY(gram_cross_stats(s->P[m].as<float>(), s->U[m].as<float>(), s->dims[m], R, Gm, C + (size_t)m * RR,
                                nullptr, s->gscr, st));
    }
    fill_kernel<<<1, 128, 0, st>>>(s->lam.as<double>(), R, 1.0);
    ALTO_LAUNCHED();
  }

  if (s->sparse) ALTO_TRY(sparse_prepare(s, b, first));
  return ALTO_OK;
}

// After the inner iterations (hs: their state): the failed-solve check,
// forgetting, prev <- current, the time rows out.
alto_status finish_batch(alto_stream_session* s, const IterState& hs, int* inner_out) {
  const int N = s->N, t = s->t, R = s->R;
  cudaStream_t st = s->st;
  const size_t RR = (size_t)R * R;
  double* G = s->G.as<double>();
  if (hs.info) {
    set_error("Cholesky of the ADMM normal equations failed (info %d)", hs.info);
    return ALTO_ERR_NOT_SPD;
  }
  if (inner_out) *inner_out = hs.done;
  if (s->sparse) ALTO_TRY(sparse_finish(s));
  // forgetting, prev <- current, time rows out
  ALTO_TRY(rr_op(G + (size_t)t * RR, nullptr, (int)RR, 2, s->forgetting, st));
  for (int n = 0; n < N; ++n)
    ALTO_TRY_CUDA(cudaMemcpyAsync(s->P[n].p, s->U[n].p, s->dims[n] * R * 4, cudaMemcpyDeviceToDevice, st));
  const size_t base = s->time_rows.size();
  s->time_rows.resize(base + s->dims[t] * R);
  ALTO_TRY_CUDA(cudaMemcpyAsync(s->time_rows.data() + base, s->time64.p, s->dims[t] * R * 8,
                                cudaMemcpyDeviceToHost, st));
  int ew[4] = {0, 0, 0, 0};  // the slice encoder's error words
  if (s->at && s->at->err.p)
    ALTO_TRY_CUDA(cudaMemcpyAsync(ew, s->at->err.p, sizeof(ew), cudaMemcpyDeviceToHost, st));
  ALTO_TRY_CUDA(cudaStreamSynchronize(st));
  if (s->at) ALTO_TRY(sort_error_status(s->at, ew, st));
  s->batches += 1;
  return ALTO_OK;
}

static double host_seconds() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// The push's inner iterations are done: their device time (the events) and
// the finish, into the session's timing.
static alto_status timed_finish(alto_stream_session* s, const IterState& hs, int* inner_out, double t_launch) {
  const double t_ran = host_seconds();
  s->t_inner += t_ran - t_launch;
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, s->inner_ev[0], s->inner_ev[1]) == cudaSuccess) s->dev_inner_ms += ms;
  int inner = 0;
  ALTO_TRY(finish_batch(s, hs, &inner));
  if (inner_out) *inner_out = inner;
  s->t_finish += host_seconds() - t_ran;
  s->pushes += 1;
  s->inner_total += (uint64_t)inner;
  return ALTO_OK;
}

alto_status push_batch(alto_stream_session* s, const alto_coo* b, const double* init_vals,
                       uint64_t n_init, int* inner_out) {
  const int N = s->N, R = s->R;
  cudaStream_t st = s->st;
  const double t0 = host_seconds();
  for (cudaEvent_t& e : s->inner_ev)
    if (!e) ALTO_TRY_CUDA(cudaEventCreate(&e));
  ALTO_TRY(prepare_batch(s, b, init_vals, n_init));
  IterState hs{};
  if (s->use_graph && stream_groupable(s)) {
    // the inner iterations as one launch of the session's own group graph,
    // captured once and relaunched for every batch
    const double t_sort0 = host_seconds();
    ALTO_TRY(group_prepare_session(s));
    s->t_sorted += host_seconds() - t_sort0;
    if (s->own_group && !group_fits(s->own_group, s)) {
      group_destroy(s->own_group);
      s->own_group = nullptr;
    }
    if (!s->own_group) ALTO_TRY(group_create(s, 1, st, &s->own_group));
    alto_stream_session* one = s;
    ALTO_TRY(group_set(s->own_group, &one, 1));
    const double t_launch = host_seconds();
    s->t_prepare += t_launch - t0;
    ALTO_TRY_CUDA(cudaEventRecord(s->inner_ev[0], st));
    ALTO_TRY(group_launch(s->own_group, s->max_inner));
    ALTO_TRY_CUDA(cudaEventRecord(s->inner_ev[1], st));
    ALTO_TRY(group_states(s->own_group, nullptr, nullptr, nullptr, nullptr));
    ALTO_TRY_CUDA(cudaMemcpyAsync(&hs, s->iter.p, sizeof(IterState), cudaMemcpyDeviceToHost, st));
    ALTO_TRY_CUDA(cudaStreamSynchronize(st));
    return timed_finish(s, hs, inner_out, t_launch);
  }
  IterLaunch L{};
  for (int n = 0; n < N; ++n) L.fac[n] = s->sparse ? s->Anz[n].p : s->U[n].p;
  // the deterministic MTTKRP where it runs, so a stream's results repeat
  // bit for bit however many other streams share the device
  L.mv = deterministic_supported(R, ALTO_F32) ? ALTO_MTTKRP_DETERMINISTIC : ALTO_MTTKRP_AUTO;
  ALTO_TRY(s->iter.ensure(sizeof(IterState)));
  ALTO_TRY_CUDA(cudaMemsetAsync(s->iter.p, 0, sizeof(IterState), st));
  const double t_launch = host_seconds();
  s->t_prepare += t_launch - t0;
  ALTO_TRY_CUDA(cudaEventRecord(s->inner_ev[0], st));
  // iteration 0 directly: sizes every buffer and builds the sorted lines
  ALTO_TRY(enqueue_iteration(s, L, st));
  if (s->use_graph && s->max_inner > 1) {
    ALTO_TRY(run_graph(s, L));
    ALTO_TRY_CUDA(cudaEventRecord(s->inner_ev[1], st));
    ALTO_TRY_CUDA(cudaMemcpyAsync(&hs, s->iter.p, sizeof(IterState), cudaMemcpyDeviceToHost, st));
    ALTO_TRY_CUDA(cudaStreamSynchronize(st));
  } else {
    while (true) {
      ALTO_TRY_CUDA(cudaEventRecord(s->inner_ev[1], st));
      ALTO_TRY_CUDA(cudaMemcpyAsync(&hs, s->iter.p, sizeof(IterState), cudaMemcpyDeviceToHost, st));
      ALTO_TRY_CUDA(cudaStreamSynchronize(st));
      if (hs.stop || hs.done >= s->max_inner) break;
      ALTO_TRY(enqueue_iteration(s, L, st));
    }
  }
  return timed_finish(s, hs, inner_out, t_launch);
}

// ------------------------------------------------- model error (cpd_error)

struct ErrArgs {
  const void* cidx[ALTO_MAX_MODES];
  const float* U[ALTO_MAX_MODES];
  uint64_t rows[ALTO_MAX_MODES];  // model rows (the time mode: X's time steps)
  uint64_t xdims[ALTO_MAX_MODES];
};

constexpr int kErrThreads = 256;

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

// Per block: sum_k v_k * sum_r prod_m F_m[i_m(k), r] and sum_k v_k^2, in a
// fixed order (cpd_error's inner product, as a per-nonzero model value
// instead of an MTTKRP of one mode; the two sums are equal).  Model rows
// past the session's dims are zero; an index outside X's dims sets *bad.
template <int IB, typename VT>
__global__ void __launch_bounds__(kErrThreads)
    model_inner_kernel(ErrArgs a, int N, int t, int R, const double* __restrict__ trow, const VT* __restrict__ vals,
                       uint64_t nnz, double* __restrict__ partial, int* __restrict__ bad) {
  double inner = 0, xx = 0;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < nnz; k += (uint64_t)gridDim.x * blockDim.x) {
    const double v = (double)vals[k];
    xx += v * v;
    uint64_t ix[ALTO_MAX_MODES];
    bool zero = false;
    for (int m = 0; m < N; ++m) {
      ix[m] = IB == 8 ? ((const uint64_t*)a.cidx[m])[k] : ((const uint32_t*)a.cidx[m])[k];
      if (ix[m] >= a.xdims[m]) {
        atomicOr(bad, 1);
        zero = true;
      } else if (ix[m] >= a.rows[m]) {
        zero = true;
      }
    }
    if (zero) continue;
    double sum = 0;
    for (int r = 0; r < R; ++r) {
      double p = trow[ix[t] * R + r];
      for (int m = 0; m < N; ++m)
        if (m != t) p *= (double)a.U[m][ix[m] * R + r];
      sum += p;
    }
    inner += v * sum;
  }
  __shared__ double sh[2][kErrThreads / 32];
  for (int o = 16; o; o >>= 1) {
    inner += __shfl_xor_sync(0xffffffffu, inner, o);
    xx += __shfl_xor_sync(0xffffffffu, xx, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sh[0][warp] = inner;
    sh[1][warp] = xx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a0 = 0, a1 = 0;
    for (int w = 0; w < kErrThreads / 32; ++w) {
      a0 += sh[0][w];
      a1 += sh[1][w];
    }
    partial[2 * blockIdx.x] = a0;
    partial[2 * blockIdx.x + 1] = a1;
  }
}

alto_status model_error(alto_stream_session* s, const alto_coo* X, double* err) {
  const int N = s->N, t = s->t, R = s->R;
  cudaStream_t st = s->st;
  const uint64_t nnz = X->nnz, T = X->dims[t];
  const uint64_t have = s->time_rows.size() / R;
  if (T > have) {
    set_error("the tensor has %llu time steps, the model %llu", (unsigned long long)T, (unsigned long long)have);
    return ALTO_ERR_INVALID;
  }
  // the last T time rows (get_prev_kruskal, src/kruskal_model.cpp:445-478)
  const double* trow_h = s->time_rows.data() + (have - T) * R;
  const int vb = X->val_dtype == ALTO_F64 ? 8 : 4;
  const unsigned nb = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((nnz + kErrThreads - 1) / kErrThreads,
                                                                         148ull * 8));
  size_t off = 0;
  const size_t o_t = off;
  off += align256(std::max<uint64_t>(T, 1) * R * 8);
  const size_t o_p = off;
  off += align256((size_t)nb * 16);
  const size_t o_b = off;
  off += 256;
  const size_t o_g = off;
  off += align256((size_t)N * R * R * 8);
  const size_t o_x = off;
  if (!X->on_device) off += align256(nnz * ((size_t)N * X->index_bytes + vb));
  DevBuf buf;
  ALTO_TRY(buf.ensure(off));
  char* b = buf.as<char>();
  ErrArgs a{};
  const void* vals = X->vals;
  for (int m = 0; m < N; ++m) {
    a.cidx[m] = X->cidx[m];
    a.U[m] = m == t ? nullptr : s->U[m].as<float>();
    a.rows[m] = m == t ? T : s->dims[m];
    a.xdims[m] = X->dims[m];
  }
  if (!X->on_device && nnz) {  // host tensor: copy it in
    for (int m = 0; m < N; ++m) {
      char* dst = b + o_x + (size_t)m * nnz * X->index_bytes;
      ALTO_TRY_CUDA(cudaMemcpyAsync(dst, X->cidx[m], nnz * X->index_bytes, cudaMemcpyHostToDevice, st));
      a.cidx[m] = dst;
    }
    char* vd = b + o_x + (size_t)N * nnz * X->index_bytes;
    ALTO_TRY_CUDA(cudaMemcpyAsync(vd, X->vals, nnz * vb, cudaMemcpyHostToDevice, st));
    vals = vd;
  }
  if (T) ALTO_TRY_CUDA(cudaMemcpyAsync(b + o_t, trow_h, T * R * 8, cudaMemcpyHostToDevice, st));
  ALTO_TRY_CUDA(cudaMemsetAsync(b + o_b, 0, 4, st));
  const double* trow = reinterpret_cast<const double*>(b + o_t);
  double* part = reinterpret_cast<double*>(b + o_p);
  int* bad = reinterpret_cast<int*>(b + o_b);
  if (X->index_bytes == 8 && X->val_dtype == ALTO_F64)
    model_inner_kernel<8, double><<<nb, kErrThreads, 0, st>>>(a, N, t, R, trow, (const double*)vals, nnz, part, bad);
  else if (X->index_bytes == 8)
    model_inner_kernel<8, float><<<nb, kErrThreads, 0, st>>>(a, N, t, R, trow, (const float*)vals, nnz, part, bad);
  else if (X->val_dtype == ALTO_F64)
    model_inner_kernel<4, double><<<nb, kErrThreads, 0, st>>>(a, N, t, R, trow, (const double*)vals, nnz, part, bad);
  else
    model_inner_kernel<4, float><<<nb, kErrThreads, 0, st>>>(a, N, t, R, trow, (const float*)vals, nnz, part, bad);
  ALTO_LAUNCHED();
  // Grams of the non-stream factors (kruskal_norm, src/kruskal_model.cpp:400-443)
  double* G = reinterpret_cast<double*>(b + o_g);
  for (int m = 0; m < N; ++m)
    if (m != t) ALTO_TRY(gram(s->U[m].as<float>(), s->dims[m], R, G + (size_t)m * R * R, s->gscr, st));
  std::vector<double> hp(2 * (size_t)nb), hg((size_t)N * R * R);
  int hbad = 0;
  ALTO_TRY_CUDA(cudaMemcpyAsync(hp.data(), part, hp.size() * 8, cudaMemcpyDeviceToHost, st));
  ALTO_TRY_CUDA(cudaMemcpyAsync(hg.data(), G, hg.size() * 8, cudaMemcpyDeviceToHost, st));
  ALTO_TRY_CUDA(cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, st));
  ALTO_TRY_CUDA(cudaStreamSynchronize(st));
  if (hbad) {
    set_error("an index of the tensor is outside its dims");
    return ALTO_ERR_INVALID;
  }
  double inner = 0, xx = 0;
  for (unsigned k = 0; k < nb; ++k) {
    inner += hp[2 * (size_t)k];
    xx += hp[2 * (size_t)k + 1];
  }
  // the time factor's Gram on the host (T x R, small)
  double* Gt = hg.data() + (size_t)t * R * R;
  for (int i = 0; i < R * R; ++i) Gt[i] = 0;
  for (uint64_t q = 0; q < T; ++q)
    for (int i = 0; i < R; ++i)
      for (int j = 0; j < R; ++j) Gt[i * R + j] += trow_h[q * R + i] * trow_h[q * R + j];
  // weights^T (Hadamard of the Grams) weights with unit weights: cpd_error
  // sets lambda to 1 before kruskal_norm (src/streaming_cpd.cpp:432)
  double z = 0;
  for (int i = 0; i < R; ++i)
    for (int j = 0; j < R; ++j) {
      double p = 1;
      for (int m = 0; m < N; ++m) p *= hg[(size_t)m * R * R + (size_t)i * R + j];
      z += p;
    }
  z = std::fabs(z);
  *err = std::sqrt(xx + z - 2 * inner) / std::sqrt(xx);
  return ALTO_OK;
}

}  // namespace

namespace alto {
// Point a session (and its encoded slice) at another CUDA stream; the
// session's previous work must be complete (every push is synchronous).
void stream_set_cuda_stream(alto_stream_session* s, cudaStream_t st) {
  s->st = st;
  if (s->at) s->at->stream = st;
}

alto_status stream_prepare_grouped(alto_stream_session* s, const alto_coo* b, const double* init_vals,
                                   uint64_t n_init, bool* grouped) {
  *grouped = false;
  if (b->nmodes != s->N || b->nnz == 0 || (n_init && !init_vals)) {
    set_error("bad batch (modes %d against %d, nnz %llu)", b->nmodes, s->N, (unsigned long long)b->nnz);
    return ALTO_ERR_INVALID;
  }
  ALTO_TRY(prepare_batch(s, b, init_vals, n_init));
  if (!s->use_graph || !stream_groupable(s)) return ALTO_OK;
  ALTO_TRY(group_prepare_session(s));
  *grouped = true;
  return ALTO_OK;
}

alto_status stream_run_ungrouped(alto_stream_session* s, int* inner) {
  const int N = s->N, R = s->R;
  cudaStream_t st = s->st;
  IterLaunch L{};
  for (int n = 0; n < N; ++n) L.fac[n] = s->sparse ? s->Anz[n].p : s->U[n].p;
  L.mv = deterministic_supported(R, ALTO_F32) ? ALTO_MTTKRP_DETERMINISTIC : ALTO_MTTKRP_AUTO;
  ALTO_TRY(s->iter.ensure(sizeof(IterState)));
  ALTO_TRY_CUDA(cudaMemsetAsync(s->iter.p, 0, sizeof(IterState), st));
  IterState hs{};
  ALTO_TRY(enqueue_iteration(s, L, st));
  if (s->use_graph && s->max_inner > 1) {
    ALTO_TRY(run_graph(s, L));
    ALTO_TRY_CUDA(cudaMemcpyAsync(&hs, s->iter.p, sizeof(IterState), cudaMemcpyDeviceToHost, st));
    ALTO_TRY_CUDA(cudaStreamSynchronize(st));
  } else {
    while (true) {
      ALTO_TRY_CUDA(cudaMemcpyAsync(&hs, s->iter.p, sizeof(IterState), cudaMemcpyDeviceToHost, st));
      ALTO_TRY_CUDA(cudaStreamSynchronize(st));
      if (hs.stop || hs.done >= s->max_inner) break;
      ALTO_TRY(enqueue_iteration(s, L, st));
    }
  }
  return finish_batch(s, hs, inner);
}

alto_status stream_finish_grouped(alto_stream_session* s, int* inner) {
  IterState hs{};
  ALTO_TRY_CUDA(cudaMemcpyAsync(&hs, s->iter.p, sizeof(IterState), cudaMemcpyDeviceToHost, s->st));
  ALTO_TRY_CUDA(cudaStreamSynchronize(s->st));
  return finish_batch(s, hs, inner);
}

bool stream_group_key_equal(const alto_stream_session* a, const alto_stream_session* b) {
  if (a->R != b->R || a->N != b->N || a->t != b->t) return false;
  for (int m = 0; m < a->N; ++m)
    if (a->det[m].hw != b->det[m].hw) return false;
  return true;
}
}  // namespace alto

extern "C" {

alto_status alto_stream_open(int nmodes, int stream_mode, int rank, alto_constraint constraint,
                             double forgetting, int max_inner_iters, double epsilon,
                             alto_cuda_stream stream, alto_stream_session** out) {
  if (!out) {
    set_error("out is NULL");
    return ALTO_ERR_INVALID;
  }
  *out = nullptr;
  if (nmodes < 2 || nmodes > ALTO_MAX_MODES || stream_mode < 0 || stream_mode >= nmodes) {
    set_error("bad nmodes %d / stream_mode %d", nmodes, stream_mode);
    return ALTO_ERR_INVALID;
  }
  if (rank < 1 || rank > 128) {
    set_error("rank %d outside 1..128", rank);
    return ALTO_ERR_UNSUPPORTED;
  }
  if (max_inner_iters < 1) {
    set_error("max_inner_iters must be >= 1");
    return ALTO_ERR_INVALID;
  }
  if (constraint != ALTO_UNCONSTRAINED && constraint != ALTO_NONNEG && constraint != ALTO_LASSO) {
    set_error("unknown constraint %d", (int)constraint);
    return ALTO_ERR_INVALID;
  }
  alto_stream_session* s = new (std::nothrow) alto_stream_session();
  if (!s) return ALTO_ERR_NOMEM;
  s->N = nmodes;
  s->t = stream_mode;
  s->R = rank;
  s->con = constraint;
  s->forgetting = forgetting;
  s->max_inner = max_inner_iters;
  s->eps = epsilon;
  s->st = (cudaStream_t)stream;
  const size_t RR = (size_t)rank * rank;
  alto_status st = ALTO_OK;
  if ((st = s->G.ensure(nmodes * RR * 8)) || (st = s->old_gram.ensure(RR * 8)) ||
      (st = s->ata.ensure(RR * 8)) || (st = s->cross.ensure(nmodes * RR * 8)) || (st = s->W.ensure(RR * 8)) ||
      (st = s->status.ensure(16)) || (st = s->rho.ensure(16)) || (st = s->lam.ensure(rank * 8)) ||
      (st = s->dstat.ensure(3 * ALTO_MAX_MODES * 8)) || (st = s->admm_state.ensure(sizeof(AdmmState)))) {
    delete s;
    return st;
  }
  if (cudaMemsetAsync(s->G.p, 0, nmodes * RR * 8, s->st) != cudaSuccess ||
      cudaMemsetAsync(s->dstat.p, 0, 3 * ALTO_MAX_MODES * 8, s->st) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->capst[0], cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->capst[1], cudaStreamNonBlocking) != cudaSuccess) {
    delete s;
    set_error("session set-up failed: %s", cudaGetErrorString(cudaGetLastError()));
    return ALTO_ERR_CUDA;
  }
  *out = s;
  return ALTO_OK;
}

alto_status alto_stream_push(alto_stream_session* s, const alto_coo* batch, const double* init_vals,
                             uint64_t n_init, int* inner_iters) {
  if (!s || !batch) {
    set_error("session or batch is NULL");
    return ALTO_ERR_INVALID;
  }
  if (batch->nmodes != s->N) {
    set_error("batch has %d modes, session %d", batch->nmodes, s->N);
    return ALTO_ERR_INVALID;
  }
  if (batch->nnz == 0) {
    set_error("empty batch (the reference asserts nnz > 0)");
    return ALTO_ERR_INVALID;
  }
  if (n_init && !init_vals) {
    set_error("init_vals is NULL");
    return ALTO_ERR_INVALID;
  }
  return push_batch(s, batch, init_vals, n_init, inner_iters);
}

alto_status alto_stream_stats(const alto_stream_session* s, double out[9]) {
  if (!s || !out) {
    set_error("session or out is NULL");
    return ALTO_ERR_INVALID;
  }
  out[0] = (double)s->pushes;
  out[1] = s->t_prepare * 1e3;
  out[2] = s->t_inner * 1e3;
  out[3] = s->dev_inner_ms;
  out[4] = s->t_finish * 1e3;
  out[5] = (double)s->inner_total;
  out[6] = s->t_grow * 1e3;
  out[7] = s->t_encode * 1e3;
  out[8] = s->t_sorted * 1e3;
  return ALTO_OK;
}

alto_status alto_stream_factor(alto_stream_session* s, int mode, double* host_out, uint64_t* rows) {
  if (!s || mode < 0 || mode >= s->N) {
    set_error("bad session or mode");
    return ALTO_ERR_INVALID;
  }
  if (mode == s->t) {
    const uint64_t r = s->time_rows.size() / s->R;
    if (rows) *rows = r;
    if (host_out) std::memcpy(host_out, s->time_rows.data(), s->time_rows.size() * sizeof(double));
    return ALTO_OK;
  }
  const uint64_t n = s->dims[mode] * (uint64_t)s->R;
  if (rows) *rows = s->dims[mode];
  if (!host_out || !n) return ALTO_OK;
  std::vector<float> tmp(n);
  ALTO_TRY_CUDA(cudaMemcpyAsync(tmp.data(), s->U[mode].p, n * 4, cudaMemcpyDeviceToHost, s->st));
  ALTO_TRY_CUDA(cudaStreamSynchronize(s->st));
  for (uint64_t q = 0; q < n; ++q) host_out[q] = tmp[q];
  return ALTO_OK;
}

alto_status alto_stream_error(alto_stream_session* s, const alto_coo* X, double* err) {
  if (!s || !X || !err || X->nmodes != s->N || !X->dims || (X->nnz && (!X->cidx || !X->vals)) ||
      (X->index_bytes != 4 && X->index_bytes != 8) || (X->val_dtype != ALTO_F64 && X->val_dtype != ALTO_F32)) {
    set_error("bad session, tensor or output");
    return ALTO_ERR_INVALID;
  }
  if (s->batches == 0) {
    set_error("the model is empty (no batch pushed)");
    return ALTO_ERR_INVALID;
  }
  return model_error(s, X, err);
}

alto_status alto_stream_lambda(alto_stream_session* s, double* host_out) {
  if (!s || !host_out) {
    set_error("session or output is NULL");
    return ALTO_ERR_INVALID;
  }
  ALTO_TRY_CUDA(cudaMemcpyAsync(host_out, s->lam.p, s->R * 8, cudaMemcpyDeviceToHost, s->st));
  ALTO_TRY_CUDA(cudaStreamSynchronize(s->st));
  return ALTO_OK;
}

alto_status alto_stream_set_model(alto_stream_session* s, alto_stream_model model) {
  if (!s || (model != ALTO_MODEL_CPSTREAM && model != ALTO_MODEL_SPCPSTREAM)) {
    set_error("bad session or model");
    return ALTO_ERR_INVALID;
  }
  if (s->batches > 0) {
    set_error("the model is chosen before the first batch");
    return ALTO_ERR_INVALID;
  }
  s->sparse = model == ALTO_MODEL_SPCPSTREAM;
  return ALTO_OK;
}

alto_status alto_stream_set_graph(alto_stream_session* s, int enable) {
  if (!s) {
    set_error("session is NULL");
    return ALTO_ERR_INVALID;
  }
  s->use_graph = enable != 0;
  return ALTO_OK;
}

alto_status alto_stream_close(alto_stream_session* s) {
  delete s;
  return ALTO_OK;
}

}  // extern "C"
