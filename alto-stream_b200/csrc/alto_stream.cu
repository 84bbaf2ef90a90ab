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
// ADMM runs as one launch per sweep over all rows (rows are independent
// except for the four global sums of the stopping test).  Each launch writes
// per-block partial sums; the last block to finish (ticket counter, no
// waiting) adds them in block order and raises a converged flag that makes
// the remaining launches return at once.
#include <cmath>
#include <cstring>
#include <vector>

#include "alto_dense.cuh"

namespace alto {
alto_status convert_f64_to_f32(const double* a, uint64_t n, float* b, cudaStream_t st);
alto_status convert_f32_to_f64(const float* a, uint64_t n, double* b, cudaStream_t st);

constexpr int kAdmmThreads = 256;
constexpr int kAdmmMaxIters = 25;

struct AdmmState {
  int converged;
  int iters;
  unsigned ticket;
  int pad;
};

// Shared row solve: x[c] = sum_k a[k] W[k][c] for the row held by the warp's
// lanes (lane owns columns lane, lane+32, ...).  a is given per lane slot.
template <int SLOTS>
__device__ __forceinline__ void row_solve(const double (&a)[SLOTS], const double* sw, int R,
                                          int lane, double (&x)[SLOTS]) {
#pragma unroll
  for (int s = 0; s < SLOTS; ++s) x[s] = 0.0;
#pragma unroll
  for (int ks = 0; ks < SLOTS; ++ks) {
    const int kbase = ks * 32;
    const int kmax = min(32, R - kbase);
    for (int k = 0; k < kmax; ++k) {
      const double ak = __shfl_sync(0xffffffffu, a[ks], k);
#pragma unroll
      for (int s = 0; s < SLOTS; ++s) {
        const int c = s * 32 + lane;
        if (c < R) x[s] += ak * sw[(kbase + k) * R + c];
      }
    }
  }
}

// First primal update (src/admm.cpp:288-327).
template <int SLOTS>
__global__ void __launch_bounds__(kAdmmThreads)
    admm_first_kernel(const double* __restrict__ rhs, double* __restrict__ primal,
                      const double* __restrict__ dual, double* __restrict__ aux,
                      double* __restrict__ init, const double* __restrict__ W,
                      const double* __restrict__ rho_p, uint64_t I, int R,
                      AdmmState* __restrict__ state) {
  extern __shared__ double sw[];
  for (int p = threadIdx.x; p < R * R; p += blockDim.x) sw[p] = W[p];
  __syncthreads();
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    state->converged = 0;
    state->iters = 0;
    state->ticket = 0;
  }
  const double rho = *rho_p;
  const int lane = threadIdx.x & 31;
  const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t i = gw; i < I; i += nw) {
    double a[SLOTS], x[SLOTS];
#pragma unroll
    for (int s = 0; s < SLOTS; ++s) {
      const int c = s * 32 + lane;
      a[s] = c < R ? rhs[i * R + c] + rho * (primal[i * R + c] + dual[i * R + c]) : 0.0;
    }
    row_solve<SLOTS>(a, sw, R, lane, x);
#pragma unroll
    for (int s = 0; s < SLOTS; ++s) {
      const int c = s * 32 + lane;
      if (c < R) {
        const size_t q = i * R + c;
        init[q] = primal[q];
        aux[q] = x[s];
        const double v = x[s] - dual[q];
        primal[q] = v < 0.0 ? 0.0 : v;
      }
    }
  }
}

// One ADMM sweep (src/admm.cpp:331-425) with the stopping test.
template <int SLOTS>
__global__ void __launch_bounds__(kAdmmThreads)
    admm_sweep_kernel(const double* __restrict__ rhs, double* __restrict__ primal,
                      double* __restrict__ dual, double* __restrict__ aux,
                      double* __restrict__ init, const double* __restrict__ W,
                      const double* __restrict__ rho_p, uint64_t I, int R,
                      double* __restrict__ partials, AdmmState* __restrict__ state, double tol) {
  if (*(volatile int*)&state->converged) return;
  extern __shared__ double sw[];
  for (int p = threadIdx.x; p < R * R; p += blockDim.x) sw[p] = W[p];
  __syncthreads();
  const double rho = *rho_p;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  double p_res = 0, d_res = 0, p_norm = 0, d_norm = 0;
  for (uint64_t i = gw; i < I; i += nw) {
    double a[SLOTS], x[SLOTS];
#pragma unroll
    for (int s = 0; s < SLOTS; ++s) {
      const int c = s * 32 + lane;
      a[s] = 0.0;
      if (c < R) {
        const size_t q = i * R + c;
        const double xv = primal[q];
        const double dd = xv - init[q];
        d_res += dd * dd;
        p_norm += xv * xv;
        const double y = xv - aux[q];
        const double di = dual[q] + y;
        dual[q] = di;
        d_norm += di * di;
        p_res += y * y;
        a[s] = rhs[q] + rho * (xv + di);
      }
    }
    row_solve<SLOTS>(a, sw, R, lane, x);
#pragma unroll
    for (int s = 0; s < SLOTS; ++s) {
      const int c = s * 32 + lane;
      if (c < R) {
        const size_t q = i * R + c;
        aux[q] = x[s];
        double v = x[s] - dual[q];
        v = v > 0.0 ? v : 0.0;
        init[q] = v;
        primal[q] = v;
      }
    }
  }
  // block partials of the four sums
  __shared__ double sred[4][kAdmmThreads / 32];
  double v4[4] = {p_res, d_res, p_norm, d_norm};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    double v = v4[k];
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) sred[k][warp] = v;
  }
  __syncthreads();
  __shared__ bool last;
  if (threadIdx.x == 0) {
    for (int k = 0; k < 4; ++k) {
      double t = 0;
      for (int w = 0; w < kAdmmThreads / 32; ++w) t += sred[k][w];
      partials[(size_t)blockIdx.x * 4 + k] = t;
    }
    __threadfence();
    const unsigned ticket = atomicAdd(&state->ticket, 1u);
    last = ticket == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double t[4] = {0, 0, 0, 0};
    for (unsigned b = 0; b < gridDim.x; ++b)
      for (int k = 0; k < 4; ++k) t[k] += ((volatile double*)partials)[(size_t)b * 4 + k];
    state->iters += 1;
    state->ticket = 0;
    if (t[0] <= tol * t[2] && t[1] <= tol * t[3]) state->converged = 1;
    __threadfence();
  }
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
  DevBuf G, old_gram, ata, hist, W, status, rho, lam, dstat, buf32, rhs, aux, init, prim, time64;
  DevBuf gscr, dscr, admm_part, admm_state, grow_stage, copy_tmp;
  std::vector<double> time_rows;  // concatenated time factor (host)
  alto_tensor* at = nullptr;
  ~alto_stream_session() { delete at; }
};

namespace {

alto_status grow_rows(DevBuf& b, uint64_t old_rows, uint64_t new_cap, size_t row_bytes, DevBuf& tmp,
                      cudaStream_t st) {
  if (b.bytes >= new_cap * row_bytes && b.p) return ALTO_OK;
  const size_t keep = old_rows * row_bytes;
  if (keep) {
    ALTO_TRY(tmp.ensure(keep));
    ALTO_TRY_CUDA(cudaMemcpyAsync(tmp.p, b.p, keep, cudaMemcpyDeviceToDevice, st));
  }
  ALTO_TRY_CUDA(cudaStreamSynchronize(st));
  b.release();
  ALTO_TRY(b.ensure(new_cap * row_bytes));
  if (keep) ALTO_TRY_CUDA(cudaMemcpyAsync(b.p, tmp.p, keep, cudaMemcpyDeviceToDevice, st));
  return ALTO_OK;
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

template <int SLOTS>
alto_status admm_run(alto_stream_session* s, uint64_t I, double* primal, double* dual,
                     cudaStream_t st) {
  const int R = s->R;
  const size_t smem = (size_t)R * R * sizeof(double);
  uint64_t blocks = std::min<uint64_t>((I * 32 + kAdmmThreads - 1) / kAdmmThreads, 148ull * 8);
  if (blocks < 1) blocks = 1;
  ALTO_TRY(s->admm_part.ensure(blocks * 4 * sizeof(double)));
  if (smem > 48 * 1024) {
    ALTO_TRY_CUDA(cudaFuncSetAttribute(admm_first_kernel<SLOTS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    ALTO_TRY_CUDA(cudaFuncSetAttribute(admm_sweep_kernel<SLOTS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  }
  AdmmState* state = s->admm_state.as<AdmmState>();
  admm_first_kernel<SLOTS><<<(unsigned)blocks, kAdmmThreads, smem, st>>>(
      s->rhs.as<double>(), primal, dual, s->aux.as<double>(), s->init.as<double>(),
      s->W.as<double>(), s->rho.as<double>(), I, R, state);
  ALTO_LAUNCHED();
  const double tol = (double)1e-6f;
  for (int k = 0; k < kAdmmMaxIters; ++k) {
    admm_sweep_kernel<SLOTS><<<(unsigned)blocks, kAdmmThreads, smem, st>>>(
        s->rhs.as<double>(), primal, dual, s->aux.as<double>(), s->init.as<double>(),
        s->W.as<double>(), s->rho.as<double>(), I, R, s->admm_part.as<double>(), state, tol);
    ALTO_LAUNCHED();
  }
  return ALTO_OK;
}

alto_status admm(alto_stream_session* s, uint64_t I, double* primal, double* dual, cudaStream_t st) {
  if (s->R <= 32) return admm_run<1>(s, I, primal, dual, st);
  if (s->R <= 64) return admm_run<2>(s, I, primal, dual, st);
  return admm_run<4>(s, I, primal, dual, st);
}

alto_status push_batch(alto_stream_session* s, const alto_coo* b, const double* init_vals,
                       uint64_t n_init, int* inner_out) {
  const int N = s->N, t = s->t, R = s->R;
  cudaStream_t st = s->st;
  const size_t RR = (size_t)R * R;
  const bool first = s->batches == 0;

  // grow the model: new rows of U from init_vals (mode order), prev rows zero
  uint64_t old[ALTO_MAX_MODES];
  uint64_t consumed = 0;
  std::vector<float> host_rows;
  for (int n = 0; n < N; ++n) {
    old[n] = s->dims[n];
    const uint64_t nd = std::max<uint64_t>(b->dims[n], old[n]);
    if (nd > s->cap[n]) {
      const uint64_t nc = std::max<uint64_t>(nd, s->cap[n] + s->cap[n] / 2);
      ALTO_TRY(grow_rows(s->U[n], old[n], nc, R * 4, s->copy_tmp, st));
      ALTO_TRY(grow_rows(s->P[n], old[n], nc, R * 4, s->copy_tmp, st));
      s->dual[n].release();
      ALTO_TRY(s->dual[n].ensure(nc * R * 8));
      s->cap[n] = nc;
    }
    if (nd > old[n]) {
      const uint64_t cnt = (nd - old[n]) * R;
      host_rows.assign(cnt, 0.0f);
      for (uint64_t q = 0; q < cnt; ++q)
        host_rows[q] = consumed + q < n_init ? (float)init_vals[consumed + q] : 0.0f;
      consumed += cnt;
      ALTO_TRY_CUDA(cudaMemcpyAsync(s->U[n].as<float>() + old[n] * R, host_rows.data(), cnt * 4,
                                    cudaMemcpyHostToDevice, st));
      ALTO_TRY_CUDA(cudaMemsetAsync(s->P[n].as<float>() + old[n] * R, 0, cnt * 4, st));
      ALTO_TRY_CUDA(cudaStreamSynchronize(st));  // host_rows is reused
    }
    s->dims[n] = nd;
  }
  uint64_t max_dim = 0;
  for (int n = 0; n < N; ++n) max_dim = std::max(max_dim, s->dims[n]);
  ALTO_TRY(s->buf32.ensure(max_dim * R * 4));
  ALTO_TRY(s->rhs.ensure(max_dim * R * 8));
  ALTO_TRY(s->aux.ensure(max_dim * R * 8));
  ALTO_TRY(s->init.ensure(max_dim * R * 8));
  ALTO_TRY(s->prim.ensure(max_dim * R * 8));
  ALTO_TRY(s->time64.ensure(s->dims[t] * R * 8));
  double* G = s->G.as<double>();
  if (first) {
    ALTO_TRY(rr_op(s->lam.as<double>(), nullptr, R, 3, 0.0, st));
    fill_kernel<<<1, 128, 0, st>>>(s->lam.as<double>(), R, 1.0);
    ALTO_LAUNCHED();
    ALTO_TRY_CUDA(cudaMemsetAsync(s->U[t].p, 0, s->dims[t] * R * 4, st));
    ALTO_TRY_CUDA(cudaMemsetAsync(G + (size_t)t * RR, 0, RR * 8, st));
  }
  for (int n = 0; n < N; ++n)
    if (n != t) ALTO_TRY(gram(s->U[n].as<float>(), s->dims[n], R, G + (size_t)n * RR, s->gscr, st));
  for (int n = 0; n < N; ++n) ALTO_TRY_CUDA(cudaMemsetAsync(s->dual[n].p, 0, s->dims[n] * R * 8, st));

  // update_salto
  alto_coo c = *b;
  uint64_t bd[ALTO_MAX_MODES];
  for (int n = 0; n < N; ++n) bd[n] = s->dims[n];
  c.dims = bd;
  if (!s->at) {
    s->at = new alto_tensor();
    s->at->key_bits = 128;
    s->at->stream_mode = t;
    s->at->stream = st;
  }
  ALTO_TRY(encode_tensor(s->at, &c, 1, st));

  // first batch: 2-norm normalise the non-stream factors, lambda = 1
  if (first) {
    for (int m = 0; m < N; ++m) {
      if (m == t) continue;
      double* Gm = G + (size_t)m * RR;
      lambda_from_gram_kernel<<<1, 128, 0, st>>>(Gm, R, s->lam.as<double>());
      ALTO_LAUNCHED();
      ALTO_TRY(scale_columns(s->U[m].as<float>(), s->dims[m], R, s->lam.as<double>(), nullptr, st));
      ALTO_TRY(gram(s->U[m].as<float>(), s->dims[m], R, Gm, s->gscr, st));
    }
    fill_kernel<<<1, 128, 0, st>>>(s->lam.as<double>(), R, 1.0);
    ALTO_LAUNCHED();
  }

  const void* fac[ALTO_MAX_MODES];
  for (int n = 0; n < N; ++n) fac[n] = s->U[n].p;
  // the deterministic MTTKRP where it runs, so a stream's results repeat
  // bit for bit however many other streams share the device
  const alto_mttkrp_variant mv =
      deterministic_supported(R, ALTO_F32) ? ALTO_MTTKRP_DETERMINISTIC : ALTO_MTTKRP_AUTO;
  const unsigned all = (1u << N) - 1;
  double* dstat = s->dstat.as<double>();  // [N][3]
  double delta = 0.0, prev_delta = 0.0;
  int it;
  for (it = 0; it < s->max_inner; ++it) {
    // time rows: MTTKRP of the stream mode, solve with the other Grams
    ALTO_TRY(run_mttkrp(s->at, t, fac, ALTO_F32, R, s->buf32.as<float>(), 0, mv, st));
    ALTO_TRY(solve_setup(G, N, all & ~(1u << t), R, kSolveRidge, 1e-12, s->W.as<double>(),
                         s->status.as<int>(), nullptr, st));
    ALTO_TRY(apply_f32_to_f64(s->buf32.as<float>(), nullptr, s->W.as<double>(), s->dims[t], R,
                              s->time64.as<double>(), st));
    ALTO_TRY(convert_f64_to_f32(s->time64.as<double>(), s->dims[t] * R, s->U[t].as<float>(), st));
    double* Gt = G + (size_t)t * RR;
    ALTO_TRY(rr_op(s->old_gram.as<double>(), Gt, (int)RR, 0, 0.0, st));
    ALTO_TRY(rank_update(Gt, s->time64.as<double>(), s->dims[t], R, st));

    for (int j = 0; j < N; ++j) {
      if (j == t) continue;
      const uint64_t I = s->dims[j];
      ALTO_TRY(run_mttkrp(s->at, j, fac, ALTO_F32, R, s->buf32.as<float>(), 0, mv, st));
      // historical term
      ALTO_TRY(rr_op(s->ata.as<double>(), s->old_gram.as<double>(), (int)RR, 0, 0.0, st));
      for (int m = 0; m < N; ++m) {
        if (m == j || m == t) continue;
        ALTO_TRY(cross_gram(s->P[m].as<float>(), s->U[m].as<float>(), s->dims[m], R,
                            s->hist.as<double>(), s->gscr, st));
        ALTO_TRY(rr_op(s->ata.as<double>(), s->hist.as<double>(), (int)RR, 1, 0.0, st));
      }
      ALTO_TRY(apply_f32_to_f64(s->P[j].as<float>(), s->buf32.as<float>(), s->ata.as<double>(), I, R,
                                s->rhs.as<double>(), st));
      if (s->con == ALTO_UNCONSTRAINED) {
        ALTO_TRY(solve_setup(G, N, all & ~(1u << j), R, kSolveRidge, 1e-12, s->W.as<double>(),
                             s->status.as<int>(), nullptr, st));
        ALTO_TRY(apply_f64_to_f32(s->rhs.as<double>(), s->W.as<double>(), I, R, s->U[j].as<float>(), st));
      } else {
        ALTO_TRY(solve_setup(G, N, all & ~(1u << j), R, kSolveAdmm, 0.0, s->W.as<double>(),
                             s->status.as<int>(), s->rho.as<double>(), st));
        ALTO_TRY(convert_f32_to_f64(s->U[j].as<float>(), I * R, s->prim.as<double>(), st));
        ALTO_TRY(admm(s, I, s->prim.as<double>(), s->dual[j].as<double>(), st));
        ALTO_TRY(convert_f64_to_f32(s->prim.as<double>(), I * R, s->U[j].as<float>(), st));
      }
      ALTO_TRY(gram(s->U[j].as<float>(), I, R, G + (size_t)j * RR, s->gscr, st));
      ALTO_TRY(dot_stats(s->P[j].as<float>(), s->U[j].as<float>(), I * R, nullptr, R, dstat + 3 * j,
                         s->dscr, st));
    }
    double h[3 * ALTO_MAX_MODES];
    ALTO_TRY_CUDA(cudaMemcpyAsync(h, dstat, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, st));
    int info = 0;
    ALTO_TRY_CUDA(cudaMemcpyAsync(&info, s->status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    ALTO_TRY_CUDA(cudaStreamSynchronize(st));
    if (info && s->con != ALTO_UNCONSTRAINED) {
      set_error("Cholesky of the ADMM normal equations failed (info %d)", info);
      return ALTO_ERR_NOT_SPD;
    }
    delta = 0.0;
    for (int j = 0; j < N; ++j)
      if (j != t) delta += std::sqrt(h[3 * j + 1]) / (std::sqrt(h[3 * j + 2]) + 1e-12);
    if (it > 0 && std::fabs(prev_delta - delta) < s->eps) {
      ++it;
      break;
    }
    prev_delta = delta;
  }
  if (inner_out) *inner_out = it;
  // forgetting, prev <- current, time rows out
  ALTO_TRY(rr_op(G + (size_t)t * RR, nullptr, (int)RR, 2, s->forgetting, st));
  for (int n = 0; n < N; ++n)
    ALTO_TRY_CUDA(cudaMemcpyAsync(s->P[n].p, s->U[n].p, s->dims[n] * R * 4, cudaMemcpyDeviceToDevice, st));
  const size_t base = s->time_rows.size();
  s->time_rows.resize(base + s->dims[t] * R);
  ALTO_TRY_CUDA(cudaMemcpyAsync(s->time_rows.data() + base, s->time64.p, s->dims[t] * R * 8,
                                cudaMemcpyDeviceToHost, st));
  ALTO_TRY_CUDA(cudaStreamSynchronize(st));
  s->batches += 1;
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
      (st = s->ata.ensure(RR * 8)) || (st = s->hist.ensure(RR * 8)) || (st = s->W.ensure(RR * 8)) ||
      (st = s->status.ensure(16)) || (st = s->rho.ensure(16)) || (st = s->lam.ensure(rank * 8)) ||
      (st = s->dstat.ensure(3 * ALTO_MAX_MODES * 8)) || (st = s->admm_state.ensure(sizeof(AdmmState)))) {
    delete s;
    return st;
  }
  if (cudaMemsetAsync(s->G.p, 0, nmodes * RR * 8, s->st) != cudaSuccess ||
      cudaMemsetAsync(s->dstat.p, 0, 3 * ALTO_MAX_MODES * 8, s->st) != cudaSuccess) {
    delete s;
    set_error("cudaMemsetAsync failed");
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

alto_status alto_stream_lambda(alto_stream_session* s, double* host_out) {
  if (!s || !host_out) {
    set_error("session or output is NULL");
    return ALTO_ERR_INVALID;
  }
  ALTO_TRY_CUDA(cudaMemcpyAsync(host_out, s->lam.p, s->R * 8, cudaMemcpyDeviceToHost, s->st));
  ALTO_TRY_CUDA(cudaStreamSynchronize(s->st));
  return ALTO_OK;
}

alto_status alto_stream_close(alto_stream_session* s) {
  delete s;
  return ALTO_OK;
}

}  // extern "C"
