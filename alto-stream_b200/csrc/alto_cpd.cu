// CP-ALS on the device and the host-buffer MTTKRP entry point.
//
// Reference: cpd_alto (jeewhanchoi/ALTO-stream include/cpd.hpp:47-191):
// per iteration, per mode j: zero U_j, MTTKRP into U_j, keep the last
// mode's MTTKRP for the fit, pseudo_inverse (Hadamard of the other Grams +
// 1e-3 I, Cholesky solve, dgelsy fallback), normalise columns (2-norm on
// the first iteration, max-norm after), update the Gram; then the fit
// (include/cpd.hpp:193-275) and the |fit - prev_fit| < epsilon stop test.
//
// Device layout: factors float32 (dims x rank, row-major), optional
// bfloat16 shadows that the MTTKRP gathers from, Grams / inverses / lambda
// float64.  The MTTKRP output goes to a separate float32 buffer that the
// solve reads, so the last mode's MTTKRP is still there for the fit.
#include <cmath>
#include <vector>

#include "alto_dense.cuh"

namespace alto {

__global__ void f64_to_f32_kernel(const double* __restrict__ a, uint64_t n, float* __restrict__ b) {
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < n;
       q += (uint64_t)gridDim.x * blockDim.x)
    b[q] = (float)a[q];
}

__global__ void add_f32_to_f64_kernel(const float* __restrict__ a, uint64_t n, double* __restrict__ b) {
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < n;
       q += (uint64_t)gridDim.x * blockDim.x)
    b[q] += (double)a[q];
}

__global__ void f32_to_f64_kernel(const float* __restrict__ a, uint64_t n, double* __restrict__ b) {
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < n;
       q += (uint64_t)gridDim.x * blockDim.x)
    b[q] = (double)a[q];
}

static unsigned ew_grid(uint64_t n) {
  uint64_t b = (n + 255) / 256;
  if (b > 148ull * 16) b = 148ull * 16;
  return (unsigned)(b ? b : 1);
}

alto_status export_keys(const alto_tensor* t, uint64_t* d_out, float* d_vals, cudaStream_t st);

alto_status convert_f64_to_f32(const double* a, uint64_t n, float* b, cudaStream_t st) {
  if (!n) return ALTO_OK;
  f64_to_f32_kernel<<<ew_grid(n), 256, 0, st>>>(a, n, b);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

alto_status convert_f32_to_f64(const float* a, uint64_t n, double* b, cudaStream_t st) {
  if (!n) return ALTO_OK;
  f32_to_f64_kernel<<<ew_grid(n), 256, 0, st>>>(a, n, b);
  ALTO_LAUNCHED();
  return ALTO_OK;
}

}  // namespace alto

using namespace alto;

// Device staging owned by one host-buffer MTTKRP call site (a thread):
// each factor's float64 copy and its float32 rounding, with the host array
// they copy (address and length) and whether they still match it.
struct HostStage {
  DevBuf f64[ALTO_MAX_MODES];
  DevBuf f32[ALTO_MAX_MODES];
  DevBuf out;
  const double* host[ALTO_MAX_MODES] = {};
  uint64_t len[ALTO_MAX_MODES] = {};
  bool f64_ok[ALTO_MAX_MODES] = {};
  bool f32_ok[ALTO_MAX_MODES] = {};
};

static alto_status mttkrp_host_impl(alto_tensor* t, int mode, double* const* factors_host, int rank,
                                    uint32_t changed, alto_cuda_stream stream);

extern "C" alto_status alto_mttkrp_host(alto_tensor* t, int mode, double* const* factors_host,
                                        int rank, alto_cuda_stream stream) {
  return mttkrp_host_impl(t, mode, factors_host, rank, ~0u, stream);
}

extern "C" alto_status alto_mttkrp_host_changed(alto_tensor* t, int mode, double* const* factors_host,
                                                int rank, uint32_t changed, alto_cuda_stream stream) {
  return mttkrp_host_impl(t, mode, factors_host, rank, changed, stream);
}

static alto_status mttkrp_host_impl(alto_tensor* t, int mode, double* const* factors_host, int rank,
                                    uint32_t changed, alto_cuda_stream stream) {
  if (!t || !factors_host) {
    set_error("tensor or factors is NULL");
    return ALTO_ERR_INVALID;
  }
  if (mode < 0 || mode >= t->nmodes || rank < 1) {
    set_error("bad mode or rank");
    return ALTO_ERR_INVALID;
  }
  for (int m = 0; m < t->nmodes; ++m)
    if (!factors_host[m]) {
      set_error("factors[%d] is NULL", m);
      return ALTO_ERR_INVALID;
    }
  cudaStream_t st = (cudaStream_t)stream;
  static thread_local HostStage* stage = nullptr;
  if (!stage) stage = new HostStage();
  const void* dev[ALTO_MAX_MODES] = {nullptr};
  for (int m = 0; m < t->nmodes; ++m) {
    const uint64_t n = t->dims[m] * (uint64_t)rank;
    const bool same = stage->f64_ok[m] && !((changed >> m) & 1u) && stage->host[m] == factors_host[m] &&
                      stage->len[m] == n && stage->f64[m].p;
    if (!same) {
      stage->f64_ok[m] = stage->f32_ok[m] = false;
      ALTO_TRY(stage->f64[m].ensure(n * 8));
      ALTO_TRY_CUDA(cudaMemcpyAsync(stage->f64[m].p, factors_host[m], n * 8, cudaMemcpyHostToDevice, st));
      stage->host[m] = factors_host[m];
      stage->len[m] = n;
      stage->f64_ok[m] = true;
    }
    if (m == mode) continue;
    if (!stage->f32_ok[m]) {
      ALTO_TRY(stage->f32[m].ensure(n * 4));
      ALTO_TRY(convert_f64_to_f32(stage->f64[m].as<double>(), n, stage->f32[m].as<float>(), st));
      stage->f32_ok[m] = true;
    }
    dev[m] = stage->f32[m].p;
  }
  const uint64_t no = t->dims[mode] * (uint64_t)rank;
  // until this call completes, the output mode's copies do not match its
  // host array (an error below leaves them unmatched)
  stage->f64_ok[mode] = stage->f32_ok[mode] = false;
  ALTO_TRY(stage->out.ensure(no * 4));
  ALTO_TRY(run_mttkrp(t, mode, dev, ALTO_F32, rank, stage->out.as<float>(), 0, ALTO_MTTKRP_AUTO, st));
  if (no) {
    add_f32_to_f64_kernel<<<ew_grid(no), 256, 0, st>>>(stage->out.as<float>(), no,
                                                        stage->f64[mode].as<double>());
    ALTO_LAUNCHED();
  }
  ALTO_TRY_CUDA(cudaMemcpyAsync(factors_host[mode], stage->f64[mode].p, no * 8, cudaMemcpyDeviceToHost, st));
  ALTO_TRY_CUDA(cudaStreamSynchronize(st));
  stage->f64_ok[mode] = true;  // the device copy is what the host now holds
  return ALTO_OK;
}

extern "C" alto_status alto_cpd_als(alto_tensor* t, int rank, double* const* U_host,
                                    double* lambda_host, int max_iters, double epsilon,
                                    alto_fit_mode fit_mode, alto_dtype storage, double* fits,
                                    int* iters, alto_cuda_stream stream) {
  if (!t || !U_host || !lambda_host) {
    set_error("tensor, U or lambda is NULL");
    return ALTO_ERR_INVALID;
  }
  if (rank < 1 || rank > 128) {
    set_error("rank %d outside 1..128", rank);
    return ALTO_ERR_UNSUPPORTED;
  }
  if (storage != ALTO_F32 && storage != ALTO_BF16) {
    set_error("factor storage must be float32 or bfloat16");
    return ALTO_ERR_INVALID;
  }
  if (max_iters < 0) {
    set_error("max_iters < 0");
    return ALTO_ERR_INVALID;
  }
  const int N = t->nmodes, R = rank;
  cudaStream_t st = (cudaStream_t)stream;
  const bool bf16 = storage == ALTO_BF16;

  DevBuf U[ALTO_MAX_MODES], Ub[ALTO_MAX_MODES];
  DevBuf grams, W, status, mbuf, stats, lam, scal, gscr, dscr, stage64;
  uint64_t max_dim = 0;
  for (int m = 0; m < N; ++m) max_dim = std::max<uint64_t>(max_dim, t->dims[m]);
  ALTO_TRY(grams.ensure((size_t)N * R * R * 8));
  ALTO_TRY(W.ensure((size_t)R * R * 8));
  ALTO_TRY(status.ensure(16));
  ALTO_TRY(mbuf.ensure(max_dim * R * 4));
  ALTO_TRY(lam.ensure(R * 8));
  ALTO_TRY(scal.ensure(8 * 8));
  ALTO_TRY(stage64.ensure(max_dim * R * 8));
  for (int m = 0; m < N; ++m) {
    const uint64_t n = t->dims[m] * (uint64_t)R;
    ALTO_TRY(U[m].ensure(n * 4));
    if (bf16) ALTO_TRY(Ub[m].ensure(n * 2));
    ALTO_TRY_CUDA(cudaMemcpyAsync(stage64.p, U_host[m], n * 8, cudaMemcpyHostToDevice, st));
    ALTO_TRY(convert_f64_to_f32(stage64.as<double>(), n, U[m].as<float>(), st));
    if (bf16) ALTO_TRY(to_bf16(U[m].as<float>(), n, Ub[m].as<__nv_bfloat16>(), st));
    ALTO_TRY(gram(U[m].as<float>(), t->dims[m], R, grams.as<double>() + (size_t)m * R * R, gscr, st));
  }
  ALTO_TRY_CUDA(cudaMemcpyAsync(lam.p, lambda_host, R * 8, cudaMemcpyHostToDevice, st));
  double* d_scal = scal.as<double>();  // [0] normX, [1..3] dot stats, [4] normU
  {  // ||X||^2 over the stored (float32) values
    DevBuf v;
    ALTO_TRY(v.ensure(std::max<uint64_t>(t->nnz, 1) * 4));
    ALTO_TRY(export_keys(t, nullptr, v.as<float>(), st));
    ALTO_TRY(sum_squares(v.as<float>(), t->nnz, d_scal + 0, dscr, st));
    ALTO_TRY_CUDA(cudaStreamSynchronize(st));
  }

  const void* fac[ALTO_MAX_MODES];
  for (int m = 0; m < N; ++m) fac[m] = bf16 ? Ub[m].p : U[m].p;
  const alto_dtype fdt = bf16 ? ALTO_BF16 : ALTO_F32;
  const unsigned all = (1u << N) - 1;

  double fit = 0.0, prev_fit = 0.0;
  int it_run = max_iters;
  for (int it = 0; it < max_iters; ++it) {
    for (int j = 0; j < N; ++j) {
      const uint64_t I = t->dims[j];
      ALTO_TRY(run_mttkrp(t, j, fac, fdt, R, mbuf.as<float>(), 0, ALTO_MTTKRP_AUTO, st));
      ALTO_TRY(solve_setup(grams.as<double>(), N, all & ~(1u << j), R, kSolveRidgeDiagFallback, 1e-3,
                           W.as<double>(), status.as<int>(), nullptr, st));
      int nb = 0;
      ALTO_TRY(apply_f32(mbuf.as<float>(), W.as<double>(), I, R, U[j].as<float>(), &stats, &nb, st));
      ALTO_TRY(column_lambda(stats.as<double>(), nb, R, it == 0 ? 0 : 1, lam.as<double>(), st));
      ALTO_TRY(scale_columns(U[j].as<float>(), I, R, lam.as<double>(),
                             bf16 ? Ub[j].as<__nv_bfloat16>() : nullptr, st));
      ALTO_TRY(gram(U[j].as<float>(), I, R, grams.as<double>() + (size_t)j * R * R, gscr, st));
    }
    // fit: <X, M> from the last mode's MTTKRP, ||M||^2 from Grams and lambda
    const uint64_t IL = t->dims[N - 1];
    ALTO_TRY(dot_stats(U[N - 1].as<float>(), mbuf.as<float>(), IL * R, lam.as<double>(), R, d_scal + 1,
                       dscr, st));
    ALTO_TRY(model_norm(grams.as<double>(), N, R, lam.as<double>(), fit_mode == ALTO_FIT_EXACT ? 1 : 0,
                        d_scal + 4, st));
    double h[5];
    ALTO_TRY_CUDA(cudaMemcpyAsync(h, d_scal, sizeof(h), cudaMemcpyDeviceToHost, st));
    ALTO_TRY_CUDA(cudaStreamSynchronize(st));
    const double normX = h[0], inner = h[1], normU = h[4];
    double res = normX + normU - 2.0 * inner;
    if (res > 0.0) res = std::sqrt(res);
    fit = res / std::sqrt(normX);
    if (fits) fits[it] = fit;
    if (it > 0 && std::fabs(prev_fit - fit) < epsilon) {
      it_run = it + 1;
      break;
    }
    prev_fit = fit;
  }
  for (int m = 0; m < N; ++m) {
    const uint64_t n = t->dims[m] * (uint64_t)R;
    ALTO_TRY(convert_f32_to_f64(U[m].as<float>(), n, stage64.as<double>(), st));
    ALTO_TRY_CUDA(cudaMemcpyAsync(U_host[m], stage64.p, n * 8, cudaMemcpyDeviceToHost, st));
    ALTO_TRY_CUDA(cudaStreamSynchronize(st));
  }
  ALTO_TRY_CUDA(cudaMemcpyAsync(lambda_host, lam.p, R * 8, cudaMemcpyDeviceToHost, st));
  ALTO_TRY_CUDA(cudaStreamSynchronize(st));
  if (iters) *iters = it_run;
  return ALTO_OK;
}
