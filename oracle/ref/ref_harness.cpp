// Test infrastructure only: a thin C-callable harness around the reference
// implementation of ALTO (jeewhanchoi/ALTO-stream), compiled from the
// reference's own, unmodified sources by oracle/ref/Makefile into
// oracle/_ref/libaltoref{64,128}.so.  It is the compiled reference that pins the C
// restatement in oracle/alto_oracle.c and the timed CPU baseline of bench.py;
// nothing in the product links or loads it.
//
// The reference exposes C++ templates and free functions only, so this file
// compiles `src/streaming_cpd.cpp` into the same translation unit (to reach the
// `cpstream_alto_iter` template) and drives the reference's own building
// blocks: create_alto / init_salto / update_salto (include/alto.hpp:151-582),
// mttkrp_alto_par (include/alto.hpp:902), the COO mttkrp (src/mttkrp.cpp:122),
// and the CP-ALS and CP-stream drivers (include/cpd.hpp:47, src/streaming_cpd.cpp:26).
//
// Two drivers are re-sequenced here instead of called whole, because calling
// them whole would read uninitialised heap or the C library's rand():
//   * ref_cpd_als follows cpd_alto (include/cpd.hpp:47-191) step for step, but
//     its Gram matrices start zero-filled.  cpd_alto allocates them with
//     init_mat (src/matrix.cpp:3-11, no fill), dsyrk writes only the upper
//     triangle (src/gram.cpp:29-41), and cpd_fit_alto reads the lower one
//     (include/cpd.hpp:228-246); zero fill is what a fresh glibc heap gives.
//   * ref_cpstream follows cpstream (src/streaming_cpd.cpp:26-366) for the
//     CP-stream (ALTO) model, taking its random initial and growth values from
//     a caller-supplied array in the order KruskalModelRandomInit and
//     GrowKruskalModel would draw them (src/kruskal_model.cpp:101-178), so the
//     CUDA path can start from the identical state.
#include "streaming_cpd.cpp"
#include "streaming_sptensor.hpp"

#include <cstdint>
#include <vector>

extern "C" void openblas_set_num_threads(int);

namespace {

struct RefTensor {
  SparseTensor* X;
  AltoTensor<LIType>* AT;
};

SparseTensor* make_coo(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* cidx,
                       const double* vals) {
  SparseTensor* X = (SparseTensor*)AlignedMalloc(sizeof(SparseTensor));
  X->nmodes = nmodes;
  X->nnz = nnz;
  X->dims = (IType*)AlignedMalloc(sizeof(IType) * nmodes);
  X->cidx = (IType**)AlignedMalloc(sizeof(IType*) * nmodes);
  for (int m = 0; m < nmodes; ++m) {
    X->dims[m] = dims[m];
    X->cidx[m] = (IType*)AlignedMalloc(sizeof(IType) * (nnz ? nnz : 1));
    if (nnz) memcpy(X->cidx[m], cidx + (size_t)m * nnz, sizeof(IType) * nnz);
  }
  X->vals = (FType*)AlignedMalloc(sizeof(FType) * (nnz ? nnz : 1));
  if (nnz) memcpy(X->vals, vals, sizeof(FType) * nnz);
  return X;
}

void put_lit(LIType v, uint64_t* out) {
  out[0] = (uint64_t)v;
  if constexpr (sizeof(LIType) > 8) {
    out[1] = (uint64_t)(v >> 64);
  } else {
    out[1] = 0;
  }
}

// Sequential reader over the caller's array of initial values.
struct ValueStream {
  const double* v;
  size_t n, pos;
  double next() { return pos < n ? v[pos++] : 0.0; }
};

}  // namespace

extern "C" {

int ref_lit_bits(void) { return (int)(sizeof(LIType) * 8); }

void ref_set_threads(int n) {
  omp_set_num_threads(n);
  openblas_set_num_threads(1);
}

int ref_max_threads(void) { return omp_get_max_threads(); }

int ref_get_num_ptrn(uint64_t nnz) { return get_num_ptrn(nnz); }

// create_alto when stream_mode < 0, else init_salto + update_salto.
void* ref_alto_create(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* cidx,
                      const double* vals, int nprtn, int stream_mode) {
  RefTensor* h = new RefTensor;
  h->X = make_coo(nmodes, dims, nnz, cidx, vals);
  if (stream_mode < 0) {
    create_alto(h->X, &h->AT, nprtn);
  } else {
    init_salto(h->X, &h->AT, nprtn, stream_mode);
    update_salto(h->X, h->AT, nprtn);
  }
  return h;
}

void ref_alto_destroy(void* p) {
  RefTensor* h = (RefTensor*)p;
  destroy_alto(h->AT);
  DestroySparseTensor(h->X);
  delete h;
}

int ref_alto_nprtn(void* p) { return ((RefTensor*)p)->AT->nprtn; }

// masks: 2*nmodes words (lo, hi); alto_mask: 2 words; idx: 2*nnz words;
// prtn_ptr: nprtn+1; intervals: 2*nprtn*nmodes (start, stop), partition-major.
void ref_alto_export(void* p, uint64_t* masks, uint64_t* alto_mask, uint64_t* idx, double* vals,
                     uint64_t* prtn_ptr, uint64_t* intervals) {
  AltoTensor<LIType>* at = ((RefTensor*)p)->AT;
  int N = at->nmode;
  if (masks)
    for (int m = 0; m < N; ++m) put_lit(at->mode_masks[m], masks + 2 * m);
  if (alto_mask) put_lit(at->alto_mask, alto_mask);
  if (idx)
    for (IType i = 0; i < at->nnz; ++i) put_lit(at->idx[i], idx + 2 * i);
  if (vals) memcpy(vals, at->vals, sizeof(double) * at->nnz);
  if (prtn_ptr)
    for (int q = 0; q <= at->nprtn; ++q) prtn_ptr[q] = at->prtn_ptr[q];
  if (intervals)
    for (int q = 0; q < at->nprtn * N; ++q) {
      intervals[2 * q] = at->prtn_intervals[q].start;
      intervals[2 * q + 1] = at->prtn_intervals[q].stop;
    }
}

// One mttkrp_alto_par call (accumulates into factors[mode]), with its own
// da_mem scratch, exactly as BenchmarkAlto sets it up (src/main.cpp:486-500).
void ref_mttkrp(void* p, int mode, double** factors, int rank) {
  AltoTensor<LIType>* at = ((RefTensor*)p)->AT;
  std::vector<std::vector<size_t>> oidx;
  FType** ofibs = NULL;
  create_da_mem(mode, rank, at, &ofibs);
  mttkrp_alto_par(mode, factors, rank, at, NULL, ofibs, oidx);
  destroy_da_mem(at, ofibs, rank, mode);
}

// Seconds per repetition of mttkrp_alto_par on `mode` (all modes when -1),
// timed like BenchmarkAlto (src/main.cpp:497-512): one warm-up, then reps.
double ref_mttkrp_time(void* p, int mode, double** factors, int rank, int reps) {
  AltoTensor<LIType>* at = ((RefTensor*)p)->AT;
  std::vector<std::vector<size_t>> oidx;
  FType** ofibs = NULL;
  create_da_mem(mode, rank, at, &ofibs);
  int m0 = mode < 0 ? 0 : mode;
  int m1 = mode < 0 ? at->nmode : mode + 1;
  for (int m = m0; m < m1; ++m) mttkrp_alto_par(m, factors, rank, at, NULL, ofibs, oidx);
  double t0 = omp_get_wtime();
  for (int r = 0; r < reps; ++r)
    for (int m = m0; m < m1; ++m) mttkrp_alto_par(m, factors, rank, at, NULL, ofibs, oidx);
  double t = (omp_get_wtime() - t0) / (reps > 0 ? reps : 1);
  destroy_da_mem(at, ofibs, rank, mode);
  return t;
}

// Sequential COO MTTKRP (src/mttkrp.cpp:122-156), accumulating into factors[mode].
void ref_coo_mttkrp(void* p, int mode, double** factors, int rank) {
  SparseTensor* X = ((RefTensor*)p)->X;
  KruskalModel M;
  M.mode = X->nmodes;
  M.dims = X->dims;
  M.rank = rank;
  M.U = factors;
  M.lambda = NULL;
  mttkrp(X, &M, mode);
}

// CP-ALS on the ALTO tensor, step for step as cpd_alto (include/cpd.hpp:47-191)
// with zero-filled Gram storage.  U[n] (dims[n] x rank, row-major) and lambda
// are the initial model on entry and the result on exit.  fits[i] receives the
// value cpd_fit_alto reports after iteration i.  Returns the iterations run.
int ref_cpd_als(void* p, double** U, double* lambda, int rank, int max_iters, double epsilon,
                double* fits) {
  AltoTensor<LIType>* AT = ((RefTensor*)p)->AT;
  int nmodes = AT->nmode;
  IType* dims = AT->dims;
  KruskalModel Mv;
  Mv.mode = nmodes;
  Mv.dims = dims;
  Mv.rank = rank;
  Mv.U = U;
  Mv.lambda = lambda;
  KruskalModel* M = &Mv;

  IType nthreads = omp_get_max_threads();
  FType* scratch = (FType*)AlignedMalloc(sizeof(FType) * dims[nmodes - 1] * rank);
  FType** lambda_sp = (FType**)AlignedMalloc(sizeof(FType*) * nthreads);
  for (IType t = 0; t < nthreads; ++t) lambda_sp[t] = (FType*)AlignedMalloc(sizeof(FType) * rank);

  double fit = 0.0, prev_fit = 0.0;
  FType normAT = 0.0;
  FType* vals = AT->vals;
  IType nnz = AT->nnz;
#pragma omp parallel for reduction(+ : normAT) schedule(static)
  for (IType i = 0; i < nnz; ++i) normAT += vals[i] * vals[i];

  Matrix** grams = (Matrix**)AlignedMalloc(sizeof(Matrix*) * nmodes);
  for (int i = 0; i < nmodes; ++i) grams[i] = zero_mat(rank, rank);
  for (int i = 0; i < nmodes; ++i) update_gram(grams[i], M, i);

  std::vector<std::vector<size_t>> oidx;
  FType** ofibs = NULL;
  create_da_mem(-1, rank, AT, &ofibs);

  int iters = max_iters;
  for (int i = 0; i < max_iters; i++) {
    for (int j = 0; j < nmodes; j++) {
      ParMemset(M->U[j], 0, sizeof(FType) * dims[j] * rank);
      mttkrp_alto_par(j, M->U, rank, AT, NULL, ofibs, oidx);
      if (j == nmodes - 1) ParMemcpy(scratch, M->U[j], sizeof(FType) * dims[j] * rank);
      pseudo_inverse(grams, M, j);
      if (i == 0)
        KruskalModelNorm(M, j, MAT_NORM_2, lambda_sp);
      else
        KruskalModelNorm(M, j, MAT_NORM_MAX, lambda_sp);
      update_gram(grams[j], M, j);
    }
    fit = cpd_fit_alto(AT, M, grams, scratch, normAT);
    if (fits) fits[i] = fit;
    if ((i > 0) && (fabs(prev_fit - fit) < epsilon)) {
      iters = i + 1;
      break;
    }
    prev_fit = fit;
  }

  for (IType t = 0; t < nthreads; ++t) free(lambda_sp[t]);
  free(lambda_sp);
  free(scratch);
  destroy_da_mem(AT, ofibs, rank, -1);
  for (int i = 0; i < nmodes; ++i) free_mat(grams[i]);
  free(grams);
  return iters;
}

// CP-stream (ALTO), following cpstream (src/streaming_cpd.cpp:26-366) batch by
// batch.  Batch s has nmodes dims at batch_dims[s*nmodes..], nnz batch_nnz[s],
// coordinates at cidx (per batch: nmodes contiguous arrays of batch_nnz[s]
// entries, batches back to back) and values at vals (batches back to back).
// init_vals feeds the random initial model and every growth, in the order the
// reference would call rand().  nonneg selects apply_nonneg_constraint.
// Outputs: out_U[m] (final dims[m] x rank for m != stream_mode; for the stream
// mode the concatenated time factor, total_time x rank), out_lambda (rank),
// slice_seconds (nbatch, may be NULL).  Returns the total time steps.
static int run_stream(int nmodes, int stream_mode, int nbatch, const uint64_t* batch_dims,
                      const uint64_t* batch_nnz, const uint64_t* cidx, const double* vals, int rank,
                      int max_iters, double epsilon, int nonneg, const double* init_vals,
                      uint64_t n_init_vals, double** out_U, double* out_lambda, double* slice_seconds,
                      bool sparse) {
  ValueStream vs{init_vals, (size_t)n_init_vals, 0};
  cpd_constraint* con = init_constraint();
  if (nonneg) apply_nonneg_constraint(con);

  AltoTensor<LIType>* AT = NULL;
  KruskalModel* M = NULL;
  KruskalModel* prev_M = NULL;
  Matrix** grams = NULL;
  StreamMatrix* global_time = new StreamMatrix(rank);
  admm_ws* ws = admm_ws_init(nmodes);
  SparseCPGrams* scpgrams = sparse ? InitSparseCPGrams(nmodes, rank) : NULL;
  double t_tensor = 0.0;

  size_t off_idx = 0, off_val = 0;
  int it = 0;
  for (int s = 0; s < nbatch; ++s) {
    double w0 = omp_get_wtime();
    uint64_t nnz = batch_nnz[s];
    SparseTensor* t_batch = make_coo(nmodes, batch_dims + (size_t)s * nmodes, nnz, cidx + off_idx,
                                     vals + off_val);
    off_idx += (size_t)nmodes * nnz;
    off_val += nnz;
    if (s == 0) init_salto(t_batch, &AT, omp_get_max_threads(), stream_mode);

    if (s == 0) {
      CreateKruskalModel(t_batch->nmodes, t_batch->dims, rank, &M);
      CreateKruskalModel(t_batch->nmodes, t_batch->dims, rank, &prev_M);
      for (int r = 0; r < rank; ++r) M->lambda[r] = 1.0;
      for (int n = 0; n < nmodes; ++n)
        for (IType i = 0; i < M->dims[n] * (IType)rank; ++i) M->U[n][i] = vs.next();
      KruskalModelZeroInit(prev_M);
      memset(M->U[stream_mode], 0, sizeof(FType) * t_batch->dims[stream_mode] * rank);
      grams = (Matrix**)AlignedMalloc(sizeof(Matrix*) * nmodes);
      for (int i = 0; i < nmodes; ++i) grams[i] = zero_mat(rank, rank);
      for (int i = 0; i < nmodes; ++i) update_gram(grams[i], M, i);
      for (int i = 0; i < rank * rank; ++i) grams[stream_mode]->vals[i] = 0.0;
    } else {
      std::vector<IType> old_dims(M->dims, M->dims + nmodes);
      GrowKruskalModel(t_batch->dims, M, FILL_ZEROS, 0);
      for (int n = 0; n < nmodes; ++n)
        for (IType i = old_dims[n] * rank; i < t_batch->dims[n] * (IType)rank; ++i)
          M->U[n][i] = vs.next();
      GrowKruskalModel(t_batch->dims, prev_M, FILL_ZEROS, 0);
      for (int j = 0; j < M->mode; ++j)
        if (j != stream_mode) update_gram(grams[j], M, j);
    }

    int max_dim = 0;
    for (int m = 0; m < nmodes; ++m) {
      ws->duals[m] = zero_mat(t_batch->dims[m], rank);
      if ((int)t_batch->dims[m] > max_dim) max_dim = t_batch->dims[m];
    }
    ws->mttkrp_buf = zero_mat(max_dim, rank);
    ws->auxil = zero_mat(max_dim, rank);
    ws->mat_init = zero_mat(max_dim, rank);

    if (sparse) {
      spcpstream_alto_iter(t_batch, AT, M, prev_M, grams, scpgrams, max_iters, epsilon, stream_mode, it, con, ws,
                           &t_tensor);
    } else {
      int num_partitions = get_num_ptrn(t_batch->nnz);
      FType** ofibs = NULL;
      update_salto(t_batch, AT, num_partitions);
      create_da_mem(-1, rank, AT, &ofibs);
      cpstream_alto_iter(AT, ofibs, M, prev_M, grams, max_iters, epsilon, stream_mode, it, con, ws,
                         &t_tensor);
      destroy_da_mem(AT, ofibs, rank, -1);
    }

    it += t_batch->dims[stream_mode];
    CopyKruskalModel(prev_M, M);
    global_time->grow_zero(it);
    memcpy(&(global_time->mat()->vals[rank * (it - t_batch->dims[stream_mode])]),
           M->U[stream_mode], M->dims[stream_mode] * rank * sizeof(FType));

    for (int m = 0; m < nmodes; ++m) free_mat(ws->duals[m]);
    free_mat(ws->mttkrp_buf);
    free_mat(ws->auxil);
    free_mat(ws->mat_init);
    DestroySparseTensor(t_batch);
    if (slice_seconds) slice_seconds[s] = omp_get_wtime() - w0;
  }

  if (M) {
    for (int m = 0; m < nmodes; ++m) {
      if (m == stream_mode)
        memcpy(out_U[m], global_time->mat()->vals, sizeof(double) * (size_t)it * rank);
      else
        memcpy(out_U[m], M->U[m], sizeof(double) * M->dims[m] * rank);
    }
    memcpy(out_lambda, M->lambda, sizeof(double) * rank);
    for (int i = 0; i < nmodes; ++i) free_mat(grams[i]);
    free(grams);
    DestroyKruskalModel(M);
    DestroyKruskalModel(prev_M);
  }
  if (AT) destroy_alto(AT);
  if (scpgrams) DeleteSparseCPGrams(scpgrams, nmodes);
  delete global_time;
  free(ws);
  free_constraint(con);
  return it;
}

int ref_cpstream(int nmodes, int stream_mode, int nbatch, const uint64_t* batch_dims,
                 const uint64_t* batch_nnz, const uint64_t* cidx, const double* vals, int rank,
                 int max_iters, double epsilon, int nonneg, const double* init_vals,
                 uint64_t n_init_vals, double** out_U, double* out_lambda,
                 double* slice_seconds) {
  return run_stream(nmodes, stream_mode, nbatch, batch_dims, batch_nnz, cidx, vals, rank, max_iters, epsilon,
                    nonneg, init_vals, n_init_vals, out_U, out_lambda, slice_seconds, false);
}

// spcpstream (cpstream with use_spcpstream, src/streaming_cpd.cpp:26-366,
// each batch through spcpstream_alto_iter :466-1085); the constraint is
// not used by the reference on this path.
int ref_spcpstream(int nmodes, int stream_mode, int nbatch, const uint64_t* batch_dims,
                   const uint64_t* batch_nnz, const uint64_t* cidx, const double* vals, int rank,
                   int max_iters, double epsilon, const double* init_vals, uint64_t n_init_vals,
                   double** out_U, double* out_lambda, double* slice_seconds) {
  return run_stream(nmodes, stream_mode, nbatch, batch_dims, batch_nnz, cidx, vals, rank, max_iters, epsilon, 0,
                    init_vals, n_init_vals, out_U, out_lambda, slice_seconds, true);
}

// The reference's stream slicer (StreamingSparseTensor,
// src/streaming_sptensor.cpp:69-264): sorts the tensor (tt_sort by the
// stream mode, then the following modes cyclically), relabels every other
// mode in first-seen order and cuts batches with next_dynamic_batch.  The
// batches are written one after another: per batch its nmodes dims, then
// its nmodes x nnz indices and nnz values into the flat outputs; batch_nnz
// gets the sizes.  Returns the batch count (at most max_batches).
int ref_slice_stream(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* cidx, const double* vals,
                     int stream_mode, uint64_t nnz_threshold, uint64_t timeslice_limit, int max_batches,
                     uint64_t* batch_dims, uint64_t* batch_nnz, uint64_t* out_cidx, double* out_vals) {
  SparseTensor* X = make_coo(nmodes, dims, nnz, cidx, vals);
  int nb = 0;
  {
    StreamingSparseTensor sst(X, stream_mode);
    size_t off_i = 0, off_v = 0;
    while (!sst.last_batch() && nb < max_batches) {
      SparseTensor* b = sst.next_dynamic_batch(nnz_threshold, timeslice_limit);
      if (!b) break;
      for (int m = 0; m < nmodes; ++m) batch_dims[(size_t)nb * nmodes + m] = b->dims[m];
      batch_nnz[nb] = b->nnz;
      for (int m = 0; m < nmodes; ++m)
        for (IType q = 0; q < b->nnz; ++q) out_cidx[off_i + (size_t)m * b->nnz + q] = b->cidx[m][q];
      for (IType q = 0; q < b->nnz; ++q) out_vals[off_v + q] = b->vals[q];
      off_i += (size_t)nmodes * b->nnz;
      off_v += b->nnz;
      DestroySparseTensor(b);
      ++nb;
    }
  }
  DestroySparseTensor(X);
  return nb;
}

// cpd_error (src/streaming_cpd.cpp:368-464) of a model whose factors
// (factors[m]: dims[m] x rank, row-major) are given, against a COO tensor.
double ref_cpd_error(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* cidx, const double* vals,
                     double** factors, int rank) {
  SparseTensor* X = make_coo(nmodes, dims, nnz, cidx, vals);
  KruskalModel* M = nullptr;
  CreateKruskalModel(nmodes, X->dims, rank, &M);
  for (int m = 0; m < nmodes; ++m) memcpy(M->U[m], factors[m], dims[m] * rank * sizeof(FType));
  for (int r = 0; r < rank; ++r) M->lambda[r] = 1.0;
  const double e = cpd_error(X, M);
  DestroyKruskalModel(M);
  DestroySparseTensor(X);
  return e;
}

// ImportSparseTensor (src/sptensor.cpp:160-249): shape of the file's tensor.
// Returns 0, or -1 when the file cannot be opened (the reference asserts).
int ref_import_info(const char* path, int format, uint64_t zero_based, uint64_t* nmodes, uint64_t* dims,
                    uint64_t* nnz) {
  FILE* f = fopen(path, "r");
  if (!f) return -1;
  fclose(f);
  SparseTensor* X = nullptr;
  ImportSparseTensor(path, format == 1 ? BINARY_FORMAT : TEXT_FORMAT, &X, zero_based);
  *nmodes = X->nmodes;
  for (IType m = 0; m < X->nmodes; ++m) dims[m] = X->dims[m];
  *nnz = X->nnz;
  DestroySparseTensor(X);
  return 0;
}

// The same import's indices ([nmodes][nnz]) and values.
int ref_import_data(const char* path, int format, uint64_t zero_based, uint64_t* cidx, double* vals) {
  SparseTensor* X = nullptr;
  ImportSparseTensor(path, format == 1 ? BINARY_FORMAT : TEXT_FORMAT, &X, zero_based);
  for (IType m = 0; m < X->nmodes; ++m) memcpy(cidx + m * X->nnz, X->cidx[m], X->nnz * sizeof(IType));
  memcpy(vals, X->vals, X->nnz * sizeof(FType));
  DestroySparseTensor(X);
  return 0;
}

// ExportSparseTensor (src/sptensor.cpp:22-72) of a COO tensor to `path`.
void ref_export(const char* path, int format, int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* cidx,
                const double* vals) {
  SparseTensor* X = make_coo(nmodes, dims, nnz, cidx, vals);
  ExportSparseTensor(path, format == 1 ? BINARY_FORMAT : TEXT_FORMAT, X);
  DestroySparseTensor(X);
}

}  // extern "C"
