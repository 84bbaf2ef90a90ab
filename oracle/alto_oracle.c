/* ALTO oracle: a plain-C, single-threaded, FP64 restatement of the reference
 * algorithm for the hot path (jeewhanchoi/ALTO-stream).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle the CUDA path is
 * compared against; only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg load it (through oracle/oracle.py).  The product library
 * never links it and has no CPU fallback.
 *
 * Pinned against the compiled reference (oracle/_ref, built by
 * oracle/ref/Makefile) and the reference's fixture tensors
 * (tests/golden/, made by tests/golden/make_golden.py).
 *
 * Every function names the reference lines it restates.  Keys are 128-bit
 * (unsigned __int128); a 64-bit reference build produces the same values in
 * the low word, since masks never set bits at or above alto_bits.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

/* ------------------------------------------------------------------ bits */

/* Bits needed for indices 0..dim-1: 64 - clz(dim-1), with clz(0) = 64 as the
 * LZCNT instruction gives (include/alto.hpp:971, include/bitops.hpp:55-57),
 * so a mode of length 1 takes no bits. */
static int mode_bits(uint64_t dim) {
  if (dim <= 1) return 0;
  return 64 - __builtin_clzll(dim - 1);
}

/* Scatter the low bits of x into the set bits of mask (BMI2 PDEP semantics,
 * include/bitops.hpp:9-10, 60-69). */
static u128 deposit(uint64_t x, u128 mask) {
  u128 r = 0;
  int k = 0;
  for (int b = 0; b < 128; ++b) {
    if ((mask >> b) & 1) {
      if ((x >> k) & 1) r |= (u128)1 << b;
      ++k;
      if (k >= 64) break;
    }
  }
  return r;
}

/* Gather the bits of x selected by mask into the low bits (BMI2 PEXT
 * semantics, include/bitops.hpp:13-14, 71-79). */
static uint64_t extract(u128 x, u128 mask) {
  uint64_t r = 0;
  int k = 0;
  for (int b = 0; b < 128 && mask; ++b) {
    if ((mask >> b) & 1) {
      if ((x >> b) & 1) r |= (uint64_t)1 << k;
      ++k;
      mask &= ~((u128)1 << b);
    }
  }
  return r;
}

/* setup_packed_alto(LSB_FIRST, SHORT_FIRST), include/alto.hpp:955-1057.
 * Modes are ordered by bit count ascending; ties keep the mode order (the
 * reference's std::sort on <= 16 elements is an insertion sort, hence
 * stable).  Then bits are dealt LSB first, one per still-active mode per
 * level.  mode_pos receives the ALT_PEXT field offsets (prefix sums of the
 * bit counts in mode order, include/alto.hpp:982-988).  Returns the total
 * bits, or -1 if they exceed max_bits. */
int ora_setup_masks(int nmodes, const uint64_t* dims, int max_bits, uint64_t* masks_lohi,
                    uint64_t* alto_mask_lohi, int* mode_pos) {
  int bits[8], order[8], total = 0;
  u128 masks[8];
  for (int n = 0; n < nmodes; ++n) {
    bits[n] = mode_bits(dims[n]);
    order[n] = n;
    total += bits[n];
    masks[n] = 0;
  }
  if (total > max_bits) return -1;
  for (int i = 1; i < nmodes; ++i) { /* stable insertion sort by bits */
    int o = order[i], j = i - 1;
    while (j >= 0 && bits[order[j]] > bits[o]) {
      order[j + 1] = order[j];
      --j;
    }
    order[j + 1] = o;
  }
  int shift = 0;
  for (int level = 0;; ++level) {
    int any = 0;
    for (int k = 0; k < nmodes; ++k) {
      int n = order[k];
      if (level < bits[n]) {
        masks[n] |= (u128)1 << shift;
        ++shift;
        any = 1;
      }
    }
    if (!any) break;
  }
  u128 all = 0;
  for (int n = 0; n < nmodes; ++n) {
    all |= masks[n];
    if (masks_lohi) {
      masks_lohi[2 * n] = (uint64_t)masks[n];
      masks_lohi[2 * n + 1] = (uint64_t)(masks[n] >> 64);
    }
  }
  if (alto_mask_lohi) {
    alto_mask_lohi[0] = (uint64_t)all;
    alto_mask_lohi[1] = (uint64_t)(all >> 64);
  }
  if (mode_pos) {
    mode_pos[0] = 0;
    for (int n = 1; n < nmodes; ++n) mode_pos[n] = mode_pos[n - 1] + bits[n - 1];
  }
  return total;
}

static u128 load_key(const uint64_t* lohi, uint64_t i) {
  return ((u128)lohi[2 * i + 1] << 64) | lohi[2 * i];
}

static void load_masks(int nmodes, const uint64_t* masks_lohi, u128* masks) {
  for (int n = 0; n < nmodes; ++n) masks[n] = load_key(masks_lohi, n);
}

/* ------------------------------------------------------------- encoding */

typedef struct {
  u128 key;
  double val;
  uint64_t pos;
} KeyRec;

static int cmp_key(const void* a, const void* b) {
  u128 x = ((const KeyRec*)a)->key, y = ((const KeyRec*)b)->key;
  return (x > y) - (x < y);
}

/* prtn_alto, include/alto.hpp:1128-1226: equal-nnz partitions
 * prtn_ptr[p+1] = min((p+1) * ceil(nnz/P), nnz), and per partition per mode
 * the [min, max] decoded index (dims[n] / 0 sentinels; an empty partition
 * reports start = stop = 0). */
void ora_partition(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* idx_lohi,
                   const uint64_t* masks_lohi, int nprtn, uint64_t* prtn_ptr,
                   uint64_t* intervals) {
  u128 masks[8];
  load_masks(nmodes, masks_lohi, masks);
  uint64_t per = (nnz + nprtn - 1) / nprtn;
  prtn_ptr[0] = 0;
  for (int p = 0; p < nprtn; ++p) {
    uint64_t s = (uint64_t)p * per, e = (uint64_t)(p + 1) * per;
    if (e > nnz) e = nnz;
    if (s > e) s = e;
    prtn_ptr[p + 1] = e;
    for (int n = 0; n < nmodes; ++n) {
      uint64_t lo = dims[n], hi = 0;
      for (uint64_t i = s; i < e; ++i) {
        uint64_t v = extract(load_key(idx_lohi, i), masks[n]);
        if (v < lo) lo = v;
        if (v > hi) hi = v;
      }
      if (lo > hi) lo = hi;
      intervals[2 * ((size_t)p * nmodes + n)] = lo;
      intervals[2 * ((size_t)p * nmodes + n) + 1] = hi;
    }
  }
}

/* create_alto / update_salto, include/alto.hpp:436-582 and 195-299:
 * linearise every nonzero (OR over modes of PDEP(index, mask)), sort the
 * {key, value} pairs by key (include/alto.hpp:1066-1090; keys are unique for
 * unique coordinates so the order is total), then partition.  perm (may be
 * NULL) receives, for each sorted position, the input position it came from.
 * Returns the total key bits or -1 when they exceed max_bits. */
int ora_alto_build(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* cidx,
                   const double* vals, int max_bits, int nprtn, uint64_t* masks_lohi,
                   uint64_t* alto_mask_lohi, uint64_t* idx_lohi, double* vals_out,
                   uint64_t* perm, uint64_t* prtn_ptr, uint64_t* intervals) {
  int total = ora_setup_masks(nmodes, dims, max_bits, masks_lohi, alto_mask_lohi, NULL);
  if (total < 0) return -1;
  u128 masks[8];
  load_masks(nmodes, masks_lohi, masks);
  KeyRec* rec = (KeyRec*)malloc(sizeof(KeyRec) * (nnz ? nnz : 1));
  for (uint64_t i = 0; i < nnz; ++i) {
    u128 k = 0;
    for (int n = 0; n < nmodes; ++n) k |= deposit(cidx[(size_t)n * nnz + i], masks[n]);
    rec[i].key = k;
    rec[i].val = vals[i];
    rec[i].pos = i;
  }
  qsort(rec, nnz, sizeof(KeyRec), cmp_key);
  for (uint64_t i = 0; i < nnz; ++i) {
    idx_lohi[2 * i] = (uint64_t)rec[i].key;
    idx_lohi[2 * i + 1] = (uint64_t)(rec[i].key >> 64);
    if (vals_out) vals_out[i] = rec[i].val;
    if (perm) perm[i] = rec[i].pos;
  }
  free(rec);
  if (prtn_ptr && nprtn > 0)
    ora_partition(nmodes, dims, nnz, idx_lohi, masks_lohi, nprtn, prtn_ptr, intervals);
  return total;
}

/* Decode every nonzero's mode indices (PEXT per mode). */
void ora_decode(int nmodes, uint64_t nnz, const uint64_t* idx_lohi, const uint64_t* masks_lohi,
                uint64_t* cidx_out) {
  u128 masks[8];
  load_masks(nmodes, masks_lohi, masks);
  for (uint64_t i = 0; i < nnz; ++i) {
    u128 k = load_key(idx_lohi, i);
    for (int n = 0; n < nmodes; ++n) cidx_out[(size_t)n * nnz + i] = extract(k, masks[n]);
  }
}

/* --------------------------------------------------------------- MTTKRP */

/* Sequential ALTO MTTKRP, include/alto.hpp:739-824: for every nonzero in
 * line order, row = val * prod_{m != mode} U_m[i_m, :], accumulated into
 * factors[mode] (the caller zeroes it first, as the drivers do). */
void ora_mttkrp(int nmodes, uint64_t nnz, const uint64_t* idx_lohi, const double* vals,
                const uint64_t* masks_lohi, int mode, double** factors, int rank) {
  u128 masks[8];
  load_masks(nmodes, masks_lohi, masks);
  double* row = (double*)malloc(sizeof(double) * rank);
  for (uint64_t i = 0; i < nnz; ++i) {
    u128 k = load_key(idx_lohi, i);
    for (int r = 0; r < rank; ++r) row[r] = vals[i];
    for (int m = 0; m < nmodes; ++m) {
      if (m == mode) continue;
      const double* u = factors[m] + extract(k, masks[m]) * (uint64_t)rank;
      for (int r = 0; r < rank; ++r) row[r] *= u[r];
    }
    double* out = factors[mode] + extract(k, masks[mode]) * (uint64_t)rank;
    for (int r = 0; r < rank; ++r) out[r] += row[r];
  }
  free(row);
}

/* Sequential COO MTTKRP, src/mttkrp.cpp:122-156. */
void ora_coo_mttkrp(int nmodes, uint64_t nnz, const uint64_t* cidx, const double* vals, int mode,
                    double** factors, int rank) {
  double* row = (double*)malloc(sizeof(double) * rank);
  for (uint64_t i = 0; i < nnz; ++i) {
    for (int r = 0; r < rank; ++r) row[r] = vals[i];
    for (int m = 0; m < nmodes; ++m) {
      if (m == mode) continue;
      const double* u = factors[m] + cidx[(size_t)m * nnz + i] * (uint64_t)rank;
      for (int r = 0; r < rank; ++r) row[r] *= u[r];
    }
    double* out = factors[mode] + cidx[(size_t)mode * nnz + i] * (uint64_t)rank;
    for (int r = 0; r < rank; ++r) out[r] += row[r];
  }
  free(row);
}

/* ------------------------------------------------------- dense R x R kit */

/* Gram G = U^T U (rank x rank, full symmetric).  The reference stores only
 * the row-major upper triangle (cblas_dsyrk Upper, src/gram.cpp:29-41); the
 * callers below read only that triangle except where noted. */
static void gram(const double* U, uint64_t I, int R, double* G) {
  memset(G, 0, sizeof(double) * R * R);
  for (uint64_t i = 0; i < I; ++i) {
    const double* u = U + i * R;
    for (int a = 0; a < R; ++a)
      for (int b = a; b < R; ++b) G[a * R + b] += u[a] * u[b];
  }
  for (int a = 0; a < R; ++a)
    for (int b = 0; b < a; ++b) G[a * R + b] = G[b * R + a];
}

/* In-place Cholesky V = L L^T of a symmetric positive definite matrix, read
 * from its upper triangle (LAPACK dpotrf 'L' on the column-major view of a
 * row-major matrix, as every reference call does).  On return L is stored
 * row-major in the lower triangle.  Returns 0, or k+1 if the leading minor of
 * order k+1 is not positive (LAPACK's info). */
static int cholesky(double* A, int R) {
  for (int j = 0; j < R; ++j) {
    double d = A[j * R + j];
    for (int k = 0; k < j; ++k) d -= A[j * R + k] * A[j * R + k];
    if (!(d > 0.0)) return j + 1;
    d = sqrt(d);
    A[j * R + j] = d;
    for (int i = j + 1; i < R; ++i) {
      double s = A[j * R + i]; /* upper triangle holds the input */
      for (int k = 0; k < j; ++k) s -= A[i * R + k] * A[j * R + k];
      A[i * R + j] = s / d;
    }
  }
  return 0;
}

/* Solve (L L^T) x = b for each of nrows row vectors b (LAPACK dpotrs). */
static void cholesky_solve(const double* L, int R, double* B, uint64_t nrows) {
  for (uint64_t q = 0; q < nrows; ++q) {
    double* x = B + q * R;
    for (int i = 0; i < R; ++i) {
      double s = x[i];
      for (int k = 0; k < i; ++k) s -= L[i * R + k] * x[k];
      x[i] = s / L[i * R + i];
    }
    for (int i = R - 1; i >= 0; --i) {
      double s = x[i];
      for (int k = i + 1; k < R; ++k) s -= L[k * R + i] * x[k];
      x[i] = s / L[i * R + i];
    }
  }
}

/* Column normalisation, src/kruskal_model.cpp:227-353 (KruskalModelNorm).
 * which 0: lambda_r = sqrt(max(sum_i U_ir^2, 1e-12)); which 1:
 * lambda_r = max(1, max_i U_ir) (signed max).  U /= lambda. */
static void normalize_cols(double* U, uint64_t I, int R, int which, double* lambda) {
  for (int r = 0; r < R; ++r) lambda[r] = which == 0 ? 0.0 : 1.0;
  for (uint64_t i = 0; i < I; ++i)
    for (int r = 0; r < R; ++r) {
      double v = U[i * R + r];
      if (which == 0)
        lambda[r] += v * v;
      else if (v > lambda[r])
        lambda[r] = v;
    }
  if (which == 0)
    for (int r = 0; r < R; ++r) lambda[r] = sqrt(lambda[r] > 1e-12 ? lambda[r] : 1e-12);
  for (uint64_t i = 0; i < I; ++i)
    for (int r = 0; r < R; ++r) U[i * R + r] /= lambda[r];
}

/* --------------------------------------------------------------- CP-ALS */

/* CP-ALS on the ALTO tensor, include/cpd.hpp:47-191, single threaded.
 * U[n] (dims[n] x rank) and lambda hold the initial model on entry and the
 * result on exit; fits[i] receives the residual that cpd_fit_alto reports
 * after iteration i.  fit_exact 0 reproduces the reference's fit, whose
 * model norm keeps only the diagonal of the Gram Hadamard product (its Gram
 * lower triangles stay zero, include/cpd.hpp:228-256); 1 uses the full
 * product.  Returns iterations run, or -(n+1) if the rank-deficient fallback
 * for mode n would be needed and could not run. */
int ora_cpd_als(int nmodes, const uint64_t* dims, uint64_t nnz, const uint64_t* idx_lohi,
                const double* vals, const uint64_t* masks_lohi, double** U, double* lambda,
                int rank, int max_iters, double epsilon, int fit_exact, double* fits) {
  int R = rank;
  double* G[8];
  for (int n = 0; n < nmodes; ++n) {
    G[n] = (double*)malloc(sizeof(double) * R * R);
    gram(U[n], dims[n], R, G[n]);
  }
  double* V = (double*)malloc(sizeof(double) * R * R);
  uint64_t Ilast = dims[nmodes - 1];
  double* scratch = (double*)malloc(sizeof(double) * Ilast * R);
  double normX = 0.0;
  for (uint64_t i = 0; i < nnz; ++i) normX += vals[i] * vals[i];

  double fit = 0.0, prev_fit = 0.0;
  int iters = max_iters;
  for (int it = 0; it < max_iters; ++it) {
    for (int j = 0; j < nmodes; ++j) {
      memset(U[j], 0, sizeof(double) * dims[j] * R);
      ora_mttkrp(nmodes, nnz, idx_lohi, vals, masks_lohi, j, U, R);
      if (j == nmodes - 1) memcpy(scratch, U[j], sizeof(double) * Ilast * R);
      /* pseudo_inverse, include/cpd.hpp:377-480 */
      for (int q = 0; q < R * R; ++q) V[q] = 1.0;
      for (int m = 0; m < nmodes; ++m)
        if (m != j)
          for (int q = 0; q < R * R; ++q) V[q] *= G[m][q];
      for (int r = 0; r < R; ++r) V[r * R + r] += 1e-3;
      if (cholesky(V, R) == 0) {
        cholesky_solve(V, R, U[j], dims[j]);
      } else {
        /* dgelsy fallback (include/cpd.hpp:436-476): the reference first
         * restores V without the ridge and mirrors its row-major lower
         * triangle, which is zero there, into the upper one; the system it
         * solves is therefore diag(V) X = B (minimum norm for zero pivots). */
        for (int r = 0; r < R; ++r) {
          double d = 1.0;
          for (int m = 0; m < nmodes; ++m)
            if (m != j) d *= G[m][r * R + r];
          for (uint64_t i = 0; i < dims[j]; ++i) U[j][i * R + r] = d != 0.0 ? U[j][i * R + r] / d : 0.0;
        }
      }
      normalize_cols(U[j], dims[j], R, it == 0 ? 0 : 1, lambda);
      gram(U[j], dims[j], R, G[j]);
    }
    /* cpd_fit_alto, include/cpd.hpp:193-275 */
    double inner = 0.0;
    for (int r = 0; r < R; ++r) {
      double acc = 0.0;
      for (uint64_t i = 0; i < Ilast; ++i) acc += U[nmodes - 1][i * R + r] * scratch[i * R + r];
      inner += acc * lambda[r];
    }
    double normU = 0.0;
    for (int a = 0; a < R; ++a)
      for (int b = 0; b <= a; ++b) {
        if (!fit_exact && b != a) continue;
        double t = lambda[a] * lambda[b];
        for (int m = 0; m < nmodes; ++m) t *= G[m][a * R + b];
        normU += (b == a) ? t : 2.0 * t;
      }
    normU = fabs(normU);
    double res = normX + normU - 2.0 * inner;
    if (res > 0.0) res = sqrt(res);
    fit = res / sqrt(normX);
    if (fits) fits[it] = fit;
    if (it > 0 && fabs(prev_fit - fit) < epsilon) {
      iters = it + 1;
      break;
    }
    prev_fit = fit;
  }
  for (int n = 0; n < nmodes; ++n) free(G[n]);
  free(V);
  free(scratch);
  return iters;
}

/* ------------------------------------------------------------ CP-stream */

typedef struct {
  const double* v;
  uint64_t n, pos;
} Stream;

static double next_val(Stream* s) { return s->pos < s->n ? s->v[s->pos++] : 0.0; }

/* admm_cf_ (src/admm.cpp:216-429) for one factor, single threaded.
 * mttkrp holds the right-hand side (I x R), primal the factor (I x R, updated
 * in place), dual the persistent dual (I x R), Phi the Hadamard product of the
 * other modes' Grams.  Unconstrained: Phi + 1e-12 I, Cholesky solve.
 * Constrained (non-negativity, the only projection the reference applies):
 * rho = tr(Phi)/R, Cholesky of Phi + rho I, a first primal update, then up to
 * 25 sweeps with the global residual test at tolerance (double)1e-6f.
 * Returns sweeps run (0 unconstrained), or -1 if the factorisation fails. */
static int admm_cf(double* Phi, int R, const double* mttkrp, double* primal, double* dual,
                   uint64_t I, int nonneg) {
  if (!nonneg) {
    for (int r = 0; r < R; ++r) Phi[r * R + r] += 1e-12;
    if (cholesky(Phi, R) != 0) return -1; /* reference prints and keeps the MTTKRP */
    memcpy(primal, mttkrp, sizeof(double) * I * R);
    cholesky_solve(Phi, R, primal, I);
    return 0;
  }
  double rho = 0.0;
  for (int r = 0; r < R; ++r) rho += Phi[r * R + r];
  rho /= (double)R;
  for (int r = 0; r < R; ++r) Phi[r * R + r] += rho;
  if (cholesky(Phi, R) != 0) return -1; /* reference exits */
  uint64_t N = I * (uint64_t)R;
  double* aux = (double*)malloc(sizeof(double) * (N ? N : 1));
  double* init = (double*)malloc(sizeof(double) * (N ? N : 1));
  for (uint64_t q = 0; q < N; ++q) aux[q] = mttkrp[q] + rho * (primal[q] + dual[q]);
  cholesky_solve(Phi, R, aux, I);
  for (uint64_t q = 0; q < N; ++q) {
    init[q] = primal[q];
    double x = aux[q] - dual[q];
    primal[q] = x < 0.0 ? 0.0 : x;
  }
  const double tol = (double)1e-6f;
  int it;
  for (it = 0; it < 25; ++it) {
    double p_res = 0, d_res = 0, p_norm = 0, d_norm = 0;
    for (uint64_t q = 0; q < N; ++q) {
      double x = primal[q];
      double dd = x - init[q];
      d_res += dd * dd;
      p_norm += x * x;
      double y = x - aux[q];
      double di = dual[q] + y;
      dual[q] = di;
      d_norm += di * di;
      p_res += y * y;
      aux[q] = mttkrp[q] + rho * (x + di);
    }
    cholesky_solve(Phi, R, aux, I);
    for (uint64_t q = 0; q < N; ++q) {
      double x = aux[q] - dual[q];
      x = x > 0.0 ? x : 0.0;
      init[q] = x;
      primal[q] = x;
    }
    if (p_res <= tol * p_norm && d_res <= tol * d_norm) {
      ++it;
      break;
    }
  }
  free(aux);
  free(init);
  return it;
}

/* CP-stream (ALTO), single threaded: the batch loop of cpstream
 * (src/streaming_cpd.cpp:26-366) around cpstream_alto_iter
 * (src/streaming_cpd.cpp:1198-1519).  Arguments as ref_cpstream in
 * oracle/ref/ref_harness.cpp, plus `forgetting` (the reference hard-codes
 * 0.99, src/streaming_cpd.cpp:18) and `inner_iters` (may be NULL: inner
 * iterations run per batch).  Returns the total time steps, or -1 when a
 * factorisation fails. */
int ora_cpstream(int nmodes, int stream_mode, int nbatch, const uint64_t* batch_dims,
                 const uint64_t* batch_nnz, const uint64_t* cidx, const double* vals, int rank,
                 int max_iters, double epsilon, int nonneg, double forgetting,
                 const double* init_vals, uint64_t n_init_vals, double** out_U,
                 double* out_lambda, int* inner_iters) {
  const int R = rank, t = stream_mode;
  Stream st = {init_vals, n_init_vals, 0};
  uint64_t dims[8] = {0}, old_dims[8] = {0};
  double *U[8] = {0}, *P[8] = {0}, *G[8], *dual[8] = {0};
  for (int n = 0; n < nmodes; ++n) {
    G[n] = (double*)calloc(R * R, sizeof(double));
  }
  double* lambda = out_lambda;
  double* Phi = (double*)malloc(sizeof(double) * R * R);
  double* old_gram = (double*)malloc(sizeof(double) * R * R);
  double* ata = (double*)malloc(sizeof(double) * R * R);
  double* hist = (double*)malloc(sizeof(double) * R * R);
  double* time_rows = NULL;
  uint64_t total_time = 0;
  size_t off_idx = 0, off_val = 0;
  int status = 0;

  for (int s = 0; s < nbatch && status == 0; ++s) {
    const uint64_t* bd = batch_dims + (size_t)s * nmodes;
    uint64_t nnz = batch_nnz[s];
    const uint64_t* bc = cidx + off_idx;
    const double* bv = vals + off_val;
    off_idx += (size_t)nmodes * nnz;
    off_val += nnz;
    for (int n = 0; n < nmodes; ++n) {
      old_dims[n] = dims[n];
      dims[n] = bd[n];
      U[n] = (double*)realloc(U[n], sizeof(double) * (dims[n] ? dims[n] : 1) * R);
      P[n] = (double*)realloc(P[n], sizeof(double) * (dims[n] ? dims[n] : 1) * R);
      for (uint64_t q = old_dims[n] * R; q < dims[n] * R; ++q) {
        U[n][q] = next_val(&st); /* KruskalModelRandomInit / GrowKruskalModel(FILL_RANDOM) */
        P[n][q] = 0.0;           /* prev model grows with zeros */
      }
    }
    if (s == 0) {
      for (int r = 0; r < R; ++r) lambda[r] = 1.0;
      memset(U[t], 0, sizeof(double) * dims[t] * R);
      for (int n = 0; n < nmodes; ++n)
        if (n != t) gram(U[n], dims[n], R, G[n]);
      memset(G[t], 0, sizeof(double) * R * R);
    } else {
      for (int n = 0; n < nmodes; ++n)
        if (n != t) gram(U[n], dims[n], R, G[n]);
    }
    uint64_t max_dim = 0;
    for (int n = 0; n < nmodes; ++n) {
      free(dual[n]);
      dual[n] = (double*)calloc((dims[n] ? dims[n] : 1) * R, sizeof(double));
      if (dims[n] > max_dim) max_dim = dims[n];
    }
    double* buf = (double*)calloc(max_dim * R, sizeof(double));

    /* update_salto: encode and sort this batch (the MTTKRP below visits the
     * nonzeros in line order). */
    uint64_t* idx = (uint64_t*)malloc(sizeof(uint64_t) * 2 * (nnz ? nnz : 1));
    double* sv = (double*)malloc(sizeof(double) * (nnz ? nnz : 1));
    uint64_t masks[16];
    ora_alto_build(nmodes, dims, nnz, bc, bv, 128, 0, masks, NULL, idx, sv, NULL, NULL, NULL);

    /* cpstream_alto_iter, src/streaming_cpd.cpp:1198-1519 */
    if (s == 0) {
      for (int m = 0; m < nmodes; ++m) {
        if (m == t) continue;
        normalize_cols(U[m], dims[m], R, 0, lambda);
        gram(U[m], dims[m], R, G[m]);
      }
      for (int r = 0; r < R; ++r) lambda[r] = 1.0;
    }
    double delta = 0.0, prev_delta = 0.0;
    int it;
    for (it = 0; it < max_iters; ++it) {
      delta = 0.0;
      memset(U[t], 0, sizeof(double) * dims[t] * R);
      ora_mttkrp(nmodes, nnz, idx, sv, masks, t, U, R);
      for (int q = 0; q < R * R; ++q) Phi[q] = 1.0;
      for (int m = 0; m < nmodes; ++m)
        if (m != t)
          for (int q = 0; q < R * R; ++q) Phi[q] *= G[m][q];
      for (int r = 0; r < R; ++r) Phi[r * R + r] += 1e-12;
      if (cholesky(Phi, R) == 0) cholesky_solve(Phi, R, U[t], dims[t]);
      /* copy_upper_tri keeps G_t symmetric; then G_t += sum_rows s s^T */
      memcpy(old_gram, G[t], sizeof(double) * R * R);
      for (uint64_t q = 0; q < dims[t]; ++q) {
        const double* sr = U[t] + q * R;
        for (int a = 0; a < R; ++a)
          for (int b = 0; b < R; ++b) G[t][a * R + b] += sr[b] * sr[a];
      }
      for (int j = 0; j < nmodes; ++j) {
        if (j == t) continue;
        memset(buf, 0, sizeof(double) * dims[j] * R);
        double* keep = U[j];
        U[j] = buf;
        ora_mttkrp(nmodes, nnz, idx, sv, masks, j, U, R);
        U[j] = keep;
        /* historical term, src/streaming_cpd.cpp:1375-1415 */
        memcpy(ata, old_gram, sizeof(double) * R * R);
        for (int m = 0; m < nmodes; ++m) {
          if (m == j || m == t) continue;
          memset(hist, 0, sizeof(double) * R * R);
          for (uint64_t i = 0; i < dims[m]; ++i)
            for (int a = 0; a < R; ++a)
              for (int b = 0; b < R; ++b) hist[a * R + b] += P[m][i * R + a] * U[m][i * R + b];
          for (int q = 0; q < R * R; ++q) ata[q] *= hist[q];
        }
        for (uint64_t i = 0; i < dims[j]; ++i)
          for (int b = 0; b < R; ++b) {
            double acc = 0.0;
            for (int a = 0; a < R; ++a) acc += P[j][i * R + a] * ata[a * R + b];
            buf[i * R + b] += acc;
          }
        /* admm_cf with Phi = Hadamard of every Gram but mode j */
        for (int q = 0; q < R * R; ++q) Phi[q] = 1.0;
        for (int m = 0; m < nmodes; ++m)
          if (m != j)
            for (int q = 0; q < R * R; ++q) Phi[q] *= G[m][q];
        if (admm_cf(Phi, R, buf, U[j], dual[j], dims[j], nonneg) < 0) {
          status = -1;
          break;
        }
        gram(U[j], dims[j], R, G[j]);
        double nd = 0.0, nu = 0.0;
        for (uint64_t q = 0; q < dims[j] * R; ++q) {
          double d = P[j][q] - U[j][q];
          nd += d * d;
          nu += U[j][q] * U[j][q];
        }
        delta += sqrt(nd) / (sqrt(nu) + 1e-12);
      }
      if (status) break;
      if (it > 0 && fabs(prev_delta - delta) < epsilon) {
        ++it;
        break;
      }
      prev_delta = delta;
    }
    if (inner_iters) inner_iters[s] = it;
    for (int q = 0; q < R * R; ++q) G[t][q] *= forgetting;

    /* prev_M <- M; append the time rows */
    for (int n = 0; n < nmodes; ++n) memcpy(P[n], U[n], sizeof(double) * dims[n] * R);
    time_rows = (double*)realloc(time_rows, sizeof(double) * (total_time + dims[t]) * R);
    memcpy(time_rows + total_time * R, U[t], sizeof(double) * dims[t] * R);
    total_time += dims[t];
    free(buf);
    free(idx);
    free(sv);
  }
  if (status == 0) {
    for (int n = 0; n < nmodes; ++n) {
      if (n == t)
        memcpy(out_U[n], time_rows, sizeof(double) * total_time * R);
      else
        memcpy(out_U[n], U[n], sizeof(double) * dims[n] * R);
    }
  }
  for (int n = 0; n < nmodes; ++n) {
    free(U[n]);
    free(P[n]);
    free(G[n]);
    free(dual[n]);
  }
  free(Phi);
  free(old_gram);
  free(ata);
  free(hist);
  free(time_rows);
  return status == 0 ? (int)total_time : -1;
}

/* ------------------------------------------------------------ spCP-stream */

/* C = A^T B over the rows listed in `rows` (or all I rows when rows is
 * NULL) of row-major I x R matrices (full R x R result). */
static void rows_atb(const double* A, const double* B, const uint64_t* rows, uint64_t n, int R, double* C) {
  memset(C, 0, sizeof(double) * R * R);
  for (uint64_t k = 0; k < n; ++k) {
    const uint64_t i = rows ? rows[k] : k;
    for (int a = 0; a < R; ++a)
      for (int b = 0; b < R; ++b) C[a * R + b] += A[i * R + a] * B[i * R + b];
  }
}

/* C = A B (R x R). */
static void mm(const double* A, const double* B, int R, double* C) {
  for (int a = 0; a < R; ++a)
    for (int b = 0; b < R; ++b) {
      double s = 0.0;
      for (int k = 0; k < R; ++k) s += A[a * R + k] * B[k * R + b];
      C[a * R + b] = s;
    }
}

/* pseudo_inverse (src/matrix.cpp:226-250): rows of B <- rows of B times
 * Phi^{-1} by Cholesky; on failure B is left as it is. */
static void solve_rows_keep(const double* Phi, int R, double* B, uint64_t nrows, double* work) {
  memcpy(work, Phi, sizeof(double) * R * R);
  if (cholesky(work, R) == 0) cholesky_solve(work, R, B, nrows);
}

static double trace(const double* A, int R) {
  double s = 0.0;
  for (int r = 0; r < R; ++r) s += A[r * R + r];
  return s;
}

/* spCP-stream: cpstream (src/streaming_cpd.cpp:26-366) with use_spcpstream,
 * each batch through spcpstream_alto_iter (:466-1085).  Per batch, for every
 * mode, the rows the batch touches (nonzero_slices, :1127-1161) are
 * gathered into compact factors A_nz (and A_nz_prev from the previous
 * model); the MTTKRPs run over the batch with its indices renumbered to
 * those rows (update_salto_rowsparse).  The Gram bookkeeping keeps, per
 * mode, c = U^T U and h = prev_U^T U split into the touched rows (c_nz,
 * h_nz) and the untouched rows (c_z, h_z, updated in closed form through
 * Q Phi^{-1}); after the inner loop the untouched rows become
 * prev_U Q Phi^{-1} and the touched rows A_nz.  The constraint is not used
 * (the reference solves with pseudo_inverse).  Initial and growth values as
 * in ora_cpstream; forgetting as there.  Returns the total time steps, or
 * -1 on failure. */
int ora_spcpstream(int nmodes, int stream_mode, int nbatch, const uint64_t* batch_dims,
                   const uint64_t* batch_nnz, const uint64_t* cidx, const double* vals, int rank,
                   int max_iters, double epsilon, double forgetting, const double* init_vals,
                   uint64_t n_init_vals, double** out_U, double* out_lambda, int* inner_iters) {
  const int R = rank, t = stream_mode, RR = rank * rank;
  Stream st = {init_vals, n_init_vals, 0};
  uint64_t dims[8] = {0}, old_dims[8] = {0};
  double *U[8] = {0}, *P[8] = {0}, *G[8];
  double *c[8], *h[8], *c_prev[8], *c_nz_prev[8], *c_nz[8], *c_z[8], *h_nz[8], *h_z[8], *c_z_prev[8], *QPi[8];
  double** all[] = {G, c, h, c_prev, c_nz_prev, c_nz, c_z, h_nz, h_z, c_z_prev, QPi};
  for (size_t k = 0; k < sizeof(all) / sizeof(all[0]); ++k)
    for (int n = 0; n < nmodes; ++n) all[k][n] = (double*)calloc(RR, sizeof(double));
  double* lambda = out_lambda;
  double* Phi = (double*)malloc(sizeof(double) * RR);
  double* Q = (double*)malloc(sizeof(double) * RR);
  double* work = (double*)malloc(sizeof(double) * RR);
  double* tmp = (double*)malloc(sizeof(double) * RR);
  double* old_gram = (double*)malloc(sizeof(double) * RR);
  double* time_rows = NULL;
  uint64_t total_time = 0;
  size_t off_idx = 0, off_val = 0;

  for (int s = 0; s < nbatch; ++s) {
    const uint64_t* bd = batch_dims + (size_t)s * nmodes;
    const uint64_t nnz = batch_nnz[s];
    const uint64_t* bc = cidx + off_idx;
    const double* bv = vals + off_val;
    off_idx += (size_t)nmodes * nnz;
    off_val += nnz;
    for (int n = 0; n < nmodes; ++n) {
      old_dims[n] = dims[n];
      dims[n] = bd[n];
      U[n] = (double*)realloc(U[n], sizeof(double) * (dims[n] ? dims[n] : 1) * R);
      P[n] = (double*)realloc(P[n], sizeof(double) * (dims[n] ? dims[n] : 1) * R);
      for (uint64_t q = old_dims[n] * R; q < dims[n] * R; ++q) {
        U[n][q] = next_val(&st);
        P[n][q] = 0.0;
      }
    }
    if (s == 0) {
      for (int r = 0; r < R; ++r) lambda[r] = 1.0;
      memset(U[t], 0, sizeof(double) * dims[t] * R);
      memset(G[t], 0, sizeof(double) * RR);
      /* iteration 0: 2-norm normalise the non-stream factors (:585-598) */
      for (int m = 0; m < nmodes; ++m) {
        if (m == t) continue;
        normalize_cols(U[m], dims[m], R, 0, lambda);
        gram(U[m], dims[m], R, G[m]);
      }
      for (int r = 0; r < R; ++r) lambda[r] = 1.0;
    }

    /* nonzero_slices for every mode: sorted touched rows and their map */
    uint64_t* nz[8];
    int64_t* ridx[8];
    uint64_t nnzr[8];
    for (int m = 0; m < nmodes; ++m) {
      ridx[m] = (int64_t*)malloc(sizeof(int64_t) * (dims[m] ? dims[m] : 1));
      for (uint64_t i = 0; i < dims[m]; ++i) ridx[m][i] = -1;
      for (uint64_t q = 0; q < nnz; ++q) ridx[m][bc[(size_t)m * nnz + q]] = 0;
      nnzr[m] = 0;
      for (uint64_t i = 0; i < dims[m]; ++i)
        if (ridx[m][i] == 0) ++nnzr[m];
      nz[m] = (uint64_t*)malloc(sizeof(uint64_t) * (nnzr[m] ? nnzr[m] : 1));
      uint64_t k = 0;
      for (uint64_t i = 0; i < dims[m]; ++i)
        if (ridx[m][i] == 0) {
          nz[m][k] = i;
          ridx[m][i] = (int64_t)k++;
        }
    }
    /* A_nz_prev, c = U^T U, h = prev_U^T U, A_nz (:614-676) */
    double *Anz[8], *Aprev[8];
    for (int m = 0; m < nmodes; ++m) {
      Anz[m] = (double*)malloc(sizeof(double) * (nnzr[m] ? nnzr[m] : 1) * R);
      Aprev[m] = (double*)malloc(sizeof(double) * (nnzr[m] ? nnzr[m] : 1) * R);
      for (uint64_t k = 0; k < nnzr[m]; ++k)
        for (int r = 0; r < R; ++r) {
          Anz[m][k * R + r] = U[m][nz[m][k] * R + r];
          Aprev[m][k * R + r] = P[m][nz[m][k] * R + r];
        }
      rows_atb(U[m], U[m], NULL, dims[m], R, c[m]);
      rows_atb(P[m], U[m], NULL, dims[m], R, h[m]);
    }
    /* c_z_prev = c_prev - c_nz_prev over the touched rows (:679-693) */
    if (s > 0)
      for (int m = 0; m < nmodes; ++m) {
        if (m == t) continue;
        rows_atb(P[m], P[m], nz[m], nnzr[m], R, c_nz_prev[m]);
        for (int q = 0; q < RR; ++q) c_z_prev[m][q] = c_prev[m][q] - c_nz_prev[m][q];
      }
    /* the batch with its indices renumbered to the touched rows */
    uint64_t* cc = (uint64_t*)malloc(sizeof(uint64_t) * nmodes * (nnz ? nnz : 1));
    for (int m = 0; m < nmodes; ++m)
      for (uint64_t q = 0; q < nnz; ++q) cc[(size_t)m * nnz + q] = (uint64_t)ridx[m][bc[(size_t)m * nnz + q]];

    double delta = 0.0, prev_delta = 0.0;
    int it, done = 0;
    for (it = 0; it < max_iters; ++it) {
      delta = 0.0;
      /* s_t: MTTKRP of the stream mode, solve with Hadamard(c) but t (:716-744) */
      memset(Anz[t], 0, sizeof(double) * nnzr[t] * R);
      ora_coo_mttkrp(nmodes, nnz, cc, bv, t, Anz, R);
      for (int q = 0; q < RR; ++q) Phi[q] = 1.0;
      for (int m = 0; m < nmodes; ++m)
        if (m != t)
          for (int q = 0; q < RR; ++q) Phi[q] *= c[m][q];
      for (int r = 0; r < R; ++r) Phi[r * R + r] += 1e-12;
      solve_rows_keep(Phi, R, Anz[t], nnzr[t], work);
      /* G_t: old_gram, then += s s^T over the stream rows (:748-780) */
      memcpy(old_gram, G[t], sizeof(double) * RR);
      for (uint64_t q = 0; q < dims[t]; ++q) {
        const double* sr = Anz[t] + q * R;
        for (int a = 0; a < R; ++a)
          for (int b = 0; b < R; ++b) G[t][a * R + b] += sr[b] * sr[a];
      }
      memcpy(h[t], old_gram, sizeof(double) * RR);
      memcpy(c[t], G[t], sizeof(double) * RR);
      for (int m = 0; m < nmodes; ++m) {
        if (m == t) continue;
        /* Q = Hadamard(h) but m, Phi = Hadamard(c) but m + 1e-12 I (:800-806) */
        for (int q = 0; q < RR; ++q) Q[q] = Phi[q] = 1.0;
        for (int k = 0; k < nmodes; ++k)
          if (k != m)
            for (int q = 0; q < RR; ++q) {
              Q[q] *= h[k][q];
              Phi[q] *= c[k][q];
            }
        for (int r = 0; r < R; ++r) Phi[r * R + r] += 1e-12;
        /* row-sparse MTTKRP, historical term, solve (:826-892) */
        memset(Anz[m], 0, sizeof(double) * nnzr[m] * R);
        ora_coo_mttkrp(nmodes, nnz, cc, bv, m, Anz, R);
        for (uint64_t k = 0; k < nnzr[m]; ++k)
          for (int b = 0; b < R; ++b) {
            double acc = 0.0;
            for (int a = 0; a < R; ++a) acc += Aprev[m][k * R + a] * Q[a * R + b];
            Anz[m][k * R + b] += acc;
          }
        solve_rows_keep(Phi, R, Anz[m], nnzr[m], work);
        /* c_nz, h_nz; Q Phi^{-1}; h_z = c_z_prev Q Phi^{-1}; c_z = (Q Phi^{-1})^T h_z (:903-942) */
        rows_atb(Anz[m], Anz[m], NULL, nnzr[m], R, c_nz[m]);
        rows_atb(Aprev[m], Anz[m], NULL, nnzr[m], R, h_nz[m]);
        memcpy(QPi[m], Q, sizeof(double) * RR);
        solve_rows_keep(Phi, R, QPi[m], R, work);
        mm(c_z_prev[m], QPi[m], R, h_z[m]);
        for (int a = 0; a < R; ++a)
          for (int b = 0; b < R; ++b) {
            double sum = 0.0;
            for (int k = 0; k < R; ++k) sum += QPi[m][k * R + a] * h_z[m][k * R + b];
            tmp[a * R + b] = sum;
          }
        memcpy(c_z[m], tmp, sizeof(double) * RR);
        for (int q = 0; q < RR; ++q) {
          c[m][q] = c_nz[m][q] + c_z[m][q];
          h[m][q] = h_nz[m][q] + h_z[m][q];
        }
        const double trc = trace(c[m], R), trh = trace(h[m], R), trp = trace(c_prev[m], R);
        delta += sqrt(fabs((trc + trp - 2.0 * trh) / (trc + 1e-12)));
      }
      if (it > 0 && fabs(prev_delta - delta) < epsilon) {
        done = it + 1;
        break;
      }
      prev_delta = delta;
      done = it + 1;
    }
    if (inner_iters) inner_iters[s] = done;
    /* untouched rows <- prev rows Q Phi^{-1}; touched rows <- A_nz (:985-1024) */
    for (int m = 0; m < nmodes; ++m) {
      for (uint64_t i = 0; i < dims[m]; ++i) {
        if (ridx[m][i] >= 0) {
          memcpy(U[m] + i * R, Anz[m] + (uint64_t)ridx[m][i] * R, sizeof(double) * R);
        } else if (m != t) {
          for (int b = 0; b < R; ++b) {
            double acc = 0.0;
            for (int a = 0; a < R; ++a) acc += P[m][i * R + a] * QPi[m][a * R + b];
            U[m][i * R + b] = acc;
          }
        }
      }
    }
    for (int q = 0; q < RR; ++q) G[t][q] *= forgetting;
    for (int m = 0; m < nmodes; ++m) {
      if (m == t) continue;
      memcpy(c_prev[m], c[m], sizeof(double) * RR);
      memcpy(c_nz_prev[m], c_nz[m], sizeof(double) * RR);
    }
    for (int n = 0; n < nmodes; ++n) memcpy(P[n], U[n], sizeof(double) * dims[n] * R);
    time_rows = (double*)realloc(time_rows, sizeof(double) * (total_time + dims[t]) * R);
    memcpy(time_rows + total_time * R, U[t], sizeof(double) * dims[t] * R);
    total_time += dims[t];
    for (int m = 0; m < nmodes; ++m) {
      free(nz[m]);
      free(ridx[m]);
      free(Anz[m]);
      free(Aprev[m]);
    }
    free(cc);
  }
  for (int n = 0; n < nmodes; ++n) {
    if (n == t)
      memcpy(out_U[n], time_rows, sizeof(double) * total_time * R);
    else
      memcpy(out_U[n], U[n], sizeof(double) * dims[n] * R);
  }
  for (size_t k = 0; k < sizeof(all) / sizeof(all[0]); ++k)
    for (int n = 0; n < nmodes; ++n) free(all[k][n]);
  for (int n = 0; n < nmodes; ++n) {
    free(U[n]);
    free(P[n]);
  }
  free(Phi);
  free(Q);
  free(work);
  free(tmp);
  free(old_gram);
  free(time_rows);
  return (int)total_time;
}
