// Dense float64 helpers shared by CP-ALS and CP-stream (alto_dense.cu).
#pragma once

#include "alto_internal.cuh"

namespace alto {

// Solve set-up kinds.  On a failed Cholesky: kSolveRidge gives W = 0,
// kSolveRidgeDiagFallback the CP-ALS diagonal fallback, kSolveRidgeKeep
// W = I (the right-hand side stays as it is, as pseudo_inverse leaves it,
// src/matrix.cpp:226-250).
enum { kSolveRidge = 0, kSolveRidgeDiagFallback = 1, kSolveAdmm = 2, kSolveRidgeKeep = 3 };

// G = A^T A (R x R float64) of a float32 I x R matrix.
alto_status gram(const float* A, uint64_t I, int R, double* out, DevBuf& scratch, cudaStream_t st);
// G = A^T B.
alto_status cross_gram(const float* A, const float* B, uint64_t I, int R, double* out,
                       DevBuf& scratch, cudaStream_t st);
// One pass over P and U: G = U^T U, C = P^T U and stats3 = {sum p u,
// sum (p - u)^2, sum u^2} (stats3 may be NULL).
alto_status gram_cross_stats(const float* P, const float* U, uint64_t I, int R, double* G, double* C,
                             double* stats3, DevBuf& scratch, cudaStream_t st);
// W = (prod_{m in mask} grams[m] + shift I)^{-1}; see the kernel comment.
alto_status solve_setup(const double* grams, int nmodes, unsigned mask, int R, int kind,
                        double ridge, double* W, int* status, double* rho, cudaStream_t st);
// X = B W (+ C); apply_f32 also writes per-block column statistics
// (sum x^2, max x) when stats is given.
alto_status apply_f32(const float* B, const double* W, uint64_t I, int R, float* X,
                      DevBuf* stats, int* nblocks, cudaStream_t st);
alto_status apply_f64_to_f32(const double* B, const double* W, uint64_t I, int R, float* X,
                             cudaStream_t st);
alto_status apply_f32_to_f64(const float* B, const float* C, const double* W, uint64_t I, int R,
                             double* X, cudaStream_t st);
alto_status column_lambda(const double* stats, int nblocks, int R, int which, double* lambda,
                          cudaStream_t st);
alto_status scale_columns(float* X, uint64_t I, int R, const double* lambda, __nv_bfloat16* shadow,
                          cudaStream_t st);
alto_status to_bf16(const float* X, uint64_t n, __nv_bfloat16* Y, cudaStream_t st);
// out3 = {sum a*b*colw, sum (a-b)^2, sum b^2}.
alto_status dot_stats(const float* a, const float* b, uint64_t n, const double* colw, int R,
                      double* out3, DevBuf& scratch, cudaStream_t st);
alto_status dot_stats_f64(const double* a, const float* b, uint64_t n, double* out3,
                          DevBuf& scratch, cudaStream_t st);
alto_status sum_squares(const float* v, uint64_t n, double* out, DevBuf& scratch, cudaStream_t st);
alto_status model_norm(const double* grams, int nmodes, int R, const double* lambda, int exact,
                       double* out, cudaStream_t st);
// op 0: dst = a; 1: dst *= a; 2: dst *= alpha; 3: dst = 0 (n elements).
alto_status rr_op(double* dst, const double* a, int n, int op, double alpha, cudaStream_t st);
alto_status rank_update(double* G, const double* S, uint64_t rows, int R, cudaStream_t st);

}  // namespace alto
