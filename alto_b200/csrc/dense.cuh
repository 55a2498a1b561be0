// dense.cuh -- dense kernels of the CP-ALS / CP-APR updates.
//
// Reference operations replaced (IntelLabs/ALTO):
//   update_gram (SYRK)          src/kruskal_model.cpp:11-24   -> k_gram (FP64 accumulate),
//                                                               k_apply_gram (R <= 64, FP64 MMA)
//   pseudo_inverse (POTRF/POTRS, GELSY fallback)
//                               include/cpd.hpp:546-646       -> k_solve_setup + k_apply
//   KruskalModelNorm            src/kruskal_model.cpp:224-341 -> k_apply (fused) + k_lambda
//   cpd_fit_alto                include/cpd.hpp:189-271       -> k_gram(inner) + k_fit
//   KruskalModelNormalizeMode   src/kruskal_model.cpp:178-222 -> k_colsum_abs + k_div_cols
//   RedistributeLambda          src/kruskal_model.cpp:355-378 -> k_mul_cols
#pragma once

#include "internal.cuh"

namespace altob {

constexpr int DN_THREADS = 256;
constexpr int SOLVE_MAX_RANK = 112;  // two R x R FP64 matrices in shared memory
constexpr int APPLY_GRAM_MAX_RANK = 64;  // fused row update + Gram (up to eight 8-column MMA blocks)

enum NormKind { NORM_NONE = 0, NORM_2 = 1, NORM_MAX = 2 };

// Argument checks shared by the CP-ALS / CP-APR entry points (cpd.cu).
altob_status check_model(const altob_tensor* t, altob_dtype ft, void* const* dU, u64 rank);

// Host launchers (dense.cu).  All FP64 internally; FT = storage type.
template <typename FT>
altob_status gram(const FT* U, u64 I, int R, double* G, const double* div, FT* Uout, const FT* M,
                  double* inner, cudaStream_t st);
altob_status solve_setup(const double* G, int nmode, int target, int R, double* W, int* info, cudaStream_t st);
template <typename FT>
altob_status apply_w(FT* U, u64 I, int R, const double* W, NormKind nk, double* colacc, cudaStream_t st);
altob_status lambda_from(const double* colacc, int R, NormKind nk, double* lam, cudaStream_t st);
// Fused U <- U W with column statistics, G = U^T U and (inner given) the fit's
// inner product, all before normalisation; lambda_finish then sets lambda,
// G /= lambda lambda^T, inner /= lambda; normalize_cols divides U by lambda.
template <typename FT>
altob_status apply_gram(FT* U, u64 I, int R, const double* W, NormKind nk, double* colacc, double* G, double* inner,
                        cudaStream_t st);
altob_status lambda_finish(const double* colacc, int R, NormKind nk, double* lam, double* G, double* inner,
                           cudaStream_t st);
template <typename FT>
altob_status normalize_cols(FT* U, u64 I, int R, const double* lam, cudaStream_t st);
altob_status fit_from(const double* G, int nmode, int R, const double* lam, const double* inner, double normAT,
                      double* fit, cudaStream_t st);
template <typename FT>
altob_status colsum_abs(const FT* U, u64 I, int R, double* acc, cudaStream_t st);
template <typename FT>
altob_status div_cols(FT* U, u64 I, int R, const double* d, cudaStream_t st);
template <typename FT>
altob_status mul_cols(FT* U, u64 I, int R, const double* d, cudaStream_t st);
template <typename FT>
altob_status sum_all(const FT* U, u64 n, double* acc, cudaStream_t st);
altob_status vec_mul(double* lam, const double* d, int R, cudaStream_t st);
altob_status vec_fill(double* v, int R, double x, cudaStream_t st);
template <typename FT>
altob_status vec_to(FT* dst, const double* src, int R, cudaStream_t st);
template <typename FT>
altob_status vec_from(double* dst, const FT* src, int R, cudaStream_t st);
// Sum of squared values of the stored tensor (normAT, cpd.hpp:73-79).
altob_status value_sumsq(const altob_tensor* t, double* acc, cudaStream_t st);

}  // namespace altob
