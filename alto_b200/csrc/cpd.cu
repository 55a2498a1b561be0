// cpd.cu -- CP-ALS on the device.
//
// Replaces cpd_alto (IntelLabs/ALTO include/cpd.hpp:43-186) and
// cpd_fit_alto (:189-271).  Per iteration and mode j, in the reference's
// order: U_j = MTTKRP_j (U_j zeroed first), keep a copy of the last mode's
// MTTKRP for the fit, U_j <- U_j V^{-1} with V the Hadamard product of the
// other Grams (FP64), column norms (2-norm on the first iteration, max-norm
// floored at 1 afterwards) into lambda, U_j /= lambda, Gram of U_j.  The fit
// is evaluated on the device; one 8-byte read per iteration drives the
// |fit - prev| < epsilon stopping rule.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "dense.cuh"
#include "mttkrp_plan.h"

namespace altob {

struct AlsScratch {
    double *G, *W, *colacc, *lam, *inner, *normAT, *fit;
    int* info;
    void* M;
};

// Cross-GPU reduction of a sharded solve (nullptr: one GPU holds the
// whole tensor).
struct Reducer {
    altob_allreduce_fn fn = nullptr;
    void* user = nullptr;
    altob_status operator()(void* buf, u64 count, altob_dtype dt, int op, cudaStream_t st) const
    {
        if (!fn) return ALTOB_OK;
        const altob_status r = fn(buf, count, dt, op, st, user);
        return r == ALTOB_OK ? r : fail(r, "the all-reduce callback failed");
    }
};

template <typename FT>
static altob_status cpd_als_impl(altob_tensor* t, FT** U, FT* lam_out, int R, int max_iters, double eps,
                                 double* fits, int* iters, cudaStream_t st, const Reducer& red = Reducer())
{
    const int N = t->nmode;
    const u64 IN = t->dims[N - 1];
    // R <= 64: one fused pass (row update, statistics, Gram, inner product)
    // and one division pass per mode instead of the row-apply and Gram passes;
    // the fused pass reads the last mode's MTTKRP before overwriting it, so the
    // copy of it for the fit is not needed
    const bool fused = R <= APPLY_GRAM_MAX_RANK && env_int("ALTOB_FUSED_APPLY", 1);
    size_t nd = (size_t)N * R * R + (size_t)R * R + 3 * (size_t)R + 8;
    size_t bytes = nd * sizeof(double) + 256 + (fused ? 0 : IN * R * sizeof(FT)) + 256;
    void* base = nullptr;
    ALTOB_TRY(tensor_scratch(t, bytes, &base));
    AlsScratch s;
    double* d = (double*)base;
    s.G = d;
    d += (size_t)N * R * R;
    s.W = d;
    d += (size_t)R * R;
    s.colacc = d;
    d += R;
    s.lam = d;
    d += R;
    s.inner = d;
    d += R;
    s.normAT = d++;
    s.fit = d++;
    s.info = (int*)d;
    d += 2;
    s.M = (void*)(((uintptr_t)d + 255) & ~(uintptr_t)255);
    ALTOB_CUDA(cudaMemsetAsync(s.info, 0, sizeof(int), st));

    ALTOB_TRY(value_sumsq(t, s.normAT, st));
    ALTOB_TRY(red(s.normAT, 1, ALTOB_F64, ALTOB_REDUCE_SUM, st));  // ||X||^2 over all shards
    double normAT = 0.0;
    ALTOB_CUDA(cudaMemcpyAsync(&normAT, s.normAT, sizeof(double), cudaMemcpyDeviceToHost, st));
    for (int m = 0; m < N; ++m)
        ALTOB_TRY(gram<FT>(U[m], t->dims[m], R, s.G + (size_t)m * R * R, nullptr, nullptr, nullptr, nullptr, st));
    ALTOB_CUDA(cudaStreamSynchronize(st));

    const altob_dtype ft = sizeof(FT) == 8 ? ALTOB_F64 : ALTOB_F32;
    double prev = 0.0;
    int done = 0;
    for (int i = 0; i < max_iters; ++i) {
        const NormKind nk = i == 0 ? NORM_2 : NORM_MAX;
        for (int j = 0; j < N; ++j) {
            ALTOB_TRY(mttkrp_device(t, j, ft, (void* const*)U, (u64)R, 0, ALTOB_ALGO_AUTO, st));
            // a shard's partial MTTKRP summed over the GPUs; the dense update
            // below then runs on identical data on every GPU
            ALTOB_TRY(red(U[j], t->dims[j] * (u64)R, ft, ALTOB_REDUCE_SUM, st));
            if (fused) {
                double* Gj = s.G + (size_t)j * R * R;
                double* inner = j == N - 1 ? s.inner : nullptr;
                ALTOB_TRY(solve_setup(s.G, N, j, R, s.W, s.info, st));
                ALTOB_TRY(apply_gram<FT>(U[j], t->dims[j], R, s.W, nk, s.colacc, Gj, inner, st));
                ALTOB_TRY(lambda_finish(s.colacc, R, nk, s.lam, Gj, inner, st));
                ALTOB_TRY(normalize_cols<FT>(U[j], t->dims[j], R, s.lam, st));
                continue;
            }
            if (j == N - 1)
                ALTOB_CUDA(cudaMemcpyAsync(s.M, U[j], IN * R * sizeof(FT), cudaMemcpyDeviceToDevice, st));
            ALTOB_TRY(solve_setup(s.G, N, j, R, s.W, s.info, st));
            ALTOB_TRY(apply_w<FT>(U[j], t->dims[j], R, s.W, nk, s.colacc, st));
            ALTOB_TRY(lambda_from(s.colacc, R, nk, s.lam, st));
            ALTOB_TRY(gram<FT>(U[j], t->dims[j], R, s.G + (size_t)j * R * R, s.lam, U[j],
                               j == N - 1 ? (const FT*)s.M : nullptr, s.inner, st));
        }
        ALTOB_TRY(fit_from(s.G, N, R, s.lam, s.inner, normAT, s.fit, st));
        // one fit for every GPU (the dense passes add with atomics, so the
        // copies may differ in the last bits): the stopping rule agrees
        ALTOB_TRY(red(s.fit, 1, ALTOB_F64, ALTOB_REDUCE_MAX, st));
        double fit = 0.0;
        ALTOB_CUDA(cudaMemcpyAsync(&fit, s.fit, sizeof(double), cudaMemcpyDeviceToHost, st));
        ALTOB_CUDA(cudaStreamSynchronize(st));
        if (fits) fits[i] = fit;
        done = i + 1;
        if (i > 0 && std::fabs(prev - fit) < eps) break;
        prev = fit;
    }
    if (lam_out) ALTOB_TRY(vec_to<FT>(lam_out, s.lam, R, st));
    ALTOB_CUDA(cudaStreamSynchronize(st));
    if (iters) *iters = done;
    return ALTOB_OK;
}

altob_status check_model(const altob_tensor* t, altob_dtype ft, void* const* dU, u64 rank)
{
    if (!t || !dU) return fail(ALTOB_ERR_ARG, "NULL argument");
    if (ft != ALTOB_F64 && ft != ALTOB_F32) return fail(ALTOB_ERR_ARG, "model dtype must be F64 or F32");
    if (rank < 1) return fail(ALTOB_ERR_ARG, "rank must be >= 1");
    if (rank > (u64)SOLVE_MAX_RANK) return fail(ALTOB_ERR_UNSUPPORTED, "rank above 112");
    for (int m = 0; m < t->nmode; ++m)
        if (!dU[m]) return fail(ALTOB_ERR_ARG, "a factor pointer is NULL");
    if (ft == ALTOB_F32 && t->vdt == ALTOB_F64)
        return fail(ALTOB_ERR_UNSUPPORTED, "FP32 model on FP64 values: create the tensor with F32 values");
    if (ft == ALTOB_F64 && t->vdt == ALTOB_F32)
        return fail(ALTOB_ERR_UNSUPPORTED, "FP64 model on FP32 values: create the tensor with F64 values");
    return ALTOB_OK;
}

}  // namespace altob

using namespace altob;

extern "C" altob_status altob_pseudo_inverse(const double* d_grams, int nmode, int mode, uint64_t rank, void* d_U,
                                             uint64_t rows, altob_dtype ftype, int* used_pinv, void* stream)
{
    if (!d_grams || !d_U) return fail(ALTOB_ERR_ARG, "NULL argument");
    if (nmode < 2 || nmode > ALTOB_MAX_MODES || mode < 0 || mode >= nmode) return fail(ALTOB_ERR_ARG, "bad mode");
    if (ftype != ALTOB_F64 && ftype != ALTOB_F32) return fail(ALTOB_ERR_ARG, "dtype must be F64 or F32");
    if (rank < 1) return fail(ALTOB_ERR_ARG, "rank must be >= 1");
    if (rank > (u64)SOLVE_MAX_RANK) return fail(ALTOB_ERR_UNSUPPORTED, "rank above 112");
    cudaStream_t st = (cudaStream_t)stream;
    StreamScope scope(st);
    const int R = (int)rank;
    double* W = nullptr;
    ALTOB_TRY(dmalloc_t(&W, (size_t)R * R + 1));
    int* info = (int*)(W + (size_t)R * R);
    altob_status s = ALTOB_OK;
    cudaError_t e = cudaMemsetAsync(info, 0, sizeof(int), st);
    if (e != cudaSuccess) s = fail(ALTOB_ERR_CUDA, std::string("memset: ") + cudaGetErrorString(e));
    if (s == ALTOB_OK) s = solve_setup(d_grams, nmode, mode, R, W, info, st);
    if (s == ALTOB_OK)
        s = ftype == ALTOB_F64 ? apply_w<double>((double*)d_U, rows, R, W, NORM_NONE, nullptr, st)
                               : apply_w<float>((float*)d_U, rows, R, W, NORM_NONE, nullptr, st);
    int used = 0;
    if (s == ALTOB_OK) {
        e = cudaMemcpyAsync(&used, info, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) s = fail(ALTOB_ERR_CUDA, std::string("pseudo_inverse: ") + cudaGetErrorString(e));
    }
    dfree(W);
    if (used_pinv) *used_pinv = used;
    return s;
}

extern "C" altob_status altob_cpd_als(altob_tensor* t, altob_dtype ftype, void* const* d_factors, void* d_lambda,
                                      uint64_t rank, int max_iters, double epsilon, double* fits, int* iters,
                                      void* stream)
{
    ALTOB_TRY(check_model(t, ftype, d_factors, rank));
    if (max_iters < 1) return fail(ALTOB_ERR_ARG, "max_iters must be >= 1");
    if (t->nmode < 2) return fail(ALTOB_ERR_ARG, "CP-ALS needs at least two modes");
    if (t->nnz == 0) return fail(ALTOB_ERR_ARG, "CP-ALS on an empty tensor (the fit divides by its norm)");
    cudaStream_t st = (cudaStream_t)stream;
    StreamScope scope(st);
    if (ftype == ALTOB_F64)
        return cpd_als_impl<double>(t, (double**)d_factors, (double*)d_lambda, (int)rank, max_iters, epsilon, fits,
                                    iters, st);
    return cpd_als_impl<float>(t, (float**)d_factors, (float*)d_lambda, (int)rank, max_iters, epsilon, fits, iters,
                               st);
}

extern "C" altob_status altob_cpd_als_sharded(altob_tensor* t, altob_dtype ftype, void* const* d_factors,
                                              void* d_lambda, uint64_t rank, int max_iters, double epsilon,
                                              double* fits, int* iters, altob_allreduce_fn allreduce, void* user,
                                              void* stream)
{
    ALTOB_TRY(check_model(t, ftype, d_factors, rank));
    if (!allreduce) return fail(ALTOB_ERR_ARG, "allreduce callback is NULL");
    if (max_iters < 1) return fail(ALTOB_ERR_ARG, "max_iters must be >= 1");
    if (t->nmode < 2) return fail(ALTOB_ERR_ARG, "CP-ALS needs at least two modes");
    cudaStream_t st = (cudaStream_t)stream;
    StreamScope scope(st);
    Reducer red;
    red.fn = allreduce;
    red.user = user;
    if (ftype == ALTOB_F64)
        return cpd_als_impl<double>(t, (double**)d_factors, (double*)d_lambda, (int)rank, max_iters, epsilon, fits,
                                    iters, st, red);
    return cpd_als_impl<float>(t, (float**)d_factors, (float*)d_lambda, (int)rank, max_iters, epsilon, fits, iters,
                               st, red);
}
