// dense.cu -- host launchers of the dense CP-ALS / CP-APR kernels
// (dense_kernels.cuh).  Every reduction accumulates in FP64; factor storage
// is FT (float/double).
#include <algorithm>
#include <atomic>
#include <cmath>

#include "dense_kernels.cuh"

namespace altob {

template <typename FT>
altob_status gram(const FT* U, u64 I, int R, double* G, const double* div, FT* Uout, const FT* M, double* inner,
                  cudaStream_t st)
{
    if (R > 128) return fail(ALTOB_ERR_UNSUPPORTED, "rank above 128 in the Gram kernel");
    ALTOB_CUDA(cudaMemsetAsync(G, 0, (size_t)R * R * sizeof(double), st));
    if (M) ALTOB_CUDA(cudaMemsetAsync(inner, 0, (size_t)R * sizeof(double), st));
    if (I == 0) return ALTOB_OK;
    size_t smem = (size_t)(GR_ELEMS + 2 * R) * sizeof(double);  // < 48 KB for R <= 128
    const int g = dn_grid(I, 2 * (GR_ELEMS / R));
    if (R <= GR_SMALL) k_gram<FT, 1><<<g, DN_THREADS, smem, st>>>(U, I, R, G, div, Uout, M, inner);
    else k_gram<FT, 3><<<g, DN_THREADS, smem, st>>>(U, I, R, G, div, Uout, M, inner);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

// ----------------------------------------------------------- R x R solve
// V = Hadamard product of the Grams of all modes but `target` (only the
// lower triangle is meaningful, as in the reference's POTRF('L')).  If V is
// positive definite: Cholesky V = L L^T and W = V^{-1} = L^{-T} L^{-1}.
// Otherwise W = V^+ from a cyclic Jacobi eigendecomposition (eigenvalues
// below R * eps * max|lambda| dropped).  info[0] += 1 on every fallback.

altob_status solve_setup(const double* G, int nmode, int target, int R, double* W, int* info, cudaStream_t st)
{
    if (R > SOLVE_MAX_RANK) return fail(ALTOB_ERR_UNSUPPORTED, "rank above 112 in the R x R solve");
    size_t smem = (size_t)2 * R * R * sizeof(double);
    static std::atomic<size_t> configured{0};
    if (smem > 48 * 1024 && smem > configured.load()) {
        ALTOB_CUDA(cudaFuncSetAttribute(k_solve_setup, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        size_t cur = configured.load();
        while (cur < smem && !configured.compare_exchange_weak(cur, smem)) {
        }
    }
    k_solve_setup<<<1, DN_THREADS, smem, st>>>(G, nmode, target, R, W, info);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

// ------------------------------------------------------------ row apply
// U[i,:] <- U[i,:] W (FP64), lanes per row chosen by the rank; column norms of the
// result are accumulated on the fly (2-norm: sum of squares; max-norm:
// running max floored at 1, src/kruskal_model.cpp:264-305).

template <typename FT, int LPR, int CJ>
static altob_status launch_apply(FT* U, u64 I, int R, const double* W, NormKind nk, double* colacc, int grid,
                                 size_t smem, cudaStream_t st)
{
    static std::atomic<size_t> cfg{0};  // one per instantiation
    if (smem > 48 * 1024 && smem > cfg.load()) {
        ALTOB_CUDA(cudaFuncSetAttribute(k_apply<FT, LPR, CJ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        size_t cur = cfg.load();
        while (cur < smem && !cfg.compare_exchange_weak(cur, smem)) {
        }
    }
    k_apply<FT, LPR, CJ><<<grid, DN_THREADS, smem, st>>>(U, I, R, W, (int)nk, colacc);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

template <typename FT>
altob_status apply_w(FT* U, u64 I, int R, const double* W, NormKind nk, double* colacc, cudaStream_t st)
{
    if (R > 128) return fail(ALTOB_ERR_UNSUPPORTED, "rank above 128 in the row apply");
    if (nk != NORM_NONE) {
        if (nk == NORM_2) ALTOB_CUDA(cudaMemsetAsync(colacc, 0, (size_t)R * sizeof(double), st));
        else ALTOB_TRY(vec_fill(colacc, R, 1.0, st));
    }
    if (I == 0) return ALTOB_OK;
    size_t smem = (size_t)(R * R + R) * sizeof(double);
    const int g = dn_grid(I, (DN_THREADS / 32) * AP_RW * 8);
    switch (rank_class(R)) {
    case 0: return launch_apply<FT, 8, 1>(U, I, R, W, nk, colacc, g, smem, st);
    case 1: return launch_apply<FT, 16, 1>(U, I, R, W, nk, colacc, g, smem, st);
    case 2: return launch_apply<FT, 32, 1>(U, I, R, W, nk, colacc, g, smem, st);
    case 3: return launch_apply<FT, 32, 2>(U, I, R, W, nk, colacc, g, smem, st);
    default: return launch_apply<FT, 32, 4>(U, I, R, W, nk, colacc, g, smem, st);
    }
}

// ------------------------------------------- fused row update + Gram (R <= 64)

template <typename FT, int MB>
static altob_status launch_apply_gram(FT* U, u64 I, int R, const double* W, NormKind nk, double* colacc, double* G,
                                      double* inner, cudaStream_t st)
{
    static std::atomic<int> per_sm{0};  // resident blocks per SM (one value per instantiation)
    if (per_sm.load() == 0) {
        int n = 0;
        ALTOB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_apply_gram<FT, MB>, AG_THREADS,
                                                                 apply_gram_smem<MB>()));
        per_sm.store(std::max(1, n));
    }
    const u64 groups = (I + 7) / 8;
    const int per_block = AG_THREADS / 32 * 4;  // at least 4 row groups per warp
    const u64 want = (groups + per_block - 1) / per_block;
    const int grid = (int)std::max<u64>(1, std::min<u64>(want, (u64)num_sms() * per_sm.load()));
    const int vec_ok = ((uintptr_t)U & 15) == 0;
    k_apply_gram<FT, MB><<<grid, AG_THREADS, apply_gram_smem<MB>(), st>>>(U, I, R, W, (int)nk, colacc, G, inner,
                                                                        vec_ok);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

template <typename FT>
altob_status apply_gram(FT* U, u64 I, int R, const double* W, NormKind nk, double* colacc, double* G, double* inner,
                        cudaStream_t st)
{
    if (R > APPLY_GRAM_MAX_RANK) return fail(ALTOB_ERR_UNSUPPORTED, "rank above 64 in the fused row update");
    if (nk == NORM_2) ALTOB_CUDA(cudaMemsetAsync(colacc, 0, (size_t)R * sizeof(double), st));
    else if (nk == NORM_MAX) ALTOB_TRY(vec_fill(colacc, R, 1.0, st));
    ALTOB_CUDA(cudaMemsetAsync(G, 0, (size_t)R * R * sizeof(double), st));
    if (inner) ALTOB_CUDA(cudaMemsetAsync(inner, 0, (size_t)R * sizeof(double), st));
    if (I == 0) return ALTOB_OK;
    switch ((R + 7) / 8) {
    case 1: return launch_apply_gram<FT, 1>(U, I, R, W, nk, colacc, G, inner, st);
    case 2: return launch_apply_gram<FT, 2>(U, I, R, W, nk, colacc, G, inner, st);
    case 3: return launch_apply_gram<FT, 3>(U, I, R, W, nk, colacc, G, inner, st);
    case 4: return launch_apply_gram<FT, 4>(U, I, R, W, nk, colacc, G, inner, st);
    case 5: return launch_apply_gram<FT, 5>(U, I, R, W, nk, colacc, G, inner, st);
    case 6: return launch_apply_gram<FT, 6>(U, I, R, W, nk, colacc, G, inner, st);
    case 7: return launch_apply_gram<FT, 7>(U, I, R, W, nk, colacc, G, inner, st);
    default: return launch_apply_gram<FT, 8>(U, I, R, W, nk, colacc, G, inner, st);
    }
}

altob_status lambda_finish(const double* colacc, int R, NormKind nk, double* lam, double* G, double* inner,
                           cudaStream_t st)
{
    k_lambda_finish<<<1, DN_THREADS, 0, st>>>(colacc, R, (int)nk, lam, G, inner);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

template <typename FT>
altob_status normalize_cols(FT* U, u64 I, int R, const double* lam, cudaStream_t st)
{
    if (I == 0) return ALTOB_OK;
    constexpr int V = 16 / sizeof(FT);
    const bool vec = R % V == 0 && ((uintptr_t)U & 15) == 0;
    const u64 n = I * (u64)R;
    const size_t smem = (size_t)R * sizeof(double);
    if (vec) k_div_cols<FT, V><<<dn_grid(n / V, DN_THREADS * 4), DN_THREADS, smem, st>>>(U, I, R, lam);
    else k_div_cols<FT, 1><<<dn_grid(n, DN_THREADS * 4), DN_THREADS, smem, st>>>(U, I, R, lam);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

// ------------------------------------------------------------- small ops

altob_status lambda_from(const double* colacc, int R, NormKind nk, double* lam, cudaStream_t st)
{
    k_lambda<<<1, 128, 0, st>>>(colacc, R, (int)nk, lam);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

altob_status fit_from(const double* G, int nmode, int R, const double* lam, const double* inner, double normAT,
                      double* fit, cudaStream_t st)
{
    k_fit<<<1, DN_THREADS, 0, st>>>(G, nmode, R, lam, inner, normAT, fit);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

template <typename FT>
altob_status colsum_abs(const FT* U, u64 I, int R, double* acc, cudaStream_t st)
{
    ALTOB_CUDA(cudaMemsetAsync(acc, 0, (size_t)R * sizeof(double), st));
    if (I == 0) return ALTOB_OK;
    k_colsum_abs<FT><<<dn_grid(I * R, DN_THREADS * 16), DN_THREADS, R * sizeof(double), st>>>(U, I, R, acc);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

template <typename FT>
altob_status div_cols(FT* U, u64 I, int R, const double* d, cudaStream_t st)
{
    if (I == 0) return ALTOB_OK;
    k_scale_cols<FT><<<dn_grid(I * R, DN_THREADS * 8), DN_THREADS, 0, st>>>(U, I, R, d, 1);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

template <typename FT>
altob_status mul_cols(FT* U, u64 I, int R, const double* d, cudaStream_t st)
{
    if (I == 0) return ALTOB_OK;
    k_scale_cols<FT><<<dn_grid(I * R, DN_THREADS * 8), DN_THREADS, 0, st>>>(U, I, R, d, 0);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

template <typename FT>
altob_status sum_all(const FT* U, u64 n, double* acc, cudaStream_t st)
{
    ALTOB_CUDA(cudaMemsetAsync(acc, 0, sizeof(double), st));
    if (n == 0) return ALTOB_OK;
    k_sum_all<FT><<<dn_grid(n, DN_THREADS * 16), DN_THREADS, 0, st>>>(U, n, acc);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

altob_status vec_mul(double* lam, const double* d, int R, cudaStream_t st)
{
    k_vec<<<1, 128, 0, st>>>(lam, d, R, 0.0, 0);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

altob_status vec_fill(double* v, int R, double x, cudaStream_t st)
{
    k_vec<<<1, 128, 0, st>>>(v, nullptr, R, x, 1);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

template <typename FT>
altob_status vec_to(FT* dst, const double* src, int R, cudaStream_t st)
{
    k_conv<FT, double><<<1, 128, 0, st>>>(dst, src, R);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

template <typename FT>
altob_status vec_from(double* dst, const FT* src, int R, cudaStream_t st)
{
    k_conv<double, FT><<<1, 128, 0, st>>>(dst, src, R);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

altob_status value_sumsq(const altob_tensor* t, double* acc, cudaStream_t st)
{
    ALTOB_CUDA(cudaMemsetAsync(acc, 0, sizeof(double), st));
    if (t->nnz == 0) return ALTOB_OK;
    int g = dn_grid(t->nnz, DN_THREADS * 16);
    if (t->vdt == ALTOB_F64) k_sumsq<double><<<g, DN_THREADS, 0, st>>>((const double*)t->d_vals, t->nnz, acc);
    else if (t->vdt == ALTOB_F32) k_sumsq<float><<<g, DN_THREADS, 0, st>>>((const float*)t->d_vals, t->nnz, acc);
    else k_sumsq<u32><<<g, DN_THREADS, 0, st>>>((const u32*)t->d_vals, t->nnz, acc);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

#define ALTOB_DENSE_INST(FT)                                                                                 \
    template altob_status gram<FT>(const FT*, u64, int, double*, const double*, FT*, const FT*, double*,     \
                                   cudaStream_t);                                                            \
    template altob_status apply_w<FT>(FT*, u64, int, const double*, NormKind, double*, cudaStream_t);        \
    template altob_status apply_gram<FT>(FT*, u64, int, const double*, NormKind, double*, double*, double*,  \
                                         cudaStream_t);                                                      \
    template altob_status normalize_cols<FT>(FT*, u64, int, const double*, cudaStream_t);                    \
    template altob_status colsum_abs<FT>(const FT*, u64, int, double*, cudaStream_t);                        \
    template altob_status div_cols<FT>(FT*, u64, int, const double*, cudaStream_t);                          \
    template altob_status mul_cols<FT>(FT*, u64, int, const double*, cudaStream_t);                          \
    template altob_status sum_all<FT>(const FT*, u64, double*, cudaStream_t);                                \
    template altob_status vec_to<FT>(FT*, const double*, int, cudaStream_t);                                 \
    template altob_status vec_from<FT>(double*, const FT*, int, cudaStream_t);

ALTOB_DENSE_INST(float)
ALTOB_DENSE_INST(double)

}  // namespace altob
