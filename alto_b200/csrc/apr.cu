// apr.cu -- CP-APR (multiplicative update) on the device.
//
// Replaces cp_apr_alto (IntelLabs/ALTO include/apr.hpp:984-1376) and
// tt_logLikelihood<LIT> (:851-982).  Order of operations follows the
// reference: KruskalModelNormalize, then per outer iteration and mode n the
// kappa fix (iter > 0), RedistributeLambda, up to max_inner rounds of
// {Phi, KKT violation, B *= Phi} with the early exit when the violation is
// below epsilon (skipped in bench mode), and KruskalModelNormalizeMode.  The
// KKT violation and the log-likelihood accumulate in FP64.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "dense.cuh"
#include "mttkrp_plan.h"

namespace altob {

// |min(B, 1 - Phi)| max-reduced (apr.hpp:1210-1216); with `mult`, also
// B *= Phi (apr.hpp:1226-1231) in the same pass.
template <typename FT>
__global__ void k_kkt(FT* __restrict__ B, const FT* __restrict__ Phi, u64 n, double* __restrict__ kkt, int mult)
{
    double m = 0.0;
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (u64)gridDim.x * blockDim.x) {
        const double b = (double)B[e], p = (double)Phi[e];
        m = fmax(m, fabs(fmin(b, 1.0 - p)));
        if (mult) B[e] = (FT)(b * p);
    }
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0)
        atomicMax(reinterpret_cast<unsigned long long*>(kkt), (unsigned long long)__double_as_longlong(m));
}

template <typename FT>
__global__ void k_mult(FT* __restrict__ B, const FT* __restrict__ Phi, u64 n)
{
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (u64)gridDim.x * blockDim.x)
        B[e] = (FT)((double)B[e] * (double)Phi[e]);
}

// Kappa fix (apr.hpp:1176-1189).
template <typename FT>
__global__ void k_kappa(FT* __restrict__ B, const FT* __restrict__ Phi, u64 n, double kappa_tol, double kappa)
{
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (u64)gridDim.x * blockDim.x)
        if ((double)B[e] < kappa_tol && (double)Phi[e] > 1.0) B[e] = (FT)((double)B[e] + kappa);
}

template <typename FT>
struct LLArgs {
    KeySrc key;
    const void* vals;
    u64 nnz;
    int nmode, R;
    double eps;
    const FT* U[ALTOB_MAX_MODES];
    Fields fld;
};

// sum_nnz v * log(max(sum_r prod_n U_n[i_n, r], eps)) (apr.hpp:913-943).
template <typename FT, typename VT>
__global__ void __launch_bounds__(256) k_loglik(LLArgs<FT> a, double* __restrict__ acc)
{
    const VT* vals = reinterpret_cast<const VT*>(a.vals);
    double s = 0.0;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < a.nnz; i += (u64)gridDim.x * blockDim.x) {
        const u64 lo = a.key.klo[i], hi = key_hi(a.key, i);
        const FT* rows[ALTOB_MAX_MODES];
#pragma unroll
        for (int m = 0; m < ALTOB_MAX_MODES; ++m)
            if (m < a.nmode) rows[m] = a.U[m] + (size_t)field(lo, hi, a.fld.pos[m], a.fld.mask[m]) * a.R;
        double tmp = 0.0;
        for (int r = 0; r < a.R; ++r) {
            double p = 1.0;
            for (int m = 0; m < a.nmode; ++m) p *= (double)__ldg(rows[m] + r);
            tmp += p;
        }
        if (tmp < a.eps) tmp = a.eps;
        s += (double)vals[i] * log(tmp);
    }
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(acc, s);
}

static int ew_grid(u64 n)
{
    u64 b = (n + 256 * 8 - 1) / (256 * 8);
    return (int)std::max<u64>(1, std::min<u64>(b, (u64)num_sms() * 8));
}

template <typename FT>
static altob_status loglik_sum(const altob_tensor* t, FT** U, int R, double eps, double* acc, cudaStream_t st)
{
    ALTOB_CUDA(cudaMemsetAsync(acc, 0, sizeof(double), st));
    if (t->nnz == 0) return ALTOB_OK;
    LLArgs<FT> a;
    memset(&a, 0, sizeof(a));
    a.key = key_src(t);
    a.vals = t->d_vals;
    a.nnz = t->nnz;
    a.nmode = t->nmode;
    a.R = R;
    a.eps = eps;
    for (int m = 0; m < t->nmode; ++m) a.U[m] = U[m];
    a.fld = t->fld;
    const int g = ew_grid(t->nnz);
#define LLK(VT) k_loglik<FT, VT><<<g, 256, 0, st>>>(a, acc)
    if (t->vdt == ALTOB_U32) LLK(u32);
    else if (t->vdt == ALTOB_F64) LLK(double);
    else LLK(float);
#undef LLK
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

struct AprScratch {
    double *lam, *colacc, *kkt, *G, *inner, *fit, *normAT, *ll, *fsum;
    int* info;
};

// tt_logLikelihood (apr.hpp:851-982): lambda into mode 0, log-likelihood
// minus sum(U_0), then mode 0 renormalised by its column 1-norms.
// The caller provides every scratch word (lam, colacc, ll, fsum): this
// function and the helpers it calls must not allocate device memory, since
// altob_loglik_noalloc passes its fixed array here.
template <typename FT>
static altob_status loglik_impl(altob_tensor* t, FT** U, double* lam, double* colacc, double* ll, double* fsum,
                                int R, double eps, double* out, cudaStream_t st)
{
    ALTOB_TRY(mul_cols<FT>(U[0], t->dims[0], R, lam, st));
    ALTOB_TRY(vec_fill(lam, R, 1.0, st));
    ALTOB_TRY(loglik_sum<FT>(t, U, R, eps, ll, st));
    ALTOB_TRY(sum_all<FT>(U[0], t->dims[0] * (u64)R, fsum, st));
    ALTOB_TRY(colsum_abs<FT>(U[0], t->dims[0], R, colacc, st));
    ALTOB_TRY(div_cols<FT>(U[0], t->dims[0], R, colacc, st));
    ALTOB_TRY(vec_mul(lam, colacc, R, st));
    double h[2];
    ALTOB_CUDA(cudaMemcpyAsync(&h[0], ll, sizeof(double), cudaMemcpyDeviceToHost, st));
    ALTOB_CUDA(cudaMemcpyAsync(&h[1], fsum, sizeof(double), cudaMemcpyDeviceToHost, st));
    ALTOB_CUDA(cudaStreamSynchronize(st));
    *out = h[0] - h[1];
    return ALTOB_OK;
}

// How Phi is formed: precomputed Khatri-Rao rows (the reference's PRE build)
// when a mode runs more than one inner iteration, in the row-ordered stream
// (PHI_ROWS: rows, values and stream positions kept per mode) when that fits
// in a quarter of free memory, else in ALTO order (PHI_PRE, the tiled
// kernel), else on the fly (PHI_OTF).  ALTOB_APR_PHI=rows|pre|otf forces one.
enum AprPhi { PHI_OTF = 0, PHI_PRE = 1, PHI_ROWS = 2 };

static AprPhi apr_phi_kind(const altob_tensor* t, int R, size_t fsz, int max_inner)
{
    const char* v = getenv("ALTOB_APR_PHI");
    if (v && !strcmp(v, "otf")) return PHI_OTF;
    if (v && !strcmp(v, "pre")) return PHI_PRE;
    if (v && !strcmp(v, "rows")) return PHI_ROWS;
    if (max_inner < 2) return PHI_OTF;
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return PHI_OTF;
    const double nnz = (double)t->nnz;
    if (nnz * ((double)R * fsz + t->nmode * (8.0 + fsz) + 24.0) <= 0.25 * (double)fr) return PHI_ROWS;
    return nnz * R * fsz <= 0.25 * (double)fr ? PHI_PRE : PHI_OTF;
}

template <typename FT>
static altob_status cp_apr_impl(altob_tensor* t, FT** U, FT* lam_io, int R, int max_iters, int max_inner,
                                double eps, double eps_div_zero, double kappa_tol, double kappa, int dobench,
                                double* summary, cudaStream_t st)
{
    const int N = t->nmode;
    const altob_dtype ft = sizeof(FT) == 8 ? ALTOB_F64 : ALTOB_F32;
    size_t phi_elems = 0;
    std::vector<size_t> phi_off(N);
    for (int n = 0; n < N; ++n) {
        phi_off[n] = phi_elems;
        phi_elems += (t->dims[n] * R + 63) & ~(size_t)63;
    }
    size_t nd = 4 * (size_t)R + (size_t)N * R * R + 16;
    size_t bytes = nd * sizeof(double) + 256 + phi_elems * sizeof(FT) + 256;
    void* base = nullptr;
    ALTOB_TRY(tensor_scratch(t, bytes, &base));
    double* d = (double*)base;
    AprScratch s;
    s.lam = d;
    d += R;
    s.colacc = d;
    d += R;
    s.inner = d;
    d += R;
    s.G = d;
    d += (size_t)N * R * R;
    s.kkt = d;
    d += 8;  // one per mode
    s.fit = d++;
    s.normAT = d++;
    s.ll = d++;
    s.fsum = d++;
    s.info = (int*)d;
    d += 2;
    FT* phi_base = (FT*)(((uintptr_t)d + 255) & ~(uintptr_t)255);
    std::vector<FT*> Phi(N);
    for (int n = 0; n < N; ++n) Phi[n] = phi_base + phi_off[n];

    // KruskalModelNormalize (src/kruskal_model.cpp:128-176)
    ALTOB_TRY(vec_from<FT>(s.lam, lam_io, R, st));
    for (int n = 0; n < N; ++n) {
        ALTOB_TRY(colsum_abs<FT>(U[n], t->dims[n], R, s.colacc, st));
        ALTOB_TRY(div_cols<FT>(U[n], t->dims[n], R, s.colacc, st));
        ALTOB_TRY(vec_mul(s.lam, s.colacc, R, st));
    }
    std::vector<double> kkt_iter(max_iters + 1, 0.0), kmode(N, 0.0);
    std::vector<int> ninner(max_iters + 1, 0);
    void* pi = nullptr;  // nnz x R precomputed rows
    u32 *rows = nullptr, *inv = nullptr;  // row-ordered stream: N x nnz each
    FT* svals = nullptr;
    struct PiFree {
        void *p, *r, *i, *v;
        ~PiFree()
        {
            dfree(p);
            dfree(r);
            dfree(i);
            dfree(v);
        }
    } pi_free{nullptr, nullptr, nullptr, nullptr};
    const u64 nnz = t->nnz;
    // per-mode stride of the row-ordered stream: a multiple of 4 elements, so
    // every mode's arrays start 16-byte aligned and may be read to a multiple
    // of 4 past their end (bulk copies of whole 16-byte units)
    const u64 nnzp = (nnz + 3) & ~3ull;
    AprPhi kind = nnz ? apr_phi_kind(t, R, sizeof(FT), max_inner) : PHI_OTF;
    // Memory can go to other streams between the choice and the allocations
    // (concurrent requests of a server): an allocation that fails falls back
    // to the next path, which gives the same Phi.
    auto drop_stream = [&]() {
        dfree(rows);
        dfree(inv);
        dfree(svals);
        rows = inv = nullptr;
        svals = nullptr;
        pi_free.r = pi_free.i = pi_free.v = nullptr;
    };
    if (kind == PHI_ROWS) {
        altob_status a = dmalloc_t(&rows, (size_t)N * nnzp);
        pi_free.r = rows;
        if (a == ALTOB_OK) a = dmalloc_t(&inv, (size_t)N * nnzp);
        pi_free.i = inv;
        if (a == ALTOB_OK) a = dmalloc_t(&svals, (size_t)N * nnzp);
        pi_free.v = svals;
        for (int n = 0; n < N && a == ALTOB_OK; ++n)
            a = mode_order_device(t, n, ft, rows + (size_t)n * nnzp, svals + (size_t)n * nnzp,
                                  inv + (size_t)n * nnzp, st);
        if (a == ALTOB_ERR_NOMEM) {
            drop_stream();
            kind = PHI_PRE;
        } else if (a != ALTOB_OK) {
            return a;
        }
    }
    if (kind != PHI_OTF) {
        const altob_status a = dmalloc(&pi, nnz * (size_t)R * sizeof(FT));
        if (a == ALTOB_ERR_NOMEM) {
            drop_stream();
            pi = nullptr;
            kind = PHI_OTF;
        } else if (a != ALTOB_OK) {
            return a;
        }
        pi_free.p = pi;
    }
    int iter;
    for (iter = 0; iter < max_iters; ++iter) {
        bool converged = false;
        if (dobench) ALTOB_CUDA(cudaMemsetAsync(s.kkt, 0, N * sizeof(double), st));
        for (int n = 0; n < N; ++n) {
            const u64 sz = t->dims[n] * (u64)R;
            FT* B = U[n];
            if (iter > 0 && sz) {
                k_kappa<FT><<<ew_grid(sz), 256, 0, st>>>(B, Phi[n], sz, kappa_tol, kappa);
                ALTOB_LAUNCH_CHECK();
            }
            ALTOB_TRY(mul_cols<FT>(B, t->dims[n], R, s.lam, st));  // RedistributeLambda
            ALTOB_TRY(vec_fill(s.lam, R, 1.0, st));
            const u32* inv_n = rows ? inv + (size_t)n * nnzp : nullptr;
            if (pi) ALTOB_TRY(pi_device(t, n, ft, (void* const*)U, (u64)R, pi, st, inv_n));
            for (int inner = 0; inner < max_inner; ++inner) {
                ninner[iter]++;
                if (rows)
                    ALTOB_TRY(phi_rows_device(t, n, ft, pi, rows + (size_t)n * nnzp, svals + (size_t)n * nnzp, B,
                                              (u64)R, eps_div_zero, Phi[n], st, true));
                else if (pi) ALTOB_TRY(phi_pre_device(t, n, ft, pi, B, (u64)R, eps_div_zero, Phi[n], st));
                else ALTOB_TRY(phi_device(t, n, ft, (void* const*)U, (u64)R, eps_div_zero, Phi[n], st));
                if (dobench) {
                    // no early exit: the violation of the last round is what the reference reports
                    ALTOB_CUDA(cudaMemsetAsync(s.kkt + n, 0, sizeof(double), st));
                    if (sz) k_kkt<FT><<<ew_grid(sz), 256, 0, st>>>(B, Phi[n], sz, s.kkt + n, 1);
                    ALTOB_LAUNCH_CHECK();
                } else {
                    ALTOB_CUDA(cudaMemsetAsync(s.kkt + n, 0, sizeof(double), st));
                    if (sz) k_kkt<FT><<<ew_grid(sz), 256, 0, st>>>(B, Phi[n], sz, s.kkt + n, 0);
                    ALTOB_LAUNCH_CHECK();
                    double kv = 0.0;
                    ALTOB_CUDA(cudaMemcpyAsync(&kv, s.kkt + n, sizeof(double), cudaMemcpyDeviceToHost, st));
                    ALTOB_CUDA(cudaStreamSynchronize(st));
                    kmode[n] = kv;
                    if (kv < eps) break;
                    if (sz) k_mult<FT><<<ew_grid(sz), 256, 0, st>>>(B, Phi[n], sz);
                    ALTOB_LAUNCH_CHECK();
                }
            }
            // KruskalModelNormalizeMode (src/kruskal_model.cpp:178-222)
            ALTOB_TRY(colsum_abs<FT>(B, t->dims[n], R, s.colacc, st));
            ALTOB_TRY(div_cols<FT>(B, t->dims[n], R, s.colacc, st));
            ALTOB_TRY(vec_mul(s.lam, s.colacc, R, st));
        }
        if (dobench) {
            ALTOB_CUDA(cudaMemcpyAsync(kmode.data(), s.kkt, N * sizeof(double), cudaMemcpyDeviceToHost, st));
            ALTOB_CUDA(cudaStreamSynchronize(st));
        }
        kkt_iter[iter] = kmode[0];
        for (int n = 1; n < N; ++n) kkt_iter[iter] = std::fmax(kkt_iter[iter], kmode[n]);
        // apr.hpp:1261; the first iteration has no predecessor to compare with
        if (iter > 0 && std::fabs(kkt_iter[iter] - kkt_iter[iter - 1]) <= eps * eps && !dobench) converged = true;
        if (converged) break;
    }
    int tot_inner = 0;
    for (int i = 0; i < iter; ++i) tot_inner += ninner[i];
    double ll = 0.0;
    ALTOB_TRY(loglik_impl<FT>(t, U, s.lam, s.colacc, s.ll, s.fsum, R, eps_div_zero, &ll, st));

    // least-squares fit of the final model (apr.hpp:1301-1330)
    for (int n = 0; n < N - 1; ++n)
        ALTOB_TRY(gram<FT>(U[n], t->dims[n], R, s.G + (size_t)n * R * R, nullptr, nullptr, nullptr, nullptr, st));
    FT* mt = Phi[N - 1];
    {
        std::vector<void*> tmpU(N);
        for (int n = 0; n < N; ++n) tmpU[n] = U[n];
        tmpU[N - 1] = mt;
        ALTOB_TRY(mttkrp_device(t, N - 1, ft, tmpU.data(), (u64)R, 0, ALTOB_ALGO_AUTO, st));
    }
    ALTOB_TRY(gram<FT>(U[N - 1], t->dims[N - 1], R, s.G + (size_t)(N - 1) * R * R, nullptr, nullptr, mt, s.inner,
                       st));
    ALTOB_TRY(value_sumsq(t, s.normAT, st));
    double normAT = 0.0;
    ALTOB_CUDA(cudaMemcpyAsync(&normAT, s.normAT, sizeof(double), cudaMemcpyDeviceToHost, st));
    ALTOB_CUDA(cudaStreamSynchronize(st));
    ALTOB_TRY(fit_from(s.G, N, R, s.lam, s.inner, normAT, s.fit, st));
    double fit = 0.0;
    ALTOB_CUDA(cudaMemcpyAsync(&fit, s.fit, sizeof(double), cudaMemcpyDeviceToHost, st));
    ALTOB_TRY(vec_to<FT>(lam_io, s.lam, R, st));
    ALTOB_CUDA(cudaStreamSynchronize(st));
    if (t->h_tma_err && *t->h_tma_err)
        return fail(ALTOB_ERR_CUDA, "a bulk-copy-staged Phi pass ran out of a wait limit");
    if (summary) {
        summary[0] = ll;
        summary[1] = fit;
        summary[2] = iter > 0 ? kkt_iter[iter - 1] : kkt_iter[0];
        summary[3] = iter;
        summary[4] = tot_inner;
    }
    return ALTOB_OK;
}

}  // namespace altob

using namespace altob;

extern "C" {

altob_status altob_cp_apr(altob_tensor* t, altob_dtype ftype, void* const* d_factors, void* d_lambda, uint64_t rank,
                          int max_iters, int max_inner, double epsilon, double eps_div_zero, double kappa_tol,
                          double kappa, int dobench, double* summary, void* stream)
{
    ALTOB_TRY(check_model(t, ftype, d_factors, rank));
    if (!d_lambda) return fail(ALTOB_ERR_ARG, "lambda is NULL");
    if (max_iters < 1 || max_inner < 1) return fail(ALTOB_ERR_ARG, "iteration counts must be >= 1");
    if (t->nnz == 0) return fail(ALTOB_ERR_ARG, "CP-APR on an empty tensor");
    cudaStream_t st = (cudaStream_t)stream;
    StreamScope scope(st);
    if (ftype == ALTOB_F64)
        return cp_apr_impl<double>(t, (double**)d_factors, (double*)d_lambda, (int)rank, max_iters, max_inner,
                                   epsilon, eps_div_zero, kappa_tol, kappa, dobench, summary, st);
    return cp_apr_impl<float>(t, (float**)d_factors, (float*)d_lambda, (int)rank, max_iters, max_inner, epsilon,
                              eps_div_zero, kappa_tol, kappa, dobench, summary, st);
}

altob_status altob_loglik(altob_tensor* t, altob_dtype ftype, void* const* d_factors, void* d_lambda, uint64_t rank,
                          double eps_div_zero, double* loglik, void* stream)
{
    ALTOB_TRY(check_model(t, ftype, d_factors, rank));
    if (!d_lambda || !loglik) return fail(ALTOB_ERR_ARG, "NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    StreamScope scope(st);
    const int R = (int)rank;
    void* base = nullptr;
    ALTOB_TRY(tensor_scratch(t, (4 * (size_t)R + 8) * sizeof(double), &base));
    double* d = (double*)base;
    double *lam = d, *colacc = d + R, *ll = d + 2 * R, *fsum = d + 2 * R + 1;
    if (ftype == ALTOB_F64) {
        ALTOB_TRY(vec_from<double>(lam, (const double*)d_lambda, R, st));
        ALTOB_TRY(loglik_impl<double>(t, (double**)d_factors, lam, colacc, ll, fsum, R, eps_div_zero, loglik, st));
        ALTOB_TRY(vec_to<double>((double*)d_lambda, lam, R, st));
    } else {
        ALTOB_TRY(vec_from<float>(lam, (const float*)d_lambda, R, st));
        ALTOB_TRY(loglik_impl<float>(t, (float**)d_factors, lam, colacc, ll, fsum, R, eps_div_zero, loglik, st));
        ALTOB_TRY(vec_to<float>((float*)d_lambda, lam, R, st));
    }
    ALTOB_CUDA(cudaStreamSynchronize(st));
    return ALTOB_OK;
}

}  // extern "C"


// ---------------------------------------------------------------------------
// altob_loglik_noalloc: the log-likelihood for callers that cannot allocate
// device memory.  Some callers own every byte of device memory through their
// own pool or arena, run where the CUDA allocator must not be entered, or
// need a call whose memory footprint is fixed before it runs; altob_loglik
// takes its scratch from the tensor handle's cache, which may call
// cudaMalloc.  This variant keeps its scratch in the file-scope array below
// instead.  The caller still passes the tensor, factors and lambda.

namespace altob {

// Largest rank the fixed scratch holds (the library's model rank limit):
// lambda and column sums (2R doubles) plus the two accumulators;
// 2 * 112 + 8 doubles = 1856 bytes per device.
constexpr int LOGLIK_NOALLOC_MAX_RANK = 112;
static __device__ __align__(256) double g_loglik_scratch[2 * LOGLIK_NOALLOC_MAX_RANK + 8];

// Device address of g_loglik_scratch on the current device.  Host code may
// not use the array's name as a device pointer, so the address is looked up
// once per device (on the first call there) and cached.
static altob_status loglik_scratch_address(double** out)
{
    static std::mutex mu;
    static std::vector<double*> addr;
    int dev = 0;
    ALTOB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if ((size_t)dev >= addr.size()) addr.resize((size_t)dev + 1, nullptr);
    if (!addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_loglik_scratch);
        if (e != cudaSuccess || !p)
            return fail(ALTOB_ERR_CUDA, std::string("cudaGetSymbolAddress(g_loglik_scratch): ") + cudaGetErrorString(e));
        addr[dev] = (double*)p;
    }
    *out = addr[dev];
    return ALTOB_OK;
}

}  // namespace altob

extern "C" altob_status altob_loglik_noalloc(altob_tensor* t, altob_dtype ftype, void* const* d_factors,
                                             void* d_lambda, uint64_t rank, double eps_div_zero, double* loglik,
                                             void* stream)
{
    if (rank > (uint64_t)LOGLIK_NOALLOC_MAX_RANK)
        return fail(ALTOB_ERR_ARG, "altob_loglik_noalloc: rank " + std::to_string(rank) +
                                       " exceeds the fixed scratch (maximum rank " +
                                       std::to_string(LOGLIK_NOALLOC_MAX_RANK) + ")");
    ALTOB_TRY(check_model(t, ftype, d_factors, rank));
    if (!d_lambda || !loglik) return fail(ALTOB_ERR_ARG, "NULL argument");
    double* d = nullptr;
    ALTOB_TRY(loglik_scratch_address(&d));
    cudaStream_t st = (cudaStream_t)stream;
    const int R = (int)rank;
    // every scratch word is written before it is read in this call:
    // lambda is loaded from d_lambda, the others are zeroed by their kernels
    double *lam = d, *colacc = d + R, *ll = d + 2 * R, *fsum = d + 2 * R + 1;
    if (ftype == ALTOB_F64) {
        ALTOB_TRY(vec_from<double>(lam, (const double*)d_lambda, R, st));
        ALTOB_TRY(loglik_impl<double>(t, (double**)d_factors, lam, colacc, ll, fsum, R, eps_div_zero, loglik, st));
        ALTOB_TRY(vec_to<double>((double*)d_lambda, lam, R, st));
    } else {
        ALTOB_TRY(vec_from<float>(lam, (const float*)d_lambda, R, st));
        ALTOB_TRY(loglik_impl<float>(t, (float**)d_factors, lam, colacc, ll, fsum, R, eps_div_zero, loglik, st));
        ALTOB_TRY(vec_to<float>((float*)d_lambda, lam, R, st));
    }
    ALTOB_CUDA(cudaStreamSynchronize(st));
    return ALTOB_OK;
}
