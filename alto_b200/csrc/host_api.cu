// host_api.cu -- solver entry points on host-resident models, the calling
// convention of the reference's cpd_alto / cp_apr_alto (KruskalModel in host
// memory): the model is copied to the device, solved, and copied back.
#include <vector>

#include "internal.cuh"

using namespace altob;

namespace {

struct DevModel {
    std::vector<void*> U;
    void* lam = nullptr;
    ~DevModel()
    {
        for (void* p : U) dfree(p);
        dfree(lam);
    }
};

altob_status upload(const altob_tensor* t, size_t fsz, void* const* hU, const void* hl, u64 R, DevModel& m,
                    cudaStream_t st)
{
    m.U.assign(t->nmode, nullptr);
    for (int n = 0; n < t->nmode; ++n) {
        if (!hU[n]) return fail(ALTOB_ERR_ARG, "a host factor pointer is NULL");
        ALTOB_TRY(dmalloc(&m.U[n], t->dims[n] * R * fsz));
        ALTOB_CUDA(cudaMemcpyAsync(m.U[n], hU[n], t->dims[n] * R * fsz, cudaMemcpyHostToDevice, st));
    }
    ALTOB_TRY(dmalloc(&m.lam, R * fsz));
    ALTOB_CUDA(cudaMemcpyAsync(m.lam, hl, R * fsz, cudaMemcpyHostToDevice, st));
    return ALTOB_OK;
}

altob_status download(const altob_tensor* t, size_t fsz, void* const* hU, void* hl, u64 R, DevModel& m,
                      cudaStream_t st)
{
    for (int n = 0; n < t->nmode; ++n)
        ALTOB_CUDA(cudaMemcpyAsync(hU[n], m.U[n], t->dims[n] * R * fsz, cudaMemcpyDeviceToHost, st));
    ALTOB_CUDA(cudaMemcpyAsync(hl, m.lam, R * fsz, cudaMemcpyDeviceToHost, st));
    ALTOB_CUDA(cudaStreamSynchronize(st));
    return ALTOB_OK;
}

}  // namespace

extern "C" {

altob_status altob_cpd_als_host(altob_tensor* t, altob_dtype ftype, void* const* h_factors, void* h_lambda,
                                uint64_t rank, int max_iters, double epsilon, double* fits, int* iters,
                                void* stream)
{
    if (!t || !h_factors || !h_lambda) return fail(ALTOB_ERR_ARG, "NULL argument");
    if (ftype != ALTOB_F64 && ftype != ALTOB_F32) return fail(ALTOB_ERR_ARG, "dtype must be F64 or F32");
    cudaStream_t st = (cudaStream_t)stream;
    StreamScope scope(st);
    const size_t fsz = ftype == ALTOB_F64 ? 8 : 4;
    DevModel m;
    ALTOB_TRY(upload(t, fsz, h_factors, h_lambda, rank, m, st));
    ALTOB_TRY(altob_cpd_als(t, ftype, m.U.data(), m.lam, rank, max_iters, epsilon, fits, iters, stream));
    return download(t, fsz, h_factors, h_lambda, rank, m, st);
}

altob_status altob_cp_apr_host(altob_tensor* t, altob_dtype ftype, void* const* h_factors, void* h_lambda,
                               uint64_t rank, int max_iters, int max_inner, double epsilon, double eps_div_zero,
                               double kappa_tol, double kappa, int dobench, double* summary, void* stream)
{
    if (!t || !h_factors || !h_lambda) return fail(ALTOB_ERR_ARG, "NULL argument");
    if (ftype != ALTOB_F64 && ftype != ALTOB_F32) return fail(ALTOB_ERR_ARG, "dtype must be F64 or F32");
    cudaStream_t st = (cudaStream_t)stream;
    StreamScope scope(st);
    const size_t fsz = ftype == ALTOB_F64 ? 8 : 4;
    DevModel m;
    ALTOB_TRY(upload(t, fsz, h_factors, h_lambda, rank, m, st));
    ALTOB_TRY(altob_cp_apr(t, ftype, m.U.data(), m.lam, rank, max_iters, max_inner, epsilon, eps_div_zero,
                           kappa_tol, kappa, dobench, summary, stream));
    return download(t, fsz, h_factors, h_lambda, rank, m, st);
}

}  // extern "C"
