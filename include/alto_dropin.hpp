// alto_dropin.hpp -- C++ drop-in for IntelLabs/ALTO's operator surface,
// header only, over the C ABI of libaltob.so (include/altob.h).
//
// The reference's names, argument meanings and host data structures are
// kept so a caller of the reference compiles against this header instead:
//
//   SparseTensor, ImportSparseTensor, ExportSparseTensor,
//   DestroySparseTensor                 include/sptensor.hpp:8-47
//   KruskalModel, CreateKruskalModel, KruskalModelRandomInit,
//   DestroyKruskalModel                 include/kruskal_model.hpp:8-45
//   AltoTensor<LIT>, create_alto, destroy_alto, create_da_mem,
//   destroy_da_mem, mttkrp_alto_par     include/alto.hpp:27-80, 617
//   cpd_alto                            include/cpd.hpp:27
//   cp_apr_alto                         include/apr.hpp:34
//
// Differences: the ALTO encoding lives on the GPU (AltoTensor holds a
// handle, not host arrays); create_da_mem / destroy_da_mem are no-ops
// because the per-segment temporary rows live in shared memory; errors throw
// std::runtime_error with the library's status text instead of asserting.
// FType is double unless ALTOB_FP32 is defined (the FP32 model of the
// B200 path); values are stored as FType unless ALTOB_VAL_UINT32 is defined.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "altob.h"

typedef unsigned long long IType;
#ifdef ALTOB_FP32
typedef float FType;
static const altob_dtype ALTOB_FTYPE = ALTOB_F32;
#else
typedef double FType;
static const altob_dtype ALTOB_FTYPE = ALTOB_F64;
#endif
#ifdef ALTOB_VAL_UINT32
static const altob_dtype ALTOB_VTYPE = ALTOB_U32;
#else
static const altob_dtype ALTOB_VTYPE = ALTOB_FTYPE;
#endif

namespace altob_detail {
inline void check(altob_status s, const char* what)
{
    if (s != ALTOB_OK)
        throw std::runtime_error(std::string(what) + ": " + altob_status_string(s) + ": " + altob_last_error());
}
}  // namespace altob_detail

// ---------------------------------------------------------------- COO
struct SparseTensor {
    int nmodes;
    IType* dims;
    IType nnz;
    IType** cidx;  // nmodes pointers into one SoA block
    FType* vals;
};

typedef enum FileFormat_ { TEXT_FORMAT = 0, BINARY_FORMAT = 1 } FileFormat;

inline void DestroySparseTensor(SparseTensor* X)
{
    if (!X) return;
    free(X->dims);
    if (X->cidx) free(X->cidx[0]);
    free(X->cidx);
    free(X->vals);
    free(X);
}

inline void ImportSparseTensor(const char* file_path, FileFormat f, SparseTensor** X_, IType zero_based)
{
    altob_coo* c = nullptr;
    altob_detail::check(f == TEXT_FORMAT ? altob_read_tns(file_path, (int)zero_based, &c)
                                         : altob_read_bin(file_path, &c),
                        "ImportSparseTensor");
    SparseTensor* X = (SparseTensor*)calloc(1, sizeof(SparseTensor));
    X->nmodes = c->nmode;
    X->nnz = c->nnz;
    X->dims = (IType*)malloc(sizeof(IType) * c->nmode);
    X->cidx = (IType**)malloc(sizeof(IType*) * c->nmode);
    IType* block = (IType*)malloc(sizeof(IType) * c->nmode * (c->nnz ? c->nnz : 1));
    memcpy(block, c->cidx, sizeof(IType) * c->nmode * c->nnz);
    for (int n = 0; n < c->nmode; ++n) {
        X->dims[n] = c->dims[n];
        X->cidx[n] = block + (size_t)n * c->nnz;
    }
    X->vals = (FType*)malloc(sizeof(FType) * (c->nnz ? c->nnz : 1));
    for (IType i = 0; i < c->nnz; ++i) X->vals[i] = (FType)c->vals[i];
    altob_coo_free(c);
    *X_ = X;
}

inline altob_coo as_coo(const SparseTensor* X, double* vals64)
{
    altob_coo c;
    memset(&c, 0, sizeof(c));
    c.nmode = X->nmodes;
    c.nnz = X->nnz;
    for (int n = 0; n < X->nmodes; ++n) c.dims[n] = X->dims[n];
    c.cidx = (uint64_t*)X->cidx[0];
    for (IType i = 0; i < X->nnz; ++i) vals64[i] = (double)X->vals[i];
    c.vals = vals64;
    return c;
}

inline void ExportSparseTensor(const char* file_path, FileFormat f, SparseTensor* X)
{
    // cidx rows must be one contiguous block (as ImportSparseTensor builds it)
    double* v = (double*)malloc(sizeof(double) * (X->nnz ? X->nnz : 1));
    altob_coo c = as_coo(X, v);
    altob_status s = f == TEXT_FORMAT ? altob_write_tns(file_path, &c) : altob_write_bin(file_path, &c);
    free(v);
    altob_detail::check(s, "ExportSparseTensor");
}

// ------------------------------------------------- Poisson generator
// PoissonGenerator / PoissonGeneratorRun (src/poisson_generator.cpp:
// 99-375) on top of altob_poisson_tensor: the random streams of the
// caller's OpenMP thread count, the edges drawn and merged on the device.
struct PoissonGenerator {
    int mode;
    IType* dims;
};

inline void CreatePoissonGenerator(int mode, IType* dims, PoissonGenerator** pg_)
{
    PoissonGenerator* pg = (PoissonGenerator*)calloc(1, sizeof(PoissonGenerator));
    pg->mode = mode;
    pg->dims = (IType*)malloc(sizeof(IType) * mode);
    memcpy(pg->dims, dims, sizeof(IType) * mode);
    *pg_ = pg;
}

inline void DestroyPoissonGenerator(PoissonGenerator* pg)
{
    if (!pg) return;
    free(pg->dims);
    free(pg);
}

struct KruskalModel;
inline void CreateKruskalModel(int mode, IType* dims, IType rank, KruskalModel** M_);
inline void PoissonGeneratorRun(PoissonGenerator* pg, IType num_edges, IType rank, KruskalModel** M_,
                                SparseTensor** X_, int nthreads);

// ------------------------------------------------------- Kruskal model
struct KruskalModel {
    int mode;
    IType* dims;
    IType rank;
    FType** U;
    FType* lambda;
};

inline void CreateKruskalModel(int mode, IType* dims, IType rank, KruskalModel** M_)
{
    KruskalModel* M = (KruskalModel*)calloc(1, sizeof(KruskalModel));
    M->mode = mode;
    M->rank = rank;
    M->dims = (IType*)malloc(sizeof(IType) * mode);
    memcpy(M->dims, dims, sizeof(IType) * mode);
    M->U = (FType**)malloc(sizeof(FType*) * mode);
    for (int n = 0; n < mode; ++n) M->U[n] = (FType*)malloc(sizeof(FType) * dims[n] * rank);
    M->lambda = (FType*)malloc(sizeof(FType) * rank);
    *M_ = M;
}

// nthreads: the OpenMP thread count whose random streams are replayed (the
// reference uses omp_get_max_threads()).
inline void PoissonGeneratorRun(PoissonGenerator* pg, IType num_edges, IType rank, KruskalModel** M_,
                                SparseTensor** X_, int nthreads)
{
    const int N = pg->mode;
    std::vector<std::vector<double>> U(N);
    std::vector<double*> up(N);
    for (int n = 0; n < N; ++n) {
        U[n].resize(pg->dims[n] * rank);
        up[n] = U[n].data();
    }
    std::vector<double> lam(rank);
    std::vector<uint64_t> d(pg->dims, pg->dims + N);
    altob_coo* c = nullptr;
    altob_detail::check(altob_poisson_tensor(N, d.data(), num_edges, rank, nthreads, up.data(), lam.data(), &c, nullptr),
                        "PoissonGeneratorRun");
    KruskalModel* M = nullptr;
    CreateKruskalModel(N, pg->dims, rank, &M);
    for (int n = 0; n < N; ++n)
        for (IType i = 0; i < pg->dims[n] * rank; ++i) M->U[n][i] = (FType)U[n][i];
    for (IType r = 0; r < rank; ++r) M->lambda[r] = (FType)lam[r];
    SparseTensor* X = (SparseTensor*)calloc(1, sizeof(SparseTensor));
    X->nmodes = c->nmode;
    X->nnz = c->nnz;
    X->dims = (IType*)malloc(sizeof(IType) * c->nmode);
    X->cidx = (IType**)malloc(sizeof(IType*) * c->nmode);
    IType* block = (IType*)malloc(sizeof(IType) * c->nmode * (c->nnz ? c->nnz : 1));
    memcpy(block, c->cidx, sizeof(IType) * c->nmode * c->nnz);
    for (int n = 0; n < c->nmode; ++n) {
        X->dims[n] = c->dims[n];
        X->cidx[n] = block + (size_t)n * c->nnz;
    }
    X->vals = (FType*)malloc(sizeof(FType) * (c->nnz ? c->nnz : 1));
    for (IType i = 0; i < c->nnz; ++i) X->vals[i] = (FType)c->vals[i];
    altob_coo_free(c);
    *M_ = M;
    *X_ = X;
}

inline void KruskalModelRandomInit(KruskalModel* M, unsigned int seed)
{
    altob_detail::check(altob_kruskal_random_init(M->mode, (const uint64_t*)M->dims, M->rank, seed, ALTOB_FTYPE,
                                                  (void* const*)M->U, M->lambda),
                        "KruskalModelRandomInit");
}

inline void DestroyKruskalModel(KruskalModel* M)
{
    if (!M) return;
    for (int n = 0; n < M->mode; ++n) free(M->U[n]);
    free(M->U);
    free(M->lambda);
    free(M->dims);
    free(M);
}

// -------------------------------------------------------- ALTO tensor
template <typename LIT>
struct AltoTensor {
    int nmode;
    int nprtn;
    IType nnz;
    IType* dims;
    altob_tensor* handle;  // device-resident encoding
};

template <typename LIT>
inline void create_alto(SparseTensor* spt, AltoTensor<LIT>** at, int nprtn)
{
    const int lit_bits = (int)sizeof(LIT) * 8;
    void* vals = nullptr;
    std::vector<double> v64;
    std::vector<float> v32;
    std::vector<uint32_t> vu;
    if (ALTOB_VTYPE == ALTOB_F64) {
        v64.assign(spt->vals, spt->vals + spt->nnz);
        vals = v64.data();
    } else if (ALTOB_VTYPE == ALTOB_F32) {
        v32.assign(spt->vals, spt->vals + spt->nnz);
        vals = v32.data();
    } else {
        vu.resize(spt->nnz);
        for (IType i = 0; i < spt->nnz; ++i) vu[i] = (uint32_t)spt->vals[i];
        vals = vu.data();
    }
    // cidx rows may be separate allocations: gather them into SoA
    std::vector<uint64_t> cidx((size_t)spt->nmodes * spt->nnz);
    for (int n = 0; n < spt->nmodes; ++n)
        memcpy(cidx.data() + (size_t)n * spt->nnz, spt->cidx[n], sizeof(uint64_t) * spt->nnz);
    altob_tensor* h = nullptr;
    altob_detail::check(altob_create(spt->nmodes, (const uint64_t*)spt->dims, spt->nnz, cidx.data(), vals,
                                     ALTOB_VTYPE, nprtn, lit_bits, nullptr, &h),
                        "create_alto");
    AltoTensor<LIT>* t = new AltoTensor<LIT>();
    t->nmode = spt->nmodes;
    t->nprtn = nprtn;
    t->nnz = spt->nnz;
    t->dims = new IType[spt->nmodes];
    memcpy(t->dims, spt->dims, sizeof(IType) * spt->nmodes);
    t->handle = h;
    *at = t;
}

template <typename LIT>
inline void destroy_alto(AltoTensor<LIT>* at)
{
    if (!at) return;
    altob_destroy(at->handle);
    delete[] at->dims;
    delete at;
}

// Per-segment temporary rows live in shared memory on the GPU: nothing to
// allocate (alto.hpp:324-398 allocated ofibs on the host).
template <typename LIT>
inline void create_da_mem(int, IType, AltoTensor<LIT>*, FType*** ofibs)
{
    if (ofibs) *ofibs = nullptr;
}

template <typename LIT>
inline void destroy_da_mem(AltoTensor<LIT>*, FType**, IType, int)
{
}

// factors[target_mode] += MTTKRP (alto.hpp:617-623), factors in host memory.
template <typename LIT>
inline void mttkrp_alto_par(int target_mode, FType** factors, IType rank, AltoTensor<LIT>* at, void* /*wlocks*/,
                            FType** /*ofibs*/)
{
    altob_detail::check(altob_mttkrp_host(at->handle, target_mode, ALTOB_FTYPE, (void* const*)factors, rank,
                                          ALTOB_ALGO_AUTO, nullptr),
                        "mttkrp_alto_par");
}

// cpd_alto (cpd.hpp:43-186): prints the reference's per-iteration line.
template <typename LIT>
inline void cpd_alto(AltoTensor<LIT>* AT, KruskalModel* M, int max_iters, double epsilon)
{
    fprintf(stdout, "Running ALTO CP-ALS with %d max iterations and %.2e epsilon\n", max_iters, epsilon);
    std::vector<double> fits(max_iters, 0.0);
    int iters = 0;
    altob_detail::check(altob_cpd_als_host(AT->handle, ALTOB_FTYPE, (void* const*)M->U, M->lambda, M->rank,
                                           max_iters, epsilon, fits.data(), &iters, nullptr),
                        "cpd_alto");
    double prev = 0.0;
    for (int i = 0; i < iters; ++i) {
        printf("it: %d\t fit: %g\t fit-delta: %g\n", i, fits[i], fabs(prev - fits[i]));
        prev = fits[i];
    }
}

// cp_apr_alto (apr.hpp:984-1376): prints the reference's summary lines.
template <typename LIT>
inline void cp_apr_alto(AltoTensor<LIT>* AT, KruskalModel* M, int max_iters, int max_inner_iters, FType epsilon,
                        FType eps_div_zero, FType kappa_tol, FType kappa, bool dobench)
{
    double s[5] = {0, 0, 0, 0, 0};
    altob_detail::check(altob_cp_apr_host(AT->handle, ALTOB_FTYPE, (void* const*)M->U, M->lambda, M->rank,
                                          max_iters, max_inner_iters, epsilon, eps_div_zero, kappa_tol, kappa,
                                          dobench ? 1 : 0, s, nullptr),
                        "cp_apr_alto");
    fprintf(stdout, "  Final log-likelihood = %e\n", s[0]);
    fprintf(stdout, "  Final least squares fit = %e\n", s[1]);
    fprintf(stdout, "  Final KKT violation = %7.7e\n", s[2]);
    fprintf(stdout, "  Total outer iterations = %d\n", (int)s[3]);
    fprintf(stdout, "  Total inner iterations = %d\n", (int)s[4]);
}
