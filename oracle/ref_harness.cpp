// ref_harness.cpp -- a thin C-ABI harness around the UNMODIFIED reference
// (IntelLabs/ALTO headers include/alto.hpp, cpd.hpp, apr.hpp and sources
// src/kruskal_model.cpp, src/sptensor.cpp, src/common.cpp, compiled in place
// by oracle/build_ref.sh into oracle/_ref/libaltoref.so).
//
// TEST INFRASTRUCTURE ONLY.  It lets tests/golden/make_golden.py write
// fixtures from the reference itself and lets bench.py time the reference's
// OpenMP CPU path.  Nothing in alto_b200/ links or loads it.
//
// Every entry point builds the reference's own SparseTensor / KruskalModel /
// AltoTensor and calls the reference's functions unchanged:
//   create_alto         include/alto.hpp:108
//   create_da_mem       include/alto.hpp:324
//   mttkrp_alto_par     include/alto.hpp:617
//   cpd_alto            include/cpd.hpp:43
//   cp_apr_alto         include/apr.hpp:984
//   KruskalModelRandomInit  src/kruskal_model.cpp:109
// Per-iteration fits and the APR summary are only printed by the reference,
// so they are recovered by capturing its stdout.
#include "alto.hpp"
#include "cpd.hpp"
#include "apr.hpp"

#include <cstring>
#include <type_traits>
#include <string>
#include <vector>

namespace {

SparseTensor* make_spt(int nmode, const uint64_t* dims, uint64_t nnz,
                       const uint64_t* cidx, const double* vals)
{
    SparseTensor* X = (SparseTensor*)AlignedMalloc(sizeof(SparseTensor));
    X->nmodes = nmode;
    X->nnz = nnz;
    X->dims = (IType*)AlignedMalloc(sizeof(IType) * nmode);
    X->cidx = (IType**)AlignedMalloc(sizeof(IType*) * nmode);
    for (int n = 0; n < nmode; ++n) {
        X->dims[n] = dims[n];
        X->cidx[n] = (IType*)AlignedMalloc(sizeof(IType) * nnz);
        memcpy(X->cidx[n], cidx + (uint64_t)n * nnz, sizeof(IType) * nnz);
    }
    X->vals = (FType*)AlignedMalloc(sizeof(FType) * nnz);
    memcpy(X->vals, vals, sizeof(FType) * nnz);
    return X;
}

template <typename LIT>
void put_lit(LIT v, uint64_t* out)
{
    out[0] = (uint64_t)v;
    out[1] = sizeof(LIT) > 8 ? (uint64_t)((unsigned __int128)v >> 64) : 0;
}

template <typename LIT>
void dump(AltoTensor<LIT>* AT, uint64_t* idx, double* vals, uint64_t* prtn_ptr,
          uint64_t* intervals, uint64_t* masks, uint64_t* cr_masks,
          uint64_t* oidx, int* info)
{
    uint64_t nnz = AT->nnz;
    int nm = AT->nmode, np = AT->nprtn;
    for (uint64_t i = 0; i < nnz; ++i) {
        put_lit<LIT>(AT->idx[i], idx + 2 * i);
        vals[i] = (double)AT->vals[i];
    }
    for (int p = 0; p <= np; ++p) prtn_ptr[p] = AT->prtn_ptr[p];
    for (int k = 0; k < np * nm; ++k) {
        intervals[2 * k] = AT->prtn_intervals[k].start;
        intervals[2 * k + 1] = AT->prtn_intervals[k].stop;
    }
    for (int n = 0; n < nm; ++n) {
        put_lit<LIT>(AT->mode_masks[n], masks + 2 * n);
        put_lit<LIT>(AT->cr_masks[n], cr_masks + 2 * n);
        if (AT->is_oidx && AT->oidx[n])
            memcpy(oidx + (uint64_t)n * nnz, AT->oidx[n], sizeof(IType) * nnz);
    }
    info[0] = popcount(AT->alto_mask);
    info[1] = AT->is_oidx ? 1 : 0;
}

// Runs fn with stdout redirected to a temporary file; returns the text.
template <typename F>
std::string capture_stdout(F fn)
{
    fflush(stdout);
    FILE* tmp = tmpfile();
    int saved = dup(fileno(stdout));
    dup2(fileno(tmp), fileno(stdout));
    fn();
    fflush(stdout);
    dup2(saved, fileno(stdout));
    close(saved);
    std::string text;
    rewind(tmp);
    char buf[4096];
    size_t n;
    while ((n = fread(buf, 1, sizeof(buf), tmp)) > 0) text.append(buf, n);
    fclose(tmp);
    return text;
}

void copy_model_out(KruskalModel* M, double* const* U_out, double* lambda_out)
{
    for (int n = 0; n < M->mode; ++n)
        memcpy(U_out[n], M->U[n], sizeof(FType) * M->dims[n] * M->rank);
    memcpy(lambda_out, M->lambda, sizeof(FType) * M->rank);
}

template <typename LIT>
int run_create(SparseTensor* X, int nprtn, uint64_t* idx, double* vals,
               uint64_t* prtn_ptr, uint64_t* intervals, uint64_t* masks,
               uint64_t* cr_masks, uint64_t* oidx, int* info)
{
    AltoTensor<LIT>* AT = nullptr;
    capture_stdout([&] { create_alto(X, &AT, nprtn); });
    dump(AT, idx, vals, prtn_ptr, intervals, masks, cr_masks, oidx, info);
    destroy_alto(AT);
    return 0;
}

template <typename LIT>
int run_mttkrp(SparseTensor* X, int nprtn, int mode, double* const* factors,
               uint64_t rank)
{
    AltoTensor<LIT>* AT = nullptr;
    FType** ofibs = nullptr;
    capture_stdout([&] {
        create_alto(X, &AT, nprtn);
        create_da_mem(-1, rank, AT, &ofibs);
        mttkrp_alto_par(mode, (FType**)factors, rank, AT, NULL, ofibs);
    });
    destroy_da_mem(AT, ofibs, rank, -1);
    destroy_alto(AT);
    return 0;
}

template <typename LIT>
int run_cpd(SparseTensor* X, int nprtn, uint64_t rank, int max_iters,
            double eps, unsigned seed, double* const* U_out,
            double* lambda_out, double* fits)
{
    KruskalModel* M = nullptr;
    CreateKruskalModel(X->nmodes, X->dims, rank, &M);
    KruskalModelRandomInit(M, seed);
    AltoTensor<LIT>* AT = nullptr;
    std::string out = capture_stdout([&] {
        create_alto(X, &AT, nprtn);
        cpd_alto(AT, M, max_iters, eps);
    });
    int iters = 0;
    size_t pos = 0;
    while ((pos = out.find("it: ", pos)) != std::string::npos) {
        int it;
        double fit;
        if (sscanf(out.c_str() + pos, "it: %d\t fit: %lf", &it, &fit) == 2 &&
            it >= 0 && it < max_iters) {
            fits[it] = fit;
            iters = it + 1;
        }
        pos += 4;
    }
    copy_model_out(M, U_out, lambda_out);
    destroy_alto(AT);
    DestroyKruskalModel(M);
    return iters;
}

double find_num(const std::string& s, const char* key)
{
    size_t p = s.find(key);
    if (p == std::string::npos) return NAN;
    return atof(s.c_str() + p + strlen(key));
}

template <typename LIT>
int run_apr(SparseTensor* X, int nprtn, uint64_t rank, int max_iters,
            int max_inner, double eps, double eps_div_zero, double kappa_tol,
            double kappa, int dobench, unsigned seed, double* const* U_out,
            double* lambda_out, double* summary)
{
    KruskalModel* M = nullptr;
    CreateKruskalModel(X->nmodes, X->dims, rank, &M);
    KruskalModelRandomInit(M, seed);
    AltoTensor<LIT>* AT = nullptr;
    std::string out = capture_stdout([&] {
        create_alto(X, &AT, nprtn);
        cp_apr_alto(AT, M, max_iters, max_inner, eps, eps_div_zero, kappa_tol,
                    kappa, dobench != 0);
    });
    summary[0] = find_num(out, "Final log-likelihood = ");
    summary[1] = find_num(out, "Final least squares fit = ");
    summary[2] = find_num(out, "Final KKT violation = ");
    summary[3] = find_num(out, "Total outer iterations = ");
    summary[4] = find_num(out, "Total inner iterations = ");
    copy_model_out(M, U_out, lambda_out);
    destroy_alto(AT);
    DestroyKruskalModel(M);
    return 0;
}

template <typename LIT>
double run_bench(SparseTensor* X, int nprtn, uint64_t rank, int iters,
                 unsigned seed, double* create_s)
{
    // BenchmarkAlto (src/main.cpp:386-518), ALS branch: warm-up sweep, then
    // `iters` sweeps of mttkrp_alto_par over every mode, factors never reset.
    int nm = X->nmodes;
    KruskalModel* M = nullptr;
    CreateKruskalModel(nm, X->dims, rank, &M);
    KruskalModelRandomInit(M, seed);
    AltoTensor<LIT>* AT = nullptr;
    FType** ofibs = nullptr;
    double t = 0.0;
    capture_stdout([&] {
        double t0 = omp_get_wtime();
        create_alto(X, &AT, nprtn);
        *create_s = omp_get_wtime() - t0;
        create_da_mem(-1, rank, AT, &ofibs);
        for (int m = 0; m < nm; ++m) mttkrp_alto_par(m, M->U, rank, AT, NULL, ofibs);
        t0 = omp_get_wtime();
        for (int i = 0; i < iters; ++i)
            for (int m = 0; m < nm; ++m) mttkrp_alto_par(m, M->U, rank, AT, NULL, ofibs);
        t = omp_get_wtime() - t0;
    });
    destroy_da_mem(AT, ofibs, rank, -1);
    destroy_alto(AT);
    DestroyKruskalModel(M);
    return t;
}

} // namespace

extern "C" {

int ref_max_threads(void) { return omp_get_max_threads(); }

// The reference's file reader, ImportSparseTensor (src/sptensor.cpp:165-258,
// text format :75-161): ref_read_open reads the file (the path must name a
// readable file; the reference asserts otherwise) and reports its order and
// nonzero count; ref_read_take copies dims, the mode-major coordinates and
// the values out and frees the tensor.
void* ref_read_open(const char* path, int binary, uint64_t zero_based, int* nmode, uint64_t* nnz)
{
    SparseTensor* X = nullptr;
    ImportSparseTensor(path, binary ? BINARY_FORMAT : TEXT_FORMAT, &X, (IType)zero_based);
    *nmode = X->nmodes;
    *nnz = X->nnz;
    return X;
}

// The reference's writer, ExportSparseTensor (src/sptensor.cpp:23-70).
void ref_write(const char* path, int binary, int nmode, const uint64_t* dims, uint64_t nnz,
               const uint64_t* cidx, const double* vals)
{
    SparseTensor* X = make_spt(nmode, dims, nnz, cidx, vals);
    ExportSparseTensor(path, binary ? BINARY_FORMAT : TEXT_FORMAT, X);
    DestroySparseTensor(X);
}

void ref_read_take(void* p, uint64_t* dims, uint64_t* cidx, double* vals)
{
    SparseTensor* X = static_cast<SparseTensor*>(p);
    const uint64_t nnz = X->nnz;
    for (int n = 0; n < X->nmodes; ++n) {
        dims[n] = X->dims[n];
        memcpy(cidx + (size_t)n * nnz, X->cidx[n], nnz * sizeof(uint64_t));
    }
    memcpy(vals, X->vals, nnz * sizeof(double));
    DestroySparseTensor(X);
}

int ref_create_dump(int nmode, const uint64_t* dims, uint64_t nnz,
                    const uint64_t* cidx, const double* vals, int nprtn,
                    int lit_bits, uint64_t* idx, double* vals_out,
                    uint64_t* prtn_ptr, uint64_t* intervals, uint64_t* masks,
                    uint64_t* cr_masks, uint64_t* oidx, int* info)
{
    SparseTensor* X = make_spt(nmode, dims, nnz, cidx, vals);
    int rc = lit_bits == 128
        ? run_create<unsigned __int128>(X, nprtn, idx, vals_out, prtn_ptr, intervals, masks, cr_masks, oidx, info)
        : run_create<unsigned long long>(X, nprtn, idx, vals_out, prtn_ptr, intervals, masks, cr_masks, oidx, info);
    DestroySparseTensor(X);
    return rc;
}

int ref_mttkrp(int nmode, const uint64_t* dims, uint64_t nnz,
               const uint64_t* cidx, const double* vals, int nprtn,
               int lit_bits, int mode, double* const* factors, uint64_t rank)
{
    SparseTensor* X = make_spt(nmode, dims, nnz, cidx, vals);
    int rc = lit_bits == 128
        ? run_mttkrp<unsigned __int128>(X, nprtn, mode, factors, rank)
        : run_mttkrp<unsigned long long>(X, nprtn, mode, factors, rank);
    DestroySparseTensor(X);
    return rc;
}

int ref_cpd(int nmode, const uint64_t* dims, uint64_t nnz,
            const uint64_t* cidx, const double* vals, int nprtn, int lit_bits,
            uint64_t rank, int max_iters, double eps, unsigned seed,
            double* const* U_out, double* lambda_out, double* fits)
{
    SparseTensor* X = make_spt(nmode, dims, nnz, cidx, vals);
    int it = lit_bits == 128
        ? run_cpd<unsigned __int128>(X, nprtn, rank, max_iters, eps, seed, U_out, lambda_out, fits)
        : run_cpd<unsigned long long>(X, nprtn, rank, max_iters, eps, seed, U_out, lambda_out, fits);
    DestroySparseTensor(X);
    return it;
}

int ref_apr(int nmode, const uint64_t* dims, uint64_t nnz,
            const uint64_t* cidx, const double* vals, int nprtn, int lit_bits,
            uint64_t rank, int max_iters, int max_inner, double eps,
            double eps_div_zero, double kappa_tol, double kappa, int dobench,
            unsigned seed, double* const* U_out, double* lambda_out,
            double* summary)
{
    SparseTensor* X = make_spt(nmode, dims, nnz, cidx, vals);
    int rc = lit_bits == 128
        ? run_apr<unsigned __int128>(X, nprtn, rank, max_iters, max_inner, eps, eps_div_zero, kappa_tol, kappa, dobench, seed, U_out, lambda_out, summary)
        : run_apr<unsigned long long>(X, nprtn, rank, max_iters, max_inner, eps, eps_div_zero, kappa_tol, kappa, dobench, seed, U_out, lambda_out, summary);
    DestroySparseTensor(X);
    return rc;
}

double ref_bench_mttkrp(int nmode, const uint64_t* dims, uint64_t nnz,
                        const uint64_t* cidx, const double* vals, int nprtn,
                        int lit_bits, uint64_t rank, int iters, unsigned seed,
                        double* create_s)
{
    SparseTensor* X = make_spt(nmode, dims, nnz, cidx, vals);
    double t = lit_bits == 128
        ? run_bench<unsigned __int128>(X, nprtn, rank, iters, seed, create_s)
        : run_bench<unsigned long long>(X, nprtn, rank, iters, seed, create_s);
    DestroySparseTensor(X);
    return t;
}

// OPT_ALTO partition subspace ids (alto.hpp:838-868) of the encoding
// create_alto builds; -1 in builds without OPT_ALTO.
int ref_prtn_ids(int nmode, const uint64_t* dims, uint64_t nnz, const uint64_t* cidx, const double* vals, int nprtn,
                 int lit_bits, uint64_t* prtn_id, uint64_t* prtn_mask, uint64_t* prtn_mode_masks)
{
#ifdef OPT_ALTO
    SparseTensor* X = make_spt(nmode, dims, nnz, cidx, vals);
    auto run = [&](auto* tag) {
        using LIT = std::remove_pointer_t<decltype(tag)>;
        AltoTensor<LIT>* AT = nullptr;
        capture_stdout([&] { create_alto(X, &AT, nprtn); });
        for (int p = 0; p < nprtn; ++p) {
            prtn_id[p] = AT->prtn_id[p];
            prtn_mask[p] = AT->prtn_mask[p];
            for (int n = 0; n < nmode; ++n) prtn_mode_masks[(size_t)p * nmode + n] = AT->prtn_mode_masks[p * nmode + n];
        }
        destroy_alto(AT);
    };
    if (lit_bits == 128) run((unsigned __int128*)nullptr);
    else run((unsigned long long*)nullptr);
    DestroySparseTensor(X);
    return 0;
#else
    (void)nmode; (void)dims; (void)nnz; (void)cidx; (void)vals; (void)nprtn; (void)lit_bits;
    (void)prtn_id; (void)prtn_mask; (void)prtn_mode_masks;
    return -1;
#endif
}

} // extern "C"
