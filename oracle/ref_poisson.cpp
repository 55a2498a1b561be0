// ref_poisson.cpp -- C-ABI harness around the UNMODIFIED reference generator
// (IntelLabs/ALTO src/poisson_generator.cpp, src/rng.cpp, src/rng_stream.cpp,
// compiled in place by oracle/build_ref.sh into
// oracle/_ref/libaltoref_poisson.so).
//
// TEST INFRASTRUCTURE ONLY: tests compare alto_b200's device generator with
// the reference's PoissonGeneratorRun (poisson_generator.cpp:337-375) for a
// fixed OpenMP thread count.  Nothing in alto_b200/ links or loads it.
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "poisson_generator.hpp"

extern "C" {

// Runs the reference's generator with `nthreads` OpenMP threads and the C
// library's rand() reset to its initial state (as at the start of the
// reference's cpd64 -d); returns the tensor handle and its nonzero count.
// The generator's progress lines go to /dev/null.
void* refp_run(int nmode, const uint64_t* dims, uint64_t num_edges, uint64_t rank, int nthreads, uint64_t* nnz,
               double* const* U_out, double* lambda_out)
{
    omp_set_num_threads(nthreads);
    srand(1);
    IType d[16];
    for (int n = 0; n < nmode; ++n) d[n] = dims[n];
    fflush(stdout);
    int saved = dup(fileno(stdout));
    FILE* devnull = fopen("/dev/null", "w");
    dup2(fileno(devnull), fileno(stdout));
    PoissonGenerator* pg = nullptr;
    CreatePoissonGenerator(nmode, d, &pg);
    KruskalModel* M = nullptr;
    SparseTensor* X = nullptr;
    PoissonGeneratorRun(pg, num_edges, rank, &M, &X);
    DestroyPoissonGenerator(pg);
    fflush(stdout);
    dup2(saved, fileno(stdout));
    close(saved);
    fclose(devnull);
    for (int n = 0; n < nmode; ++n)
        if (U_out && U_out[n]) memcpy(U_out[n], M->U[n], sizeof(FType) * dims[n] * rank);
    if (lambda_out) memcpy(lambda_out, M->lambda, sizeof(FType) * rank);
    DestroyKruskalModel(M);
    *nnz = X->nnz;
    return X;
}

// Copies the tensor out (mode-major coordinates, values) and frees it.
void refp_take(void* p, uint64_t* cidx, double* vals)
{
    SparseTensor* X = static_cast<SparseTensor*>(p);
    for (int n = 0; n < X->nmodes; ++n) memcpy(cidx + (size_t)n * X->nnz, X->cidx[n], X->nnz * sizeof(IType));
    memcpy(vals, X->vals, X->nnz * sizeof(FType));
    DestroySparseTensor(X);
}

}  // extern "C"
