// cpd64.cpp -- command-line driver with the reference's flags
// (IntelLabs/ALTO src/main.cpp:70-92), written against the C++ drop-in
// header include/alto_dropin.hpp, so it also shows that header in use.
//
//   cpd64 -l als|apr -i file.tns | -b file.bin [--rank R] [-m iters]
//         [-n inner] [-e eps] [-x seed] [-t mode] [-z] [-c] [-p]
//
// -c   MTTKRP check against a sequential COO MTTKRP on the host
//      (RunAltoCheck, main.cpp:520-650; absolute tolerance 1e-6)
// -p   benchmark (BenchmarkAlto, main.cpp:386-518): prints "ALTO runtime"
// Built twice: cpd64 (FP64 model) and cpd64_fp32 (-DALTOB_FP32).
// -d (the reference's built-in Poisson generator) is not provided.
#include <getopt.h>
#include <omp.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <string>
#include <vector>

#include "alto_dropin.hpp"

typedef unsigned __int128 LIT128;
typedef unsigned long long LIT64;

static const struct option long_opt[] = {
    {"help", 0, NULL, 'h'},        {"version", 0, NULL, 'v'},     {"input", 1, NULL, 'i'},
    {"output", 1, NULL, 'o'},      {"bin", 1, NULL, 'b'},         {"model", 1, NULL, 'l'},
    {"rank", 1, NULL, 'r'},        {"max-iter", 1, NULL, 'm'},    {"max-inner", 1, NULL, 'n'},
    {"seed", 1, NULL, 'x'},        {"dims", 1, NULL, 'd'},        {"target-mode", 1, NULL, 't'},
    {"sparsity", 1, NULL, 's'},    {"epsilon", 1, NULL, 'e'},     {"file", 1, NULL, 'f'},
    {"zero-based", 0, NULL, 'z'},  {"check", 0, NULL, 'c'},       {"bench", 0, NULL, 'p'},
    {"nprtn", 1, NULL, 'P'},       {NULL, 0, NULL, 0}};

static void usage(const char* call)
{
    printf("Usage: %s [options]\n"
           "  -i, --input <file>     .tns text tensor\n"
           "  -b, --bin <file>       binary tensor\n"
           "  -d, --dims <I,J,...>   generate a Poisson count tensor of these dims (rank -r)\n"
           "  -s, --sparsity <f>     with -d: draws = f x prod(dims) (default 0.1)\n"
           "  -l, --model als|apr    decomposition\n"
           "  -r, --rank <R>         rank (default 16)\n"
           "  -m, --max-iter <N>     iterations (default 10)\n"
           "  -n, --max-inner <N>    CP-APR inner iterations (default 10)\n"
           "  -e, --epsilon <e>      tolerance (default 1e-5)\n"
           "  -x, --seed <s>         random seed (default time)\n"
           "  -t, --target-mode <n>  mode for -c / -p (default all)\n"
           "  -z, --zero-based       0-based .tns indices\n"
           "  -c, --check            MTTKRP check against a COO MTTKRP\n"
           "  -p, --bench            benchmark mode\n"
           "      --nprtn <P>        partitions of the encoding (default: OpenMP threads)\n",
           call);
}

static double now()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <typename LIT>
static int run(SparseTensor* X, bool is_apr, bool do_check, bool do_bench, IType rank, int max_iters, int max_inner,
               double epsilon, int seed, int target_mode, int nprtn)
{
    KruskalModel* M = nullptr;
    CreateKruskalModel(X->nmodes, X->dims, rank, &M);
    KruskalModelRandomInit(M, (unsigned)seed);
    if (do_check) {
        // truth: sequential COO MTTKRP (cpd.hpp:509-543) onto the initial factors
        int n0 = target_mode < 0 ? 0 : target_mode, n1 = target_mode < 0 ? X->nmodes : target_mode + 1;
        AltoTensor<LIT>* AT = nullptr;
        create_alto(X, &AT, nprtn);
        for (int m = n0; m < n1; ++m) {
            std::vector<FType> truth(M->U[m], M->U[m] + X->dims[m] * rank);
            std::vector<FType> row(rank);
            for (IType i = 0; i < X->nnz; ++i) {
                for (IType r = 0; r < rank; ++r) row[r] = X->vals[i];
                for (int q = 0; q < X->nmodes; ++q)
                    if (q != m)
                        for (IType r = 0; r < rank; ++r) row[r] *= M->U[q][X->cidx[q][i] * rank + r];
                for (IType r = 0; r < rank; ++r) truth[X->cidx[m][i] * rank + r] += row[r];
            }
            std::vector<FType> saved(M->U[m], M->U[m] + X->dims[m] * rank);
            mttkrp_alto_par(m, M->U, rank, AT, nullptr, nullptr);
            IType bad = 0;
            for (IType k = 0; k < X->dims[m] * rank; ++k)
                if (std::fabs(truth[k] - M->U[m][k]) > 1.0e-6) ++bad;
            if (bad == 0) fprintf(stderr, "mode %d: Results of mttkrp_alto is correct\n", m);
            else fprintf(stderr, "mode %d: Results of mttkrp_alto is incorrect by %llu\n", m, bad);
            std::copy(saved.begin(), saved.end(), M->U[m]);
            if (bad) {
                destroy_alto(AT);
                DestroyKruskalModel(M);
                return 2;
            }
        }
        destroy_alto(AT);
        DestroyKruskalModel(M);
        return 0;
    }
    AltoTensor<LIT>* AT = nullptr;
    double t0 = now();
    create_alto(X, &AT, nprtn);
    printf("ALTO creation time:   %f\n", now() - t0);
    if (do_bench && !is_apr) {
        int n0 = target_mode < 0 ? 0 : target_mode, n1 = target_mode < 0 ? X->nmodes : target_mode + 1;
        for (int m = n0; m < n1; ++m) mttkrp_alto_par(m, M->U, rank, AT, nullptr, nullptr);  // warm-up
        t0 = now();
        for (int it = 0; it < max_iters; ++it)
            for (int m = n0; m < n1; ++m) mttkrp_alto_par(m, M->U, rank, AT, nullptr, nullptr);
        printf("ALTO runtime:   %f\n", now() - t0);
    } else if (is_apr) {
        t0 = now();
        cp_apr_alto(AT, M, max_iters, max_inner, do_bench ? 0.0 : epsilon, do_bench ? 0.0 : 1.0e-10, 1.0e-10,
                    1.0e-2, do_bench);
        printf("APR (ALTO): %f s\n", now() - t0);
    } else {
        t0 = now();
        cpd_alto(AT, M, max_iters, epsilon);
        printf("ALS (ALTO): %f s\n", now() - t0);
    }
    destroy_alto(AT);
    DestroyKruskalModel(M);
    return 0;
}

int main(int argc, char** argv)
{
    int max_iters = 10, max_inner = 10, target_mode = -1, seed = (int)time(NULL), nprtn = omp_get_max_threads();
    IType rank = 16, zero_based = 0;
    double epsilon = 1e-5;
    std::string text_file, binary_file, model, dims_arg;
    double sparsity = 0.1;  // -s (main.cpp:127)
    bool do_check = false, do_bench = false;
    int c;
    while ((c = getopt_long(argc, argv, "hvi:o:b:l:r:m:n:x:d:t:s:e:f:zcp", long_opt, NULL)) != -1) {
        switch (c) {
        case 'h': usage(argv[0]); return 0;
        case 'v': printf("%s\n", altob_version()); return 0;
        case 'i': text_file = optarg; break;
        case 'b': binary_file = optarg; break;
        case 'l': model = optarg; break;
        case 'r': rank = (IType)atoll(optarg); break;
        case 'm': max_iters = atoi(optarg); break;
        case 'n': max_inner = atoi(optarg); break;
        case 'x': seed = atoi(optarg); break;
        case 't': target_mode = atoi(optarg); break;
        case 'e': epsilon = atof(optarg); break;
        case 'z': zero_based = 1; break;
        case 'c': do_check = true; break;
        case 'p': do_bench = true; break;
        case 'P': nprtn = atoi(optarg); break;
        case 'd': dims_arg = optarg; break;
        case 's': sparsity = atof(optarg); break;
        case 'o': case 'f': break;
        default: usage(argv[0]); return -1;
        }
    }
    if (rank < 1 || max_iters < 1 || max_inner < 1 || seed < 0 || target_mode < -1) {
        fprintf(stderr, "invalid argument\n");
        return -1;
    }
    if (model != "als" && model != "ALS" && model != "apr" && model != "APR" && !do_check) {
        fprintf(stderr, "choose a model with -l als|apr\n");
        return -1;
    }
    const bool is_apr = model == "apr" || model == "APR";
    SparseTensor* X = nullptr;
    try {
        if (!binary_file.empty()) ImportSparseTensor(binary_file.c_str(), BINARY_FORMAT, &X, zero_based);
        else if (!text_file.empty()) ImportSparseTensor(text_file.c_str(), TEXT_FORMAT, &X, zero_based);
        else if (!dims_arg.empty()) {
            // MakeSparseTensor (main.cpp:652-675): sparsity x prod(dims) Poisson
            // draws from a random rank-`rank` model
            std::vector<IType> dims;
            size_t pos = 0;
            while (pos <= dims_arg.size()) {
                const size_t e = dims_arg.find(',', pos);
                dims.push_back((IType)atoll(dims_arg.substr(pos, e == std::string::npos ? e : e - pos).c_str()));
                if (e == std::string::npos) break;
                pos = e + 1;
            }
            IType total = 1;
            for (IType d : dims) total *= d;
            const IType edges = (IType)(sparsity * (double)total);
            PoissonGenerator* pg = nullptr;
            CreatePoissonGenerator((int)dims.size(), dims.data(), &pg);
            KruskalModel* truth = nullptr;
            double t0 = now();
            PoissonGeneratorRun(pg, edges, rank, &truth, &X, omp_get_max_threads());
            printf("Creating a new tensor: %f s (%llu nonzeros)\n", now() - t0, (unsigned long long)X->nnz);
            DestroyPoissonGenerator(pg);
            DestroyKruskalModel(truth);
        } else {
            fprintf(stderr, "no input: use -i, -b or -d\n");
            return -1;
        }
        if (target_mode >= X->nmodes) {
            fprintf(stderr, "invalid target mode\n");
            return -1;
        }
        int bits = 0;
        for (int n = 0; n < X->nmodes; ++n)
            if (X->dims[n] > 1) bits += 64 - __builtin_clzll(X->dims[n] - 1);
        int rc = bits <= 64 ? run<LIT64>(X, is_apr, do_check, do_bench, rank, max_iters, max_inner, epsilon, seed,
                                          target_mode, nprtn)
                            : run<LIT128>(X, is_apr, do_check, do_bench, rank, max_iters, max_inner, epsilon, seed,
                                          target_mode, nprtn);
        DestroySparseTensor(X);
        return rc;
    } catch (const std::exception& e) {
        fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
}
