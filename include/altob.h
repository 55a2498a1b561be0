/*
 * altob.h -- C ABI of alto_b200, a B200-native (sm_100a) implementation of
 * the ALTO hot path: linearized-tensor build, MTTKRP on every mode from one
 * tensor copy, and the CP-ALS / CP-APR updates that consume it.
 *
 * Plain C types only: host pointers, device pointers (void*), sizes and a
 * cudaStream_t passed as void* (NULL = the legacy default stream).  Every
 * entry point returns an altob_status; none asserts or exits.  A tensor
 * handle is device resident, stream ordered, and must be used by one host
 * thread at a time.
 *
 * Each declaration names the reference interface it replaces
 * (IntelLabs/ALTO v0.1.2, file:line).
 */
#ifndef ALTOB_H_
#define ALTOB_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define ALTOB_API __attribute__((visibility("default")))
#else
#define ALTOB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define ALTOB_MAX_MODES 5 /* config.mk:27 MAX_NUM_MODES */

typedef enum {
    ALTOB_OK = 0,
    ALTOB_ERR_ARG = 1,         /* invalid argument */
    ALTOB_ERR_BITS = 2,        /* ALTO bits exceed the index width (alto.hpp:709) */
    ALTOB_ERR_CUDA = 3,        /* a CUDA runtime call or kernel failed */
    ALTOB_ERR_NOMEM = 4,       /* device or host allocation failed */
    ALTOB_ERR_IO = 5,          /* file missing or malformed */
    ALTOB_ERR_UNSUPPORTED = 6, /* dtype / size combination not built */
    ALTOB_ERR_NOT_FOUND = 7    /* no CUDA device */
} altob_status;

typedef enum {
    ALTOB_F64 = 0, /* double (reference FType/ValType default, common.hpp:45-69) */
    ALTOB_F32 = 1, /* float  (FP_TYPE32) */
    ALTOB_U32 = 2  /* uint32 counts (VAL_TYPE_INT32), values only */
} altob_dtype;

/* MTTKRP conflict-resolution strategy.  AUTO follows the reference dispatch
 * (alto.hpp:554-563): fiber reuse nnz/I_n > 4 -> TILED (the GPU form of
 * da_mem_pull), else OPSCHED when oidx exists, else ATOMIC_CR / ATOMIC. */
typedef enum {
    ALTOB_ALGO_AUTO = 0,
    ALTOB_ALGO_TILED = 1,     /* per-tile shared-memory row accumulators, atomic flush */
    ALTOB_ALGO_ATOMIC = 2,    /* mttkrp_alto_atomic (alto.hpp:1030-1088) */
    ALTOB_ALGO_ATOMIC_CR = 3, /* mttkrp_alto_atomic_cr (alto.hpp:1090-1158) */
    ALTOB_ALGO_OPSCHED = 4    /* mttkrp_alto_op_sched (alto.hpp:1320-1415) */
} altob_algo;

typedef struct altob_tensor altob_tensor;

/* Scalars and masks of an encoding (AltoTensor<LIT>, alto.hpp:27-54).
 * 128-bit quantities are (lo, hi) word pairs. */
typedef struct {
    int nmode;
    int nprtn;
    int lit_bits;  /* 64 or 128 */
    int alto_bits; /* popcount(alto_mask) */
    int is_oidx;
    int val_dtype; /* altob_dtype of the stored values */
    uint64_t nnz;
    uint64_t dims[ALTOB_MAX_MODES];
    uint64_t mode_masks[ALTOB_MAX_MODES][2];
    uint64_t cr_masks[ALTOB_MAX_MODES][2];
    uint64_t alto_mask[2];
    uint64_t alto_cr_mask[2];
    uint64_t device_bytes; /* HBM held by the handle */
    uint64_t key_bytes;    /* bytes of index stored per nonzero on the device */
    int nruns;             /* high index words kept as a run table (0: none) */
    int plan_modes;        /* bit n set: mode n has a tile plan (MTTKRP) */
    uint64_t plan_bytes;   /* HBM held by the tile plans (2 B per nonzero and mode) */
    int tma_err;           /* 1: a TMA-staged MTTKRP ran out of a wait limit (read after the
                              stream of that call has been synchronised) */
} altob_info;

/* COO tensor in host memory (SparseTensor, sptensor.hpp:8-25): cidx is
 * mode-major SoA, cidx[n*nnz + i], 0-based; vals are FP64. */
typedef struct {
    int nmode;
    uint64_t nnz;
    uint64_t dims[ALTOB_MAX_MODES];
    uint64_t* cidx;
    double* vals;
} altob_coo;

ALTOB_API const char* altob_status_string(altob_status s);
/* Text of the last error raised on the calling thread ("" if none). */
ALTOB_API const char* altob_last_error(void);
/* Library version string. */
ALTOB_API const char* altob_version(void);

/* ---- tensor build ------------------------------------------------------
 * Replaces create_alto<LIT>(SparseTensor*, AltoTensor<LIT>**, int nprtn)
 * (alto.hpp:108-294): packed LSB-first / shortest-first masks (:669-770),
 * linearization (:184-202), sort (:772-803), oidx (:246-285), equal-nnz
 * partitions, per-mode intervals and CR bits (:805-1028).  nprtn has the
 * reference's meaning (it fixes prtn_ptr, intervals and the CR bits).
 * lit_bits: 64, 128, or 0 = the smallest width that holds the ALTO bits.
 * Host inputs; cidx as in altob_coo; vals in val_dtype. */
ALTOB_API altob_status altob_create(int nmode, const uint64_t* dims, uint64_t nnz,
                          const uint64_t* cidx, const void* vals,
                          altob_dtype val_dtype, int nprtn, int lit_bits,
                          void* stream, altob_tensor** out);

/* Same, with cidx / vals already in device memory. */
ALTOB_API altob_status altob_create_device(int nmode, const uint64_t* dims, uint64_t nnz,
                                 const uint64_t* d_cidx, const void* d_vals,
                                 altob_dtype val_dtype, int nprtn, int lit_bits,
                                 void* stream, altob_tensor** out);

/* Replaces destroy_alto (alto.hpp:296-322). */
ALTOB_API altob_status altob_destroy(altob_tensor* t);

/* One GPU's share of a sharded MTTKRP / CP-ALS: nonzeros [begin, end) of
 * t's ALTO stream (the reference's contiguous equal-nnz partitions,
 * prtn_alto, alto.hpp:822-836, with one partition per GPU) as a tensor of
 * its own with nprtn partitions, mode intervals (alto.hpp:874-899) and oidx
 * (alto.hpp:246-285) computed for the slice; t is unchanged and may be
 * destroyed afterwards.  The slice has no conflict-resolution masks. */
ALTOB_API altob_status altob_slice(const altob_tensor* t, uint64_t begin,
                                   uint64_t end, int nprtn, void* stream,
                                   altob_tensor** out);

ALTOB_API altob_status altob_get_info(const altob_tensor* t, altob_info* out);

/* Copies the encoding back to the host in the reference's layout (for
 * parity checks): idx as (lo, hi) words per nonzero, vals in the stored
 * dtype, prtn_ptr[nprtn+1], intervals[nprtn*nmode] (start, stop) pairs
 * (prtn_intervals, alto.hpp:42), oidx as nmode rows of nnz (rows of modes
 * without oidx are left untouched).  Any output pointer may be NULL. */
ALTOB_API altob_status altob_dump(const altob_tensor* t, uint64_t* idx, void* vals,
                        uint64_t* prtn_ptr, uint64_t* intervals,
                        uint64_t* oidx, void* stream);

/* The keys and mode masks a -DALT_PEXT build of the reference holds
 * (alto.hpp:212-244): every mode index re-encoded as a bit field at
 * mode_pos[n] (the running sum of bit counts in mode order, alto.hpp:
 * 695-700), CR bits kept; masks (1 << bits) - 1.  idx: nnz (lo, hi) pairs;
 * mode_masks: nmode (lo, hi) pairs; mode_pos: nmode; any may be NULL.  Modes
 * of 31 or more bits are refused (the reference's int mask expression is
 * undefined there). */
ALTOB_API altob_status altob_dump_alt_pext(const altob_tensor* t, uint64_t* idx,
                                           uint64_t* mode_masks, int* mode_pos,
                                           void* stream);

/* The partition subspace ids of a -DOPT_ALTO build (alto.hpp:838-868), per
 * partition p: the ALTO bits its first and last keys share (before CR bits),
 * prtn_id[p] = those bits, prtn_mask[p] = their mask, prtn_mode_masks[p *
 * nmode + n] = mode n's mask restricted to them; 64-bit words as in the
 * reference; empty partitions 0. */
ALTOB_API altob_status altob_partition_ids(const altob_tensor* t, uint64_t* prtn_id,
                                           uint64_t* prtn_mask,
                                           uint64_t* prtn_mode_masks, void* stream);

/* ---- MTTKRP ------------------------------------------------------------
 * Replaces mttkrp_alto_par(int target_mode, FType** factors, IType rank,
 * AltoTensor*, omp_lock_t*, FType** ofibs) (alto.hpp:617-623).
 * d_factors: nmode device pointers, row-major I_n x rank in ftype.
 * accumulate = 1 keeps the reference's += semantics; 0 overwrites. */
ALTOB_API altob_status altob_mttkrp(altob_tensor* t, int mode, altob_dtype ftype,
                          void* const* d_factors, uint64_t rank,
                          int accumulate, altob_algo algo, void* stream);

/* The same call with the factor matrices in HOST memory (the reference's
 * calling convention): copies the factors in, runs, copies factors[mode]
 * back.  Synchronous. */
ALTOB_API altob_status altob_mttkrp_host(altob_tensor* t, int mode, altob_dtype ftype,
                               void* const* h_factors, uint64_t rank,
                               altob_algo algo, void* stream);

/* `iters` sweeps of mttkrp over every mode with host factors, as the
 * reference's benchmark loop (main.cpp:476-495): factors copied in once,
 * += into each mode in turn, all factors copied back.  Synchronous. */
ALTOB_API altob_status altob_mttkrp_sweep_host(altob_tensor* t, altob_dtype ftype,
                                     void* const* h_factors, uint64_t rank,
                                     int iters, altob_algo algo, void* stream);

/* ---- CP-ALS ------------------------------------------------------------
 * Replaces cpd_alto(AltoTensor*, KruskalModel*, int max_iters,
 * double epsilon) (cpd.hpp:43-186).  d_factors / d_lambda (ftype) hold the
 * initial model and receive the result.  fits[max_iters] (host, may be
 * NULL) receives cpd_fit_alto (cpd.hpp:189-271) per iteration; *iters the
 * number run.  The R x R Gram, solve, norms and fit run in FP64. */
ALTOB_API altob_status altob_cpd_als(altob_tensor* t, altob_dtype ftype,
                           void* const* d_factors, void* d_lambda,
                           uint64_t rank, int max_iters, double epsilon,
                           double* fits, int* iters, void* stream);

/* Sharded CP-ALS (no counterpart in the reference, which runs on one
 * node): every GPU holds one slice of the tensor (altob_slice) and the whole
 * model, and runs cpd_alto (cpd.hpp:43-186) with three exchanges, made by the
 * caller's allreduce callback (for example an NCCL all-reduce on `stream`):
 * the norm of the tensor once (sum), each mode's partial MTTKRP (sum over
 * the GPUs, dims[mode] x rank values of ftype, in place) and each
 * iteration's fit (max, so every GPU takes the same stopping decision).  The
 * dense update then runs on identical data on every GPU.  Every GPU must call
 * this with the same model, rank, max_iters and epsilon; the callback must
 * return ALTOB_OK after the reduction, or an error status, which ends the
 * solve on that GPU (the others then fail in their next exchange). */
#define ALTOB_REDUCE_SUM 0
#define ALTOB_REDUCE_MAX 1
typedef altob_status (*altob_allreduce_fn)(void* d_buf, uint64_t count,
                                           altob_dtype dtype, int op,
                                           void* stream, void* user);
ALTOB_API altob_status altob_cpd_als_sharded(altob_tensor* slice, altob_dtype ftype,
                                             void* const* d_factors, void* d_lambda,
                                             uint64_t rank, int max_iters, double epsilon,
                                             double* fits, int* iters,
                                             altob_allreduce_fn allreduce, void* user,
                                             void* stream);

/* Replaces pseudo_inverse (cpd.hpp:546-646): U <- U V^-1 with V the
 * Hadamard product of the Grams of every mode but `mode` (d_grams: nmode
 * R x R FP64 matrices, lower triangles used), by Cholesky when V is positive
 * definite, else by V's pseudo-inverse (Jacobi eigendecomposition,
 * eigenvalues below R * eps * max|lambda| dropped; the reference falls back
 * to GELSY, the same minimum-norm solution).  d_U: rows x rank (ftype), in
 * place.  *used_pinv (host, may be NULL) = 1 when the pseudo-inverse was
 * used.  Synchronous. */
ALTOB_API altob_status altob_pseudo_inverse(const double* d_grams, int nmode, int mode,
                                            uint64_t rank, void* d_U, uint64_t rows,
                                            altob_dtype ftype, int* used_pinv, void* stream);

/* cpd_alto's own calling convention: the model (factors, lambda) in HOST
 * memory, copied to the device, solved, and copied back.  Synchronous. */
ALTOB_API altob_status altob_cpd_als_host(altob_tensor* t, altob_dtype ftype,
                                          void* const* h_factors, void* h_lambda,
                                          uint64_t rank, int max_iters,
                                          double epsilon, double* fits,
                                          int* iters, void* stream);

/* ---- CP-APR ------------------------------------------------------------
 * Replaces cp_apr_alto(AltoTensor*, KruskalModel*, int max_iters,
 * int max_inner_iters, FType epsilon, FType eps_div_zero, FType kappa_tol,
 * FType kappa, bool dobench) (apr.hpp:984-1376).  summary[5] (host) =
 * {log-likelihood, least-squares fit, final KKT violation, outer
 * iterations, total inner iterations}.  KKT and log-likelihood in FP64. */
ALTOB_API altob_status altob_cp_apr(altob_tensor* t, altob_dtype ftype,
                          void* const* d_factors, void* d_lambda,
                          uint64_t rank, int max_iters, int max_inner,
                          double epsilon, double eps_div_zero,
                          double kappa_tol, double kappa, int dobench,
                          double* summary, void* stream);

/* cp_apr_alto's calling convention: host model, copied in and out. */
ALTOB_API altob_status altob_cp_apr_host(altob_tensor* t, altob_dtype ftype,
                                         void* const* h_factors, void* h_lambda,
                                         uint64_t rank, int max_iters,
                                         int max_inner, double epsilon,
                                         double eps_div_zero, double kappa_tol,
                                         double kappa, int dobench,
                                         double* summary, void* stream);

/* Replaces CalculatePhi_alto_par (apr.hpp:297-303): d_phi (I_mode x rank,
 * ftype) is overwritten; rows without nonzeros are 0. */
ALTOB_API altob_status altob_phi(altob_tensor* t, int mode, altob_dtype ftype,
                       void* const* d_factors, uint64_t rank,
                       double eps_div_zero, void* d_phi, void* stream);

/* Replaces tt_logLikelihood<LIT> (apr.hpp:851-982), including its
 * redistribution of lambda into mode 0 and the 1-norm renormalisation. */
ALTOB_API altob_status altob_loglik(altob_tensor* t, altob_dtype ftype,
                          void* const* d_factors, void* d_lambda,
                          uint64_t rank, double eps_div_zero,
                          double* loglik, void* stream);

/* No counterpart in the reference.  altob_loglik without device allocation,
 * for callers that cannot call cudaMalloc: code that owns all device memory
 * through its own pool or arena, code running where the CUDA allocator must
 * not be entered, or callers that need a fixed memory footprint.  The caller
 * passes the same tensor, factors and lambda as to altob_loglik and gets the
 * same result.  The scratch (lambda, column sums, two accumulators) is a
 * fixed device array inside the library: rank at most 112 (1856 bytes, held
 * on every GPU that loads the library until the process exits); a larger
 * rank returns ALTOB_ERR_ARG.  The first call on a device looks up that
 * array's device address (cudaGetSymbolAddress), so make that first call
 * before any stream capture.  All calls share the array: calls that overlap
 * on the GPU (other streams, other host threads) race and must be
 * serialised by the caller.  Synchronous on `stream`. */
ALTOB_API altob_status altob_loglik_noalloc(altob_tensor* t, altob_dtype ftype,
                                            void* const* d_factors,
                                            void* d_lambda, uint64_t rank,
                                            double eps_div_zero,
                                            double* loglik, void* stream);

/* ---- batched CP-ALS ----------------------------------------------------
 * No counterpart in the reference (one tensor per run there).  Many
 * independent CP-ALS solves (cpd_alto, include/cpd.hpp:43-186, each) run
 * together: every step of an iteration (MTTKRP, R x R solve, row apply,
 * normalisation, Gram, fit) is one launch for all tensors of the batch, the
 * MTTKRP one launch per shape class, and iterations after the first are
 * replayed from a captured CUDA graph.  Each tensor stops on its own rule
 * (|fit - previous fit| < epsilon, or max_iters) and is skipped from then on,
 * so its result is the one a separate altob_cpd_als call computes (up to the
 * order of floating-point additions in the MTTKRP).
 *   tensors[b], ranks[b] (1..112), d_factors[b][m] (device, dims[m] x
 *   ranks[b], row-major, ftype) and d_lambda[b] (device, ranks[b]; the array
 *   or any entry may be NULL) belong to tensor b.  All tensors share one
 *   value dtype.  The handle keeps the pointers: factors are updated in place
 *   by every altob_batch_cpd_als call.  fit_capacity bounds max_iters. */
typedef struct altob_batch altob_batch;
ALTOB_API altob_status altob_batch_create(altob_tensor* const* tensors, int count,
                                          const uint64_t* ranks, altob_dtype ftype,
                                          void* const* const* d_factors,
                                          void* const* d_lambda, int fit_capacity,
                                          void* stream, altob_batch** out);
/* Picks, per shape class (order, lanes per nonzero (from the rank),
 * elements per lane, nnz decade, low fiber reuse), the row-slot count and
 * lane layout of the batched MTTKRP by timing
 * every candidate on that class; leaves the factors unchanged.  Choices are
 * remembered per class for the rest of the process and applied to later
 * batches at creation; force = 0 tunes only classes without one. */
ALTOB_API altob_status altob_batch_autotune(altob_batch* b, int force, void* stream);
/* fits: count x max_iters (row b = tensor b, 0 after its last iteration) or
 * NULL; iters: count or NULL.  use_graph = 0 launches every iteration
 * directly (same results).  Synchronous on `stream`. */
ALTOB_API altob_status altob_batch_cpd_als(altob_batch* b, int max_iters, double epsilon,
                                           double* fits, int* iters, int use_graph,
                                           void* stream);
/* Text description of the shape classes and their chosen schedules. */
ALTOB_API altob_status altob_batch_describe(const altob_batch* b, char* buf, size_t len);
ALTOB_API altob_status altob_batch_destroy(altob_batch* b);

/* ---- decomposition server ----------------------------------------------
 * No counterpart in the reference.  A request loop over the solvers above:
 * requests are queued in arrival order and admitted against an HBM budget
 * (footprint estimated by altob_request_footprint); `workers` requests or
 * batches run at once, each worker on its own CUDA stream.  A worker that
 * admits a CP-ALS request takes the queued CP-ALS requests behind it with
 * the same dtypes, iteration limit and tolerance (up to max_batch, within
 * the budget) into one altob_batch solve.  The request a free worker starts
 * is the queue head (policy 0) or the one with the least estimated work
 * (nonzeros x modes x iterations, x inner iterations for CP-APR, at an
 * assumed 10 Gnnz/s) after subtracting the time it has waited (policy 1:
 * short requests pass long ones, no request waits forever).  Batched CP-ALS
 * solves run on a stream of the device's highest priority, CP-APR requests
 * on one of the lowest.  With plain = 1 every request runs
 * alone through altob_cpd_als / altob_cp_apr (no batching).  Factors are
 * initialised on the device from the request's seed, identically alone or in
 * a batch.  The request's COO arrays (device, as for altob_create_device)
 * must stay valid until altob_server_wait returns for it. */
typedef enum { ALTOB_REQ_CPD_ALS = 0, ALTOB_REQ_CP_APR = 1 } altob_req_kind;

typedef struct {
    altob_req_kind kind;
    int nmode;
    uint64_t dims[ALTOB_MAX_MODES];
    uint64_t nnz;
    const void* d_cidx;  /* device, nmode x nnz uint64 (mode-major) */
    const void* d_vals;  /* device, nnz values of vdtype */
    altob_dtype vdtype;  /* F32 / F64 values (CP-ALS), U32 counts (CP-APR) */
    altob_dtype ftype;   /* model dtype, F32 or F64 */
    uint64_t rank;       /* 1..112 */
    int max_iters;       /* CP-ALS iterations / CP-APR outer iterations */
    int max_inner;       /* CP-APR inner iterations */
    double tol;          /* CP-ALS |fit change| / CP-APR KKT tolerance */
    unsigned seed;       /* factor initialisation */
    int nprtn;           /* ALTO partitions (0: 128) */
} altob_request;

typedef struct {
    altob_status status;
    int iters;        /* CP-ALS iterations / CP-APR outer iterations run */
    int batch_size;   /* requests solved together with this one */
    double fit;       /* final fit (CP-APR: its least-squares fit) */
    double loglik;    /* CP-APR log-likelihood */
    double t_submit;  /* server clock, seconds */
    double t_start;
    double t_end;
} altob_result;

typedef struct {
    uint64_t hbm_budget; /* bytes admitted requests may use together */
    int workers;         /* requests or batches in flight (1..64) */
    int max_batch;       /* CP-ALS requests per batched solve */
    int use_graph;       /* replay batched iterations from a CUDA graph */
    int autotune;        /* tune unseen shape classes on first use */
    int plain;           /* 1: no batching, altob_cpd_als per request */
    int policy;          /* 0: arrival order; 1: least estimated work first, a
                            request's estimate shrinking by 1 s per second waited */
} altob_server_config;

typedef struct altob_server altob_server;
ALTOB_API altob_status altob_request_footprint(const altob_request* r, uint64_t* bytes);
ALTOB_API altob_status altob_server_create(const altob_server_config* cfg, altob_server** out);
ALTOB_API double altob_server_clock(const altob_server* s);
ALTOB_API altob_status altob_server_submit(altob_server* s, const altob_request* r, uint64_t* id);
/* Blocks until request `id` completes; each id can be waited for once. */
ALTOB_API altob_status altob_server_wait(altob_server* s, uint64_t id, altob_result* out);
ALTOB_API altob_status altob_server_stats(const altob_server* s, uint64_t* used_bytes,
                                          uint64_t* peak_bytes, int* queued, int* running);
/* Finishes the queued requests, then stops the workers. */
ALTOB_API altob_status altob_server_destroy(altob_server* s);

/* Replaces PoissonGeneratorRun (src/poisson_generator.cpp:337-375) as
 * MakeSparseTensor (src/main.cpp:652-675, cpd64 -d) calls it: a random
 * rank-`rank` Kruskal model (GenerateRandomModel :145-194), num_edges
 * multinomial draws of its components and coordinates (GenerateEdges
 * :197-259), duplicates merged into counts (ConstructCIdx :262-334).  The
 * reference's random streams (one MT19937-64 per OpenMP thread, seeded
 * 1234 + thread id, and the C library's rand() from its initial state) are
 * replayed for `nthreads` threads; the edges are drawn and sorted on the
 * device.  For the same thread count the tensor and the model equal the
 * reference's (above one thread up to the order in which the reference's
 * OpenMP reduction adds its column sums).  *out: host COO (0-based,
 * values = counts), freed with altob_coo_free; model_U (nmode host arrays,
 * dims[n] x rank, FP64) and model_lambda (rank) receive the model and may
 * be NULL.  Every dimension must be >= rank (the reference asserts it). */
ALTOB_API altob_status altob_poisson_tensor(int nmode, const uint64_t* dims,
                                            uint64_t num_edges, uint64_t rank,
                                            int nthreads, double* const* model_U,
                                            double* model_lambda, altob_coo** out,
                                            void* stream);

/* ---- tensor files ------------------------------------------------------
 * Replaces ImportSparseTensor (sptensor.cpp:165-258).  The .tns reader
 * follows the reference (dims = largest index seen, '#' comments and empty
 * lines skipped, 1-based unless zero_based) and parses in parallel. */
ALTOB_API altob_status altob_read_tns(const char* path, int zero_based, altob_coo** out);
/* Binary layout of sptensor.cpp:57-69 / 211-258: u64 nmodes, u64
 * dims[nmodes], u64 nnz, nmodes x nnz u64 indices, nnz FP64 values. */
ALTOB_API altob_status altob_read_bin(const char* path, altob_coo** out);
ALTOB_API altob_status altob_write_bin(const char* path, const altob_coo* coo);
/* Replaces ExportSparseTensor TEXT_FORMAT (sptensor.cpp:49-56). */
ALTOB_API altob_status altob_write_tns(const char* path, const altob_coo* coo);
ALTOB_API void altob_coo_free(altob_coo* coo);

/* Replaces KruskalModelRandomInit (src/kruskal_model.cpp:109-125): lambda
 * = 1 and U = (FType)rand() / RAND_MAX from glibc srand(seed), mode by mode,
 * into host buffers (so a model initialised here equals the reference's). */
ALTOB_API altob_status altob_kruskal_random_init(int nmode, const uint64_t* dims,
                                                 uint64_t rank, unsigned seed,
                                                 altob_dtype ftype,
                                                 void* const* h_factors,
                                                 void* h_lambda);

#ifdef __cplusplus
}
#endif
#endif /* ALTOB_H_ */
