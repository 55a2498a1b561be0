/*
 * alto_oracle.h -- CPU restatement of IntelLabs/ALTO's hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This oracle is the checker for the CUDA
 * implementation in alto_b200/.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py may load it.  The product path
 * (libaltob.so) never links, calls or falls back to it.
 *
 * Parity pin: the oracle is checked against fixtures produced by the
 * reference itself (oracle/_ref, built by oracle/build_ref.sh from the
 * reference sources; fixtures and their generator live in tests/golden/).
 *
 * Every function cites the reference file:line it restates.
 */
#ifndef ALTO_ORACLE_H_
#define ALTO_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_MODES 5

typedef struct orc_alto orc_alto;

/* create_alto (include/alto.hpp:108-294): packed masks, linearize, sort,
 * oidx, partition, intervals, CR bits.  cidx is mode-major SoA
 * (cidx[n*nnz + i]), 0-based.  lit_bits is 64 or 128.  Returns 0 on
 * success, 1 if the ALTO bits exceed lit_bits, 2 on bad arguments. */
int orc_create(int nmode, const uint64_t* dims, uint64_t nnz,
               const uint64_t* cidx, const double* vals, int nprtn,
               int lit_bits, orc_alto** out);
void orc_destroy(orc_alto* at);

/* Scalars of the encoding: [alto_bits, is_oidx, nprtn, nmode]. */
void orc_info(const orc_alto* at, int* out4);

/* Dump the encoding.  idx is written as two words per nonzero (lo, hi);
 * masks / cr_masks as two words per mode; intervals as nprtn*nmode
 * (start, stop) pairs; oidx as nmode*nnz (rows of modes without oidx are
 * left untouched).  Any pointer may be NULL. */
void orc_dump(const orc_alto* at, uint64_t* idx, double* vals,
              uint64_t* prtn_ptr, uint64_t* intervals, uint64_t* masks,
              uint64_t* cr_masks, uint64_t* oidx);

/* mttkrp_alto_par (include/alto.hpp:617-623) with the reference's dispatch:
 * reuse > 4 -> da_mem_pull order, reuse <= 4 -> op_sched order.  Accumulates
 * (+=) into factors[mode] like the reference. */
void orc_mttkrp(const orc_alto* at, int mode, double* const* factors,
                uint64_t rank);

/* Plain sequential COO MTTKRP (include/cpd.hpp:509-543), += semantics. */
void orc_mttkrp_coo(int nmode, uint64_t nnz, const uint64_t* cidx,
                    const double* vals, int mode, double* const* factors,
                    uint64_t rank);

/* KruskalModelRandomInit (src/kruskal_model.cpp:109-125): glibc srand/rand. */
void orc_random_init(int nmode, const uint64_t* dims, uint64_t rank,
                     unsigned seed, double* const* U, double* lambda);

/* cpd_alto (include/cpd.hpp:43-186).  U / lambda are updated in place.
 * fits[max_iters] receives the per-iteration fit; returns iterations run. */
int orc_cpd_als(const orc_alto* at, double* const* U, double* lambda,
                uint64_t rank, int max_iters, double epsilon, double* fits);

/* cp_apr_alto (include/apr.hpp:984-1376).  out[8] = {log-likelihood,
 * least-squares fit, final KKT violation, outer iterations, total inner
 * iterations, 0, 0, 0}.  kkt_trace[max_iters] receives the per-outer KKT. */
int orc_cp_apr(const orc_alto* at, double* const* U, double* lambda,
               uint64_t rank, int max_iters, int max_inner, double epsilon,
               double eps_div_zero, double kappa_tol, double kappa,
               int dobench, double* out, double* kkt_trace);

/* CalculatePhi (include/apr.hpp:306-381 naive form; rows without nonzeros
 * are 0 as in the da_mem_pull variant, include/apr.hpp:476-499). */
void orc_phi(const orc_alto* at, int mode, double* const* U, uint64_t rank,
             double eps_div_zero, double* phi);

/* tt_logLikelihood (include/apr.hpp:851-982); renormalises mode 0. */
double orc_loglik(const orc_alto* at, double* const* U, double* lambda,
                  uint64_t rank, double eps_div_zero);

/* update_gram (src/kruskal_model.cpp:11-24): full symmetric U^T U. */
void orc_gram(const double* U, uint64_t rows, uint64_t rank, double* G);

#ifdef __cplusplus
}
#endif
#endif
