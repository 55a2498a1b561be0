/*
 * alto_oracle.c -- CPU restatement of IntelLabs/ALTO's hot path (oracle).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for alto_b200's CUDA path.  It is
 * loaded by tests/, __graft_entry__.smoke() and bench.py's CPU legs, and by
 * nothing that ships.  Plain C, single threaded, FP64 throughout.
 *
 * Pinned against the reference itself: tests/golden/ holds fixtures written
 * by the reference code (built from its own sources by oracle/build_ref.sh)
 * and tests/test_oracle_golden.py checks this file against them.
 *
 * Defined behaviour where the reference is undefined (each noted inline):
 *  - a mode of length 1 gets 0 ALTO bits (reference: clz(0));
 *  - sort ties (duplicate coordinates) keep input order (reference: std::sort
 *    order, unspecified); oidx ties keep ALTO order;
 *  - CP-APR Phi rows that no nonzero touches are 0 (reference op_sched
 *    leaves them stale);
 *  - CP-APR's first outer iteration has no predecessor for the convergence
 *    test (reference reads kktViolations[-1]);
 *  - the Cholesky fallback is a symmetric pseudo-inverse of the lower
 *    triangle (reference GELSY reads the upper triangle, which holds stale
 *    data).
 */
#include "alto_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;
typedef uint64_t u64;

#define MIN_FIBER_REUSE 4 /* include/alto.hpp:90 */

struct orc_alto {
    int nmode, nprtn, lit_bits, alto_bits, is_oidx;
    u64 nnz;
    u64 dims[ORC_MAX_MODES];
    u128 masks[ORC_MAX_MODES];
    u128 alto_mask;
    u128 cr_masks[ORC_MAX_MODES];
    u128 alto_cr_mask;
    u128* idx;
    double* vals;
    u64* prtn_ptr;
    u64* intervals; /* nprtn * nmode * 2 */
    u64* oidx[ORC_MAX_MODES];
};

/* ---- bit operations (include/bitops.hpp:17-42 portable loops, 59-106) ---- */

static u128 pdep128(u64 x, u128 m)
{
    u128 res = 0;
    for (int b = 0; b < 128 && m; ++b) {
        u128 low = m & (~m + 1); /* lowest set bit */
        if (x & 1) res |= low;
        x >>= 1;
        m &= m - 1;
        (void)b;
    }
    return res;
}

static u64 pext128(u128 x, u128 m)
{
    u64 res = 0, bit = 1;
    while (m) {
        u128 low = m & (~m + 1);
        if (x & low) res |= bit;
        bit <<= 1;
        m &= m - 1;
    }
    return res;
}

static int popcount128(u128 x)
{
    return __builtin_popcountll((u64)x) + __builtin_popcountll((u64)(x >> 64));
}

/* mbits = sizeof(IType)*8 - clz(dim-1), include/alto.hpp:686. */
static int mode_bits(u64 d)
{
    if (d <= 1) return 0;
    return 64 - __builtin_clzll(d - 1);
}

/* setup_packed_alto(LSB_FIRST, SHORT_FIRST), include/alto.hpp:669-770.
 * Modes are ordered by bit count ascending; equal counts keep mode order
 * (std::sort on <=16 elements is libstdc++'s insertion sort, which does not
 * reorder equal elements).  Then round-robin from the LSB. */
static int setup_masks(orc_alto* at)
{
    int bits[ORC_MAX_MODES], order[ORC_MAX_MODES], total = 0;
    for (int n = 0; n < at->nmode; ++n) {
        bits[n] = mode_bits(at->dims[n]);
        order[n] = n;
        total += bits[n];
        at->masks[n] = 0;
    }
    if (total > at->lit_bits) return 1; /* alto.hpp:709 assert */
    for (int i = 1; i < at->nmode; ++i) {
        int v = order[i], j = i - 1;
        while (j >= 0 && bits[order[j]] > bits[v]) {
            order[j + 1] = order[j];
            --j;
        }
        order[j + 1] = v;
    }
    int shift = 0;
    for (int level = 0;; ++level) {
        int done = 1;
        for (int k = 0; k < at->nmode; ++k) {
            int n = order[k];
            if (level < bits[n]) {
                at->masks[n] |= (u128)1 << shift;
                ++shift;
                done = 0;
            }
        }
        if (done) break;
    }
    at->alto_mask = 0;
    for (int n = 0; n < at->nmode; ++n) at->alto_mask |= at->masks[n];
    at->alto_bits = shift;
    return 0;
}

/* ---- sorting helpers (stable) ---- */

typedef struct { u128 key; u64 pos; } kp_t;

static int cmp_kp(const void* a, const void* b)
{
    const kp_t* x = (const kp_t*)a;
    const kp_t* y = (const kp_t*)b;
    if (x->key < y->key) return -1;
    if (x->key > y->key) return 1;
    return (x->pos < y->pos) ? -1 : (x->pos > y->pos);
}

/* prtn_alto, include/alto.hpp:805-1028: equal-nnz bounds, per-mode
 * intervals, CR bits through an ownership array. */
static void partition(orc_alto* at)
{
    int nm = at->nmode, np = at->nprtn;
    u64 nnz = at->nnz;
    u64 per = (nnz + (u64)np - 1) / (u64)np;
    at->prtn_ptr[0] = 0;
    for (int p = 0; p < np; ++p) {
        u64 s = (u64)p * per, e = (u64)(p + 1) * per;
        if (e > nnz) e = nnz;
        if (s > e) s = e;
        at->prtn_ptr[p + 1] = e;
    }
    for (int p = 0; p < np; ++p) {
        u64 lo[ORC_MAX_MODES], hi[ORC_MAX_MODES];
        for (int n = 0; n < nm; ++n) { lo[n] = at->dims[n]; hi[n] = 0; }
        for (u64 i = at->prtn_ptr[p]; i < at->prtn_ptr[p + 1]; ++i)
            for (int n = 0; n < nm; ++n) {
                u64 c = pext128(at->idx[i], at->masks[n]);
                if (c < lo[n]) lo[n] = c;
                if (c > hi[n]) hi[n] = c;
            }
        for (int n = 0; n < nm; ++n) {
            at->intervals[((u64)p * nm + n) * 2 + 0] = lo[n];
            at->intervals[((u64)p * nm + n) * 2 + 1] = hi[n];
        }
    }

    /* CR bits, include/alto.hpp:932-1027. */
    int free_bits = at->lit_bits - popcount128(at->alto_mask);
    int* owner[ORC_MAX_MODES] = {0};
    at->alto_cr_mask = 0;
    for (int n = 0; n < nm; ++n) {
        at->cr_masks[n] = 0;
        u64 reuse = nnz / at->dims[n];
        if (reuse <= MIN_FIBER_REUSE && free_bits) {
            at->cr_masks[n] = (u128)1 << (at->lit_bits - free_bits);
            at->alto_cr_mask |= at->cr_masks[n];
            owner[n] = (int*)calloc(at->dims[n], sizeof(int));
            --free_bits;
        }
    }
    if (!at->alto_cr_mask) return;
    /* Final owner state: 0 untouched, p+1 touched by one partition only,
     * -1 touched by two or more partitions (independent of thread order). */
    for (int p = 0; p < np; ++p)
        for (u64 i = at->prtn_ptr[p]; i < at->prtn_ptr[p + 1]; ++i)
            for (int n = 0; n < nm; ++n) {
                if (!owner[n]) continue;
                u64 c = pext128(at->idx[i], at->masks[n]);
                int o = owner[n][c];
                if (o == 0) owner[n][c] = p + 1;
                else if (o != p + 1) owner[n][c] = -1;
            }
    for (u64 i = 0; i < nnz; ++i) {
        u128 add = 0;
        for (int n = 0; n < nm; ++n) {
            if (!owner[n]) continue;
            u64 c = pext128(at->idx[i], at->masks[n]);
            if (owner[n][c] == -1) add |= at->cr_masks[n];
        }
        at->idx[i] |= add;
    }
    for (int n = 0; n < nm; ++n) free(owner[n]);
}

int orc_create(int nmode, const uint64_t* dims, uint64_t nnz,
               const uint64_t* cidx, const double* vals, int nprtn,
               int lit_bits, orc_alto** out)
{
    if (nmode < 1 || nmode > ORC_MAX_MODES || nprtn < 1 ||
        (lit_bits != 64 && lit_bits != 128) || !out)
        return 2;
    orc_alto* at = (orc_alto*)calloc(1, sizeof(orc_alto));
    at->nmode = nmode;
    at->nprtn = nprtn;
    at->lit_bits = lit_bits;
    at->nnz = nnz;
    for (int n = 0; n < nmode; ++n) {
        if (dims[n] == 0) { free(at); return 2; }
        at->dims[n] = dims[n];
    }
    if (setup_masks(at)) { free(at); return 1; }

    /* Linearize, include/alto.hpp:184-202; then sort_alto (:772-803). */
    kp_t* kp = (kp_t*)malloc((nnz ? nnz : 1) * sizeof(kp_t));
    for (u64 i = 0; i < nnz; ++i) {
        u128 a = 0;
        for (int n = 0; n < nmode; ++n) a |= pdep128(cidx[(u64)n * nnz + i], at->masks[n]);
        kp[i].key = a;
        kp[i].pos = i;
    }
    qsort(kp, nnz, sizeof(kp_t), cmp_kp);
    at->idx = (u128*)malloc((nnz ? nnz : 1) * sizeof(u128));
    at->vals = (double*)malloc((nnz ? nnz : 1) * sizeof(double));
    for (u64 i = 0; i < nnz; ++i) {
        at->idx[i] = kp[i].key;
        at->vals[i] = vals[kp[i].pos];
    }

    /* oidx, include/alto.hpp:246-285 (computed before the CR bits are set,
     * as in the reference; CR bits do not change mode indices anyway). */
    at->is_oidx = 0;
    for (int n = 0; n < nmode; ++n)
        if (nnz / dims[n] <= MIN_FIBER_REUSE) at->is_oidx = 1;
    if (at->is_oidx) {
        for (int n = 0; n < nmode; ++n) {
            if (nnz / dims[n] > MIN_FIBER_REUSE) continue;
            for (u64 i = 0; i < nnz; ++i) {
                kp[i].key = pext128(at->idx[i], at->masks[n]);
                kp[i].pos = i;
            }
            qsort(kp, nnz, sizeof(kp_t), cmp_kp);
            at->oidx[n] = (u64*)malloc((nnz ? nnz : 1) * sizeof(u64));
            for (u64 i = 0; i < nnz; ++i) at->oidx[n][i] = kp[i].pos;
        }
    }
    free(kp);

    at->prtn_ptr = (u64*)malloc((size_t)(nprtn + 1) * sizeof(u64));
    at->intervals = (u64*)malloc((size_t)nprtn * nmode * 2 * sizeof(u64));
    partition(at);
    *out = at;
    return 0;
}

void orc_destroy(orc_alto* at)
{
    if (!at) return;
    free(at->idx);
    free(at->vals);
    free(at->prtn_ptr);
    free(at->intervals);
    for (int n = 0; n < at->nmode; ++n) free(at->oidx[n]);
    free(at);
}

void orc_info(const orc_alto* at, int* out4)
{
    out4[0] = at->alto_bits;
    out4[1] = at->is_oidx;
    out4[2] = at->nprtn;
    out4[3] = at->nmode;
}

void orc_dump(const orc_alto* at, uint64_t* idx, double* vals,
              uint64_t* prtn_ptr, uint64_t* intervals, uint64_t* masks,
              uint64_t* cr_masks, uint64_t* oidx)
{
    u64 nnz = at->nnz;
    if (idx)
        for (u64 i = 0; i < nnz; ++i) {
            idx[2 * i] = (u64)at->idx[i];
            idx[2 * i + 1] = (u64)(at->idx[i] >> 64);
        }
    if (vals) memcpy(vals, at->vals, nnz * sizeof(double));
    if (prtn_ptr) memcpy(prtn_ptr, at->prtn_ptr, (size_t)(at->nprtn + 1) * sizeof(u64));
    if (intervals)
        memcpy(intervals, at->intervals, (size_t)at->nprtn * at->nmode * 2 * sizeof(u64));
    for (int n = 0; n < at->nmode; ++n) {
        if (masks) {
            masks[2 * n] = (u64)at->masks[n];
            masks[2 * n + 1] = (u64)(at->masks[n] >> 64);
        }
        if (cr_masks) {
            cr_masks[2 * n] = (u64)at->cr_masks[n];
            cr_masks[2 * n + 1] = (u64)(at->cr_masks[n] >> 64);
        }
        if (oidx && at->oidx[n]) memcpy(oidx + (u64)n * nnz, at->oidx[n], nnz * sizeof(u64));
    }
}

/* ---- MTTKRP ---- */

/* Row of the Khatri-Rao product times the value, for every mode but skip. */
static void krp_row(const orc_alto* at, u128 a, double v, int skip,
                    double* const* U, u64 R, double* row)
{
    for (u64 r = 0; r < R; ++r) row[r] = v;
    for (int m = 0; m < at->nmode; ++m) {
        if (m == skip) continue;
        const double* Um = U[m] + pext128(a, at->masks[m]) * R;
        for (u64 r = 0; r < R; ++r) row[r] *= Um[r];
    }
}

/* da_mem_pull order (include/alto.hpp:1227-1318): per-partition temp rows,
 * then a pull over partitions in ascending order for every output row. */
static void mttkrp_pull(const orc_alto* at, int mode, double* const* U, u64 R)
{
    int nm = at->nmode, np = at->nprtn;
    double** tmp = (double**)calloc((size_t)np, sizeof(double*));
    double* row = (double*)malloc(R * sizeof(double));
    for (int p = 0; p < np; ++p) {
        u64 s = at->prtn_ptr[p], e = at->prtn_ptr[p + 1];
        if (s == e) continue; /* empty partition: reference would abort */
        u64 lo = at->intervals[((u64)p * nm + mode) * 2];
        u64 hi = at->intervals[((u64)p * nm + mode) * 2 + 1];
        tmp[p] = (double*)calloc((hi - lo + 1) * R, sizeof(double));
        for (u64 i = s; i < e; ++i) {
            krp_row(at, at->idx[i], at->vals[i], mode, U, R, row);
            double* o = tmp[p] + (pext128(at->idx[i], at->masks[mode]) - lo) * R;
            for (u64 r = 0; r < R; ++r) o[r] += row[r];
        }
    }
    double* out = U[mode];
    for (u64 i = 0; i < at->dims[mode]; ++i)
        for (int p = 0; p < np; ++p) {
            if (!tmp[p]) continue;
            u64 lo = at->intervals[((u64)p * nm + mode) * 2];
            u64 hi = at->intervals[((u64)p * nm + mode) * 2 + 1];
            if (i < lo || i > hi) continue;
            const double* t = tmp[p] + (i - lo) * R;
            for (u64 r = 0; r < R; ++r) out[i * R + r] += t[r];
        }
    for (int p = 0; p < np; ++p) free(tmp[p]);
    free(tmp);
    free(row);
}

/* op_sched order (include/alto.hpp:1320-1415): walk oidx per partition and
 * flush each run of equal output rows. */
static void mttkrp_opsched(const orc_alto* at, int mode, double* const* U, u64 R)
{
    const u64* ox = at->oidx[mode];
    double* acc = (double*)malloc(R * sizeof(double));
    double* row = (double*)malloc(R * sizeof(double));
    double* out = U[mode];
    for (int p = 0; p < at->nprtn; ++p) {
        u64 s = at->prtn_ptr[p], e = at->prtn_ptr[p + 1];
        if (s == e) continue;
        u64 last = pext128(at->idx[ox[s]], at->masks[mode]);
        memset(acc, 0, R * sizeof(double));
        for (u64 i = s; i < e; ++i) {
            u128 a = at->idx[ox[i]];
            krp_row(at, a, at->vals[ox[i]], mode, U, R, row);
            u64 t = pext128(a, at->masks[mode]);
            if (t != last) {
                for (u64 r = 0; r < R; ++r) out[last * R + r] += acc[r];
                memset(acc, 0, R * sizeof(double));
            }
            last = t;
            for (u64 r = 0; r < R; ++r) acc[r] += row[r];
        }
        for (u64 r = 0; r < R; ++r) out[last * R + r] += acc[r];
    }
    free(acc);
    free(row);
}

void orc_mttkrp(const orc_alto* at, int mode, double* const* factors,
                uint64_t rank)
{
    u64 reuse = at->nnz / at->dims[mode];
    if (reuse <= MIN_FIBER_REUSE && at->is_oidx)
        mttkrp_opsched(at, mode, factors, rank);
    else
        mttkrp_pull(at, mode, factors, rank);
}

void orc_mttkrp_coo(int nmode, uint64_t nnz, const uint64_t* cidx,
                    const double* vals, int mode, double* const* factors,
                    uint64_t rank)
{
    double* row = (double*)malloc(rank * sizeof(double));
    for (u64 i = 0; i < nnz; ++i) {
        for (u64 r = 0; r < rank; ++r) row[r] = vals[i];
        for (int m = 0; m < nmode; ++m) {
            if (m == mode) continue;
            const double* Um = factors[m] + cidx[(u64)m * nnz + i] * rank;
            for (u64 r = 0; r < rank; ++r) row[r] *= Um[r];
        }
        double* o = factors[mode] + cidx[(u64)mode * nnz + i] * rank;
        for (u64 r = 0; r < rank; ++r) o[r] += row[r];
    }
    free(row);
}

/* ---- Kruskal model helpers (src/kruskal_model.cpp) ---- */

void orc_random_init(int nmode, const uint64_t* dims, uint64_t rank,
                     unsigned seed, double* const* U, double* lambda)
{
    for (u64 r = 0; r < rank; ++r) lambda[r] = 1.0;
    srand(seed);
    for (int n = 0; n < nmode; ++n)
        for (u64 i = 0; i < dims[n] * rank; ++i)
            U[n][i] = (double)rand() / RAND_MAX;
}

void orc_gram(const double* U, uint64_t rows, uint64_t R, double* G)
{
    for (u64 a = 0; a < R; ++a)
        for (u64 b = 0; b <= a; ++b) {
            double s = 0.0;
            for (u64 i = 0; i < rows; ++i) s += U[i * R + a] * U[i * R + b];
            G[a * R + b] = s;
            G[b * R + a] = s;
        }
}

/* KruskalModelNorm (src/kruskal_model.cpp:224-341). */
static void col_norm(double* U, u64 rows, u64 R, double* lambda, int use_max)
{
    for (u64 r = 0; r < R; ++r) lambda[r] = 0.0;
    if (!use_max) {
        for (u64 i = 0; i < rows; ++i)
            for (u64 r = 0; r < R; ++r) lambda[r] += U[i * R + r] * U[i * R + r];
        for (u64 r = 0; r < R; ++r) lambda[r] = sqrt(lambda[r]);
    } else {
        for (u64 i = 0; i < rows; ++i)
            for (u64 r = 0; r < R; ++r)
                if (U[i * R + r] > lambda[r]) lambda[r] = U[i * R + r];
        for (u64 r = 0; r < R; ++r)
            if (lambda[r] < 1.0) lambda[r] = 1.0;
    }
    for (u64 i = 0; i < rows; ++i)
        for (u64 r = 0; r < R; ++r) U[i * R + r] /= lambda[r];
}

/* KruskalModelNormalizeMode (src/kruskal_model.cpp:178-222): 1-norm. */
static void normalize_mode(double* U, u64 rows, u64 R, double* lambda)
{
    double* cn = (double*)calloc(R, sizeof(double));
    for (u64 i = 0; i < rows; ++i)
        for (u64 r = 0; r < R; ++r) cn[r] += fabs(U[i * R + r]);
    for (u64 i = 0; i < rows; ++i)
        for (u64 r = 0; r < R; ++r) U[i * R + r] /= cn[r];
    for (u64 r = 0; r < R; ++r) lambda[r] *= cn[r];
    free(cn);
}

/* RedistributeLambda (src/kruskal_model.cpp:355-378). */
static void redistribute(double* U, u64 rows, u64 R, double* lambda)
{
    for (u64 i = 0; i < rows; ++i)
        for (u64 r = 0; r < R; ++r) U[i * R + r] *= lambda[r];
    for (u64 r = 0; r < R; ++r) lambda[r] = 1.0;
}

/* ---- R x R solve (include/cpd.hpp:546-646) ---- */

/* Cyclic Jacobi eigen-decomposition of a symmetric matrix (A overwritten by
 * the eigenvalues on its diagonal, V the eigenvectors as columns). */
static void jacobi_eig(double* A, double* V, int n)
{
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) V[i * n + j] = (i == j);
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, tot = 0.0;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                tot += A[i * n + j] * A[i * n + j];
                if (i != j) off += A[i * n + j] * A[i * n + j];
            }
        if (off <= 1e-30 * tot) break;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) {
                double apq = A[p * n + q];
                if (apq == 0.0) continue;
                double theta = (A[q * n + q] - A[p * n + p]) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; ++k) {
                    double akp = A[k * n + p], akq = A[k * n + q];
                    A[k * n + p] = c * akp - s * akq;
                    A[k * n + q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {
                    double apk = A[p * n + k], aqk = A[q * n + k];
                    A[p * n + k] = c * apk - s * aqk;
                    A[q * n + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    double vkp = V[k * n + p], vkq = V[k * n + q];
                    V[k * n + p] = c * vkp - s * vkq;
                    V[k * n + q] = s * vkp + c * vkq;
                }
            }
    }
}

/* U <- U * V^{-1} with V = Hadamard of the Grams of the other modes.
 * Cholesky (lower) when V is positive definite, else pseudo-inverse. */
static int pseudo_inverse(double** G, int nmode, int mode, double* U, u64 rows, u64 R)
{
    double* V = (double*)malloc(R * R * sizeof(double));
    for (u64 k = 0; k < R * R; ++k) V[k] = 1.0;
    for (int m = 0; m < nmode; ++m)
        if (m != mode)
            for (u64 k = 0; k < R * R; ++k) V[k] *= G[m][k];
    double* L = (double*)calloc(R * R, sizeof(double));
    int ok = 1;
    for (u64 j = 0; j < R && ok; ++j) {
        double d = V[j * R + j];
        for (u64 k = 0; k < j; ++k) d -= L[j * R + k] * L[j * R + k];
        if (!(d > 0.0)) { ok = 0; break; }
        L[j * R + j] = sqrt(d);
        for (u64 i = j + 1; i < R; ++i) {
            double s = V[i * R + j];
            for (u64 k = 0; k < j; ++k) s -= L[i * R + k] * L[j * R + k];
            L[i * R + j] = s / L[j * R + j];
        }
    }
    double* x = (double*)malloc(R * sizeof(double));
    if (ok) {
        for (u64 i = 0; i < rows; ++i) {
            double* u = U + i * R;
            for (u64 a = 0; a < R; ++a) {
                double s = u[a];
                for (u64 k = 0; k < a; ++k) s -= L[a * R + k] * x[k];
                x[a] = s / L[a * R + a];
            }
            for (u64 a = R; a-- > 0;) {
                double s = x[a];
                for (u64 k = a + 1; k < R; ++k) s -= L[k * R + a] * x[k];
                x[a] = s / L[a * R + a];
            }
            memcpy(u, x, R * sizeof(double));
        }
    } else {
        double* A = (double*)malloc(R * R * sizeof(double));
        double* E = (double*)malloc(R * R * sizeof(double));
        for (u64 a = 0; a < R; ++a)
            for (u64 b = 0; b <= a; ++b) A[a * R + b] = A[b * R + a] = V[a * R + b];
        jacobi_eig(A, E, (int)R);
        double emax = 0.0;
        for (u64 a = 0; a < R; ++a) if (fabs(A[a * R + a]) > emax) emax = fabs(A[a * R + a]);
        double tol = emax * (double)R * 2.220446049250313e-16;
        double* P = (double*)calloc(R * R, sizeof(double));
        for (u64 k = 0; k < R; ++k) {
            double ev = A[k * R + k];
            if (fabs(ev) <= tol) continue;
            for (u64 a = 0; a < R; ++a)
                for (u64 b = 0; b < R; ++b) P[a * R + b] += E[a * R + k] * E[b * R + k] / ev;
        }
        for (u64 i = 0; i < rows; ++i) {
            double* u = U + i * R;
            for (u64 a = 0; a < R; ++a) {
                double s = 0.0;
                for (u64 b = 0; b < R; ++b) s += u[b] * P[b * R + a];
                x[a] = s;
            }
            memcpy(u, x, R * sizeof(double));
        }
        free(A); free(E); free(P);
    }
    free(x); free(L); free(V);
    return !ok;
}

/* pseudo_inverse on Grams given as one nmode x R x R array; returns 1 when
 * the pseudo-inverse (not the Cholesky solve) was used. */
int orc_pseudo_inverse(const double* grams, int nmode, int mode, double* U, uint64_t rows, uint64_t R)
{
    double* G[8];
    for (int m = 0; m < nmode; ++m) G[m] = (double*)(grams + (size_t)m * R * R);
    return pseudo_inverse(G, nmode, mode, U, rows, R);
}

/* cpd_fit_alto (include/cpd.hpp:189-271). */
static double fit_alto(int nmode, const u64* dims, double* const* U,
                       const double* lambda, double** G, const double* Umt,
                       u64 R, double normAT)
{
    int last = nmode - 1;
    double inner = 0.0;
    double* acc = (double*)calloc(R, sizeof(double));
    for (u64 i = 0; i < dims[last]; ++i)
        for (u64 r = 0; r < R; ++r) acc[r] += U[last][i * R + r] * Umt[i * R + r];
    for (u64 r = 0; r < R; ++r) inner += acc[r] * lambda[r];
    double normU = 0.0;
    for (u64 a = 0; a < R; ++a)
        for (u64 b = 0; b <= a; ++b) {
            double t = lambda[a] * lambda[b];
            for (int m = 0; m < nmode; ++m) t *= G[m][a * R + b];
            normU += (a == b) ? t : 2.0 * t;
        }
    normU = fabs(normU);
    double res = normAT + normU - 2.0 * inner;
    if (res > 0.0) res = sqrt(res);
    free(acc);
    return 1.0 - res / sqrt(normAT);
}

int orc_cpd_als(const orc_alto* at, double* const* U, double* lambda,
                uint64_t R, int max_iters, double epsilon, double* fits)
{
    int nm = at->nmode;
    double normAT = 0.0;
    for (u64 i = 0; i < at->nnz; ++i) normAT += at->vals[i] * at->vals[i];
    double* G[ORC_MAX_MODES];
    for (int m = 0; m < nm; ++m) {
        G[m] = (double*)malloc(R * R * sizeof(double));
        orc_gram(U[m], at->dims[m], R, G[m]);
    }
    double* scratch = (double*)malloc(at->dims[nm - 1] * R * sizeof(double));
    double fit = 0.0, prev = 0.0;
    int it = 0;
    for (int i = 0; i < max_iters; ++i) {
        for (int j = 0; j < nm; ++j) {
            memset(U[j], 0, at->dims[j] * R * sizeof(double));
            orc_mttkrp(at, j, U, R);
            if (j == nm - 1) memcpy(scratch, U[j], at->dims[j] * R * sizeof(double));
            pseudo_inverse(G, nm, j, U[j], at->dims[j], R);
            col_norm(U[j], at->dims[j], R, lambda, i > 0);
            orc_gram(U[j], at->dims[j], R, G[j]);
        }
        fit = fit_alto(nm, at->dims, U, lambda, G, scratch, R, normAT);
        if (fits) fits[i] = fit;
        it = i + 1;
        if (i > 0 && fabs(prev - fit) < epsilon) break;
        prev = fit;
    }
    for (int m = 0; m < nm; ++m) free(G[m]);
    free(scratch);
    return it;
}

/* ---- CP-APR (include/apr.hpp) ---- */

void orc_phi(const orc_alto* at, int mode, double* const* U, uint64_t R,
             double eps_div_zero, double* phi)
{
    const double* B = U[mode];
    double* row = (double*)malloc(R * sizeof(double));
    memset(phi, 0, at->dims[mode] * R * sizeof(double));
    for (u64 i = 0; i < at->nnz; ++i) {
        u128 a = at->idx[i];
        krp_row(at, a, 1.0, mode, U, R, row);
        u64 t = pext128(a, at->masks[mode]);
        double v = 0.0;
        for (u64 r = 0; r < R; ++r) v += B[t * R + r] * row[r];
        v = at->vals[i] / fmax(v, eps_div_zero);
        for (u64 r = 0; r < R; ++r) phi[t * R + r] += v * row[r];
    }
    free(row);
}

double orc_loglik(const orc_alto* at, double* const* U, double* lambda,
                  uint64_t R, double eps_div_zero)
{
    redistribute(U[0], at->dims[0], R, lambda);
    double logsum = 0.0;
    for (u64 i = 0; i < at->nnz; ++i) {
        double tmp = 0.0;
        for (u64 r = 0; r < R; ++r) {
            double p = 1.0;
            for (int n = 0; n < at->nmode; ++n)
                p *= U[n][pext128(at->idx[i], at->masks[n]) * R + r];
            tmp += p;
        }
        if (tmp < eps_div_zero) tmp = eps_div_zero;
        logsum += at->vals[i] * log(tmp);
    }
    double fsum = 0.0;
    for (u64 k = 0; k < at->dims[0] * R; ++k) fsum += U[0][k];
    for (u64 r = 0; r < R; ++r) {
        double t = 0.0;
        for (u64 i = 0; i < at->dims[0]; ++i) t += fabs(U[0][i * R + r]);
        for (u64 i = 0; i < at->dims[0]; ++i) U[0][i * R + r] /= t;
        lambda[r] *= t;
    }
    return logsum - fsum;
}

int orc_cp_apr(const orc_alto* at, double* const* U, double* lambda,
               uint64_t R, int max_iters, int max_inner, double epsilon,
               double eps_div_zero, double kappa_tol, double kappa,
               int dobench, double* out, double* kkt_trace)
{
    int nm = at->nmode;
    double* Phi[ORC_MAX_MODES];
    for (int n = 0; n < nm; ++n) Phi[n] = (double*)calloc(at->dims[n] * R, sizeof(double));
    double kmode[ORC_MAX_MODES] = {0};
    double* kkt = (double*)calloc((size_t)max_iters + 1, sizeof(double));
    int* ninner = (int*)calloc((size_t)max_iters + 1, sizeof(int));
    for (int n = 0; n < nm; ++n) normalize_mode(U[n], at->dims[n], R, lambda);
    int iter;
    for (iter = 0; iter < max_iters; ++iter) {
        int converged = 0;
        for (int n = 0; n < nm; ++n) {
            u64 sz = at->dims[n] * R;
            double* B = U[n];
            if (iter > 0)
                for (u64 k = 0; k < sz; ++k)
                    if (B[k] < kappa_tol && Phi[n][k] > 1.0) B[k] += kappa;
            redistribute(B, at->dims[n], R, lambda);
            for (int inner = 0; inner < max_inner; ++inner) {
                ninner[iter]++;
                orc_phi(at, n, U, R, eps_div_zero, Phi[n]);
                double kv = 0.0;
                for (u64 k = 0; k < sz; ++k) {
                    double mc = fabs(fmin(B[k], 1.0 - Phi[n][k]));
                    kv = fmax(kv, mc);
                }
                kmode[n] = kv;
                if (kv < epsilon && !dobench) break;
                for (u64 k = 0; k < sz; ++k) B[k] *= Phi[n][k];
            }
            normalize_mode(B, at->dims[n], R, lambda);
        }
        kkt[iter] = kmode[0];
        for (int n = 1; n < nm; ++n) kkt[iter] = fmax(kkt[iter], kmode[n]);
        if (kkt_trace) kkt_trace[iter] = kkt[iter];
        if (iter > 0 && fabs(kkt[iter] - kkt[iter - 1]) <= epsilon * epsilon && !dobench)
            converged = 1;
        if (converged) break;
    }
    int tot_inner = 0;
    for (int i = 0; i < iter; ++i) tot_inner += ninner[i];
    double ll = orc_loglik(at, U, lambda, R, eps_div_zero);
    /* Post-processing least-squares fit, include/apr.hpp:1301-1330. */
    double* G[ORC_MAX_MODES];
    for (int n = 0; n < nm; ++n) {
        G[n] = (double*)malloc(R * R * sizeof(double));
        orc_gram(U[n], at->dims[n], R, G[n]);
    }
    double* mt = (double*)calloc(at->dims[nm - 1] * R, sizeof(double));
    double* Utmp[ORC_MAX_MODES];
    for (int n = 0; n < nm; ++n) Utmp[n] = U[n];
    Utmp[nm - 1] = mt;
    {
        /* mttkrp_ (apr.hpp:127-186): plain sum into a zeroed matrix; it only
         * reads the other modes' factors. */
        double* row = (double*)malloc(R * sizeof(double));
        for (u64 i = 0; i < at->nnz; ++i) {
            krp_row(at, at->idx[i], at->vals[i], nm - 1, Utmp, R, row);
            double* o = mt + pext128(at->idx[i], at->masks[nm - 1]) * R;
            for (u64 r = 0; r < R; ++r) o[r] += row[r];
        }
        free(row);
    }
    double normAT = 0.0;
    for (u64 i = 0; i < at->nnz; ++i) normAT += at->vals[i] * at->vals[i];
    double fit = fit_alto(nm, at->dims, U, lambda, G, mt, R, normAT);
    if (out) {
        out[0] = ll;
        out[1] = fit;
        out[2] = iter > 0 ? kkt[iter - 1] : kkt[0];
        out[3] = iter;
        out[4] = tot_inner;
        out[5] = out[6] = out[7] = 0.0;
    }
    for (int n = 0; n < nm; ++n) { free(Phi[n]); free(G[n]); }
    free(mt); free(kkt); free(ninner);
    return iter;
}
