// dense_kernels.cuh -- device bodies and kernels of the dense CP updates
// (see dense.cuh for the reference functions they replace).  The bodies take
// an explicit block index so that the batched solver (batch.cu) can run one
// tensor per blockIdx.y with the same code.
#pragma once

#include "dense.cuh"

namespace altob {

// ------------------------------------------------------------------ helpers

__device__ __forceinline__ void atomic_max_pos(double* addr, double v)
{
    // v >= 0: IEEE order of non-negative doubles equals their integer order
    atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

static int dn_grid(u64 work, u64 per_block)
{
    u64 b = (work + per_block - 1) / per_block;
    return (int)std::max<u64>(1, std::min<u64>(b, (u64)num_sms() * 4));
}

// ------------------------------------------------------------------- Gram
// G += X^T X (FP64, full symmetric) with X = U / div (column-wise) when div
// is given; X is written back to Uout when given; inner[r] += sum_i X[i,r] *
// M[i,r] when M is given (cpd_fit_alto's inner product, cpd.hpp:207-213).
// 4x4 register tiles of the lower triangle; rows of a staged chunk are split
// across thread groups when there are fewer tiles than threads.  A chunk holds
// GR_ELEMS elements whatever the rank (GR_ELEMS / R rows), so small ranks
// still keep GR_LD loads in flight per thread between barriers.

constexpr int GR_TB = 4;
constexpr int GR_ELEMS = 4096;
constexpr int GR_LD = 8;      // staged elements in flight per thread
constexpr int GR_SMALL = 88;  // R <= 88: at most 253 tiles, one per thread

template <typename FT, int MAXT>
__device__ __forceinline__ void gram_body(const FT* __restrict__ U, u64 I, int R, double* __restrict__ G,
                                          const double* __restrict__ div, FT* __restrict__ Uout,
                                          const FT* __restrict__ M, double* __restrict__ inner, u64 bx, u64 nbx)
{
    extern __shared__ __align__(16) double gsm[];
    const int RS = (R + 3) & ~3;       // row stride in shared memory (zero padding)
    const int rows = GR_ELEMS / RS;    // rows per chunk
    double* s = gsm;                   // rows x RS (<= GR_ELEMS)
    double* si = gsm + GR_ELEMS;       // R (inner partial)
    double* sdiv = si + R;             // R (divisors)
    const int tid = threadIdx.x;
    const int T = (R + GR_TB - 1) / GR_TB;
    const int NT = T * (T + 1) / 2;
    const int groups = NT >= DN_THREADS ? 1 : DN_THREADS / NT;
    const int grp = NT >= DN_THREADS ? 0 : tid / NT;
    const bool active = NT >= DN_THREADS || tid < groups * NT;
    int ta[MAXT], tb[MAXT];
    double acc[MAXT][GR_TB * GR_TB];
#pragma unroll
    for (int k = 0; k < MAXT; ++k) {
        int t = NT >= DN_THREADS ? tid + k * DN_THREADS : tid % NT;
        if (NT < DN_THREADS && k > 0) t = NT;  // only one tile
        int a = 0;
        while ((a + 1) * (a + 2) / 2 <= t) ++a;
        ta[k] = t < NT ? a : -1;
        tb[k] = t < NT ? t - a * (a + 1) / 2 : -1;
#pragma unroll
        for (int e = 0; e < GR_TB * GR_TB; ++e) acc[k][e] = 0.0;
    }
    for (int r = tid; r < R; r += DN_THREADS) {
        si[r] = 0.0;
        sdiv[r] = div ? div[r] : 1.0;
    }
    if (RS != R)  // padding columns stay zero for every chunk
        for (int e = tid; e < rows * (RS - R); e += DN_THREADS) s[(e / (RS - R)) * RS + R + e % (RS - R)] = 0.0;
    __syncthreads();
    // element e of a chunk sits in column (e mod R); for R dividing the
    // block size that column is the same for every element of a thread
    const bool fixed_col = DN_THREADS % R == 0;
    const int col_step = DN_THREADS % R, row_step = DN_THREADS / R;
    double pin = 0.0;
    const u64 nchunks = (I + rows - 1) / rows;
    for (u64 ch = bx; ch < nchunks; ch += nbx) {
        const u64 r0 = ch * rows;
        const int nrows = (int)min((u64)rows, I - r0);
        const int tot = rows * R, valid = nrows * R;
        const u64 base = r0 * (u64)R;  // a chunk is contiguous in memory
        __syncthreads();
        int col = tid % R, row = tid / R;
        for (int e0 = 0; e0 < tot; e0 += GR_LD * DN_THREADS) {
            FT v[GR_LD], mv[GR_LD];
#pragma unroll
            for (int q = 0; q < GR_LD; ++q) {
                const int e = e0 + q * DN_THREADS + tid;
                v[q] = e < valid ? U[base + e] : FT(0);
                mv[q] = (M && e < valid) ? M[base + e] : FT(0);
            }
#pragma unroll
            for (int q = 0; q < GR_LD; ++q) {
                const int e = e0 + q * DN_THREADS + tid;
                if (e < tot) {
                    double x = (double)v[q];
                    if (e < valid) {
                        if (div) {
                            x = x / sdiv[col];
                            if (Uout) Uout[base + e] = (FT)x;
                            x = (double)(FT)x;
                        }
                        if (M) {
                            if (fixed_col) pin += x * (double)mv[q];
                            else atomicAdd(&si[col], x * (double)mv[q]);
                        }
                    }
                    s[row * RS + col] = x;
                }
                col += col_step;
                row += row_step;
                if (col >= R) {
                    col -= R;
                    ++row;
                }
            }
        }
        __syncthreads();
        if (!active) continue;
#pragma unroll
        for (int k = 0; k < MAXT; ++k) {
            if (ta[k] < 0) continue;
            const int a0 = ta[k] * GR_TB, b0 = tb[k] * GR_TB;
            for (int row = grp; row < nrows; row += groups) {
                const double* sr = s + row * RS;
                // RS and the tile offsets are multiples of 4: 16-byte aligned pairs
                const double2 a01 = *reinterpret_cast<const double2*>(sr + a0);
                const double2 a23 = *reinterpret_cast<const double2*>(sr + a0 + 2);
                const double2 b01 = *reinterpret_cast<const double2*>(sr + b0);
                const double2 b23 = *reinterpret_cast<const double2*>(sr + b0 + 2);
                double xa[GR_TB], xb[GR_TB];
                xa[0] = a01.x;
                xa[1] = a01.y;
                xa[2] = a23.x;
                xa[3] = a23.y;
                xb[0] = b01.x;
                xb[1] = b01.y;
                xb[2] = b23.x;
                xb[3] = b23.y;
#pragma unroll
                for (int p = 0; p < GR_TB; ++p)
#pragma unroll
                    for (int q = 0; q < GR_TB; ++q) acc[k][p * GR_TB + q] += xa[p] * xb[q];
            }
        }
    }
    // row groups hold partial copies of the same tiles: sum them in shared
    // memory (the staging buffer is free now) so each tile entry takes one
    // global atomic per CTA
    bool flush = active;
    if (MAXT == 1 && groups > 1) {
        __syncthreads();
        if (active)
#pragma unroll
            for (int e = 0; e < GR_TB * GR_TB; ++e) s[tid * GR_TB * GR_TB + e] = acc[0][e];
        __syncthreads();
        flush = tid < NT;
        if (flush)
            for (int g = 1; g < groups; ++g)
#pragma unroll
                for (int e = 0; e < GR_TB * GR_TB; ++e) acc[0][e] += s[(g * NT + tid) * GR_TB * GR_TB + e];
    }
    if (flush) {
#pragma unroll
        for (int k = 0; k < MAXT; ++k) {
            if (ta[k] < 0) continue;
            const int a0 = ta[k] * GR_TB, b0 = tb[k] * GR_TB;
#pragma unroll
            for (int p = 0; p < GR_TB; ++p)
#pragma unroll
                for (int q = 0; q < GR_TB; ++q) {
                    const int a = a0 + p, b = b0 + q;
                    if (a < R && b < R && a >= b) {
                        atomicAdd(&G[a * R + b], acc[k][p * GR_TB + q]);
                        if (a != b) atomicAdd(&G[b * R + a], acc[k][p * GR_TB + q]);
                    }
                }
        }
    }
    if (M) {
        if (fixed_col) atomicAdd(&si[tid % R], pin);
        __syncthreads();
        for (int r = tid; r < R; r += DN_THREADS) atomicAdd(&inner[r], si[r]);
    }
}

template <typename FT, int MAXT>
__global__ void __launch_bounds__(DN_THREADS) k_gram(const FT* __restrict__ U, u64 I, int R, double* __restrict__ G,
                                                     const double* __restrict__ div, FT* __restrict__ Uout,
                                                     const FT* __restrict__ M, double* __restrict__ inner)
{
    gram_body<FT, MAXT>(U, I, R, G, div, Uout, M, inner, blockIdx.x, gridDim.x);
}


constexpr int JAC_MAX_PAIRS = (SOLVE_MAX_RANK + 1) / 2;
constexpr int JAC_SWEEPS = 40;

__device__ __forceinline__ void solve_body(const double* __restrict__ G, int nmode, int target, int R,
                                           double* __restrict__ W, int* __restrict__ info)
{
    extern __shared__ double ssm[];
    double* A = ssm;          // R x R
    double* B = ssm + R * R;  // R x R
    __shared__ int ok;
    const int tid = threadIdx.x;
    for (int e = tid; e < R * R; e += DN_THREADS) {
        const int a = e / R, b = e - a * R;
        const int lo = a >= b ? e : b * R + a;  // symmetric from the lower triangle
        double v = 1.0;
        for (int m = 0; m < nmode; ++m)
            if (m != target) v *= G[(size_t)m * R * R + lo];
        A[e] = v;
        B[e] = v;
    }
    if (tid == 0) ok = 1;
    __syncthreads();
    // right-looking Cholesky of A (lower)
    for (int k = 0; k < R; ++k) {
        if (tid == 0) {
            double d = A[k * R + k];
            if (!(d > 0.0)) ok = 0;
            else A[k * R + k] = sqrt(d);
        }
        __syncthreads();
        if (!ok) break;
        const double dk = A[k * R + k];
        for (int i = k + 1 + tid; i < R; i += DN_THREADS) A[i * R + k] /= dk;
        __syncthreads();
        const int n = R - k - 1;
        for (int e = tid; e < n * n; e += DN_THREADS) {
            const int i = k + 1 + e / n, j = k + 1 + e % n;
            if (j <= i) A[i * R + j] -= A[i * R + k] * A[j * R + k];
        }
        __syncthreads();
    }
    if (ok) {
        // Linv (lower) into B, column by column
        for (int c = tid; c < R; c += DN_THREADS) {
            for (int i = 0; i < R; ++i) B[i * R + c] = 0.0;
            B[c * R + c] = 1.0 / A[c * R + c];
            for (int i = c + 1; i < R; ++i) {
                double s = 0.0;
                for (int k = c; k < i; ++k) s += A[i * R + k] * B[k * R + c];
                B[i * R + c] = -s / A[i * R + i];
            }
        }
        __syncthreads();
        for (int e = tid; e < R * R; e += DN_THREADS) {
            const int a = e / R, b = e - a * R;
            const int k0 = a > b ? a : b;
            double s = 0.0;
            for (int k = k0; k < R; ++k) s += B[k * R + a] * B[k * R + b];
            W[e] = s;
        }
        return;
    }
    // ---- pseudo-inverse fallback: A = V (symmetric), B = eigenvectors.
    // Two-sided Jacobi with the round-robin (tournament) ordering: each step
    // rotates n/2 disjoint index pairs at once (n = R rounded up to even; the
    // extra index is a dummy), n-1 steps make a sweep.  Sweeps stop when the
    // off-diagonal mass is below 1e-26 of the total (eigenvectors to ~1e-13),
    // at most JAC_SWEEPS of them.
    for (int e = tid; e < R * R; e += DN_THREADS) {
        const int a = e / R, b = e - a * R;
        A[e] = a >= b ? B[e] : B[b * R + a];
    }
    __syncthreads();
    for (int e = tid; e < R * R; e += DN_THREADS) B[e] = (e / R == e % R) ? 1.0 : 0.0;
    const int n = (R + 1) & ~1, half = n / 2;
    __shared__ double jc[JAC_MAX_PAIRS], js[JAC_MAX_PAIRS];
    __shared__ int jp[JAC_MAX_PAIRS], jq[JAC_MAX_PAIRS];
    __shared__ double red[2 * (DN_THREADS / 32)];
    __syncthreads();
    for (int sweep = 0; sweep < JAC_SWEEPS; ++sweep) {
        // convergence test: block sums of squares (off-diagonal, total)
        double off = 0.0, tot = 0.0;
        for (int e = tid; e < R * R; e += DN_THREADS) {
            const double x = A[e] * A[e];
            tot += x;
            if (e / R != e % R) off += x;
        }
        for (int o = 16; o; o >>= 1) {
            off += __shfl_xor_sync(0xffffffffu, off, o);
            tot += __shfl_xor_sync(0xffffffffu, tot, o);
        }
        if ((tid & 31) == 0) {
            red[2 * (tid >> 5)] = off;
            red[2 * (tid >> 5) + 1] = tot;
        }
        __syncthreads();
        if (tid == 0) {
            double o2 = 0.0, t2 = 0.0;
            for (int w = 0; w < DN_THREADS / 32; ++w) {
                o2 += red[2 * w];
                t2 += red[2 * w + 1];
            }
            ok = o2 <= 1e-26 * t2;
        }
        __syncthreads();
        if (ok) break;
        for (int step = 0; step < n - 1; ++step) {
            // pair i: positions i and n-1-i of the arrangement [0, rotating 1..n-1]
            for (int i = tid; i < half; i += DN_THREADS) {
                const int a = i == 0 ? 0 : ((i - 1 + step) % (n - 1)) + 1;
                const int bpos = n - 1 - i;
                const int b = ((bpos - 1 + step) % (n - 1)) + 1;
                const int p = a < b ? a : b, q = a < b ? b : a;
                double c = 1.0, sn = 0.0;
                if (q < R) {
                    const double apq = A[p * R + q];
                    if (apq != 0.0) {
                        const double th = (A[q * R + q] - A[p * R + p]) / (2.0 * apq);
                        const double t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
                        c = 1.0 / sqrt(t * t + 1.0);
                        sn = t * c;
                    }
                }
                jp[i] = p;
                jq[i] = q;
                jc[i] = c;
                js[i] = sn;
            }
            __syncthreads();
            // columns p, q of A for every pair
            for (int w = tid; w < half * R; w += DN_THREADS) {
                const int i = w / R, k = w - i * R;
                const int p = jp[i], q = jq[i];
                if (q >= R || js[i] == 0.0) continue;
                const double c = jc[i], sn = js[i];
                const double akp = A[k * R + p], akq = A[k * R + q];
                A[k * R + p] = c * akp - sn * akq;
                A[k * R + q] = sn * akp + c * akq;
            }
            __syncthreads();
            // rows p, q of A and columns p, q of the eigenvectors
            for (int w = tid; w < half * R; w += DN_THREADS) {
                const int i = w / R, k = w - i * R;
                const int p = jp[i], q = jq[i];
                if (q >= R || js[i] == 0.0) continue;
                const double c = jc[i], sn = js[i];
                const double apk = A[p * R + k], aqk = A[q * R + k];
                A[p * R + k] = c * apk - sn * aqk;
                A[q * R + k] = sn * apk + c * aqk;
                const double vkp = B[k * R + p], vkq = B[k * R + q];
                B[k * R + p] = c * vkp - sn * vkq;
                B[k * R + q] = sn * vkp + c * vkq;
            }
            __syncthreads();
        }
    }
    __syncthreads();
    double emax = 0.0;
    for (int k = 0; k < R; ++k) emax = fmax(emax, fabs(A[k * R + k]));
    const double tol = emax * R * 2.220446049250313e-16;
    for (int e = tid; e < R * R; e += DN_THREADS) {
        const int a = e / R, b = e - a * R;
        double s = 0.0;
        for (int k = 0; k < R; ++k) {
            const double ev = A[k * R + k];
            if (fabs(ev) > tol) s += B[a * R + k] * B[b * R + k] / ev;
        }
        W[e] = s;
    }
    if (tid == 0) atomicAdd(info, 1);
}

static __global__ void __launch_bounds__(DN_THREADS) k_solve_setup(const double* __restrict__ G, int nmode, int target,
                                                            int R, double* __restrict__ W, int* __restrict__ info)
{
    solve_body(G, nmode, target, R, W, info);
}

// Row apply: a row is held by LPR lanes, CJ columns per lane (column c =
// l + LPR * j), AP_RW rows per lane group; 32 / LPR row groups per warp, so
// small ranks keep every lane busy.  Row k of W is read from shared memory,
// the u[i][k] operand is shuffled from the lane that holds it.
constexpr int AP_RW = 4;

template <typename FT, int LPR, int CJ>
__device__ __forceinline__ void apply_body(FT* __restrict__ U, u64 I, int R, const double* __restrict__ Wg, int nk,
                                           double* __restrict__ colacc, u64 bx, u64 nbx)
{
    constexpr int NG = 32 / LPR;  // row groups per warp
    constexpr int ROWS_WARP = NG * AP_RW;
    extern __shared__ double asm_[];
    double* W = asm_;           // R x R
    double* cr = asm_ + R * R;  // R column partials
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane / LPR, l = lane % LPR;
    for (int e = tid; e < R * R; e += DN_THREADS) W[e] = Wg[e];
    for (int r = tid; r < R; r += DN_THREADS) cr[r] = nk == NORM_MAX ? 1.0 : 0.0;
    __syncthreads();
    double part[CJ];
#pragma unroll
    for (int j = 0; j < CJ; ++j) part[j] = nk == NORM_MAX ? 1.0 : 0.0;
    const u64 step = nbx * (DN_THREADS / 32) * ROWS_WARP;
    for (u64 w0 = (bx * (DN_THREADS / 32) + warp) * ROWS_WARP; w0 < I; w0 += step) {
        const u64 i0 = w0 + (u64)g * AP_RW;
        double u[AP_RW][CJ], x[AP_RW][CJ];
#pragma unroll
        for (int rw = 0; rw < AP_RW; ++rw)
#pragma unroll
            for (int j = 0; j < CJ; ++j) {
                const int c = l + LPR * j;
                const u64 i = i0 + rw;
                u[rw][j] = (c < R && i < I) ? (double)U[i * R + c] : 0.0;
                x[rw][j] = 0.0;
            }
        for (int a = 0; a < R; ++a) {
            const int ja = a / LPR, la = g * LPR + (a % LPR);
            double ua[AP_RW];
#pragma unroll
            for (int rw = 0; rw < AP_RW; ++rw) {
                double v = u[rw][0];
#pragma unroll
                for (int j = 1; j < CJ; ++j)
                    if (j == ja) v = u[rw][j];
                ua[rw] = __shfl_sync(0xffffffffu, v, la);
            }
#pragma unroll
            for (int j = 0; j < CJ; ++j) {
                const int b = l + LPR * j;
                if (b < R) {
                    const double w = W[a * R + b];
#pragma unroll
                    for (int rw = 0; rw < AP_RW; ++rw) x[rw][j] += ua[rw] * w;
                }
            }
        }
#pragma unroll
        for (int rw = 0; rw < AP_RW; ++rw) {
            const u64 i = i0 + rw;
            if (i >= I) continue;
#pragma unroll
            for (int j = 0; j < CJ; ++j) {
                const int b = l + LPR * j;
                if (b < R) {
                    const FT y = (FT)x[rw][j];
                    U[i * R + b] = y;
                    const double yd = (double)y;
                    if (nk == NORM_2) part[j] += yd * yd;
                    else if (nk == NORM_MAX) part[j] = fmax(part[j], yd);
                }
            }
        }
    }
    if (nk != NORM_NONE) {
#pragma unroll
        for (int j = 0; j < CJ; ++j) {
            const int b = l + LPR * j;
            if (b < R) {
                if (nk == NORM_2) atomicAdd(&cr[b], part[j]);
                else atomic_max_pos(&cr[b], part[j]);
            }
        }
        __syncthreads();
        for (int r = tid; r < R; r += DN_THREADS) {
            if (nk == NORM_2) atomicAdd(&colacc[r], cr[r]);
            else atomic_max_pos(&colacc[r], cr[r]);
        }
    }
}

template <typename FT, int LPR, int CJ>
__global__ void __launch_bounds__(DN_THREADS) k_apply(FT* __restrict__ U, u64 I, int R, const double* __restrict__ Wg,
                                                      int nk, double* __restrict__ colacc)
{
    apply_body<FT, LPR, CJ>(U, I, R, Wg, nk, colacc, blockIdx.x, gridDim.x);
}

// ------------------------------------------------ fused row update + Gram
// One pass over the MTTKRP output M (held in U) for R <= 8*MB:
//   Y = M W                      (FP64 tensor-core MMA, m8n8k4)
//   U <- (FT) Y                  (in place)
//   colacc: column 2-norm^2 / running max of the stored Y
//   G' += Y^T Y                  (FP64 MMA over the rows of the warp's tile)
//   inner'[r] += Y[:,r] . M[:,r] (when inner is given: the fit's inner product)
// The caller then takes lambda from colacc, G = G' / (lambda lambda^T),
// inner = inner' / lambda and divides U by lambda, which equals the
// reference's apply -> normalise -> Gram order (cpd.hpp:102-163) up to the
// rounding of the stored FT values.
//
// The product is formed transposed, Y^T = W^T M^T, so that the accumulator
// fragment of an 8-row tile (lane (g, t) holds Y[r0 + 2t + i][8mb + g],
// g = lane / 4, t = lane % 4) is directly the A and B operand of the Gram
// MMA whose k index runs over the tile's rows (row r0 + 2k + i in MMA i):
// no shuffles, no shared-memory transpose.  The k index of the row update is
// permuted (input column t*KS + kk at k-step kk, lane slot t) so that each
// lane's operand columns are contiguous in its row (vector loads).

__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

constexpr int AG_THREADS = 128;
constexpr int AG_WARPS = AG_THREADS / 32;

// W^T fragments (later the block's Gram), column statistics and inner
// partials per warp, and their block totals
template <int MB>
constexpr size_t apply_gram_smem()
{
    return (size_t)(64 * MB * MB + 2 * 8 * MB * (AG_WARPS + 1)) * sizeof(double);
}

// KS consecutive FT values of a row (columns c0.., zero beyond R).  Plain
// loads, not the read-only path: the same warp overwrites the row later.
template <typename FT, int KS>
__device__ __forceinline__ void load_run(const FT* __restrict__ p, int c0, int R, bool full, bool row_ok, FT* v)
{
    constexpr int VB = (KS * (int)sizeof(FT)) % 16 == 0 ? 16 : (KS * (int)sizeof(FT)) % 8 == 0 ? 8 : 0;
    if (VB && full && row_ok) {
        constexpr int PER = VB ? VB / (int)sizeof(FT) : 1;
#pragma unroll
        for (int q = 0; q < KS / PER; ++q) {
            if constexpr (VB == 16 && sizeof(FT) == 4) {
                const float4 x = reinterpret_cast<const float4*>(p + c0)[q];
                v[4 * q] = x.x, v[4 * q + 1] = x.y, v[4 * q + 2] = x.z, v[4 * q + 3] = x.w;
            } else if constexpr (VB == 16) {
                const double2 x = reinterpret_cast<const double2*>(p + c0)[q];
                v[2 * q] = x.x, v[2 * q + 1] = x.y;
            } else if constexpr (sizeof(FT) == 4) {
                const float2 x = reinterpret_cast<const float2*>(p + c0)[q];
                v[2 * q] = x.x, v[2 * q + 1] = x.y;
            } else {
                v[q] = p[c0 + q];
            }
        }
        return;
    }
#pragma unroll
    for (int k = 0; k < KS; ++k) v[k] = (row_ok && c0 + k < R) ? p[c0 + k] : FT(0);
}

template <typename FT, int MB>
__device__ __forceinline__ void apply_gram_body(FT* __restrict__ U, u64 I, int R, const double* __restrict__ Wg,
                                                int nk, double* __restrict__ colacc, double* __restrict__ G,
                                                double* __restrict__ inner, int vec_ok, u64 bx, u64 nbx)
{
    constexpr int KS = 2 * MB;             // k-steps of the row update (4 input columns each)
    constexpr int NB = MB * (MB + 1) / 2;  // Gram blocks a >= b
    constexpr int RP = 8 * MB;             // rank padded to the MMA tile
    // MB <= 4 keeps the column statistics in registers; larger blocks keep
    // them per warp in shared memory to stay within 255 registers
    constexpr bool SREG = MB <= 4;
    extern __shared__ __align__(16) double ags[];
    double* wf = ags;                 // MB*KS*32 W^T fragments in lane order; the Gram at the end
    double* cw = wf + 64 * MB * MB;   // AG_WARPS x RP column statistics per warp
    double* iw = cw + AG_WARPS * RP;  // AG_WARPS x RP inner partials per warp
    double* cs = iw + AG_WARPS * RP;  // RP block column statistics
    double* is = cs + RP;             // RP block inner partials
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t4 = lane & 3;
    const double sinit = nk == NORM_MAX ? 1.0 : 0.0;
    for (int e = tid; e < MB * KS * 32; e += AG_THREADS) {
        const int l = e & 31, kk = (e >> 5) % KS, mb = (e >> 5) / KS;
        const int row = (l & 3) * KS + kk, col = 8 * mb + (l >> 2);
        wf[e] = (row < R && col < R) ? Wg[row * R + col] : 0.0;
    }
    for (int e = tid; e < AG_WARPS * RP; e += AG_THREADS) {
        cw[e] = sinit;
        iw[e] = 0.0;
    }
    __syncthreads();
    const bool full = R == RP && vec_ok;  // vector loads: whole rows, 16-byte aligned base
    double gacc[NB][2], cst[SREG ? MB : 1], ipt[SREG ? MB : 1];
#pragma unroll
    for (int q = 0; q < NB; ++q) gacc[q][0] = gacc[q][1] = 0.0;
#pragma unroll
    for (int mb = 0; mb < (SREG ? MB : 1); ++mb) {
        cst[mb] = sinit;
        ipt[mb] = 0.0;
    }
    const u64 step = nbx * (u64)AG_WARPS * 8;
    for (u64 r0 = (bx * AG_WARPS + warp) * 8; r0 < I; r0 += step) {
        FT bf[KS];
        load_run<FT, KS>(U + (r0 + g) * R, t4 * KS, R, full, r0 + g < I, bf);
        double y[MB][2];
#pragma unroll
        for (int mb = 0; mb < MB; ++mb) {
            y[mb][0] = y[mb][1] = 0.0;
#pragma unroll
            for (int kk = 0; kk < KS; ++kk)
                dmma884(y[mb][0], y[mb][1], wf[(mb * KS + kk) * 32 + lane], (double)bf[kk]);
        }
        // the inner product's M operand is read by the lane that overwrites
        // it, just before the store (same thread, same address: ordered)
        FT mv[MB][2];
        if (inner) {
#pragma unroll
            for (int mb = 0; mb < MB; ++mb)
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    const u64 row = r0 + 2 * t4 + i;
                    const int col = 8 * mb + g;
                    mv[mb][i] = (row < I && col < R) ? U[row * R + col] : FT(0);
                }
        }
#pragma unroll
        for (int mb = 0; mb < MB; ++mb) {
            double c = SREG ? cst[mb] : sinit, p = SREG ? ipt[mb] : 0.0;
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const u64 row = r0 + 2 * t4 + i;
                const int col = 8 * mb + g;
                const FT yf = (FT)y[mb][i];
                const double yd = (double)yf;
                y[mb][i] = yd;  // rows past I and columns past R are exact zeros
                if (row < I && col < R) U[row * R + col] = yf;
                if (nk == NORM_2) c += yd * yd;
                else if (nk == NORM_MAX) c = fmax(c, yd);
                if (inner) p += yd * (double)mv[mb][i];
            }
            if constexpr (SREG) {
                cst[mb] = c;
                ipt[mb] = p;
            } else {
                // lanes g, t = 0..3 hold the same column: combine, one lane updates
#pragma unroll
                for (int o = 1; o <= 2; o <<= 1) {
                    const double c2 = __shfl_xor_sync(0xffffffffu, c, o);
                    c = nk == NORM_MAX ? fmax(c, c2) : c + c2;
                    if (inner) p += __shfl_xor_sync(0xffffffffu, p, o);
                }
                if (t4 == 0) {
                    double* cp = cw + warp * RP + 8 * mb + g;
                    *cp = nk == NORM_MAX ? fmax(*cp, c) : *cp + c;
                    if (inner) iw[warp * RP + 8 * mb + g] += p;
                }
            }
        }
        int q = 0;
#pragma unroll
        for (int a = 0; a < MB; ++a)
#pragma unroll
            for (int b = 0; b <= a; ++b, ++q) {
                dmma884(gacc[q][0], gacc[q][1], y[a][0], y[b][0]);
                dmma884(gacc[q][0], gacc[q][1], y[a][1], y[b][1]);
            }
    }
    if constexpr (SREG) {
#pragma unroll
        for (int mb = 0; mb < MB; ++mb) {
            double c = cst[mb], p = ipt[mb];
#pragma unroll
            for (int o = 1; o <= 2; o <<= 1) {
                const double c2 = __shfl_xor_sync(0xffffffffu, c, o);
                c = nk == NORM_MAX ? fmax(c, c2) : c + c2;
                p += __shfl_xor_sync(0xffffffffu, p, o);
            }
            if (t4 == 0) {
                cw[warp * RP + 8 * mb + g] = c;
                iw[warp * RP + 8 * mb + g] = p;
            }
        }
    }
    __syncthreads();  // every warp is done with the W fragments: reuse them for the Gram
    double* gs = wf;  // RP*RP
    for (int e = tid; e < RP * RP; e += AG_THREADS) gs[e] = 0.0;
    for (int r = tid; r < RP; r += AG_THREADS) {
        double c = sinit, p = 0.0;
        for (int w = 0; w < AG_WARPS; ++w) {
            c = nk == NORM_MAX ? fmax(c, cw[w * RP + r]) : c + cw[w * RP + r];
            p += iw[w * RP + r];
        }
        cs[r] = c;
        is[r] = p;
    }
    __syncthreads();
    {
        int q = 0;
#pragma unroll
        for (int a = 0; a < MB; ++a)
#pragma unroll
            for (int b = 0; b <= a; ++b, ++q)
#pragma unroll
                for (int i = 0; i < 2; ++i) atomicAdd(&gs[(8 * a + g) * RP + 8 * b + 2 * t4 + i], gacc[q][i]);
    }
    __syncthreads();
    for (int e = tid; e < R * R; e += AG_THREADS) {
        const int a = e / R, b = e - a * R;
        if (a < b) continue;
        const double v = gs[a * RP + b];  // block(a) >= block(b): computed
        atomicAdd(&G[a * R + b], v);
        if (a != b) atomicAdd(&G[b * R + a], v);
    }
    for (int r = tid; r < R; r += AG_THREADS) {
        if (nk == NORM_2) atomicAdd(&colacc[r], cs[r]);
        else if (nk == NORM_MAX) atomic_max_pos(&colacc[r], cs[r]);
        if (inner) atomicAdd(&inner[r], is[r]);
    }
}

template <typename FT, int MB>
__global__ void __launch_bounds__(AG_THREADS) k_apply_gram(FT* __restrict__ U, u64 I, int R,
                                                           const double* __restrict__ W, int nk,
                                                           double* __restrict__ colacc, double* __restrict__ G,
                                                           double* __restrict__ inner, int vec_ok)
{
    apply_gram_body<FT, MB>(U, I, R, W, nk, colacc, G, inner, vec_ok, blockIdx.x, gridDim.x);
}

// lambda from the column statistics, G = G' / (lambda lambda^T), inner /= lambda
__device__ __forceinline__ void lambda_finish_body(const double* __restrict__ acc, int R, int nk,
                                                   double* __restrict__ lam, double* __restrict__ G,
                                                   double* __restrict__ inner)
{
    __shared__ double sl[SOLVE_MAX_RANK + 16];
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        const double l = nk == NORM_2 ? sqrt(acc[r]) : acc[r];
        sl[r] = l;
        lam[r] = l;
        if (inner) inner[r] /= l;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < R * R; e += blockDim.x) {
        const int a = e / R, b = e - a * R;
        G[e] = G[e] / sl[a] / sl[b];
    }
}

static __global__ void k_lambda_finish(const double* acc, int R, int nk, double* lam, double* G, double* inner)
{
    lambda_finish_body(acc, R, nk, lam, G, inner);
}

// U[:, c] /= lambda[c] (FT storage, FP64 division as in the reference's
// normalisation); VEC consecutive elements per thread (R % VEC == 0; 16-byte
// vectors when VEC * sizeof(FT) == 16), the column index carried along the
// grid-stride loop.
template <typename FT, int VEC>
__device__ __forceinline__ void div_cols_body(FT* __restrict__ U, u64 I, int R, const double* __restrict__ lam,
                                              u64 bx, u64 nbx)
{
    extern __shared__ double dl_[];
    for (int r = threadIdx.x; r < R; r += blockDim.x) dl_[r] = lam[r];
    __syncthreads();
    const u64 nv = I * (u64)R / VEC;
    const u64 stride = nbx * blockDim.x;
    u64 e = bx * blockDim.x + threadIdx.x;
    if (e >= nv) return;
    int col = (int)((e * VEC) % (u64)R);
    const int cstep = (int)((stride * VEC) % (u64)R);
    for (; e < nv; e += stride) {
        union {
            uint4 q;
            FT f[VEC];
        } v;
        if constexpr (VEC * sizeof(FT) == 16) v.q = reinterpret_cast<const uint4*>(U)[e];
        else
#pragma unroll
            for (int k = 0; k < VEC; ++k) v.f[k] = U[e * VEC + k];
#pragma unroll
        for (int k = 0; k < VEC; ++k) v.f[k] = (FT)((double)v.f[k] / dl_[col + k]);  // R % VEC == 0
        if constexpr (VEC * sizeof(FT) == 16) reinterpret_cast<uint4*>(U)[e] = v.q;
        else
#pragma unroll
            for (int k = 0; k < VEC; ++k) U[e * VEC + k] = v.f[k];
        col += cstep;
        col = col >= R ? col - R : col;
    }
}

template <typename FT, int VEC>
__global__ void __launch_bounds__(DN_THREADS) k_div_cols(FT* __restrict__ U, u64 I, int R,
                                                         const double* __restrict__ lam)
{
    div_cols_body<FT, VEC>(U, I, R, lam, blockIdx.x, gridDim.x);
}

// Rank classes of the row kernels: (lanes per row, columns per lane) and
// Gram tiles per thread.
inline int rank_class(int R) { return R <= 8 ? 0 : R <= 16 ? 1 : R <= 32 ? 2 : R <= 64 ? 3 : 4; }
constexpr int NRANK_CLASSES = 5;

static __global__ void k_lambda(const double* acc, int R, int nk, double* lam)
{
    for (int r = threadIdx.x; r < R; r += blockDim.x) lam[r] = nk == NORM_2 ? sqrt(acc[r]) : acc[r];
}

// cpd_fit_alto (cpd.hpp:189-271): normU from lambda and the Grams (lower
// triangle, off-diagonal doubled), inner from the per-column partials.
__device__ __forceinline__ void fit_body(const double* __restrict__ G, int nmode, int R,
                                         const double* __restrict__ lam, const double* __restrict__ inner,
                                         double normAT, double* __restrict__ fit)
{
    __shared__ double red[DN_THREADS];
    double s = 0.0;
    for (int e = threadIdx.x; e < R * R; e += DN_THREADS) {
        const int a = e / R, b = e - a * R;
        if (b > a) continue;
        double t = lam[a] * lam[b];
        for (int m = 0; m < nmode; ++m) t *= G[(size_t)m * R * R + e];
        s += a == b ? t : 2.0 * t;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = DN_THREADS / 2; o; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double normU = fabs(red[0]);
        double ip = 0.0;
        for (int r = 0; r < R; ++r) ip += inner[r] * lam[r];
        double res = normAT + normU - 2.0 * ip;
        if (res > 0.0) res = sqrt(res);
        fit[0] = 1.0 - res / sqrt(normAT);
    }
}

static __global__ void k_fit(const double* __restrict__ G, int nmode, int R, const double* __restrict__ lam,
                      const double* __restrict__ inner, double normAT, double* __restrict__ fit)
{
    fit_body(G, nmode, R, lam, inner, normAT, fit);
}

template <typename FT>
static __global__ void k_colsum_abs(const FT* __restrict__ U, u64 I, int R, double* __restrict__ acc)
{
    extern __shared__ double cs_[];
    for (int r = threadIdx.x; r < R; r += blockDim.x) cs_[r] = 0.0;
    __syncthreads();
    const u64 n = I * (u64)R;
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (u64)gridDim.x * blockDim.x)
        atomicAdd(&cs_[e % R], fabs((double)U[e]));
    __syncthreads();
    for (int r = threadIdx.x; r < R; r += blockDim.x) atomicAdd(&acc[r], cs_[r]);
}

template <typename FT>
static __global__ void k_scale_cols(FT* __restrict__ U, u64 I, int R, const double* __restrict__ d, int divide)
{
    const u64 n = I * (u64)R;
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (u64)gridDim.x * blockDim.x) {
        const double v = (double)U[e];
        U[e] = (FT)(divide ? v / d[e % R] : v * d[e % R]);
    }
}

template <typename FT>
static __global__ void k_sum_all(const FT* __restrict__ U, u64 n, double* __restrict__ acc)
{
    double s = 0.0;
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (u64)gridDim.x * blockDim.x)
        s += (double)U[e];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(acc, s);
}

static __global__ void k_vec(double* lam, const double* d, int R, double x, int op)
{
    for (int r = threadIdx.x; r < R; r += blockDim.x) lam[r] = op == 0 ? lam[r] * d[r] : x;
}

template <typename A, typename B>
static __global__ void k_conv(A* dst, const B* src, int R)
{
    for (int r = threadIdx.x; r < R; r += blockDim.x) dst[r] = (A)src[r];
}

template <typename VT>
static __global__ void k_sumsq(const VT* __restrict__ v, u64 n, double* __restrict__ acc)
{
    double s = 0.0;
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (u64)gridDim.x * blockDim.x) {
        const double x = (double)v[e];
        s += x * x;
    }
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(acc, s);
}

}  // namespace altob
