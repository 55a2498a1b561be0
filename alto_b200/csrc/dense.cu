// dense.cu -- dense kernels for the CP-ALS / CP-APR updates (see dense.cuh).
// Every reduction accumulates in FP64; factor storage is FT (float/double).
#include <algorithm>
#include <atomic>
#include <cmath>

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
// across thread groups when there are fewer tiles than threads.

constexpr int GR_TB = 4;
constexpr int GR_ROWS = 64;
constexpr int GR_MAXT = 3;  // tiles per thread (R <= 128)

template <typename FT>
__global__ void __launch_bounds__(DN_THREADS) k_gram(const FT* __restrict__ U, u64 I, int R, double* __restrict__ G,
                                                     const double* __restrict__ div, FT* __restrict__ Uout,
                                                     const FT* __restrict__ M, double* __restrict__ inner)
{
    extern __shared__ double gsm[];
    double* s = gsm;                     // GR_ROWS x R
    double* si = gsm + GR_ROWS * R;      // R (inner partial)
    const int tid = threadIdx.x;
    const int T = (R + GR_TB - 1) / GR_TB;
    const int NT = T * (T + 1) / 2;
    const int groups = NT >= DN_THREADS ? 1 : DN_THREADS / NT;
    const int grp = NT >= DN_THREADS ? 0 : tid / NT;
    const bool active = NT >= DN_THREADS || tid < groups * NT;
    int ta[GR_MAXT], tb[GR_MAXT];
    double acc[GR_MAXT][GR_TB * GR_TB];
#pragma unroll
    for (int k = 0; k < GR_MAXT; ++k) {
        int t = NT >= DN_THREADS ? tid + k * DN_THREADS : tid % NT;
        if (NT < DN_THREADS && k > 0) t = NT;  // only one tile
        int a = 0;
        while ((a + 1) * (a + 2) / 2 <= t) ++a;
        ta[k] = t < NT ? a : -1;
        tb[k] = t < NT ? t - a * (a + 1) / 2 : -1;
#pragma unroll
        for (int e = 0; e < GR_TB * GR_TB; ++e) acc[k][e] = 0.0;
    }
    if (M)
        for (int r = tid; r < R; r += DN_THREADS) si[r] = 0.0;
    const u64 nchunks = (I + GR_ROWS - 1) / GR_ROWS;
    for (u64 ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
        const u64 r0 = ch * GR_ROWS;
        const int nrows = (int)std::min<u64>(GR_ROWS, I - r0);
        __syncthreads();
        for (int e = tid; e < GR_ROWS * R; e += DN_THREADS) {
            const int row = e / R, col = e - row * R;
            double x = 0.0;
            if (row < nrows) {
                const u64 gi = (r0 + row) * (u64)R + col;
                x = (double)U[gi];
                if (div) {
                    x = x / div[col];
                    if (Uout) Uout[gi] = (FT)x;
                    x = (double)(FT)x;
                }
                if (M) atomicAdd(&si[col], x * (double)M[gi]);
            }
            s[e] = x;
        }
        __syncthreads();
        if (!active) continue;
#pragma unroll
        for (int k = 0; k < GR_MAXT; ++k) {
            if (ta[k] < 0) continue;
            const int a0 = ta[k] * GR_TB, b0 = tb[k] * GR_TB;
            for (int row = grp; row < nrows; row += groups) {
                const double* sr = s + row * R;
                double xa[GR_TB], xb[GR_TB];
#pragma unroll
                for (int q = 0; q < GR_TB; ++q) {
                    xa[q] = a0 + q < R ? sr[a0 + q] : 0.0;
                    xb[q] = b0 + q < R ? sr[b0 + q] : 0.0;
                }
#pragma unroll
                for (int p = 0; p < GR_TB; ++p)
#pragma unroll
                    for (int q = 0; q < GR_TB; ++q) acc[k][p * GR_TB + q] += xa[p] * xb[q];
            }
        }
    }
    if (active) {
#pragma unroll
        for (int k = 0; k < GR_MAXT; ++k) {
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
        __syncthreads();
        for (int r = tid; r < R; r += DN_THREADS) atomicAdd(&inner[r], si[r]);
    }
}

template <typename FT>
altob_status gram(const FT* U, u64 I, int R, double* G, const double* div, FT* Uout, const FT* M, double* inner,
                  cudaStream_t st)
{
    if (R > 128) return fail(ALTOB_ERR_UNSUPPORTED, "rank above 128 in the Gram kernel");
    ALTOB_CUDA(cudaMemsetAsync(G, 0, (size_t)R * R * sizeof(double), st));
    if (M) ALTOB_CUDA(cudaMemsetAsync(inner, 0, (size_t)R * sizeof(double), st));
    if (I == 0) return ALTOB_OK;
    size_t smem = (size_t)(GR_ROWS * R + R) * sizeof(double);
    k_gram<FT><<<dn_grid(I, 4 * GR_ROWS), DN_THREADS, smem, st>>>(U, I, R, G, div, Uout, M, inner);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

// ----------------------------------------------------------- R x R solve
// V = Hadamard product of the Grams of all modes but `target` (only the
// lower triangle is meaningful, as in the reference's POTRF('L')).  If V is
// positive definite: Cholesky V = L L^T and W = V^{-1} = L^{-T} L^{-1}.
// Otherwise W = V^+ from a cyclic Jacobi eigendecomposition (eigenvalues
// below R * eps * max|lambda| dropped).  info[0] += 1 on every fallback.

__global__ void __launch_bounds__(DN_THREADS) k_solve_setup(const double* __restrict__ G, int nmode, int target,
                                                            int R, double* __restrict__ W, int* __restrict__ info)
{
    extern __shared__ double ssm[];
    double* A = ssm;          // R x R
    double* B = ssm + R * R;  // R x R
    __shared__ int ok;
    __shared__ double cs[2];
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
    // ---- pseudo-inverse fallback: A = V (symmetric), B = eigenvectors
    for (int e = tid; e < R * R; e += DN_THREADS) {
        const int a = e / R, b = e - a * R;
        A[e] = a >= b ? B[e] : B[b * R + a];
    }
    __syncthreads();
    for (int e = tid; e < R * R; e += DN_THREADS) B[e] = (e / R == e % R) ? 1.0 : 0.0;
    __syncthreads();
    for (int sweep = 0; sweep < 60; ++sweep) {
        // convergence test
        if (tid == 0) {
            double off = 0.0, tot = 0.0;
            for (int e = 0; e < R * R; ++e) {
                tot += A[e] * A[e];
                if (e / R != e % R) off += A[e] * A[e];
            }
            ok = off <= 1e-30 * tot;
        }
        __syncthreads();
        if (ok) break;
        for (int p = 0; p < R; ++p)
            for (int q = p + 1; q < R; ++q) {
                if (tid == 0) {
                    const double apq = A[p * R + q];
                    double c = 1.0, s = 0.0;
                    if (apq != 0.0) {
                        const double th = (A[q * R + q] - A[p * R + p]) / (2.0 * apq);
                        const double t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
                        c = 1.0 / sqrt(t * t + 1.0);
                        s = t * c;
                    }
                    cs[0] = c;
                    cs[1] = s;
                }
                __syncthreads();
                const double c = cs[0], s = cs[1];
                if (s != 0.0) {
                    for (int k = tid; k < R; k += DN_THREADS) {
                        const double akp = A[k * R + p], akq = A[k * R + q];
                        A[k * R + p] = c * akp - s * akq;
                        A[k * R + q] = s * akp + c * akq;
                    }
                    __syncthreads();
                    for (int k = tid; k < R; k += DN_THREADS) {
                        const double apk = A[p * R + k], aqk = A[q * R + k];
                        A[p * R + k] = c * apk - s * aqk;
                        A[q * R + k] = s * apk + c * aqk;
                        const double vkp = B[k * R + p], vkq = B[k * R + q];
                        B[k * R + p] = c * vkp - s * vkq;
                        B[k * R + q] = s * vkp + c * vkq;
                    }
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

altob_status solve_setup(const double* G, int nmode, int target, int R, double* W, int* info, cudaStream_t st)
{
    if (R > SOLVE_MAX_RANK) return fail(ALTOB_ERR_UNSUPPORTED, "rank above 112 in the R x R solve");
    size_t smem = (size_t)2 * R * R * sizeof(double);
    static std::atomic<size_t> configured{0};
    if (smem > 48 * 1024 && smem > configured.load()) {
        ALTOB_CUDA(cudaFuncSetAttribute(k_solve_setup, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        size_t cur = configured.load();
        while (cur < smem && !configured.compare_exchange_weak(cur, smem)) {
        }
    }
    k_solve_setup<<<1, DN_THREADS, smem, st>>>(G, nmode, target, R, W, info);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

// ------------------------------------------------------------ row apply
// U[i,:] <- U[i,:] W (FP64), four rows per warp step; column norms of the
// result are accumulated on the fly (2-norm: sum of squares; max-norm:
// running max floored at 1, src/kruskal_model.cpp:264-305).

constexpr int AP_RW = 4;
constexpr int AP_CJ = 4;  // R <= 128

template <typename FT>
__global__ void __launch_bounds__(DN_THREADS) k_apply(FT* __restrict__ U, u64 I, int R, const double* __restrict__ Wg,
                                                      int nk, double* __restrict__ colacc)
{
    extern __shared__ double asm_[];
    double* W = asm_;          // R x R
    double* cr = asm_ + R * R;  // R column partials
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int e = tid; e < R * R; e += DN_THREADS) W[e] = Wg[e];
    for (int r = tid; r < R; r += DN_THREADS) cr[r] = nk == NORM_MAX ? 1.0 : 0.0;
    __syncthreads();
    const int CJ = (R + 31) / 32;
    double part[AP_CJ];
#pragma unroll
    for (int j = 0; j < AP_CJ; ++j) part[j] = nk == NORM_MAX ? 1.0 : 0.0;
    const u64 step = (u64)gridDim.x * (DN_THREADS / 32) * AP_RW;
    for (u64 i0 = ((u64)blockIdx.x * (DN_THREADS / 32) + warp) * AP_RW; i0 < I; i0 += step) {
        double u[AP_RW][AP_CJ], x[AP_RW][AP_CJ];
#pragma unroll
        for (int rw = 0; rw < AP_RW; ++rw)
#pragma unroll
            for (int j = 0; j < AP_CJ; ++j) {
                const int c = lane + 32 * j;
                const u64 i = i0 + rw;
                u[rw][j] = (j < CJ && c < R && i < I) ? (double)U[i * R + c] : 0.0;
                x[rw][j] = 0.0;
            }
        for (int a = 0; a < R; ++a) {
            const int ja = a >> 5, la = a & 31;
            double ua[AP_RW];
#pragma unroll
            for (int rw = 0; rw < AP_RW; ++rw) {
                double v = 0.0;
#pragma unroll
                for (int j = 0; j < AP_CJ; ++j)
                    if (j == ja) v = u[rw][j];
                ua[rw] = __shfl_sync(0xffffffffu, v, la);
            }
#pragma unroll
            for (int j = 0; j < AP_CJ; ++j) {
                const int b = lane + 32 * j;
                if (j < CJ && b < R) {
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
            for (int j = 0; j < AP_CJ; ++j) {
                const int b = lane + 32 * j;
                if (j < CJ && b < R) {
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
        for (int j = 0; j < AP_CJ; ++j) {
            const int b = lane + 32 * j;
            if (j < CJ && b < R) {
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

template <typename FT>
altob_status apply_w(FT* U, u64 I, int R, const double* W, NormKind nk, double* colacc, cudaStream_t st)
{
    if (R > 128) return fail(ALTOB_ERR_UNSUPPORTED, "rank above 128 in the row apply");
    if (nk != NORM_NONE) {
        if (nk == NORM_2) ALTOB_CUDA(cudaMemsetAsync(colacc, 0, (size_t)R * sizeof(double), st));
        else ALTOB_TRY(vec_fill(colacc, R, 1.0, st));
    }
    if (I == 0) return ALTOB_OK;
    size_t smem = (size_t)(R * R + R) * sizeof(double);
    static std::atomic<size_t> cfg{0};  // one per FT instantiation
    if (smem > 48 * 1024 && smem > cfg.load()) {
        ALTOB_CUDA(cudaFuncSetAttribute(k_apply<FT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        size_t cur = cfg.load();
        while (cur < smem && !cfg.compare_exchange_weak(cur, smem)) {
        }
    }
    k_apply<FT><<<dn_grid(I, (DN_THREADS / 32) * AP_RW * 8), DN_THREADS, smem, st>>>(U, I, R, W, (int)nk, colacc);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

// ------------------------------------------------------------- small ops

__global__ void k_lambda(const double* acc, int R, int nk, double* lam)
{
    for (int r = threadIdx.x; r < R; r += blockDim.x) lam[r] = nk == NORM_2 ? sqrt(acc[r]) : acc[r];
}

altob_status lambda_from(const double* colacc, int R, NormKind nk, double* lam, cudaStream_t st)
{
    k_lambda<<<1, 128, 0, st>>>(colacc, R, (int)nk, lam);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

// cpd_fit_alto (cpd.hpp:189-271): normU from lambda and the Grams (lower
// triangle, off-diagonal doubled), inner from the per-column partials.
__global__ void k_fit(const double* __restrict__ G, int nmode, int R, const double* __restrict__ lam,
                      const double* __restrict__ inner, double normAT, double* __restrict__ fit)
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

altob_status fit_from(const double* G, int nmode, int R, const double* lam, const double* inner, double normAT,
                      double* fit, cudaStream_t st)
{
    k_fit<<<1, DN_THREADS, 0, st>>>(G, nmode, R, lam, inner, normAT, fit);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

template <typename FT>
__global__ void k_colsum_abs(const FT* __restrict__ U, u64 I, int R, double* __restrict__ acc)
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
altob_status colsum_abs(const FT* U, u64 I, int R, double* acc, cudaStream_t st)
{
    ALTOB_CUDA(cudaMemsetAsync(acc, 0, (size_t)R * sizeof(double), st));
    if (I == 0) return ALTOB_OK;
    k_colsum_abs<FT><<<dn_grid(I * R, DN_THREADS * 16), DN_THREADS, R * sizeof(double), st>>>(U, I, R, acc);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

template <typename FT>
__global__ void k_scale_cols(FT* __restrict__ U, u64 I, int R, const double* __restrict__ d, int divide)
{
    const u64 n = I * (u64)R;
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (u64)gridDim.x * blockDim.x) {
        const double v = (double)U[e];
        U[e] = (FT)(divide ? v / d[e % R] : v * d[e % R]);
    }
}

template <typename FT>
altob_status div_cols(FT* U, u64 I, int R, const double* d, cudaStream_t st)
{
    if (I == 0) return ALTOB_OK;
    k_scale_cols<FT><<<dn_grid(I * R, DN_THREADS * 8), DN_THREADS, 0, st>>>(U, I, R, d, 1);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

template <typename FT>
altob_status mul_cols(FT* U, u64 I, int R, const double* d, cudaStream_t st)
{
    if (I == 0) return ALTOB_OK;
    k_scale_cols<FT><<<dn_grid(I * R, DN_THREADS * 8), DN_THREADS, 0, st>>>(U, I, R, d, 0);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

template <typename FT>
__global__ void k_sum_all(const FT* __restrict__ U, u64 n, double* __restrict__ acc)
{
    double s = 0.0;
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (u64)gridDim.x * blockDim.x)
        s += (double)U[e];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(acc, s);
}

template <typename FT>
altob_status sum_all(const FT* U, u64 n, double* acc, cudaStream_t st)
{
    ALTOB_CUDA(cudaMemsetAsync(acc, 0, sizeof(double), st));
    if (n == 0) return ALTOB_OK;
    k_sum_all<FT><<<dn_grid(n, DN_THREADS * 16), DN_THREADS, 0, st>>>(U, n, acc);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

__global__ void k_vec(double* lam, const double* d, int R, double x, int op)
{
    for (int r = threadIdx.x; r < R; r += blockDim.x) lam[r] = op == 0 ? lam[r] * d[r] : x;
}

altob_status vec_mul(double* lam, const double* d, int R, cudaStream_t st)
{
    k_vec<<<1, 128, 0, st>>>(lam, d, R, 0.0, 0);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

altob_status vec_fill(double* v, int R, double x, cudaStream_t st)
{
    k_vec<<<1, 128, 0, st>>>(v, nullptr, R, x, 1);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

template <typename A, typename B>
__global__ void k_conv(A* dst, const B* src, int R)
{
    for (int r = threadIdx.x; r < R; r += blockDim.x) dst[r] = (A)src[r];
}

template <typename FT>
altob_status vec_to(FT* dst, const double* src, int R, cudaStream_t st)
{
    k_conv<FT, double><<<1, 128, 0, st>>>(dst, src, R);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

template <typename FT>
altob_status vec_from(double* dst, const FT* src, int R, cudaStream_t st)
{
    k_conv<double, FT><<<1, 128, 0, st>>>(dst, src, R);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

template <typename VT>
__global__ void k_sumsq(const VT* __restrict__ v, u64 n, double* __restrict__ acc)
{
    double s = 0.0;
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (u64)gridDim.x * blockDim.x) {
        const double x = (double)v[e];
        s += x * x;
    }
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(acc, s);
}

altob_status value_sumsq(const altob_tensor* t, double* acc, cudaStream_t st)
{
    ALTOB_CUDA(cudaMemsetAsync(acc, 0, sizeof(double), st));
    if (t->nnz == 0) return ALTOB_OK;
    int g = dn_grid(t->nnz, DN_THREADS * 16);
    if (t->vdt == ALTOB_F64) k_sumsq<double><<<g, DN_THREADS, 0, st>>>((const double*)t->d_vals, t->nnz, acc);
    else if (t->vdt == ALTOB_F32) k_sumsq<float><<<g, DN_THREADS, 0, st>>>((const float*)t->d_vals, t->nnz, acc);
    else k_sumsq<u32><<<g, DN_THREADS, 0, st>>>((const u32*)t->d_vals, t->nnz, acc);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

#define ALTOB_DENSE_INST(FT)                                                                                 \
    template altob_status gram<FT>(const FT*, u64, int, double*, const double*, FT*, const FT*, double*,     \
                                   cudaStream_t);                                                            \
    template altob_status apply_w<FT>(FT*, u64, int, const double*, NormKind, double*, cudaStream_t);        \
    template altob_status colsum_abs<FT>(const FT*, u64, int, double*, cudaStream_t);                        \
    template altob_status div_cols<FT>(FT*, u64, int, const double*, cudaStream_t);                          \
    template altob_status mul_cols<FT>(FT*, u64, int, const double*, cudaStream_t);                          \
    template altob_status sum_all<FT>(const FT*, u64, double*, cudaStream_t);                                \
    template altob_status vec_to<FT>(FT*, const double*, int, cudaStream_t);                                 \
    template altob_status vec_from<FT>(double*, const FT*, int, cudaStream_t);

ALTOB_DENSE_INST(float)
ALTOB_DENSE_INST(double)

}  // namespace altob
