// mttkrp.cu -- MTTKRP and Phi entry points.
//
// altob_mttkrp replaces mttkrp_alto_par (IntelLabs/ALTO include/alto.hpp:
// 617-623) including its dispatch on fiber reuse (alto.hpp:554-563) and its
// += semantics; altob_phi replaces CalculatePhi_alto_par (include/apr.hpp:
// 297-303).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <type_traits>

#include "mttkrp_launch.cuh"
#include "mttkrp_plan.h"
#include "phi_rows_tma.cuh"

namespace altob {

static int next_pow2(int x)
{
    int p = 1;
    while (p < x) p <<= 1;
    return p;
}

static int floor_pow2(long long x)
{
    int p = 1;
    while ((long long)p * 2 <= x) p <<= 1;
    return p;
}

bool ptr_aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

altob_status plan_tiled(const altob_tensor* t, u64 R, size_t fsz, bool aligned, bool cache, TiledPlan* pl)
{
    const int V = (int)(16 / fsz);
    if (R > 128) return fail(ALTOB_ERR_UNSUPPORTED, "rank above 128 in the MTTKRP kernel");
    pl->vec = (aligned && R % V == 0) ? V : 1;
    if (pl->vec == 1) {
        pl->lpn = 32;
        pl->ch = 4;
    } else {
        const int lanes = (int)((R + pl->vec - 1) / pl->vec);
        pl->lpn = std::max(2, std::min(32, next_pow2(lanes)));
        pl->ch = (int)((R + (u64)pl->lpn * pl->vec - 1) / ((u64)pl->lpn * pl->vec));
    }
    pl->grouped = env_int("ALTOB_KERNEL", 4) == 4;
    if (pl->grouped && pl->vec > 1) {
        // fewer lanes per nonzero, two chunks each: amortizes per-nonzero work
        const int want = env_int("ALTOB_LPN", 0);
        if (want == 4 || want == 8 || want == 16) {
            const u64 per = (u64)want * pl->vec;
            const u64 ch = (R + per - 1) / per;
            if (ch <= 2) {
                pl->lpn = want;
                pl->ch = (int)ch;
            }
        }
    }
    if (pl->grouped) {
        // k_grouped: fixed tile, slot table only (no accumulator rows)
        pl->tile = GT_TILE;
        const int slots = env_int("ALTOB_GROUP_SLOTS", 2048);
        pl->hslots = cache ? std::max(32, std::min(floor_pow2(slots), 8192)) : 0;
        const int mm = t->nmode >= 3 ? t->nmode : ALTOB_MAX_MODES;
        pl->hot = env_int("ALTOB_HOT_ROWS", 1) ? grouped_hot_slots((int)R, fsz) : 0;
        pl->smem = grouped_smem(pl->hslots, mm, fsz, pl->hot, (int)R);
        return ALTOB_OK;
    }
    pl->hot = 0;
    pl->tile = env_int("ALTOB_TILE", 1024);
    pl->tile = std::max(256, (pl->tile / 256) * 256);
    int cache_bytes = env_int("ALTOB_CACHE_BYTES", 32 * 1024);
    long long rows = (long long)cache_bytes / (long long)(R * fsz);
    pl->hslots = (cache && rows >= 16) ? std::min(floor_pow2(rows), 4096) : 0;
    pl->smem = tiled_smem(t->nmode, pl->tile, pl->hslots, (int)R, fsz);
    return ALTOB_OK;
}

// Per-CTA hot-row accumulator regions for a launch of `grid` CTAs (none when
// the kernel has no hot-row slots).
template <typename FT>
static altob_status set_hot_acc(altob_tensor* t, TiledArgs<FT>& a, unsigned grid, cudaStream_t st)
{
    (void)st;
    a.hot_acc = nullptr;
    if (!a.hot) return ALTOB_OK;
    void* p = nullptr;
    ALTOB_TRY(tensor_hotbuf(t, (size_t)grid * a.hot * a.R * sizeof(FT), &p));
    a.hot_acc = (FT*)p;
    return ALTOB_OK;
}

// Tile plan of `mode` (k_tile_plan), built on the first call that needs it.
// Returns false (and leaves no plan) when the 2 bytes per nonzero cannot be
// allocated; the caller then runs the grouped kernel.
static bool ensure_plan(altob_tensor* t, int mode, cudaStream_t st)
{
    if (t->d_plan[mode]) return true;
    void* p = nullptr;
    if (dmalloc(&p, (size_t)t->nnz * sizeof(uint16_t)) != ALTOB_OK) return false;
    const u64 ntiles = (t->nnz + PT_TILE - 1) / PT_TILE;
    k_tile_plan<PT_TILE><<<(unsigned)ntiles, PT_TILE / 2, 0, st>>>(key_src(t), t->fld, t->nnz, mode, (u16*)p);
    if (cudaGetLastError() != cudaSuccess) {
        dfree(p);
        return false;
    }
    t->d_plan[mode] = (uint16_t*)p;
    return true;
}

const uint16_t* tensor_plan(altob_tensor* t, int mode, cudaStream_t st)
{
    if (!env_int("ALTOB_PLAN", 1) || t->nnz == 0 || t->nnz >= (1ull << 32)) return nullptr;
    return ensure_plan(t, mode, st) ? t->d_plan[mode] : nullptr;
}

// ---------------------------------------------- TMA-staged planned MTTKRP

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled()
{
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
        cudaGetLastError();
    });
    return fn;
}

// Row-gather map of an I x R FP32 factor matrix (box: one row of R values).
static bool row_map(CUtensorMap* m, const float* U, u64 rows, int R)
{
    EncodeTiledFn fn = encode_tiled();
    if (!fn) return false;
    const cuuint64_t dim[2] = {(cuuint64_t)R, (cuuint64_t)rows};
    const cuuint64_t stride[1] = {(cuuint64_t)R * 4};
    const cuuint32_t box[2] = {(cuuint32_t)R, 1};
    const cuuint32_t estr[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void*)U, dim, stride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int LPN, int S>
static altob_status launch_tma_one(altob_tensor* t, TmaArgs& ta, const CUtensorMap& m0, const CUtensorMap& m1,
                                   cudaStream_t st)
{
    using Sh = TmaShape<LPN, S>;
    static std::atomic<size_t> configured{0};
    const size_t smem = Sh::smem(ta.a.hot);
    if (smem > configured.load()) {
        ALTOB_CUDA(cudaFuncSetAttribute(k_planned_tma<LPN, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        configured.store(smem);
    }
    int bps = 0;
    ALTOB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_planned_tma<LPN, S>, TMA_THREADS, smem));
    if (bps < 1) return fail(ALTOB_ERR_UNSUPPORTED, "TMA MTTKRP kernel does not fit on an SM");
    const unsigned grid = (unsigned)std::max<u64>(1, std::min<u64>(ta.a.ntiles, (u64)bps * num_sms()));
    ALTOB_TRY(set_hot_acc(t, ta.a, grid, st));
    k_planned_tma<LPN, S><<<grid, TMA_THREADS, smem, st>>>(ta, m0, m1);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

// FP32, order 3, R = 4 * LPN with LPN in {4, 8, 16}, a tile plan, 16-byte
// aligned factors: the TMA-staged kernel (ALTOB_TMA=1 selects it; 2 or 4
// stages with ALTOB_TMA_STAGES).  Returns false when the case does not
// qualify (the caller then runs the planned kernel).
static bool tma_eligible(const altob_tensor* t, u64 R, bool planned)
{
    return planned && t->nmode == 3 && (R == 16 || R == 32 || R == 64) && env_int("ALTOB_TMA", 0) != 0 &&
           encode_tiled() != nullptr;
}

static altob_status run_tma(altob_tensor* t, TiledArgs<float>& a, u64 R, cudaStream_t st)
{
    if (!t->d_tma_err) {
        ALTOB_TRY(dmalloc_t(&t->d_tma_err, 4));
        ALTOB_CUDA(cudaMemsetAsync(t->d_tma_err, 0, 4, st));
        ALTOB_CUDA(cudaMallocHost((void**)&t->h_tma_err, 4));
        *t->h_tma_err = 0;
    }
    if (*t->h_tma_err) return fail(ALTOB_ERR_CUDA, "an earlier TMA-staged MTTKRP ran out of a wait limit");
    CUtensorMap m[2];
    int k = 0;
    for (int m_ = 0; m_ < 3; ++m_) {
        if (m_ == a.target) continue;
        if (!row_map(&m[k], a.U[m_], t->dims[m_], (int)R)) return fail(ALTOB_ERR_CUDA, "cuTensorMapEncodeTiled failed");
        ++k;
    }
    TmaArgs ta;
    ta.a = a;
    ta.err = t->d_tma_err;
    const int stages = env_int("ALTOB_TMA_STAGES", 4) == 2 ? 2 : 4;
    altob_status s;
    if (R == 16) s = stages == 2 ? launch_tma_one<4, 2>(t, ta, m[0], m[1], st) : launch_tma_one<4, 4>(t, ta, m[0], m[1], st);
    else if (R == 32) s = stages == 2 ? launch_tma_one<8, 2>(t, ta, m[0], m[1], st) : launch_tma_one<8, 4>(t, ta, m[0], m[1], st);
    else s = stages == 2 ? launch_tma_one<16, 2>(t, ta, m[0], m[1], st) : launch_tma_one<16, 4>(t, ta, m[0], m[1], st);
    ALTOB_TRY(s);
    ALTOB_CUDA(cudaMemcpyAsync(t->h_tma_err, t->d_tma_err, 4, cudaMemcpyDeviceToHost, st));
    return ALTOB_OK;
}

template <typename FT, typename VT>
static altob_status run_tiled_vt(altob_tensor* t, int mode, void* const* dU, void* dout, u64 R, bool phi,
                                 double eps, const u32* perm, bool cache, cudaStream_t st)
{
    bool aligned = ptr_aligned16(dout);
    for (int m = 0; m < t->nmode; ++m) aligned = aligned && ptr_aligned16(dU[m]);
    TiledPlan pl;
    ALTOB_TRY(plan_tiled(t, R, sizeof(FT), aligned, cache, &pl));
    // MTTKRP of a static order 3-5 in ALTO order with one vector chunk per
    // lane: the planned kernel (ALTOB_PLAN=0 keeps the grouped kernel)
    const bool planned = pl.grouped && !phi && !perm && cache && t->nmode >= 3 && t->nmode <= 5 && pl.vec > 1 &&
                         pl.ch == 1 && t->nnz < (1ull << 32) && env_int("ALTOB_PLAN", 1) && ensure_plan(t, mode, st);
    TiledArgs<FT> a;
    memset(&a, 0, sizeof(a));
    a.key = key_src(t);
    a.vals = t->d_vals;
    a.perm = perm;
    a.nnz = t->nnz;
    a.ntiles = (t->nnz + pl.tile - 1) / pl.tile;
    a.nmode = t->nmode;
    a.target = mode;
    a.R = (int)R;
    a.tile = pl.tile;
    a.hslots = pl.hslots;
    a.eps = (FT)eps;
    for (int m = 0; m < t->nmode; ++m) a.U[m] = (const FT*)dU[m];
    a.out = (FT*)dout;
    a.fld = t->fld;
    a.hot = pl.grouped ? pl.hot : 0;
    TiledCfg c;
    c.lpn = pl.lpn;
    c.vec = pl.vec;
    c.ch = pl.ch;
    c.grouped = pl.grouped;
    c.phi = phi ? 1 : 0;
    c.smem = pl.smem;
    c.grid = dim3(0);
    int bps = 0;
    if (planned) {
        a.plan = t->d_plan[mode];
        // runs of 16 or more nonzeros through the hot-row table: fewer table
        // lookups than at 8 (2.19 -> 2.16 ms per mode on the 100.85M-nonzero
        // Zipf tensor) at the same FP32 error (1.0-1.7e-6 against FP64); below
        // 8 the lookups cost more than the atomics they save (2: 2.61 ms)
        a.hot_minrun = 16;
        a.tile = PT_TILE;
        a.ntiles = (t->nnz + PT_TILE - 1) / PT_TILE;
        a.hslots = 0;
        if constexpr (sizeof(FT) == 4 && std::is_same<VT, float>::value) {
            if (tma_eligible(t, R, true)) return run_tma(t, a, R, st);
        }
        const int nbuf = t->nmode == 3 ? planned_nbuf<FT, 3>() : 2;
        c.smem = planned_smem(t->nmode, sizeof(FT), a.hot, c.lpn, PT_TILE, nbuf);
        ALTOB_TRY((launch_planned<FT, VT>(a, c, st, &bps)));
        if (bps < 1) return fail(ALTOB_ERR_UNSUPPORTED, "planned MTTKRP kernel does not fit on an SM");
        c.grid = dim3((unsigned)std::max<u64>(1, std::min<u64>(a.ntiles, (u64)bps * num_sms())));
        ALTOB_TRY(set_hot_acc(t, a, c.grid.x, st));
        return launch_planned<FT, VT>(a, c, st, nullptr);
    }
    ALTOB_TRY((launch_tiled<FT, VT>(a, c, st, &bps)));
    if (bps < 1) return fail(ALTOB_ERR_UNSUPPORTED, "MTTKRP kernel does not fit on an SM");
    u64 cap = (u64)bps * num_sms();
    c.grid = dim3((unsigned)std::max<u64>(1, std::min<u64>(a.ntiles, cap)));
    ALTOB_TRY(set_hot_acc(t, a, c.grid.x, st));
    return launch_tiled<FT, VT>(a, c, st, nullptr);
}

template <typename FT>
static altob_status run_tiled(altob_tensor* t, int mode, void* const* dU, void* dout, u64 R, bool phi, double eps,
                              const u32* perm, bool cache, cudaStream_t st)
{
    const bool f64 = sizeof(FT) == 8;
    if (t->vdt == ALTOB_U32) return run_tiled_vt<FT, u32>(t, mode, dU, dout, R, phi, eps, perm, cache, st);
    if ((t->vdt == ALTOB_F64) == f64) return run_tiled_vt<FT, FT>(t, mode, dU, dout, R, phi, eps, perm, cache, st);
    return fail(ALTOB_ERR_UNSUPPORTED, "stored value dtype does not match the compute dtype");
}

template <typename FT>
static altob_status run_atomic_cr(altob_tensor* t, int mode, void* const* dU, u64 R, cudaStream_t st)
{
    u128 crm = t->cr_masks[mode];
    if (!crm) return fail(ALTOB_ERR_ARG, "ATOMIC_CR needs a CR bit for the target mode");
    CrArgsK<FT> a;
    memset(&a, 0, sizeof(a));
    a.key = key_src(t);
    a.vals = t->d_vals;
    a.nnz = t->nnz;
    a.nprtn = t->nprtn;
    a.per = (t->nnz + t->nprtn - 1) / t->nprtn;
    a.nmode = t->nmode;
    a.target = mode;
    a.R = (int)R;
    a.crword = (u64)crm ? 0 : 1;
    a.crbit = (u64)crm ? (u64)crm : (u64)(crm >> 64);

    for (int m = 0; m < t->nmode; ++m) a.U[m] = (const FT*)dU[m];
    a.out = (FT*)dU[mode];
    a.fld = t->fld;
    const bool f64 = sizeof(FT) == 8;
    if (t->vdt == ALTOB_U32) return launch_atomic_cr<FT, u32>(a, st);
    if ((t->vdt == ALTOB_F64) == f64) return launch_atomic_cr<FT, FT>(a, st);
    return fail(ALTOB_ERR_UNSUPPORTED, "stored value dtype does not match the compute dtype");
}

altob_algo resolve_algo(const altob_tensor* t, int mode, altob_algo algo)
{
    if (algo != ALTOB_ALGO_AUTO) return algo;
    if (fib_reuse(t, mode) > 4) return ALTOB_ALGO_TILED;
    if (t->is_oidx && t->d_oidx[mode]) return ALTOB_ALGO_OPSCHED;
    if (t->cr_masks[mode]) return ALTOB_ALGO_ATOMIC_CR;
    return ALTOB_ALGO_ATOMIC;
}

altob_status mttkrp_device(altob_tensor* t, int mode, altob_dtype ft, void* const* dU, u64 R, int accumulate,
                           altob_algo algo, cudaStream_t st)
{
    if (!t || !dU) return fail(ALTOB_ERR_ARG, "NULL argument");
    if (mode < 0 || mode >= t->nmode) return fail(ALTOB_ERR_ARG, "mode out of range");
    if (R < 1) return fail(ALTOB_ERR_ARG, "rank must be >= 1");
    if (ft != ALTOB_F64 && ft != ALTOB_F32) return fail(ALTOB_ERR_ARG, "compute dtype must be F64 or F32");
    for (int m = 0; m < t->nmode; ++m)
        if (!dU[m]) return fail(ALTOB_ERR_ARG, "a factor pointer is NULL");
    const size_t fsz = ft == ALTOB_F64 ? 8 : 4;
    ALTOB_TRY(tensor_enter(t, st));
    TensorUse use(t, st);
    if (!accumulate) ALTOB_CUDA(cudaMemsetAsync(dU[mode], 0, t->dims[mode] * R * fsz, st));
    if (t->nnz == 0) return ALTOB_OK;
    algo = resolve_algo(t, mode, algo);
    const u32* perm = nullptr;
    bool cache = true;
    switch (algo) {
    case ALTOB_ALGO_TILED: break;
    case ALTOB_ALGO_ATOMIC: cache = false; break;
    case ALTOB_ALGO_OPSCHED:
        perm = t->d_oidx[mode];
        if (!perm) return fail(ALTOB_ERR_ARG, "OPSCHED needs oidx for the target mode (fiber reuse <= 4)");
        break;
    case ALTOB_ALGO_ATOMIC_CR:
        return ft == ALTOB_F64 ? run_atomic_cr<double>(t, mode, dU, R, st) : run_atomic_cr<float>(t, mode, dU, R, st);
    default: return fail(ALTOB_ERR_ARG, "unknown algorithm");
    }
    return ft == ALTOB_F64 ? run_tiled<double>(t, mode, dU, dU[mode], R, false, 0.0, perm, cache, st)
                           : run_tiled<float>(t, mode, dU, dU[mode], R, false, 0.0, perm, cache, st);
}

altob_status phi_device(altob_tensor* t, int mode, altob_dtype ft, void* const* dU, u64 R, double eps,
                        void* dphi, cudaStream_t st)
{
    if (!t || !dU || !dphi) return fail(ALTOB_ERR_ARG, "NULL argument");
    if (mode < 0 || mode >= t->nmode) return fail(ALTOB_ERR_ARG, "mode out of range");
    if (ft != ALTOB_F64 && ft != ALTOB_F32) return fail(ALTOB_ERR_ARG, "compute dtype must be F64 or F32");
    const size_t fsz = ft == ALTOB_F64 ? 8 : 4;
    ALTOB_TRY(tensor_enter(t, st));
    TensorUse use(t, st);
    ALTOB_CUDA(cudaMemsetAsync(dphi, 0, t->dims[mode] * R * fsz, st));
    if (t->nnz == 0) return ALTOB_OK;
    return ft == ALTOB_F64 ? run_tiled<double>(t, mode, dU, dphi, R, true, eps, nullptr, true, st)
                           : run_tiled<float>(t, mode, dU, dphi, R, true, eps, nullptr, true, st);
}

// ------------------------------------------------- precomputed Phi rows
// The Khatri-Rao row of every nonzero for target mode n (the product of the
// other modes' factor rows), computed once and reused by every inner
// iteration of that mode: the reference's PRE build of cp_apr_alto
// (apr.hpp:1133-1171, precomp_row).  Same products in the same order as the
// on-the-fly path, so both give the same Phi.

template <typename FT>
struct PiArgs {
    KeySrc key;
    Fields fld;
    u64 nnz;
    int nmode, target, R;
    const FT* U[ALTOB_MAX_MODES];
    FT* Pi;
    const u32* inv;  // row of nonzero i in Pi (row-ordered stream), or nullptr: row i
};

template <typename FT, int NM, int VEC>
__global__ void __launch_bounds__(256) k_pi(PiArgs<FT> a)
{
    constexpr int MM = NM ? NM : ALTOB_MAX_MODES;
    const int nmode = NM ? NM : a.nmode;
    const int cpr = a.R / VEC;  // VEC-wide chunks per row
    const u64 total = a.nnz * (u64)cpr;
    for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (u64)gridDim.x * blockDim.x) {
        const u64 i = t / cpr;
        const int c = (int)(t - i * cpr) * VEC;
        const u64 lo = a.key.klo[i];
        const u64 hi = a.key.khi ? a.key.khi[i] : (a.key.nrun ? key_hi(a.key, i) : 0);
        FT x[VEC];
#pragma unroll
        for (int e = 0; e < VEC; ++e) x[e] = FT(1);
#pragma unroll
        for (int m = 0; m < MM; ++m) {
            if (NM == 0 && m >= nmode) break;
            if (m == a.target) continue;
            const u32 row = field(lo, hi, a.fld.pos[m], a.fld.mask[m]);
            FT y[VEC];
            vload<FT, VEC>(a.U[m] + (size_t)row * a.R + c, y);
            vmul<FT, VEC>(x, y);
        }
        typedef typename VecT<FT, VEC>::T V;
        const u64 dst = a.inv ? (u64)a.inv[i] : i;
        *reinterpret_cast<V*>(a.Pi + dst * a.R + c) = *reinterpret_cast<const V*>(x);
    }
}

template <typename FT, int NM>
static void launch_pi_nm(const PiArgs<FT>& a, int vec, int grid, cudaStream_t st)
{
    constexpr int V = 16 / sizeof(FT);
    if (vec == V) k_pi<FT, NM, V><<<grid, 256, 0, st>>>(a);
    else k_pi<FT, NM, 1><<<grid, 256, 0, st>>>(a);
}

template <typename FT>
static altob_status pi_rows(altob_tensor* t, int mode, void* const* dU, u64 R, void* dpi, const u32* inv,
                           cudaStream_t st)
{
    PiArgs<FT> a;
    memset(&a, 0, sizeof(a));
    a.key = key_src(t);
    a.fld = t->fld;
    a.nnz = t->nnz;
    a.nmode = t->nmode;
    a.target = mode;
    a.R = (int)R;
    bool aligned = ptr_aligned16(dpi);
    for (int m = 0; m < t->nmode; ++m) {
        a.U[m] = (const FT*)dU[m];
        aligned = aligned && ptr_aligned16(dU[m]);
    }
    a.Pi = (FT*)dpi;
    a.inv = inv;
    constexpr int V = 16 / sizeof(FT);
    const int vec = (aligned && R % V == 0) ? V : 1;
    const u64 work = t->nnz * (R / vec);
    const int grid = (int)std::max<u64>(1, std::min<u64>((work + 255) / 256, (u64)num_sms() * 16));
    switch (t->nmode) {
    case 3: launch_pi_nm<FT, 3>(a, vec, grid, st); break;
    case 4: launch_pi_nm<FT, 4>(a, vec, grid, st); break;
    case 5: launch_pi_nm<FT, 5>(a, vec, grid, st); break;
    default: launch_pi_nm<FT, 0>(a, vec, grid, st); break;
    }
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

altob_status pi_device(altob_tensor* t, int mode, altob_dtype ft, void* const* dU, u64 R, void* dpi, cudaStream_t st,
                       const u32* inv)
{
    if (!t || !dU || !dpi) return fail(ALTOB_ERR_ARG, "NULL argument");
    if (mode < 0 || mode >= t->nmode) return fail(ALTOB_ERR_ARG, "mode out of range");
    if (t->nnz == 0) return ALTOB_OK;
    return ft == ALTOB_F64 ? pi_rows<double>(t, mode, dU, R, dpi, inv, st)
                           : pi_rows<float>(t, mode, dU, R, dpi, inv, st);
}

// ------------------------------------- CP-APR Phi over a row-ordered stream
// For target mode n the nonzeros are put once in the order of their mode-n
// index (a stable LSD radix sort of (index, position) pairs): rows[k] is the
// target row of stream position k, vals[k] its value and inv[i] the stream
// position of nonzero i.  k_pi then writes the Khatri-Rao row of nonzero i
// to stream row inv[i], so every inner iteration reads keys-free, fully
// sequential rows: Phi[r] = sum over the run of row r of
// (v / max(B[r] . pi, eps)) pi, the products and the dot product formed as in
// the tiled Phi (apr.hpp:383-848 computes the same sums per row).  A warp
// takes PR_CHUNK consecutive stream positions; each lane group keeps the
// running sum of its current row in registers and adds it to Phi with one
// vector atomic when the row changes (rows change rarely: the runs of a
// mode are nnz / dims long on average).

constexpr u64 PR_CHUNK = 512;
constexpr int PR_THREADS = 256;

__global__ void k_mode_idx(KeySrc key, Fields fld, int mode, u64 n, u64* __restrict__ idx, u32* __restrict__ iota)
{
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const u64 lo = key.klo[i], hi = key_hi(key, i);
        idx[i] = field(lo, hi, fld.pos[mode], fld.mask[mode]);
        iota[i] = (u32)i;
    }
}

template <typename FT, typename VT>
__global__ void k_row_meta(const u64* __restrict__ sidx, const u32* __restrict__ perm, const VT* __restrict__ vals,
                           u64 n, u32* __restrict__ rows, FT* __restrict__ svals, u32* __restrict__ inv)
{
    for (u64 k = (u64)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (u64)gridDim.x * blockDim.x) {
        const u32 p = perm[k];
        rows[k] = (u32)sidx[k];
        svals[k] = (FT)vals[p];
        inv[p] = (u32)k;
    }
}

// UN nonzeros of a lane group (stream positions k, k + G, ...; rw = ~0 past k1)
template <typename FT, int VEC, int LPN, int CH, int UN>
struct RowStep {
    u32 rw[UN];
    FT v[UN], x[UN][CH][VEC];
    __device__ __forceinline__ void load(const FT* __restrict__ Pi, const u32* __restrict__ rows,
                                         const FT* __restrict__ vals, u64 k, u64 k1, int R, int sub)
    {
        constexpr int G = 32 / LPN;
#pragma unroll
        for (int u = 0; u < UN; ++u) {
            const u64 ku = k + (u64)u * G;
            const bool ok = ku < k1;
            rw[u] = ok ? __ldcs(rows + ku) : 0xffffffffu;
            v[u] = ok ? __ldcs(vals + ku) : FT(0);
#pragma unroll
            for (int ch = 0; ch < CH; ++ch) {
                const int r0 = ch * LPN * VEC + sub * VEC;
                if (ok && r0 < R) vload_stream<FT, VEC>(Pi + ku * R + r0, x[u][ch]);
                else
#pragma unroll
                    for (int e = 0; e < VEC; ++e) x[u][ch][e] = FT(0);
            }
        }
    }
};

// Adds the step's nonzeros to the lane group's run; a row change flushes the
// run with one vector atomic per lane and reloads the cached B row.
template <typename FT, int VEC, int LPN, int CH, int UN>
__device__ __forceinline__ void row_step(const RowStep<FT, VEC, LPN, CH, UN>& s, const FT* __restrict__ B,
                                         FT* __restrict__ Phi, int R, int sub, unsigned gmask, FT eps, u32& cur,
                                         FT (*acc)[VEC], FT (*bc)[VEC])
{
#pragma unroll
    for (int u = 0; u < UN; ++u) {
        if (s.rw[u] == 0xffffffffu) break;  // past the chunk (uniform in the group)
        if (s.rw[u] != cur) {
#pragma unroll
            for (int ch = 0; ch < CH; ++ch) {
                const int r0 = ch * LPN * VEC + sub * VEC;
                if (r0 < R) {
                    if (cur != 0xffffffffu) gred<FT, VEC>(Phi + (size_t)cur * R + r0, acc[ch]);
                    vload<FT, VEC>(B + (size_t)s.rw[u] * R + r0, bc[ch]);
                }
#pragma unroll
                for (int e = 0; e < VEC; ++e) acc[ch][e] = FT(0);
            }
            cur = s.rw[u];
        }
        FT dot = FT(0);
#pragma unroll
        for (int ch = 0; ch < CH; ++ch) {
            const int r0 = ch * LPN * VEC + sub * VEC;
            if (r0 < R)
#pragma unroll
                for (int e = 0; e < VEC; ++e) dot += bc[ch][e] * s.x[u][ch][e];
        }
#pragma unroll
        for (int o = LPN / 2; o > 0; o >>= 1) dot += __shfl_xor_sync(gmask, dot, o, LPN);
        const FT sc = s.v[u] / (dot > eps ? dot : eps);
#pragma unroll
        for (int ch = 0; ch < CH; ++ch)
#pragma unroll
            for (int e = 0; e < VEC; ++e) acc[ch][e] += s.x[u][ch][e] * sc;
    }
}

// Resident blocks per SM the register budget is set for: while a lane holds
// at most 16 bytes of a stream row, four (64 registers) in FP32 and three in
// FP64; else two.
template <typename FT, int VEC, int CH>
constexpr int pr_min_blocks()
{
    return CH * VEC * (int)sizeof(FT) <= 16 ? (sizeof(FT) == 4 ? 4 : 3) : 2;
}

// Two register buffers of UN steps: the loads of the next buffer are issued
// before the current one is reduced, so a warp keeps 2 x UN x G stream rows
// in flight.
template <typename FT, int VEC, int LPN, int CH>
__global__ void __launch_bounds__(PR_THREADS, pr_min_blocks<FT, VEC, CH>()) k_phi_rows(const FT* __restrict__ Pi, const u32* __restrict__ rows,
                                                         const FT* __restrict__ vals, const FT* __restrict__ B,
                                                         FT* __restrict__ Phi, u64 nnz, int R, FT eps)
{
    constexpr int G = 32 / LPN;  // nonzeros per warp step
    constexpr int UN = 2;
    constexpr u64 S = (u64)G * UN;
    const int lane = threadIdx.x & 31, grp = lane / LPN, sub = lane % LPN;
    const unsigned gmask = LPN == 32 ? 0xffffffffu : (((1u << LPN) - 1u) << (grp * LPN));
    const u64 nchunks = (nnz + PR_CHUNK - 1) / PR_CHUNK;
    const u64 nw = ((u64)gridDim.x * blockDim.x) >> 5;
    for (u64 c = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < nchunks; c += nw) {
        const u64 k1 = min(nnz, (c + 1) * PR_CHUNK);
        u32 cur = 0xffffffffu;
        FT acc[CH][VEC], bc[CH][VEC];
#pragma unroll
        for (int ch = 0; ch < CH; ++ch)
#pragma unroll
            for (int e = 0; e < VEC; ++e) acc[ch][e] = bc[ch][e] = FT(0);
        RowStep<FT, VEC, LPN, CH, UN> a, b;
        u64 k = c * PR_CHUNK + grp;
        a.load(Pi, rows, vals, k, k1, R, sub);
        while (k < k1) {
            b.load(Pi, rows, vals, k + S, k1, R, sub);
            row_step(a, B, Phi, R, sub, gmask, eps, cur, acc, bc);
            k += S;
            if (k >= k1) break;
            a.load(Pi, rows, vals, k + S, k1, R, sub);
            row_step(b, B, Phi, R, sub, gmask, eps, cur, acc, bc);
            k += S;
        }
        if (cur != 0xffffffffu)
#pragma unroll
            for (int ch = 0; ch < CH; ++ch) {
                const int r0 = ch * LPN * VEC + sub * VEC;
                if (r0 < R) gred<FT, VEC>(Phi + (size_t)cur * R + r0, acc[ch]);
            }
    }
}

template <typename FT, typename VT>
static altob_status mode_order_vt(altob_tensor* t, int mode, u32* rows, FT* svals, u32* inv, cudaStream_t st)
{
    const u64 n = t->nnz;
    u64 *mk = nullptr, *mk2 = nullptr;
    u32 *p = nullptr, *p2 = nullptr;
    altob_status s = dmalloc_t(&mk, n);
    if (s == ALTOB_OK) s = dmalloc_t(&mk2, n);
    if (s == ALTOB_OK) s = dmalloc_t(&p, n);
    if (s == ALTOB_OK) s = dmalloc_t(&p2, n);
    int bits = 0;
    while (bits < 32 && (1ull << bits) < t->dims[mode]) ++bits;
    const int grid = (int)std::max<u64>(1, std::min<u64>((n + 255) / 256, (u64)num_sms() * 8));
    bool alt = false;
    if (s == ALTOB_OK) {
        k_mode_idx<<<grid, 256, 0, st>>>(key_src(t), t->fld, mode, n, mk, p);
        s = cudaGetLastError() == cudaSuccess ? ALTOB_OK : fail(ALTOB_ERR_CUDA, "mode index launch failed");
    }
    if (s == ALTOB_OK) s = radix_sort_pairs(mk, nullptr, p, mk2, nullptr, p2, n, 1, bits, st, &alt);
    if (s == ALTOB_OK) {
        k_row_meta<FT, VT><<<grid, 256, 0, st>>>(alt ? mk2 : mk, alt ? p2 : p, (const VT*)t->d_vals, n, rows, svals,
                                                 inv);
        s = cudaGetLastError() == cudaSuccess ? ALTOB_OK : fail(ALTOB_ERR_CUDA, "row order launch failed");
    }
    dfree(mk);
    dfree(mk2);
    dfree(p);
    dfree(p2);
    return s;
}

altob_status mode_order_device(altob_tensor* t, int mode, altob_dtype ft, u32* rows, void* svals, u32* inv,
                               cudaStream_t st)
{
    if (!t || !rows || !svals || !inv) return fail(ALTOB_ERR_ARG, "NULL argument");
    if (mode < 0 || mode >= t->nmode) return fail(ALTOB_ERR_ARG, "mode out of range");
    if (t->nnz == 0) return ALTOB_OK;
    const bool f64 = ft == ALTOB_F64;
    if (t->vdt == ALTOB_U32)
        return f64 ? mode_order_vt<double, u32>(t, mode, rows, (double*)svals, inv, st)
                   : mode_order_vt<float, u32>(t, mode, rows, (float*)svals, inv, st);
    if ((t->vdt == ALTOB_F64) != f64)
        return fail(ALTOB_ERR_UNSUPPORTED, "stored value dtype does not match the compute dtype");
    return f64 ? mode_order_vt<double, double>(t, mode, rows, (double*)svals, inv, st)
               : mode_order_vt<float, float>(t, mode, rows, (float*)svals, inv, st);
}

template <typename FT, int VEC>
static void launch_phi_rows(int lpn, int ch, int grid, const FT* pi, const u32* rows, const FT* vals, const FT* B,
                            FT* phi, u64 nnz, int R, FT eps, cudaStream_t st)
{
#define PRK(L, C) k_phi_rows<FT, VEC, L, C><<<grid, PR_THREADS, 0, st>>>(pi, rows, vals, B, phi, nnz, R, eps)
    if (ch == 4) PRK(32, 4);
    else if (ch == 2) PRK(32, 2);
    else if (lpn == 32) PRK(32, 1);
    else if (lpn == 16) PRK(16, 1);
    else if (lpn == 8) PRK(8, 1);
    else if (lpn == 4) PRK(4, 1);
    else if (lpn == 2) PRK(2, 1);
    else PRK(1, 1);
#undef PRK
}

// The handle's error word of the kernels with bounded waits (allocated on
// first use); fails when an earlier launch ran out of a wait limit.
static altob_status wait_error_word(altob_tensor* t, cudaStream_t st, unsigned** out)
{
    if (!t->d_tma_err) {
        ALTOB_TRY(dmalloc_t(&t->d_tma_err, 4));
        ALTOB_CUDA(cudaMemsetAsync(t->d_tma_err, 0, 4, st));
        ALTOB_CUDA(cudaMallocHost((void**)&t->h_tma_err, 4));
        *t->h_tma_err = 0;
    }
    if (*t->h_tma_err) return fail(ALTOB_ERR_CUDA, "an earlier bulk-copy-staged kernel ran out of a wait limit");
    *out = t->d_tma_err;
    return ALTOB_OK;
}

// Row-ordered Phi with the stream staged by bulk copies (phi_rows_tma.cuh).
template <typename FT, int VEC>
static altob_status launch_phi_rows_tma(altob_tensor* t, int lpn, const FT* pi, const u32* rows, const FT* vals,
                                        const FT* B, FT* phi, u64 nnz, int R, FT eps, cudaStream_t st)
{
    PhiTmaArgs<FT> a;
    a.Pi = pi;
    a.rows = rows;
    a.vals = vals;
    a.B = B;
    a.Phi = phi;
    a.nnz = nnz;
    a.R = R;
    a.eps = eps;
    a.wait_limit = TMA_WAIT_LIMIT;
    a.stall = 0;
    if (env_int("ALTOB_TEST_STALL_PHI", 0)) {
        // failure test: the producer warp issues nothing, so the consumers'
        // waits run out after a short limit (no copy is ever in flight) and
        // the kernel reports it through the handle's error word
        a.stall = 1;
        a.wait_limit = 1u << 12;
    }
    ALTOB_TRY(wait_error_word(t, st, &a.err));
    const u64 vg = (u64)PX_CONSUMERS * (32 / lpn);
    a.S = std::max<u64>(vg, (u64)PX_ROW_BYTES / ((u64)R * sizeof(FT)) / vg * vg);
    a.nstage = (nnz + a.S - 1) / a.S;
    const u64 grid0 = std::min<u64>(a.nstage, (u64)num_sms() * 2);
    a.per_cta = (a.nstage + grid0 - 1) / grid0;
    const unsigned grid = (unsigned)((a.nstage + a.per_cta - 1) / a.per_cta);
    const size_t smem = phi_tma_smem(a.S, R, (int)sizeof(FT));
    // the shared-memory limit is set once per kernel instance (one slot per
    // lane count; every instance of an FT has the same function type)
    static std::atomic<size_t> configured[6] = {};
    auto go = [&](void (*kern)(const PhiTmaArgs<FT>), int slot) -> altob_status {
        if (smem > configured[slot].load()) {
            ALTOB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            configured[slot].store(smem);
        }
        kern<<<grid, PX_THREADS, smem, st>>>(a);
        return ALTOB_OK;
    };
    altob_status s;
    switch (lpn) {
    case 1: s = go(k_phi_rows_tma<FT, VEC, 1>, 0); break;
    case 2: s = go(k_phi_rows_tma<FT, VEC, 2>, 1); break;
    case 4: s = go(k_phi_rows_tma<FT, VEC, 4>, 2); break;
    case 8: s = go(k_phi_rows_tma<FT, VEC, 8>, 3); break;
    case 16: s = go(k_phi_rows_tma<FT, VEC, 16>, 4); break;
    default: s = go(k_phi_rows_tma<FT, VEC, 32>, 5); break;
    }
    ALTOB_TRY(s);
    ALTOB_LAUNCH_CHECK();
    ALTOB_CUDA(cudaMemcpyAsync(t->h_tma_err, t->d_tma_err, 4, cudaMemcpyDeviceToHost, st));
    return ALTOB_OK;
}

altob_status phi_rows_device(altob_tensor* t, int mode, altob_dtype ft, const void* dpi, const u32* rows,
                             const void* svals, const void* dB, u64 R, double eps, void* dphi, cudaStream_t st,
                             bool pad4)
{
    if (!t || !dpi || !rows || !svals || !dB || !dphi) return fail(ALTOB_ERR_ARG, "NULL argument");
    if (mode < 0 || mode >= t->nmode) return fail(ALTOB_ERR_ARG, "mode out of range");
    if (R == 0 || R > 128) return fail(ALTOB_ERR_UNSUPPORTED, "rank must be 1..128");
    const size_t fsz = ft == ALTOB_F64 ? 8 : 4;
    ALTOB_CUDA(cudaMemsetAsync(dphi, 0, t->dims[mode] * R * fsz, st));
    if (t->nnz == 0) return ALTOB_OK;
    const int V = (int)(16 / fsz);
    const bool vec = R % V == 0 && ptr_aligned16(dpi) && ptr_aligned16(dB) && ptr_aligned16(dphi);
    const int ve = vec ? V : 1;
    int lpn = 1;
    while (lpn < 32 && (u64)lpn * ve < R) lpn <<= 1;
    const int ch = (int)((R + (u64)lpn * ve - 1) / ((u64)lpn * ve));  // 1, 2 or 4 (only with 32 lanes)
    const u64 nchunks = (t->nnz + PR_CHUNK - 1) / PR_CHUNK;
    const int per_sm = ch * ve * (int)fsz <= 16 ? (fsz == 4 ? 4 : 3) : 2;  // pr_min_blocks: one wave
    const int grid = (int)std::max<u64>(1, std::min<u64>((nchunks + 7) / 8, (u64)num_sms() * per_sm));
    const u64 nnz = t->nnz;
    // the stream staged by bulk copies (ALTOB_PHI_TMA=1; measured no faster
    // than the register-staged kernel): one vector chunk per lane, whole
    // 16-byte rows, stream arrays readable to a multiple of 4 past the end
    if (pad4 && vec && ch == 1 && (R * fsz) % 16 == 0 && env_int("ALTOB_PHI_TMA", 0)) {
        if (ft == ALTOB_F64)
            return launch_phi_rows_tma<double, 2>(t, lpn, (const double*)dpi, rows, (const double*)svals,
                                                  (const double*)dB, (double*)dphi, nnz, (int)R, eps, st);
        return launch_phi_rows_tma<float, 4>(t, lpn, (const float*)dpi, rows, (const float*)svals, (const float*)dB,
                                             (float*)dphi, nnz, (int)R, (float)eps, st);
    }
    if (ft == ALTOB_F64) {
        if (vec) launch_phi_rows<double, 2>(lpn, ch, grid, (const double*)dpi, rows, (const double*)svals,
                                            (const double*)dB, (double*)dphi, nnz, (int)R, eps, st);
        else launch_phi_rows<double, 1>(lpn, ch, grid, (const double*)dpi, rows, (const double*)svals,
                                        (const double*)dB, (double*)dphi, nnz, (int)R, eps, st);
    } else {
        if (vec) launch_phi_rows<float, 4>(lpn, ch, grid, (const float*)dpi, rows, (const float*)svals,
                                           (const float*)dB, (float*)dphi, nnz, (int)R, (float)eps, st);
        else launch_phi_rows<float, 1>(lpn, ch, grid, (const float*)dpi, rows, (const float*)svals,
                                       (const float*)dB, (float*)dphi, nnz, (int)R, (float)eps, st);
    }
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

// Phi of mode `mode` from precomputed rows `dpi` and the current factor B.
template <typename FT, typename VT>
static altob_status run_phi_pre_vt(altob_tensor* t, int mode, const void* dpi, const void* dB, void* dphi, u64 R,
                                   double eps, cudaStream_t st)
{
    const bool aligned = ptr_aligned16(dpi) && ptr_aligned16(dB) && ptr_aligned16(dphi);
    TiledPlan pl;
    ALTOB_TRY(plan_tiled(t, R, sizeof(FT), aligned, true, &pl));
    TiledArgs<FT> a;
    memset(&a, 0, sizeof(a));
    a.key = key_src(t);
    a.vals = t->d_vals;
    a.perm = nullptr;
    a.nnz = t->nnz;
    a.ntiles = (t->nnz + GT_TILE - 1) / GT_TILE;
    a.nmode = t->nmode;
    a.target = mode;
    a.R = (int)R;
    a.tile = GT_TILE;
    a.hslots = pl.hslots ? pl.hslots : 2048;
    a.eps = (FT)eps;
    a.U[0] = (const FT*)dpi;
    a.U[1] = (const FT*)dB;
    a.out = (FT*)dphi;
    a.fld = t->fld;
    a.hot = env_int("ALTOB_HOT_ROWS", 1) ? grouped_hot_slots((int)R, sizeof(FT)) : 0;
    TiledCfg c;
    c.lpn = pl.lpn;
    c.vec = pl.vec;
    c.ch = pl.ch;
    c.phi = 1;
    c.grouped = 1;
    c.pre = 1;
    c.smem = grouped_smem(a.hslots, 2, sizeof(FT), a.hot, (int)R);
    c.grid = dim3(0);
    int bps = 0;
    ALTOB_TRY((launch_tiled<FT, VT>(a, c, st, &bps)));
    if (bps < 1) return fail(ALTOB_ERR_UNSUPPORTED, "Phi kernel does not fit on an SM");
    const u64 cap = (u64)bps * num_sms();
    c.grid = dim3((unsigned)std::max<u64>(1, std::min<u64>(a.ntiles, cap)));
    ALTOB_TRY(set_hot_acc(t, a, c.grid.x, st));
    return launch_tiled<FT, VT>(a, c, st, nullptr);
}

altob_status phi_pre_device(altob_tensor* t, int mode, altob_dtype ft, const void* dpi, const void* dB, u64 R,
                            double eps, void* dphi, cudaStream_t st)
{
    if (!t || !dpi || !dB || !dphi) return fail(ALTOB_ERR_ARG, "NULL argument");
    if (mode < 0 || mode >= t->nmode) return fail(ALTOB_ERR_ARG, "mode out of range");
    const size_t fsz = ft == ALTOB_F64 ? 8 : 4;
    ALTOB_TRY(tensor_enter(t, st));
    TensorUse use(t, st);
    ALTOB_CUDA(cudaMemsetAsync(dphi, 0, t->dims[mode] * R * fsz, st));
    if (t->nnz == 0) return ALTOB_OK;
    const bool f64 = ft == ALTOB_F64;
    if (t->vdt == ALTOB_U32)
        return f64 ? run_phi_pre_vt<double, u32>(t, mode, dpi, dB, dphi, R, eps, st)
                   : run_phi_pre_vt<float, u32>(t, mode, dpi, dB, dphi, R, eps, st);
    if ((t->vdt == ALTOB_F64) != f64) return fail(ALTOB_ERR_UNSUPPORTED, "stored value dtype does not match the compute dtype");
    return f64 ? run_phi_pre_vt<double, double>(t, mode, dpi, dB, dphi, R, eps, st)
               : run_phi_pre_vt<float, float>(t, mode, dpi, dB, dphi, R, eps, st);
}

// Copies host factors into the handle's cached scratch (no per-call
// allocation once the scratch is large enough).
static altob_status upload_factors(altob_tensor* t, void* const* h, size_t fsz, u64 R, void** d, cudaStream_t st)
{
    size_t total = 0, offs[ALTOB_MAX_MODES];
    for (int m = 0; m < t->nmode; ++m) {
        if (!h[m]) return fail(ALTOB_ERR_ARG, "a host factor pointer is NULL");
        offs[m] = total;
        total += (t->dims[m] * R * fsz + 255) & ~(size_t)255;
    }
    void* base = nullptr;
    ALTOB_TRY(tensor_scratch(t, total, &base));
    for (int m = 0; m < t->nmode; ++m) {
        d[m] = (char*)base + offs[m];
        ALTOB_CUDA(cudaMemcpyAsync(d[m], h[m], t->dims[m] * R * fsz, cudaMemcpyHostToDevice, st));
    }
    return ALTOB_OK;
}

}  // namespace altob

using namespace altob;

extern "C" {

altob_status altob_mttkrp(altob_tensor* t, int mode, altob_dtype ftype, void* const* d_factors, uint64_t rank,
                          int accumulate, altob_algo algo, void* stream)
{
    StreamScope scope((cudaStream_t)stream);
    return mttkrp_device(t, mode, ftype, d_factors, rank, accumulate, algo, (cudaStream_t)stream);
}

altob_status altob_phi(altob_tensor* t, int mode, altob_dtype ftype, void* const* d_factors, uint64_t rank,
                       double eps_div_zero, void* d_phi, void* stream)
{
    StreamScope scope((cudaStream_t)stream);
    return phi_device(t, mode, ftype, d_factors, rank, eps_div_zero, d_phi, (cudaStream_t)stream);
}

altob_status altob_mttkrp_host(altob_tensor* t, int mode, altob_dtype ftype, void* const* h_factors, uint64_t rank,
                               altob_algo algo, void* stream)
{
    if (!t || !h_factors) return fail(ALTOB_ERR_ARG, "NULL argument");
    if (mode < 0 || mode >= t->nmode) return fail(ALTOB_ERR_ARG, "mode out of range");
    cudaStream_t st = (cudaStream_t)stream;
    StreamScope scope(st);
    const size_t fsz = ftype == ALTOB_F64 ? 8 : 4;
    void* d[ALTOB_MAX_MODES];
    altob_status s = upload_factors(t, h_factors, fsz, rank, d, st);
    if (s == ALTOB_OK) s = mttkrp_device(t, mode, ftype, d, rank, 1, algo, st);
    if (s == ALTOB_OK) {
        cudaError_t e = cudaMemcpyAsync(h_factors[mode], d[mode], t->dims[mode] * rank * fsz,
                                        cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) s = fail(ALTOB_ERR_CUDA, std::string("mttkrp_host: ") + cudaGetErrorString(e));
    }
    cudaStreamSynchronize(st);
    return s;
}

altob_status altob_mttkrp_sweep_host(altob_tensor* t, altob_dtype ftype, void* const* h_factors, uint64_t rank,
                                     int iters, altob_algo algo, void* stream)
{
    if (!t || !h_factors) return fail(ALTOB_ERR_ARG, "NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    StreamScope scope(st);
    const size_t fsz = ftype == ALTOB_F64 ? 8 : 4;
    void* d[ALTOB_MAX_MODES];
    altob_status s = upload_factors(t, h_factors, fsz, rank, d, st);
    // In the last sweep, factor m is final once mode m is done: its copy back
    // runs on a second stream while the later modes compute.
    cudaStream_t cs = nullptr;
    cudaEvent_t ev[ALTOB_MAX_MODES] = {nullptr};
    if (s == ALTOB_OK && iters > 0) {
        if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) cs = nullptr;
        for (int m = 0; cs && m < t->nmode; ++m)
            if (cudaEventCreateWithFlags(&ev[m], cudaEventDisableTiming) != cudaSuccess) ev[m] = nullptr;
    }
    for (int i = 0; i < iters && s == ALTOB_OK; ++i)
        for (int m = 0; m < t->nmode && s == ALTOB_OK; ++m) {
            s = mttkrp_device(t, m, ftype, d, rank, 1, algo, st);
            if (s == ALTOB_OK && i == iters - 1 && cs && ev[m]) {
                cudaEventRecord(ev[m], st);
                cudaStreamWaitEvent(cs, ev[m], 0);
                cudaError_t e = cudaMemcpyAsync(h_factors[m], d[m], t->dims[m] * rank * fsz, cudaMemcpyDeviceToHost,
                                                cs);
                if (e != cudaSuccess) s = fail(ALTOB_ERR_CUDA, std::string("sweep copy-out: ") + cudaGetErrorString(e));
            }
        }
    for (int m = 0; m < t->nmode && s == ALTOB_OK; ++m) {
        if (cs && ev[m] && iters > 0) continue;  // already copied on the second stream
        cudaError_t e = cudaMemcpyAsync(h_factors[m], d[m], t->dims[m] * rank * fsz, cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) s = fail(ALTOB_ERR_CUDA, std::string("sweep copy-out: ") + cudaGetErrorString(e));
    }
    if (cs) {
        cudaError_t e = cudaStreamSynchronize(cs);
        if (s == ALTOB_OK && e != cudaSuccess) s = fail(ALTOB_ERR_CUDA, std::string("sweep: ") + cudaGetErrorString(e));
        cudaStreamDestroy(cs);
    }
    for (int m = 0; m < ALTOB_MAX_MODES; ++m)
        if (ev[m]) cudaEventDestroy(ev[m]);
    cudaError_t e = cudaStreamSynchronize(st);
    if (s == ALTOB_OK && e != cudaSuccess) s = fail(ALTOB_ERR_CUDA, std::string("sweep: ") + cudaGetErrorString(e));
    return s;
}

}  // extern "C"
