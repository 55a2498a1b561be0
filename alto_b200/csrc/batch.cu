// batch.cu -- many independent CP-ALS solves in batched launches.
//
// No counterpart in the reference (it decomposes one tensor per process).
// Every tensor of the batch keeps its own device model and follows exactly
// the per-tensor algorithm of cpd_alto (include/cpd.hpp:43-186, as in
// cpd.cu), but each step runs for all tensors in one launch:
//   zero U_j | MTTKRP (one launch per shape class) | prepare |
//   R x R solve (one CTA per tensor) | fused row update + column norms +
//   Gram (+ fit inner product) | lambda, Gram scaling | U_j /= lambda
//   -- for every mode j; rank classes above 64 keep the separate passes
//   (copy of the last mode, row apply + column norms, lambda, Gram of the
//   normalised factor) --
//   then the fit, which also records the per-iteration fit and clears the
//   tensor's active flag when |fit - prev| < epsilon or max_iters is reached.
// Inactive tensors are skipped by every kernel, so a tensor's result equals
// its stand-alone solve.  Iterations after the first are captured once as a
// CUDA graph and replayed.  A shape class is (order, lanes per nonzero,
// elements per lane, chunks, nnz decade, whether a mode reads through oidx);
// its row-slot count and lane layout are picked by altob_batch_autotune.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "dense_kernels.cuh"
#include "mttkrp_launch.cuh"
#include "mttkrp_plan.h"

namespace altob {

template <typename FT>
struct BDesc {
    FT* U[ALTOB_MAX_MODES];
    u64 dims[ALTOB_MAX_MODES];
    int nmode, R;
    double *G, *W, *colacc, *lam, *inner, *fit_tmp, *fits;
    FT* M;
    FT* lam_out;
    double normAT;
    int* info;
};

// ------------------------------------------------------------ kernels

// Flattened per-mode grid: tensor list[i] owns blocks [prefix[i], prefix[i+1]),
// so small tensors get few CTAs and large ones many.
struct BlkMap {
    const int* list;
    const int* prefix;  // n + 1
    int n;
};

__device__ __forceinline__ int blk_owner(const BlkMap& m, int* bx, int* nbx)
{
    const int blk = (int)blockIdx.x;
    int lo = 0, hi = m.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (m.prefix[mid] <= blk) lo = mid;
        else hi = mid - 1;
    }
    *bx = blk - m.prefix[lo];
    *nbx = m.prefix[lo + 1] - m.prefix[lo];
    return m.list[lo];
}

template <typename FT>
__global__ void k_b_zero(const BDesc<FT>* __restrict__ d, BlkMap map, const int* __restrict__ active, int j)
{
    int bx, nbx;
    const int b = blk_owner(map, &bx, &nbx);
    if (!active[b]) return;
    const BDesc<FT>& t = d[b];
    const u64 n = t.dims[j] * (u64)t.R;
    FT* U = t.U[j];
    for (u64 e = (u64)bx * blockDim.x + threadIdx.x; e < n; e += (u64)nbx * blockDim.x) U[e] = FT(0);
}

template <typename FT>
__global__ void k_b_copym(const BDesc<FT>* __restrict__ d, BlkMap map, const int* __restrict__ active, int j)
{
    int bx, nbx;
    const int b = blk_owner(map, &bx, &nbx);
    if (!active[b]) return;
    const BDesc<FT>& t = d[b];
    if (j != t.nmode - 1 || t.R <= APPLY_GRAM_MAX_RANK) return;  // the fused pass reads M itself
    const u64 n = t.dims[j] * (u64)t.R;
    for (u64 e = (u64)bx * blockDim.x + threadIdx.x; e < n; e += (u64)nbx * blockDim.x) t.M[e] = t.U[j][e];
}

template <typename FT>
__global__ void k_b_prep(const BDesc<FT>* __restrict__ d, const int* __restrict__ list,
                         const int* __restrict__ active, int j, int nk)
{
    const int b = list[blockIdx.x];
    if (!active[b]) return;
    const BDesc<FT>& t = d[b];
    const int R = t.R;
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        t.colacc[r] = nk == NORM_MAX ? 1.0 : 0.0;
        if (j == t.nmode - 1) t.inner[r] = 0.0;
    }
    double* G = t.G + (size_t)j * R * R;
    for (int e = threadIdx.x; e < R * R; e += blockDim.x) G[e] = 0.0;
}

template <typename FT>
__global__ void __launch_bounds__(DN_THREADS) k_b_solve(const BDesc<FT>* __restrict__ d,
                                                        const int* __restrict__ list,
                                                        const int* __restrict__ active, int j)
{
    const int b = list[blockIdx.x];
    if (!active[b]) return;
    const BDesc<FT>& t = d[b];
    solve_body(t.G, t.nmode, j, t.R, t.W, t.info);
}

template <typename FT, int LPR, int CJ>
__global__ void __launch_bounds__(DN_THREADS) k_b_apply(const BDesc<FT>* __restrict__ d, BlkMap map,
                                                        const int* __restrict__ active, int j, int nk)
{
    int bx, nbx;
    const int b = blk_owner(map, &bx, &nbx);
    if (!active[b]) return;
    const BDesc<FT>& t = d[b];
    apply_body<FT, LPR, CJ>(t.U[j], t.dims[j], t.R, t.W, nk, t.colacc, bx, nbx);
}

// fused row update + Gram of U_j (R <= 64, see apply_gram_body), one launch
// per rank class
template <typename FT, int MB>
__global__ void __launch_bounds__(AG_THREADS) k_b_apply_gram(const BDesc<FT>* __restrict__ d, BlkMap map,
                                                             const int* __restrict__ active, int j, int nk)
{
    int bx, nbx;
    const int b = blk_owner(map, &bx, &nbx);
    if (!active[b]) return;
    const BDesc<FT>& t = d[b];
    const int R = t.R;
    const int vec_ok = ((uintptr_t)t.U[j] & 15) == 0;
    apply_gram_body<FT, MB>(t.U[j], t.dims[j], R, t.W, nk, t.colacc, t.G + (size_t)j * R * R,
                            j == t.nmode - 1 ? t.inner : nullptr, vec_ok, bx, nbx);
}

// U_j /= lambda after the fused pass
template <typename FT>
__global__ void __launch_bounds__(DN_THREADS) k_b_div_cols(const BDesc<FT>* __restrict__ d, BlkMap map,
                                                           const int* __restrict__ active, int j)
{
    int bx, nbx;
    const int b = blk_owner(map, &bx, &nbx);
    if (!active[b]) return;
    const BDesc<FT>& t = d[b];
    constexpr int V = 16 / sizeof(FT);
    if (t.R % V == 0 && ((uintptr_t)t.U[j] & 15) == 0) div_cols_body<FT, V>(t.U[j], t.dims[j], t.R, t.lam, bx, nbx);
    else div_cols_body<FT, 1>(t.U[j], t.dims[j], t.R, t.lam, bx, nbx);
}

// lambda from the column statistics; after the fused pass (R <= 64) also
// G_j /= lambda lambda^T and the inner product /= lambda
template <typename FT>
__global__ void k_b_lambda(const BDesc<FT>* __restrict__ d, const int* __restrict__ list,
                           const int* __restrict__ active, int nk, int j)
{
    const int b = list[blockIdx.x];
    if (!active[b]) return;
    const BDesc<FT>& t = d[b];
    if (t.R <= APPLY_GRAM_MAX_RANK) {
        lambda_finish_body(t.colacc, t.R, nk, t.lam, t.G + (size_t)j * t.R * t.R,
                           j == t.nmode - 1 ? t.inner : nullptr);
        return;
    }
    for (int r = threadIdx.x; r < t.R; r += blockDim.x) t.lam[r] = nk == NORM_2 ? sqrt(t.colacc[r]) : t.colacc[r];
}

// Gram of U_j; with `scaled`, U_j /= lambda first (written back) and the
// fit's inner product with the saved MTTKRP of the last mode.
template <typename FT, int MAXT>
__global__ void __launch_bounds__(DN_THREADS) k_b_gram(const BDesc<FT>* __restrict__ d, BlkMap map,
                                                       const int* __restrict__ active, int j, int scaled)
{
    int bx, nbx;
    const int b = blk_owner(map, &bx, &nbx);
    if (!active[b]) return;
    const BDesc<FT>& t = d[b];
    const int R = t.R;
    const bool last = j == t.nmode - 1;
    gram_body<FT, MAXT>(t.U[j], t.dims[j], R, t.G + (size_t)j * R * R, scaled ? t.lam : nullptr,
                        scaled ? t.U[j] : nullptr, (scaled && last) ? t.M : nullptr, t.inner, bx, nbx);
}

template <typename FT>
__global__ void __launch_bounds__(DN_THREADS) k_b_fit(const BDesc<FT>* __restrict__ d, int* __restrict__ active,
                                                      int* __restrict__ iters, double eps, int max_iters)
{
    const int b = blockIdx.x;
    if (!active[b]) return;
    const BDesc<FT>& t = d[b];
    fit_body(t.G, t.nmode, t.R, t.lam, t.inner, t.normAT, t.fit_tmp);
    if (threadIdx.x == 0) {
        const double f = *t.fit_tmp;
        const int it = iters[b];
        t.fits[it] = f;
        iters[b] = it + 1;
        if ((it > 0 && fabs(t.fits[it - 1] - f) < eps) || it + 1 >= max_iters) active[b] = 0;
    }
}

template <typename FT>
__global__ void k_b_lamout(const BDesc<FT>* __restrict__ d, int count)
{
    const int b = blockIdx.x;
    if (b >= count) return;
    const BDesc<FT>& t = d[b];
    if (!t.lam_out) return;
    for (int r = threadIdx.x; r < t.R; r += blockDim.x) t.lam_out[r] = (FT)t.lam[r];
}

template <typename FT, typename VT>
__global__ void k_b_sumsq(BDesc<FT>* __restrict__ d, const void* const* __restrict__ vals,
                          const u64* __restrict__ nnz)
{
    const int b = blockIdx.y;
    const VT* v = reinterpret_cast<const VT*>(vals[b]);
    double s = 0.0;
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < nnz[b]; e += (u64)gridDim.x * blockDim.x) {
        const double x = (double)v[e];
        s += x * x;
    }
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&d[b].normAT, s);
}

// ---------------------------------------------------------------- host

// Choices of the autotuner, remembered per (factor type, shape class) for
// every later batch in the process.
struct TuneChoice {
    int hslots, lpn, ch;
    float ms;
};
static std::mutex g_tune_mu;
static std::map<std::string, TuneChoice> g_tune;

static bool tune_lookup(const std::string& k, TuneChoice* out)
{
    std::lock_guard<std::mutex> g(g_tune_mu);
    auto it = g_tune.find(k);
    if (it == g_tune.end()) return false;
    *out = it->second;
    return true;
}

static void tune_store(const std::string& k, const TuneChoice& c)
{
    std::lock_guard<std::mutex> g(g_tune_mu);
    g_tune[k] = c;
}

// The tiles of the tensors whose target mode has a tile plan, per mode
// (batched planned kernel; the rest of a class runs the grouped kernel).
template <typename FT>
struct PlannedPart {
    int count[ALTOB_MAX_MODES] = {0};
    TiledArgs<FT>* d_args[ALTOB_MAX_MODES] = {nullptr};
    u64* d_prefix[ALTOB_MAX_MODES] = {nullptr};
    int* d_bid[ALTOB_MAX_MODES] = {nullptr};
    u64 total_tiles[ALTOB_MAX_MODES] = {0};
    unsigned gridx = 1;
    size_t smem = 0;
    void free_args()
    {
        for (int j = 0; j < ALTOB_MAX_MODES; ++j) {
            dfree(d_args[j]);
            dfree(d_prefix[j]);
            dfree(d_bid[j]);
            d_args[j] = nullptr;
            d_prefix[j] = nullptr;
            d_bid[j] = nullptr;
            total_tiles[j] = 0;
            count[j] = 0;
        }
    }
};

template <typename FT>
struct ClassRun {
    int nm = 0;  // order 3-5 (static loops), or 0 (generic)
    altob_dtype vdt = ALTOB_F32;
    int lpn = 32, vec = 1, ch = 4;
    int hslots = 0;      // row slots of the grouped kernel (0: no grouping)
    unsigned gridx = 1;  // resident CTAs for the current choice
    size_t smem = 0;
    std::vector<int> members;  // batch indices
    int mode_count[ALTOB_MAX_MODES] = {0};
    TiledArgs<FT>* d_args[ALTOB_MAX_MODES] = {nullptr};
    u64* d_prefix[ALTOB_MAX_MODES] = {nullptr};
    int* d_bid[ALTOB_MAX_MODES] = {nullptr};
    u64 total_tiles[ALTOB_MAX_MODES] = {0};
    std::string key;
    float tuned_ms = -1.f;
    PlannedPart<FT> pp;

    TiledCfg cfg(unsigned gx) const
    {
        TiledCfg c;
        c.lpn = lpn;
        c.vec = vec;
        c.ch = ch;
        c.phi = 0;
        c.grouped = 1;
        c.grid = dim3(gx);
        c.smem = smem;
        return c;
    }
    void free_args()
    {
        for (int j = 0; j < ALTOB_MAX_MODES; ++j) {
            dfree(d_args[j]);
            dfree(d_prefix[j]);
            dfree(d_bid[j]);
            d_args[j] = nullptr;
            d_prefix[j] = nullptr;
            d_bid[j] = nullptr;
            total_tiles[j] = 0;
        }
        pp.free_args();
    }
};

// Classes that share a kernel template (order, lanes, elements per lane,
// chunks, value type) after tuning run in one launch per mode; each tensor
// keeps its class's row-slot count (the slot table is laid out for the
// largest one).
template <typename FT>
struct LaunchGroup {
    int nm = 0;
    altob_dtype vdt = ALTOB_F32;
    int lpn = 32, vec = 1, ch = 4;
    int hmax = 0;
    unsigned gridx = 1;
    size_t smem = 0;
    PlannedPart<FT> pp;
    int count[ALTOB_MAX_MODES] = {0};
    TiledArgs<FT>* d_args[ALTOB_MAX_MODES] = {nullptr};
    u64* d_prefix[ALTOB_MAX_MODES] = {nullptr};
    int* d_bid[ALTOB_MAX_MODES] = {nullptr};
    u64 total_tiles[ALTOB_MAX_MODES] = {0};

    TiledCfg cfg(unsigned gx) const
    {
        TiledCfg c;
        c.lpn = lpn;
        c.vec = vec;
        c.ch = ch;
        c.phi = 0;
        c.grouped = 1;
        c.grid = dim3(gx);
        c.smem = smem;
        return c;
    }
    void free_args()
    {
        for (int j = 0; j < ALTOB_MAX_MODES; ++j) {
            dfree(d_args[j]);
            dfree(d_prefix[j]);
            dfree(d_bid[j]);
            d_args[j] = nullptr;
            d_prefix[j] = nullptr;
            d_bid[j] = nullptr;
            total_tiles[j] = 0;
        }
        pp.free_args();
    }
};

struct BatchBase {
    virtual ~BatchBase() {}
    virtual altob_status autotune(int force, cudaStream_t st) = 0;
    virtual altob_status solve(int max_iters, double eps, double* fits, int* iters, int use_graph,
                               cudaStream_t st) = 0;
    virtual void describe(std::string* out) const = 0;
};

template <typename FT>
struct BatchImpl : BatchBase {
    int count = 0, maxN = 0, maxR = 0, cap = 0;
    std::vector<altob_tensor*> ts;
    std::vector<BDesc<FT>> hdesc;
    BDesc<FT>* d_desc = nullptr;
    int* d_active = nullptr;
    int* d_iters = nullptr;
    int* d_list[ALTOB_MAX_MODES] = {nullptr};
    int nlist[ALTOB_MAX_MODES] = {0};
    void* d_scratch = nullptr;
    std::vector<std::unique_ptr<ClassRun<FT>>> classes;
    std::vector<std::unique_ptr<LaunchGroup<FT>>> groups;
    cudaStream_t cap_stream = nullptr;  // graph capture (never the legacy stream)
    int prio = 0;                       // priority of the internal streams
    static constexpr int NFORK = 4;     // streams the launch groups of a mode spread over
    cudaStream_t fork_st[NFORK] = {nullptr};
    cudaEvent_t fork_ev = nullptr, join_ev[NFORK] = {nullptr};
    cudaGraphExec_t gexec = nullptr;
    double g_eps = -1.0;
    int g_iters = -1;
    // per mode: flattened block maps of the row kernels (apply, Gram) and of
    // the element kernels (zero, copy)
    // (mode, rank class): tensor list, row-block map, largest rank
    int* d_clist[ALTOB_MAX_MODES][NRANK_CLASSES] = {};
    int* d_rowpre[ALTOB_MAX_MODES][NRANK_CLASSES] = {};
    int ncl[ALTOB_MAX_MODES][NRANK_CLASSES] = {};
    int nrowblk[ALTOB_MAX_MODES][NRANK_CLASSES] = {};
    int cmaxR[NRANK_CLASSES] = {};
    int* d_elpre[ALTOB_MAX_MODES] = {nullptr};
    int nelblk[ALTOB_MAX_MODES] = {0};
    static constexpr u64 ROWS_PER_CTA = 512;
    static constexpr u64 ELEMS_PER_CTA = 16384;
    static constexpr u64 MAX_CTAS_PER_TENSOR = 64;
    int launches_per_iter = 0;  // kernels one iteration launches (last count)

    ~BatchImpl() override
    {
        StreamScope scope(0);
        if (gexec) cudaGraphExecDestroy(gexec);
        if (cap_stream) cudaStreamDestroy(cap_stream);
        for (int i = 0; i < NFORK; ++i) {
            if (fork_st[i]) cudaStreamDestroy(fork_st[i]);
            if (join_ev[i]) cudaEventDestroy(join_ev[i]);
        }
        if (fork_ev) cudaEventDestroy(fork_ev);
        dfree(d_desc);
        dfree(d_active);
        dfree(d_iters);
        for (int j = 0; j < ALTOB_MAX_MODES; ++j) {
            dfree(d_list[j]);
            dfree(d_elpre[j]);
            for (int c = 0; c < NRANK_CLASSES; ++c) {
                dfree(d_clist[j][c]);
                dfree(d_rowpre[j][c]);
            }
        }
        dfree(d_scratch);
        for (auto& c : classes) c->free_args();
        for (auto& g : groups) g->free_args();
    }

    void drop_graph()
    {
        if (gexec) cudaGraphExecDestroy(gexec);
        gexec = nullptr;
    }

    altob_status launch_mt(int nm, altob_dtype vdt, const BatchTiles<FT>& bt, const TiledCfg& cfg, cudaStream_t st,
                           int* bps)
    {
        if (vdt == ALTOB_U32) return launch_batch<FT, u32>(bt, nm, cfg, st, bps);
        return launch_batch<FT, FT>(bt, nm, cfg, st, bps);
    }
    altob_status launch_mt(const ClassRun<FT>& c, const BatchTiles<FT>& bt, const TiledCfg& cfg, cudaStream_t st,
                           int* bps)
    {
        return launch_mt(c.nm, c.vdt, bt, cfg, st, bps);
    }

    // MTTKRP arguments of tensor b for target mode j with `hslots` row slots
    // (and the mode's tile plan when it is read in ALTO order).
    TiledArgs<FT> make_args(int b, int j, int hslots, bool want_plan, cudaStream_t st) const
    {
        altob_tensor* t = ts[b];
        TiledArgs<FT> a;
        memset(&a, 0, sizeof(a));
        a.key = key_src(t);
        a.vals = t->d_vals;
        // low fiber reuse: read in the target mode's order (oidx), as the
        // reference's op_sched dispatch does (alto.hpp:637-664)
        a.perm = (fib_reuse(t, j) <= 4 && t->d_oidx[j]) ? t->d_oidx[j] : nullptr;
        a.nnz = t->nnz;
        a.ntiles = (t->nnz + GT_TILE - 1) / GT_TILE;
        a.nmode = t->nmode;
        a.target = j;
        a.R = hdesc[b].R;
        a.tile = GT_TILE;
        a.hslots = hslots;
        a.eps = FT(0);
        for (int m = 0; m < t->nmode; ++m) a.U[m] = hdesc[b].U[m];
        a.out = hdesc[b].U[j];
        a.fld = t->fld;
        a.plan = (want_plan && !a.perm) ? tensor_plan(t, j, st) : nullptr;
        return a;
    }

    // Uploads per-mode tables for (tensor, slots) members; returns counts.
    // planned: 1 = the members whose mode has a tile plan, 0 = the others
    // (a class whose kernel shape has no planned form keeps every member in
    // the grouped tables)
    altob_status upload_tables(const std::vector<std::pair<int, int>>& mem, int planned, bool plan_shape,
                               TiledArgs<FT>** d_args, u64** d_prefix, int** d_bid, u64* total_tiles, int* count,
                               cudaStream_t st)
    {
        for (int j = 0; j < maxN; ++j) {
            std::vector<TiledArgs<FT>> args;
            std::vector<u64> prefix;
            std::vector<int> bid;
            u64 tiles = 0;
            for (const auto& m : mem) {
                if (ts[m.first]->nmode <= j) continue;
                TiledArgs<FT> a = make_args(m.first, j, m.second, plan_shape, st);
                if ((a.plan != nullptr) != (planned != 0)) continue;
                args.push_back(a);
                prefix.push_back(tiles);
                bid.push_back(m.first);
                tiles += args.back().ntiles;
            }
            prefix.push_back(tiles);
            count[j] = (int)args.size();
            total_tiles[j] = tiles;
            d_args[j] = nullptr;
            d_prefix[j] = nullptr;
            d_bid[j] = nullptr;
            if (args.empty()) continue;
            ALTOB_TRY(dmalloc_t(&d_args[j], args.size()));
            ALTOB_TRY(dmalloc_t(&d_prefix[j], prefix.size()));
            ALTOB_TRY(dmalloc_t(&d_bid[j], bid.size()));
            ALTOB_CUDA(cudaMemcpyAsync(d_args[j], args.data(), args.size() * sizeof(TiledArgs<FT>),
                                       cudaMemcpyHostToDevice, st));
            ALTOB_CUDA(cudaMemcpyAsync(d_prefix[j], prefix.data(), prefix.size() * sizeof(u64),
                                       cudaMemcpyHostToDevice, st));
            ALTOB_CUDA(cudaMemcpyAsync(d_bid[j], bid.data(), bid.size() * sizeof(int), cudaMemcpyHostToDevice, st));
            ALTOB_CUDA(cudaStreamSynchronize(st));  // host vectors go out of scope
        }
        return ALTOB_OK;
    }

    // Whether a kernel shape has a planned form (static order, one vector
    // chunk per lane) and tile plans are on.
    static bool plan_shape(int nm, int vec, int ch)
    {
        return nm >= 3 && ch == 1 && vec == (int)(16 / sizeof(FT)) && env_int("ALTOB_PLAN", 1);
    }

    // Tables, shared memory and grid of the planned tiles of (nm, lanes).
    altob_status setup_planned(PlannedPart<FT>& pp, const std::vector<std::pair<int, int>>& mem, int nm,
                               altob_dtype vdt, int lpn, int vec, int ch, cudaStream_t st)
    {
        pp.free_args();
        if (!plan_shape(nm, vec, ch)) return ALTOB_OK;
        ALTOB_TRY(upload_tables(mem, 1, true, pp.d_args, pp.d_prefix, pp.d_bid, pp.total_tiles, pp.count, st));
        pp.smem = planned_batch_smem(nm, sizeof(FT));
        BatchTiles<FT> bt;
        memset(&bt, 0, sizeof(bt));
        int bps = 0;
        ALTOB_TRY(launch_mt(nm, vdt, bt, planned_cfg(pp, lpn, vec, ch, 0), st, &bps));
        if (bps < 1) return fail(ALTOB_ERR_UNSUPPORTED, "batched planned MTTKRP kernel does not fit on an SM");
        pp.gridx = (unsigned)(bps * num_sms());
        return ALTOB_OK;
    }

    static TiledCfg planned_cfg(const PlannedPart<FT>& pp, int lpn, int vec, int ch, unsigned gx)
    {
        TiledCfg c;
        c.lpn = lpn;
        c.vec = vec;
        c.ch = ch;
        c.phi = 0;
        c.grouped = 1;
        c.planned = 1;
        c.grid = dim3(gx);
        c.smem = pp.smem;
        return c;
    }

    altob_status mttkrp_planned(const PlannedPart<FT>& pp, int nm, altob_dtype vdt, int lpn, int vec, int ch, int j,
                                cudaStream_t st)
    {
        if (!pp.d_args[j] || pp.total_tiles[j] == 0) return ALTOB_OK;
        BatchTiles<FT> bt;
        memset(&bt, 0, sizeof(bt));
        bt.args = pp.d_args[j];
        bt.tile_prefix = pp.d_prefix[j];
        bt.bid = pp.d_bid[j];
        bt.active = d_active;
        bt.ntensors = pp.count[j];
        bt.total_tiles = pp.total_tiles[j];
        const unsigned gx = (unsigned)std::max<u64>(1, std::min<u64>(pp.total_tiles[j], pp.gridx));
        return launch_mt(nm, vdt, bt, planned_cfg(pp, lpn, vec, ch, gx), st, nullptr);
    }

    // Launch groups from the classes' current choices.
    altob_status rebuild_groups(cudaStream_t st)
    {
        drop_graph();
        for (auto& g : groups) g->free_args();
        groups.clear();
        std::map<std::string, std::vector<ClassRun<FT>*>> by;
        for (auto& c : classes) {
            char k[96];
            snprintf(k, sizeof(k), "%d/%d/%d/%d/%d", c->nm, (int)c->vdt, c->lpn, c->vec, c->ch);
            by[k].push_back(c.get());
        }
        for (auto& kv : by) {
            auto g = std::make_unique<LaunchGroup<FT>>();
            const ClassRun<FT>& c0 = *kv.second[0];
            g->nm = c0.nm;
            g->vdt = c0.vdt;
            g->lpn = c0.lpn;
            g->vec = c0.vec;
            g->ch = c0.ch;
            std::vector<std::pair<int, int>> mem;
            for (ClassRun<FT>* c : kv.second) {
                g->hmax = std::max(g->hmax, c->hslots);
                for (int b : c->members) mem.push_back({b, c->hslots});
            }
            g->smem = grouped_smem(g->hmax, g->nm ? g->nm : ALTOB_MAX_MODES, sizeof(FT));
            const bool ps = plan_shape(g->nm, g->vec, g->ch);
            ALTOB_TRY(upload_tables(mem, 0, ps, g->d_args, g->d_prefix, g->d_bid, g->total_tiles, g->count, st));
            ALTOB_TRY(setup_planned(g->pp, mem, g->nm, g->vdt, g->lpn, g->vec, g->ch, st));
            BatchTiles<FT> bt;
            memset(&bt, 0, sizeof(bt));
            bt.hslots = g->hmax;
            int bps = 0;
            ALTOB_TRY(launch_mt(g->nm, g->vdt, bt, g->cfg(0), st, &bps));
            if (bps < 1) return fail(ALTOB_ERR_UNSUPPORTED, "batched MTTKRP kernel does not fit on an SM");
            g->gridx = (unsigned)(bps * num_sms());
            groups.push_back(std::move(g));
        }
        return ALTOB_OK;
    }

    altob_status mttkrp_group(LaunchGroup<FT>& g, int j, cudaStream_t st)
    {
        ALTOB_TRY(mttkrp_planned(g.pp, g.nm, g.vdt, g.lpn, g.vec, g.ch, j, st));
        if (!g.d_args[j] || g.total_tiles[j] == 0) return ALTOB_OK;
        BatchTiles<FT> bt;
        bt.args = g.d_args[j];
        bt.tile_prefix = g.d_prefix[j];
        bt.bid = g.d_bid[j];
        bt.active = d_active;
        bt.ntensors = g.count[j];
        bt.hslots = g.hmax;
        bt.total_tiles = g.total_tiles[j];
        const unsigned gx = (unsigned)std::max<u64>(1, std::min<u64>(g.total_tiles[j], g.gridx));
        return launch_mt(g.nm, g.vdt, bt, g.cfg(gx), st, nullptr);
    }

    // Per-mode argument tables of a class for its current slot count.
    altob_status build_class_args(ClassRun<FT>& c, cudaStream_t st)
    {
        c.free_args();
        std::vector<std::pair<int, int>> mem;
        for (int b : c.members) mem.push_back({b, c.hslots});
        ALTOB_TRY(upload_tables(mem, 0, plan_shape(c.nm, c.vec, c.ch), c.d_args, c.d_prefix, c.d_bid,
                                c.total_tiles, c.mode_count, st));
        return setup_planned(c.pp, mem, c.nm, c.vdt, c.lpn, c.vec, c.ch, st);
    }

    // slot count and lane layout of a class -> argument tables and grid
    altob_status set_choice(ClassRun<FT>& c, int hslots, int lpn, int ch, cudaStream_t st)
    {
        c.hslots = hslots;
        c.lpn = lpn;
        c.ch = ch;
        c.smem = grouped_smem(hslots, c.nm ? c.nm : ALTOB_MAX_MODES, sizeof(FT));
        ALTOB_TRY(build_class_args(c, st));
        BatchTiles<FT> bt;
        memset(&bt, 0, sizeof(bt));
        bt.hslots = hslots;
        int bps = 0;
        ALTOB_TRY(launch_mt(c, bt, c.cfg(0), st, &bps));  // sets the smem limit, reports occupancy
        if (bps < 1) return fail(ALTOB_ERR_UNSUPPORTED, "batched MTTKRP kernel does not fit on an SM");
        c.gridx = (unsigned)(bps * num_sms());
        return ALTOB_OK;
    }

    altob_status mttkrp_class(ClassRun<FT>& c, int j, cudaStream_t st)
    {
        ALTOB_TRY(mttkrp_planned(c.pp, c.nm, c.vdt, c.lpn, c.vec, c.ch, j, st));
        if (!c.d_args[j] || c.total_tiles[j] == 0) return ALTOB_OK;
        BatchTiles<FT> bt;
        bt.args = c.d_args[j];
        bt.tile_prefix = c.d_prefix[j];
        bt.bid = c.d_bid[j];
        bt.active = d_active;
        bt.ntensors = c.mode_count[j];
        bt.hslots = c.hslots;
        bt.total_tiles = c.total_tiles[j];
        const unsigned gx = (unsigned)std::max<u64>(1, std::min<u64>(c.total_tiles[j], c.gridx));
        return launch_mt(c, bt, c.cfg(gx), st, nullptr);
    }

    size_t smem_solve() const { return (size_t)2 * maxR * maxR * sizeof(double); }
    static size_t smem_apply(int R) { return (size_t)(R * R + R) * sizeof(double); }
    static size_t smem_gram(int R) { return (size_t)(GR_ELEMS + 2 * R) * sizeof(double); }

    // fused row update + Gram of mode j for the rank classes up to 64
    void launch_apply_gram(int j, int nk, cudaStream_t st)
    {
        for (int c = 0; c < NRANK_CLASSES; ++c) {
            if (!ncl[j][c] || !fused_class(c)) continue;
            const BlkMap m = {d_clist[j][c], d_rowpre[j][c], ncl[j][c]};
            const int g = nrowblk[j][c];
            switch (c) {
            case 0: k_b_apply_gram<FT, 1><<<g, AG_THREADS, apply_gram_smem<1>(), st>>>(d_desc, m, d_active, j, nk); break;
            case 1: k_b_apply_gram<FT, 2><<<g, AG_THREADS, apply_gram_smem<2>(), st>>>(d_desc, m, d_active, j, nk); break;
            case 2: k_b_apply_gram<FT, 4><<<g, AG_THREADS, apply_gram_smem<4>(), st>>>(d_desc, m, d_active, j, nk); break;
            default: k_b_apply_gram<FT, 8><<<g, AG_THREADS, apply_gram_smem<8>(), st>>>(d_desc, m, d_active, j, nk); break;
            }
        }
    }
    // U_j /= lambda for the fused rank classes (after k_b_lambda)
    void launch_div_cols(int j, cudaStream_t st)
    {
        for (int c = 0; c < NRANK_CLASSES; ++c) {
            if (!ncl[j][c] || !fused_class(c)) continue;
            const BlkMap m = {d_clist[j][c], d_rowpre[j][c], ncl[j][c]};
            k_b_div_cols<FT><<<nrowblk[j][c], DN_THREADS, cmaxR[c] * sizeof(double), st>>>(d_desc, m, d_active, j);
        }
    }
    static bool fused_class(int c) { return c <= 3; }  // rank classes up to R = 64
    // row kernels of mode j for the rank classes above 64, one launch per class
    void launch_apply(int j, int nk, cudaStream_t st)
    {
        for (int c = 0; c < NRANK_CLASSES; ++c) {
            if (!ncl[j][c] || fused_class(c)) continue;
            const BlkMap m = {d_clist[j][c], d_rowpre[j][c], ncl[j][c]};
            const size_t sm = smem_apply(cmaxR[c]);
            const int g = nrowblk[j][c];
            switch (c) {
            case 0: k_b_apply<FT, 8, 1><<<g, DN_THREADS, sm, st>>>(d_desc, m, d_active, j, nk); break;
            case 1: k_b_apply<FT, 16, 1><<<g, DN_THREADS, sm, st>>>(d_desc, m, d_active, j, nk); break;
            case 2: k_b_apply<FT, 32, 1><<<g, DN_THREADS, sm, st>>>(d_desc, m, d_active, j, nk); break;
            case 3: k_b_apply<FT, 32, 2><<<g, DN_THREADS, sm, st>>>(d_desc, m, d_active, j, nk); break;
            default: k_b_apply<FT, 32, 4><<<g, DN_THREADS, sm, st>>>(d_desc, m, d_active, j, nk); break;
            }
        }
    }
    void launch_gram(int j, int scaled, cudaStream_t st)
    {
        for (int c = 0; c < NRANK_CLASSES; ++c) {
            if (!ncl[j][c] || (scaled && fused_class(c))) continue;
            const BlkMap m = {d_clist[j][c], d_rowpre[j][c], ncl[j][c]};
            const size_t sm = smem_gram(cmaxR[c]);
            const int g = nrowblk[j][c];
            if (cmaxR[c] <= GR_SMALL) k_b_gram<FT, 1><<<g, DN_THREADS, sm, st>>>(d_desc, m, d_active, j, scaled);
            else k_b_gram<FT, 3><<<g, DN_THREADS, sm, st>>>(d_desc, m, d_active, j, scaled);
        }
    }
    int row_launches(int j) const
    {
        int n = 0;
        for (int c = 0; c < NRANK_CLASSES; ++c) n += ncl[j][c] ? 1 : 0;
        return n;
    }
    altob_status set_smem_limits()
    {
        const int big = (int)smem_apply(SOLVE_MAX_RANK), bigg = (int)smem_gram(SOLVE_MAX_RANK);
        ALTOB_CUDA(cudaFuncSetAttribute(k_b_solve<FT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)(2 * SOLVE_MAX_RANK * SOLVE_MAX_RANK * sizeof(double))));
        ALTOB_CUDA(cudaFuncSetAttribute(k_b_apply<FT, 32, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
        ALTOB_CUDA(cudaFuncSetAttribute(k_b_apply<FT, 32, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
        ALTOB_CUDA(cudaFuncSetAttribute(k_b_gram<FT, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bigg));
        ALTOB_CUDA(cudaFuncSetAttribute(k_b_gram<FT, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, bigg));
        return ALTOB_OK;
    }

    // one CP-ALS iteration over all active tensors (cpd.hpp:96-160 per tensor)
    altob_status iteration(int nk, double eps, int max_iters, cudaStream_t st)
    {
        int launches = 1;  // the fit
        for (int j = 0; j < maxN; ++j) {
            const int n = nlist[j];
            if (!n) continue;
            const int* L = d_list[j];
            const BlkMap els = {L, d_elpre[j], n};
            k_b_zero<FT><<<nelblk[j], 256, 0, st>>>(d_desc, els, d_active, j);
            // the launch groups of mode j are independent: spread them over
            // forked streams so one group's last wave overlaps the others
            ALTOB_CUDA(cudaEventRecord(fork_ev, st));
            int used = 0;
            for (size_t gi = 0; gi < groups.size(); ++gi) {
                LaunchGroup<FT>& g = *groups[gi];
                const int parts = (g.d_args[j] && g.total_tiles[j] ? 1 : 0) +
                                  (g.pp.d_args[j] && g.pp.total_tiles[j] ? 1 : 0);
                if (!parts) continue;
                cudaStream_t fs = fork_st[used % NFORK];
                if (used < NFORK) ALTOB_CUDA(cudaStreamWaitEvent(fs, fork_ev, 0));
                ALTOB_TRY(mttkrp_group(g, j, fs));
                ++used;
                launches += parts;
            }
            for (int i = 0; i < std::min(used, NFORK); ++i) {
                ALTOB_CUDA(cudaEventRecord(join_ev[i], fork_st[i]));
                ALTOB_CUDA(cudaStreamWaitEvent(st, join_ev[i], 0));
            }
            launches += 5 + 2 * row_launches(j);
            k_b_copym<FT><<<nelblk[j], 256, 0, st>>>(d_desc, els, d_active, j);
            k_b_prep<FT><<<n, 128, 0, st>>>(d_desc, L, d_active, j, nk);
            k_b_solve<FT><<<n, DN_THREADS, smem_solve(), st>>>(d_desc, L, d_active, j);
            launch_apply_gram(j, nk, st);
            launch_apply(j, nk, st);
            k_b_lambda<FT><<<n, 128, 0, st>>>(d_desc, L, d_active, nk, j);
            launch_div_cols(j, st);
            launch_gram(j, 1, st);
            ALTOB_LAUNCH_CHECK();
        }
        k_b_fit<FT><<<count, DN_THREADS, 0, st>>>(d_desc, d_active, d_iters, eps, max_iters);
        ALTOB_LAUNCH_CHECK();
        launches_per_iter = launches;
        return ALTOB_OK;
    }

    altob_status capture(double eps, int max_iters)
    {
        drop_graph();
        if (!cap_stream) ALTOB_CUDA(cudaStreamCreateWithPriority(&cap_stream, cudaStreamNonBlocking, prio));
        cudaGraph_t g = nullptr;
        ALTOB_CUDA(cudaStreamBeginCapture(cap_stream, cudaStreamCaptureModeThreadLocal));
        altob_status s = iteration(NORM_MAX, eps, max_iters, cap_stream);
        cudaError_t e = cudaStreamEndCapture(cap_stream, &g);
        if (s != ALTOB_OK) {
            if (g) cudaGraphDestroy(g);
            return s;
        }
        if (e != cudaSuccess) return fail(ALTOB_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&gexec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            gexec = nullptr;
            return fail(ALTOB_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        }
        g_eps = eps;
        g_iters = max_iters;
        return ALTOB_OK;
    }

    altob_status any_active(cudaStream_t st, bool* any)
    {
        std::vector<int> a(count);
        ALTOB_CUDA(cudaMemcpyAsync(a.data(), d_active, count * sizeof(int), cudaMemcpyDeviceToHost, st));
        ALTOB_CUDA(cudaStreamSynchronize(st));
        *any = std::any_of(a.begin(), a.end(), [](int v) { return v != 0; });
        return ALTOB_OK;
    }

    altob_status solve(int max_iters, double eps, double* fits, int* iters, int use_graph, cudaStream_t st) override
    {
        if (max_iters < 1 || max_iters > cap) return fail(ALTOB_ERR_ARG, "max_iters must be 1..fit capacity");
        ALTOB_TRY(set_smem_limits());
        // all tensors active, no fits yet; Grams of the initial factors
        std::vector<int> ones(count, 1);
        ALTOB_CUDA(cudaMemcpyAsync(d_active, ones.data(), count * sizeof(int), cudaMemcpyHostToDevice, st));
        ALTOB_CUDA(cudaMemsetAsync(d_iters, 0, count * sizeof(int), st));
        for (int j = 0; j < maxN; ++j) {
            if (!nlist[j]) continue;
            k_b_prep<FT><<<nlist[j], 128, 0, st>>>(d_desc, d_list[j], d_active, j, NORM_2);
            launch_gram(j, 0, st);
        }
        ALTOB_LAUNCH_CHECK();
        // the first iteration normalises with the 2-norm, later ones with the max-norm
        ALTOB_TRY(iteration(NORM_2, eps, max_iters, st));
        int done = 1;
        constexpr int CHUNK = 4;  // iterations between host checks for early exit
        if (use_graph && max_iters > 1 && (!gexec || g_eps != eps || g_iters != max_iters))
            ALTOB_TRY(capture(eps, max_iters));
        while (done < max_iters) {
            const int n = std::min(CHUNK, max_iters - done);
            for (int i = 0; i < n; ++i) {
                if (use_graph) ALTOB_CUDA(cudaGraphLaunch(gexec, st));
                else ALTOB_TRY(iteration(NORM_MAX, eps, max_iters, st));
            }
            done += n;
            if (done < max_iters) {
                bool any = true;
                ALTOB_TRY(any_active(st, &any));
                if (!any) break;
            }
        }
        k_b_lamout<FT><<<count, 128, 0, st>>>(d_desc, count);
        ALTOB_LAUNCH_CHECK();
        std::vector<int> hit(count);
        ALTOB_CUDA(cudaMemcpyAsync(hit.data(), d_iters, count * sizeof(int), cudaMemcpyDeviceToHost, st));
        std::vector<double> hf((size_t)count * cap);
        ALTOB_CUDA(cudaMemcpyAsync(hf.data(), hdesc[0].fits, hf.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        ALTOB_CUDA(cudaStreamSynchronize(st));
        for (int b = 0; b < count; ++b) {
            if (iters) iters[b] = hit[b];
            if (fits)
                for (int i = 0; i < max_iters; ++i)
                    fits[(size_t)b * max_iters + i] = i < hit[b] ? hf[(size_t)b * cap + i] : 0.0;
        }
        return ALTOB_OK;
    }

    // Autotuner: per shape class, times each candidate (slot count x lane
    // layout) on the class's MTTKRP of every mode and keeps the fastest.  The
    // target factors are saved before and restored after, so the model the
    // caller passed in is unchanged.
    std::string tune_key(const ClassRun<FT>& c) const { return std::to_string(sizeof(FT)) + "|" + c.key; }

    altob_status autotune(int force, cudaStream_t st) override
    {
        drop_graph();
        std::vector<int> ones(count, 1);
        ALTOB_CUDA(cudaMemcpyAsync(d_active, ones.data(), count * sizeof(int), cudaMemcpyHostToDevice, st));
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        ALTOB_CUDA(cudaEventCreate(&e0));
        ALTOB_CUDA(cudaEventCreate(&e1));
        altob_status s = ALTOB_OK;
        for (auto& cp : classes) {
            ClassRun<FT>& c = *cp;
            TuneChoice known;
            if (!force && tune_lookup(tune_key(c), &known)) continue;  // applied at creation
            // save the factors this class writes
            size_t bytes = 0;
            for (int b : c.members)
                for (int m = 0; m < ts[b]->nmode; ++m) bytes += ts[b]->dims[m] * hdesc[b].R * sizeof(FT);
            void* save = nullptr;
            s = dmalloc(&save, bytes);
            if (s != ALTOB_OK) break;
            size_t off = 0;
            for (int b : c.members)
                for (int m = 0; m < ts[b]->nmode; ++m) {
                    const size_t nb = ts[b]->dims[m] * hdesc[b].R * sizeof(FT);
                    cudaMemcpyAsync((char*)save + off, hdesc[b].U[m], nb, cudaMemcpyDeviceToDevice, st);
                    off += nb;
                }
            struct Cand {
                int hs, lpn, ch;
            };
            std::vector<Cand> cand;
            const int lpn0 = c.lpn, ch0 = c.ch;
            for (int hs : {0, 512, 1024, 2048, 4096}) {
                cand.push_back({hs, lpn0, ch0});
                if (ch0 == 1 && c.vec > 1 && lpn0 >= 8) cand.push_back({hs, lpn0 / 2, 2});
            }
            Cand best = {c.hslots, lpn0, ch0};
            float best_ms = 1e30f;
            for (const Cand& k : cand) {
                if (set_choice(c, k.hs, k.lpn, k.ch, st) != ALTOB_OK) continue;
                float t_best = 1e30f;
                bool ok = true;
                for (int rep = 0; rep < 3 && ok; ++rep) {
                    cudaEventRecord(e0, st);
                    for (int j = 0; j < maxN && ok; ++j) ok = mttkrp_class(c, j, st) == ALTOB_OK;
                    cudaEventRecord(e1, st);
                    if (cudaEventSynchronize(e1) != cudaSuccess) ok = false;
                    float ms = 0.f;
                    cudaEventElapsedTime(&ms, e0, e1);
                    if (rep > 0) t_best = std::min(t_best, ms);  // first run warms up
                }
                if (ok && t_best < best_ms) {
                    best_ms = t_best;
                    best = k;
                }
            }
            off = 0;
            for (int b : c.members)
                for (int m = 0; m < ts[b]->nmode; ++m) {
                    const size_t nb = ts[b]->dims[m] * hdesc[b].R * sizeof(FT);
                    cudaMemcpyAsync(hdesc[b].U[m], (char*)save + off, nb, cudaMemcpyDeviceToDevice, st);
                    off += nb;
                }
            dfree(save);
            s = set_choice(c, best.hs, best.lpn, best.ch, st);
            if (s != ALTOB_OK) break;
            c.tuned_ms = best_ms;
            tune_store(tune_key(c), {best.hs, best.lpn, best.ch, best_ms});
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        ALTOB_CUDA(cudaGetLastError());
        if (s == ALTOB_OK) s = rebuild_groups(st);
        ALTOB_CUDA(cudaStreamSynchronize(st));
        return s;
    }

    void describe(std::string* out) const override
    {
        char line[320];
        snprintf(line, sizeof(line),
                 "tensors=%d classes=%zu launch_groups=%zu max_modes=%d max_rank=%d launches_per_iteration=%d\n",
                 count, classes.size(), groups.size(), maxN, maxR, launches_per_iter);
        *out += line;
        for (auto& c : classes) {
            snprintf(line, sizeof(line), "class %s: tensors=%zu slots=%d lanes=%d chunks=%d tuned_ms=%.4f\n",
                     c->key.c_str(), c->members.size(), c->hslots, c->lpn, c->ch, c->tuned_ms);
            *out += line;
        }
    }

    altob_status create(altob_tensor* const* tensors, int n, const uint64_t* ranks, void* const* const* dU,
                        void* const* dlam, int fit_cap, cudaStream_t st)
    {
        count = n;
        cap = fit_cap;
        ts.assign(tensors, tensors + n);
        hdesc.resize(n);
        // per-tensor FP64 block (Grams, W, colacc, lambda, inner, fit) and the
        // saved MTTKRP of the last mode, then the fit history and info
        auto dbl_block = [](int N, int R) {
            const size_t nd = (size_t)N * R * R + (size_t)R * R + 3 * (size_t)R + 2;
            return (nd * 8 + 255) & ~(size_t)255;
        };
        size_t total = 0;
        std::vector<size_t> off(n);
        for (int b = 0; b < n; ++b) {
            altob_tensor* t = ts[b];
            const int R = (int)ranks[b];
            maxN = std::max(maxN, t->nmode);
            maxR = std::max(maxR, R);
            off[b] = total;
            total += dbl_block(t->nmode, R);
            total += (t->dims[t->nmode - 1] * R * sizeof(FT) + 255) & ~(size_t)255;
        }
        const size_t fits_off = total;
        total += ((size_t)n * cap * 8 + 255) & ~(size_t)255;
        const size_t info_off = total;
        total += 256;
        ALTOB_TRY(dmalloc(&d_scratch, total));
        char* base = (char*)d_scratch;
        ALTOB_CUDA(cudaMemsetAsync(base + info_off, 0, 256, st));
        std::vector<const void*> hv(n);
        std::vector<u64> hnnz(n);
        for (int b = 0; b < n; ++b) {
            altob_tensor* t = ts[b];
            BDesc<FT>& d = hdesc[b];
            memset(&d, 0, sizeof(d));
            const int R = (int)ranks[b];
            d.nmode = t->nmode;
            d.R = R;
            for (int m = 0; m < t->nmode; ++m) {
                d.U[m] = (FT*)dU[b][m];
                d.dims[m] = t->dims[m];
            }
            double* p = (double*)(base + off[b]);
            d.G = p;
            p += (size_t)t->nmode * R * R;
            d.W = p;
            p += (size_t)R * R;
            d.colacc = p;
            p += R;
            d.lam = p;
            p += R;
            d.inner = p;
            p += R;
            d.fit_tmp = p;
            d.M = (FT*)(base + off[b] + dbl_block(t->nmode, R));
            d.fits = (double*)(base + fits_off) + (size_t)b * cap;
            d.lam_out = dlam ? (FT*)dlam[b] : nullptr;
            d.normAT = 0.0;
            d.info = (int*)(base + info_off);
            hv[b] = t->d_vals;
            hnnz[b] = t->nnz;
        }
        ALTOB_TRY(dmalloc_t(&d_desc, n));
        ALTOB_TRY(dmalloc_t(&d_active, n));
        ALTOB_TRY(dmalloc_t(&d_iters, n));
        ALTOB_CUDA(cudaMemcpyAsync(d_desc, hdesc.data(), n * sizeof(BDesc<FT>), cudaMemcpyHostToDevice, st));
        // squared norm of every tensor's values (cpd.hpp:73-79)
        {
            const void** d_vals = nullptr;
            u64* d_nnz = nullptr;
            ALTOB_TRY(dmalloc_t(&d_vals, n));
            ALTOB_TRY(dmalloc_t(&d_nnz, n));
            ALTOB_CUDA(cudaMemcpyAsync(d_vals, hv.data(), n * sizeof(void*), cudaMemcpyHostToDevice, st));
            ALTOB_CUDA(cudaMemcpyAsync(d_nnz, hnnz.data(), n * sizeof(u64), cudaMemcpyHostToDevice, st));
            if (ts[0]->vdt == ALTOB_U32)
                k_b_sumsq<FT, u32><<<dim3(64, n), 256, 0, st>>>(d_desc, (const void* const*)d_vals, d_nnz);
            else
                k_b_sumsq<FT, FT><<<dim3(64, n), 256, 0, st>>>(d_desc, (const void* const*)d_vals, d_nnz);
            ALTOB_LAUNCH_CHECK();
            ALTOB_CUDA(cudaStreamSynchronize(st));
            dfree((void*)d_vals);
            dfree(d_nnz);
        }
        // per-mode lists of the tensors that have that mode, element-block
        // maps, and per rank class the row-block maps
        for (int b = 0; b < n; ++b) {
            const int c = rank_class(hdesc[b].R);
            cmaxR[c] = std::max(cmaxR[c], hdesc[b].R);
        }
        for (int j = 0; j < maxN; ++j) {
            std::vector<int> L, ep(1, 0);
            std::vector<int> CL[NRANK_CLASSES], RP[NRANK_CLASSES];
            for (int c = 0; c < NRANK_CLASSES; ++c) RP[c].push_back(0);
            for (int b = 0; b < n; ++b)
                if (ts[b]->nmode > j) {
                    L.push_back(b);
                    const u64 I = ts[b]->dims[j], R = (u64)hdesc[b].R;
                    const u64 rb = std::min<u64>(MAX_CTAS_PER_TENSOR, std::max<u64>(1, (I + ROWS_PER_CTA - 1) / ROWS_PER_CTA));
                    const u64 eb = std::min<u64>(MAX_CTAS_PER_TENSOR,
                                                 std::max<u64>(1, (I * R + ELEMS_PER_CTA - 1) / ELEMS_PER_CTA));
                    ep.push_back(ep.back() + (int)eb);
                    const int c = rank_class((int)R);
                    CL[c].push_back(b);
                    RP[c].push_back(RP[c].back() + (int)rb);
                }
            nlist[j] = (int)L.size();
            if (L.empty()) continue;
            nelblk[j] = ep.back();
            ALTOB_TRY(dmalloc_t(&d_list[j], L.size()));
            ALTOB_TRY(dmalloc_t(&d_elpre[j], ep.size()));
            ALTOB_CUDA(cudaMemcpyAsync(d_list[j], L.data(), L.size() * sizeof(int), cudaMemcpyHostToDevice, st));
            ALTOB_CUDA(cudaMemcpyAsync(d_elpre[j], ep.data(), ep.size() * sizeof(int), cudaMemcpyHostToDevice, st));
            for (int c = 0; c < NRANK_CLASSES; ++c) {
                ncl[j][c] = (int)CL[c].size();
                if (CL[c].empty()) continue;
                nrowblk[j][c] = RP[c].back();
                ALTOB_TRY(dmalloc_t(&d_clist[j][c], CL[c].size()));
                ALTOB_TRY(dmalloc_t(&d_rowpre[j][c], RP[c].size()));
                ALTOB_CUDA(cudaMemcpyAsync(d_clist[j][c], CL[c].data(), CL[c].size() * sizeof(int),
                                           cudaMemcpyHostToDevice, st));
                ALTOB_CUDA(cudaMemcpyAsync(d_rowpre[j][c], RP[c].data(), RP[c].size() * sizeof(int),
                                           cudaMemcpyHostToDevice, st));
            }
            ALTOB_CUDA(cudaStreamSynchronize(st));
        }
        // shape classes: (order, lanes, elements per lane, chunks, nnz decade,
        // low-reuse flag) -- ALTOB_BATCH_CLASS_NNZ=0 drops the last two
        const char* cn = getenv("ALTOB_BATCH_CLASS_NNZ");
        const bool by_nnz = !(cn && atoi(cn) == 0);
        std::map<std::string, ClassRun<FT>*> byk;
        for (int b = 0; b < n; ++b) {
            altob_tensor* t = ts[b];
            bool aligned = true;
            for (int m = 0; m < t->nmode; ++m) aligned = aligned && ptr_aligned16(hdesc[b].U[m]);
            TiledPlan pl;
            ALTOB_TRY(plan_tiled(t, (u64)hdesc[b].R, sizeof(FT), aligned, true, &pl));
            const int nm = t->nmode >= 3 ? t->nmode : 0;
            char k[128];
            snprintf(k, sizeof(k), "order=%d lanes=%d vec=%d chunks=%d", t->nmode, pl.lpn, pl.vec,
                     pl.ch);
            if (by_nnz) {
                bool low = false;
                for (int m = 0; m < t->nmode; ++m) low = low || (fib_reuse(t, m) <= 4 && t->d_oidx[m]);
                const int dec = t->nnz < 100000 ? 4 : t->nnz < 1000000 ? 5 : 6;
                const size_t l = strlen(k);
                snprintf(k + l, sizeof(k) - l, " nnz=1e%d%s", dec, low ? " low-reuse" : "");
            }
            auto it = byk.find(k);
            if (it == byk.end()) {
                auto c = std::make_unique<ClassRun<FT>>();
                c->nm = nm;
                c->vdt = t->vdt;
                c->key = k;
                c->lpn = pl.lpn;
                c->vec = pl.vec;
                c->ch = pl.ch;
                c->hslots = 2048;
                it = byk.emplace(k, c.get()).first;
                classes.push_back(std::move(c));
            }
            it->second->members.push_back(b);
        }
        for (auto& c : classes) {
            TuneChoice known;
            if (tune_lookup(tune_key(*c), &known)) {
                c->tuned_ms = known.ms;
                ALTOB_TRY(set_choice(*c, known.hslots, known.lpn, known.ch, st));
            } else {
                ALTOB_TRY(set_choice(*c, c->hslots, c->lpn, c->ch, st));
            }
        }
        ALTOB_TRY(rebuild_groups(st));
        // the internal streams take the priority of the caller's stream (a
        // server runs short batched solves at a higher priority than long
        // CP-APR requests)
        if (cudaStreamGetPriority(st, &prio) != cudaSuccess) {
            cudaGetLastError();
            prio = 0;
        }
        for (int i = 0; i < NFORK; ++i) {
            ALTOB_CUDA(cudaStreamCreateWithPriority(&fork_st[i], cudaStreamNonBlocking, prio));
            ALTOB_CUDA(cudaEventCreateWithFlags(&join_ev[i], cudaEventDisableTiming));
        }
        ALTOB_CUDA(cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming));
        ALTOB_CUDA(cudaStreamSynchronize(st));
        return ALTOB_OK;
    }
};

}  // namespace altob

struct altob_batch {
    std::unique_ptr<altob::BatchBase> impl;
};

using namespace altob;

extern "C" {

altob_status altob_batch_create(altob_tensor* const* tensors, int count, const uint64_t* ranks, altob_dtype ftype,
                                void* const* const* d_factors, void* const* d_lambda, int fit_capacity, void* stream,
                                altob_batch** out)
{
    if (!out) return fail(ALTOB_ERR_ARG, "NULL output handle");
    *out = nullptr;
    if (!tensors || !ranks || !d_factors || count < 1) return fail(ALTOB_ERR_ARG, "NULL or empty argument");
    if (count > 65535) return fail(ALTOB_ERR_UNSUPPORTED, "more than 65535 tensors in one batch");
    if (ftype != ALTOB_F64 && ftype != ALTOB_F32) return fail(ALTOB_ERR_ARG, "dtype must be F64 or F32");
    if (fit_capacity < 1) return fail(ALTOB_ERR_ARG, "fit capacity must be >= 1");
    for (int b = 0; b < count; ++b) {
        altob_tensor* t = tensors[b];
        if (!t || !d_factors[b]) return fail(ALTOB_ERR_ARG, "NULL tensor or factor list");
        ALTOB_TRY(check_model(t, ftype, d_factors[b], ranks[b]));
        if (t->nmode < 2) return fail(ALTOB_ERR_ARG, "CP-ALS needs at least two modes");
        if (t->nnz == 0) return fail(ALTOB_ERR_ARG, "CP-ALS on an empty tensor (the fit divides by its norm)");
        if (t->vdt != tensors[0]->vdt) return fail(ALTOB_ERR_ARG, "all tensors of a batch need one value dtype");
    }
    cudaStream_t st = (cudaStream_t)stream;
    StreamScope scope(st);
    std::unique_ptr<altob_batch> bh(new altob_batch());
    altob_status s;
    if (ftype == ALTOB_F64) {
        auto* impl = new BatchImpl<double>();
        bh->impl.reset(impl);
        s = impl->create(tensors, count, ranks, d_factors, d_lambda, fit_capacity, st);
    } else {
        auto* impl = new BatchImpl<float>();
        bh->impl.reset(impl);
        s = impl->create(tensors, count, ranks, d_factors, d_lambda, fit_capacity, st);
    }
    if (s != ALTOB_OK) return s;
    *out = bh.release();
    return ALTOB_OK;
}

altob_status altob_batch_autotune(altob_batch* b, int force, void* stream)
{
    if (!b) return fail(ALTOB_ERR_ARG, "NULL batch");
    StreamScope scope((cudaStream_t)stream);
    return b->impl->autotune(force, (cudaStream_t)stream);
}

altob_status altob_batch_cpd_als(altob_batch* b, int max_iters, double epsilon, double* fits, int* iters,
                                 int use_graph, void* stream)
{
    if (!b) return fail(ALTOB_ERR_ARG, "NULL batch");
    StreamScope scope((cudaStream_t)stream);
    return b->impl->solve(max_iters, epsilon, fits, iters, use_graph, (cudaStream_t)stream);
}

altob_status altob_batch_describe(const altob_batch* b, char* buf, size_t len)
{
    if (!b || !buf || !len) return fail(ALTOB_ERR_ARG, "NULL argument");
    std::string s;
    b->impl->describe(&s);
    const size_t n = std::min(len - 1, s.size());
    memcpy(buf, s.data(), n);
    buf[n] = 0;
    return ALTOB_OK;
}

altob_status altob_batch_destroy(altob_batch* b)
{
    // every call on a handle returns with its work finished, so the memory
    // is released without waiting for the device
    if (!b) return ALTOB_OK;
    delete b;
    return ALTOB_OK;
}

}  // extern "C"
