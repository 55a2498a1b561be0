// mttkrp_launch.cuh -- typed launchers for the MTTKRP / Phi kernels.  Each
// (FT, VT) pair is instantiated in its own translation unit
// (mttkrp_<ft>_<vt>.cu) so the kernels compile in parallel.
#pragma once

#include <atomic>

#include "mttkrp_tma.cuh"

namespace altob {

struct TiledCfg {
    int lpn = 32, vec = 1, ch = 4, phi = 0;
    int grouped = 1;  // 1: k_grouped, 0: k_tiled
    int pre = 0;      // Phi from precomputed Khatri-Rao rows (grouped only)
    int planned = 0;  // batched MTTKRP: tiles with a tile plan
    dim3 grid;
    size_t smem = 0;
};

template <typename FT, typename VT>
altob_status launch_tiled(const TiledArgs<FT>& a, const TiledCfg& c, cudaStream_t st, int* max_blocks_per_sm);

template <typename FT, typename VT>
altob_status launch_atomic_cr(const CrArgsK<FT>& a, cudaStream_t st);

// Planned MTTKRP (static order 3-5, one VEC-wide chunk per lane, a.plan set).
template <typename FT, typename VT>
altob_status launch_planned(const TiledArgs<FT>& a, const TiledCfg& c, cudaStream_t st, int* bps);

// Batched grouped MTTKRP over the tensors of one shape class (nm = order 3-5, or 0).
template <typename FT, typename VT>
altob_status launch_batch(const BatchTiles<FT>& bt, int nm, const TiledCfg& c, cudaStream_t st, int* bps);

// Sets the kernel's shared-memory limit once and launches it (or only
// reports occupancy when grid.x == 0).
template <typename K>
altob_status launch_kernel(K k, std::atomic<size_t>& configured, const void* args_ptr, const TiledCfg& c,
                           cudaStream_t st, int* bps)
{
    if (c.smem > configured.load()) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c.smem);
        if (e != cudaSuccess) return fail(ALTOB_ERR_CUDA, std::string("smem attribute: ") + cudaGetErrorString(e));
        size_t cur = configured.load();
        while (cur < c.smem && !configured.compare_exchange_weak(cur, c.smem)) {
        }
    }
    if (bps) {
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, MT_THREADS, c.smem);
        *bps = n;
    }
    if (c.grid.x == 0) return ALTOB_OK;
    void* args[] = {const_cast<void*>(args_ptr)};
    cudaError_t e = cudaLaunchKernel((const void*)k, c.grid, dim3(MT_THREADS), args, c.smem, st);
    if (e != cudaSuccess) return fail(ALTOB_ERR_CUDA, std::string("MTTKRP launch: ") + cudaGetErrorString(e));
    return ALTOB_OK;
}

template <typename FT, typename VT, int NM, int LPN, int VEC, int CH, bool PHI>
altob_status launch_grouped(const TiledArgs<FT>& a, const TiledCfg& c, cudaStream_t st, int* bps)
{
    static std::atomic<size_t> configured{0};
    constexpr int mb = grouped_min_blocks<FT, NM, CH, PHI>();
    if constexpr (mb > 0)
        return launch_kernel(k_grouped_mb<FT, VT, NM, LPN, VEC, CH, PHI, mb>, configured, &a, c, st, bps);
    else
        return launch_kernel(k_grouped<FT, VT, NM, LPN, VEC, CH, PHI>, configured, &a, c, st, bps);
}

template <typename FT, typename VT, int NM, int LPN, int VEC, int CH, bool PHI>
altob_status launch_one(const TiledArgs<FT>& a, const TiledCfg& c, cudaStream_t st, int* bps)
{
    if (c.grouped) return launch_grouped<FT, VT, NM, LPN, VEC, CH, PHI>(a, c, st, bps);
    // k_tiled is built for order 3 and the generic order only
    if constexpr (NM == 1) {
        return fail(ALTOB_ERR_UNSUPPORTED, "precomputed rows need the grouped kernel");
    } else if constexpr (NM == 4 || NM == 5) {
        return launch_one<FT, VT, 0, LPN, VEC, CH, PHI>(a, c, st, bps);
    } else {
        static std::atomic<size_t> configured{0};
        return launch_kernel(k_tiled<FT, VT, NM, LPN, VEC, CH, PHI>, configured, &a, c, st, bps);
    }
}

// (lanes per nonzero, elements per lane, chunks) -> kernel
template <typename FT, typename VT, int NM, bool PHI>
altob_status launch_shape(const TiledArgs<FT>& a, const TiledCfg& c, cudaStream_t st, int* bps)
{
    constexpr int V = 16 / sizeof(FT);
    if (c.vec == 1) return launch_one<FT, VT, NM, 32, 1, 4, PHI>(a, c, st, bps);
    if (c.ch == 2) {
        if (c.lpn == 32) return launch_one<FT, VT, NM, 32, V, 2, PHI>(a, c, st, bps);
        if (!c.grouped) return fail(ALTOB_ERR_UNSUPPORTED, "shape needs the grouped kernel");
        switch (c.lpn) {
        case 4: return launch_grouped<FT, VT, NM, 4, V, 2, PHI>(a, c, st, bps);
        case 8: return launch_grouped<FT, VT, NM, 8, V, 2, PHI>(a, c, st, bps);
        case 16: return launch_grouped<FT, VT, NM, 16, V, 2, PHI>(a, c, st, bps);
        }
        return fail(ALTOB_ERR_UNSUPPORTED, "lanes per nonzero");
    }
    switch (c.lpn) {
    case 2: return launch_one<FT, VT, NM, 2, V, 1, PHI>(a, c, st, bps);
    case 4: return launch_one<FT, VT, NM, 4, V, 1, PHI>(a, c, st, bps);
    case 8: return launch_one<FT, VT, NM, 8, V, 1, PHI>(a, c, st, bps);
    case 16: return launch_one<FT, VT, NM, 16, V, 1, PHI>(a, c, st, bps);
    case 32: return launch_one<FT, VT, NM, 32, V, 1, PHI>(a, c, st, bps);
    }
    return fail(ALTOB_ERR_UNSUPPORTED, "lanes per nonzero");
}

template <typename FT, typename VT, int NM, int LPN, int V>
altob_status launch_planned_one(const TiledArgs<FT>& a, const TiledCfg& c, cudaStream_t st, int* bps)
{
    static std::atomic<size_t> configured{0};
    constexpr int mb = planned_min_blocks<FT, NM, LPN>();
    if constexpr (mb > 0)
        return launch_kernel(k_planned_mb<FT, VT, NM, LPN, V, mb, PT_TILE, planned_nbuf<FT, NM>()>, configured, &a, c, st,
                             bps);
    else
        return launch_kernel(k_planned<FT, VT, NM, LPN, V>, configured, &a, c, st, bps);
}

template <typename FT, typename VT, int NM>
altob_status launch_planned_shape(const TiledArgs<FT>& a, const TiledCfg& c, cudaStream_t st, int* bps)
{
    constexpr int V = 16 / sizeof(FT);
    if (c.ch != 1) return fail(ALTOB_ERR_UNSUPPORTED, "planned kernel shape");
    if (c.vec != V) return fail(ALTOB_ERR_UNSUPPORTED, "planned kernel shape");
    switch (c.lpn) {
    case 2: return launch_planned_one<FT, VT, NM, 2, V>(a, c, st, bps);
    case 4: return launch_planned_one<FT, VT, NM, 4, V>(a, c, st, bps);
    case 8: return launch_planned_one<FT, VT, NM, 8, V>(a, c, st, bps);
    case 16: return launch_planned_one<FT, VT, NM, 16, V>(a, c, st, bps);
    case 32: return launch_planned_one<FT, VT, NM, 32, V>(a, c, st, bps);
    }
    return fail(ALTOB_ERR_UNSUPPORTED, "lanes per nonzero");
}

template <typename FT, typename VT, int NM, int LPN, int VEC, int CH>
altob_status launch_batch_one(const BatchTiles<FT>& bt, const TiledCfg& c, cudaStream_t st, int* bps)
{
    static std::atomic<size_t> configured{0};
    constexpr int mb = grouped_min_blocks<FT, NM, CH, false>();
    if constexpr (mb > 0)
        return launch_kernel(k_grouped_batch_mb<FT, VT, NM, LPN, VEC, CH, false, mb>, configured, &bt, c, st, bps);
    else
        return launch_kernel(k_grouped_batch<FT, VT, NM, LPN, VEC, CH, false>, configured, &bt, c, st, bps);
}

template <typename FT, typename VT, int NM, int LPN>
altob_status launch_planned_batch_one(const BatchTiles<FT>& bt, const TiledCfg& c, cudaStream_t st, int* bps)
{
    static std::atomic<size_t> configured{0};
    constexpr int V = 16 / sizeof(FT);
    constexpr int mb = planned_min_blocks<FT, NM, LPN>();
    if constexpr (mb > 0)
        return launch_kernel(k_planned_batch_mb<FT, VT, NM, LPN, V, mb>, configured, &bt, c, st, bps);
    else
        return launch_kernel(k_planned_batch<FT, VT, NM, LPN, V>, configured, &bt, c, st, bps);
}

template <typename FT, typename VT, int NM>
altob_status launch_batch_shape(const BatchTiles<FT>& bt, const TiledCfg& c, cudaStream_t st, int* bps)
{
    constexpr int V = 16 / sizeof(FT);
    if (c.planned) {
        if constexpr (NM >= 3) {
            if (c.vec != V || c.ch != 1) return fail(ALTOB_ERR_UNSUPPORTED, "planned batch shape");
            switch (c.lpn) {
            case 2: return launch_planned_batch_one<FT, VT, NM, 2>(bt, c, st, bps);
            case 4: return launch_planned_batch_one<FT, VT, NM, 4>(bt, c, st, bps);
            case 8: return launch_planned_batch_one<FT, VT, NM, 8>(bt, c, st, bps);
            case 16: return launch_planned_batch_one<FT, VT, NM, 16>(bt, c, st, bps);
            case 32: return launch_planned_batch_one<FT, VT, NM, 32>(bt, c, st, bps);
            }
        }
        return fail(ALTOB_ERR_UNSUPPORTED, "planned batch shape");
    }
    if (c.vec == 1) return launch_batch_one<FT, VT, NM, 32, 1, 4>(bt, c, st, bps);
    if (c.ch == 2) {
        switch (c.lpn) {
        case 4: return launch_batch_one<FT, VT, NM, 4, V, 2>(bt, c, st, bps);
        case 8: return launch_batch_one<FT, VT, NM, 8, V, 2>(bt, c, st, bps);
        case 16: return launch_batch_one<FT, VT, NM, 16, V, 2>(bt, c, st, bps);
        case 32: return launch_batch_one<FT, VT, NM, 32, V, 2>(bt, c, st, bps);
        }
        return fail(ALTOB_ERR_UNSUPPORTED, "lanes per nonzero");
    }
    switch (c.lpn) {
    case 2: return launch_batch_one<FT, VT, NM, 2, V, 1>(bt, c, st, bps);
    case 4: return launch_batch_one<FT, VT, NM, 4, V, 1>(bt, c, st, bps);
    case 8: return launch_batch_one<FT, VT, NM, 8, V, 1>(bt, c, st, bps);
    case 16: return launch_batch_one<FT, VT, NM, 16, V, 1>(bt, c, st, bps);
    case 32: return launch_batch_one<FT, VT, NM, 32, V, 1>(bt, c, st, bps);
    }
    return fail(ALTOB_ERR_UNSUPPORTED, "lanes per nonzero");
}

#define ALTOB_INSTANTIATE_MTTKRP(FT, VT)                                                                 \
    template <>                                                                                        \
    altob_status launch_tiled<FT, VT>(const TiledArgs<FT>& a, const TiledCfg& c, cudaStream_t st,      \
                                      int* bps)                                                        \
    {                                                                                                  \
        if (c.pre) return launch_shape<FT, VT, 1, true>(a, c, st, bps);                                \
        switch (a.nmode) {                                                                             \
        case 3: return c.phi ? launch_shape<FT, VT, 3, true>(a, c, st, bps)                            \
                             : launch_shape<FT, VT, 3, false>(a, c, st, bps);                          \
        case 4: return c.phi ? launch_shape<FT, VT, 4, true>(a, c, st, bps)                            \
                             : launch_shape<FT, VT, 4, false>(a, c, st, bps);                          \
        case 5: return c.phi ? launch_shape<FT, VT, 5, true>(a, c, st, bps)                            \
                             : launch_shape<FT, VT, 5, false>(a, c, st, bps);                          \
        }                                                                                              \
        return c.phi ? launch_shape<FT, VT, 0, true>(a, c, st, bps) : launch_shape<FT, VT, 0, false>(a, c, st, bps); \
    }                                                                                                  \
    template <>                                                                                        \
    altob_status launch_batch<FT, VT>(const BatchTiles<FT>& bt, int nm, const TiledCfg& c, cudaStream_t st, \
                                      int* bps)                                                        \
    {                                                                                                  \
        switch (nm) {                                                                                  \
        case 3: return launch_batch_shape<FT, VT, 3>(bt, c, st, bps);                                  \
        case 4: return launch_batch_shape<FT, VT, 4>(bt, c, st, bps);                                  \
        case 5: return launch_batch_shape<FT, VT, 5>(bt, c, st, bps);                                  \
        }                                                                                              \
        return launch_batch_shape<FT, VT, 0>(bt, c, st, bps);                                          \
    }                                                                                                  \
    template <>                                                                                        \
    altob_status launch_planned<FT, VT>(const TiledArgs<FT>& a, const TiledCfg& c, cudaStream_t st,    \
                                        int* bps)                                                      \
    {                                                                                                  \
        switch (a.nmode) {                                                                             \
        case 3: return launch_planned_shape<FT, VT, 3>(a, c, st, bps);                                 \
        case 4: return launch_planned_shape<FT, VT, 4>(a, c, st, bps);                                 \
        case 5: return launch_planned_shape<FT, VT, 5>(a, c, st, bps);                                 \
        }                                                                                              \
        return fail(ALTOB_ERR_UNSUPPORTED, "planned kernel: order 3-5");                               \
    }                                                                                                  \
    template <>                                                                                        \
    altob_status launch_atomic_cr<FT, VT>(const CrArgsK<FT>& a, cudaStream_t st)                       \
    {                                                                                                  \
        int blocks = (a.nprtn * 32 + MT_THREADS - 1) / MT_THREADS;                                      \
        if (blocks < 1) blocks = 1;                                                                    \
        k_atomic_cr<FT, VT><<<blocks, MT_THREADS, 0, st>>>(a);                                          \
        cudaError_t e = cudaGetLastError();                                                            \
        if (e != cudaSuccess) return fail(ALTOB_ERR_CUDA, std::string("k_atomic_cr: ") + cudaGetErrorString(e)); \
        return ALTOB_OK;                                                                               \
    }

}  // namespace altob
