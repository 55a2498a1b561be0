// mttkrp_launch.cuh -- typed launchers for the MTTKRP / Phi kernels.  Each
// (FT, VT) pair is instantiated in its own translation unit
// (mttkrp_<ft>_<vt>.cu) so the kernels compile in parallel.
#pragma once

#include "mttkrp_kernels.cuh"

namespace altob {

struct TiledCfg {
    int kw, lpn, vec, phi;
    dim3 grid;
    size_t smem;
};

template <typename FT, typename VT>
altob_status launch_tiled(const TiledArgs<FT>& a, const TiledCfg& c, cudaStream_t st, int* max_blocks_per_sm);

template <typename FT, typename VT>
altob_status launch_atomic_cr(const CrArgsK<FT>& a, int kw, cudaStream_t st);

// Resolves the kernel for (KW, LPN, VEC, PHI), sets its shared-memory limit
// once, and launches it (or only reports occupancy when grid.x == 0).
template <typename FT, typename VT, int KW, int LPN, int VEC, bool PHI>
altob_status launch_one(const TiledArgs<FT>& a, const TiledCfg& c, cudaStream_t st, int* bps)
{
    auto k = k_tiled<FT, VT, KW, LPN, VEC, PHI>;
    static size_t configured = 0;
    if (c.smem > configured) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c.smem);
        if (e != cudaSuccess) return fail(ALTOB_ERR_CUDA, std::string("smem attribute: ") + cudaGetErrorString(e));
        configured = c.smem;
    }
    if (bps) {
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, MT_THREADS, c.smem);
        *bps = n;
    }
    if (c.grid.x == 0) return ALTOB_OK;
    k<<<c.grid, MT_THREADS, c.smem, st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(ALTOB_ERR_CUDA, std::string("k_tiled launch: ") + cudaGetErrorString(e));
    return ALTOB_OK;
}

template <typename FT, typename VT, int KW, bool PHI>
altob_status launch_lpn(const TiledArgs<FT>& a, const TiledCfg& c, cudaStream_t st, int* bps)
{
    constexpr int V = 16 / sizeof(FT);
    if (c.vec == 1) return launch_one<FT, VT, KW, 32, 1, PHI>(a, c, st, bps);
    switch (c.lpn) {
    case 2: return launch_one<FT, VT, KW, 2, V, PHI>(a, c, st, bps);
    case 4: return launch_one<FT, VT, KW, 4, V, PHI>(a, c, st, bps);
    case 8: return launch_one<FT, VT, KW, 8, V, PHI>(a, c, st, bps);
    case 16: return launch_one<FT, VT, KW, 16, V, PHI>(a, c, st, bps);
    case 32: return launch_one<FT, VT, KW, 32, V, PHI>(a, c, st, bps);
    }
    return fail(ALTOB_ERR_UNSUPPORTED, "lanes per nonzero");
}

#define ALTOB_INSTANTIATE_MTTKRP(FT, VT)                                                                 \
    template <>                                                                                        \
    altob_status launch_tiled<FT, VT>(const TiledArgs<FT>& a, const TiledCfg& c, cudaStream_t st,      \
                                      int* bps)                                                        \
    {                                                                                                  \
        if (c.kw == 2)                                                                                 \
            return c.phi ? launch_lpn<FT, VT, 2, true>(a, c, st, bps)                                  \
                         : launch_lpn<FT, VT, 2, false>(a, c, st, bps);                                \
        return c.phi ? launch_lpn<FT, VT, 1, true>(a, c, st, bps) : launch_lpn<FT, VT, 1, false>(a, c, st, bps); \
    }                                                                                                  \
    template <>                                                                                        \
    altob_status launch_atomic_cr<FT, VT>(const CrArgsK<FT>& a, int kw, cudaStream_t st)               \
    {                                                                                                  \
        int warps = a.nprtn;                                                                           \
        int blocks = (warps * 32 + MT_THREADS - 1) / MT_THREADS;                                        \
        if (blocks < 1) blocks = 1;                                                                    \
        if (kw == 2) k_atomic_cr<FT, VT, 2><<<blocks, MT_THREADS, 0, st>>>(a);                          \
        else k_atomic_cr<FT, VT, 1><<<blocks, MT_THREADS, 0, st>>>(a);                                  \
        cudaError_t e = cudaGetLastError();                                                            \
        if (e != cudaSuccess) return fail(ALTOB_ERR_CUDA, std::string("k_atomic_cr: ") + cudaGetErrorString(e)); \
        return ALTOB_OK;                                                                               \
    }

}  // namespace altob
