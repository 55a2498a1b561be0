// mttkrp_planned.cuh -- MTTKRP on the ALTO stream with a per-mode tile plan.
//
// Replaces mttkrp_alto_da_mem_pull (IntelLabs/ALTO include/alto.hpp:
// 1227-1318) for modes with fiber reuse above 4.  The grouped kernel
// (mttkrp_kernels.cuh) sorts every tile of the stream by output row on each
// launch: slot claims, a scan and a counting-sort scatter, about 40% of its
// instructions.  That order depends only on the tensor and the mode, so it is
// computed once (k_tile_plan) and kept beside the stream as a 16-bit position
// per nonzero and mode ("tile plan": where the nonzero goes in its tile's
// records sorted by the mode's index, ties in stream order).  A launch then
// reads key, value and plan entry (14 B per nonzero instead of 12), decodes
// the mode indices and writes each record straight to its sorted slot in
// shared memory; the run phase is the grouped kernel's (lean_runs: running
// row sums in registers, one vector atomic per run, per-CTA hot-row
// accumulators for long runs).  Two record buffers alternate between tiles,
// so one barrier per tile separates the scatter from the run phase.
//
// The plan is the tile-local analogue of the reference's oidx (alto.hpp:
// 246-285: a full permutation per low-reuse mode); it is built on the first
// MTTKRP of a mode and freed with the tensor.
#pragma once

#include "mttkrp_kernels.cuh"

namespace altob {

typedef uint16_t u16;

// Default tile of the planned kernels (nonzeros per tile; plan entries are
// below the tile size).
constexpr int PT_TILE = 1024;

// Decoded high key word of the nonzeros of one tile: one value for the whole
// tile unless it spans a run boundary of the high-word table (then two), or
// more than two runs (then a search per nonzero).
struct TileHi {
    u64 hcur = 0, hnext = 0, nstart = ~0ull;
    bool slow = false;
    __device__ __forceinline__ void init(const KeySrc& k, u64 g0, int tile)
    {
        if (k.khi || k.nrun == 0) return;
        const int r = run_of(k, g0);
        hcur = k.run_val[r];
        if (r + 1 < k.nrun) {
            nstart = k.run_start[r + 1];
            hnext = k.run_val[r + 1];
            if (r + 2 < k.nrun && k.run_start[r + 2] < g0 + (u64)tile) slow = true;
        }
    }
    __device__ __forceinline__ u64 get(const KeySrc& k, u64 g) const
    {
        if (k.khi) return k.khi[g];
        if (k.nrun == 0) return 0;
        if (slow) return key_hi(k, g);
        return g >= nstart ? hnext : hcur;
    }
};

// ------------------------------------------------------------ plan build
//
// One CTA per tile: (mode index << 32 | position in the tile) keys sorted by
// a bitonic network in shared memory; entry g of the plan is the sorted rank
// of nonzero g inside its tile.  Positions past the end of the stream sort
// last and are not written.
template <int TILE>
__global__ void __launch_bounds__(TILE / 2) k_tile_plan(KeySrc key, Fields fld, u64 nnz, int mode, u16* plan)
{
    __shared__ unsigned long long s[TILE];
    const int tid = threadIdx.x;
    const u64 g0 = (u64)blockIdx.x * TILE;
    const int nvalid = (int)min((u64)TILE, nnz - g0);
    for (int i = tid; i < TILE; i += TILE / 2) {
        unsigned long long k = ~0ull;
        if (i < nvalid) {
            const u64 g = g0 + i;
            const u64 lo = key.klo[g];
            const u64 hi = key.khi ? key.khi[g] : (key.nrun ? key_hi(key, g) : 0);
            const u32 row = field(lo, hi, fld.pos[mode], fld.mask[mode]);
            k = ((unsigned long long)row << 32) | (u32)i;
        }
        s[i] = k;
    }
    __syncthreads();
    for (int k = 2; k <= TILE; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = tid; i < TILE; i += TILE / 2) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const unsigned long long x = s[i], y = s[ixj];
                    const bool up = (i & k) == 0;
                    if ((x > y) == up) {
                        s[i] = y;
                        s[ixj] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (int p = tid; p < nvalid; p += TILE / 2) plan[g0 + (u32)s[p]] = (u16)p;
}

// --------------------------------------------------------- planned MTTKRP

// Resident blocks per SM each instance is compiled for (register cap), FP32:
// 5 blocks of 8 warps for order 3 (48 registers; the run loop waits on its
// row gathers, so more resident warps hide more of that latency: 2.31 ms per
// mode at 4 blocks, 2.17 ms at 5 on the 100.85M-nonzero Zipf tensor; 3
// blocks: 2.53 ms) and 3 for orders 4-5 (80-86 registers uncapped would
// allow only 2).  Ranks above 64 (32 lanes per nonzero) keep 4 blocks: at 48
// registers their run loop spills.  FP64 order 3: 4 blocks (53-56
// registers, one record buffer; 80 registers and 3 blocks uncapped: 23.1 ->
// 21.9 ms per FP64 sweep of the same tensor; 5 blocks measured the same).
template <typename FT, int NM, int LPN>
constexpr int planned_min_blocks()
{
    if (sizeof(FT) != 4) return NM == 3 ? 4 : 0;
    return NM == 3 ? (LPN <= 16 ? 5 : 4) : 3;
}

// Record buffers of the planned kernel: two (the next tile's scatter
// overlaps this tile's runs) unless the records are 32 bytes and the kernel
// targets 4 blocks per SM (order-3 FP64: two 33 KB buffers would leave room
// for 3).
template <typename FT, int NM>
constexpr int planned_nbuf()
{
    return (sizeof(FT) == 8 && NM == 3) ? 1 : 2;
}

// Nonzeros whose key, value and plan entry a thread loads together in the
// scatter phase.  Four in flight were the register peak of the kernel; the
// order-3 instances keep one, which is what lets them fit their register
// caps without spilling in the run loop.
template <typename FT, int NM>
constexpr int planned_scatter_q()
{
    return NM == 3 ? 1 : 4;
}

// Records a lane group takes per tile (lpn lanes per nonzero).
constexpr int planned_ipg(int pt, int lpn) { return pt / (MT_WARPS * (32 / lpn)); }
constexpr int log2c(int x) { return x <= 1 ? 0 : 1 + log2c(x / 2); }

// Dynamic shared memory of the planned kernel: nbuf run-ordered record
// buffers (one padding record per lane-group stretch) and the hot-row tags.
inline size_t planned_smem(int nmode, size_t fsz, int hot, int lpn, int pt, int nbuf)
{
    const int rw = (nmode + (int)(fsz / 4) + 3) & ~3;
    return (size_t)nbuf * (size_t)(pt + pt / planned_ipg(pt, lpn)) * rw * 4 + (size_t)hot * 4;
}

// Phase A of a planned tile: every thread loads key, value and plan entry
// of its nonzeros (four in flight at a time), decodes the mode indices and
// writes the record [target, other modes..., value] to its run-ordered slot
// (one padding record per 2^PSH).
template <typename FT, typename VT, int MM, int PT, int PSH, int QM = 4>
__device__ __forceinline__ void planned_scatter(const TiledArgs<FT>& a, u64 g0, int nvalid, u32* srec)
{
    constexpr int RW = RecWords<FT, MM>::n;
    constexpr int FW = (int)(sizeof(FT) / 4);
    constexpr int IPT = PT / MT_THREADS;
    constexpr int IPQ = IPT < QM ? IPT : QM;
    const int tid = threadIdx.x, target = a.target;
    const VT* vals = reinterpret_cast<const VT*>(a.vals);
    TileHi th;
    th.init(a.key, g0, PT);
#pragma unroll
    for (int k0 = 0; k0 < IPT; k0 += IPQ) {
        u64 lo[IPQ];
        VT vv[IPQ];
        u32 ps[IPQ];
#pragma unroll
        for (int k = 0; k < IPQ; ++k) {
            const int it = tid + (k0 + k) * MT_THREADS;
            if (it < nvalid) {
                const u64 g = g0 + it;
                lo[k] = __ldcs(reinterpret_cast<const unsigned long long*>(a.key.klo) + g);
                vv[k] = ldcs_val(vals + g);
                ps[k] = __ldcs(reinterpret_cast<const unsigned short*>(a.plan) + g);
            }
        }
#pragma unroll
        for (int k = 0; k < IPQ; ++k) {
            const int it = tid + (k0 + k) * MT_THREADS;
            if (it < nvalid) {
                const u64 g = g0 + it;
                const u64 hi = th.get(a.key, g);
                u32 c[MM];
#pragma unroll
                for (int m = 0; m < MM; ++m) c[m] = field(lo[k], hi, a.fld.pos[m], a.fld.mask[m]);
                u32 w[RW];
#pragma unroll
                for (int x = 0; x < RW; ++x) w[x] = 0u;
                w[0] = c[0];
#pragma unroll
                for (int m = 1; m < MM; ++m)
                    if (m == target) w[0] = c[m];
#pragma unroll
                for (int s = 1; s < MM; ++s) w[s] = s - 1 < target ? c[s - 1] : c[s];
                const FT fv = (FT)vv[k];
                if constexpr (FW == 1) {
                    w[MM] = __float_as_uint((float)fv);
                } else {
                    const unsigned long long bits = (unsigned long long)__double_as_longlong((double)fv);
                    w[MM] = (u32)bits;
                    w[MM + 1] = (u32)(bits >> 32);
                }
                u32* dst = srec + (size_t)rslot_t<PSH>((int)ps[k]) * RW;
#pragma unroll
                for (int x = 0; x < RW; x += 4)
                    *reinterpret_cast<uint4*>(dst + x) = make_uint4(w[x], w[x + 1], w[x + 2], w[x + 3]);
            }
        }
    }
}

// One planned tile with one record buffer (the batched kernel): scatter,
// barrier, runs, barrier.  The records use the grouped kernel's padding (one
// per 32), so the buffer is the grouped kernel's run-ordered record area.
template <typename FT, typename VT, int NM, int LPN, int VEC>
__device__ __forceinline__ void planned_tile(const TiledArgs<FT>& a, u64 ti, const GroupedSmem& gs)
{
    constexpr int NPW = 32 / LPN;
    constexpr int IPG = PT_TILE / (MT_WARPS * NPW);
    static_assert(NM >= 3 && NM <= ALTOB_MAX_MODES, "static order 3..5");
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int sub = lane % LPN, q = lane / LPN;
    const unsigned gmask = (0xffffffffu >> (32 - LPN)) << (q * LPN);
    const u64 g0 = ti * (u64)PT_TILE;
    const int nvalid = (int)min((u64)PT_TILE, a.nnz - g0);
    planned_scatter<FT, VT, NM, PT_TILE, 5, planned_scatter_q<FT, NM>()>(a, g0, nvalid, gs.srec);
    __syncthreads();
    const int p0 = (warp * NPW + q) * IPG;
    const FT* Uo[NM - 1];
#pragma unroll
    for (int k = 0; k < NM - 1; ++k) Uo[k] = a.U[k < a.target ? k : k + 1];
    lean_runs<FT, NM, LPN, VEC, 5>(a, gs, Uo, p0, min(p0 + IPG, nvalid), a.R, sub, gmask);
    __syncthreads();
}

// PT: nonzeros per tile (the plan's tile); NBUF: record buffers (2: the
// next tile's scatter overlaps this tile's runs, one barrier per tile; 1:
// two barriers per tile, half the shared memory, so more of the SM's
// 256 KB stays L1 cache for the row gathers).
template <typename FT, typename VT, int NM, int LPN, int VEC, int PT, int NBUF>
__device__ __forceinline__ void planned_body(const TiledArgs<FT>& a)
{
    constexpr int MM = NM;
    constexpr int RW = RecWords<FT, MM>::n;
    constexpr int NPW = 32 / LPN;
    constexpr int NGRP = MT_WARPS * NPW;
    constexpr int IPG = PT / NGRP;
    constexpr int PSH = log2c(IPG);
    constexpr int SREC = PT + PT / IPG;
    static_assert(IPG == planned_ipg(PT, LPN) && (1 << PSH) == IPG, "lane-group stretch");
    static_assert(NM >= 3 && NM <= ALTOB_MAX_MODES, "static order 3..5");
    static_assert(NBUF == 1 || NBUF == 2, "record buffers");
    extern __shared__ __align__(16) unsigned char smem[];
    u32* buf0 = reinterpret_cast<u32*>(smem);
    u32* buf1 = buf0 + (NBUF - 1) * (size_t)SREC * RW;
    GroupedSmem gs = {};
    gs.htag = buf1 + (size_t)SREC * RW;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int R = a.R, target = a.target;
    const int sub = lane % LPN, q = lane / LPN;
    const int grp = warp * NPW + q;
    const unsigned gmask = (0xffffffffu >> (32 - LPN)) << (q * LPN);
    if (a.hot) {
        FT* hacc = a.hot_acc + (size_t)blockIdx.x * a.hot * R;
        for (int k = tid; k < a.hot; k += MT_THREADS) gs.htag[k] = 0;
        for (int k = tid; k < a.hot * R; k += MT_THREADS) hacc[k] = FT(0);
    }
    __syncthreads();  // the zeroed accumulators precede every run flush

    int b = 0;
    for (u64 ti = blockIdx.x; ti < a.ntiles; ti += gridDim.x, b ^= 1) {
        u32* srec = b ? buf1 : buf0;
        const u64 g0 = ti * (u64)PT;
        const int nvalid = (int)min((u64)PT, a.nnz - g0);
        // ---- A: load key, value and plan entry; record into its sorted slot
        planned_scatter<FT, VT, MM, PT, PSH, planned_scatter_q<FT, NM>()>(a, g0, nvalid, srec);
        // with two buffers one barrier per tile: the buffer written next tile
        // was last read before this barrier
        __syncthreads();
        // ---- B: runs of equal output rows (grouped kernel's run loop)
        gs.srec = srec;
        const int p0 = grp * IPG;
        const int pend = min(p0 + IPG, nvalid);
        const FT* Uo[MM - 1];  // from the parameters each tile: fewer live registers
#pragma unroll
        for (int k = 0; k < MM - 1; ++k) Uo[k] = a.U[k < target ? k : k + 1];
        lean_runs<FT, MM, LPN, VEC, PSH>(a, gs, Uo, p0, pend, R, sub, gmask);
        if constexpr (NBUF == 1) __syncthreads();  // the records are overwritten next tile
    }
    if (a.hot) {  // the CTA's hot-row sums, once each
        const FT* hacc = a.hot_acc + (size_t)blockIdx.x * a.hot * R;
        __syncthreads();
        for (int k = tid; k < a.hot * R; k += MT_THREADS) {
            const int sl = k / R;
            const u32 tg = gs.htag[sl];
            if (tg) atomicAdd(a.out + (size_t)(tg - 1u) * R + (k - sl * R), __ldcg(hacc + k));
        }
    }
}

template <typename FT, typename VT, int NM, int LPN, int VEC, int PT = PT_TILE, int NBUF = 2>
__global__ void __launch_bounds__(MT_THREADS) k_planned(TiledArgs<FT> a)
{
    planned_body<FT, VT, NM, LPN, VEC, PT, NBUF>(a);
}

template <typename FT, typename VT, int NM, int LPN, int VEC, int MINB, int PT = PT_TILE, int NBUF = 2>
__global__ void __launch_bounds__(MT_THREADS, MINB) k_planned_mb(TiledArgs<FT> a)
{
    planned_body<FT, VT, NM, LPN, VEC, PT, NBUF>(a);
}

// Batched form: the tiles of many tensors (one TiledArgs each, same shape
// class and slot count) in one persistent launch.  tile_prefix[b] is the
// first global tile of tensor b; tensors whose active flag is 0 are skipped.
template <typename FT>
struct BatchTiles {
    const TiledArgs<FT>* args;
    const u64* tile_prefix;  // ntensors + 1
    const int* bid;          // batch index of each entry (for `active`)
    const int* active;
    int ntensors;
    int hslots;
    u64 total_tiles;
};

template <typename FT, typename VT, int NM, int LPN, int VEC, int CH, bool PHI>
__device__ __forceinline__ void grouped_batch_body(const BatchTiles<FT>& bt)
{
    constexpr int MM = grouped_mm<NM>();
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ u32 statics[2 + MT_WARPS];
    const GroupedSmem gs = grouped_smem_ptrs<FT, MM>(smem, bt.hslots, statics);
    grouped_init(gs, bt.hslots);
    for (u64 gt = blockIdx.x; gt < bt.total_tiles; gt += gridDim.x) {
        int lo = 0, hi = bt.ntensors - 1;  // last tensor whose first tile <= gt
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (bt.tile_prefix[mid] <= gt) lo = mid;
            else hi = mid - 1;
        }
        if (!bt.active[bt.bid[lo]]) continue;
        grouped_tile<FT, VT, NM, LPN, VEC, CH, PHI>(bt.args[lo], gt - bt.tile_prefix[lo], gs);
    }
}

template <typename FT, typename VT, int NM, int LPN, int VEC, int CH, bool PHI>
__global__ void __launch_bounds__(MT_THREADS) k_grouped_batch(BatchTiles<FT> bt)
{
    grouped_batch_body<FT, VT, NM, LPN, VEC, CH, PHI>(bt);
}

template <typename FT, typename VT, int NM, int LPN, int VEC, int CH, bool PHI, int MINB>
__global__ void __launch_bounds__(MT_THREADS, MINB) k_grouped_batch_mb(BatchTiles<FT> bt)
{
    grouped_batch_body<FT, VT, NM, LPN, VEC, CH, PHI>(bt);
}

// Batched planned MTTKRP: the tiles of the tensors whose target mode has a
// tile plan (same shape class), one persistent launch; single record buffer.
template <typename FT, typename VT, int NM, int LPN, int VEC>
__device__ __forceinline__ void planned_batch_body(const BatchTiles<FT>& bt)
{
    extern __shared__ __align__(16) unsigned char smem[];
    GroupedSmem gs = {};
    gs.srec = reinterpret_cast<u32*>(smem);
    for (u64 gt = blockIdx.x; gt < bt.total_tiles; gt += gridDim.x) {
        int lo = 0, hi = bt.ntensors - 1;  // last tensor whose first tile <= gt
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (bt.tile_prefix[mid] <= gt) lo = mid;
            else hi = mid - 1;
        }
        if (!bt.active[bt.bid[lo]]) continue;
        planned_tile<FT, VT, NM, LPN, VEC>(bt.args[lo], gt - bt.tile_prefix[lo], gs);
    }
}

template <typename FT, typename VT, int NM, int LPN, int VEC>
__global__ void __launch_bounds__(MT_THREADS) k_planned_batch(BatchTiles<FT> bt)
{
    planned_batch_body<FT, VT, NM, LPN, VEC>(bt);
}

template <typename FT, typename VT, int NM, int LPN, int VEC, int MINB>
__global__ void __launch_bounds__(MT_THREADS, MINB) k_planned_batch_mb(BatchTiles<FT> bt)
{
    planned_batch_body<FT, VT, NM, LPN, VEC>(bt);
}

// Shared memory of the batched planned kernel: one run-ordered record buffer.
inline size_t planned_batch_smem(int nmode, size_t fsz)
{
    const int rw = (nmode + (int)(fsz / 4) + 3) & ~3;
    return (size_t)(PT_TILE + PT_TILE / 32) * rw * 4;
}

}  // namespace altob
