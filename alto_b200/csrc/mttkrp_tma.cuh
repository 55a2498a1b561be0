// mttkrp_tma.cuh -- planned MTTKRP with the factor rows staged by TMA.
//
// The planned kernel (mttkrp_planned.cuh) gathers the other modes' factor
// rows with 16-byte loads issued by the lane groups themselves; it spends
// most of its time waiting for them (long-scoreboard stalls on L2 latency).
// Here a producer warp stages the rows in shared memory with the Tensor
// Memory Accelerator's row gather (cp.async.bulk.tensor.2d.tile::gather4:
// four rows of one factor matrix, chosen by index, per instruction, into
// consecutive shared memory, completion counted on an mbarrier), several
// steps ahead of the consumers, so the row loads in flight no longer hold
// registers and the consumer warps read their rows from shared memory.
//
// Per tile of 1024 nonzeros (the plan's tile): the 8 consumer warps decode
// and scatter the records to their run-ordered slots (planned_scatter),
// then every lane group walks its stretch of IPG records, four records per
// step.  Step s of a tile is one stage of the ring: the rows of records
// 4s..4s+3 of every lane group, mode by mode (gather4 of lane group g and
// mode k lands at stage + (k * G + g) * 4 rows).  full[stage] completes when
// the stage's bytes have arrived; empty[stage] when the 8 consumer warps
// have read it.  Runs of equal output rows are added as in lean_runs (sums
// in registers, one vector atomic per run, per-CTA hot-row accumulators).
//
// Only FP32 order-3 tensors whose rank R has a power-of-two R/4 (rows of
// 16 to 256 bytes, R = 4..64) take this path.  Every wait is bounded: when
// one runs out the kernel records it in *err and goes on without the data
// (the host reports the failure); the copies a CTA issued are waited for
// before it exits.
#pragma once

#include <cuda.h>

#include "mttkrp_planned.cuh"

namespace altob {

constexpr int TMA_CONSUMERS = 8;                          // consumer warps
constexpr int TMA_THREADS = (TMA_CONSUMERS + 1) * 32;     // + one producer warp
constexpr int TMA_STAGE_BYTES = 32 * 1024;                // rows of one step
constexpr unsigned TMA_WAIT_LIMIT = 1u << 24;             // polls per wait

struct TmaArgs {
    TiledArgs<float> a;
    unsigned* err;  // set to 1 when a wait runs out
};

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Waits (bounded) for the phase of the given parity; false when it ran out
// or when another thread of the CTA has given up already (*abort set): after
// the first wait that runs out, every later one returns at once.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, volatile int* abort,
                                          unsigned limit = TMA_WAIT_LIMIT)
{
    for (unsigned it = 0; it < limit; ++it) {
        unsigned done;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if ((it & 255) == 255 && *abort) return false;
    }
    *abort = 1;
    return false;
}

// Four rows (r0..r3) of the 2-D tensor map into dst (consecutive rows).
__device__ __forceinline__ void tma_gather4(unsigned dst, const CUtensorMap* map, int r0, int r1, int r2, int r3,
                                           unsigned bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
        "l"(map), "r"(0), "r"(r0), "r"(r1), "r"(r2), "r"(r3), "r"(bar)
        : "memory");
}

template <int LPN, int S>
struct TmaShape {
    static constexpr int NPW = 32 / LPN;
    static constexpr int G = TMA_CONSUMERS * NPW;   // lane groups
    static constexpr int IPG = PT_TILE / G;         // records per lane group and tile
    static constexpr int PSH = log2c(IPG);
    static constexpr int STEPS = IPG / 4;           // stages per tile
    static constexpr int SREC = PT_TILE + PT_TILE / IPG;
    static constexpr int ROW = LPN * 16;            // bytes per factor row (R = 4 * LPN)
    static_assert(2 * 4 * G * ROW == TMA_STAGE_BYTES, "stage size");
    static constexpr size_t REC_BYTES = 2 * (size_t)SREC * 16;  // two record buffers
    static constexpr size_t smem(int hot)
    {
        // records | hot-row tags | 2 S mbarriers | stages (1024-byte aligned)
        return ((REC_BYTES + (size_t)hot * 4 + 2 * S * 8 + 1023) & ~(size_t)1023) + (size_t)S * TMA_STAGE_BYTES + 1024;
    }
};

template <int LPN, int S>
__global__ void __launch_bounds__(TMA_THREADS, 1)
    k_planned_tma(const TmaArgs ta, const __grid_constant__ CUtensorMap map0, const __grid_constant__ CUtensorMap map1)
{
    using Sh = TmaShape<LPN, S>;
    constexpr int VEC = 4, MM = 3, RW = 4;
    const TiledArgs<float>& a = ta.a;
    extern __shared__ __align__(16) unsigned char smem[];  // stages aligned below (smem() has the slack)
    u32* buf0 = reinterpret_cast<u32*>(smem);
    u32* buf1 = buf0 + (size_t)Sh::SREC * RW;
    GroupedSmem gs = {};
    gs.htag = buf1 + (size_t)Sh::SREC * RW;
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(
        (reinterpret_cast<uintptr_t>(gs.htag + a.hot) + 7) & ~(uintptr_t)7);
    unsigned char* stages = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(bars + 2 * S) + 1023) & ~(uintptr_t)1023);
    const unsigned full0 = smem_addr(bars), empty0 = smem_addr(bars + S), st0 = smem_addr(stages);

    __shared__ int abort_flag;
    volatile int* abort = &abort_flag;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool producer = warp == TMA_CONSUMERS;
    const int R = a.R;
    if (tid == 0) {
        abort_flag = 0;
        for (int s = 0; s < S; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, TMA_CONSUMERS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (a.hot) {
        float* hacc = a.hot_acc + (size_t)blockIdx.x * a.hot * R;
        for (int k = tid; k < a.hot; k += TMA_THREADS) gs.htag[k] = 0;
        for (int k = tid; k < a.hot * R; k += TMA_THREADS) hacc[k] = 0.f;
    }
    __syncthreads();

    const int sub = lane % LPN, q = lane / LPN;
    const int grp = warp * Sh::NPW + q;  // consumers only
    const unsigned gmask = (0xffffffffu >> (32 - LPN)) << (q * LPN);
    bool ok = true;
    u64 chunk = 0;  // stages used so far (all tiles)
    int b = 0;
    for (u64 ti = blockIdx.x; ti < a.ntiles; ti += gridDim.x, b ^= 1) {
        u32* srec = b ? buf1 : buf0;
        const u64 g0 = ti * (u64)PT_TILE;
        const int nvalid = (int)min((u64)PT_TILE, a.nnz - g0);
        if (!producer) planned_scatter<float, float, MM, PT_TILE, Sh::PSH>(a, g0, nvalid, srec);
        __syncthreads();  // records of this tile ready (two buffers: one barrier per tile)
        if (producer) {
            // the rows of every step, one stage each, as the ring frees up
            for (int s = 0; s < Sh::STEPS; ++s, ++chunk) {
                const int st = (int)(chunk % S);
                const unsigned par = (unsigned)((chunk / S) & 1);
                ok = mbar_wait(empty0 + 8 * st, par ^ 1u, abort) && ok;
                if (lane == 0) mbar_expect_tx(full0 + 8 * st, TMA_STAGE_BYTES);
                __syncwarp();
                for (int x = lane; x < 2 * Sh::G; x += 32) {
                    const int g = x >> 1, k = x & 1;
                    int r[4];
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const int p = g * Sh::IPG + 4 * s + i;  // past the tile's end: row 0 (read, not used)
                        r[i] = p < nvalid ? (int)srec[(size_t)rslot_t<Sh::PSH>(p) * RW + 1 + k] : 0;
                    }
                    tma_gather4(st0 + st * TMA_STAGE_BYTES + (k * Sh::G + g) * 4 * Sh::ROW, k ? &map1 : &map0,
                                r[0], r[1], r[2], r[3], full0 + 8 * st);
                }
            }
            continue;
        }
        // consumers: the lane group's stretch, four records per stage
        const int p0 = grp * Sh::IPG, pend = min(p0 + Sh::IPG, nvalid);
        u32 cur = 0xffffffffu;
        int len = 0;
        float acc[1][VEC] = {{0.f, 0.f, 0.f, 0.f}};
        for (int s = 0; s < Sh::STEPS; ++s, ++chunk) {
            const int st = (int)(chunk % S);
            const unsigned par = (unsigned)((chunk / S) & 1);
            // one decision per warp (the run flushes shuffle within lane groups)
            const bool arrived = __all_sync(0xffffffffu, mbar_wait(full0 + 8 * st, par, abort));
            ok = arrived && ok;
            const unsigned char* rows = stages + (size_t)st * TMA_STAGE_BYTES;
            if (arrived) {
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int p = p0 + 4 * s + i;
                    if (p >= pend) break;
                    const uint4 w = *reinterpret_cast<const uint4*>(srec + (size_t)rslot_t<Sh::PSH>(p) * RW);
                    const float4 y0 = *reinterpret_cast<const float4*>(rows + (grp * 4 + i) * Sh::ROW + sub * 16);
                    const float4 y1 =
                        *reinterpret_cast<const float4*>(rows + ((Sh::G + grp) * 4 + i) * Sh::ROW + sub * 16);
                    const float v = __uint_as_float(w.w);
                    float x[1][VEC] = {{v, v, v, v}};
                    const float ya[VEC] = {y0.x, y0.y, y0.z, y0.w}, yb[VEC] = {y1.x, y1.y, y1.z, y1.w};
                    vmul<float, VEC>(x[0], ya);
                    vmul<float, VEC>(x[0], yb);
                    if (w.x != cur) {
                        if (cur != 0xffffffffu)
                            flush_run<float, VEC, 1, LPN>(a.out, gs, len >= GT_HOT_MINRUN ? a.hot : 0, a.hot_acc,
                                                          gmask, cur, R, sub, acc);
                        cur = w.x;
                        len = 1;
#pragma unroll
                        for (int e = 0; e < VEC; ++e) acc[0][e] = x[0][e];
                    } else {
                        run_add<float, VEC, 1>(acc, x);
                        ++len;
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(empty0 + 8 * st);
        }
        if (cur != 0xffffffffu)
            flush_run<float, VEC, 1, LPN>(a.out, gs, len >= GT_HOT_MINRUN ? a.hot : 0, a.hot_acc, gmask, cur, R,
                                          sub, acc);
    }
    // every copy the producer issued has landed before the CTA exits: the
    // last phase of each stage (complete already unless a wait gave up)
    if (producer) {
        for (int st = 0; st < S; ++st) {
            const u64 uses = chunk / S + (st < (int)(chunk % S) ? 1 : 0);
            if (uses) {
                volatile int keep_waiting = 0;  // these waits do not give up early
                mbar_wait(full0 + 8 * st, (unsigned)((uses - 1) & 1), &keep_waiting);
            }
        }
    }
    if (!ok && lane == 0) atomicExch(ta.err, 1u);
    if (a.hot) {  // the CTA's hot-row sums, once each
        const float* hacc = a.hot_acc + (size_t)blockIdx.x * a.hot * R;
        __syncthreads();
        for (int k = tid; k < a.hot * R; k += TMA_THREADS) {
            const int sl = k / R;
            const u32 tg = gs.htag[sl];
            if (tg) atomicAdd(a.out + (size_t)(tg - 1u) * R + (k - sl * R), __ldcg(hacc + k));
        }
    }
}

}  // namespace altob
