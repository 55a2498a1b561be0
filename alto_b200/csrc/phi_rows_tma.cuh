// phi_rows_tma.cuh -- CP-APR Phi over the row-ordered stream, with the
// stream staged in shared memory by bulk asynchronous copies.
//
// Replaces the inner-iteration Phi of CalculatePhi_alto_par with
// precomputed rows (IntelLabs/ALTO include/apr.hpp:383-848, the PRE build of
// :1133-1171).  The stream of mode n holds, per nonzero in mode-index order,
// its precomputed Khatri-Rao row (R values), its target row and its value
// (mttkrp.cu, mode_order_device / pi_device).  An inner iteration is one
// sequential read of it: Phi[i, :] = sum over the nonzeros of row i of
// v / max(<B[i, :], krp>, eps) * krp.
//
// k_phi_rows (mttkrp.cu) loads the stream into registers and spends its time
// waiting on those loads (long-scoreboard stalls at 0.71 of the copy
// bandwidth).  Here a producer warp streams it into a ring of shared-memory
// stages with cp.async.bulk (one-dimensional bulk copies, completion counted
// on an mbarrier), several stages ahead of the sixteen consumer warps, so the
// bytes in flight no longer hold registers.  Each CTA takes a contiguous
// range of stages; a lane group ("virtual group" vg of the CTA) takes the
// stream positions congruent to vg modulo the CTA's group count, so it sees
// the positions of one row in order and keeps its run sum across stages,
// flushing with one vector atomic per lane when the row changes.
//
// Every wait is bounded: a wait that runs out sets *err and the CTA goes on
// without the data; the copies a CTA issued are waited for before it exits.
#pragma once

#include "mttkrp_tma.cuh"

namespace altob {

constexpr int PX_CONSUMERS = 16;                      // consumer warps
constexpr int PX_THREADS = (PX_CONSUMERS + 1) * 32;   // + one producer warp
constexpr int PX_STAGES = 3;
constexpr int PX_ROW_BYTES = 24 * 1024;               // Khatri-Rao rows per stage (at most)

__device__ __forceinline__ void bulk_g2s(unsigned dst, const void* src, unsigned bytes, unsigned bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

template <typename FT>
struct PhiTmaArgs {
    const FT* Pi;      // stream-ordered Khatri-Rao rows, nnz x R
    const u32* rows;   // target row per stream position (readable up to a multiple of 4 past nnz)
    const FT* vals;    // value per stream position (the same)
    const FT* B;       // current factor of the mode
    FT* Phi;           // output, zeroed by the caller
    u64 nnz;
    u64 S;             // stream positions per stage (a multiple of the CTA's lane groups)
    u64 nstage;        // stages in the stream
    u64 per_cta;       // contiguous stages per CTA
    int R;
    FT eps;
    unsigned* err;
    unsigned wait_limit;  // polls per mbarrier wait
    int stall;            // 1: the producer issues no copies (a failure test: every
                          // consumer wait then runs out and the kernel reports it)
};

// Byte offsets of one stage: rows of the Khatri-Rao stream | target rows |
// values, each 16-byte aligned.
struct PxLayout {
    unsigned pi, rw, vl, stage;
    __host__ __device__ PxLayout(u64 S, int R, int fsz)
    {
        pi = 0;
        rw = (unsigned)((S * (u64)R * fsz + 15) & ~15ull);
        vl = rw + (unsigned)((S * 4 + 15) & ~15ull);
        stage = (vl + (unsigned)((S * (u64)fsz + 15) & ~15ull) + 127) & ~127u;
    }
};

inline size_t phi_tma_smem(u64 S, int R, int fsz)
{
    const PxLayout L(S, R, fsz);
    return (size_t)PX_STAGES * L.stage + 2 * PX_STAGES * 8 + 128 + 256;
}

template <typename FT, int VEC, int LPN>
__global__ void __launch_bounds__(PX_THREADS, 2) k_phi_rows_tma(const PhiTmaArgs<FT> a)
{
    constexpr int G = 32 / LPN;               // lane groups per warp
    constexpr int VG = PX_CONSUMERS * G;      // lane groups per CTA
    constexpr int FSZ = (int)sizeof(FT);
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // stages on a 128-byte boundary (phi_tma_smem has the slack)
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
    const PxLayout L(a.S, a.R, FSZ);
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem + (size_t)PX_STAGES * L.stage);
    const unsigned st0 = smem_addr(smem), full0 = smem_addr(bars), empty0 = smem_addr(bars + PX_STAGES);
    __shared__ int abort_flag;
    volatile int* abort = &abort_flag;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool producer = warp == PX_CONSUMERS;
    if (tid == 0) {
        abort_flag = 0;
        for (int s = 0; s < PX_STAGES; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, PX_CONSUMERS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    const u64 t0 = (u64)blockIdx.x * a.per_cta;
    const u64 t1 = min(a.nstage, t0 + a.per_cta);
    const int R = a.R;
    bool ok = true;
    u64 used = 0;  // stages of the ring used so far
    if (producer) {
        if (lane == 0 && !a.stall) {
            for (u64 t = t0; t < t1; ++t, ++used) {
                const int sl = (int)(used % PX_STAGES);
                const unsigned par = (unsigned)((used / PX_STAGES) & 1);
                ok = mbar_wait(empty0 + 8 * sl, par ^ 1u, abort, a.wait_limit) && ok;
                if (!ok || *abort) break;  // a wait gave up: issue nothing more
                const u64 p0 = t * a.S;
                const u64 n = min(a.S, a.nnz - p0);
                const u64 n4 = (n + 3) & ~3ull;  // the stream arrays are readable to a multiple of 4
                const unsigned bpi = (unsigned)(n * (u64)R * FSZ);
                const unsigned brw = (unsigned)(n4 * 4);
                const unsigned bvl = (unsigned)((n4 * FSZ + 15) & ~15ull);
                const unsigned dst = st0 + (unsigned)sl * L.stage;
                mbar_expect_tx(full0 + 8 * sl, bpi + brw + bvl);
                bulk_g2s(dst + L.pi, a.Pi + p0 * (u64)R, bpi, full0 + 8 * sl);
                bulk_g2s(dst + L.rw, a.rows + p0, brw, full0 + 8 * sl);
                bulk_g2s(dst + L.vl, a.vals + p0, bvl, full0 + 8 * sl);
            }
            // every issued copy lands before the CTA exits
            for (int sl = 0; sl < PX_STAGES; ++sl) {
                const u64 uses = used / PX_STAGES + ((u64)sl < used % PX_STAGES ? 1 : 0);
                if (uses) {
                    volatile int keep_waiting = 0;
                    mbar_wait(full0 + 8 * sl, (unsigned)((uses - 1) & 1), &keep_waiting, a.wait_limit);
                }
            }
        }
    } else {
        const int q = lane / LPN, sub = lane % LPN;
        const int vg = warp * G + q;
        const unsigned gmask = LPN == 32 ? 0xffffffffu : (((1u << LPN) - 1u) << (q * LPN));
        const int r0 = sub * VEC;
        const bool live = r0 < R;
        u32 cur = 0xffffffffu;
        FT acc[VEC], bc[VEC];
#pragma unroll
        for (int e = 0; e < VEC; ++e) acc[e] = bc[e] = FT(0);
        for (u64 t = t0; t < t1; ++t, ++used) {
            const int sl = (int)(used % PX_STAGES);
            const unsigned par = (unsigned)((used / PX_STAGES) & 1);
            const bool arrived = __all_sync(0xffffffffu, mbar_wait(full0 + 8 * sl, par, abort, a.wait_limit));
            ok = arrived && ok;
            if (arrived) {
                const unsigned char* sb = smem + (size_t)sl * L.stage;
                const FT* spi = reinterpret_cast<const FT*>(sb + L.pi);
                const u32* srw = reinterpret_cast<const u32*>(sb + L.rw);
                const FT* svl = reinterpret_cast<const FT*>(sb + L.vl);
                const int n = (int)min(a.S, a.nnz - t * a.S);
                for (int p = vg; p < n; p += VG) {
                    const u32 rw = srw[p];
                    const FT v = svl[p];
                    FT x[VEC];
                    if (live) {
                        if constexpr (VEC * FSZ == 16) {
                            const uint4 w = *reinterpret_cast<const uint4*>(spi + (size_t)p * R + r0);
                            const FT* f = reinterpret_cast<const FT*>(&w);
#pragma unroll
                            for (int e = 0; e < VEC; ++e) x[e] = f[e];
                        } else {
#pragma unroll
                            for (int e = 0; e < VEC; ++e) x[e] = spi[(size_t)p * R + r0 + e];
                        }
                    } else {
#pragma unroll
                        for (int e = 0; e < VEC; ++e) x[e] = FT(0);
                    }
                    if (rw != cur) {
                        if (live) {
                            if (cur != 0xffffffffu) gred<FT, VEC>(a.Phi + (size_t)cur * R + r0, acc);
                            vload<FT, VEC>(a.B + (size_t)rw * R + r0, bc);
                        }
#pragma unroll
                        for (int e = 0; e < VEC; ++e) acc[e] = FT(0);
                        cur = rw;
                    }
                    FT dot = FT(0);
#pragma unroll
                    for (int e = 0; e < VEC; ++e) dot += bc[e] * x[e];
#pragma unroll
                    for (int o = LPN / 2; o > 0; o >>= 1) dot += __shfl_xor_sync(gmask, dot, o, LPN);
                    const FT sc = v / (dot > a.eps ? dot : a.eps);
#pragma unroll
                    for (int e = 0; e < VEC; ++e) acc[e] += x[e] * sc;
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(empty0 + 8 * sl);
        }
        if (cur != 0xffffffffu && live) gred<FT, VEC>(a.Phi + (size_t)cur * R + r0, acc);
    }
    if (!ok && lane == 0) atomicExch(a.err, 1u);
}

}  // namespace altob
