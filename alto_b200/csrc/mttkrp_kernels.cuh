// mttkrp_kernels.cuh -- MTTKRP and CP-APR Phi kernels on the ALTO stream.
//
// Reference kernels replaced (IntelLabs/ALTO) and the kernel that runs them:
//   mttkrp_alto_da_mem_pull   include/alto.hpp:1227-1318  -> k_planned (mttkrp_planned.cuh),
//                                                            k_grouped without a tile plan
//   mttkrp_alto_op_sched      include/alto.hpp:1320-1415  -> k_grouped reading through oidx
//   mttkrp_alto_atomic        include/alto.hpp:1030-1088  -> k_grouped without row slots
//   mttkrp_alto_atomic_cr     include/alto.hpp:1090-1158  -> k_atomic_cr
//   CalculatePhi_alto_*       include/apr.hpp:383-848     -> k_grouped<..., PHI=true>
//   batched MTTKRP (no counterpart)                       -> k_grouped_batch
//
// k_grouped (below, the default when no tile plan exists): a persistent CTA
// walks tiles of 1024 consecutive nonzeros of the ALTO-ordered stream (the
// GPU analogue of the reference's line segments), sorts each tile's records
// by output row in shared memory (slot claims, a scan, a counting-sort
// scatter), and lane groups walk runs of equal output rows keeping their sums
// in registers, one vector atomic per run (the reference's pull reduction).
// k_planned does the same with the tile order precomputed per mode.
//
// k_tiled (kept as an alternative: ALTOB_KERNEL other than 4): per-tile shared-memory
// accumulator rows claimed by output index, flushed once per tile.
#pragma once

#include "internal.cuh"

namespace altob {

constexpr int MT_THREADS = 256;
constexpr int MT_WARPS = MT_THREADS / 32;

template <typename FT, int VEC>
struct VecT;
template <>
struct VecT<float, 1> { typedef float T; };
template <>
struct VecT<float, 4> { typedef float4 T; };
template <>
struct VecT<double, 1> { typedef double T; };
template <>
struct VecT<double, 2> { typedef double2 T; };

template <typename FT, int VEC>
__device__ __forceinline__ void vload(const FT* p, FT* x)
{
    typedef typename VecT<FT, VEC>::T V;
    V v = __ldg(reinterpret_cast<const V*>(p));
    const FT* f = reinterpret_cast<const FT*>(&v);
#pragma unroll
    for (int e = 0; e < VEC; ++e) x[e] = f[e];
}

template <typename FT, int VEC>
__device__ __forceinline__ void vload_plain(const FT* p, FT* x)
{
    typedef typename VecT<FT, VEC>::T V;
    V v = *reinterpret_cast<const V*>(p);
    const FT* f = reinterpret_cast<const FT*>(&v);
#pragma unroll
    for (int e = 0; e < VEC; ++e) x[e] = f[e];
}

template <typename FT, int VEC>
__device__ __forceinline__ void vload_stream(const FT* p, FT* x)
{
    typedef typename VecT<FT, VEC>::T V;
    V v = __ldcs(reinterpret_cast<const V*>(p));
    const FT* f = reinterpret_cast<const FT*>(&v);
#pragma unroll
    for (int e = 0; e < VEC; ++e) x[e] = f[e];
}

template <typename FT, int VEC>
__device__ __forceinline__ void vstore_zero(FT* p)
{
    typedef typename VecT<FT, VEC>::T V;
    V z;
    FT* f = reinterpret_cast<FT*>(&z);
#pragma unroll
    for (int e = 0; e < VEC; ++e) f[e] = FT(0);
    *reinterpret_cast<V*>(p) = z;
}

// Global accumulate of VEC consecutive elements.
template <typename FT, int VEC>
__device__ __forceinline__ void gred(FT* p, const FT* x)
{
    if constexpr (sizeof(FT) == 4 && VEC == 4) {
        atomicAdd(reinterpret_cast<float4*>(p), make_float4(x[0], x[1], x[2], x[3]));
    } else {
#pragma unroll
        for (int e = 0; e < VEC; ++e) atomicAdd(p + e, x[e]);
    }
}

// y[e] = x[(e + r) % VEC] with r fixed per lane (branch-free selects).
template <typename FT, int VEC>
__device__ __forceinline__ void rotate(const FT* x, int r, FT* y)
{
    if constexpr (VEC == 1) {
        y[0] = x[0];
    } else if constexpr (VEC == 2) {
        const bool s = r & 1;
        y[0] = s ? x[1] : x[0];
        y[1] = s ? x[0] : x[1];
    } else {
        FT t[4];
        const bool s1 = r & 1, s2 = r & 2;
#pragma unroll
        for (int e = 0; e < 4; ++e) t[e] = s1 ? x[(e + 1) & 3] : x[e];
#pragma unroll
        for (int e = 0; e < 4; ++e) y[e] = s2 ? t[(e + 2) & 3] : t[e];
    }
}

// x[e] *= y[e]; FP32 pairs use the packed FP32x2 multiply of sm_100 (same
// IEEE round-to-nearest result as two scalar multiplies).
template <typename FT, int VEC>
__device__ __forceinline__ void vmul(FT* x, const FT* y)
{
    if constexpr (sizeof(FT) == 4 && VEC % 2 == 0) {
#pragma unroll
        for (int e = 0; e < VEC; e += 2) {
            const float2 r = __fmul2_rn(make_float2(x[e], x[e + 1]), make_float2(y[e], y[e + 1]));
            x[e] = r.x;
            x[e + 1] = r.y;
        }
    } else {
#pragma unroll
        for (int e = 0; e < VEC; ++e) x[e] *= y[e];
    }
}

// Index of the high-word run that contains nonzero g (uniform per tile).
__device__ __forceinline__ int run_of(const KeySrc& k, u64 g)
{
    int lo = 0, hi = k.nrun - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (k.run_start[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <typename FT>
struct TiledArgs {
    KeySrc key;
    const void* vals;
    const u32* perm;  // read order (oidx) or nullptr for ALTO order
    u64 nnz;
    u64 ntiles;
    int nmode;
    int target;
    int R;
    int tile;
    int hslots;  // power of two; 0 disables the row cache
    FT eps;      // Phi: eps_div_zero
    const FT* U[ALTOB_MAX_MODES];
    FT* out;
    Fields fld;
    int hot;       // per-CTA hot-row slots (power of two; 0: none), grouped kernel only
    FT* hot_acc;   // gridDim.x x hot x R accumulators, one private region per CTA
    const uint16_t* plan;  // tile plan of the target mode (planned kernel only)
    int hot_minrun;        // shortest run through the hot-row table (0: GT_HOT_MINRUN)
};

// Dynamic shared-memory bytes of k_tiled.
inline size_t tiled_smem(int nmode, int tile, int hslots, int R, size_t fsz)
{
    size_t b = (size_t)nmode * tile * 4 + (size_t)tile * 4;  // indices + slot
    b += (size_t)tile * fsz;                                  // values
    b = (b + 15) & ~(size_t)15;
    b += (size_t)hslots * 8;  // tag + used list
    b = (b + 15) & ~(size_t)15;
    b += (size_t)hslots * R * fsz;
    return b;
}

// NM: number of modes (0 = any, read from the arguments).  R <= LPN*VEC*CH.
template <typename FT, typename VT, int NM, int LPN, int VEC, int CH, bool PHI>
__global__ void __launch_bounds__(MT_THREADS) k_tiled(TiledArgs<FT> a)
{
    constexpr int MM = NM ? NM : ALTOB_MAX_MODES;
    constexpr int NPW = 32 / LPN;
    constexpr int UNR = 2;  // warp steps issued together in phase B
    extern __shared__ __align__(16) unsigned char smem[];
    const int tile = a.tile, R = a.R, H = a.hslots;
    const int nmode = NM ? NM : a.nmode;
    u32* crd = reinterpret_cast<u32*>(smem);
    int* slot = reinterpret_cast<int*>(crd + (size_t)nmode * tile);
    FT* val = reinterpret_cast<FT*>(slot + tile);
    size_t off = (size_t)nmode * tile * 4 + (size_t)tile * 4 + (size_t)tile * sizeof(FT);
    off = (off + 15) & ~(size_t)15;
    u32* tag = reinterpret_cast<u32*>(smem + off);
    u32* used = tag + H;
    off += (size_t)H * 8;
    off = (off + 15) & ~(size_t)15;
    FT* acc = reinterpret_cast<FT*>(smem + off);
    __shared__ u32 nused;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int k = tid; k < H; k += MT_THREADS) tag[k] = 0;
    for (size_t k = (size_t)tid; k < (size_t)H * R; k += MT_THREADS) acc[k] = FT(0);
    if (tid == 0) nused = 0;
    __syncthreads();

    const VT* vals = reinterpret_cast<const VT*>(a.vals);
    const int target = a.target;
    const int sub = lane % LPN, q = lane / LPN;
    const int rot = q % VEC;
    const int per_warp = tile / MT_WARPS;
    const u32 lt_mask = (1u << lane) - 1u;
    // the other modes' factor matrices and index rows (static register indices)
    const FT* Uo[MM - 1];
    int oo[MM - 1];
#pragma unroll
    for (int k = 0; k < MM - 1; ++k) {
        const int m = k < target ? k : k + 1;
        Uo[k] = a.U[k < target ? k : (k + 1 < MM ? k + 1 : k)];
        oo[k] = m * tile;
    }
    const int nother = nmode - 1;

    for (u64 ti = blockIdx.x; ti < a.ntiles; ti += gridDim.x) {
        // ---- phase A: load, read mode indices, claim accumulator rows
        const u64 g0 = ti * (u64)tile;
        // high key word: one compare per nonzero unless the tile spans
        // several runs (or reads through a permutation)
        u64 hcur = 0, hnext = 0, nstart = ~0ull;
        bool slow_hi = a.perm != nullptr;
        if (!a.key.khi && a.key.nrun && !slow_hi) {
            const int r = run_of(a.key, g0);
            hcur = a.key.run_val[r];
            if (r + 1 < a.key.nrun) {
                nstart = a.key.run_start[r + 1];
                hnext = a.key.run_val[r + 1];
                if (r + 2 < a.key.nrun && a.key.run_start[r + 2] < g0 + (u64)tile) slow_hi = true;
            }
        }
        for (int it = tid; it < tile; it += MT_THREADS) {
            const u64 g = g0 + it;
            int sl = -2;
            bool claimed = false;
            u32 h = 0;
            if (g < a.nnz) {
                const u64 pos = a.perm ? (u64)a.perm[g] : g;
                const u64 lo = a.key.klo[pos];
                const VT vv = vals[pos];
                u64 hi;
                if (a.key.khi) hi = a.key.khi[pos];
                else if (a.key.nrun == 0) hi = 0;
                else if (slow_hi) hi = key_hi(a.key, pos);
                else hi = g >= nstart ? hnext : hcur;
                val[it] = (FT)vv;
                u32 trow = 0;
#pragma unroll
                for (int m = 0; m < MM; ++m) {
                    if (NM == 0 && m >= nmode) break;
                    const u32 c = field(lo, hi, a.fld.pos[m], a.fld.mask[m]);
                    crd[(size_t)m * tile + it] = c;
                    if (m == target) trow = c;
                }
                sl = -1;
                if (H) {
                    h = trow & (u32)(H - 1);
                    const u32 old = atomicCAS(&tag[h], 0u, trow + 1u);
                    if (old == 0u) {
                        claimed = true;
                        sl = (int)h;
                    } else if (old == trow + 1u) {
                        sl = (int)h;
                    }
                }
            } else {
                // tail of the last tile: harmless index 0, value 0, no writes
#pragma unroll
                for (int m = 0; m < MM; ++m) {
                    if (NM == 0 && m >= nmode) break;
                    crd[(size_t)m * tile + it] = 0u;
                }
                val[it] = FT(0);
            }
            slot[it] = sl;
            // append this warp's claims to the list with one atomic
            const u32 cm = __ballot_sync(0xffffffffu, claimed);
            if (cm) {
                u32 base = 0;
                if (lane == 0) base = atomicAdd(&nused, (u32)__popc(cm));
                base = __shfl_sync(0xffffffffu, base, 0);
                if (claimed) used[base + __popc(cm & lt_mask)] = h;
            }
        }
        __syncthreads();

        // ---- phase B: gather factor rows (UNR steps in flight), accumulate
        for (int j = warp * per_warp; j < (warp + 1) * per_warp; j += NPW * UNR) {
            int its[UNR], sls[UNR];
            FT vs[UNR];
            FT x[UNR][CH][VEC];
#pragma unroll
            for (int u = 0; u < UNR; ++u) {
                its[u] = j + u * NPW + q;
                sls[u] = slot[its[u]];  // -2: no nonzero (kept for the Phi shuffles)
                vs[u] = val[its[u]];
#pragma unroll
                for (int ch = 0; ch < CH; ++ch)
#pragma unroll
                    for (int e = 0; e < VEC; ++e) x[u][ch][e] = PHI ? FT(1) : vs[u];
            }
            FT y[UNR][MM - 1][CH][VEC];
#pragma unroll
            for (int k = 0; k < MM - 1; ++k) {
                if (NM == 0 && k >= nother) break;
#pragma unroll
                for (int u = 0; u < UNR; ++u) {
                    const FT* row = Uo[k] + (size_t)crd[oo[k] + its[u]] * R;
#pragma unroll
                    for (int ch = 0; ch < CH; ++ch) {
                        const int r0 = ch * LPN * VEC + sub * VEC;
                        if (r0 < R) vload<FT, VEC>(row + r0, y[u][k][ch]);
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < MM - 1; ++k) {
                if (NM == 0 && k >= nother) break;
#pragma unroll
                for (int u = 0; u < UNR; ++u)
#pragma unroll
                    for (int ch = 0; ch < CH; ++ch) {
                        const int r0 = ch * LPN * VEC + sub * VEC;
                        if (r0 < R) vmul<FT, VEC>(x[u][ch], y[u][k][ch]);
                    }
            }
#pragma unroll
            for (int u = 0; u < UNR; ++u) {
                const u32 trow = crd[(size_t)target * tile + its[u]];
                if constexpr (PHI) {
                    // v / max(<B[trow,:], krp>, eps), apr.hpp:452-462
                    const FT* brow = a.U[target] + (size_t)trow * R;
                    FT dot = FT(0);
#pragma unroll
                    for (int ch = 0; ch < CH; ++ch) {
                        const int r0 = ch * LPN * VEC + sub * VEC;
                        if (r0 < R) {
                            FT b[VEC];
                            vload<FT, VEC>(brow + r0, b);
#pragma unroll
                            for (int e = 0; e < VEC; ++e) dot += b[e] * x[u][ch][e];
                        }
                    }
#pragma unroll
                    for (int o = LPN / 2; o > 0; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o, LPN);
                    const FT sc = vs[u] / (dot > a.eps ? dot : a.eps);
#pragma unroll
                    for (int ch = 0; ch < CH; ++ch)
#pragma unroll
                        for (int e = 0; e < VEC; ++e) x[u][ch][e] *= sc;
                }
                const int sl = sls[u];
                if (sl == -2) continue;
#pragma unroll
                for (int ch = 0; ch < CH; ++ch) {
                    const int r0 = ch * LPN * VEC + sub * VEC;
                    if (r0 < R) {
                        if (sl >= 0) {
                            FT z[VEC];
                            rotate<FT, VEC>(x[u][ch], rot, z);
                            FT* dst = acc + (size_t)sl * R + r0;
#pragma unroll
                            for (int e = 0; e < VEC; ++e) atomicAdd(dst + ((e + rot) % VEC), z[e]);
                        } else {
                            gred<FT, VEC>(a.out + (size_t)trow * R + r0, x[u][ch]);
                        }
                    }
                }
            }
        }
        __syncthreads();

        // ---- phase C: flush claimed rows (NPW rows per warp step)
        if (H) {
            const u32 nu = nused;
            for (u32 k = (u32)warp * NPW; k < nu; k += MT_WARPS * NPW) {
                const u32 kk = k + q;
                if (kk < nu) {
                    const u32 hh = used[kk];
                    FT* src = acc + (size_t)hh * R;
                    FT* dst = a.out + (size_t)(tag[hh] - 1u) * R;
#pragma unroll
                    for (int ch = 0; ch < CH; ++ch) {
                        const int r0 = ch * LPN * VEC + sub * VEC;
                        if (r0 < R) {
                            FT z[VEC];
                            vload_plain<FT, VEC>(src + r0, z);
                            gred<FT, VEC>(dst + r0, z);
                            vstore_zero<FT, VEC>(src + r0);
                        }
                    }
                }
            }
            __syncthreads();
            for (u32 k = tid; k < nu; k += MT_THREADS) tag[used[k]] = 0;
            __syncthreads();
            if (tid == 0) nused = 0;
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------- k_grouped
//
// Second MTTKRP / Phi kernel: no shared-memory accumulators at all.  Per tile
// of GT_TILE nonzeros:
//   A1  load keys and values (coalesced), form one record per nonzero
//       (mode indices + value) in registers, claim a slot for the output
//       row in a direct-mapped tag table, and take a rank inside the slot
//       with one atomic per group of equal slots in a warp (match_any);
//   A2  exclusive scan of the slot counts in claim order;
//   A3  write each record once to shared memory at its place in slot order
//       (a counting sort), so nonzeros with the same output row are
//       contiguous;
//   B   each lane group walks a contiguous range of the sorted list, gathers
//       the other modes' rows, keeps the running sum of equal output rows in
//       registers and adds each finished run to global memory with one
//       vector atomic.
// Nonzeros whose slot is held by another row form single-element runs.
// The run is the reference's fiber and the flush its pull.

constexpr int GT_TILE = 1024;
constexpr int GT_IPT = GT_TILE / MT_THREADS;
// Streaming (evict-first) loads for data read once per launch (the key/value
// stream, precomputed Khatri-Rao rows), so L2 keeps the gathered factor rows.
__device__ __forceinline__ float ldcs_val(const float* p) { return __ldcs(p); }
__device__ __forceinline__ double ldcs_val(const double* p) { return __ldcs(p); }
__device__ __forceinline__ u32 ldcs_val(const u32* p) { return __ldcs(reinterpret_cast<const unsigned int*>(p)); }

// L2 prefetch of one row (R elements).  Phase A of the precomputed-row Phi
// kernel issues it for the rows phase B will read, so they arrive from DRAM
// while the tile is being sorted (measured: +9 % on CP-APR; the factor-row
// gathers of MTTKRP are mostly L2 hits and lose 7 % to the extra issue).
template <typename FT>
__device__ __forceinline__ void prefetch_row(const FT* p, int R)
{
    const char* c = reinterpret_cast<const char*>(p);
    for (int off = 0; off < R * (int)sizeof(FT); off += 128) asm volatile("prefetch.global.L2 [%0];" ::"l"(c + off));
}

// Nonzeros a lane group takes per step in the run phase of the grouped kernels.
#ifndef GT_NZS
#define GT_NZS 2
#endif

// Resident blocks per SM that a grouped kernel instance is compiled for (a
// register cap of 65536 / (256 n); 0: the compiler's own choice).  The
// kernel is latency-bound: the order-3 FP32 MTTKRP with its records in
// registers takes 2.88 ms per mode at 4 blocks (64 registers) against 3.27 ms
// at 3 (the 3-mode Zipf tensor, 100.8M nonzeros, rank 32).  Order 5 (3
// blocks), the generic-order two-chunk instances (2) and the precomputed-row
// Phi (4) are held at the occupancy they had with every record staged in
// shared memory; order 4 reaches 4 blocks uncapped.
template <typename FT, int NM, int CH, bool PHI>
constexpr int grouped_min_blocks()
{
    if (sizeof(FT) != 4) return 0;
    if (NM == 0 && CH == 2) return 2;
    if (CH != 1) return 0;
    if (NM == 1) return 4;
    if (PHI) return 0;
    return NM == 3 ? 4 : NM == 5 ? 3 : 0;
}

// Record modes of a grouped kernel instance: NM = 3..5 (static order), 0
// (any order, loops bounded at run time) or 1 (precomputed Khatri-Rao rows:
// records hold the target row and the nonzero's position).
template <int NM>
constexpr int grouped_mm()
{
    return NM == 1 ? 2 : NM ? NM : ALTOB_MAX_MODES;
}

// 32-bit words of one shared record: output index, the other modes' indices,
// the value, padding to 16 B.
template <typename FT, int MM>
struct RecWords {
    static constexpr int n = (MM + (int)(sizeof(FT) / 4) + 3) & ~3;
};

inline size_t grouped_smem(int hslots, int mm, size_t fsz, int hot = 0, int R = 0)
{
    const int rw = (mm + (int)(fsz / 4) + 3) & ~3;
    size_t b = (size_t)(GT_TILE + GT_TILE / 32) * rw * 4;  // records in run order (padded)
    if (rw > 4) b += (size_t)GT_TILE * rw * 4;             // records in stream order
    b += (size_t)hslots * 8;                  // tags + counts
    b += (size_t)GT_TILE * 4;                 // claimed-slot list
    b += (size_t)hot * 4;                     // hot-row tags
    (void)R;
    return b;
}

// Runs shorter than GT_HOT_MINRUN nonzeros skip the hot-row lookup (rows
// that are hot fill long runs in a tile).
#ifndef GT_HOT_MINRUN
#define GT_HOT_MINRUN 8
#endif

// Hot-row cache of the grouped kernel: per CTA, `hot` direct-mapped rows
// (row & (hot - 1), claimed first come, tags in shared memory) whose run sums
// go to a region of global memory private to the CTA (L2-resident, no
// contention) and reach the output once per CTA instead of once per tile.
// Rows that many tiles touch (the head of a skewed mode) then take a few
// hundred FP32 additions instead of one per tile, which keeps their rounding
// error near the per-tile level.  16 KB per CTA; FP32 only.
inline int grouped_hot_slots(int R, size_t fsz)
{
    if (fsz != 4 || R < 1) return 0;
    int h = 1;
    while (h * 2 <= 256 && (size_t)(h * 2) * R * fsz <= 16384) h *= 2;
    return h >= 16 ? h : 0;
}

// Slot of run-ordered record p: one padding record after every 32, so the
// stretches that the lane groups of a warp read at the same time start in
// different 16-byte bank groups (unpadded they are 512 bytes apart: one bank
// group, a 4-way conflict on every record load).
__device__ __forceinline__ int rslot(int p) { return p + (p >> 5); }
// The same with one padding record after every 2^PSH (stretches of 2^PSH
// records per lane group).
template <int PSH>
__device__ __forceinline__ int rslot_t(int p) { return p + (p >> PSH); }
constexpr int GT_SREC = GT_TILE + GT_TILE / 32;  // run-ordered record slots

template <typename FT, int RW>
__device__ __forceinline__ void load_rec(const u32* r, u32* w)
{
#pragma unroll
    for (int w4 = 0; w4 < RW; w4 += 4) {
        const uint4 t4 = *reinterpret_cast<const uint4*>(r + w4);
        w[w4] = t4.x;
        w[w4 + 1] = t4.y;
        w[w4 + 2] = t4.z;
        w[w4 + 3] = t4.w;
    }
}

template <typename FT, int MM>
__device__ __forceinline__ FT rec_val(const u32* w)
{
    if constexpr (sizeof(FT) == 4) return (FT)__uint_as_float(w[MM]);
    else return (FT)__longlong_as_double((long long)(((unsigned long long)w[MM + 1] << 32) | w[MM]));
}

struct GroupedSmem {
    u32* srec;
    u32* rec;  // records in stream order (records wider than 4 words only)
    u32* tag;
    u32* cnt;
    u32* used;
    u32* htag;   // hot-row tags (row + 1; 0 free)
    u32* nused;
    u32* ndirect;
    u32* wsum;
};

// One run sum into its output row: into the CTA's hot-row slot when the row
// holds (or can claim) it, else with vector atomics into the output.
template <typename FT, int VEC, int CH, int LPN>
__device__ __forceinline__ void flush_run(FT* out, const GroupedSmem& gs, int hot, FT* hot_acc, unsigned gmask,
                                          u32 row, int R, int sub, FT (*racc)[VEC])
{
    if (hot) {
        const u32 sl = row & (u32)(hot - 1);
        u32 tg = 0;
        if (sub == 0) {
            tg = gs.htag[sl];
            if (tg == 0u) {
                const u32 old = atomicCAS(&gs.htag[sl], 0u, row + 1u);
                tg = old == 0u ? row + 1u : old;
            }
        }
        tg = __shfl_sync(gmask, tg, __ffs(gmask) - 1);
        if (tg == row + 1u) {
            FT* h = hot_acc + ((size_t)blockIdx.x * hot + sl) * R;
#pragma unroll
            for (int ch = 0; ch < CH; ++ch) {
                const int r0 = ch * LPN * VEC + sub * VEC;
                if (r0 < R) gred<FT, VEC>(h + r0, racc[ch]);
            }
            return;
        }
    }
#pragma unroll
    for (int ch = 0; ch < CH; ++ch) {
        const int r0 = ch * LPN * VEC + sub * VEC;
        if (r0 < R) gred<FT, VEC>(out + (size_t)row * R + r0, racc[ch]);
    }
}

// One nonzero of a lane group: val * (Khatri-Rao row of the other modes), or
// the Phi contribution.  Record words: [target index, other indices..., value].
template <typename FT, int MM, int NM, int LPN, int VEC, int CH, bool PHI>
__device__ __forceinline__ void nz_row(const u32* w, const FT* const* Uo, const FT* Ut, int R, int sub, int nother,
                                       FT eps, unsigned gmask, FT (*x)[VEC])
{
    const FT v = rec_val<FT, MM>(w);
#pragma unroll
    for (int ch = 0; ch < CH; ++ch)
#pragma unroll
        for (int e = 0; e < VEC; ++e) x[ch][e] = PHI ? FT(1) : v;
    FT y[MM - 1][CH][VEC];
#pragma unroll
    for (int k = 0; k < MM - 1; ++k) {
        if (NM == 0 && k >= nother) break;
        const FT* row = Uo[k] + (size_t)w[1 + k] * R;
#pragma unroll
        for (int ch = 0; ch < CH; ++ch) {
            const int r0 = ch * LPN * VEC + sub * VEC;
            if (r0 < R) {
                if constexpr (NM == 1) vload_stream<FT, VEC>(row + r0, y[k][ch]);  // precomputed row, read once
                else vload<FT, VEC>(row + r0, y[k][ch]);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < MM - 1; ++k) {
        if (NM == 0 && k >= nother) break;
#pragma unroll
        for (int ch = 0; ch < CH; ++ch) {
            const int r0 = ch * LPN * VEC + sub * VEC;
            if (r0 < R) vmul<FT, VEC>(x[ch], y[k][ch]);
        }
    }
    if constexpr (PHI) {
        const FT* brow = Ut + (size_t)w[0] * R;
        FT dot = FT(0);
#pragma unroll
        for (int ch = 0; ch < CH; ++ch) {
            const int r0 = ch * LPN * VEC + sub * VEC;
            if (r0 < R) {
                FT b[VEC];
                vload<FT, VEC>(brow + r0, b);
#pragma unroll
                for (int e = 0; e < VEC; ++e) dot += b[e] * x[ch][e];
            }
        }
#pragma unroll
        for (int o = LPN / 2; o > 0; o >>= 1) dot += __shfl_xor_sync(gmask, dot, o, LPN);
        const FT sc = v / (dot > eps ? dot : eps);
#pragma unroll
        for (int ch = 0; ch < CH; ++ch)
#pragma unroll
            for (int e = 0; e < VEC; ++e) x[ch][e] *= sc;
    }
}

template <typename FT, int VEC, int CH>
__device__ __forceinline__ void run_add(FT (*racc)[VEC], FT (*x)[VEC])
{
#pragma unroll
    for (int ch = 0; ch < CH; ++ch) {
        if constexpr (sizeof(FT) == 4 && VEC % 2 == 0) {
#pragma unroll
            for (int e = 0; e < VEC; e += 2) {
                const float2 r = __fadd2_rn(make_float2(racc[ch][e], racc[ch][e + 1]), make_float2(x[ch][e], x[ch][e + 1]));
                racc[ch][e] = r.x;
                racc[ch][e + 1] = r.y;
            }
        } else {
#pragma unroll
            for (int e = 0; e < VEC; ++e) racc[ch][e] += x[ch][e];
        }
    }
}

// Phase B of the MTTKRP for a static order and one VEC-wide chunk per lane:
// the lane group walks its stretch [p0, pe) of the run-ordered records two at
// a time (both records' gathers issued before either is added), forms
// v * row_1 * ... * row_{N-1} in the order of nz_row, and keeps the run sum
// of its current output row in registers.  The same arithmetic as the
// generic loop, written so that the per-nonzero work is the record load, the
// row loads with 32-bit-operand address products, the products and the run
// test (23% fewer instructions and 28% less time on the 3-mode Zipf tensor).
template <typename FT, int MM, int LPN, int VEC, int PSH = 5>
__device__ __forceinline__ void lean_runs(const TiledArgs<FT>& a, const GroupedSmem& gs, const FT* const* Uo,
                                          int p0, int pe, int R, int sub, unsigned gmask)
{
    constexpr int RW = RecWords<FT, MM>::n;
    const u32 Ru = (u32)R;
    // Lanes past the rank (R below LPN * VEC) load the row's last elements,
    // so every load stays inside its row; flush_run writes only r0 < R.
    const int col = min(sub * VEC, R - VEC);
    const FT* Ub[MM - 1];
#pragma unroll
    for (int k = 0; k < MM - 1; ++k) Ub[k] = Uo[k] + col;
    u32 cur = 0xffffffffu;
    int len = 0;
    const int hmin = a.hot_minrun ? a.hot_minrun : GT_HOT_MINRUN;
    FT acc[1][VEC];
#pragma unroll
    for (int e = 0; e < VEC; ++e) acc[0][e] = FT(0);
    auto add = [&](const u32* w, FT (*y)[VEC]) {
        const FT v = rec_val<FT, MM>(w);
        FT x[1][VEC];
#pragma unroll
        for (int e = 0; e < VEC; ++e) x[0][e] = v;
#pragma unroll
        for (int k = 0; k < MM - 1; ++k) vmul<FT, VEC>(x[0], y[k]);
        if (w[0] != cur) {
            if (cur != 0xffffffffu)
                flush_run<FT, VEC, 1, LPN>(a.out, gs, len >= hmin ? a.hot : 0, a.hot_acc, gmask, cur, R,
                                           sub, acc);
            cur = w[0];
            len = 1;
#pragma unroll
            for (int e = 0; e < VEC; ++e) acc[0][e] = x[0][e];
        } else {
            run_add<FT, VEC, 1>(acc, x);
            ++len;
        }
    };
    int p = p0;
    for (; p + 1 < pe; p += 2) {
        u32 w0[RW], w1[RW];
        load_rec<FT, RW>(gs.srec + (size_t)rslot_t<PSH>(p) * RW, w0);
        load_rec<FT, RW>(gs.srec + (size_t)rslot_t<PSH>(p + 1) * RW, w1);
        FT y0[MM - 1][VEC], y1[MM - 1][VEC];
#pragma unroll
        for (int k = 0; k < MM - 1; ++k) {
            vload<FT, VEC>(Ub[k] + (size_t)w0[1 + k] * Ru, y0[k]);
            vload<FT, VEC>(Ub[k] + (size_t)w1[1 + k] * Ru, y1[k]);
        }
        add(w0, y0);
        add(w1, y1);
    }
    if (p < pe) {
        u32 w0[RW];
        load_rec<FT, RW>(gs.srec + (size_t)rslot_t<PSH>(p) * RW, w0);
        FT y0[MM - 1][VEC];
#pragma unroll
        for (int k = 0; k < MM - 1; ++k) vload<FT, VEC>(Ub[k] + (size_t)w0[1 + k] * Ru, y0[k]);
        add(w0, y0);
    }
    if (cur != 0xffffffffu)
        flush_run<FT, VEC, 1, LPN>(a.out, gs, len >= hmin ? a.hot : 0, a.hot_acc, gmask, cur, R, sub, acc);
}

// Shared-memory work areas of the grouped kernels (tags and counts must be
// zero between tiles; grouped_tile leaves them zero).

template <typename FT, int MM>
__device__ __forceinline__ GroupedSmem grouped_smem_ptrs(unsigned char* smem, int H, u32* statics, int hot = 0)
{
    constexpr int RW = RecWords<FT, MM>::n;
    GroupedSmem g;
    g.srec = reinterpret_cast<u32*>(smem);
    g.rec = RW > 4 ? g.srec + (size_t)GT_SREC * RW : nullptr;
    g.tag = g.srec + (size_t)GT_SREC * RW + (RW > 4 ? (size_t)GT_TILE * RW : 0);
    g.cnt = g.tag + H;
    g.used = g.cnt + H;
    g.htag = g.used + GT_TILE;
    (void)hot;
    g.nused = statics;
    g.ndirect = statics + 1;
    g.wsum = statics + 2;
    return g;
}

__device__ __forceinline__ void grouped_init(const GroupedSmem& g, int H)
{
    for (int k = threadIdx.x; k < H; k += MT_THREADS) {
        g.tag[k] = 0;
        g.cnt[k] = 0;
    }
    if (threadIdx.x == 0) {
        *g.nused = 0;
        *g.ndirect = 0;
    }
    __syncthreads();
}

// One tile of nonzeros [ti * GT_TILE, ...) of the tensor described by `a`.
template <typename FT, typename VT, int NM, int LPN, int VEC, int CH, bool PHI>
__device__ __forceinline__ void grouped_tile(const TiledArgs<FT>& a, u64 ti, const GroupedSmem& gs)
{
    constexpr bool PRE = NM == 1;  // a.U[0]: precomputed rows (nnz x R), a.U[1]: target factor
    constexpr int MM = grouped_mm<NM>();
    constexpr int NPW = 32 / LPN;
    constexpr int RW = RecWords<FT, MM>::n;
    constexpr int NGRP = MT_WARPS * NPW;
    constexpr int IPG = GT_TILE / NGRP;  // sorted nonzeros per lane group
    constexpr int FW = (int)(sizeof(FT) / 4);
    const int R = a.R, H = a.hslots;
    const int nmode = PRE ? 2 : NM ? NM : a.nmode;
    u32* srec = gs.srec;
    u32* tag = gs.tag;
    u32* cnt = gs.cnt;
    u32* used = gs.used;
    u32& nused = *gs.nused;
    u32& ndirect = *gs.ndirect;
    u32* wsum = gs.wsum;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const VT* vals = reinterpret_cast<const VT*>(a.vals);
    const int target = a.target;
    const int sub = lane % LPN, q = lane / LPN;
    const int grp = warp * NPW + q;
    const unsigned gmask = (0xffffffffu >> (32 - LPN)) << (q * LPN);
    const u32 lt_mask = (1u << lane) - 1u;
    const FT* Uo[MM - 1];
    if constexpr (PRE) {
        Uo[0] = a.U[0];
    } else {
#pragma unroll
        for (int k = 0; k < MM - 1; ++k) Uo[k] = a.U[k < target ? k : (k + 1 < MM ? k + 1 : k)];
    }
    const FT* Ut = PRE ? a.U[1] : a.U[target];
    const int nother = nmode - 1;
    const u64 g0 = ti * (u64)GT_TILE;
    const int nvalid = (int)min((u64)GT_TILE, a.nnz - g0);
    u64 hcur = 0, hnext = 0, nstart = ~0ull;
    bool slow_hi = a.perm != nullptr;
    if (!a.key.khi && a.key.nrun && !slow_hi) {
        const int r = run_of(a.key, g0);
        hcur = a.key.run_val[r];
        if (r + 1 < a.key.nrun) {
            nstart = a.key.run_start[r + 1];
            hnext = a.key.run_val[r + 1];
            if (r + 2 < a.key.nrun && a.key.run_start[r + 2] < g0 + (u64)GT_TILE) slow_hi = true;
        }
    }
    // ---- A1: records [target, others..., value], slot claims, ranks.
    // Records of 4 words stay in registers until A3 writes them once, in run
    // order; wider ones are staged in shared memory (a thread's GT_IPT wide
    // records held in registers would cost occupancy).
    u64 lo[GT_IPT];
    u32 pv[GT_IPT];  // read position when reading through a permutation
    VT vv[GT_IPT];
#pragma unroll
    for (int k = 0; k < GT_IPT; ++k) {
        const int it = tid + k * MT_THREADS;
        const u64 g = g0 + it;
        pv[k] = 0;
        if (it < nvalid) {
            if (a.perm) pv[k] = a.perm[g];
            const u64 pos = a.perm ? (u64)pv[k] : g;
            if (!a.perm) {  // the stream is read once: keep L2 for factor rows
                lo[k] = __ldcs(reinterpret_cast<const unsigned long long*>(a.key.klo) + pos);
                vv[k] = ldcs_val(vals + pos);
            } else {
                lo[k] = a.key.klo[pos];
                vv[k] = vals[pos];
            }
        }
    }
    constexpr bool REGREC = RW == 4;
    // slot and rank inside the slot (or among the direct nonzeros); packed as
    // (slot + 2) << 16 | rank when the records are in registers (fewer live
    // registers there, more in the shared-memory form)
    u32 slr[GT_IPT];
    int slv[GT_IPT];
    u32 rankv[GT_IPT];
    u32 rg[GT_IPT][RW];  // the records (static indices only: registers)
#pragma unroll
    for (int k = 0; k < GT_IPT; ++k) {
        const int it = tid + k * MT_THREADS;
        const u64 g = g0 + it;
        int sl = -2;
        bool claimed = false;
        u32 h = 0;
#pragma unroll
        for (int w = 0; w < RW; ++w) rg[k][w] = 0u;
        if (it < nvalid) {
            const u64 pos = a.perm ? (u64)pv[k] : g;
            u64 hi;
            if (a.key.khi) hi = a.key.khi[pos];
            else if (a.key.nrun == 0) hi = 0;
            else if (slow_hi) hi = key_hi(a.key, pos);
            else hi = g >= nstart ? hnext : hcur;
            if constexpr (!REGREC) {
                // wide records: each word straight to shared memory (word 0:
                // the target index; then the other modes in order; the value)
                u32* r = gs.rec + (size_t)it * RW;
                u32 trow = 0;
#pragma unroll
                for (int m = 0; m < MM; ++m) {
                    if (NM == 0 && m >= nmode) break;
                    const u32 c = field(lo[k], hi, a.fld.pos[m], a.fld.mask[m]);
                    r[m == target ? 0 : (m < target ? m + 1 : m)] = c;
                    if (m == target) trow = c;
                }
                rg[k][0] = trow;
                const FT fv = (FT)vv[k];
                if constexpr (FW == 1) {
                    r[MM] = __float_as_uint((float)fv);
                } else {
                    const unsigned long long b = (unsigned long long)__double_as_longlong((double)fv);
                    r[MM] = (u32)b;
                    r[MM + 1] = (u32)(b >> 32);
                }
            } else {
                if constexpr (PRE) {
                    rg[k][0] = field(lo[k], hi, a.fld.pos[target], a.fld.mask[target]);
                    rg[k][1] = (u32)pos;
                    // the precomputed row comes from DRAM: start fetching it now
                    prefetch_row<FT>(Uo[0] + (size_t)pos * R, R);
                } else {
                    // word 0: the target index; word s >= 1: mode s-1 below
                    // the target, mode s above it
                    u32 c[MM];
#pragma unroll
                    for (int m = 0; m < MM; ++m)
                        c[m] = (NM == 0 && m >= nmode) ? 0u : field(lo[k], hi, a.fld.pos[m], a.fld.mask[m]);
                    u32 trow = c[0];
#pragma unroll
                    for (int m = 1; m < MM; ++m)
                        if (m == target) trow = c[m];
                    rg[k][0] = trow;
#pragma unroll
                    for (int s = 1; s < MM; ++s) rg[k][s] = s - 1 < target ? c[s - 1] : c[s];
                }
                const FT fv = (FT)vv[k];
                if constexpr (FW == 1) {
                    rg[k][MM] = __float_as_uint((float)fv);
                } else {
                    const unsigned long long b = (unsigned long long)__double_as_longlong((double)fv);
                    rg[k][MM] = (u32)b;
                    rg[k][MM + 1] = (u32)(b >> 32);
                }
            }
            sl = -1;
            h = rg[k][0] & (u32)(H - 1);
            if constexpr (!REGREC) {
                if (H) {
                    const u32 old = atomicCAS(&tag[h], 0u, rg[k][0] + 1u);
                    if (old == 0u) {
                        claimed = true;
                        sl = (int)h;
                    } else if (old == rg[k][0] + 1u) {
                        sl = (int)h;
                    }
                }
            }
        }
        u32 peers;
        if constexpr (REGREC) {
            // lanes with the same output row form one group (rows are below
            // 0xffffffff: the tags store row + 1); its first lane claims the
            // slot for all of them, so a row repeated across the warp (the
            // head of a skewed mode) costs one compare-and-swap, not one per
            // nonzero
            peers = __match_any_sync(0xffffffffu, sl == -2 ? 0xffffffffu : rg[k][0]);
            const int leader = __ffs(peers) - 1;
            if (H) {
                u32 old = 0;
                if (sl == -1 && lane == leader) old = atomicCAS(&tag[h], 0u, rg[k][0] + 1u);
                old = __shfl_sync(0xffffffffu, old, leader);
                if (sl == -1) {
                    if (old == 0u) {
                        claimed = lane == leader;
                        sl = (int)h;
                    } else if (old == rg[k][0] + 1u) {
                        sl = (int)h;
                    }
                }
            }
        } else {
            // one compare-and-swap per nonzero (above), then groups of equal
            // slots (fewer registers than grouping first: wide records)
            peers = __match_any_sync(0xffffffffu, sl >= 0 ? (u32)sl : (0x80000000u | (u32)lane));
        }
        const int leader = __ffs(peers) - 1;
        const u32 cm = __ballot_sync(0xffffffffu, claimed);
        if (cm) {
            u32 base = 0;
            if (lane == 0) base = atomicAdd(&nused, (u32)__popc(cm));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (claimed) used[base + __popc(cm & lt_mask)] = h;
        }
        u32 base = 0;
        if (sl >= 0 && lane == leader) base = atomicAdd(&cnt[sl], (u32)__popc(peers));
        base = __shfl_sync(0xffffffffu, base, leader);
        u32 rank = base + __popc(peers & lt_mask);
        const u32 dm = __ballot_sync(0xffffffffu, sl == -1);
        if (dm) {
            u32 db = 0;
            if (lane == 0) db = atomicAdd(&ndirect, (u32)__popc(dm));
            db = __shfl_sync(0xffffffffu, db, 0);
            if (sl == -1) rank = db + __popc(dm & lt_mask);
        }
        if constexpr (REGREC) {
            slr[k] = ((u32)(sl + 2) << 16) | rank;
        } else {
            slv[k] = sl;
            rankv[k] = rank;
        }
    }
    __syncthreads();
    // ---- A2: exclusive scan of the counts in claim order
    const u32 nu = nused;
    {
        u32 c[GT_IPT], sum = 0;
#pragma unroll
        for (int k = 0; k < GT_IPT; ++k) {
            const u32 e = (u32)(tid * GT_IPT + k);
            c[k] = e < nu ? cnt[used[e]] : 0u;
            sum += c[k];
        }
        u32 xs = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const u32 y = __shfl_up_sync(0xffffffffu, xs, o);
            if (lane >= o) xs += y;
        }
        if (lane == 31) wsum[warp] = xs;
        __syncthreads();
        u32 wbase = 0;
#pragma unroll
        for (int w = 0; w < MT_WARPS; ++w)
            if (w < warp) wbase += wsum[w];
        u32 run = wbase + xs - sum;
#pragma unroll
        for (int k = 0; k < GT_IPT; ++k) {
            const u32 e = (u32)(tid * GT_IPT + k);
            if (e < nu) {
                const u32 hh = used[e];
                tag[hh] = 0;    // tags are not read again in this tile
                cnt[hh] = run;  // count -> start offset
            }
            run += c[k];
        }
    }
    __syncthreads();
    // ---- A3: records into run order (counting-sort scatter)
    u32 slotted = 0;
#pragma unroll
    for (int w = 0; w < MT_WARPS; ++w) slotted += wsum[w];
#pragma unroll
    for (int k = 0; k < GT_IPT; ++k) {
        const int it = tid + k * MT_THREADS;
        if (it < nvalid) {
            const int sl = REGREC ? (int)(slr[k] >> 16) - 2 : slv[k];
            const u32 rank = REGREC ? slr[k] & 0xffffu : rankv[k];
            const u32 pos = sl >= 0 ? cnt[sl] + rank : slotted + rank;
            u32* dst = srec + (size_t)rslot((int)pos) * RW;
            if constexpr (REGREC) {
                *reinterpret_cast<uint4*>(dst) = make_uint4(rg[k][0], rg[k][1], rg[k][2], rg[k][3]);
            } else {
                const u32* src = gs.rec + (size_t)it * RW;
#pragma unroll
                for (int w4 = 0; w4 < RW; w4 += 4)
                    *reinterpret_cast<uint4*>(dst + w4) = *reinterpret_cast<const uint4*>(src + w4);
            }
        }
    }
    __syncthreads();
    // ---- B: runs of equal output rows, one atomic per run
    u32 prow = 0xffffffffu;
    int rlen = 0;  // nonzeros in the current run
    FT racc[CH][VEC];
#pragma unroll
    for (int ch = 0; ch < CH; ++ch)
#pragma unroll
        for (int e = 0; e < VEC; ++e) racc[ch][e] = FT(0);
    const int p0 = grp * IPG;
    const int pend = min(p0 + IPG, nvalid);
    if constexpr (!PHI && NM >= 3 && CH == 1) {
        lean_runs<FT, MM, LPN, VEC>(a, gs, Uo, p0, pend, R, sub, gmask);
        __syncthreads();
        for (u32 e = tid; e < nu; e += MT_THREADS) cnt[used[e]] = 0;
        if (tid == 0) {
            nused = 0;
            ndirect = 0;
        }
        __syncthreads();
        return;
    }
    int p = p0;
    // GT_NZS nonzeros per step: all their gathers in flight before the run logic
    for (; p + GT_NZS - 1 < pend; p += GT_NZS) {
        u32 w[GT_NZS][RW];
#pragma unroll
        for (int q = 0; q < GT_NZS; ++q) load_rec<FT, RW>(srec + (size_t)rslot(p + q) * RW, w[q]);
        FT x[GT_NZS][CH][VEC];
#pragma unroll
        for (int q = 0; q < GT_NZS; ++q)
            nz_row<FT, MM, NM, LPN, VEC, CH, PHI>(w[q], Uo, Ut, R, sub, nother, a.eps, gmask, x[q]);
#pragma unroll
        for (int q = 0; q < GT_NZS; ++q) {
            if (w[q][0] != prow) {
                if (prow != 0xffffffffu) flush_run<FT, VEC, CH, LPN>(a.out, gs, rlen >= GT_HOT_MINRUN ? a.hot : 0, a.hot_acc, gmask, prow, R, sub, racc);
                prow = w[q][0];
                rlen = 1;
#pragma unroll
                for (int ch = 0; ch < CH; ++ch)
#pragma unroll
                    for (int e = 0; e < VEC; ++e) racc[ch][e] = x[q][ch][e];
            } else {
                run_add<FT, VEC, CH>(racc, x[q]);
                ++rlen;
            }
        }
    }
    for (; p < pend; ++p) {
        u32 w0[RW];
        load_rec<FT, RW>(srec + (size_t)rslot(p) * RW, w0);
        FT x0[CH][VEC];
        nz_row<FT, MM, NM, LPN, VEC, CH, PHI>(w0, Uo, Ut, R, sub, nother, a.eps, gmask, x0);
        if (w0[0] != prow) {
            if (prow != 0xffffffffu) flush_run<FT, VEC, CH, LPN>(a.out, gs, rlen >= GT_HOT_MINRUN ? a.hot : 0, a.hot_acc, gmask, prow, R, sub, racc);
            prow = w0[0];
            rlen = 1;
#pragma unroll
            for (int ch = 0; ch < CH; ++ch)
#pragma unroll
                for (int e = 0; e < VEC; ++e) racc[ch][e] = x0[ch][e];
        } else {
            run_add<FT, VEC, CH>(racc, x0);
            ++rlen;
        }
    }
    if (prow != 0xffffffffu) flush_run<FT, VEC, CH, LPN>(a.out, gs, rlen >= GT_HOT_MINRUN ? a.hot : 0, a.hot_acc, gmask, prow, R, sub, racc);
    __syncthreads();
    // counts back to zero for the next tile (tags were cleared in A2)
    for (u32 e = tid; e < nu; e += MT_THREADS) cnt[used[e]] = 0;
    if (tid == 0) {
        nused = 0;
        ndirect = 0;
    }
    __syncthreads();
}

template <typename FT, typename VT, int NM, int LPN, int VEC, int CH, bool PHI>
__device__ __forceinline__ void grouped_kernel_body(const TiledArgs<FT>& a)
{
    constexpr int MM = grouped_mm<NM>();
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ u32 statics[2 + MT_WARPS];
    const GroupedSmem gs = grouped_smem_ptrs<FT, MM>(smem, a.hslots, statics, a.hot);
    FT* hacc = a.hot ? a.hot_acc + (size_t)blockIdx.x * a.hot * a.R : nullptr;
    for (int k = threadIdx.x; k < a.hot; k += MT_THREADS) gs.htag[k] = 0;
    for (int k = threadIdx.x; k < a.hot * a.R; k += MT_THREADS) hacc[k] = FT(0);
    grouped_init(gs, a.hslots);  // ends with a barrier: the zeroed region precedes every run flush
    for (u64 ti = blockIdx.x; ti < a.ntiles; ti += gridDim.x)
        grouped_tile<FT, VT, NM, LPN, VEC, CH, PHI>(a, ti, gs);
    if (a.hot) {  // the CTA's hot-row sums, once each (read from L2, where the atomics landed)
        __syncthreads();
        for (int k = threadIdx.x; k < a.hot * a.R; k += MT_THREADS) {
            const int sl = k / a.R;
            const u32 tg = gs.htag[sl];
            if (tg) atomicAdd(a.out + (size_t)(tg - 1u) * a.R + (k - sl * a.R), __ldcg(hacc + k));
        }
    }
}

template <typename FT, typename VT, int NM, int LPN, int VEC, int CH, bool PHI>
__global__ void __launch_bounds__(MT_THREADS) k_grouped(TiledArgs<FT> a)
{
    grouped_kernel_body<FT, VT, NM, LPN, VEC, CH, PHI>(a);
}

template <typename FT, typename VT, int NM, int LPN, int VEC, int CH, bool PHI, int MINB>
__global__ void __launch_bounds__(MT_THREADS, MINB) k_grouped_mb(TiledArgs<FT> a)
{
    grouped_kernel_body<FT, VT, NM, LPN, VEC, CH, PHI>(a);
}

template <typename FT>
struct CrArgsK {
    KeySrc key;
    const void* vals;
    u64 nnz;
    u64 per;  // nonzeros per reference partition
    int nprtn;
    int nmode;
    int target;
    int R;
    int crword;  // 0 = lo, 1 = hi
    u64 crbit;   // bit mask inside that word
    const FT* U[ALTOB_MAX_MODES];
    FT* out;
    Fields fld;
};

// mttkrp_alto_atomic_cr (alto.hpp:1090-1158): one warp owns one reference
// partition and walks it in order, so rows owned by that partition (CR bit
// clear) are updated with plain read-modify-write and shared rows (CR bit
// set) with atomics.
template <typename FT, typename VT>
__global__ void __launch_bounds__(MT_THREADS) k_atomic_cr(CrArgsK<FT> a)
{
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * MT_THREADS + threadIdx.x) >> 5;
    const int nw = (gridDim.x * MT_THREADS) >> 5;
    const VT* vals = reinterpret_cast<const VT*>(a.vals);
    for (int p = gw; p < a.nprtn; p += nw) {
        u64 s = (u64)p * a.per, e = (u64)(p + 1) * a.per;
        if (s > a.nnz) s = a.nnz;
        if (e > a.nnz) e = a.nnz;
        for (u64 i = s; i < e; ++i) {
            const u64 lo = a.key.klo[i], hi = key_hi(a.key, i);
            const bool shared = ((a.crword ? hi : lo) & a.crbit) != 0;
            const FT v = (FT)vals[i];
            u32 c[ALTOB_MAX_MODES];
            for (int m = 0; m < a.nmode; ++m) c[m] = field(lo, hi, a.fld.pos[m], a.fld.mask[m]);
            for (int r = lane; r < a.R; r += 32) {
                FT x = v;
                for (int m = 0; m < a.nmode; ++m)
                    if (m != a.target) x *= __ldg(a.U[m] + (size_t)c[m] * a.R + r);
                FT* o = a.out + (size_t)c[a.target] * a.R + r;
                if (shared) atomicAdd(o, x);
                else *o += x;
            }
            __syncwarp();
        }
    }
}

}  // namespace altob
