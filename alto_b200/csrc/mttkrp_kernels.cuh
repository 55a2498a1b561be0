// mttkrp_kernels.cuh -- MTTKRP and CP-APR Phi kernels on the ALTO stream.
//
// Reference kernels replaced (IntelLabs/ALTO):
//   mttkrp_alto_da_mem_pull   include/alto.hpp:1227-1318  -> k_tiled<..., PHI=false>
//   mttkrp_alto_op_sched      include/alto.hpp:1320-1415  -> k_tiled reading through oidx
//   mttkrp_alto_atomic        include/alto.hpp:1030-1088  -> k_tiled without row cache
//   mttkrp_alto_atomic_cr     include/alto.hpp:1090-1158  -> k_atomic_cr
//   CalculatePhi_alto_*       include/apr.hpp:383-848     -> k_tiled<..., PHI=true>
//
// k_tiled: a persistent CTA walks tiles of TILE consecutive nonzeros of the
// ALTO-ordered stream.  Phase A (one thread per nonzero) loads the key and
// value with coalesced loads, decodes every mode index with the compress
// network and claims a shared-memory accumulator row for the output index
// (direct-mapped on its low bits).  Phase B (a group of LPN lanes per
// nonzero, VEC elements per lane, 16-byte loads) gathers the factor rows,
// forms val * Khatri-Rao row (or the Phi row) and adds it to the claimed
// shared-memory row, or straight to global memory when the slot belongs to
// another index.  Phase C flushes every claimed row once with vector
// atomics.  This is the GPU form of the reference's per-partition temporary
// rows plus pull reduction: the tile is the partition and the flush is the
// pull.
#pragma once

#include "internal.cuh"

namespace altob {

constexpr int MT_THREADS = 256;
constexpr int MT_WARPS = MT_THREADS / 32;
constexpr int MT_CHMAX = 4;  // rank chunks kept in registers

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

template <typename FT>
struct TiledArgs {
    const u64* klo;
    const u64* khi;
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
    Decoder dec;
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

template <typename FT, typename VT, int KW, int LPN, int VEC, bool PHI>
__global__ void __launch_bounds__(MT_THREADS) k_tiled(TiledArgs<FT> a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int tile = a.tile, nmode = a.nmode, R = a.R, H = a.hslots;
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
    constexpr int NPW = 32 / LPN;
    const int sub = lane % LPN, q = lane / LPN;
    const int per_warp = tile / MT_WARPS;
    const int nch = (R + LPN * VEC - 1) / (LPN * VEC);

    for (u64 ti = blockIdx.x; ti < a.ntiles; ti += gridDim.x) {
        // ---- phase A: load, decode, claim accumulator rows
        const u64 g0 = ti * (u64)tile;
        for (int it = tid; it < tile; it += MT_THREADS) {
            const u64 g = g0 + it;
            int sl = -2;
            if (g < a.nnz) {
                const u64 pos = a.perm ? (u64)a.perm[g] : g;
                u32 w[4];
                split_key(a.klo[pos], KW == 2 ? a.khi[pos] : 0ull, w);
                val[it] = (FT)vals[pos];
                u32 trow = 0;
                for (int m = 0; m < nmode; ++m) {
                    u32 c = decode_mode(w, a.dec.md[m], a.dec.nwords);
                    crd[(size_t)m * tile + it] = c;
                    if (m == target) trow = c;
                }
                sl = -1;
                if (H) {
                    u32 h = trow & (u32)(H - 1);
                    u32 old = atomicCAS(&tag[h], 0u, trow + 1u);
                    if (old == 0u) {
                        used[atomicAdd(&nused, 1u)] = h;
                        sl = (int)h;
                    } else if (old == trow + 1u) {
                        sl = (int)h;
                    }
                }
            }
            else {
                // tail of the last tile: harmless index 0, value 0, no writes
                for (int m = 0; m < nmode; ++m) crd[(size_t)m * tile + it] = 0u;
                val[it] = FT(0);
            }
            slot[it] = sl;
        }
        __syncthreads();

        // ---- phase B: gather factor rows, accumulate
        for (int j = warp * per_warp; j < (warp + 1) * per_warp; j += NPW) {
            const int it = j + q;
            const int sl = slot[it];  // -2: no nonzero (kept in the loop for the Phi shuffles)
            const FT v = val[it];
            FT x[MT_CHMAX][VEC];
#pragma unroll
            for (int ch = 0; ch < MT_CHMAX; ++ch)
#pragma unroll
                for (int e = 0; e < VEC; ++e) x[ch][e] = PHI ? FT(1) : v;
            for (int m = 0; m < nmode; ++m) {
                if (m == target) continue;
                const FT* row = a.U[m] + (size_t)crd[(size_t)m * tile + it] * R;
#pragma unroll
                for (int ch = 0; ch < MT_CHMAX; ++ch) {
                    const int r0 = ch * LPN * VEC + sub * VEC;
                    if (ch < nch && r0 < R) {
                        FT y[VEC];
                        vload<FT, VEC>(row + r0, y);
#pragma unroll
                        for (int e = 0; e < VEC; ++e) x[ch][e] *= y[e];
                    }
                }
            }
            const u32 trow = crd[(size_t)target * tile + it];
            if constexpr (PHI) {
                // v / max(<B[trow,:], krp>, eps), apr.hpp:452-462
                const FT* brow = a.U[target] + (size_t)trow * R;
                FT dot = FT(0);
#pragma unroll
                for (int ch = 0; ch < MT_CHMAX; ++ch) {
                    const int r0 = ch * LPN * VEC + sub * VEC;
                    if (ch < nch && r0 < R) {
                        FT y[VEC];
                        vload<FT, VEC>(brow + r0, y);
#pragma unroll
                        for (int e = 0; e < VEC; ++e) dot += y[e] * x[ch][e];
                    }
                }
#pragma unroll
                for (int o = LPN / 2; o > 0; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o, LPN);
                const FT s = v / (dot > a.eps ? dot : a.eps);
#pragma unroll
                for (int ch = 0; ch < MT_CHMAX; ++ch)
#pragma unroll
                    for (int e = 0; e < VEC; ++e) x[ch][e] *= s;
            }
#pragma unroll
            for (int ch = 0; ch < MT_CHMAX; ++ch) {
                const int r0 = ch * LPN * VEC + sub * VEC;
                if (ch < nch && r0 < R && sl != -2) {
                    if (sl >= 0) {
                        FT* dst = acc + (size_t)sl * R + r0;
#pragma unroll
                        for (int e = 0; e < VEC; ++e) atomicAdd(dst + e, x[ch][e]);
                    } else {
                        gred<FT, VEC>(a.out + (size_t)trow * R + r0, x[ch]);
                    }
                }
            }
        }
        __syncthreads();

        // ---- phase C: flush claimed rows
        if (H) {
            const u32 nu = nused;
            for (u32 k = warp; k < nu; k += MT_WARPS) {
                const u32 h = used[k];
                const u32 row = tag[h] - 1u;
                FT* src = acc + (size_t)h * R;
                FT* dst = a.out + (size_t)row * R;
                for (int r = lane * VEC; r < R; r += 32 * VEC) {
                    FT y[VEC];
                    vload_plain<FT, VEC>(src + r, y);
                    gred<FT, VEC>(dst + r, y);
                    vstore_zero<FT, VEC>(src + r);
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

template <typename FT>
struct CrArgsK {
    const u64* klo;
    const u64* khi;
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
    Decoder dec;
};

// mttkrp_alto_atomic_cr (alto.hpp:1090-1158): one warp owns one reference
// partition and walks it in order, so rows owned by that partition (CR bit
// clear) are updated with plain read-modify-write and shared rows (CR bit
// set) with atomics.
template <typename FT, typename VT, int KW>
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
            u64 lo = a.klo[i], hi = KW == 2 ? a.khi[i] : 0ull;
            u32 w[4];
            split_key(lo, hi, w);
            const bool shared = ((a.crword ? hi : lo) & a.crbit) != 0;
            const FT v = (FT)vals[i];
            u32 c[ALTOB_MAX_MODES];
            for (int m = 0; m < a.nmode; ++m) c[m] = decode_mode(w, a.dec.md[m], a.dec.nwords);
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
