// build.cu -- ALTO tensor build on the device.
//
// Replaces create_alto (IntelLabs/ALTO include/alto.hpp:108-294):
//   setup_packed_alto  (alto.hpp:669-770)  -> host, make_masks()
//   pdep linearization (alto.hpp:184-202)  -> k_linearize (expand network)
//   sort_alto          (alto.hpp:772-803)  -> radix_sort_pairs (LSD, 8-bit digits)
//   oidx               (alto.hpp:246-285)  -> radix sort of mode indices
//   prtn_alto          (alto.hpp:805-899)  -> k_intervals
//   CR bits            (alto.hpp:930-1027) -> k_cr_owner + k_cr_set
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "internal.cuh"

namespace altob {

// ------------------------------------------------------------- errors

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

altob_status fail(altob_status s, const std::string& msg)
{
    set_error(msg);
    return s;
}

static thread_local cudaStream_t g_alloc_stream = 0;

StreamScope::StreamScope(cudaStream_t s) : prev(g_alloc_stream) { g_alloc_stream = s; }
StreamScope::~StreamScope() { g_alloc_stream = prev; }

altob_status dmalloc(void** p, size_t bytes)
{
    *p = nullptr;
    cudaError_t e = cudaMallocAsync(p, bytes ? bytes : 1, g_alloc_stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return fail(e == cudaErrorMemoryAllocation ? ALTOB_ERR_NOMEM : ALTOB_ERR_CUDA,
                    std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e));
    }
    return ALTOB_OK;
}

void dfree(void* p)
{
    if (p) cudaFreeAsync(p, g_alloc_stream);
}

altob_status tensor_scratch(altob_tensor* t, size_t bytes, void** out)
{
    if (bytes > t->scratch_bytes) {
        if (t->scratch) {
            dfree(t->scratch);  // stream-ordered: after this stream's earlier uses
            t->scratch = nullptr;
            t->scratch_bytes = 0;
        }
        size_t want = std::max(bytes, (size_t)1 << 20);
        ALTOB_TRY(dmalloc(&t->scratch, want));
        t->scratch_bytes = want;
    }
    *out = t->scratch;
    return ALTOB_OK;
}

altob_status tensor_hotbuf(altob_tensor* t, size_t bytes, void** out)
{
    if (bytes > t->hotbuf_bytes) {
        if (t->hotbuf) {
            dfree(t->hotbuf);
            t->hotbuf = nullptr;
            t->hotbuf_bytes = 0;
        }
        ALTOB_TRY(dmalloc(&t->hotbuf, bytes));
        t->hotbuf_bytes = bytes;
    }
    *out = t->hotbuf;
    return ALTOB_OK;
}

static bool capturing(cudaStream_t st)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return cs != cudaStreamCaptureStatusNone;
}

altob_status tensor_enter(altob_tensor* t, cudaStream_t st)
{
    if (!t->use_ev || t->use_stream == st || capturing(st)) return ALTOB_OK;
    ALTOB_CUDA(cudaStreamWaitEvent(st, t->use_ev, 0));
    return ALTOB_OK;
}

altob_status tensor_leave(altob_tensor* t, cudaStream_t st)
{
    if (capturing(st)) return ALTOB_OK;
    if (!t->use_ev) ALTOB_CUDA(cudaEventCreateWithFlags(&t->use_ev, cudaEventDisableTiming));
    ALTOB_CUDA(cudaEventRecord(t->use_ev, st));
    t->use_stream = st;
    return ALTOB_OK;
}

// SM count of the current device, cached per device ordinal.
int num_sms()
{
    static std::mutex mu;
    static std::vector<int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    if (dev >= (int)cache.size()) cache.resize(dev + 1, 0);
    if (cache[dev] <= 0) {
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cache[dev] = sms > 0 ? sms : 148;
    }
    return cache[dev];
}

// ------------------------------------------------------------ masks

static int mode_bits(u64 d) { return d <= 1 ? 0 : 64 - __builtin_clzll(d - 1); }

// setup_packed_alto(LSB_FIRST, SHORT_FIRST), alto.hpp:669-770: modes in
// ascending bit count (ties in mode order), one bit per mode per level,
// starting at the least significant bit.
static int make_masks(int nmode, const u64* dims, u128* masks, int* order)
{
    int bits[ALTOB_MAX_MODES], total = 0;
    for (int n = 0; n < nmode; ++n) {
        bits[n] = mode_bits(dims[n]);
        order[n] = n;
        total += bits[n];
        masks[n] = 0;
    }
    std::stable_sort(order, order + nmode, [&](int a, int b) { return bits[a] < bits[b]; });
    int shift = 0;
    for (int level = 0;; ++level) {
        bool done = true;
        for (int k = 0; k < nmode; ++k) {
            int n = order[k];
            if (level < bits[n]) {
                masks[n] |= (u128)1 << shift;
                ++shift;
                done = false;
            }
        }
        if (done) break;
    }
    return total;
}

Decoder make_decoder(int nmode, const u128* masks, int alto_bits)
{
    Decoder d;
    memset(&d, 0, sizeof(d));
    d.nmode = nmode;
    d.nwords = std::max(1, (alto_bits + 31) / 32);
    for (int n = 0; n < nmode; ++n) {
        u32 off = 0;
        for (int w = 0; w < 4; ++w) {
            u32 m = (u32)(masks[n] >> (32 * w));
            WordDec& wd = d.md[n].w[w];
            wd.m = m;
            wd.off = m ? off : 0;
            compress_moves(m, wd.mv);
            off += __builtin_popcount(m);
        }
    }
    return d;
}

// ----------------------------------------------------------- scans
// Exclusive prefix sum of u32 values in place (sum < 2^32).

static constexpr int SC_THREADS = 1024;
static constexpr int SC_IPT = 4;
static constexpr int SC_CHUNK = SC_THREADS * SC_IPT;

__device__ __forceinline__ u32 block_excl_scan(u32 v, u32* total, u32* warp_sums)
{
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    u32 x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        u32 y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        u32 s = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            u32 y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) warp_sums[lane] = s;
    }
    __syncthreads();
    u32 base = warp ? warp_sums[warp - 1] : 0;
    *total = warp_sums[nw - 1];
    __syncthreads();
    return base + x - v;
}

__global__ void k_scan_reduce(const u32* in, u64 n, u32* bsum)
{
    __shared__ u32 ws[32];
    u64 base = (u64)blockIdx.x * SC_CHUNK + (u64)threadIdx.x * SC_IPT;
    u32 s = 0;
#pragma unroll
    for (int k = 0; k < SC_IPT; ++k)
        if (base + k < n) s += in[base + k];
    u32 tot;
    block_excl_scan(s, &tot, ws);
    if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

__global__ void k_scan_top(u32* bsum, u32 nb)
{
    __shared__ u32 ws[32];
    u32 carry = 0;
    for (u32 b0 = 0; b0 < nb; b0 += blockDim.x) {
        u32 i = b0 + threadIdx.x;
        u32 v = i < nb ? bsum[i] : 0;
        u32 tot;
        u32 ex = block_excl_scan(v, &tot, ws);
        if (i < nb) bsum[i] = carry + ex;
        carry += tot;
    }
}

__global__ void k_scan_down(u32* data, u64 n, const u32* bsum)
{
    __shared__ u32 ws[32];
    u64 base = (u64)blockIdx.x * SC_CHUNK + (u64)threadIdx.x * SC_IPT;
    u32 v[SC_IPT];
    u32 s = 0;
#pragma unroll
    for (int k = 0; k < SC_IPT; ++k) {
        v[k] = base + k < n ? data[base + k] : 0;
        s += v[k];
    }
    u32 tot;
    u32 ex = block_excl_scan(s, &tot, ws) + bsum[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SC_IPT; ++k) {
        if (base + k < n) data[base + k] = ex;
        ex += v[k];
    }
}

static altob_status excl_scan_u32(u32* data, u64 n, u32* bsum, cudaStream_t st)
{
    u32 nb = (u32)((n + SC_CHUNK - 1) / SC_CHUNK);
    if (nb == 0) return ALTOB_OK;
    k_scan_reduce<<<nb, SC_THREADS, 0, st>>>(data, n, bsum);
    ALTOB_LAUNCH_CHECK();
    k_scan_top<<<1, SC_THREADS, 0, st>>>(bsum, nb);
    ALTOB_LAUNCH_CHECK();
    k_scan_down<<<nb, SC_THREADS, 0, st>>>(data, n, bsum);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

// ------------------------------------------------------- radix sort
// LSD radix sort, 8-bit digits.  Per pass: tile histograms (digit-major),
// one exclusive scan, then a stable scatter in which every tile ranks its
// keys with warp match + a per-round scan over the eight warps.

static constexpr int RS_THREADS = 256;
static constexpr int RS_IPT = 16;
static constexpr int RS_TILE = RS_THREADS * RS_IPT;
static constexpr int RS_WARPS = RS_THREADS / 32;

template <int KW>
__device__ __forceinline__ u32 rs_digit(u64 lo, u64 hi, int shift)
{
    u64 w = (KW == 2 && shift >= 64) ? hi : lo;
    return (u32)(w >> (shift & 63)) & 0xffu;
}

template <int KW>
__global__ void __launch_bounds__(RS_THREADS) k_rs_hist(const u64* __restrict__ klo, const u64* __restrict__ khi,
                                                        u64 n, int shift, u32* __restrict__ hist, u32 ntiles)
{
    __shared__ u32 h[RS_WARPS][256];
    for (int j = threadIdx.x; j < RS_WARPS * 256; j += RS_THREADS) (&h[0][0])[j] = 0;
    __syncthreads();
    int warp = threadIdx.x >> 5;
    u64 base = (u64)blockIdx.x * RS_TILE;
#pragma unroll 4
    for (int k = 0; k < RS_IPT; ++k) {
        u64 i = base + (u64)k * RS_THREADS + threadIdx.x;
        if (i < n) {
            u64 lo = (KW == 1 || shift < 64) ? klo[i] : 0;
            u64 hi = (KW == 2 && shift >= 64) ? khi[i] : 0;
            atomicAdd(&h[warp][rs_digit<KW>(lo, hi, shift)], 1u);
        }
    }
    __syncthreads();
    u32 d = threadIdx.x;
    u32 s = 0;
#pragma unroll
    for (int w = 0; w < RS_WARPS; ++w) s += h[w][d];
    hist[(u64)d * ntiles + blockIdx.x] = s;
}

template <int KW>
__global__ void __launch_bounds__(RS_THREADS) k_rs_scatter(const u64* __restrict__ klo, const u64* __restrict__ khi,
                                                           const u32* __restrict__ pay, u64* __restrict__ olo,
                                                           u64* __restrict__ ohi, u32* __restrict__ opay, u64 n,
                                                           int shift, const u32* __restrict__ offs, u32 ntiles)
{
    __shared__ u32 run[256];
    __shared__ u32 wcnt[RS_WARPS][256];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    run[tid] = offs[(u64)tid * ntiles + blockIdx.x];
    const u64 base = (u64)blockIdx.x * RS_TILE;
    for (int k = 0; k < RS_IPT; ++k) {
        const u64 i = base + (u64)k * RS_THREADS + tid;
        const bool valid = i < n;
        u64 lo = 0, hi = 0;
        u32 p = 0, d = 256;
        if (valid) {
            lo = klo[i];
            if (KW == 2) hi = khi[i];
            p = pay[i];
            d = rs_digit<KW>(lo, hi, shift);
        }
        for (int j = tid; j < RS_WARPS * 256; j += RS_THREADS) (&wcnt[0][0])[j] = 0;
        __syncthreads();
        const u32 peers = __match_any_sync(0xffffffffu, d);
        const u32 rank = __popc(peers & ((1u << lane) - 1u));
        if (valid && lane == __ffs(peers) - 1) wcnt[warp][d] = __popc(peers);
        __syncthreads();
        {
            u32 r = run[tid];
#pragma unroll
            for (int w = 0; w < RS_WARPS; ++w) {
                u32 c = wcnt[w][tid];
                wcnt[w][tid] = r;
                r += c;
            }
            run[tid] = r;
        }
        __syncthreads();
        if (valid) {
            u32 dst = wcnt[warp][d] + rank;
            olo[dst] = lo;
            if (KW == 2) ohi[dst] = hi;
            opay[dst] = p;
        }
        __syncthreads();
    }
}

altob_status radix_sort_pairs(u64* klo, u64* khi, u32* pay, u64* klo_alt, u64* khi_alt, u32* pay_alt, u64 n,
                              int kw, int nbits, cudaStream_t st, bool* result_in_alt)
{
    *result_in_alt = false;
    if (n <= 1 || nbits <= 0) return ALTOB_OK;
    u32 ntiles = (u32)((n + RS_TILE - 1) / RS_TILE);
    u64 hn = (u64)ntiles * 256;
    u32* hist = nullptr;
    u32* bsum = nullptr;
    ALTOB_TRY(dmalloc_t(&hist, hn));
    altob_status s = dmalloc_t(&bsum, hn / SC_CHUNK + 2);
    if (s != ALTOB_OK) {
        dfree(hist);
        return s;
    }
    bool alt = false;
    for (int shift = 0; shift < nbits; shift += 8) {
        u64* slo = alt ? klo_alt : klo;
        u64* shi = alt ? khi_alt : khi;
        u32* sp = alt ? pay_alt : pay;
        u64* dlo = alt ? klo : klo_alt;
        u64* dhi = alt ? khi : khi_alt;
        u32* dp = alt ? pay : pay_alt;
        if (kw == 2) {
            k_rs_hist<2><<<ntiles, RS_THREADS, 0, st>>>(slo, shi, n, shift, hist, ntiles);
        } else {
            k_rs_hist<1><<<ntiles, RS_THREADS, 0, st>>>(slo, shi, n, shift, hist, ntiles);
        }
        s = excl_scan_u32(hist, hn, bsum, st);
        if (s != ALTOB_OK) break;
        if (kw == 2) {
            k_rs_scatter<2><<<ntiles, RS_THREADS, 0, st>>>(slo, shi, sp, dlo, dhi, dp, n, shift, hist, ntiles);
        } else {
            k_rs_scatter<1><<<ntiles, RS_THREADS, 0, st>>>(slo, shi, sp, dlo, dhi, dp, n, shift, hist, ntiles);
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            s = fail(ALTOB_ERR_CUDA, std::string("radix scatter: ") + cudaGetErrorString(e));
            break;
        }
        alt = !alt;
    }
    cudaStreamSynchronize(st);
    dfree(hist);
    dfree(bsum);
    *result_in_alt = alt;
    return s;
}

// ------------------------------------------------------ build kernels

// pdep linearization: key = OR over modes of expand(coord, mask).  Also
// validates every coordinate against its dimension.
__global__ void k_linearize(const u64* __restrict__ cidx, u64 nnz, Decoder dec, u64 dmax0, u64 dmax1, u64 dmax2,
                            u64 dmax3, u64 dmax4, int kw, u64* __restrict__ klo, u64* __restrict__ khi,
                            u32* __restrict__ perm, int* __restrict__ bad)
{
    const u64 dm[5] = {dmax0, dmax1, dmax2, dmax3, dmax4};
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += (u64)gridDim.x * blockDim.x) {
        u32 w[4] = {0, 0, 0, 0};
        for (int m = 0; m < dec.nmode; ++m) {
            u64 c64 = cidx[(u64)m * nnz + i];
            if (c64 >= dm[m]) {
                atomicExch(bad, 1);
                c64 = 0;
            }
            u32 c = (u32)c64;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const WordDec& wd = dec.md[m].w[q];
                if (q < dec.nwords && wd.m) w[q] |= expand32(c >> wd.off, wd);
            }
        }
        klo[i] = (u64)w[0] | ((u64)w[1] << 32);
        if (kw == 2) khi[i] = (u64)w[2] | ((u64)w[3] << 32);
        perm[i] = (u32)i;
    }
}

template <typename VI, typename VO>
__global__ void k_gather_vals(const VI* __restrict__ in, const u32* __restrict__ perm, u64 n, VO* __restrict__ out)
{
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
        out[i] = (VO)in[perm[i]];
}

// Interleaved ALTO key -> field layout (same sort order).  CR bits are not
// set yet at this point.
__global__ void k_reencode(u64* __restrict__ klo, u64* __restrict__ khi, int kw, u64 n, Decoder dec, Fields f)
{
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        u32 w[4];
        split_key(klo[i], kw == 2 ? khi[i] : 0ull, w);
        u64 lo = 0, hi = 0;
        for (int m = 0; m < dec.nmode; ++m) {
            const u64 c = decode_mode(w, dec.md[m], dec.nwords);
            const u32 p = f.pos[m];
            if (p < 64) {
                lo |= c << p;
                if (p > 0 && p + 32 > 64) hi |= c >> (64 - p);
            } else {
                hi |= c << (p - 64);
            }
        }
        klo[i] = lo;
        if (kw == 2) khi[i] = hi;
    }
}

// Field layout -> interleaved ALTO key (for altob_dump); bits at and above
// alto_bits (the CR bits) are copied unchanged.
__global__ void k_interleave(const u64* __restrict__ klo, KeySrc ks, int alto_bits, u64 n, Decoder dec, Fields f,
                             u64* __restrict__ olo, u64* __restrict__ ohi)
{
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const u64 lo = klo[i], hi = key_hi(ks, i);
        u32 w[4] = {0, 0, 0, 0};
        for (int m = 0; m < dec.nmode; ++m) {
            const u32 c = field(lo, hi, f.pos[m], f.mask[m]);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const WordDec& wd = dec.md[m].w[q];
                if (q < dec.nwords && wd.m) w[q] |= expand32(c >> wd.off, wd);
            }
        }
        u64 ilo = (u64)w[0] | ((u64)w[1] << 32), ihi = (u64)w[2] | ((u64)w[3] << 32);
        if (alto_bits < 64) ilo |= lo & (~0ull << alto_bits);
        if (alto_bits <= 64) ihi |= hi;  // every high bit is a CR bit
        else ihi |= hi & (~0ull << (alto_bits - 64));
        olo[i] = ilo;
        ohi[i] = ihi;
    }
}

// Mode indices of the sorted keys (for the oidx sort).
__global__ void k_mode_keys(const u64* __restrict__ klo, const u64* __restrict__ khi, u64 n, Fields f, int mode,
                            u64* __restrict__ out, u32* __restrict__ iota)
{
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        out[i] = field(klo[i], khi ? khi[i] : 0ull, f.pos[mode], f.mask[mode]);
        iota[i] = (u32)i;
    }
}

__global__ void k_init_intervals(u64* iv, int nprtn, int nmode, u64 d0, u64 d1, u64 d2, u64 d3, u64 d4)
{
    const u64 dm[5] = {d0, d1, d2, d3, d4};
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nprtn * nmode) {
        iv[2 * k] = dm[k % nmode];
        iv[2 * k + 1] = 0;
    }
}

// Per-partition min / max of every mode index (prtn_alto, alto.hpp:874-899).
// A warp whose 32 keys lie in one partition reduces in registers first.
__global__ void k_intervals(const u64* __restrict__ klo, const u64* __restrict__ khi, u64 n, Fields f, u64 per,
                            u64* __restrict__ iv)
{
    const int lane = threadIdx.x & 31;
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 base = (u64)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
        u64 i = base + lane;
        bool valid = i < n;
        u64 p = valid ? i / per : ~0ull;
        u64 p0 = __shfl_sync(0xffffffffu, p, 0);
        u64 pl = __shfl_sync(0xffffffffu, p, 31);
        bool uniform = (p0 == pl) || (base + 31 >= n && __all_sync(0xffffffffu, !valid || p == p0));
        u64 lo = valid ? klo[i] : 0, hi = (valid && khi) ? khi[i] : 0;
        for (int m = 0; m < f.nmode; ++m) {
            u32 c = valid ? field(lo, hi, f.pos[m], f.mask[m]) : 0;
            if (uniform) {
                u32 mn = valid ? c : 0xffffffffu, mx = valid ? c : 0;
#pragma unroll
                for (int o = 16; o; o >>= 1) {
                    mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
                    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
                }
                if (lane == 0) {
                    u64* e = iv + (p0 * f.nmode + m) * 2;
                    atomicMin((unsigned long long*)e, (unsigned long long)mn);
                    atomicMax((unsigned long long*)(e + 1), (unsigned long long)mx);
                }
            } else if (valid) {
                u64* e = iv + (p * f.nmode + m) * 2;
                atomicMin((unsigned long long*)e, (unsigned long long)c);
                atomicMax((unsigned long long*)(e + 1), (unsigned long long)c);
            }
        }
    }
}

struct CrArgs {
    int* owner[ALTOB_MAX_MODES];
    int bitpos[ALTOB_MAX_MODES];  // -1 = no CR bit for this mode
};

// Fiber ownership (alto.hpp:970-996): 0 untouched, p+1 one partition, -1 shared.
__global__ void k_cr_owner(const u64* __restrict__ klo, const u64* __restrict__ khi, u64 n, Fields f, u64 per,
                           CrArgs a)
{
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const u64 lo = klo[i], hi = khi ? khi[i] : 0;
        int p1 = (int)(i / per) + 1;
        for (int m = 0; m < f.nmode; ++m) {
            if (a.bitpos[m] < 0) continue;
            u32 c = field(lo, hi, f.pos[m], f.mask[m]);
            int old = atomicCAS(&a.owner[m][c], 0, p1);
            if (old != 0 && old != p1 && old != -1) atomicExch(&a.owner[m][c], -1);
        }
    }
}

// Sets the CR bits of nonzeros whose fiber is shared (alto.hpp:998-1019).
__global__ void k_cr_set(u64* __restrict__ klo, u64* __restrict__ khi, u64 n, Fields f, CrArgs a)
{
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const u64 lo = klo[i], hi = khi ? khi[i] : 0;
        u64 add_lo = 0, add_hi = 0;
        for (int m = 0; m < f.nmode; ++m) {
            int b = a.bitpos[m];
            if (b < 0) continue;
            u32 c = field(lo, hi, f.pos[m], f.mask[m]);
            if (a.owner[m][c] == -1) {
                if (b < 64) add_lo |= 1ull << b;
                else add_hi |= 1ull << (b - 64);
            }
        }
        if (add_lo) klo[i] = lo | add_lo;
        if (add_hi && khi) khi[i] = hi | add_hi;
    }
}

// Positions where the high key word changes (for the run table) and a
// check that it never decreases.
__global__ void k_hi_runs(const u64* __restrict__ khi, u64 n, u64* __restrict__ starts, u32 cap,
                          u32* __restrict__ count, u32* __restrict__ decreasing)
{
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        if (i == 0 || khi[i] != khi[i - 1]) {
            if (i > 0 && khi[i] < khi[i - 1]) atomicExch(decreasing, 1u);
            u32 k = atomicAdd(count, 1u);
            if (k < cap) starts[k] = i;
        }
    }
}

__global__ void k_gather_u64(const u64* __restrict__ src, const u64* __restrict__ idx, u32 n, u64* __restrict__ out)
{
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = src[idx[i]];
}

// Explicit high key word of every nonzero of a tensor that keeps them as a
// run table.
__global__ void k_expand_hi(KeySrc key, u64 n, u64* __restrict__ hi)
{
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
        hi[i] = key_hi(key, i);
}

static int grid_for(u64 n, int threads)
{
    u64 blocks = (n + threads - 1) / threads;
    u64 cap = (u64)num_sms() * 16;
    return (int)std::max<u64>(1, std::min(blocks, cap));
}

// ------------------------------------------------------------ create

static altob_status build(altob_tensor* t, const u64* d_cidx, const void* d_vals_in, altob_dtype vin,
                          cudaStream_t st)
{
    const u64 nnz = t->nnz;
    const int kw = t->kw;
    u64 *klo = nullptr, *khi = nullptr, *klo2 = nullptr, *khi2 = nullptr;
    u32 *perm = nullptr, *perm2 = nullptr;
    int* bad = nullptr;
    altob_status s = ALTOB_OK;
    auto cleanup = [&] {
        cudaStreamSynchronize(st);
        dfree(klo2);
        dfree(khi2);
        dfree(perm);
        dfree(perm2);
        dfree(bad);
        if (s != ALTOB_OK) {
            dfree(klo);
            dfree(khi);
        }
    };
#define BTRY(x)             \
    do {                    \
        s = (x);            \
        if (s != ALTOB_OK) { \
            cleanup();      \
            return s;       \
        }                   \
    } while (0)
    BTRY(dmalloc_t(&klo, nnz));
    BTRY(dmalloc_t(&klo2, nnz));
    if (kw == 2) {
        BTRY(dmalloc_t(&khi, nnz));
        BTRY(dmalloc_t(&khi2, nnz));
    }
    BTRY(dmalloc_t(&perm, nnz));
    BTRY(dmalloc_t(&perm2, nnz));
    BTRY(dmalloc_t(&bad, 1));
    cudaMemsetAsync(bad, 0, sizeof(int), st);
    u64 dm[5] = {1, 1, 1, 1, 1};
    for (int n = 0; n < t->nmode; ++n) dm[n] = t->dims[n];
    if (nnz) {
        k_linearize<<<grid_for(nnz, 256), 256, 0, st>>>(d_cidx, nnz, t->dec, dm[0], dm[1], dm[2], dm[3], dm[4], kw,
                                                        klo, khi, perm, bad);
        if (cudaGetLastError() != cudaSuccess) BTRY(fail(ALTOB_ERR_CUDA, "k_linearize launch failed"));
        int hbad = 0;
        cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) BTRY(fail(ALTOB_ERR_CUDA, "linearize failed"));
        if (hbad) BTRY(fail(ALTOB_ERR_ARG, "a coordinate is not below its dimension"));
    }
    bool in_alt = false;
    BTRY(radix_sort_pairs(klo, khi, perm, klo2, khi2, perm2, nnz, kw, t->alto_bits, st, &in_alt));
    if (in_alt) {
        std::swap(klo, klo2);
        std::swap(khi, khi2);
        std::swap(perm, perm2);
    }
    // interleaved -> field layout (same order)
    if (nnz) {
        k_reencode<<<grid_for(nnz, 256), 256, 0, st>>>(klo, khi, kw, nnz, t->dec, t->fld);
        if (cudaGetLastError() != cudaSuccess) BTRY(fail(ALTOB_ERR_CUDA, "k_reencode launch failed"));
    }
    // values in sorted order, converted to the stored dtype
    size_t vsz = val_size(t->vdt);
    BTRY(dmalloc(&t->d_vals, nnz * vsz + 16));
    if (nnz) {
        int g = grid_for(nnz, 256);
#define GATHER(VI, VO) \
    k_gather_vals<VI, VO><<<g, 256, 0, st>>>((const VI*)d_vals_in, perm, nnz, (VO*)t->d_vals)
        if (vin == ALTOB_F64 && t->vdt == ALTOB_F64) GATHER(double, double);
        else if (vin == ALTOB_F64 && t->vdt == ALTOB_F32) GATHER(double, float);
        else if (vin == ALTOB_F32 && t->vdt == ALTOB_F32) GATHER(float, float);
        else if (vin == ALTOB_F32 && t->vdt == ALTOB_F64) GATHER(float, double);
        else if (vin == ALTOB_U32 && t->vdt == ALTOB_U32) GATHER(u32, u32);
        else if (vin == ALTOB_F64 && t->vdt == ALTOB_U32) GATHER(double, u32);
        else BTRY(fail(ALTOB_ERR_UNSUPPORTED, "value dtype conversion not supported"));
#undef GATHER
        if (cudaGetLastError() != cudaSuccess) BTRY(fail(ALTOB_ERR_CUDA, "gather launch failed"));
    }

    // oidx for low-reuse modes (alto.hpp:246-285)
    t->is_oidx = 0;
    for (int n = 0; n < t->nmode; ++n)
        if (fib_reuse(t, n) <= 4) t->is_oidx = 1;
    if (t->is_oidx && nnz) {
        for (int n = 0; n < t->nmode; ++n) {
            if (fib_reuse(t, n) > 4) continue;
            // klo2 / perm2 are free at this point: mode keys + iota
            u64* mk = klo2;
            u64* mk2 = nullptr;
            u32* ox2 = nullptr;
            BTRY(dmalloc_t(&mk2, nnz));
            s = dmalloc_t(&ox2, nnz);
            if (s != ALTOB_OK) {
                dfree(mk2);
                cleanup();
                return s;
            }
            k_mode_keys<<<grid_for(nnz, 256), 256, 0, st>>>(klo, khi, nnz, t->fld, n, mk, perm2);
            bool alt2 = false;
            s = radix_sort_pairs(mk, nullptr, perm2, mk2, nullptr, ox2, nnz, 1, mode_bits(t->dims[n]), st, &alt2);
            dfree(mk2);
            if (s != ALTOB_OK) {
                dfree(ox2);
                cleanup();
                return s;
            }
            if (alt2) {
                t->d_oidx[n] = ox2;
            } else {
                t->d_oidx[n] = perm2;
                perm2 = ox2;
            }
        }
    }

    // partitions (alto.hpp:822-836) and intervals (:874-899)
    const int np = t->nprtn, nm = t->nmode;
    const u64 per = (nnz + (u64)np - 1) / (u64)np;
    t->prtn_ptr.assign(np + 1, 0);
    for (int p = 0; p < np; ++p) t->prtn_ptr[p + 1] = std::min<u64>((u64)(p + 1) * per, nnz);
    u64* d_iv = nullptr;
    BTRY(dmalloc_t(&d_iv, (u64)np * nm * 2));
    k_init_intervals<<<(np * nm + 255) / 256, 256, 0, st>>>(d_iv, np, nm, dm[0], dm[1], dm[2], dm[3], dm[4]);
    if (nnz) k_intervals<<<grid_for(nnz, 256), 256, 0, st>>>(klo, khi, nnz, t->fld, per, d_iv);
    t->intervals.assign((size_t)np * nm * 2, 0);
    cudaMemcpyAsync(t->intervals.data(), d_iv, t->intervals.size() * sizeof(u64), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    dfree(d_iv);
    if (e != cudaSuccess) BTRY(fail(ALTOB_ERR_CUDA, std::string("intervals: ") + cudaGetErrorString(e)));

    // CR bits (alto.hpp:932-1027)
    CrArgs ca;
    memset(&ca, 0, sizeof(ca));
    int free_bits = t->lit_bits - t->alto_bits;
    bool any_cr = false;
    t->alto_cr_mask = 0;
    for (int n = 0; n < nm; ++n) {
        ca.bitpos[n] = -1;
        t->cr_masks[n] = 0;
        if (fib_reuse(t, n) <= 4 && free_bits) {
            int b = t->lit_bits - free_bits;
            ca.bitpos[n] = b;
            t->cr_masks[n] = (u128)1 << b;
            t->alto_cr_mask |= t->cr_masks[n];
            --free_bits;
            any_cr = true;
        }
    }
    if (any_cr && nnz) {
        for (int n = 0; n < nm; ++n) {
            if (ca.bitpos[n] < 0) continue;
            s = dmalloc_t(&ca.owner[n], t->dims[n]);
            if (s == ALTOB_OK) cudaMemsetAsync(ca.owner[n], 0, t->dims[n] * sizeof(int), st);
            if (s != ALTOB_OK) break;
        }
        if (s == ALTOB_OK) {
            k_cr_owner<<<grid_for(nnz, 256), 256, 0, st>>>(klo, khi, nnz, t->fld, per, ca);
            k_cr_set<<<grid_for(nnz, 256), 256, 0, st>>>(klo, khi, nnz, t->fld, ca);
            e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) s = fail(ALTOB_ERR_CUDA, std::string("CR bits: ") + cudaGetErrorString(e));
        }
        for (int n = 0; n < nm; ++n) dfree(ca.owner[n]);
        if (s != ALTOB_OK) {
            cleanup();
            return s;
        }
    }
    // high key words: a run table when they never decrease along the stream
    // (the usual case: they are the top ALTO bits), else one word per nonzero
    if (kw == 2 && nnz) {
        const u32 cap = 1u << 16;
        u64* starts = nullptr;
        u32* cnt = nullptr;
        BTRY(dmalloc_t(&starts, cap));
        s = dmalloc_t(&cnt, 2);
        if (s != ALTOB_OK) {
            dfree(starts);
            cleanup();
            return s;
        }
        cudaMemsetAsync(cnt, 0, 2 * sizeof(u32), st);
        k_hi_runs<<<grid_for(nnz, 256), 256, 0, st>>>(khi, nnz, starts, cap, cnt, cnt + 1);
        u32 hc[2] = {0, 0};
        cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, st);
        e = cudaStreamSynchronize(st);
        if (e == cudaSuccess && hc[1] == 0 && hc[0] <= cap) {
            std::vector<u64> hs(hc[0]);
            cudaMemcpyAsync(hs.data(), starts, hc[0] * sizeof(u64), cudaMemcpyDeviceToHost, st);
            cudaStreamSynchronize(st);
            std::sort(hs.begin(), hs.end());
            u64 *rs = nullptr, *rv = nullptr;
            s = dmalloc_t(&rs, hc[0]);
            if (s == ALTOB_OK) s = dmalloc_t(&rv, hc[0]);
            if (s == ALTOB_OK) {
                cudaMemcpyAsync(rs, hs.data(), hc[0] * sizeof(u64), cudaMemcpyHostToDevice, st);
                k_gather_u64<<<std::max(1u, (hc[0] + 255) / 256), 256, 0, st>>>(khi, rs, hc[0], rv);
                e = cudaStreamSynchronize(st);
                if (e == cudaSuccess) {
                    t->d_run_start = rs;
                    t->d_run_val = rv;
                    t->nrun = (int)hc[0];
                    dfree(khi);
                    khi = nullptr;
                } else {
                    dfree(rs);
                    dfree(rv);
                }
            } else {
                dfree(rs);
            }
        }
        dfree(starts);
        dfree(cnt);
        if (e != cudaSuccess) BTRY(fail(ALTOB_ERR_CUDA, std::string("high-word runs: ") + cudaGetErrorString(e)));
        if (s != ALTOB_OK) BTRY(s);
    }
    t->d_klo = klo;
    t->d_khi = khi;
    cleanup();
#undef BTRY
    t->device_bytes = nnz * (8 * (khi ? 2 : 1) + vsz) + (u64)t->nrun * 16;
    for (int n = 0; n < nm; ++n)
        if (t->d_oidx[n]) t->device_bytes += nnz * 4;
    return ALTOB_OK;
}

static altob_status create_common(int nmode, const u64* dims, u64 nnz, const u64* d_cidx, const void* d_vals,
                                  altob_dtype vdt, int nprtn, int lit_bits, cudaStream_t st, altob_tensor** out)
{
    if (!out) return fail(ALTOB_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (nmode < 1 || nmode > ALTOB_MAX_MODES) return fail(ALTOB_ERR_ARG, "nmode must be 1..5");
    if (nprtn < 1) return fail(ALTOB_ERR_ARG, "nprtn must be >= 1");
    if (lit_bits != 0 && lit_bits != 64 && lit_bits != 128) return fail(ALTOB_ERR_ARG, "lit_bits must be 0, 64 or 128");
    if (nnz >= (1ull << 32)) return fail(ALTOB_ERR_UNSUPPORTED, "nnz must be below 2^32");
    if (vdt != ALTOB_F64 && vdt != ALTOB_F32 && vdt != ALTOB_U32) return fail(ALTOB_ERR_ARG, "bad value dtype");
    for (int n = 0; n < nmode; ++n) {
        if (dims[n] == 0) return fail(ALTOB_ERR_ARG, "a dimension is 0");
        if (dims[n] >= (1ull << 32)) return fail(ALTOB_ERR_UNSUPPORTED, "dimensions of 2^32 or more are not supported");
    }
    if (nnz && (!d_cidx || !d_vals)) return fail(ALTOB_ERR_ARG, "cidx / vals is NULL");
    altob_tensor* t = new altob_tensor();
    cudaGetDevice(&t->device);
    t->nmode = nmode;
    t->nprtn = nprtn;
    t->nnz = nnz;
    t->vdt = vdt;
    for (int n = 0; n < nmode; ++n) t->dims[n] = dims[n];
    int total = make_masks(nmode, dims, t->masks, t->order);
    if (lit_bits == 0) lit_bits = total <= 64 ? 64 : 128;
    if (total > lit_bits) {
        delete t;
        return fail(ALTOB_ERR_BITS, "ALTO bits (" + std::to_string(total) + ") exceed the " +
                                        std::to_string(lit_bits) + "-bit index");
    }
    t->lit_bits = lit_bits;
    t->alto_bits = total;
    t->alto_mask = 0;
    for (int n = 0; n < nmode; ++n) t->alto_mask |= t->masks[n];
    int ncr = 0, fb = lit_bits - total;
    for (int n = 0; n < nmode; ++n)
        if (fib_reuse(t, n) <= 4 && fb) {
            ++ncr;
            --fb;
        }
    t->kw = (total + ncr > 64) ? 2 : 1;
    t->dec = make_decoder(nmode, t->masks, total);
    t->fld.nmode = nmode;
    {
        u32 p = 0;
        for (int k = 0; k < nmode; ++k) {
            const int n = t->order[k];
            const int b = mode_bits(dims[n]);
            t->fld.pos[n] = p;
            t->fld.mask[n] = b >= 32 ? 0xffffffffu : ((1u << b) - 1u);
            p += b;
        }
    }
    altob_status s = build(t, d_cidx, d_vals, vdt, st);
    if (s != ALTOB_OK) {
        altob_destroy(t);
        return s;
    }
    *out = t;
    return ALTOB_OK;
}

// The reference's interleaved keys (default encoding, CR bits included) of
// every nonzero, into device arrays.
altob_status interleaved_keys(const altob_tensor* t, u64* olo, u64* ohi, cudaStream_t st)
{
    if (!t->nnz) return ALTOB_OK;
    k_interleave<<<grid_for(t->nnz, 256), 256, 0, st>>>(t->d_klo, key_src(t), t->alto_bits, t->nnz, t->dec, t->fld,
                                                        olo, ohi);
    ALTOB_LAUNCH_CHECK();
    return ALTOB_OK;
}

// A contiguous range [begin, end) of a tensor's ALTO stream as a tensor of
// its own (one GPU's share of a sharded MTTKRP or CP-ALS; the split follows
// the reference's equal-nnz partition rule, alto.hpp:822-836).  Keys, values
// and high words are copied; oidx (for the slice's own low-reuse modes, as
// alto.hpp:246-285 decides them from its nonzero count), partitions and
// intervals (alto.hpp:822-899) are computed for the slice.  The slice has no
// CR masks: its keys keep the parent's CR bits, which no mode field reads.
static altob_status slice_impl(const altob_tensor* t, u64 begin, u64 end, int nprtn, cudaStream_t st,
                               altob_tensor* s)
{
    const u64 n = end - begin;
    s->device = t->device;
    s->nmode = t->nmode;
    s->nprtn = nprtn;
    s->lit_bits = t->lit_bits;
    s->alto_bits = t->alto_bits;
    s->kw = t->kw;
    s->vdt = t->vdt;
    s->nnz = n;
    for (int m = 0; m < ALTOB_MAX_MODES; ++m) {
        s->dims[m] = t->dims[m];
        s->masks[m] = t->masks[m];
        s->order[m] = t->order[m];
    }
    s->alto_mask = t->alto_mask;
    s->dec = t->dec;
    s->fld = t->fld;
    const size_t vsz = val_size(t->vdt);
    ALTOB_TRY(dmalloc_t(&s->d_klo, n));
    ALTOB_TRY(dmalloc(&s->d_vals, n * vsz + 16));
    if (n) {
        ALTOB_CUDA(cudaMemcpyAsync(s->d_klo, t->d_klo + begin, n * 8, cudaMemcpyDeviceToDevice, st));
        ALTOB_CUDA(cudaMemcpyAsync(s->d_vals, (const char*)t->d_vals + begin * vsz, n * vsz, cudaMemcpyDeviceToDevice,
                                   st));
    }
    if (t->d_khi) {
        ALTOB_TRY(dmalloc_t(&s->d_khi, n));
        if (n) ALTOB_CUDA(cudaMemcpyAsync(s->d_khi, t->d_khi + begin, n * 8, cudaMemcpyDeviceToDevice, st));
    } else if (t->nrun) {  // the runs that overlap the range, starts relative to it
        std::vector<u64> rs(t->nrun), rv(t->nrun), ns, nv;
        ALTOB_CUDA(cudaMemcpyAsync(rs.data(), t->d_run_start, rs.size() * 8, cudaMemcpyDeviceToHost, st));
        ALTOB_CUDA(cudaMemcpyAsync(rv.data(), t->d_run_val, rv.size() * 8, cudaMemcpyDeviceToHost, st));
        ALTOB_CUDA(cudaStreamSynchronize(st));
        for (int r = 0; r < t->nrun; ++r) {
            const u64 stop = r + 1 < t->nrun ? rs[r + 1] : t->nnz;
            if (stop <= begin || rs[r] >= end) continue;
            ns.push_back(std::max(rs[r], begin) - begin);
            nv.push_back(rv[r]);
        }
        if (ns.empty()) {  // empty slice
            ns.push_back(0);
            nv.push_back(0);
        }
        ALTOB_TRY(dmalloc_t(&s->d_run_start, ns.size()));
        ALTOB_TRY(dmalloc_t(&s->d_run_val, nv.size()));
        ALTOB_CUDA(cudaMemcpyAsync(s->d_run_start, ns.data(), ns.size() * 8, cudaMemcpyHostToDevice, st));
        ALTOB_CUDA(cudaMemcpyAsync(s->d_run_val, nv.data(), nv.size() * 8, cudaMemcpyHostToDevice, st));
        s->nrun = (int)ns.size();
    }
    // explicit high words for the oidx and interval kernels (a run table is
    // expanded into a temporary array)
    const u64* hi = s->d_khi;
    u64* hi_tmp = nullptr;
    struct HiFree {
        u64** p;
        ~HiFree() { dfree(*p); }
    } hi_free{&hi_tmp};
    if (!hi && s->nrun && n) {
        ALTOB_TRY(dmalloc_t(&hi_tmp, n));
        k_expand_hi<<<grid_for(n, 256), 256, 0, st>>>(key_src(s), n, hi_tmp);
        if (cudaGetLastError() != cudaSuccess) return fail(ALTOB_ERR_CUDA, "k_expand_hi launch failed");
        hi = hi_tmp;
    }
    // oidx of the slice's low-reuse modes
    s->is_oidx = 0;
    for (int m = 0; m < s->nmode; ++m)
        if (fib_reuse(s, m) <= 4) s->is_oidx = 1;
    if (s->is_oidx && n) {
        for (int m = 0; m < s->nmode; ++m) {
            if (fib_reuse(s, m) > 4) continue;
            u64 *mk = nullptr, *mk2 = nullptr;
            u32 *io = nullptr, *io2 = nullptr;
            altob_status a = dmalloc_t(&mk, n);
            if (a == ALTOB_OK) a = dmalloc_t(&mk2, n);
            if (a == ALTOB_OK) a = dmalloc_t(&io, n);
            if (a == ALTOB_OK) a = dmalloc_t(&io2, n);
            bool alt = false;
            if (a == ALTOB_OK) {
                k_mode_keys<<<grid_for(n, 256), 256, 0, st>>>(s->d_klo, hi, n, s->fld, m, mk, io);
                if (cudaGetLastError() != cudaSuccess) a = fail(ALTOB_ERR_CUDA, "k_mode_keys launch failed");
            }
            if (a == ALTOB_OK) a = radix_sort_pairs(mk, nullptr, io, mk2, nullptr, io2, n, 1, mode_bits(s->dims[m]), st, &alt);
            dfree(mk);
            dfree(mk2);
            if (a == ALTOB_OK) {
                s->d_oidx[m] = alt ? io2 : io;
                dfree(alt ? io : io2);
            } else {
                dfree(io);
                dfree(io2);
                return a;
            }
        }
    }
    // partitions and intervals of the slice
    const int np = nprtn, nm = s->nmode;
    const u64 per = (n + (u64)np - 1) / (u64)np;
    s->prtn_ptr.assign(np + 1, 0);
    for (int p = 0; p < np; ++p) s->prtn_ptr[p + 1] = std::min<u64>((u64)(p + 1) * per, n);
    u64 dm[5] = {1, 1, 1, 1, 1};
    for (int m = 0; m < nm; ++m) dm[m] = s->dims[m];
    u64* d_iv = nullptr;
    ALTOB_TRY(dmalloc_t(&d_iv, (u64)np * nm * 2));
    k_init_intervals<<<(np * nm + 255) / 256, 256, 0, st>>>(d_iv, np, nm, dm[0], dm[1], dm[2], dm[3], dm[4]);
    if (n) k_intervals<<<grid_for(n, 256), 256, 0, st>>>(s->d_klo, hi, n, s->fld, per, d_iv);
    s->intervals.assign((size_t)np * nm * 2, 0);
    cudaMemcpyAsync(s->intervals.data(), d_iv, s->intervals.size() * sizeof(u64), cudaMemcpyDeviceToHost, st);
    const cudaError_t e = cudaStreamSynchronize(st);
    dfree(d_iv);
    if (e != cudaSuccess) return fail(ALTOB_ERR_CUDA, std::string("slice: ") + cudaGetErrorString(e));
    s->device_bytes = n * (8 * (s->d_khi ? 2 : 1) + vsz) + (u64)s->nrun * 16;
    for (int m = 0; m < nm; ++m)
        if (s->d_oidx[m]) s->device_bytes += n * 4;
    return ALTOB_OK;
}

}  // namespace altob

using namespace altob;

extern "C" {

const char* altob_status_string(altob_status s)
{
    switch (s) {
    case ALTOB_OK: return "ok";
    case ALTOB_ERR_ARG: return "invalid argument";
    case ALTOB_ERR_BITS: return "ALTO bits exceed the index width";
    case ALTOB_ERR_CUDA: return "CUDA error";
    case ALTOB_ERR_NOMEM: return "out of memory";
    case ALTOB_ERR_IO: return "I/O error";
    case ALTOB_ERR_UNSUPPORTED: return "unsupported";
    case ALTOB_ERR_NOT_FOUND: return "no CUDA device";
    }
    return "unknown status";
}

const char* altob_last_error(void) { return g_last_error.c_str(); }

const char* altob_version(void) { return "alto_b200 0.1.0 (sm_100a)"; }

altob_status altob_create(int nmode, const uint64_t* dims, uint64_t nnz, const uint64_t* cidx, const void* vals,
                          altob_dtype val_dtype, int nprtn, int lit_bits, void* stream, altob_tensor** out)
{
    if (!dims) return fail(ALTOB_ERR_ARG, "dims is NULL");
    if (nmode < 1 || nmode > ALTOB_MAX_MODES) return fail(ALTOB_ERR_ARG, "nmode must be 1..5");
    cudaStream_t st = (cudaStream_t)stream;
    StreamScope scope(st);
    u64* d_cidx = nullptr;
    void* d_vals = nullptr;
    size_t vsz = val_size(val_dtype);
    if (nnz) {
        if (!cidx || !vals) return fail(ALTOB_ERR_ARG, "cidx / vals is NULL");
        ALTOB_TRY(dmalloc_t(&d_cidx, (u64)nmode * nnz));
        altob_status s = dmalloc(&d_vals, nnz * vsz);
        if (s != ALTOB_OK) {
            dfree(d_cidx);
            return s;
        }
        cudaMemcpyAsync(d_cidx, cidx, (u64)nmode * nnz * sizeof(u64), cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_vals, vals, nnz * vsz, cudaMemcpyHostToDevice, st);
    }
    altob_status s = create_common(nmode, dims, nnz, d_cidx, d_vals, val_dtype, nprtn, lit_bits, st, out);
    cudaStreamSynchronize(st);
    dfree(d_cidx);
    dfree(d_vals);
    return s;
}

altob_status altob_create_device(int nmode, const uint64_t* dims, uint64_t nnz, const uint64_t* d_cidx,
                                 const void* d_vals, altob_dtype val_dtype, int nprtn, int lit_bits, void* stream,
                                 altob_tensor** out)
{
    if (!dims) return fail(ALTOB_ERR_ARG, "dims is NULL");
    StreamScope scope((cudaStream_t)stream);
    return create_common(nmode, dims, nnz, d_cidx, d_vals, val_dtype, nprtn, lit_bits, (cudaStream_t)stream, out);
}

altob_status altob_slice(const altob_tensor* t, uint64_t begin, uint64_t end, int nprtn, void* stream,
                         altob_tensor** out)
{
    if (!t || !out) return fail(ALTOB_ERR_ARG, "NULL argument");
    *out = nullptr;
    if (begin > end || end > t->nnz) return fail(ALTOB_ERR_ARG, "slice range outside the tensor");
    if (nprtn < 1) return fail(ALTOB_ERR_ARG, "nprtn must be >= 1");
    cudaStream_t st = (cudaStream_t)stream;
    StreamScope scope(st);
    ALTOB_TRY(tensor_enter(const_cast<altob_tensor*>(t), st));
    altob_tensor* s = new altob_tensor();
    const altob_status r = slice_impl(t, begin, end, nprtn, st, s);
    tensor_leave(const_cast<altob_tensor*>(t), st);
    if (r != ALTOB_OK) {
        altob_destroy(s);
        return r;
    }
    *out = s;
    return ALTOB_OK;
}

altob_status altob_destroy(altob_tensor* t)
{
    if (!t) return ALTOB_OK;
    // frees are ordered on the legacy default stream, i.e. after the work
    // already issued on blocking streams; work on non-blocking streams that
    // uses the tensor must be finished by the caller first
    StreamScope scope(0);
    if (t->use_ev) {  // after the last call that used the handle, on any stream
        cudaStreamWaitEvent(0, t->use_ev, 0);
        cudaEventDestroy(t->use_ev);
    }
    dfree(t->d_klo);
    dfree(t->d_khi);
    dfree(t->d_run_start);
    dfree(t->d_run_val);
    dfree(t->d_vals);
    for (int n = 0; n < ALTOB_MAX_MODES; ++n) dfree(t->d_oidx[n]);
    for (int n = 0; n < ALTOB_MAX_MODES; ++n) dfree(t->d_plan[n]);
    dfree(t->scratch);
    dfree(t->hotbuf);
    dfree(t->d_tma_err);
    if (t->h_tma_err) {
        cudaStreamSynchronize(0);  // the flag's last copy was ordered before the frees above
        cudaFreeHost(t->h_tma_err);
    }
    delete t;
    return ALTOB_OK;
}

altob_status altob_get_info(const altob_tensor* t, altob_info* o)
{
    if (!t || !o) return fail(ALTOB_ERR_ARG, "NULL argument");
    memset(o, 0, sizeof(*o));
    o->nmode = t->nmode;
    o->nprtn = t->nprtn;
    o->lit_bits = t->lit_bits;
    o->alto_bits = t->alto_bits;
    o->is_oidx = t->is_oidx;
    o->val_dtype = t->vdt;
    o->nnz = t->nnz;
    for (int n = 0; n < t->nmode; ++n) {
        o->dims[n] = t->dims[n];
        o->mode_masks[n][0] = (u64)t->masks[n];
        o->mode_masks[n][1] = (u64)(t->masks[n] >> 64);
        o->cr_masks[n][0] = (u64)t->cr_masks[n];
        o->cr_masks[n][1] = (u64)(t->cr_masks[n] >> 64);
    }
    o->alto_mask[0] = (u64)t->alto_mask;
    o->alto_mask[1] = (u64)(t->alto_mask >> 64);
    o->alto_cr_mask[0] = (u64)t->alto_cr_mask;
    o->alto_cr_mask[1] = (u64)(t->alto_cr_mask >> 64);
    o->device_bytes = t->device_bytes;
    o->key_bytes = t->d_khi ? 16 : 8;
    o->nruns = t->nrun;
    o->tma_err = t->h_tma_err ? (int)*t->h_tma_err : 0;
    for (int n = 0; n < t->nmode; ++n)
        if (t->d_plan[n]) {
            o->plan_modes |= 1 << n;
            o->plan_bytes += t->nnz * sizeof(uint16_t);
        }
    return ALTOB_OK;
}

altob_status altob_dump(const altob_tensor* t, uint64_t* idx, void* vals, uint64_t* prtn_ptr, uint64_t* intervals,
                        uint64_t* oidx, void* stream)
{
    if (!t) return fail(ALTOB_ERR_ARG, "NULL tensor");
    cudaStream_t st = (cudaStream_t)stream;
    StreamScope scope(st);
    const u64 nnz = t->nnz;
    if (idx && nnz) {
        u64 *olo = nullptr, *ohi = nullptr;
        ALTOB_TRY(dmalloc_t(&olo, nnz));
        altob_status s = dmalloc_t(&ohi, nnz);
        if (s != ALTOB_OK) {
            dfree(olo);
            return s;
        }
        k_interleave<<<grid_for(nnz, 256), 256, 0, st>>>(t->d_klo, key_src(t), t->alto_bits, nnz, t->dec, t->fld,
                                                         olo, ohi);
        std::vector<u64> lo(nnz), hi(nnz);
        cudaMemcpyAsync(lo.data(), olo, nnz * 8, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(hi.data(), ohi, nnz * 8, cudaMemcpyDeviceToHost, st);
        cudaError_t e = cudaStreamSynchronize(st);
        dfree(olo);
        dfree(ohi);
        if (e != cudaSuccess) return fail(ALTOB_ERR_CUDA, std::string("dump: ") + cudaGetErrorString(e));
        for (u64 i = 0; i < nnz; ++i) {
            idx[2 * i] = lo[i];
            idx[2 * i + 1] = hi[i];
        }
    }
    if (vals && nnz) ALTOB_CUDA(cudaMemcpyAsync(vals, t->d_vals, nnz * val_size(t->vdt), cudaMemcpyDeviceToHost, st));
    if (prtn_ptr) memcpy(prtn_ptr, t->prtn_ptr.data(), t->prtn_ptr.size() * sizeof(u64));
    if (intervals) memcpy(intervals, t->intervals.data(), t->intervals.size() * sizeof(u64));
    if (oidx && nnz) {
        std::vector<u32> tmp(nnz);
        for (int n = 0; n < t->nmode; ++n) {
            if (!t->d_oidx[n]) continue;
            ALTOB_CUDA(cudaMemcpyAsync(tmp.data(), t->d_oidx[n], nnz * 4, cudaMemcpyDeviceToHost, st));
            ALTOB_CUDA(cudaStreamSynchronize(st));
            for (u64 i = 0; i < nnz; ++i) oidx[(u64)n * nnz + i] = tmp[i];
        }
    }
    ALTOB_CUDA(cudaStreamSynchronize(st));
    return ALTOB_OK;
}

}  // extern "C"
