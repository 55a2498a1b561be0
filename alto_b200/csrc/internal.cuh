// internal.cuh -- shared definitions of the alto_b200 CUDA library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>

#include <string>
#include <vector>

#include "../../include/altob.h"

typedef unsigned __int128 u128;
typedef uint64_t u64;
typedef uint32_t u32;

namespace altob {

// ---------------------------------------------------------------- errors

void set_error(const std::string& msg);
altob_status fail(altob_status s, const std::string& msg);

#define ALTOB_CUDA(call)                                                          \
    do {                                                                          \
        cudaError_t e_ = (call);                                                  \
        if (e_ != cudaSuccess)                                                    \
            return ::altob::fail(ALTOB_ERR_CUDA, std::string(#call) + ": " +      \
                                                     cudaGetErrorString(e_));     \
    } while (0)

#define ALTOB_TRY(expr)                                                           \
    do {                                                                          \
        altob_status s_ = (expr);                                                 \
        if (s_ != ALTOB_OK) return s_;                                            \
    } while (0)

// Checks the launch that was just issued.
#define ALTOB_LAUNCH_CHECK() ALTOB_CUDA(cudaGetLastError())

// ------------------------------------------------ bit compress / expand
//
// pext / pdep replacement.  For a 32-bit mask m the published "compress"
// method (H. S. Warren, Hacker's Delight, 2nd ed., section 7-4) moves the
// selected bits right in five steps whose move masks mv[0..4] depend only
// on m; "expand" (section 7-5) applies the same moves in reverse.  The move
// masks are computed once per tensor on the host, so decoding a mode index
// from a key is at most five (and, xor/or, shift) triples per key word.

struct WordDec {
    u32 m;       // mask bits of this mode inside the 32-bit key word
    u32 off;     // bit offset of this word's bits inside the mode index
    u32 mv[5];   // move masks
};

struct ModeDec {
    WordDec w[4];
};

struct Decoder {
    int nmode;
    int nwords;  // 32-bit key words spanned by the ALTO bits
    ModeDec md[ALTOB_MAX_MODES];
};

// Host: move masks of the compress/expand network for mask m.
inline void compress_moves(u32 m, u32 mv[5])
{
    u32 mk = ~m << 1;
    for (int i = 0; i < 5; ++i) {
        u32 mp = mk ^ (mk << 1);
        mp ^= mp << 2;
        mp ^= mp << 4;
        mp ^= mp << 8;
        mp ^= mp << 16;
        u32 v = mp & m;
        mv[i] = v;
        m = (m ^ v) | (v >> (1u << i));
        mk &= ~mp;
    }
}

__host__ __device__ __forceinline__ u32 compress32(u32 x, const WordDec& d)
{
    x &= d.m;
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        u32 v = d.mv[i];
        if (v) {
            u32 t = x & v;
            x = (x ^ t) | (t >> (1u << i));
        }
    }
    return x;
}

__host__ __device__ __forceinline__ u32 expand32(u32 x, const WordDec& d)
{
#pragma unroll
    for (int i = 4; i >= 0; --i) {
        u32 v = d.mv[i];
        if (v) {
            u32 t = x << (1u << i);
            x = (x & ~v) | (t & v);
        }
    }
    return x & d.m;
}

// Mode index of a key given as up to four 32-bit words.
__host__ __device__ __forceinline__ u32 decode_mode(const u32* kw, const ModeDec& md, int nwords)
{
    u32 c = 0;
#pragma unroll
    for (int w = 0; w < 4; ++w)
        if (w < nwords && md.w[w].m) c |= compress32(kw[w], md.w[w]) << md.w[w].off;
    return c;
}

__host__ __device__ __forceinline__ void split_key(u64 lo, u64 hi, u32 kw[4])
{
    kw[0] = (u32)lo;
    kw[1] = (u32)(lo >> 32);
    kw[2] = (u32)hi;
    kw[3] = (u32)(hi >> 32);
}

Decoder make_decoder(int nmode, const u128* masks, int alto_bits);

// ------------------------------------------------ device key layout
//
// On the device a key keeps the ALTO sort order but stores each mode index
// as a contiguous bit field (the reference's ALT_PEXT re-encode,
// alto.hpp:212-244), so reading a mode index is one funnel shift and a mask
// instead of a bit gather.  Fields are laid out in the ALTO level order
// (shortest mode first), which puts the longest mode's top bits at the top of
// the key: those are exactly the most significant ALTO bits, so the key bits
// above bit 63 are non-decreasing along the sorted stream and can be kept as
// a short run table instead of a second word per nonzero.  CR bits stay at
// the reference's positions (alto_bits + k).

struct Fields {
    int nmode;
    u32 pos[ALTOB_MAX_MODES];
    u32 mask[ALTOB_MAX_MODES];
};

__host__ __device__ __forceinline__ u32 field(u64 lo, u64 hi, u32 pos, u32 mask)
{
    u64 v;
    if (pos >= 64) v = hi >> (pos - 64);
    else if (pos == 0) v = lo;
    else v = (lo >> pos) | (hi << (64 - pos));
    return (u32)v & mask;
}

// Where the high key word of nonzero i comes from.
struct KeySrc {
    const u64* klo;
    const u64* khi;        // one high word per nonzero, or nullptr
    const u64* run_start;  // else: sorted run starts of the high word ...
    const u64* run_val;    // ... and its value on each run
    int nrun;              // 0: the high word is 0
};

__device__ __forceinline__ u64 key_hi(const KeySrc& k, u64 i)
{
    if (k.khi) return k.khi[i];
    if (k.nrun == 0) return 0;
    int lo = 0, hi = k.nrun - 1;  // last run with start <= i
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (k.run_start[mid] <= i) lo = mid;
        else hi = mid - 1;
    }
    return k.run_val[lo];
}

// ------------------------------------------------------------- tensor

}  // namespace altob

struct altob_tensor {
    int device = 0;
    int nmode = 0, nprtn = 0, lit_bits = 64, alto_bits = 0, is_oidx = 0;
    int kw = 1;  // u64 key words kept on the device (1: key incl. CR bits < 2^64)
    altob_dtype vdt = ALTOB_F64;
    u64 nnz = 0;
    u64 dims[ALTOB_MAX_MODES] = {0};
    u128 masks[ALTOB_MAX_MODES] = {0};
    u128 cr_masks[ALTOB_MAX_MODES] = {0};
    u128 alto_mask = 0, alto_cr_mask = 0;
    altob::Decoder dec;   // interleaved <-> fields conversion (build / dump)
    altob::Fields fld;    // device key layout
    int order[ALTOB_MAX_MODES] = {0};  // ALTO level order of the modes
    // device arrays
    u64* d_klo = nullptr;
    u64* d_khi = nullptr;       // explicit high words (or nullptr)
    u64* d_run_start = nullptr; // implicit high words: run table
    u64* d_run_val = nullptr;
    int nrun = 0;
    void* d_vals = nullptr;
    u32* d_oidx[ALTOB_MAX_MODES] = {nullptr};
    // host copies of the small partition tables
    std::vector<u64> prtn_ptr;   // nprtn + 1
    std::vector<u64> intervals;  // nprtn * nmode * 2
    u64 device_bytes = 0;
    // cached scratch (grown on demand, freed with the handle)
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    // per-CTA hot-row accumulators of the grouped kernel (grown on demand)
    void* hotbuf = nullptr;
    size_t hotbuf_bytes = 0;
    // tile plans of the planned MTTKRP kernel, one per mode (built on first use)
    uint16_t* d_plan[ALTOB_MAX_MODES] = {nullptr};
    // the TMA-staged kernel's wait-limit flag: on the device, and a pinned
    // host copy refreshed after each of its launches
    unsigned* d_tma_err = nullptr;
    unsigned* h_tma_err = nullptr;
    // the stream of the last call that used the cached buffers or plans, and
    // an event recorded there: a call on another stream waits for it first
    cudaEvent_t use_ev = nullptr;
    cudaStream_t use_stream = nullptr;
};

namespace altob {

inline size_t val_size(altob_dtype d) { return d == ALTOB_F64 ? 8 : 4; }

inline KeySrc key_src(const altob_tensor* t)
{
    KeySrc k;
    k.klo = t->d_klo;
    k.khi = t->d_khi;
    k.run_start = t->d_run_start;
    k.run_val = t->d_run_val;
    k.nrun = t->nrun;
    return k;
}
inline u64 fib_reuse(const altob_tensor* t, int n) { return t->nnz / t->dims[n]; }

// Device allocation helpers that record failures as ALTOB_ERR_NOMEM.  They
// use the stream-ordered allocator on the stream of the entry point that is
// running on this thread (StreamScope), so freeing never waits for work on
// other streams.
struct StreamScope {
    cudaStream_t prev;
    explicit StreamScope(cudaStream_t s);
    ~StreamScope();
};
altob_status dmalloc(void** p, size_t bytes);
template <typename T>
altob_status dmalloc_t(T** p, size_t count)
{
    return dmalloc(reinterpret_cast<void**>(p), count * sizeof(T) + (count == 0));
}
void dfree(void* p);

// Per-tensor scratch: returns a device buffer of at least `bytes`, reused
// across calls on the same handle.
altob_status tensor_scratch(altob_tensor* t, size_t bytes, void** out);
altob_status tensor_hotbuf(altob_tensor* t, size_t bytes, void** out);

// Stream ordering of a handle's shared state (scratch, hot-row buffers, tile
// plans): tensor_enter makes stream st wait for the last call that used the
// handle on a different stream; tensor_leave records that this call's work
// was issued on st.  Both do nothing while st is being captured.
altob_status tensor_enter(altob_tensor* t, cudaStream_t st);
altob_status tensor_leave(altob_tensor* t, cudaStream_t st);
struct TensorUse {
    altob_tensor* t;
    cudaStream_t st;
    TensorUse(altob_tensor* t_, cudaStream_t st_) : t(t_), st(st_) {}
    ~TensorUse() { if (t) tensor_leave(t, st); }
};

int num_sms();

// Integer setting from the environment (dflt when unset or empty).
inline int env_int(const char* name, int dflt)
{
    const char* v = getenv(name);
    return v && *v ? atoi(v) : dflt;
}

// Stable LSD radix sort of (key, payload) pairs on key bits [0, nbits).
// Keys are kw u64 words (lo[], hi[]); payload is u32.  Ping-pong buffers
// are provided by the caller; the result ends in the *_out arrays.
altob_status radix_sort_pairs(u64* klo, u64* khi, u32* pay, u64* klo_alt,
                              u64* khi_alt, u32* pay_alt, u64 n, int kw,
                              int nbits, cudaStream_t st, bool* result_in_alt);

}  // namespace altob
