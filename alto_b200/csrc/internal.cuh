// internal.cuh -- shared definitions of the alto_b200 CUDA library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

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
    altob::Decoder dec;
    // device arrays
    u64* d_klo = nullptr;
    u64* d_khi = nullptr;
    void* d_vals = nullptr;
    u32* d_oidx[ALTOB_MAX_MODES] = {nullptr};
    // host copies of the small partition tables
    std::vector<u64> prtn_ptr;   // nprtn + 1
    std::vector<u64> intervals;  // nprtn * nmode * 2
    u64 device_bytes = 0;
    // cached scratch (grown on demand, freed with the handle)
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
};

namespace altob {

inline size_t val_size(altob_dtype d) { return d == ALTOB_F64 ? 8 : 4; }
inline u64 fib_reuse(const altob_tensor* t, int n) { return t->nnz / t->dims[n]; }

// Device allocation helpers that record failures as ALTOB_ERR_NOMEM.
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

int num_sms();

// Stable LSD radix sort of (key, payload) pairs on key bits [0, nbits).
// Keys are kw u64 words (lo[], hi[]); payload is u32.  Ping-pong buffers
// are provided by the caller; the result ends in the *_out arrays.
altob_status radix_sort_pairs(u64* klo, u64* khi, u32* pay, u64* klo_alt,
                              u64* khi_alt, u32* pay_alt, u64 n, int kw,
                              int nbits, cudaStream_t st, bool* result_in_alt);

}  // namespace altob
