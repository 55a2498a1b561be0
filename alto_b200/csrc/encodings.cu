// encodings.cu -- the reference's alternative ALTO encodings, from a tensor
// handle.
//
// ALT_PEXT (IntelLabs/ALTO include/alto.hpp:35-37, 212-244, 695-700): after
// the sort, every key is re-encoded with each mode's index as a contiguous
// bit field at mode_pos[n], the running sum of the bit counts in mode order
// (setup_packed_alto computes it before ordering the modes, alto.hpp:
// 695-700), and the mode masks become (1 << bits) - 1.  The device keys of
// this library already keep every mode as a contiguous field (that layout is
// what makes a mode index one funnel shift on the GPU), placed in ALTO level
// order so that the high key word is monotone; the re-encode is a
// relabelling of fields.  altob_dump_alt_pext writes the keys and masks a
// -DALT_PEXT build of the reference holds, CR bits included.
//
// OPT_ALTO (alto.hpp:18-20, 49-53, 838-868): per partition, the ALTO bits
// its first and last keys share (prefix_bits, counted from the top ALTO
// bit), the partition's id (those bits), their mask, and each mode mask
// restricted to them.  The reference computes them before setting the CR
// bits and keeps them as 64-bit words; altob_partition_ids returns the same.
#include <algorithm>
#include <cstring>
#include <vector>

#include "internal.cuh"

namespace altob {

namespace {

__device__ __forceinline__ int clz128(u128 x, int width)
{
    const u64 hi = (u64)(x >> 64), lo = (u64)x;
    if (width == 64) return lo ? __clzll((long long)lo) : 64;
    if (hi) return __clzll((long long)hi);
    return 64 + (lo ? __clzll((long long)lo) : 64);
}

// ALT_PEXT keys: fields at mode_pos, CR bits (alto_bits and up) kept.
__global__ void k_alt_pext(const u64* __restrict__ klo, KeySrc ks, int alto_bits, u64 n, Fields f, int nmode,
                           const int* __restrict__ mode_pos, u64* __restrict__ out)
{
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const u64 lo = klo[i], hi = key_hi(ks, i);
        u128 key = 0;
        for (int m = 0; m < nmode; ++m) key |= (u128)field(lo, hi, f.pos[m], f.mask[m]) << mode_pos[m];
        const u128 full = ((u128)hi << 64) | lo;
        key |= (full >> alto_bits) << alto_bits;
        out[2 * i] = (u64)key;
        out[2 * i + 1] = (u64)(key >> 64);
    }
}

// OPT_ALTO partition ids from the interleaved keys without CR bits.
__global__ void k_prtn_ids(const u64* __restrict__ ilo, const u64* __restrict__ ihi, const u64* __restrict__ ptr,
                           int nprtn, int nmode, int lit_bits, int alto_bits, u128 alto_mask,
                           const u64* __restrict__ masks, u64* __restrict__ id, u64* __restrict__ pmask,
                           u64* __restrict__ mmask)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nprtn) return;
    const u64 s = ptr[p], e = ptr[p + 1];
    id[p] = 0;
    pmask[p] = 0;
    for (int m = 0; m < nmode; ++m) mmask[(u64)p * nmode + m] = 0;
    if (s == e) return;  // empty partition: left zero (alto.hpp:865)
    const u128 a = (((u128)ihi[s] << 64) | ilo[s]) & alto_mask;
    const u128 b = (((u128)ihi[e - 1] << 64) | ilo[e - 1]) & alto_mask;
    const int prefix = clz128(a ^ b, lit_bits) - (lit_bits - alto_bits);
    // bits 0 .. prefix-1 set one by one as 64-bit words (alto.hpp:849-851); a
    // prefix of 64 bits or more sets every bit
    const u64 pm = prefix >= 64 ? ~0ull : ((1ull << prefix) - 1ull);
    const int sh = alto_bits - prefix;
    pmask[p] = pm;
    id[p] = (u64)(a >> sh) & pm;
    for (int m = 0; m < nmode; ++m) {
        const u128 mm = ((u128)masks[2 * m + 1] << 64) | masks[2 * m];
        mmask[(u64)p * nmode + m] = (u64)(mm >> sh) & pm;
    }
}

// Key bits per mode and the reference's mode_pos (running sum in mode order).
void alt_pext_layout(const altob_tensor* t, int* pos, int* bits)
{
    for (int n = 0; n < t->nmode; ++n) {
        const u64 d = t->dims[n];
        bits[n] = d <= 1 ? 0 : 64 - __builtin_clzll(d - 1);
    }
    pos[0] = 0;
    for (int n = 1; n < t->nmode; ++n) pos[n] = pos[n - 1] + bits[n - 1];
}

int grid_of(u64 n)
{
    return (int)std::max<u64>(1, std::min<u64>((n + 255) / 256, (u64)num_sms() * 16));
}

}  // namespace

}  // namespace altob

using namespace altob;

extern "C" altob_status altob_dump_alt_pext(const altob_tensor* t, uint64_t* idx, uint64_t* mode_masks, int* mode_pos,
                                            void* stream)
{
    if (!t) return fail(ALTOB_ERR_ARG, "NULL tensor");
    int pos[ALTOB_MAX_MODES], bits[ALTOB_MAX_MODES];
    alt_pext_layout(t, pos, bits);
    for (int n = 0; n < t->nmode; ++n) {
        if (bits[n] >= 31)
            return fail(ALTOB_ERR_UNSUPPORTED, "ALT_PEXT: the reference's mode mask (1 << bits) - 1 is an int "
                                               "expression, undefined for 31 or more bits");
        if (pos[n] + bits[n] > t->lit_bits) return fail(ALTOB_ERR_BITS, "ALT_PEXT: a field passes the index width");
    }
    if (mode_pos) memcpy(mode_pos, pos, t->nmode * sizeof(int));
    if (mode_masks)
        for (int n = 0; n < t->nmode; ++n) {
            mode_masks[2 * n] = (1ull << bits[n]) - 1ull;
            mode_masks[2 * n + 1] = 0;
        }
    const u64 nnz = t->nnz;
    if (!idx || !nnz) return ALTOB_OK;
    cudaStream_t st = (cudaStream_t)stream;
    StreamScope scope(st);
    u64* out = nullptr;
    int* dpos = nullptr;
    ALTOB_TRY(dmalloc_t(&out, 2 * nnz));
    altob_status s = dmalloc_t(&dpos, ALTOB_MAX_MODES);
    if (s == ALTOB_OK) {
        cudaMemcpyAsync(dpos, pos, sizeof(pos), cudaMemcpyHostToDevice, st);
        k_alt_pext<<<grid_of(nnz), 256, 0, st>>>(t->d_klo, key_src(t), t->alto_bits, nnz, t->fld, t->nmode, dpos, out);
        cudaMemcpyAsync(idx, out, 2 * nnz * 8, cudaMemcpyDeviceToHost, st);
        const cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) s = fail(ALTOB_ERR_CUDA, std::string("ALT_PEXT dump: ") + cudaGetErrorString(e));
    }
    dfree(out);
    dfree(dpos);
    return s;
}

// Interleaved keys (the reference's default encoding) of a handle, on the
// device; implemented beside the encoder.
namespace altob {
altob_status interleaved_keys(const altob_tensor* t, u64* olo, u64* ohi, cudaStream_t st);
}

extern "C" altob_status altob_partition_ids(const altob_tensor* t, uint64_t* prtn_id, uint64_t* prtn_mask,
                                            uint64_t* prtn_mode_masks, void* stream)
{
    if (!t || !prtn_id || !prtn_mask || !prtn_mode_masks) return fail(ALTOB_ERR_ARG, "NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    StreamScope scope(st);
    const int np = t->nprtn, nm = t->nmode;
    const u64 nnz = t->nnz;
    u64 *lo = nullptr, *hi = nullptr, *ptr = nullptr, *masks = nullptr, *id = nullptr, *pm = nullptr, *mm = nullptr;
    struct Free {
        std::vector<void*> v;
        ~Free()
        {
            for (void* p : v) dfree(p);
        }
    } fr;
    auto get = [&](u64** p, u64 n) {
        const altob_status s = dmalloc_t(p, std::max<u64>(1, n));
        if (s == ALTOB_OK) fr.v.push_back(*p);
        return s;
    };
    ALTOB_TRY(get(&lo, nnz));
    ALTOB_TRY(get(&hi, nnz));
    ALTOB_TRY(get(&ptr, np + 1));
    ALTOB_TRY(get(&masks, 2 * ALTOB_MAX_MODES));
    ALTOB_TRY(get(&id, np));
    ALTOB_TRY(get(&pm, np));
    ALTOB_TRY(get(&mm, (u64)np * nm));
    if (nnz) ALTOB_TRY(interleaved_keys(t, lo, hi, st));
    u64 hm[2 * ALTOB_MAX_MODES] = {0};
    for (int n = 0; n < nm; ++n) {
        hm[2 * n] = (u64)t->masks[n];
        hm[2 * n + 1] = (u64)(t->masks[n] >> 64);
    }
    ALTOB_CUDA(cudaMemcpyAsync(ptr, t->prtn_ptr.data(), (np + 1) * 8, cudaMemcpyHostToDevice, st));
    ALTOB_CUDA(cudaMemcpyAsync(masks, hm, sizeof(hm), cudaMemcpyHostToDevice, st));
    k_prtn_ids<<<(np + 127) / 128, 128, 0, st>>>(lo, hi, ptr, np, nm, t->lit_bits, t->alto_bits, t->alto_mask, masks,
                                                id, pm, mm);
    ALTOB_LAUNCH_CHECK();
    ALTOB_CUDA(cudaMemcpyAsync(prtn_id, id, np * 8, cudaMemcpyDeviceToHost, st));
    ALTOB_CUDA(cudaMemcpyAsync(prtn_mask, pm, np * 8, cudaMemcpyDeviceToHost, st));
    ALTOB_CUDA(cudaMemcpyAsync(prtn_mode_masks, mm, (u64)np * nm * 8, cudaMemcpyDeviceToHost, st));
    ALTOB_CUDA(cudaStreamSynchronize(st));
    return ALTOB_OK;
}
