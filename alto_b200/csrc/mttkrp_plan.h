// mttkrp_plan.h -- host-side MTTKRP / Phi helpers shared by the solvers.
#pragma once

#include "internal.cuh"

namespace altob {

struct TiledPlan {
    int vec, lpn, ch, tile, hslots, grouped;
    int hot;  // hot-row slots per CTA (grouped kernel, FP32)
    size_t smem;
};

bool ptr_aligned16(const void* p);
altob_status plan_tiled(const altob_tensor* t, u64 R, size_t fsz, bool aligned, bool cache, TiledPlan* pl);
altob_algo resolve_algo(const altob_tensor* t, int mode, altob_algo algo);
// The tile plan of `mode` (built on first use; nullptr when plans are off or
// cannot be allocated).
const uint16_t* tensor_plan(altob_tensor* t, int mode, cudaStream_t st);
altob_status mttkrp_device(altob_tensor* t, int mode, altob_dtype ft, void* const* dU, u64 R, int accumulate,
                           altob_algo algo, cudaStream_t st);
altob_status phi_device(altob_tensor* t, int mode, altob_dtype ft, void* const* dU, u64 R, double eps,
                        void* dphi, cudaStream_t st);
// Khatri-Rao rows of every nonzero for `mode` (nnz x R, ALTO order) and Phi
// computed from them (CP-APR with precomputed rows).
// inv given: row i goes to stream row inv[i] (the row-ordered stream below).
altob_status pi_device(altob_tensor* t, int mode, altob_dtype ft, void* const* dU, u64 R, void* dpi,
                       cudaStream_t st, const u32* inv = nullptr);
altob_status phi_pre_device(altob_tensor* t, int mode, altob_dtype ft, const void* dpi, const void* dB, u64 R,
                            double eps, void* dphi, cudaStream_t st);
// Row-ordered stream of `mode` (CP-APR): rows[k], vals[k] (compute dtype)
// of the k-th nonzero in mode-index order, inv[i] = stream position of
// nonzero i; and Phi computed from it and the stream-ordered Khatri-Rao rows.
altob_status mode_order_device(altob_tensor* t, int mode, altob_dtype ft, u32* rows, void* svals, u32* inv,
                               cudaStream_t st);
// pad4: rows and svals may be read up to a multiple of 4 elements past the
// mode's nnz (and start 16-byte aligned), which lets the stream be staged by
// bulk copies.
altob_status phi_rows_device(altob_tensor* t, int mode, altob_dtype ft, const void* dpi, const u32* rows,
                             const void* svals, const void* dB, u64 R, double eps, void* dphi, cudaStream_t st,
                             bool pad4 = false);

}  // namespace altob
