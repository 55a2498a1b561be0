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
altob_status mttkrp_device(altob_tensor* t, int mode, altob_dtype ft, void* const* dU, u64 R, int accumulate,
                           altob_algo algo, cudaStream_t st);
altob_status phi_device(altob_tensor* t, int mode, altob_dtype ft, void* const* dU, u64 R, double eps,
                        void* dphi, cudaStream_t st);
// Khatri-Rao rows of every nonzero for `mode` (nnz x R, ALTO order) and Phi
// computed from them (CP-APR with precomputed rows).
altob_status pi_device(altob_tensor* t, int mode, altob_dtype ft, void* const* dU, u64 R, void* dpi,
                       cudaStream_t st);
altob_status phi_pre_device(altob_tensor* t, int mode, altob_dtype ft, const void* dpi, const void* dB, u64 R,
                            double eps, void* dphi, cudaStream_t st);

}  // namespace altob
