// hilbert_tc.cu -- tensor-core (tcgen05) Toeplitz GEMM form of the Hilbert filter.
#include "internal.h"

namespace ctr {

size_t hilbert_tc_kappa_bytes(const FilterPlan& plan, int nviews, int mode) {
    (void)plan; (void)nviews; (void)mode;
    return 0;
}

Status launch_split_kappa(cudaStream_t s, const FilterPlan& plan, const float* X, int nviews,
                          void* Xsplit, int mode) {
    (void)s; (void)plan; (void)X; (void)nviews; (void)Xsplit; (void)mode;
    return make_status(CTRECON_ERR_UNSUPPORTED, "tensor-core Hilbert filter not built");
}

Status launch_hilbert_tc(ctrecon_ctx* ctx, cudaStream_t s, FilterPlan& plan, const void* Xsplit,
                         int nviews, float* d_fproj_chunk, int mode) {
    (void)ctx; (void)s; (void)plan; (void)Xsplit; (void)nviews; (void)d_fproj_chunk; (void)mode;
    return make_status(CTRECON_ERR_UNSUPPORTED, "tensor-core Hilbert filter not built");
}

}  // namespace ctr
