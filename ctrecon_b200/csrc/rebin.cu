// rebin.cu -- arc-to-flat detector rebin (rebinToPanel.m:1-36) on the device.
//
// The host builds, in FP64, one entry per flat-panel column: the two arc columns around its
// fan angle and their weights, with the reference's clamps (a column it skips gets no entry
// and stays zero; a fan position exactly on a cell centre gets weight 0 on both cells, as the
// reference's weights use the clamped indices). One thread per output element then blends two
// input elements of its row: HBM-bound, 8 (FP32) or 16 (FP64) bytes read and 4 or 8 written per
// element. The FP64 kernel multiplies and adds without contraction, in the reference's order.
#include "internal.h"

#include <cmath>
#include <vector>

namespace ctr {
void set_noctx_error(const std::string& m);
}
using namespace ctr;

namespace {

struct PanelEntry { int lo, hi; double wl, wh; };  // lo < 0: column stays zero

// rebinToPanel.m:6-33 in FP64; returns the panel width (:9)
double panel_table(int N, double c, double w, double D, std::vector<PanelEntry>& t) {
    const double oneFanAngle = std::atan(w / 2 / D) * 2.0;
    const double a1 = (c + 0.5) * oneFanAngle, a2 = (N - 1 - c + 0.5) * oneFanAngle;
    const double largerAngle = a1 > a2 ? a1 : a2;
    const double detWidth = std::tan(largerAngle) * D * 2;
    const double newW = detWidth / N;
    t.assign(N, PanelEntry{-1, -1, 0.0, 0.0});
    for (int ii = 1; ii <= N; ++ii) {
        const double fanAngle = std::atan((ii - (N + 1) / 2.0) * newW / D);
        const double idx = fanAngle / oneFanAngle + c + 1;
        double lowIdx = std::floor(idx), higIdx = std::ceil(idx);
        if (lowIdx < 1) lowIdx = 1;
        if (higIdx < 1) continue;
        if (lowIdx > N) continue;
        if (higIdx > N) higIdx = N;
        t[ii - 1] = PanelEntry{(int)lowIdx - 1, (int)higIdx - 1, higIdx - idx, idx - lowIdx};
    }
    return detWidth;
}

template <typename T>
__global__ void k_rebin_panel(const T* __restrict__ in, T* __restrict__ out,
                              const PanelEntry* __restrict__ tab, int N, size_t total) {
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(e % (size_t)N);
        const PanelEntry t = tab[i];
        const T* row = in + (e - i);
        T v = T(0);
        if (t.lo >= 0) {
            if constexpr (sizeof(T) == 8)
                v = __dadd_rn(__dmul_rn(row[t.lo], t.wl), __dmul_rn(row[t.hi], t.wh));
            else
                v = fmaf(row[t.lo], (float)t.wl, row[t.hi] * (float)t.wh);
        }
        out[e] = v;
    }
}

template <typename T>
ctrecon_status rebin_dev(ctrecon_ctx* ctx, cudaStream_t s, const T* d_in, int N, int H, int P,
                         double c, double w, double D, T* d_out, double* width) {
    if (!ctx) return CTRECON_ERR_INVALID_ARGUMENT;
    auto fin = [&](const Status& st) {
        if (!st.ok()) ctx->last_error = st.msg;
        else ctx->last_error.clear();
        return st.code;
    };
    if (!d_in || !d_out || N < 1 || H < 1 || P < 1 || !(D > 0) || !(w > 0) || !std::isfinite(c))
        return fin(make_status(CTRECON_ERR_INVALID_ARGUMENT, "bad panel-rebin arguments"));
    if (d_in == d_out)
        return fin(make_status(CTRECON_ERR_INVALID_ARGUMENT, "panel rebin needs distinct input and output"));
    try {
        cudaError_t e = cudaSetDevice(ctx->device);
        if (e != cudaSuccess) return fin(cuda_status(e, "cudaSetDevice"));
        std::vector<PanelEntry> tab;
        const double wd = panel_table(N, c, w, D, tab);
        if (width) *width = wd;
        // the table lives in the context's panel buffer; the upload waits for the device, so
        // a previous rebin still reading it has finished
        Status st = ctx->ws_panel.ensure(tab.size() * sizeof(PanelEntry), "panel-rebin table");
        if (st.ok()) st = upload_now(ctx->ws_panel.ptr, tab.data(), tab.size() * sizeof(PanelEntry));
        if (!st.ok()) return fin(st);
        const size_t total = (size_t)N * H * P;
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
        const size_t want = (total + 255) / 256;
        const unsigned grid = (unsigned)std::min<size_t>(want, (size_t)sms * 16);
        k_rebin_panel<T><<<grid, 256, 0, s>>>(d_in, d_out, ctx->ws_panel.as<PanelEntry>(), N, total);
        e = cudaGetLastError();
        if (e != cudaSuccess) return fin(cuda_status(e, "k_rebin_panel"));
        return fin(Status::Ok());
    } catch (const std::exception& ex) {
        return fin(make_status(CTRECON_ERR_INTERNAL, ex.what()));
    }
}

}  // namespace

extern "C" {

ctrecon_status ctrecon_rebin_to_panel_dev_f32(ctrecon_ctx* ctx, void* stream, const float* d_proj,
                                              int det_num, int det_hei, int prj_num,
                                              double det_center_idx, double det_cell_width,
                                              double sour_to_det, float* d_out,
                                              double* det_width) {
    return rebin_dev<float>(ctx, (cudaStream_t)stream, d_proj, det_num, det_hei, prj_num,
                            det_center_idx, det_cell_width, sour_to_det, d_out, det_width);
}

ctrecon_status ctrecon_rebin_to_panel_dev_f64(ctrecon_ctx* ctx, void* stream, const double* d_proj,
                                              int det_num, int det_hei, int prj_num,
                                              double det_center_idx, double det_cell_width,
                                              double sour_to_det, double* d_out,
                                              double* det_width) {
    return rebin_dev<double>(ctx, (cudaStream_t)stream, d_proj, det_num, det_hei, prj_num,
                             det_center_idx, det_cell_width, sour_to_det, d_out, det_width);
}

}  // extern "C"
