// rebin.cu -- arc-to-flat detector rebin (rebinToPanel.m:1-36) on the device.
//
// The host builds, in FP64, one entry per flat-panel column: the two arc columns around its
// fan angle and their weights, with the reference's clamps (a column it skips gets no entry
// and stays zero; a fan position exactly on a cell centre gets weight 0 on both cells, as the
// reference's weights use the clamped indices). Blocks keep the table in shared memory and walk
// detector rows, one thread per output column blending two input elements of its row:
// HBM-bound, one read and one write per sample. The FP64 kernel multiplies and adds without
// contraction, in the reference's order.
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

// One block per group of rows: the column table goes to shared memory once, then the block
// walks its rows (row r = all N columns of one detector row of one view), thread per column.
template <typename T>
__global__ void k_rebin_panel(const T* __restrict__ in, T* __restrict__ out,
                              const PanelEntry* __restrict__ tab, int N, size_t rows) {
    extern __shared__ PanelEntry st[];
    for (int i = threadIdx.x; i < N; i += blockDim.x) st[i] = tab[i];
    __syncthreads();
    constexpr int RB = sizeof(T) == 8 ? 2 : 4;  // rows per step: independent loads in flight
    for (size_t r0 = (size_t)blockIdx.x * RB; r0 < rows; r0 += (size_t)gridDim.x * RB) {
        const int nr = (int)(rows - r0 < (size_t)RB ? rows - r0 : (size_t)RB);
        for (int i = threadIdx.x; i < N; i += blockDim.x) {
            const PanelEntry t = st[i];
            T a[RB], b[RB];
#pragma unroll
            for (int q = 0; q < RB; ++q) {
                a[q] = T(0);
                b[q] = T(0);
                if (q < nr && t.lo >= 0) {
                    const T* row = in + (r0 + q) * (size_t)N;
                    a[q] = row[t.lo];
                    b[q] = row[t.hi];
                }
            }
#pragma unroll
            for (int q = 0; q < RB; ++q) {
                if (q >= nr) break;
                T v = T(0);
                if (t.lo >= 0) {
                    if constexpr (sizeof(T) == 8)
                        v = __dadd_rn(__dmul_rn(a[q], t.wl), __dmul_rn(b[q], t.wh));
                    else
                        v = fmaf(a[q], (float)t.wl, b[q] * (float)t.wh);
                }
                out[(r0 + q) * (size_t)N + i] = v;
            }
        }
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
        const size_t rows = (size_t)H * P;
        const size_t smem = (size_t)N * sizeof(PanelEntry);
        if (smem > 200 * 1024)
            return fin(make_status(CTRECON_ERR_UNSUPPORTED, "panel rebin: more than 8533 columns"));
        if (smem > 48 * 1024) {
            e = cudaFuncSetAttribute(k_rebin_panel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem);
            if (e != cudaSuccess) return fin(cuda_status(e, "cudaFuncSetAttribute"));
        }
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
        const int threads = N >= 512 ? 256 : 128;
        const unsigned grid = (unsigned)std::min<size_t>((rows + 3) / 4, (size_t)sms * 8);
        k_rebin_panel<T><<<grid, threads, smem, s>>>(d_in, d_out, ctx->ws_panel.as<PanelEntry>(), N,
                                                     rows);
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
