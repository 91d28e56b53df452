/*
 * KatsevichFiltering_GPU -- MEX entry point with the reference's call contract
 * (KatsevichFiltering_GPU.cu:939-978; caller KatsevichFiltering.m:37-38):
 *
 *   KatsevichFiltering_GPU(Proj, ProjScale, DecWidth, DecHeigh, ScanR, StdDis, HelicP,
 *                          FilterCoeFF, DeltaAngle, FilteringMode, YL, ZL, ProjNumber, FProj)
 *
 * 14 double inputs, no outputs; the filtered projections are written in place into the
 * 14th argument (the caller pre-sets FProj = Proj). Integer arguments arrive as doubles
 * and are truncated, as the reference does (:957-959). Unlike the reference, the sizes
 * are checked against the arrays before anything is read.
 *
 * Build against MATLAB's mex.h for MATLAB, or against the project's shim for the
 * standalone harness (ctrecon_b200/csrc/Makefile).
 */
#include "mex.h"

#include "ctrecon.h"

#include <cstdio>
#include <cstdlib>
#include <string>

static ctrecon_ctx* g_ctx = nullptr;

static ctrecon_ctx* context() {
    if (!g_ctx) {
        const char* dev = std::getenv("CTRECON_DEVICE");
        ctrecon_status s = ctrecon_ctx_create(dev ? std::atoi(dev) : 0, &g_ctx);
        if (s != CTRECON_OK) {
            static char msg[512];
            std::snprintf(msg, sizeof msg, "KatsevichFiltering_GPU: %s", ctrecon_last_error(nullptr));
            g_ctx = nullptr;
            mexErrMsgTxt(msg);
        }
        const char* h = std::getenv("CTRECON_HILBERT");
        if (h) ctrecon_set_option(g_ctx, CTRECON_OPT_HILBERT, std::atoi(h));
    }
    return g_ctx;
}

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    (void)nlhs;
    (void)plhs;
    if (nrhs != 14) mexErrMsgTxt("KatsevichFiltering_GPU requires 14 input arguments.");
    for (int i = 0; i < 14; ++i)
        if (!mxIsDouble(prhs[i]) || mxGetNumberOfElements(prhs[i]) < 1)
            mexErrMsgTxt("KatsevichFiltering_GPU: all arguments must be non-empty double arrays.");
    ctrecon_filter_params p;
    p.proj_scale = (double)(int)mxGetPr(prhs[1])[0];  // passed to an int parameter (:860)
    p.dec_width = mxGetPr(prhs[2])[0];
    p.dec_height = mxGetPr(prhs[3])[0];
    p.scan_r = mxGetPr(prhs[4])[0];
    p.std_dis = mxGetPr(prhs[5])[0];
    p.helic_p = mxGetPr(prhs[6])[0];
    p.filter_coeff = mxGetPr(prhs[7])[0];
    p.delta_angle = mxGetPr(prhs[8])[0];
    p.filtering_mode = (int)mxGetPr(prhs[9])[0];
    p.yl = (int)mxGetPr(prhs[10])[0];
    p.zl = (int)mxGetPr(prhs[11])[0];
    p.proj_number = (int)mxGetPr(prhs[12])[0];
    const size_t n = (size_t)(p.yl > 0 ? p.yl : 0) * (size_t)(p.zl > 0 ? p.zl : 0) *
                     (size_t)(p.proj_number > 0 ? p.proj_number : 0);
    if (n == 0 || mxGetNumberOfElements(prhs[0]) < n || mxGetNumberOfElements(prhs[13]) < n)
        mexErrMsgTxt("KatsevichFiltering_GPU: Proj and FProj must hold YL*ZL*ProjNumber elements.");
    ctrecon_ctx* ctx = context();
    ctrecon_status s = ctrecon_filter_host_f64(ctx, &p, mxGetPr(prhs[0]), mxGetPr(prhs[13]));
    if (s != CTRECON_OK) {
        static char msg[1024];
        std::snprintf(msg, sizeof msg, "KatsevichFiltering_GPU: %s (%s)", ctrecon_last_error(ctx),
                      ctrecon_status_string(s));
        mexErrMsgTxt(msg);
    }
}
