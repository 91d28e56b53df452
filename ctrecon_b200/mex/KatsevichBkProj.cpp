/*
 * KatsevichBkProj / KatsevichBkProj_GPU -- MEX entry point with the reference's call contract
 * (KatsevichBkProj.cpp:314-352, KatsevichBkProj_GPU.cu:332-429; callers
 * FunctionKat_v6.m:113, katsevichReconForGUI.m:107-109):
 *
 *   KatsevichBkProj(geom, FProj, RecMatrix)
 *
 * geom is the struct built at FunctionKat_v6.m:110-112 (fields read by position: Locus,
 * Detector, Object); FProj is double YL x ZL x (ProjEndIndex-ProjBeginIndex+1); RecMatrix
 * is the double volume, written in place with the image index (x*NY + y)*NZ + z. Voxels
 * the reference's CPU backprojector leaves untouched (outside the ObjR cylinder, or with
 * no PI interval inside the scan) keep their values. The argument checks and their
 * messages are the CPU MEX's own (KatsevichBkProj.cpp:321-326, :338-342).
 *
 * The same source builds both MEX names; both run on the GPU.
 */
#include "mex.h"

#include "ctrecon.h"

#include <cstdio>
#include <cstdlib>

static ctrecon_ctx* g_ctx = nullptr;

static ctrecon_ctx* context() {
    if (!g_ctx) {
        const char* dev = std::getenv("CTRECON_DEVICE");
        ctrecon_status s = ctrecon_ctx_create(dev ? std::atoi(dev) : 0, &g_ctx);
        if (s != CTRECON_OK) {
            static char msg[512];
            std::snprintf(msg, sizeof msg, "KatsevichBkProj: %s", ctrecon_last_error(nullptr));
            g_ctx = nullptr;
            mexErrMsgTxt(msg);
        }
        const char* pi = std::getenv("CTRECON_PI_SOLVER");
        if (pi) ctrecon_set_option(g_ctx, CTRECON_OPT_PI_SOLVER, std::atoi(pi));
    }
    return g_ctx;
}

static int read_field(const mxArray* s, int field, double* out, int maxn, int minn) {
    const mxArray* f = mxGetFieldByNumber(s, 0, field);
    if (!f || !mxIsDouble(f)) return -1;
    int n = (int)mxGetNumberOfElements(f);
    if (n < minn) return -1;
    if (n > maxn) n = maxn;
    const double* d = mxGetPr(f);
    for (int i = 0; i < n; ++i) out[i] = d[i];
    return n;
}

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    (void)plhs;
    if (nrhs != 3) mexErrMsgTxt("bkproj requires two input arguments.");
    if (nlhs != 0) mexErrMsgTxt("bkproj requires one output argument.");
    if (!mxIsStruct(prhs[0]) || mxGetNumberOfFields(prhs[0]) < 3)
        mexErrMsgTxt("bkproj: geom must be a struct with Locus, Detector and Object fields.");
    ctrecon_bp_geom g = {};
    if (read_field(prhs[0], 0, g.locus, 7, 7) < 0)
        mexErrMsgTxt("bkproj: geom.Locus must hold 7 doubles.");
    g.n_detector = read_field(prhs[0], 1, g.detector, 6, 4);
    if (g.n_detector < 0) mexErrMsgTxt("bkproj: geom.Detector must hold at least 4 doubles.");
    g.n_object = read_field(prhs[0], 2, g.object, 7, 4);
    if (g.n_object < 0) mexErrMsgTxt("bkproj: geom.Object must hold at least 4 doubles.");
    if (mxGetClassID(prhs[1]) == mxSINGLE_CLASS)
        mexErrMsgTxt("Single precision is not supported in this version.\n");
    if (!mxIsDouble(prhs[1]) || !mxIsDouble(prhs[2]))
        mexErrMsgTxt("bkproj: FProj and RecMatrix must be double arrays.");
    const long long P = (long long)(int)g.locus[5] - (int)g.locus[4] + 1;
    const long long nproj = P * (int)g.detector[1] * (int)g.detector[3];
    const long long nvox = (long long)(int)g.object[1] * (int)g.object[2] * (int)g.object[3];
    if (P < 1 || nproj < 1 || nvox < 1 || (long long)mxGetNumberOfElements(prhs[1]) < nproj ||
        (long long)mxGetNumberOfElements(prhs[2]) < nvox)
        mexErrMsgTxt("bkproj: FProj or RecMatrix is smaller than geom describes.");
    ctrecon_ctx* ctx = context();
    ctrecon_status s = ctrecon_bkproj_host_f64(ctx, &g, mxGetPr(prhs[1]), mxGetPr(prhs[2]));
    if (s != CTRECON_OK) {
        static char msg[1024];
        std::snprintf(msg, sizeof msg, "bkproj: %s (%s)", ctrecon_last_error(ctx),
                      ctrecon_status_string(s));
        mexErrMsgTxt(msg);
    }
}
