// api.cpp -- the C ABI of include/ctrecon.h: contexts, plan caching and the host (FP64,
// MEX-equivalent) and device (FP32) entry points.
#include "internal.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <new>
#include <vector>

namespace ctr {

DevBuf::~DevBuf() { release(); }

void DevBuf::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

Status DevBuf::ensure(size_t b, const char* what) {
    if (b <= bytes && ptr) return Status::Ok();
    release();
    if (b == 0) b = 16;
    cudaError_t e = cudaMalloc(&ptr, b);
    if (e != cudaSuccess) {
        ptr = nullptr;
        cudaGetLastError();
        return make_status(CTRECON_ERR_OUT_OF_MEMORY,
                           std::string("cudaMalloc(") + std::to_string(b) + " B) for " + what +
                               ": " + cudaGetErrorString(e));
    }
    bytes = b;
    return Status::Ok();
}

template <class T>
static Status upload(DevBuf& buf, const std::vector<T>& host, const char* what) {
    CTR_TRY(buf.ensure(host.size() * sizeof(T), what));
    CTR_CUDA(cudaMemcpy(buf.ptr, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice));
    return Status::Ok();
}

static bool same_filter_params(const ctrecon_filter_params& a, const ctrecon_filter_params& b) {
    return std::memcmp(&a, &b, sizeof a) == 0;
}

Status get_filter_plan(ctrecon_ctx* ctx, const ctrecon_filter_params& p, FilterPlan** out) {
    FilterPlan& plan = ctx->fplan;
    if (ctx->fplan_valid && same_filter_params(plan.p, p)) {
        *out = &plan;
        return Status::Ok();
    }
    ctx->fplan_valid = false;
    CTR_TRY(build_filter_plan(p, plan));
    ctx->fplan_valid = true;
    *out = &plan;
    return Status::Ok();
}

Status build_filter_plan(const ctrecon_filter_params& p, FilterPlan& plan) {
    plan.p = p;
    plan.tc_mode = -1;
    CTR_TRY(build_filter_tables(p, plan.t));
    const FilterTables& t = plan.t;
    plan.YLp = (t.YL + 63) / 64 * 64;
    const size_t ay = (size_t)t.AL * t.YL, zy = (size_t)t.ZL * t.YL;
    std::vector<FwEntry> fw(ay);
    for (size_t i = 0; i < ay; ++i) fw[i] = FwEntry{t.r0[i], t.r1[i], (float)t.wa[i], (float)t.wb[i]};
    std::vector<BkEntry> bk(zy);
    for (size_t i = 0; i < zy; ++i) bk[i] = BkEntry{t.b[i], t.e[i], (float)t.gb[i], (float)t.ge[i]};
    std::vector<float2> cuy(t.YL);
    for (int j = 0; j < t.YL; ++j) cuy[j] = make_float2((float)t.cu[j], (float)t.y[j]);
    std::vector<float> zcv(t.ZL);
    for (int k = 0; k < t.ZL; ++k) zcv[k] = (float)(t.z[k] * t.cv);
    const int HOFF = plan.YLp + 64;
    std::vector<float> hpad(2 * (size_t)HOFF, 0.f);
    for (int m = -(t.YL - 1); m <= t.YL - 1; ++m)
        if (m & 1) hpad[(size_t)(HOFF + m)] = (float)t.h[(size_t)(m + t.YL - 1)];
    CTR_TRY(upload(plan.fw, fw, "forward-rebin table"));
    CTR_TRY(upload(plan.bk, bk, "backward-rebin table"));
    CTR_TRY(upload(plan.cuy, cuy, "derivative coefficients"));
    CTR_TRY(upload(plan.zcv, zcv, "derivative coefficients"));
    CTR_TRY(upload(plan.h, hpad, "Hilbert taps"));
    plan.inv2dl = (float)(1.0 / (2 * t.DeltaL));
    return Status::Ok();
}

static bool same_geom(const BPGeom& a, const BPGeom& b) { return std::memcmp(&a, &b, sizeof a) == 0; }

Status get_bp_plan(ctrecon_ctx* ctx, const ctrecon_bp_geom& gin, BPPlan** out) {
    BPGeom g;
    std::memset(&g, 0, sizeof g);
    CTR_TRY(parse_bp_geom(gin, g));
    BPPlan& plan = ctx->bplan;
    if (ctx->bplan_valid && same_geom(plan.g, g)) {
        *out = &plan;
        return Status::Ok();
    }
    ctx->bplan_valid = false;
    CTR_TRY(build_bp_plan(g, plan));
    ctx->bplan_valid = true;
    *out = &plan;
    return Status::Ok();
}

Status build_bp_plan(const BPGeom& g, BPPlan& plan) {
    plan.g = g;
    plan.kp = make_bp_params(g);
    const double PI = kRefPi;
    std::vector<float4> views(g.ProjNum);
    for (int k = 0; k < g.ProjNum; ++k) {  // KatsevichBkProj.cpp:130-140, FP64 then rounded
        double temp = (k + g.ProjBegin - g.ProjCtr) * g.DeltaL;
        views[k] = make_float4((float)std::cos(temp), (float)std::sin(temp),
                               (float)(g.HelicP * temp / (2 * PI)), 0.f);
    }
    std::vector<float> xyz((size_t)g.NX + g.NY + g.NZ);
    for (int i = 0; i < g.NX; ++i) xyz[i] = (float)((i - g.XC) * g.dx);
    for (int i = 0; i < g.NY; ++i) xyz[(size_t)g.NX + i] = (float)((i - g.YC) * g.dy);
    for (int i = 0; i < g.NZ; ++i) xyz[(size_t)g.NX + g.NY + i] = (float)((i - g.ZC) * g.dz);
    CTR_TRY(upload(plan.views, views, "view geometry"));
    CTR_TRY(upload(plan.xyz, xyz, "voxel coordinates"));
    return Status::Ok();
}

size_t phantom_ell_bytes(int n_ell);
void phantom_pack(const double* ell, int n_ell, void* out);

}  // namespace ctr

using namespace ctr;

static thread_local std::string g_noctx_error;

namespace ctr {
// the message ctrecon_last_error(NULL) returns, for entry points that take no context
void set_noctx_error(const std::string& m) { g_noctx_error = m; }
}  // namespace ctr

static ctrecon_status finish(ctrecon_ctx* ctx, const Status& s) {
    if (!s.ok()) {
        if (ctx) ctx->last_error = s.msg;
        else g_noctx_error = s.msg;
        if (ctx && ctx->opt_verbose) std::fprintf(stderr, "ctrecon: %s\n", s.msg.c_str());
    } else if (ctx) {
        ctx->last_error.clear();
    }
    return s.code;
}

#define API_BEGIN try {
#define API_END(ctx)                                                                 \
    }                                                                                \
    catch (const std::bad_alloc&) {                                                  \
        return finish(ctx, make_status(CTRECON_ERR_OUT_OF_MEMORY, "host allocation failed")); \
    }                                                                                \
    catch (const std::exception& ex) {                                               \
        return finish(ctx, make_status(CTRECON_ERR_INTERNAL, ex.what()));            \
    }                                                                                \
    catch (...) {                                                                    \
        return finish(ctx, make_status(CTRECON_ERR_INTERNAL, "unknown exception"));  \
    }

static Status use_device(ctrecon_ctx* ctx) {
    CTR_CUDA(cudaSetDevice(ctx->device));
    return Status::Ok();
}

// After a synchronisation: the device error word is set by a bounded wait that gave up.
static Status check_device_flag(ctrecon_ctx* ctx) {
    if (!ctx->ws_flag.ptr) return Status::Ok();
    int flag = 0;
    CTR_CUDA(cudaMemcpy(&flag, ctx->ws_flag.ptr, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag)
        return make_status(CTRECON_ERR_TIMEOUT, "a device-side wait gave up (code " +
                                                    std::to_string(flag) + ")");
    return Status::Ok();
}

extern "C" {

int ctrecon_abi_version(void) { return CTRECON_ABI_VERSION; }

const char* ctrecon_status_string(ctrecon_status s) {
    switch (s) {
    case CTRECON_OK: return "ok";
    case CTRECON_ERR_INVALID_ARGUMENT: return "invalid argument";
    case CTRECON_ERR_GEOMETRY: return "geometry outside the reference's index range";
    case CTRECON_ERR_CUDA: return "CUDA error";
    case CTRECON_ERR_OUT_OF_MEMORY: return "out of memory";
    case CTRECON_ERR_NO_DEVICE: return "no usable device";
    case CTRECON_ERR_TIMEOUT: return "device wait timed out";
    case CTRECON_ERR_UNSUPPORTED: return "unsupported";
    case CTRECON_ERR_INTERNAL: return "internal error";
    }
    return "unknown status";
}

const char* ctrecon_last_error(const ctrecon_ctx* ctx) {
    return ctx ? ctx->last_error.c_str() : g_noctx_error.c_str();
}

ctrecon_status ctrecon_ctx_create(int device, ctrecon_ctx** out) {
    API_BEGIN
    if (!out) return finish(nullptr, make_status(CTRECON_ERR_INVALID_ARGUMENT, "out is NULL"));
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        return finish(nullptr, make_status(CTRECON_ERR_NO_DEVICE,
                                           std::string("no CUDA device: ") + cudaGetErrorString(e)));
    }
    if (device < 0 || device >= n)
        return finish(nullptr, make_status(CTRECON_ERR_INVALID_ARGUMENT, "device index out of range"));
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return finish(nullptr, cuda_status(e, "cudaGetDeviceProperties"));
    if (prop.major != 10)
        return finish(nullptr, make_status(CTRECON_ERR_NO_DEVICE,
                                           "this build targets sm_100a (B200); device is sm_" +
                                               std::to_string(prop.major * 10 + prop.minor)));
    ctrecon_ctx* ctx = new ctrecon_ctx();
    ctx->device = device;
    Status s = use_device(ctx);
    if (s.ok()) {
        e = cudaStreamCreateWithFlags(&ctx->host_stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) s = cuda_status(e, "cudaStreamCreate");
    }
    if (!s.ok()) {
        delete ctx;
        return finish(nullptr, s);
    }
    *out = ctx;
    return CTRECON_OK;
    API_END(nullptr)
}

void ctrecon_ctx_destroy(ctrecon_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->host_stream) {
        cudaStreamSynchronize(ctx->host_stream);
        cudaStreamDestroy(ctx->host_stream);
    }
    delete ctx;
}

ctrecon_status ctrecon_set_option(ctrecon_ctx* ctx, ctrecon_option opt, int value) {
    if (!ctx) return CTRECON_ERR_INVALID_ARGUMENT;
    switch (opt) {
    case CTRECON_OPT_HILBERT:
        if (value < CTRECON_HILBERT_FP32 || value > CTRECON_HILBERT_TF32)
            return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT, "bad Hilbert mode"));
        ctx->opt_hilbert = value;
        break;
    case CTRECON_OPT_PI_SOLVER:
        if (value < CTRECON_PI_BISECT || value > CTRECON_PI_LEARNED)
            return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT, "bad PI solver"));
        ctx->opt_pi = value;
        break;
    case CTRECON_OPT_FILTER_CHUNK:
        if (value < 1)
            return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT, "chunk must be >= 1"));
        ctx->opt_filter_chunk = value;
        break;
    case CTRECON_OPT_BP_VARIANT: ctx->opt_bp_variant = value; break;
    case CTRECON_OPT_VERBOSE: ctx->opt_verbose = value; break;
    default: return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT, "unknown option"));
    }
    return finish(ctx, Status::Ok());
}

ctrecon_status ctrecon_get_option(const ctrecon_ctx* ctx, ctrecon_option opt, int* value) {
    if (!ctx || !value) return CTRECON_ERR_INVALID_ARGUMENT;
    switch (opt) {
    case CTRECON_OPT_HILBERT: *value = ctx->opt_hilbert; break;
    case CTRECON_OPT_PI_SOLVER: *value = ctx->opt_pi; break;
    case CTRECON_OPT_FILTER_CHUNK: *value = ctx->opt_filter_chunk; break;
    case CTRECON_OPT_BP_VARIANT: *value = ctx->opt_bp_variant; break;
    case CTRECON_OPT_VERBOSE: *value = ctx->opt_verbose; break;
    default: return CTRECON_ERR_INVALID_ARGUMENT;
    }
    return CTRECON_OK;
}

int ctrecon_num_kappa(int zl) { return 2 * (int)std::ceil(zl * 1.3 * 0.5) + 1; }

ctrecon_status ctrecon_find_tau(double ratio, double tol, double* tau) {
    if (!tau || !(ratio > 0 && ratio < 1) || !(tol > 0))
        return finish(nullptr, make_status(CTRECON_ERR_INVALID_ARGUMENT,
                                           "find_tau: need 0 < ratio < 1 and tol > 0"));
    const double pi = 3.141592653589793;  // MATLAB's pi (FindTau.m:7 uses the built-in)
    const double am = 2 * pi - 2 * std::acos(ratio);
    double tu = 0.5, td = 0, delta = 1, t = 0;
    int guard = 0;
    while (delta > tol && guard++ < 200) {  // FindTau.m:13-22
        t = (td + tu) / 2;
        const double f = t * std::cos(am) - std::cos(t * am) + 1 - t;
        delta = std::fabs(f);
        if (f > 0) tu = t;
        else td = t;
    }
    *tau = t;
    return CTRECON_OK;
}

void ctrecon_geometry_sizing(double ScanR, double StdDis, double HelicP, double ObjR, int YL,
                             int ZL, double* DecWidth, double* DecHeigh, double* delta) {
    const double PI = 3.1415926;  // FunctionKat_v6.m:49
    double U_HelicP = HelicP / ObjR;
    double U_ScanR = ScanR / ObjR;
    double U_DW = 2 * (U_ScanR / std::pow(U_ScanR * U_ScanR - 1, 0.5)) * YL / (YL - 2);
    double d = 2 * std::acos(ObjR / ScanR);
    double coef = (2 * PI - d) / (2 * PI * (1 - std::cos(d)));
    double U_DH = 2 * coef * U_HelicP * ZL / (ZL - 2);
    if (DecWidth) *DecWidth = U_DW * StdDis / U_ScanR;
    if (DecHeigh) *DecHeigh = U_DH * StdDis / U_ScanR;
    if (delta) *delta = d;
}

ctrecon_status ctrecon_filter_tables(const ctrecon_filter_params* p, int* r0, int* r1,
                                     double* wa, double* wb, int* b, int* e, double* gb,
                                     double* ge) {
    API_BEGIN
    if (!p) return finish(nullptr, make_status(CTRECON_ERR_INVALID_ARGUMENT, "params NULL"));
    FilterTables t;
    Status s = build_filter_tables(*p, t);
    if (!s.ok()) return finish(nullptr, s);
    const size_t ay = (size_t)t.AL * t.YL, zy = (size_t)t.ZL * t.YL;
    if (r0) std::memcpy(r0, t.r0.data(), ay * sizeof(int));
    if (r1) std::memcpy(r1, t.r1.data(), ay * sizeof(int));
    if (wa) std::memcpy(wa, t.wa.data(), ay * sizeof(double));
    if (wb) std::memcpy(wb, t.wb.data(), ay * sizeof(double));
    if (b) std::memcpy(b, t.b.data(), zy * sizeof(int));
    if (e) std::memcpy(e, t.e.data(), zy * sizeof(int));
    if (gb) std::memcpy(gb, t.gb.data(), zy * sizeof(double));
    if (ge) std::memcpy(ge, t.ge.data(), zy * sizeof(double));
    return CTRECON_OK;
    API_END(nullptr)
}

ctrecon_status ctrecon_pi_table_bytes(const ctrecon_bp_geom* g, size_t* bytes) {
    API_BEGIN
    if (!g || !bytes) return finish(nullptr, make_status(CTRECON_ERR_INVALID_ARGUMENT, "NULL"));
    BPGeom bg;
    Status s = parse_bp_geom(*g, bg);
    if (!s.ok()) return finish(nullptr, s);
    *bytes = (size_t)bg.NX * bg.NY * bg.NZ * sizeof(PiRecord);
    return CTRECON_OK;
    API_END(nullptr)
}

// ---- device entry points --------------------------------------------------------------------
ctrecon_status ctrecon_filter_dev_f32(ctrecon_ctx* ctx, void* stream,
                                      const ctrecon_filter_params* p, const float* d_proj,
                                      float* d_fproj) {
    if (!ctx) return CTRECON_ERR_INVALID_ARGUMENT;
    API_BEGIN
    if (!p || !d_proj || !d_fproj)
        return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT, "NULL argument"));
    if ((const void*)d_proj == (const void*)d_fproj)
        return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT,
                                       "device filter needs distinct input and output"));
    Status s = use_device(ctx);
    FilterPlan* plan = nullptr;
    if (s.ok()) s = get_filter_plan(ctx, *p, &plan);
    if (s.ok())
        s = launch_filter(ctx, (cudaStream_t)stream, *plan, d_proj, 0, p->proj_number, d_fproj,
                          0, 0, p->proj_number);
    return finish(ctx, s);
    API_END(ctx)
}

ctrecon_status ctrecon_pi_dev(ctrecon_ctx* ctx, void* stream, const ctrecon_bp_geom* g,
                              void* d_pitab, unsigned long long* d_updates) {
    if (!ctx) return CTRECON_ERR_INVALID_ARGUMENT;
    API_BEGIN
    if (!g || !d_pitab) return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT, "NULL argument"));
    Status s = use_device(ctx);
    BPPlan* plan = nullptr;
    if (s.ok()) s = get_bp_plan(ctx, *g, &plan);
    if (s.ok()) s = launch_pi(ctx, (cudaStream_t)stream, *plan, (PiRecord*)d_pitab, d_updates);
    return finish(ctx, s);
    API_END(ctx)
}

ctrecon_status ctrecon_bkproj_dev_f32(ctrecon_ctx* ctx, void* stream, const ctrecon_bp_geom* g,
                                      const float* d_fproj, const void* d_pitab,
                                      float* d_image) {
    if (!ctx) return CTRECON_ERR_INVALID_ARGUMENT;
    API_BEGIN
    if (!g || !d_fproj || !d_image)
        return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT, "NULL argument"));
    cudaStream_t st = (cudaStream_t)stream;
    Status s = use_device(ctx);
    BPPlan* plan = nullptr;
    if (s.ok()) s = get_bp_plan(ctx, *g, &plan);
    const PiRecord* pit = (const PiRecord*)d_pitab;
    if (s.ok() && !pit) {
        const size_t nvox = (size_t)plan->kp.NX * plan->kp.NY * plan->kp.NZ;
        s = ctx->ws_pitab.ensure(nvox * sizeof(PiRecord), "PI table");
        if (s.ok()) s = launch_pi(ctx, st, *plan, ctx->ws_pitab.as<PiRecord>(), nullptr);
        pit = ctx->ws_pitab.as<PiRecord>();
    }
    if (s.ok()) s = launch_bkproj_f32(ctx, st, *plan, d_fproj, pit, d_image);
    return finish(ctx, s);
    API_END(ctx)
}

ctrecon_status ctrecon_phantom_project_dev(ctrecon_ctx* ctx, void* stream,
                                           const ctrecon_bp_geom* g, const double* ell,
                                           int n_ell, double photons, uint64_t seed,
                                           float* d_proj) {
    if (!ctx) return CTRECON_ERR_INVALID_ARGUMENT;
    API_BEGIN
    if (!g || !d_proj || (n_ell > 0 && !ell) || n_ell < 0)
        return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT, "bad phantom arguments"));
    Status s = use_device(ctx);
    BPGeom bg;
    std::memset(&bg, 0, sizeof bg);
    if (s.ok()) s = parse_bp_geom(*g, bg);
    std::vector<unsigned char> packed(phantom_ell_bytes(n_ell));
    phantom_pack(ell, n_ell, packed.data());
    cudaStream_t st = (cudaStream_t)stream;
    if (s.ok()) s = ctx->ws_ell.ensure(packed.size() + 256, "phantom ellipsoids");
    if (s.ok()) {
        cudaError_t e = cudaMemcpyAsync(ctx->ws_ell.ptr, packed.data(), packed.size(),
                                        cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) s = cuda_status(e, "cudaMemcpyAsync");
        else {
            // the host copy must outlive the transfer
            e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) s = cuda_status(e, "cudaStreamSynchronize");
        }
    }
    if (s.ok()) {
        float* dmax = (float*)((char*)ctx->ws_ell.ptr + ((packed.size() + 127) / 128) * 128);
        s = launch_phantom(st, bg, (const double*)ctx->ws_ell.ptr, n_ell, photons, seed, d_proj,
                           dmax);
    }
    return finish(ctx, s);
    API_END(ctx)
}

ctrecon_status ctrecon_sync(ctrecon_ctx* ctx, void* stream) {
    if (!ctx) return CTRECON_ERR_INVALID_ARGUMENT;
    API_BEGIN
    Status s = use_device(ctx);
    if (s.ok()) {
        cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
        if (e != cudaSuccess) s = cuda_status(e, "cudaStreamSynchronize");
    }
    if (s.ok()) s = check_device_flag(ctx);
    return finish(ctx, s);
    API_END(ctx)
}

// ---- host (FP64, MEX-equivalent) entry points -----------------------------------------------
static Status host_filter_to_device(ctrecon_ctx* ctx, const ctrecon_filter_params& p,
                                    const double* proj, float** d_fproj_out) {
    cudaStream_t st = ctx->host_stream;
    FilterPlan* plan = nullptr;
    CTR_TRY(get_filter_plan(ctx, p, &plan));
    const size_t n = (size_t)p.proj_number * p.yl * p.zl;
    CTR_TRY(ctx->ws_a.ensure(n * sizeof(double), "FP64 staging"));
    CTR_TRY(ctx->ws_b.ensure(n * sizeof(float), "projections"));
    CTR_TRY(ctx->ws_c.ensure(n * sizeof(float), "filtered projections"));
    CTR_CUDA(cudaMemcpyAsync(ctx->ws_a.ptr, proj, n * sizeof(double), cudaMemcpyHostToDevice, st));
    CTR_TRY(launch_convert_f64_to_f32(st, ctx->ws_a.as<double>(), ctx->ws_b.as<float>(), n));
    CTR_TRY(launch_filter(ctx, st, *plan, ctx->ws_b.as<float>(), 0, p.proj_number,
                          ctx->ws_c.as<float>(), 0, 0, p.proj_number));
    *d_fproj_out = ctx->ws_c.as<float>();
    return Status::Ok();
}

static Status check_filter_bp_shapes(const ctrecon_filter_params& p, const BPGeom& g) {
    if (p.yl != g.YL || p.zl != g.ZL || p.proj_number != g.ProjNum)
        return make_status(CTRECON_ERR_INVALID_ARGUMENT,
                           "filter and backprojection geometries disagree on YL/ZL/views");
    return Status::Ok();
}

static Status host_bkproj_from_device(ctrecon_ctx* ctx, BPPlan& plan, const float* d_fproj,
                                      double* image) {
    cudaStream_t st = ctx->host_stream;
    const size_t nvox = (size_t)plan.kp.NX * plan.kp.NY * plan.kp.NZ;
    CTR_TRY(ctx->ws_pitab.ensure(nvox * sizeof(PiRecord), "PI table"));
    CTR_TRY(ctx->ws_d.ensure(nvox * sizeof(double), "FP64 image"));
    CTR_CUDA(cudaMemcpyAsync(ctx->ws_d.ptr, image, nvox * sizeof(double), cudaMemcpyHostToDevice, st));
    CTR_TRY(launch_pi(ctx, st, plan, ctx->ws_pitab.as<PiRecord>(), nullptr));
    CTR_TRY(launch_bkproj_f64out(ctx, st, plan, d_fproj, ctx->ws_pitab.as<PiRecord>(),
                                 ctx->ws_d.as<double>()));
    CTR_CUDA(cudaMemcpyAsync(image, ctx->ws_d.ptr, nvox * sizeof(double), cudaMemcpyDeviceToHost, st));
    CTR_CUDA(cudaStreamSynchronize(st));
    return check_device_flag(ctx);
}

ctrecon_status ctrecon_filter_host_f64(ctrecon_ctx* ctx, const ctrecon_filter_params* p,
                                       const double* proj, double* fproj) {
    if (!ctx) return CTRECON_ERR_INVALID_ARGUMENT;
    API_BEGIN
    if (!p || !proj || !fproj)
        return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT, "NULL argument"));
    Status s = use_device(ctx);
    float* d_f = nullptr;
    if (s.ok()) s = host_filter_to_device(ctx, *p, proj, &d_f);
    const size_t n = (size_t)p->proj_number * p->yl * p->zl;
    if (s.ok()) s = launch_convert_f32_to_f64(ctx->host_stream, d_f, ctx->ws_a.as<double>(), n);
    if (s.ok()) {
        cudaError_t e = cudaMemcpyAsync(fproj, ctx->ws_a.ptr, n * sizeof(double),
                                        cudaMemcpyDeviceToHost, ctx->host_stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->host_stream);
        if (e != cudaSuccess) s = cuda_status(e, "filter result copy");
    }
    if (s.ok()) s = check_device_flag(ctx);
    return finish(ctx, s);
    API_END(ctx)
}

ctrecon_status ctrecon_bkproj_host_f64(ctrecon_ctx* ctx, const ctrecon_bp_geom* g,
                                       const double* fproj, double* image) {
    if (!ctx) return CTRECON_ERR_INVALID_ARGUMENT;
    API_BEGIN
    if (!g || !fproj || !image)
        return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT, "NULL argument"));
    Status s = use_device(ctx);
    BPPlan* plan = nullptr;
    if (s.ok()) s = get_bp_plan(ctx, *g, &plan);
    if (s.ok()) {
        const size_t n = (size_t)plan->g.ProjNum * plan->g.YL * plan->g.ZL;
        cudaStream_t st = ctx->host_stream;
        s = ctx->ws_a.ensure(n * sizeof(double), "FP64 staging");
        if (s.ok()) s = ctx->ws_c.ensure(n * sizeof(float), "filtered projections");
        if (s.ok()) {
            cudaError_t e = cudaMemcpyAsync(ctx->ws_a.ptr, fproj, n * sizeof(double),
                                            cudaMemcpyHostToDevice, st);
            if (e != cudaSuccess) s = cuda_status(e, "FProj upload");
        }
        if (s.ok()) s = launch_convert_f64_to_f32(st, ctx->ws_a.as<double>(), ctx->ws_c.as<float>(), n);
        if (s.ok()) s = host_bkproj_from_device(ctx, *plan, ctx->ws_c.as<float>(), image);
    }
    return finish(ctx, s);
    API_END(ctx)
}

ctrecon_status ctrecon_recon_host_f64(ctrecon_ctx* ctx, const ctrecon_filter_params* p,
                                      const ctrecon_bp_geom* g, const double* proj,
                                      double* image) {
    if (!ctx) return CTRECON_ERR_INVALID_ARGUMENT;
    API_BEGIN
    if (!p || !g || !proj || !image)
        return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT, "NULL argument"));
    Status s = use_device(ctx);
    BPPlan* plan = nullptr;
    if (s.ok()) s = get_bp_plan(ctx, *g, &plan);
    if (s.ok()) s = check_filter_bp_shapes(*p, plan->g);
    float* d_f = nullptr;
    if (s.ok()) s = host_filter_to_device(ctx, *p, proj, &d_f);
    if (s.ok()) s = host_bkproj_from_device(ctx, *plan, d_f, image);
    return finish(ctx, s);
    API_END(ctx)
}

}  // extern "C"
