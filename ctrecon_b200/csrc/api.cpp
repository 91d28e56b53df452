// api.cpp -- the C ABI of include/ctrecon.h: contexts, plan caching and the host (FP64,
// MEX-equivalent) and device (FP32) entry points.
#include "internal.h"
#include "host_convert.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <condition_variable>
#include <mutex>
#include <new>
#include <thread>
#include <vector>


namespace ctr {

DevBuf::~DevBuf() { release(); }

void DevBuf::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

static std::atomic<unsigned long long> g_devbuf_epoch{0};
unsigned long long devbuf_epoch() { return g_devbuf_epoch.load(); }

Status upload_now(void* dst, const void* src, size_t bytes) {
    CTR_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
    CTR_CUDA(cudaDeviceSynchronize());
    return Status::Ok();
}

Status DevBuf::ensure(size_t b, const char* what) {
    if (b <= bytes && ptr) return Status::Ok();
    release();
    g_devbuf_epoch.fetch_add(1);
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

PinnedBuf::~PinnedBuf() { release(); }

void PinnedBuf::release() {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    bytes = 0;
}

Status PinnedBuf::ensure(size_t b, const char* what) {
    if (b <= bytes && ptr) return Status::Ok();
    release();
    if (b == 0) b = 16;
    cudaError_t e = cudaHostAlloc(&ptr, b, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        ptr = nullptr;
        cudaGetLastError();
        return make_status(CTRECON_ERR_OUT_OF_MEMORY,
                           std::string("cudaHostAlloc(") + std::to_string(b) + " B) for " + what +
                               ": " + cudaGetErrorString(e));
    }
    bytes = b;
    return Status::Ok();
}

template <class T>
static Status upload(DevBuf& buf, const std::vector<T>& host, const char* what) {
    CTR_TRY(buf.ensure(host.size() * sizeof(T), what));
    return upload_now(buf.ptr, host.data(), host.size() * sizeof(T));
}

// Most-recently-used lookup in a plan list; `make` builds a new plan on a miss. The least
// recently used plan is dropped when the list is full, after a device synchronisation (work
// already queued may still read its tables).
template <class Plan, class Match, class Make>
static Status plan_lookup(std::vector<std::unique_ptr<Plan>>& list, Match match, Make make,
                          Plan** out) {
    for (size_t i = 0; i < list.size(); ++i) {
        if (match(*list[i])) {
            std::rotate(list.begin(), list.begin() + i, list.begin() + i + 1);
            *out = list.front().get();
            return Status::Ok();
        }
    }
    std::unique_ptr<Plan> plan(new Plan());
    CTR_TRY(make(*plan));
    if (list.size() >= kPlanCacheSize) {
        CTR_CUDA(cudaDeviceSynchronize());
        list.pop_back();
    }
    list.insert(list.begin(), std::move(plan));
    *out = list.front().get();
    return Status::Ok();
}

static bool same_filter_params(const ctrecon_filter_params& a, const ctrecon_filter_params& b) {
    return std::memcmp(&a, &b, sizeof a) == 0;
}

Status get_filter_plan(ctrecon_ctx* ctx, const ctrecon_filter_params& p, FilterPlan** out) {
    return plan_lookup(
        ctx->fplans, [&](const FilterPlan& f) { return same_filter_params(f.p, p); },
        [&](FilterPlan& f) { return build_filter_plan(p, f); }, out);
}

Status build_filter_plan(const ctrecon_filter_params& p, FilterPlan& plan) {
    plan.p = p;
    plan.tc_mode = -1;
    CTR_TRY(build_filter_tables(p, plan.t));
    const FilterTables& t = plan.t;
    plan.YLp = (t.YL + 127) / 128 * 128;  // halves of 64 columns for the parity split
    const size_t ay = (size_t)t.AL * t.YL, zy = (size_t)t.ZL * t.YL;
    std::vector<FwEntry> fw(ay);
    for (size_t i = 0; i < ay; ++i) fw[i] = FwEntry{t.r0[i], t.r1[i], (float)t.wa[i], (float)t.wb[i]};
    std::vector<BkEntry> bk(zy);
    for (size_t i = 0; i < zy; ++i) bk[i] = BkEntry{t.b[i], t.e[i], (float)t.gb[i], (float)t.ge[i]};
    std::vector<float2> cuy(t.YL);
    for (int j = 0; j < t.YL; ++j) cuy[j] = make_float2((float)t.cu[j], (float)t.y[j]);
    std::vector<float> zcv(t.ZL);
    for (int k = 0; k < t.ZL; ++k) zcv[k] = (float)(t.z[k] * t.cv);
    std::vector<float> hpad;
    build_simt_taps(t, plan.YLp, hpad);
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
    return plan_lookup(
        ctx->bplans, [&](const BPPlan& b) { return same_geom(b.g, g); },
        [&](BPPlan& b) { return build_bp_plan(g, b); }, out);
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

Status ctr::reset_device_flag(ctrecon_ctx* ctx, cudaStream_t s) {
    CTR_TRY(ctx->ws_flag.ensure(256, "device error word"));
    CTR_CUDA(cudaMemsetAsync(ctx->ws_flag.ptr, 0, sizeof(int), s));
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

ctrecon_status ctrecon_selftest_bounded_wait(ctrecon_ctx* ctx, void* stream, int limit_ms) {
    if (!ctx) return CTRECON_ERR_INVALID_ARGUMENT;
    API_BEGIN
    if (limit_ms < 1 || limit_ms > 10000)
        return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT, "limit_ms must be 1..10000"));
    Status s = use_device(ctx);
    if (s.ok()) s = selftest_bounded_wait(ctx, (cudaStream_t)stream, limit_ms);
    return finish(ctx, s);
    API_END(ctx)
}

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
        for (cudaStream_t* st :
             {&ctx->host_stream, &ctx->up_stream, &ctx->down_stream, &ctx->up2_stream}) {
            e = cudaStreamCreateWithFlags(st, cudaStreamNonBlocking);
            if (e != cudaSuccess) {
                s = cuda_status(e, "cudaStreamCreate");
                break;
            }
        }
    }
    if (s.ok()) s = reset_device_flag(ctx, ctx->host_stream);
    if (s.ok()) {
        e = cudaStreamSynchronize(ctx->host_stream);
        if (e != cudaSuccess) s = cuda_status(e, "cudaStreamSynchronize");
    }
    if (!s.ok()) {
        ctrecon_ctx_destroy(ctx);
        return finish(nullptr, s);
    }
    *out = ctx;
    return CTRECON_OK;
    API_END(nullptr)
}

void ctrecon_ctx_destroy(ctrecon_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    for (cudaStream_t st : {ctx->host_stream, ctx->up_stream, ctx->down_stream, ctx->up2_stream}) {
        if (!st) continue;
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    for (cudaEvent_t e : ctx->events) cudaEventDestroy(e);
    for (const ctr::KernelSpan& k : ctx->kspans) {
        cudaEventDestroy(k.a);
        cudaEventDestroy(k.b);
    }
    for (cudaEvent_t e : ctx->kev_free) cudaEventDestroy(e);
    delete ctx;
}

namespace ctr {
// A timing event from the context's pool (created on demand); nullptr on failure.
static cudaEvent_t take_timing_event(ctrecon_ctx* ctx) {
    if (!ctx->kev_free.empty()) {
        cudaEvent_t e = ctx->kev_free.back();
        ctx->kev_free.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    return cudaEventCreate(&e) == cudaSuccess ? e : nullptr;
}

// at most this many launches are kept between two queries; later ones go untimed
constexpr size_t kMaxKernelSpans = 1 << 20;

KernelTimer::KernelTimer(ctrecon_ctx* c, cudaStream_t st, int k) : ctx(c), s(st), kind(k) {
    if (!ctx || !ctx->opt_kernel_timing || ctx->kspans.size() >= kMaxKernelSpans) {
        ctx = nullptr;
        return;
    }
    a = take_timing_event(ctx);
    if (!a || cudaEventRecord(a, s) != cudaSuccess) {
        if (a) ctx->kev_free.push_back(a);
        a = nullptr;
        ctx = nullptr;
    }
}

void KernelTimer::stop() {
    if (!ctx || !a) return;
    cudaEvent_t b = take_timing_event(ctx);
    if (b && cudaEventRecord(b, s) == cudaSuccess) {
        ctx->kspans.push_back(KernelSpan{kind, a, b});
    } else {
        ctx->kev_free.push_back(a);
        if (b) ctx->kev_free.push_back(b);
    }
    a = nullptr;
    ctx = nullptr;
}
}  // namespace ctr

ctrecon_status ctrecon_kernel_times(ctrecon_ctx* ctx, double* ms, unsigned long long* launches,
                                    int n) {
    if (!ctx || (n > 0 && (!ms || !launches)) || n < 0) return CTRECON_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < n; ++i) {
        ms[i] = 0;
        launches[i] = 0;
    }
    Status st;
    cudaSetDevice(ctx->device);
    for (const KernelSpan& k : ctx->kspans) {
        float t = 0.f;
        cudaError_t e = cudaEventSynchronize(k.b);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&t, k.a, k.b);
        if (e != cudaSuccess && st.ok()) st = cuda_status(e, "kernel timing events");
        if (e == cudaSuccess && k.kind >= 0 && k.kind < n) {
            ms[k.kind] += t;
            launches[k.kind] += 1;
        }
        ctx->kev_free.push_back(k.a);
        ctx->kev_free.push_back(k.b);
    }
    ctx->kspans.clear();
    return finish(ctx, st);
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
    case CTRECON_OPT_BP_VARIANT:
        if (!(value == CTRECON_BP_AUTO || (value >= 0 && value <= kMaxBPVariant) || value == 100))
            return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT,
                                           "backprojector variant must be -1, 0..12 or 100"));
        ctx->opt_bp_variant = value;
        break;
    case CTRECON_OPT_VERBOSE: ctx->opt_verbose = value; break;
    case CTRECON_OPT_DERIVATIVE:
        if (value != CTRECON_DERIV_DIRECT && value != CTRECON_DERIV_CHAIN)
            return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT, "bad derivative mode"));
        ctx->opt_deriv = value;
        break;
    case CTRECON_OPT_BP_WINDOW:
        if (value < 0)
            return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT, "window must be >= 0"));
        ctx->opt_bp_window = value;
        break;
    case CTRECON_OPT_PINET_MODE:
        if (value < CTRECON_PINET_VOXEL_FP32 || value > CTRECON_PINET_GRID)
            return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT, "bad network mode"));
        ctx->opt_pinet_mode = value;
        break;
    case CTRECON_OPT_KERNEL_TIMING: ctx->opt_kernel_timing = value != 0; break;
    case CTRECON_OPT_TC_FORM:
        if (value != CTRECON_TC_PARITY_SPLIT && value != CTRECON_TC_SINGLE_PASS)
            return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT, "bad tensor-core form"));
        ctx->opt_tc_form = value;
        break;
    case CTRECON_OPT_K1_FORM:
        if (value != CTRECON_K1_STAGED && value != CTRECON_K1_PER_VIEW)
            return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT, "bad K1 form"));
        ctx->opt_k1_form = value;
        break;
    case CTRECON_OPT_HOST_THREADS:
        if (value < -1 || value > 256)
            return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT,
                                           "host threads must be -1, 0 or 1..256"));
        ctx->opt_host_threads = value;
        break;
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
    case CTRECON_OPT_DERIVATIVE: *value = ctx->opt_deriv; break;
    case CTRECON_OPT_BP_WINDOW: *value = ctx->opt_bp_window; break;
    case CTRECON_OPT_PINET_MODE: *value = ctx->opt_pinet_mode; break;
    case CTRECON_OPT_KERNEL_TIMING: *value = ctx->opt_kernel_timing; break;
    case CTRECON_OPT_TC_FORM: *value = ctx->opt_tc_form; break;
    case CTRECON_OPT_K1_FORM: *value = ctx->opt_k1_form; break;
    case CTRECON_OPT_HOST_THREADS: *value = ctx->opt_host_threads; break;
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
    if (s.ok()) s = reset_device_flag(ctx, (cudaStream_t)stream);
    if (s.ok())
        s = launch_filter(ctx, (cudaStream_t)stream, *plan, d_proj, 0, p->proj_number, d_fproj,
                          0, 0, p->proj_number);
    return finish(ctx, s);
    API_END(ctx)
}

ctrecon_status ctrecon_filter_mode1_dev_f32(ctrecon_ctx* ctx, void* stream,
                                            const ctrecon_filter_params* p, const float* d_proj,
                                            float* d_fproj) {
    if (!ctx) return CTRECON_ERR_INVALID_ARGUMENT;
    API_BEGIN
    if (!p || !d_proj || !d_fproj)
        return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT, "NULL argument"));
    if ((const void*)d_proj == (const void*)d_fproj)
        return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT,
                                       "device filter needs distinct input and output"));
    cudaStream_t st = (cudaStream_t)stream;
    ctrecon_filter_params p1 = *p;
    p1.filter_coeff = 1.0 - p->filter_coeff;  // the second pass of FunctionKat_v6.m:88
    Status s = use_device(ctx);
    FilterPlan* plan0 = nullptr;
    FilterPlan* plan1 = nullptr;
    if (s.ok()) s = get_filter_plan(ctx, *p, &plan0);
    if (s.ok()) s = get_filter_plan(ctx, p1, &plan1);
    const size_t n = (size_t)p->proj_number * p->yl * p->zl;
    if (s.ok()) s = ctx->ws_dual.ensure(n * sizeof(float), "FilteringMode 1 second result");
    if (s.ok()) s = reset_device_flag(ctx, st);
    if (s.ok())
        s = launch_filter(ctx, st, *plan0, d_proj, 0, p->proj_number, d_fproj, 0, 0, p->proj_number);
    if (s.ok())
        s = launch_filter(ctx, st, *plan1, d_proj, 0, p->proj_number, ctx->ws_dual.as<float>(), 0,
                          0, p->proj_number);
    if (s.ok()) s = launch_average_into(st, d_fproj, ctx->ws_dual.as<float>(), n);
    return finish(ctx, s);
    API_END(ctx)
}

ctrecon_status ctrecon_pi_dev(ctrecon_ctx* ctx, void* stream, const ctrecon_bp_geom* g,
                              void* d_pitab, unsigned long long* d_updates) {
    if (!ctx) return CTRECON_ERR_INVALID_ARGUMENT;
    API_BEGIN
    if (!g || !d_pitab) return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT, "NULL argument"));
    Status s = check_pitab_alignment(d_pitab);
    if (s.ok()) s = use_device(ctx);
    BPPlan* plan = nullptr;
    if (s.ok()) s = get_bp_plan(ctx, *g, &plan);
    if (s.ok()) s = reset_device_flag(ctx, (cudaStream_t)stream);
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
    Status s = check_pitab_alignment(d_pitab);
    if (s.ok()) s = use_device(ctx);
    BPPlan* plan = nullptr;
    if (s.ok()) s = get_bp_plan(ctx, *g, &plan);
    const PiRecord* pit = (const PiRecord*)d_pitab;
    if (s.ok()) s = reset_device_flag(ctx, st);
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
// The host calls pipeline their transfers: projections go up in chunks of views on the up
// stream (converted to FP32 there), each chunk is filtered on the host stream as soon as it
// and its neighbour view are resident, and results go down on the down stream while later
// chunks are still being filtered; the PI solve overlaps the FProj upload. With pinned host
// buffers the copies run concurrently with the kernels (and H2D with D2H); with pageable
// buffers each copy blocks the calling thread and the call degrades to sequential order.
constexpr int kHostChunkViews = 256;

// Clears the device error word before the host call's three streams start.
static Status host_reset(ctrecon_ctx* ctx) {
    CTR_TRY(reset_device_flag(ctx, ctx->host_stream));
    CTR_CUDA(cudaStreamSynchronize(ctx->host_stream));
    return Status::Ok();
}

static Status event_at(ctrecon_ctx* ctx, size_t i, cudaEvent_t* out) {
    while (ctx->events.size() <= i) {
        cudaEvent_t e;
        CTR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ctx->events.push_back(e);
    }
    *out = ctx->events[i];
    return Status::Ok();
}

// Host-side FP64 -> FP32 conversion of the host calls' views (projections, or filtered
// projections for the backprojection). Worker threads convert slots of kSlotViews views into a
// ring of kRingSlots page-locked FP32 slots (ctx->pin_ring), each worker a fixed share of every
// slot; the calling thread copies each slot to the device as soon as every worker is done with
// it (issue_upto), and a worker reuses a slot only after the copy out of it has completed. The
// FP32 values are the round-to-nearest casts the device conversion makes, so the result is the
// same bit for bit; half the bytes cross the host link, and pageable host arrays are read by
// the threads at memory speed instead of going through the driver's staged copies.
constexpr int kSlotViews = 64;
constexpr int kRingSlots = 8;

class HostConverter {
public:
    ~HostConverter() { stop(); }

    // converts the views of the given ranges [v0, v1) (increasing) of src into d_dst
    Status start(ctrecon_ctx* ctx, const double* src, float* d_dst, size_t S,
                 const std::vector<std::pair<int, int>>& ranges, int threads, cudaStream_t up) {
        src_ = src;
        dst_ = d_dst;
        S_ = S;
        up_ = up;
        device_ = ctx->device;
        for (const auto& r : ranges)
            for (int v = r.first; v < r.second; v += kSlotViews)
                slots_.push_back({v, std::min(kSlotViews, r.second - v)});
        nslot_ = (int)slots_.size();
        const size_t slot_elems = (size_t)kSlotViews * S;
        CTR_TRY(ctx->pin_ring.ensure(kRingSlots * slot_elems * sizeof(float), "conversion ring"));
        ring_ = ctx->pin_ring.as<float>();
        for (cudaEvent_t& e : ev_) {
            if (!e) CTR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        }
        parts_.assign(nslot_, 0);
        nthreads_ = threads;
        for (int t = 0; t < threads; ++t) workers_.emplace_back([this, t] { work(t); });
        return Status::Ok();
    }

    // enqueues on the up stream the copies of every slot holding views below v (waiting for
    // their conversion)
    Status issue_upto(int v) {
        while (issued_ < nslot_ && slots_[issued_].first < v) {
            const int q = issued_;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return parts_[q] == nthreads_ || failed_; });
                if (failed_) return make_status(CTRECON_ERR_CUDA, "host conversion: " + why_);
            }
            const size_t v0 = (size_t)slots_[q].first, nv = (size_t)slots_[q].second;
            CTR_CUDA(cudaMemcpyAsync(dst_ + v0 * S_, slot(q), nv * S_ * sizeof(float),
                                     cudaMemcpyHostToDevice, up_));
            CTR_CUDA(cudaEventRecord(ev_[q % kRingSlots], up_));
            {
                std::lock_guard<std::mutex> lk(mu_);
                ++issued_;
            }
            cv_.notify_all();
        }
        return Status::Ok();
    }

    // joins the workers (abandoning what they have not converted)
    void stop() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stopping_ = true;
        }
        cv_.notify_all();
        for (std::thread& w : workers_) w.join();
        workers_.clear();
        for (cudaEvent_t& e : ev_) {
            if (e) {
                cudaEventSynchronize(e);  // no copy may still read the ring
                cudaEventDestroy(e);
            }
            e = nullptr;
        }
    }

private:
    float* slot(int q) const { return ring_ + (size_t)(q % kRingSlots) * kSlotViews * S_; }

    void work(int t) {
        cudaSetDevice(device_);
        for (int q = 0; q < nslot_; ++q) {
            if (q >= kRingSlots) {
                // the copy out of this slot (slot q - kRingSlots) has been enqueued ...
                {
                    std::unique_lock<std::mutex> lk(mu_);
                    cv_.wait(lk, [&] { return issued_ > q - kRingSlots || stopping_ || failed_; });
                    if (stopping_ || failed_) return;
                }
                // ... and has completed
                const cudaError_t e = cudaEventSynchronize(ev_[q % kRingSlots]);
                if (e != cudaSuccess) {
                    std::lock_guard<std::mutex> lk(mu_);
                    failed_ = true;
                    why_ = cudaGetErrorString(e);
                    cv_.notify_all();
                    return;
                }
            }
            const size_t v0 = (size_t)slots_[q].first, n = (size_t)slots_[q].second * S_;
            const size_t a = n * t / nthreads_, b = n * (t + 1) / nthreads_;
            const double* s = src_ + v0 * S_;
            float* d = slot(q);
            convert_stream(s + a, d + a, b - a);
            {
                std::lock_guard<std::mutex> lk(mu_);
                if (stopping_) return;
                ++parts_[q];
            }
            cv_.notify_all();
        }
    }

    const double* src_ = nullptr;
    float* dst_ = nullptr;
    float* ring_ = nullptr;
    size_t S_ = 0;
    std::vector<std::pair<int, int>> slots_;  // (first view, views) of each slot, in order
    int nslot_ = 0, nthreads_ = 0, device_ = 0;
    cudaStream_t up_ = nullptr;
    cudaEvent_t ev_[kRingSlots] = {};
    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::vector<int> parts_;  // workers done with each slot
    int issued_ = 0;          // slots whose copies are enqueued
    bool stopping_ = false, failed_ = false;
    std::string why_;
};

// The reverse of HostConverter, for results going to pageable host arrays: each slot of
// kSlotViews FP32 views comes down from the device into a ring of kRingSlots page-locked slots
// (ctx->pin_ring_down) on the down stream, and worker threads widen it to FP64 into the
// caller's array; the calling thread reuses a slot only after the workers are done with it.
// Half the bytes cross the host link, and the pageable array is written by the threads at
// memory speed instead of through the driver's staged copies.
class HostWidener {
public:
    ~HostWidener() { stop(); }

    Status start(ctrecon_ctx* ctx, const float* d_src, double* dst, size_t S, int nviews,
                 int threads, cudaStream_t down) {
        src_ = d_src;
        dst_ = dst;
        S_ = S;
        down_ = down;
        device_ = ctx->device;
        for (int v = 0; v < nviews; v += kSlotViews)
            slots_.push_back({v, std::min(kSlotViews, nviews - v)});
        nslot_ = (int)slots_.size();
        CTR_TRY(ctx->pin_ring_down.ensure((size_t)kRingSlots * kSlotViews * S * sizeof(float),
                                          "widening ring"));
        ring_ = ctx->pin_ring_down.as<float>();
        for (cudaEvent_t& e : ev_) {
            if (!e) CTR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        }
        parts_.assign(nslot_, 0);
        nthreads_ = threads;
        for (int t = 0; t < threads; ++t) workers_.emplace_back([this, t] { work(t); });
        return Status::Ok();
    }

    // enqueues on the down stream, after `ready` (recorded where views [0, v) of d_src are
    // final), the copies of every slot below view v, each once its ring slot is free again
    Status issue_upto(int v, cudaEvent_t ready) {
        bool waited = false;
        while (issued_ < nslot_ && slots_[issued_].first < v) {
            const int q = issued_;
            if (q >= kRingSlots) {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return parts_[q - kRingSlots] == nthreads_ || failed_; });
                if (failed_) return make_status(CTRECON_ERR_CUDA, "host widening: " + why_);
            }
            if (!waited) {
                CTR_CUDA(cudaStreamWaitEvent(down_, ready, 0));
                waited = true;
            }
            const size_t v0 = (size_t)slots_[q].first, nv = (size_t)slots_[q].second;
            CTR_CUDA(cudaMemcpyAsync(slot(q), src_ + v0 * S_, nv * S_ * sizeof(float),
                                     cudaMemcpyDeviceToHost, down_));
            CTR_CUDA(cudaEventRecord(ev_[q % kRingSlots], down_));
            {
                std::lock_guard<std::mutex> lk(mu_);
                ++issued_;
            }
            cv_.notify_all();
        }
        return Status::Ok();
    }

    // waits until every slot is widened into the caller's array
    Status finish() {
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] {
                return failed_ || nslot_ == 0 || parts_[nslot_ - 1] == nthreads_;
            });
            if (failed_) return make_status(CTRECON_ERR_CUDA, "host widening: " + why_);
        }
        stop();
        return Status::Ok();
    }

    // joins the workers (abandoning what they have not widened)
    void stop() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stopping_ = true;
        }
        cv_.notify_all();
        for (std::thread& w : workers_) w.join();
        workers_.clear();
        for (cudaEvent_t& e : ev_) {
            if (e) {
                cudaEventSynchronize(e);  // no copy may still write the ring
                cudaEventDestroy(e);
            }
            e = nullptr;
        }
    }

private:
    float* slot(int q) const { return ring_ + (size_t)(q % kRingSlots) * kSlotViews * S_; }

    void work(int t) {
        cudaSetDevice(device_);
        for (int q = 0; q < nslot_; ++q) {
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return issued_ > q || stopping_ || failed_; });
                if (stopping_ || failed_) return;
            }
            const cudaError_t e = cudaEventSynchronize(ev_[q % kRingSlots]);
            if (e != cudaSuccess) {
                std::lock_guard<std::mutex> lk(mu_);
                failed_ = true;
                why_ = cudaGetErrorString(e);
                cv_.notify_all();
                return;
            }
            const size_t v0 = (size_t)slots_[q].first, n = (size_t)slots_[q].second * S_;
            const size_t a = n * t / nthreads_, b = n * (t + 1) / nthreads_;
            widen_stream(slot(q) + a, dst_ + v0 * S_ + a, b - a);
            {
                std::lock_guard<std::mutex> lk(mu_);
                ++parts_[q];
            }
            cv_.notify_all();
        }
    }

    const float* src_ = nullptr;
    double* dst_ = nullptr;
    float* ring_ = nullptr;
    size_t S_ = 0;
    std::vector<std::pair<int, int>> slots_;
    int nslot_ = 0, nthreads_ = 0, device_ = 0;
    cudaStream_t down_ = nullptr;
    cudaEvent_t ev_[kRingSlots] = {};
    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::vector<int> parts_;
    int issued_ = 0;
    bool stopping_ = false, failed_ = false;
    std::string why_;
};

// Host memory the driver copies through staging buffers (not page-locked or registered).
static bool is_pageable(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return a.type == cudaMemoryTypeUnregistered;
}

static int host_threads(const ctrecon_ctx* ctx) {
    if (ctx->opt_host_threads >= 0) return ctx->opt_host_threads;
    const unsigned hw = std::thread::hardware_concurrency();
    return hw == 0 ? 4 : (int)std::min(16u, hw);
}

// Uploads proj (FP64 host) and filters it into ctx->ws_c (FP32, device); if fproj_host is not
// NULL the result also comes down into it (FP64). Returns after enqueueing, except that it
// waits for the down copies when fproj_host is given. The host stream holds the filter work.
static Status host_filter_pipeline(ctrecon_ctx* ctx, const ctrecon_filter_params& p,
                                   const double* proj, double* fproj_host) {
    FilterPlan* plan = nullptr;
    CTR_TRY(get_filter_plan(ctx, p, &plan));
    const int P = p.proj_number;
    const size_t S = (size_t)p.yl * p.zl, n = S * P;
    const int threads = host_threads(ctx);
    if (threads == 0) CTR_TRY(ctx->ws_a.ensure(n * sizeof(double), "FP64 staging"));
    CTR_TRY(ctx->ws_b.ensure(n * sizeof(float), "projections"));
    CTR_TRY(ctx->ws_c.ensure(n * sizeof(float), "filtered projections"));
    // results for a pageable array come down in FP32 and are widened by host threads
    const bool widen = fproj_host && threads > 0 && is_pageable(fproj_host);
    if (fproj_host && !widen) CTR_TRY(ctx->ws_d.ensure(n * sizeof(double), "FP64 result staging"));
    const int nch = (P + kHostChunkViews - 1) / kHostChunkViews;
    cudaStream_t up = ctx->up_stream, comp = ctx->host_stream, down = ctx->down_stream;
    HostWidener wid;
    if (widen) CTR_TRY(wid.start(ctx, ctx->ws_c.as<float>(), fproj_host, S, P, threads, down));
    // the projections go up converted to FP32 by host threads (slots on the second up stream),
    // or in FP64 on the up stream, converted on the compute stream (a conversion kernel on the
    // up stream would wait for SMs behind the filter and stall the copy engine)
    HostConverter cvt;
    if (threads > 0) {
        CTR_TRY(cvt.start(ctx, proj, ctx->ws_b.as<float>(), S, {{0, P}}, threads, ctx->up2_stream));
    } else {
        for (int c = 0; c < nch; ++c) {
            const size_t v0 = (size_t)c * kHostChunkViews, v1 = std::min<size_t>(P, v0 + kHostChunkViews);
            CTR_CUDA(cudaMemcpyAsync(ctx->ws_a.as<double>() + v0 * S, proj + v0 * S,
                                     (v1 - v0) * S * sizeof(double), cudaMemcpyHostToDevice, up));
            cudaEvent_t e = nullptr;
            CTR_TRY(event_at(ctx, c, &e));
            CTR_CUDA(cudaEventRecord(e, up));
        }
    }
    int converted = 0;  // chunks [0, converted) are in FP32 once the compute stream gets there
    for (int c = 0; c < nch; ++c) {
        const int v0 = c * kHostChunkViews, v1 = std::min(P, v0 + kHostChunkViews);
        // this chunk and the first view of the next (derivative neighbour)
        const int need = std::min(c + 1, nch - 1);
        for (; converted <= need; ++converted) {
            const size_t w0 = (size_t)converted * kHostChunkViews;
            const size_t w1 = std::min<size_t>(P, w0 + kHostChunkViews);
            cudaEvent_t e = nullptr;
            CTR_TRY(event_at(ctx, converted, &e));
            if (threads > 0) {
                CTR_TRY(cvt.issue_upto((int)w1));
                CTR_CUDA(cudaEventRecord(e, ctx->up2_stream));
            }
            CTR_CUDA(cudaStreamWaitEvent(comp, e, 0));
            if (threads == 0)
                CTR_TRY(launch_convert_f64_to_f32(comp, ctx->ws_a.as<double>() + w0 * S,
                                                  ctx->ws_b.as<float>() + w0 * S, (w1 - w0) * S));
        }
        CTR_TRY(launch_filter(ctx, comp, *plan, ctx->ws_b.as<float>(), 0, P,
                              ctx->ws_c.as<float>(), 0, v0, v1));
        if (widen) {
            cudaEvent_t done = nullptr;
            CTR_TRY(event_at(ctx, nch + c, &done));
            CTR_CUDA(cudaEventRecord(done, comp));
            CTR_TRY(wid.issue_upto(v1, done));
        } else if (fproj_host) {
            const size_t o = (size_t)v0 * S, m = (size_t)(v1 - v0) * S;
            CTR_TRY(launch_convert_f32_to_f64(comp, ctx->ws_c.as<float>() + o,
                                              ctx->ws_d.as<double>() + o, m));
            cudaEvent_t done = nullptr;
            CTR_TRY(event_at(ctx, nch + c, &done));
            CTR_CUDA(cudaEventRecord(done, comp));
            CTR_CUDA(cudaStreamWaitEvent(down, done, 0));
            CTR_CUDA(cudaMemcpyAsync(fproj_host + o, ctx->ws_d.as<double>() + o,
                                     m * sizeof(double), cudaMemcpyDeviceToHost, down));
        }
    }
    cvt.stop();
    if (widen) CTR_TRY(wid.finish());
    if (fproj_host) {
        CTR_CUDA(cudaStreamSynchronize(down));
        CTR_CUDA(cudaStreamSynchronize(comp));
    }
    return Status::Ok();
}

static Status check_filter_bp_shapes(const ctrecon_filter_params& p, const BPGeom& g) {
    if (p.yl != g.YL || p.zl != g.ZL || p.proj_number != g.ProjNum)
        return make_status(CTRECON_ERR_INVALID_ARGUMENT,
                           "filter and backprojection geometries disagree on YL/ZL/views");
    return Status::Ok();
}

ctrecon_status ctrecon_filter_host_f64(ctrecon_ctx* ctx, const ctrecon_filter_params* p,
                                       const double* proj, double* fproj) {
    if (!ctx) return CTRECON_ERR_INVALID_ARGUMENT;
    API_BEGIN
    if (!p || !proj || !fproj)
        return finish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT, "NULL argument"));
    Status s = use_device(ctx);
    if (s.ok()) s = host_reset(ctx);
    if (s.ok()) s = host_filter_pipeline(ctx, *p, proj, fproj);
    if (s.ok()) s = check_device_flag(ctx);
    return finish(ctx, s);
    API_END(ctx)
}

// KatsevichBkProj with FProj from host memory, with the transfer overlapping the work: the
// image goes up first, the PI solve runs meanwhile, the valid voxels are zeroed, then the views
// go up in windows of about 2048 and each window is backprojected (accumulating) as soon as it
// is resident; the image comes down at the end. Summing per window reorders the FP32 sums of a
// voxel (the windows' partial sums are added in FP64).
static Status host_bkproj_windowed(ctrecon_ctx* ctx, BPPlan& plan, const double* fproj,
                                   double* image) {
    cudaStream_t up = ctx->up_stream, comp = ctx->host_stream, side = ctx->down_stream;
    const int P = plan.g.ProjNum;
    const size_t S = (size_t)plan.g.YL * plan.g.ZL, n = S * P;
    const size_t nvox = (size_t)plan.kp.NX * plan.kp.NY * plan.kp.NZ;
    const int threads = host_threads(ctx);
    if (threads == 0) CTR_TRY(ctx->ws_a.ensure(n * sizeof(double), "FP64 staging"));
    CTR_TRY(ctx->ws_c.ensure(n * sizeof(float), "filtered projections"));
    CTR_TRY(ctx->ws_pitab.ensure(nvox * sizeof(PiRecord), "PI table"));
    CTR_TRY(ctx->ws_e.ensure(nvox * sizeof(double), "FP64 image"));
    cudaEvent_t pi_done = nullptr, img_up = nullptr;
    CTR_TRY(event_at(ctx, 0, &pi_done));
    CTR_TRY(event_at(ctx, 1, &img_up));
    CTR_TRY(launch_pi(ctx, side, plan, ctx->ws_pitab.as<PiRecord>(), nullptr));
    CTR_CUDA(cudaEventRecord(pi_done, side));
    CTR_CUDA(cudaMemcpyAsync(ctx->ws_e.ptr, image, nvox * sizeof(double), cudaMemcpyHostToDevice, up));
    CTR_CUDA(cudaEventRecord(img_up, up));
    // the views go up converted to FP32 by host threads (slots on the second up stream), or
    // in FP64, converted per window on the compute stream
    HostConverter cvt;
    if (threads > 0)
        CTR_TRY(cvt.start(ctx, fproj, ctx->ws_c.as<float>(), S, {{0, P}}, threads, ctx->up2_stream));
    CTR_CUDA(cudaStreamWaitEvent(comp, pi_done, 0));
    CTR_CUDA(cudaStreamWaitEvent(comp, img_up, 0));
    CTR_TRY(launch_zero_valid_f64(comp, ctx->ws_pitab.as<PiRecord>(), ctx->ws_e.as<double>(), nvox));
    // windows: whole upload chunks, about 2048 views each
    const int per_win = std::max(kHostChunkViews, (2048 / kHostChunkViews) * kHostChunkViews);
    const BPParams saved = plan.kp;
    Status st;
    int w = 0;
    for (int v0 = 0; st.ok() && v0 < P; v0 += per_win, ++w) {
        const int v1 = std::min(P, v0 + per_win);
        for (int c0 = v0; st.ok() && threads == 0 && c0 < v1; c0 += kHostChunkViews) {
            const size_t m = (size_t)(std::min(v1, c0 + kHostChunkViews) - c0) * S;
            cudaError_t e = cudaMemcpyAsync(ctx->ws_a.as<double>() + (size_t)c0 * S,
                                            fproj + (size_t)c0 * S, m * sizeof(double),
                                            cudaMemcpyHostToDevice, up);
            if (e != cudaSuccess) st = cuda_status(e, "FProj upload");
        }
        if (st.ok() && threads > 0) st = cvt.issue_upto(v1);
        cudaEvent_t ev = nullptr;
        if (st.ok()) st = event_at(ctx, 2 + (size_t)w, &ev);
        if (st.ok()) {
            cudaError_t e = cudaEventRecord(ev, threads > 0 ? ctx->up2_stream : up);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(comp, ev, 0);
            if (e != cudaSuccess) st = cuda_status(e, "window event");
        }
        // the window's conversion on the compute stream (copies only on the up stream: a
        // kernel there would wait for SMs behind the backprojection and stall the copy engine)
        if (st.ok() && threads == 0)
            st = launch_convert_f64_to_f32(comp, ctx->ws_a.as<double>() + (size_t)v0 * S,
                                           ctx->ws_c.as<float>() + (size_t)v0 * S,
                                           (size_t)(v1 - v0) * S);
        if (st.ok()) {
            plan.kp.win0 = v0;
            plan.kp.win1 = v1 - 1;
            plan.kp.accum = 1;
            st = launch_bkproj_f64out(ctx, comp, plan, ctx->ws_c.as<float>(),
                                      ctx->ws_pitab.as<PiRecord>(), ctx->ws_e.as<double>());
            plan.kp = saved;
        }
    }
    plan.kp = saved;
    cvt.stop();
    CTR_TRY(st);
    CTR_CUDA(cudaMemcpyAsync(image, ctx->ws_e.ptr, nvox * sizeof(double), cudaMemcpyDeviceToHost, comp));
    CTR_CUDA(cudaStreamSynchronize(comp));
    CTR_CUDA(cudaStreamSynchronize(side));
    CTR_CUDA(cudaStreamSynchronize(up));
    CTR_CUDA(cudaStreamSynchronize(ctx->up2_stream));
    return check_device_flag(ctx);
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
    if (s.ok()) s = host_reset(ctx);
    if (s.ok()) s = host_bkproj_windowed(ctx, *plan, fproj, image);
    return finish(ctx, s);
    API_END(ctx)
}

// The whole chain with FP64 host buffers (FunctionKat_v6.m:85-113 without the FProj round
// trip), pipelined so that the host copies hide the work: the image goes up first and the PI
// solve runs beside the uploads; the projections go up in chunks, each chunk is converted and
// filtered as soon as it and its neighbour view are resident, and each window of about 2048
// views is backprojected (accumulating into the zeroed valid voxels) as soon as its views are
// filtered, while later chunks are still on their way; the image comes down at the end.

static Status host_recon_pipeline(ctrecon_ctx* ctx, const ctrecon_filter_params& p, BPPlan& plan,
                                  const double* proj, double* image) {
    FilterPlan* fplan = nullptr;
    CTR_TRY(get_filter_plan(ctx, p, &fplan));
    cudaStream_t up = ctx->up_stream, comp = ctx->host_stream, side = ctx->down_stream;
    const int P = p.proj_number;
    const size_t S = (size_t)p.yl * p.zl, n = S * P;
    const size_t nvox = (size_t)plan.kp.NX * plan.kp.NY * plan.kp.NZ;
    const int threads = host_threads(ctx);
    const int nch = (P + kHostChunkViews - 1) / kHostChunkViews;
    // every chunk converted by the host threads, or (no threads) copied up in FP64 and
    // converted on the device. Sending a third or a quarter of the chunks up in FP64 beside the
    // host conversion measured slower (0.34 and 0.31 s against 0.27 s at 512^3): the DMA
    // reads of host memory slow the conversion more than they relieve the link.
    std::vector<char> on_host(nch, threads > 0 ? 1 : 0);
    if (threads == 0) CTR_TRY(ctx->ws_a.ensure(n * sizeof(double), "FP64 staging"));
    CTR_TRY(ctx->ws_b.ensure(n * sizeof(float), "projections"));
    CTR_TRY(ctx->ws_c.ensure(n * sizeof(float), "filtered projections"));
    CTR_TRY(ctx->ws_pitab.ensure(nvox * sizeof(PiRecord), "PI table"));
    CTR_TRY(ctx->ws_e.ensure(nvox * sizeof(double), "FP64 image"));
    cudaEvent_t pi_done = nullptr, img_up = nullptr;
    CTR_TRY(event_at(ctx, 0, &pi_done));
    CTR_TRY(event_at(ctx, 1, &img_up));
    // image first (the first window needs it) on the up stream, then the projections: FP64
    // chunks on the same stream, or the host-converted slots on the second up stream
    CTR_CUDA(cudaMemcpyAsync(ctx->ws_e.ptr, image, nvox * sizeof(double), cudaMemcpyHostToDevice, up));
    CTR_CUDA(cudaEventRecord(img_up, up));
    std::vector<std::pair<int, int>> host_views;
    for (int c = 0; c < nch; ++c) {
        const int v0 = c * kHostChunkViews, v1 = std::min(P, v0 + kHostChunkViews);
        if (on_host[c]) {
            host_views.push_back({v0, v1});
            continue;
        }
        CTR_CUDA(cudaMemcpyAsync(ctx->ws_a.as<double>() + (size_t)v0 * S, proj + (size_t)v0 * S,
                                 (size_t)(v1 - v0) * S * sizeof(double), cudaMemcpyHostToDevice, up));
        cudaEvent_t e = nullptr;
        CTR_TRY(event_at(ctx, 2 + (size_t)c, &e));
        CTR_CUDA(cudaEventRecord(e, up));
    }
    HostConverter cvt;
    if (!host_views.empty())
        CTR_TRY(cvt.start(ctx, proj, ctx->ws_b.as<float>(), S, host_views, threads, ctx->up2_stream));
    CTR_TRY(launch_pi(ctx, side, plan, ctx->ws_pitab.as<PiRecord>(), nullptr));
    CTR_CUDA(cudaEventRecord(pi_done, side));
    CTR_CUDA(cudaStreamWaitEvent(comp, pi_done, 0));
    CTR_CUDA(cudaStreamWaitEvent(comp, img_up, 0));
    CTR_TRY(launch_zero_valid_f64(comp, ctx->ws_pitab.as<PiRecord>(), ctx->ws_e.as<double>(), nvox));
    // windows of whole chunks, about 2048 views each
    const int cpw = std::max(1, 2048 / kHostChunkViews);
    const BPParams saved = plan.kp;
    Status st;
    int resident = 0;  // chunks [0, resident) are in FP32 once the host stream gets there
    for (int w0 = 0; st.ok() && w0 < nch; w0 += cpw) {
        const int w1 = std::min(nch, w0 + cpw);
        for (int c = w0; st.ok() && c < w1; ++c) {
            const int v0 = c * kHostChunkViews, v1 = std::min(P, v0 + kHostChunkViews);
            // this chunk and the first view of the next (derivative neighbour)
            const int need = std::min(c + 1, nch - 1);
            for (; st.ok() && resident <= need; ++resident) {
                const size_t x0 = (size_t)resident * kHostChunkViews;
                const size_t x1 = std::min<size_t>(P, x0 + kHostChunkViews);
                cudaEvent_t e = nullptr;
                st = event_at(ctx, 2 + (size_t)resident, &e);
                if (st.ok() && on_host[resident]) {
                    st = cvt.issue_upto((int)x1);
                    if (st.ok()) {
                        const cudaError_t ce = cudaEventRecord(e, ctx->up2_stream);
                        if (ce != cudaSuccess) st = cuda_status(ce, "chunk event");
                    }
                }
                if (st.ok()) {
                    const cudaError_t ce = cudaStreamWaitEvent(comp, e, 0);
                    if (ce != cudaSuccess) st = cuda_status(ce, "chunk event");
                }
                if (st.ok() && !on_host[resident])
                    st = launch_convert_f64_to_f32(comp, ctx->ws_a.as<double>() + x0 * S,
                                                   ctx->ws_b.as<float>() + x0 * S, (x1 - x0) * S);
            }
            if (st.ok())
                st = launch_filter(ctx, comp, *fplan, ctx->ws_b.as<float>(), 0, P,
                                   ctx->ws_c.as<float>(), 0, v0, v1);
        }
        if (st.ok()) {
            plan.kp.win0 = w0 * kHostChunkViews;
            plan.kp.win1 = std::min(P, w1 * kHostChunkViews) - 1;
            plan.kp.accum = 1;
            st = launch_bkproj_f64out(ctx, comp, plan, ctx->ws_c.as<float>(),
                                      ctx->ws_pitab.as<PiRecord>(), ctx->ws_e.as<double>());
            plan.kp = saved;
        }
    }
    plan.kp = saved;
    cvt.stop();
    CTR_TRY(st);
    CTR_CUDA(cudaMemcpyAsync(image, ctx->ws_e.ptr, nvox * sizeof(double), cudaMemcpyDeviceToHost, comp));
    CTR_CUDA(cudaStreamSynchronize(comp));
    CTR_CUDA(cudaStreamSynchronize(side));
    CTR_CUDA(cudaStreamSynchronize(up));
    CTR_CUDA(cudaStreamSynchronize(ctx->up2_stream));
    return check_device_flag(ctx);
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
    if (s.ok()) s = host_reset(ctx);
    if (s.ok()) s = host_recon_pipeline(ctx, *p, *plan, proj, image);
    return finish(ctx, s);
    API_END(ctx)
}

}  // extern "C"
