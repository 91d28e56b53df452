// autotune.cpp -- the project's autotuner for the backprojector forms: times each candidate
// form (tile shape, view-block depth, staging ring) on the caller's data with CUDA events,
// keeps the fastest per geometry in the context's table, and saves / loads that table as
// text. The batched form is tuned in batch.cpp with the same candidates.
#include "internal.h"

#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <sstream>

namespace ctr {

// candidate forms: second form (tile shapes 8x8, 4x8, 8x4 slices x views), third form
// (blocks of 4 views), fourth form (producer-warp staging: 2, 3, 4 producer warps), fifth form
// (cell records copied from global memory: three rings)
const int kTuneCandidates[] = {2, 3, 4, 0, 7, 8, 9, 10, 11, 12};
const int kNumTuneCandidates = (int)(sizeof(kTuneCandidates) / sizeof(kTuneCandidates[0]));

std::string tune_key(const BPGeom& g) {
    char buf[512];
    std::snprintf(buf, sizeof buf,
                  "R%.6g_D%.6g_H%.6g_Ps%d_P%d_Ctr%.6g_Beg%d_det%dx%d_%.6gx%.6g_c%.6g,%.6g_"
                  "vol%dx%dx%d_%.6gx%.6gx%.6g_r%.6g",
                  g.ScanR, g.StdDis, g.HelicP, g.ProjScale, g.ProjNum, g.ProjCtr, g.ProjBegin,
                  g.YL, g.ZL, g.DecWidth, g.DecHeigh, g.HalfY, g.HalfZ, g.NX, g.NY, g.NZ, g.dx,
                  g.dy, g.dz, g.ObjR);
    return buf;
}

int bp_variant_for(const ctrecon_ctx* ctx, const BPGeom& g) {
    if (ctx->opt_bp_variant != CTRECON_BP_AUTO) return ctx->opt_bp_variant;
    auto it = ctx->tune.find(tune_key(g));
    return it == ctx->tune.end() ? kDefaultBPVariant : it->second.first;
}

}  // namespace ctr

using namespace ctr;

namespace {

ctrecon_status tfinish(ctrecon_ctx* ctx, const Status& s) {
    if (!s.ok()) ctx->last_error = s.msg;
    else ctx->last_error.clear();
    return s.code;
}

// mean device time of `reps` runs of fn on stream s, after one untimed run
template <class F>
Status time_launches(cudaStream_t s, int reps, F fn, float* ms) {
    CTR_TRY(fn());
    cudaEvent_t e0, e1;
    CTR_CUDA(cudaEventCreate(&e0));
    cudaError_t e = cudaEventCreate(&e1);
    if (e != cudaSuccess) {
        cudaEventDestroy(e0);
        return cuda_status(e, "cudaEventCreate");
    }
    Status st;
    e = cudaEventRecord(e0, s);
    for (int r = 0; st.ok() && e == cudaSuccess && r < reps; ++r) st = fn();
    if (st.ok() && e == cudaSuccess) e = cudaEventRecord(e1, s);
    if (st.ok() && e == cudaSuccess) e = cudaEventSynchronize(e1);
    float t = 0.f;
    if (st.ok() && e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st.ok() && e != cudaSuccess) st = cuda_status(e, "autotuner timing");
    *ms = t / reps;
    return st;
}

Status cuda_status_or_ok(cudaError_t e, const char* what) {
    return e == cudaSuccess ? Status::Ok() : cuda_status(e, what);
}

}  // namespace

namespace ctr {
// Status of a candidate that cannot launch for this geometry (shared memory too large): the
// candidate is skipped. Sticky device errors are not swallowed.
bool launch_does_not_fit(const Status& st) {
    if (st.ok() || st.code != CTRECON_ERR_CUDA) return false;
    return st.msg.find("cudaFuncSetAttribute") != std::string::npos ||
           st.msg.find("invalid argument") != std::string::npos ||
           st.msg.find("too many resources") != std::string::npos;
}

Status tune_candidates(ctrecon_tune_result* res, cudaStream_t s,
                       const std::function<Status(int)>& prepare,
                       const std::function<Status(int)>& run_one, int max_variant) {
    std::memset(res, 0, sizeof *res);
    res->best_variant = -1;
    res->best_ms = -1.f;
    for (int c = 0; c < kNumTuneCandidates && res->n < CTRECON_TUNE_MAX; ++c) {
        const int v = kTuneCandidates[c];
        if (v > max_variant) continue;
        float ms = -1.f;
        Status st = prepare ? prepare(v) : Status::Ok();
        if (st.ok()) st = time_launches(s, 2, [&] { return run_one(v); }, &ms);
        if (launch_does_not_fit(st)) {
            cudaGetLastError();  // clear the non-sticky launch error
            ms = -1.f;
        } else if (!st.ok()) {
            return st;
        }
        res->variants[res->n] = v;
        res->ms[res->n] = ms;
        res->n++;
        if (ms >= 0.f && (res->best_ms < 0.f || ms < res->best_ms)) {
            res->best_ms = ms;
            res->best_variant = v;
        }
    }
    if (res->best_variant < 0)
        return make_status(CTRECON_ERR_UNSUPPORTED, "no backprojector form fits this geometry");
    return Status::Ok();
}
}  // namespace ctr

extern "C" {

ctrecon_status ctrecon_tune_bkproj(ctrecon_ctx* ctx, void* stream, const ctrecon_bp_geom* g,
                                   const float* d_fproj, const void* d_pitab, float* d_image,
                                   ctrecon_tune_result* out) {
    if (!ctx) return CTRECON_ERR_INVALID_ARGUMENT;
    if (!g || !d_fproj || !d_image || !out)
        return tfinish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT, "NULL argument"));
    try {
        cudaStream_t s = (cudaStream_t)stream;
        const cudaError_t e0 = cudaSetDevice(ctx->device);
        Status st = e0 == cudaSuccess ? Status::Ok() : cuda_status(e0, "cudaSetDevice");
        if (st.ok()) st = check_pitab_alignment(d_pitab);
        BPPlan* plan = nullptr;
        if (st.ok()) st = get_bp_plan(ctx, *g, &plan);
        if (st.ok()) st = reset_device_flag(ctx, s);
        const PiRecord* pit = (const PiRecord*)d_pitab;
        if (st.ok() && !pit) {
            const size_t nvox = (size_t)plan->kp.NX * plan->kp.NY * plan->kp.NZ;
            st = ctx->ws_pitab.ensure(nvox * sizeof(PiRecord), "PI table");
            if (st.ok()) st = launch_pi(ctx, s, *plan, ctx->ws_pitab.as<PiRecord>(), nullptr);
            pit = ctx->ws_pitab.as<PiRecord>();
        }
        const int saved = ctx->opt_bp_variant;
        if (st.ok())
            st = tune_candidates(out, s, nullptr, [&](int v) {
                ctx->opt_bp_variant = v;
                return launch_bkproj_f32(ctx, s, *plan, d_fproj, pit, d_image);
            });
        if (st.ok()) {  // leave the winner's backprojection in the image
            ctx->opt_bp_variant = out->best_variant;
            st = launch_bkproj_f32(ctx, s, *plan, d_fproj, pit, d_image);
        }
        ctx->opt_bp_variant = saved;
        if (st.ok()) st = cuda_status_or_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize");
        if (st.ok()) {
            int flag = 0;
            cudaError_t e = cudaMemcpy(&flag, ctx->ws_flag.ptr, sizeof(int), cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) st = cuda_status(e, "device error word");
            else if (flag) st = make_status(CTRECON_ERR_TIMEOUT, "a device-side wait gave up");
        }
        if (st.ok()) ctx->tune[tune_key(plan->g)] = {out->best_variant, out->best_ms};
        return tfinish(ctx, st);
    } catch (const std::exception& e) {
        return tfinish(ctx, make_status(CTRECON_ERR_INTERNAL, e.what()));
    }
}

ctrecon_status ctrecon_tune_save(const ctrecon_ctx* ctx, const char* path) {
    if (!ctx || !path) return CTRECON_ERR_INVALID_ARGUMENT;
    std::ofstream f(path);
    if (!f) return CTRECON_ERR_INVALID_ARGUMENT;
    f << "# ctrecon backprojector tuning table: key variant ms\n";
    for (const auto& kv : ctx->tune)
        f << kv.first << ' ' << kv.second.first << ' ' << kv.second.second << '\n';
    return f ? CTRECON_OK : CTRECON_ERR_INVALID_ARGUMENT;
}

ctrecon_status ctrecon_tune_load(ctrecon_ctx* ctx, const char* path) {
    if (!ctx || !path) return CTRECON_ERR_INVALID_ARGUMENT;
    std::ifstream f(path);
    if (!f) return tfinish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT, "cannot open tuning table"));
    std::string line;
    while (std::getline(f, line)) {
        if (line.empty() || line[0] == '#') continue;
        std::istringstream is(line);
        std::string key;
        int v = 0;
        float ms = 0.f;
        if (!(is >> key >> v >> ms) || !((v >= 0 && v <= kMaxBPVariant) || v == 100))
            return tfinish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT, "bad tuning table line"));
        ctx->tune[key] = {v, ms};
    }
    return tfinish(ctx, Status::Ok());
}

}  // extern "C"
