// noalloc.cu -- the Katsevich filter for callers that cannot allocate GPU memory.
//
// Some hosts cannot call cudaMalloc from the place where they run the filter: a plug-in
// loaded into an application that owns every device allocation through its own pool, code
// running under a memory budget enforced by the host process, or a real-time pipeline that
// forbids allocation after start-up (cudaMalloc can synchronise the device and block). For
// them, ctrecon_filter_noalloc_dev_f32 runs the plain FP32 filter with all of its working
// memory -- the filter tables and the kappa-row scratch between the two kernels -- inside
// one file-scope device array of fixed size, loaded with the library (every GPU that loads
// the library holds it until the process exits). It calls no cudaMalloc, no cudaFree and no
// allocating library routine; only the caller's projection buffers and this array are used.
#include "internal.h"

#include <cstring>
#include <mutex>
#include <vector>

namespace ctr {

Status launch_filter_fp32_preplaced(cudaStream_t s, const FilterTables& t, int YLp,
                                    const FwEntry* fw, const BkEntry* bk, const float2* cuy,
                                    const float* zcv, const float* hso, float inv2dl,
                                    float* kappa, int chunk, const float* d_proj,
                                    float* d_fproj);
void set_noctx_error(const std::string& m);

// The whole working set: 16 MiB. This fits, for example, a 736 x 64 detector (tables 1.8 MB,
// then 56 views of kappa rows per pass) or 1024 x 128 (tables 4.9 MB, 16 views per pass).
constexpr size_t kNoAllocBytes = (size_t)16 << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// In host code g_noalloc_scratch names a host-side stand-in, not device memory; the device
// address is looked up once per device (with that device current) and cached here for the life
// of the process. The cache assumes that the device's primary context (the one the CUDA runtime
// uses) stays alive: after cudaDeviceReset the cached address is stale.
static std::mutex g_addr_mu;
static void* g_addr[128];

static Status scratch_address(void** out) {
    int dev = 0;
    CTR_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 128) return make_status(CTRECON_ERR_UNSUPPORTED, "device index > 127");
    std::lock_guard<std::mutex> lk(g_addr_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(no-allocation scratch)");
        if (!p) return make_status(CTRECON_ERR_CUDA, "no-allocation scratch has no device address");
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return Status::Ok();
}

static size_t align256(size_t x) { return (x + 255) / 256 * 256; }

static Status filter_noalloc(cudaStream_t s, const ctrecon_filter_params& p, const float* d_proj,
                             float* d_fproj) {
    FilterTables t;
    CTR_TRY(build_filter_tables(p, t));
    const int YL = t.YL, ZL = t.ZL, AL = t.AL;
    const int YLp = (YL + 63) / 64 * 64;
    std::vector<float> hso;
    build_simt_taps(t, YLp, hso);
    const size_t ay = (size_t)AL * YL, zy = (size_t)ZL * YL;
    // layout of the array: tables, then the kappa-row scratch
    const size_t o_fw = 0;
    const size_t o_bk = align256(o_fw + ay * sizeof(FwEntry));
    const size_t o_cuy = align256(o_bk + zy * sizeof(BkEntry));
    const size_t o_zcv = align256(o_cuy + (size_t)YL * sizeof(float2));
    const size_t o_h = align256(o_zcv + (size_t)ZL * sizeof(float));
    const size_t o_kappa = align256(o_h + hso.size() * sizeof(float));
    const size_t per_view = (size_t)AL * YLp * sizeof(float);
    if (o_kappa + per_view > kNoAllocBytes)
        return make_status(CTRECON_ERR_UNSUPPORTED,
                           "scan too large for the no-allocation filter: it needs " +
                               std::to_string(o_kappa + per_view) + " bytes (tables " +
                               std::to_string(o_kappa) + " + one view of kappa rows " +
                               std::to_string(per_view) + "), the fixed scratch holds " +
                               std::to_string(kNoAllocBytes));
    const int chunk = (int)std::min<size_t>((kNoAllocBytes - o_kappa) / per_view, (size_t)t.P);

    std::vector<unsigned char> blob(o_kappa, 0);
    FwEntry* fw = reinterpret_cast<FwEntry*>(blob.data() + o_fw);
    for (size_t i = 0; i < ay; ++i) fw[i] = FwEntry{t.r0[i], t.r1[i], (float)t.wa[i], (float)t.wb[i]};
    BkEntry* bk = reinterpret_cast<BkEntry*>(blob.data() + o_bk);
    for (size_t i = 0; i < zy; ++i) bk[i] = BkEntry{t.b[i], t.e[i], (float)t.gb[i], (float)t.ge[i]};
    float2* cuy = reinterpret_cast<float2*>(blob.data() + o_cuy);
    for (int j = 0; j < YL; ++j) cuy[j] = make_float2((float)t.cu[j], (float)t.y[j]);
    float* zcv = reinterpret_cast<float*>(blob.data() + o_zcv);
    for (int k = 0; k < ZL; ++k) zcv[k] = (float)(t.z[k] * t.cv);
    std::memcpy(blob.data() + o_h, hso.data(), hso.size() * sizeof(float));

    void* base = nullptr;
    CTR_TRY(scratch_address(&base));
    unsigned char* b = static_cast<unsigned char*>(base);
    // pageable source: the copy is staged before cudaMemcpyAsync returns, so `blob` may go
    CTR_CUDA(cudaMemcpyAsync(b, blob.data(), blob.size(), cudaMemcpyHostToDevice, s));
    return launch_filter_fp32_preplaced(
        s, t, YLp, reinterpret_cast<const FwEntry*>(b + o_fw),
        reinterpret_cast<const BkEntry*>(b + o_bk), reinterpret_cast<const float2*>(b + o_cuy),
        reinterpret_cast<const float*>(b + o_zcv), reinterpret_cast<const float*>(b + o_h),
        (float)(1.0 / (2 * t.DeltaL)), reinterpret_cast<float*>(b + o_kappa), chunk, d_proj,
        d_fproj);
}

}  // namespace ctr

extern "C" ctrecon_status ctrecon_filter_noalloc_dev_f32(void* stream,
                                                         const ctrecon_filter_params* p,
                                                         const float* d_proj, float* d_fproj) {
    using namespace ctr;
    Status s;
    try {
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        const cudaError_t ce = cudaStreamIsCapturing((cudaStream_t)stream, &cap);
        if (!p || !d_proj || !d_fproj)
            s = make_status(CTRECON_ERR_INVALID_ARGUMENT, "NULL argument");
        else if ((const void*)d_proj == (const void*)d_fproj)
            s = make_status(CTRECON_ERR_INVALID_ARGUMENT, "input and output must differ");
        else if (ce != cudaSuccess)
            s = cuda_status(ce, "cudaStreamIsCapturing");
        else if (cap != cudaStreamCaptureStatusNone)
            // every call copies its tables from a temporary host buffer; a captured copy would
            // keep reading that buffer after it is gone, so nothing is enqueued
            s = make_status(CTRECON_ERR_UNSUPPORTED,
                            "the no-allocation filter cannot be called on a stream that is "
                            "being captured");
        else
            s = filter_noalloc((cudaStream_t)stream, *p, d_proj, d_fproj);
    } catch (const std::exception& e) {
        s = make_status(CTRECON_ERR_INTERNAL, e.what());
    }
    set_noctx_error(s.ok() ? std::string() : s.msg);
    return s.code;
}
