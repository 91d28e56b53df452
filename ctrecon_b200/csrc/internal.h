// internal.h -- shared host/device definitions of ctrecon-b200 (not part of the C ABI).
#pragma once

#include "ctrecon.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace ctr {

// The reference's pi for the filter and the backprojector (KatsevichFiltering.m:32,
// KatsevichBkProj.cpp:25); geometry must use the same constant to agree with it.
constexpr double kRefPi = 3.14159265358979;

// ---- status plumbing ---------------------------------------------------------------------
struct Status {
    ctrecon_status code = CTRECON_OK;
    std::string msg;
    bool ok() const { return code == CTRECON_OK; }
    static Status Ok() { return {}; }
};
Status make_status(ctrecon_status c, const std::string& m);
Status cuda_status(cudaError_t e, const char* what);
#define CTR_CUDA(call)                                                   \
    do {                                                                 \
        cudaError_t _e = (call);                                         \
        if (_e != cudaSuccess) return ::ctr::cuda_status(_e, #call);     \
    } while (0)
#define CTR_TRY(expr)                                                    \
    do {                                                                 \
        ::ctr::Status _s = (expr);                                       \
        if (!_s.ok()) return _s;                                         \
    } while (0)

// ---- device memory owned by a context (grow-only cache) ------------------------------------
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf();
    Status ensure(size_t b, const char* what);
    void release();
    template <class T> T* as() const { return static_cast<T*>(ptr); }
};
// Page-locked host memory of the library (cudaHostAlloc), kept for reuse like a DevBuf.
struct PinnedBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    PinnedBuf() = default;
    PinnedBuf(const PinnedBuf&) = delete;
    PinnedBuf& operator=(const PinnedBuf&) = delete;
    ~PinnedBuf();
    Status ensure(size_t b, const char* what);
    void release();
    template <class T> T* as() const { return static_cast<T*>(ptr); }
};
// Number of device allocations made by DevBuf::ensure so far (process-wide); a captured CUDA
// graph that baked in work-buffer pointers is stale once this has moved.
unsigned long long devbuf_epoch();
// Copies host -> device and waits for the device: a synchronous cudaMemcpy from pageable
// memory may return before its DMA lands, and the kernels reading the buffer run on other
// (non-blocking) streams.
Status upload_now(void* dst, const void* src, size_t bytes);
constexpr size_t kPlanCacheSize = 32;

// ---- filter tables -----------------------------------------------------------------------
// forward rebin entry per (kappa row a, column y): X = wa*GF[r0] + wb*GF[r1]
struct alignas(16) FwEntry { int r0, r1; float wa, wb; };
// backward rebin entry per (row z, column y): FProj = gb*H[b] + ge*H[e], H the unsigned
// Hilbert sum (the sign and the post-weight 1/coef are folded into gb/ge)
struct alignas(16) BkEntry { int b, e; float gb, ge; };

struct FilterTables {
    int YL = 0, ZL = 0, AL = 0, QQ = 0, P = 0;
    double DeltaL = 0, DeltaU = 0, DeltaV = 0;
    std::vector<double> y, z, AZCor, coef, Rato;
    std::vector<int> r0, r1, b, e;          // forward [AL*YL], backward [ZL*YL]
    std::vector<double> wa, wb, gb, ge;     // FP64 weights
    std::vector<double> cu;                 // u-derivative coefficient per column
    double cv = 0;                          // v-derivative coefficient 1/(2 dV D)
    std::vector<double> h;                  // Hilbert taps h[m + YL - 1]
    // DerMode 0 derivative (KatsevichFiltering_T.m:50-94), for the source rotated by -dL/2
    // (index 0, applied to the next view) and +dL/2 (index 1): per column the clamped 0-based
    // columns YD, YU and fraction alfa of the resampled position, and its row scale Dzc (the
    // row position is (k + 1 - HalfZ) * Dzc + HalfZ, one-based)
    std::vector<int> dres_yd[2], dres_yu[2];  // [YL]
    std::vector<double> dres_alfa[2], dres_dzc[2];
};
// Builds the tables of KatsevichFiltering.m:40-153 and :191-287 on the host in FP64.
Status build_filter_tables(const ctrecon_filter_params& p, FilterTables& t);

// DerMode 0 resampling of one column (one side): columns, fraction, row scale
struct alignas(16) DresCol { int yd, yu; float alfa, dzc; };

// Device form of the tables for one parameter set.
struct FilterPlan {
    ctrecon_filter_params p{};
    FilterTables t;
    int YLp = 0;  // padded row length of the kappa-row buffers (multiple of 128)
    DevBuf fw, bk, cuy, zcv, h;
    float inv2dl = 0;
    // tensor-core Hilbert operands (Toeplitz hi/lo in BF16, or TF32), built on first use: the
    // full Toeplitz with its columns in the kappa rows' de-interleaved order (single-pass form,
    // hilbert_tc.cu), and the two parity halves with the backward-rebin table by parity
    // (parity-split form, hilbert_tc2.cu)
    DevBuf tcT0, tcT1;
    int tc_mode = -1;
    DevBuf tc2T0, tc2T1, bkp;
    int tc2_mode = -1;
    bool bkp_ready = false;
    // DerMode 0 resampling (DresCol per column and side, [column][side]), built on first use
    DevBuf dres;
    bool dres_ready = false;
};

// ---- backprojection geometry ----------------------------------------------------------------
struct BPGeom {
    // reference quantities (KatsevichBkProj.cpp:80-147)
    double ScanR, StdDis, HelicP, ProjCtr, ObjR, DecWidth, DecHeigh;
    int ProjScale, ProjBegin, ProjNum, YL, ZL, NX, NY, NZ;
    double DeltaL, DeltaU, DeltaV, HalfY, HalfZ, dx, dy, dz, XC, YC, ZC;
};
Status parse_bp_geom(const ctrecon_bp_geom& g, BPGeom& out);

// Per-voxel PI-interval record (16 bytes): B = bi + bf and T = ti + tf are the fractional
// view indices of KatsevichBkProj.cpp:177-178; bi == kPiInvalid marks an unwritten voxel.
struct alignas(16) PiRecord { int bi; float bf; int ti; float tf; };
constexpr int kPiInvalid = 0x7fffffff;
// A caller's PI table is read and written as 16-byte records: it must be 16-byte aligned.
inline Status check_pitab_alignment(const void* p) {
    return ((uintptr_t)p & 15u)
               ? make_status(CTRECON_ERR_INVALID_ARGUMENT, "PI table must be 16-byte aligned")
               : Status::Ok();
}

// Kernel parameter block of the PI solve and the backprojector.
struct BPParams {
    int NX, NY, NZ, P, YL, ZL;
    double ScanR, HelicP, DeltaL, CtrMinusBeg, ObjR2;
    double XC, YC, ZC, dx, dy, dz;
    float Rf, DdU, DdV, HalfY, HalfZ, invPs, dzf;
    // view window of the backprojection: only loop views in [win0, win1] are summed; accum = 1
    // adds the window's sum to the image instead of assigning it (the full scan, assign, is the
    // default from make_bp_params)
    int win0, win1, accum;
};
BPParams make_bp_params(const BPGeom& g);

struct BPPlan {
    BPGeom g{};
    BPParams kp{};
    DevBuf views;   // float4 per view: cos, sin, source z, 0
    DevBuf xyz;     // float voxel coordinates x[NX], y[NY], z[NZ]
    int caps_cells = 0, caps_raw = 0;  // fourth-form staging capacities (bp4_caps)
    int caps_box = 0;                  // fifth form: cell records per staged view (boxes)
};
// the cell records and view count a box-map table was made for
struct BoxMapKey {
    const void* rec = nullptr;
    int RW = 0, RH = 0, nviews = 0;
    bool operator==(const BoxMapKey& o) const {
        return rec == o.rec && RW == o.RW && RH == o.RH && nviews == o.nviews;
    }
};
// Sizes the fourth form's staging capacities of a plan (once).
void bp4_caps(BPPlan& plan);
// Autotuner (autotune.cpp): the tuning-table key of a geometry, the form to use for a plan
// (the option, or the table's entry under CTRECON_BP_AUTO), and the candidate forms.
std::string tune_key(const BPGeom& g);
int bp_variant_for(const ctrecon_ctx* ctx, const BPGeom& g);
extern const int kTuneCandidates[];
extern const int kNumTuneCandidates;
// The form used when CTRECON_OPT_BP_VARIANT is CTRECON_BP_AUTO (the default) and the tuning
// table has no entry for the geometry: the fifth form with blocks of 8 views (the tuner's choice
// on every benchmark scan). Its cell records are written in view windows sized to the free
// memory, so it runs at any scan length.
constexpr int kDefaultBPVariant = 12;
// A batch's default form: the second form, since a batch holds the cell records of all of its
// fifth-form scans at once.
constexpr int kDefaultBatchVariant = 2;
// Times every candidate form: prepare(v) (untimed, may be empty) then run_one(v) three times,
// the last two timed with CUDA events on s; candidates that cannot launch are marked -1.
Status tune_candidates(ctrecon_tune_result* res, cudaStream_t s,
                       const std::function<Status(int)>& prepare,
                       const std::function<Status(int)>& run_one, int max_variant = 1000);

// Per-kernel device timing (CTRECON_OPT_KERNEL_TIMING): a KernelTimer records a pair of CUDA
// events around the launches of one kernel kind on the launching stream; ctrecon_kernel_times
// sums the pairs per kind (api.cpp). With the option off (or no context) it does nothing.
struct KernelSpan {
    int kind;
    cudaEvent_t a, b;
};
struct KernelTimer {
    KernelTimer(ctrecon_ctx* ctx, cudaStream_t s, int kind);
    ~KernelTimer() { stop(); }
    void stop();
    KernelTimer(const KernelTimer&) = delete;
    KernelTimer& operator=(const KernelTimer&) = delete;
    ctrecon_ctx* ctx;
    cudaStream_t s;
    int kind;
    cudaEvent_t a = nullptr;
};

// One scan of a batched backprojection (batch.cpp, bkproj2.cu)
struct BatchScanDev {
    BPParams kp;
    const float* fproj;
    const PiRecord* pit;
    const float4* views;
    const float* xyz;
    float* image;
    long long first_tile;
    // fifth form: the scan's box-map table (CUtensorMap[256] over its cell records) and the
    // view of its first record plane
    const void* tmaps;
    int rec_p0;
};

// The learned PI-line initialiser (pinet.cu): FP32 master parameters, Adam state, training
// data, and the BF16 inference copy.
struct PinetState {
    DevBuf theta, adam_m, adam_v, grad, data, infer, guess;
    DevBuf grid_feat, grid_out;  // CTRECON_PINET_GRID: features and outputs on the (r, psi) grid
    bool trained = false;
    double r_max = 0;
    int version = 0;        // bumped by every training run
    int infer_version = -1; // version the inference copy was made from
};

}  // namespace ctr

// ---- the context (opaque in the C ABI) -------------------------------------------------------
struct ctrecon_ctx {
    int device = 0;
    std::string last_error;
    int opt_hilbert = CTRECON_HILBERT_FP32;
    int opt_pi = CTRECON_PI_BISECT;
    int opt_filter_chunk = 2048;  // larger chunks fill the GPU better (c2: 512 -> 2048, -4 %)
    int opt_bp_variant = CTRECON_BP_AUTO;  // the tuning table's form, else kDefaultBPVariant
    int opt_verbose = 0;
    int opt_deriv = CTRECON_DERIV_CHAIN;
    int opt_bp_window = 0;
    int opt_pinet_mode = CTRECON_PINET_GRID;  // CTRECON_OPT_PINET_MODE
    int opt_kernel_timing = 0;                // CTRECON_OPT_KERNEL_TIMING
    int opt_tc_form = CTRECON_TC_PARITY_SPLIT;  // CTRECON_OPT_TC_FORM
    int opt_k1_form = CTRECON_K1_STAGED;        // CTRECON_OPT_K1_FORM
    int opt_host_threads = -1;                  // CTRECON_OPT_HOST_THREADS
    std::vector<ctr::KernelSpan> kspans;      // timed launches since the last query
    std::vector<cudaEvent_t> kev_free;        // timing events for reuse
    cudaStream_t host_stream = nullptr;  // stream for the synchronous host calls
    cudaStream_t up_stream = nullptr;    // host -> device copies of the host calls
    cudaStream_t down_stream = nullptr;  // device -> host copies of the host calls
    cudaStream_t up2_stream = nullptr;   // host -> device copies of host-converted projections
    std::vector<cudaEvent_t> events;     // reusable (timing-disabled) events of the host calls
    // plans by geometry, most recently used first; a plan is never rebuilt in place (kernels
    // still queued may read it) and evicting one synchronises the device first
    std::vector<std::unique_ptr<ctr::FilterPlan>> fplans;
    std::vector<std::unique_ptr<ctr::BPPlan>> bplans;
    ctr::DevBuf ws_kappa;    // kappa-row chunk buffer of the filter
    ctr::DevBuf ws_pitab;    // PI table when the caller does not pass one
    ctr::DevBuf ws_count;    // update counter
    ctr::DevBuf ws_a, ws_b, ws_c, ws_d;  // host-call staging (f64 in, f32, f32 out, f64 out)
    ctr::DevBuf ws_e;        // FP64 image of the host backprojection
    ctr::PinnedBuf pin_ring; // FP32 slots of the host calls' input conversion
    ctr::PinnedBuf pin_ring_down;  // FP32 slots of the results widened on the host
    ctr::DevBuf ws_panel;    // arc-to-flat rebin table
    ctr::DevBuf ws_dual;     // second filter result of FilteringMode 1
    ctr::DevBuf ws_ell;      // phantom ellipsoids
    ctr::DevBuf ws_flag;     // device error word
    ctr::DevBuf ws_rec;      // cell records of the fifth-form backprojection (one window)
    ctr::DevBuf ws_boxmaps;  // tensor maps over ws_rec (one per box shape)
    ctr::BoxMapKey boxmap_key;
    ctr::PinetState pinet;   // learned PI-line initialiser
    // autotuner: backprojector form per geometry key (tune_key), with its time
    std::map<std::string, std::pair<int, float>> tune;
};

namespace ctr {
Status get_filter_plan(ctrecon_ctx* ctx, const ctrecon_filter_params& p, FilterPlan** out);
Status get_bp_plan(ctrecon_ctx* ctx, const ctrecon_bp_geom& g, BPPlan** out);
Status build_filter_plan(const ctrecon_filter_params& p, FilterPlan& plan);
Status build_bp_plan(const BPGeom& g, BPPlan& plan);
// Clears the device error word on stream s (allocating it on first use). Every entry point
// that launches a kernel with a bounded wait calls it once before its launches, so the word
// reports the waits that gave up since the last such call.
Status reset_device_flag(ctrecon_ctx* ctx, cudaStream_t s);

// kernel launchers (filter.cu, pi.cu, bkproj.cu, phantom.cu)
// Odd-lag Hilbert taps of the FP32 filter: hso[simt_koff(YLp) + K] = h(2K + 1) for
// |2K + 1| <= YL - 1, zero beyond; 2 * simt_koff(YLp) entries (geometry.cpp).
__host__ __device__ inline int simt_koff(int YLp) { return YLp / 2 + 32; }
void build_simt_taps(const FilterTables& t, int YLp, std::vector<float>& hso);
// tensor-core Hilbert (hilbert_tc.cu: single pass; hilbert_tc2.cu: parity split, persistent).
// In the tensor-core modes the kappa rows are stored de-interleaved: column j of a row at
// (j & 1) * YLp / 2 + (j >> 1).
int hilbert_tc_views_per_tile(int AL);
bool hilbert_tc2_fits(const FilterPlan& plan);
Status launch_hilbert_tc2(ctrecon_ctx* ctx, cudaStream_t s, FilterPlan& plan, const void* X,
                          int nviews, float* d_fproj_chunk, int mode);
Status launch_filter(ctrecon_ctx* ctx, cudaStream_t s, FilterPlan& plan, const float* d_proj,
                     int proj_view0, int proj_nviews, float* d_fproj, int out_view0,
                     int view_begin, int view_end);
Status launch_pi(ctrecon_ctx* ctx, cudaStream_t s, BPPlan& plan, PiRecord* d_pitab,
                 unsigned long long* d_updates);
Status launch_bkproj_f32(ctrecon_ctx* ctx, cudaStream_t s, BPPlan& plan, const float* d_fproj,
                         const PiRecord* d_pitab, float* d_image);
Status launch_bkproj_f64out(ctrecon_ctx* ctx, cudaStream_t s, BPPlan& plan,
                            const float* d_fproj, const PiRecord* d_pitab, double* d_image);
Status launch_convert_f64_to_f32(cudaStream_t s, const double* in, float* out, size_t n);
Status launch_zero_valid_f64(cudaStream_t s, const PiRecord* d_pitab, double* d_image, size_t n);
// Fifth form (variants 10..12, bkproj2.cu): cell records of at most kRecBudget bytes of views
// at a time in `recbuf` (and no more than half of the free device memory), then the
// backprojection of those views.
constexpr size_t kRecBudget = (size_t)32 << 30;
constexpr int kMaxBPVariant = 12;
// selftest.cu: a bounded wait that nothing completes must give up within limit_ms and be
// reported (returns CTRECON_ERR_TIMEOUT when the mechanism works)
Status selftest_bounded_wait(ctrecon_ctx* ctx, cudaStream_t s, int limit_ms);
// the driver's cuTensorMapEncodeTiled (nullptr when unavailable), hilbert_tc.cu
void* tensor_map_encoder();
// K1 with its projection rows staged by tensor copies (k1_staged.cu): whether it applies to a
// shape and buffer, and its launch over views [c0, c0 + n) of a buffer holding views
// [proj_view0, proj_view0 + proj_nviews); the kappa rows are bit-identical to k_deriv_rebin's.
bool k1_staged_fits(int YL, int ZL, int AL, int YLp, const void* d_proj);
Status launch_k1_staged(ctrecon_ctx* ctx, cudaStream_t s, const float* d_proj, int proj_view0,
                        int proj_nviews, int P, int YL, int ZL, int AL, int YLp, int c0, int n,
                        const FwEntry* fw, const float2* cuy, const float* zcv, float inv2dl,
                        void* X, size_t plane, int mode);
// Fifth form building blocks (bkproj2.cu): the box-map table over cell records of `nviews`
// views (kBoxMaps CUtensorMap entries written to `out`, host memory), the records of views
// [p0, p0 + nviews) of fproj, and the capacity (records per staged view) of a plan.
constexpr int kBoxMaps = 256;
Status encode_box_maps(void* out, const void* rec, int RW, int RH, int nviews);
Status launch_cell_records(cudaStream_t s, const float* d_fproj, void* rec, int p0, int nviews,
                           int YL, int ZL);
template <typename OutT>
Status launch_bkproj_v5(int variant, cudaStream_t s, BPPlan& plan, const float* d_fproj,
                        const PiRecord* d_pitab, OutT* d_image, int* err, DevBuf& recbuf,
                        DevBuf& maps, BoxMapKey& mkey, int max_views,
                        ctrecon_ctx* tctx = nullptr);
// kinds of KernelTimer (the index into ctrecon_kernel_times' arrays)
enum KernelKind {
    kKDerivRebin = 0,   // K1 k_deriv_rebin
    kKHilbertSimt = 1,  // K2 k_hilbert_simt (FP32)
    kKHilbertTc = 2,    // K2 k_hilbert_tc (tensor cores)
    kKPiSolve = 3,      // K3 PI solve (with the learned start's network)
    kKCellRecords = 4,  // k_cell_records of the fifth form
    kKBackproject = 5,  // K4, any form
    kNumKernelKinds = 6
};
Status launch_convert_f32_to_f64(cudaStream_t s, const float* in, double* out, size_t n);
Status launch_average_into(cudaStream_t s, float* a, const float* b, size_t n);
Status launch_phantom(cudaStream_t s, const BPGeom& g, const double* d_ell, int n_ell,
                      double photons, uint64_t seed, float* d_proj, float* d_max);
}  // namespace ctr
