// k1_staged.cu -- K1 with its projection rows brought in by tensor copies: the chain-rule
// derivative of KatsevichFiltering.m:52-95 and the forward height rebin onto the kappa lines
// with the pre-weight (:131-153), the same arithmetic in the same order as k_deriv_rebin
// (filter.cu), so the kappa rows are bit-identical to that kernel's.
//
// Layout of the work: the detector is cut into strips of 32 columns. CTA b (one per SM at a
// time) takes strip b % strips and the (b / strips)-th of the equal runs of the chunk's views
// (as many runs as fill the SMs in the fewest waves, staged_runs), and walks its views in
// order. The strips of one run are neighbouring CTAs working on the same views at the same
// time (they start in the same wave), so the 128-byte lines a strip's halo columns share with
// its neighbours, and the lines of the kappa rows the strips write side by side, meet in L2:
// DRAM sees each projection line read once and each kappa-row line written whole.
//
// The derivative of view p reads views pc - 1, pc, pc + 1 (pc = p clamped to [1, P - 2]) and p
// itself, so walking the views in order, each view of the strip is copied in ONCE (rows
// 0 .. ZL - 1, the strip's 32 columns plus 4 each side for the u stencil: the copies start on
// a 16-byte boundary) into a ring of SLOTS slots, up to SLOTS - VIEWS - 2 views ahead of the
// step being computed. The forward-rebin entries (the two weights and the two derivative rows of
// each (kappa line, column)) of a thread's column and its warp's kappa lines stay in registers
// for the whole run: the only global traffic of the loop is the tensor copies in and the
// kappa-row stores out, and shared memory carries only the staged rows and the derivative.
//
// A step takes VIEWS consecutive views: wait for the views its window gains; the derivative of
// the strip's ZL x 32 samples of each view into one of two sets of VIEWS shared buffers (a warp
// per ROWS rows, a lane per column, the v stencil's rows in registers); ONE barrier; the copies
// of the views the next window frees; the AL x 32 kappa samples of each view from its buffer
// (a warp per kappa line, the entries in registers), stored de-interleaved as every Hilbert
// form reads them. The next step's derivatives write the other set, so the rebins need no
// barrier of their own; taking several views a step shares the wait, the barrier and the loop
// among them.
#include "internal.h"
#include "tc_util.cuh"

#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <string>

namespace ctr {

namespace {

constexpr int kStrip = 32;                 // detector columns per strip, one per lane
constexpr int kHalo = 4;                   // staged columns each side (16 bytes: copy alignment)
constexpr int kRowW = kStrip + 2 * kHalo;  // floats per staged row
constexpr int kThreadsK1 = 512;
constexpr int kWarpsK1 = kThreadsK1 / 32;
constexpr size_t kSmemBudget = 227 * 1024 - 128 - 128;  // less alignment slack and barriers

// The two shapes of the kernel: derivative rows a warp takes at a time (ROWS), kappa lines per
// warp with their entries in registers (LINES), views in the ring (SLOTS), views a step
// (VIEWS). Tall detectors (up to 176 kappa lines) take 8 rows and 11 lines a warp, 2 views a
// step; short ones (at most 64 rows and 96 kappa lines) 4 rows and 6 lines, so that all 16
// warps share the derivative and no warp loads entries of lines past AL, and 4 views a step,
// which their smaller staged views leave room for.
struct K1Shape {
    int rows, lines, slots, views;
};
constexpr K1Shape kTall{8, 11, 6, 2};
constexpr K1Shape kShort{4, 6, 10, 4};

struct K1sParams {
    int P, YL, ZL, AL, YLp;
    int proj_view0;       // view held at index 0 of the projection buffer (the map's view 0)
    int c0, n;            // the chunk: views [c0, c0 + n)
    int nstrips;          // strips of YLp; CTA b takes strip b % nstrips
    int ngroups;          // runs of views per strip; CTA b takes run b / nstrips
    int slot_floats;      // floats per slot (a multiple of 32: 128-byte aligned slots)
    uint32_t box_bytes;   // bytes one tensor copy writes (the full box, fill included)
    float inv2dl;
    size_t plane;         // lo-plane offset of the BF16x3 kappa rows, in elements
    const FwEntry* fw;
    const float2* cuy;
    const float* zcv;
    void* X;
    int* err;
};

__device__ __forceinline__ void tma_load_rows(uint32_t dst, const CUtensorMap* map, int x, int y,
                                              int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(tcu::smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tcu::smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// shared-memory accesses by 32-bit address. Volatile keeps them on their side of the barriers
// and the mbarrier waits; nothing else in the kernel touches the ring or the derivative buffers.
__device__ __forceinline__ float lds_f32(uint32_t a) {
    float v;
    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ void sts_f32(uint32_t a, float v) {
    asm volatile("st.shared.f32 [%0], %1;" ::"r"(a), "f"(v));
}

__host__ __device__ __forceinline__ int clamp_view(int p, int P) {
    return p < 1 ? 1 : (p > P - 2 ? P - 2 : p);
}

// one derivative sample (:52-95) in the operations and order of k_deriv_rebin:
// (Pp - Pm) * inv2dl, then + (row[jr] - row[jl]) * cu, then + (zcv[k] * cy) * (Pv[kr] - Pv[kl])
__device__ __forceinline__ float deriv_sample(float pp, float pm, float ur, float ul, float cux,
                                              float zc, float vr, float vl, float inv2dl) {
    float g = (pp - pm) * inv2dl;
    g = fmaf(ur - ul, cux, g);
    return fmaf(zc, vr - vl, g);
}

template <int MODE, int ROWS, int LINES, int SLOTS, int VIEWS>
__global__ void __launch_bounds__(kThreadsK1, 1)
k_deriv_rebin_staged(const __grid_constant__ CUtensorMap pmap, const K1sParams k) {
    // a step's window (VIEWS + 2 views) fits in the ring, so every wait has its copy issued
    static_assert(SLOTS >= VIEWS + 2, "ring too small for a step");
    extern __shared__ __align__(128) unsigned char k1dyn[];
    __shared__ __align__(8) uint64_t full[SLOTS];
    unsigned char* base = k1dyn + ((128u - (tcu::smem_u32(k1dyn) & 127u)) & 127u);
    const int ZL = k.ZL, AL = k.AL, YL = k.YL, P = k.P;
    float* ring = reinterpret_cast<float*>(base);
    float* gfb = ring + (size_t)SLOTS * k.slot_floats;  // 2 x VIEWS buffers of ZL x 32 samples
    float* zs = gfb + (size_t)2 * VIEWS * ZL * kStrip;     // zcv
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        for (int s = 0; s < SLOTS; ++s) tcu::mbar_init(&full[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < ZL; i += kThreadsK1) zs[i] = k.zcv[i];

    // this CTA's strip and run of views
    const int strip = blockIdx.x % k.nstrips;
    const int grp = blockIdx.x / k.nstrips;
    const int pfirst = k.c0 + (int)((long long)k.n * grp / k.ngroups);
    const int plast = k.c0 + (int)((long long)k.n * (grp + 1) / k.ngroups) - 1;
    const int j0 = strip * kStrip;
    const int j = j0 + lane;
    const bool real = j < YL;
    // the forward-rebin entries of this thread's column and the warp's kappa lines
    // a = warp + 16 i, for the whole run: {wa, wb, byte offsets of gf[r0][lane], gf[r1][lane]};
    // columns past YL get zero weights (zero padding)
    float4 te[LINES];
#pragma unroll
    for (int i = 0; i < LINES; ++i) {
        const int a = warp + i * kWarpsK1;
        FwEntry e{0, 0, 0.f, 0.f};
        if (a < AL && real) e = k.fw[(size_t)a * YL + j];
        te[i] = make_float4(e.wa, e.wb, __uint_as_float((uint32_t)(e.r0 * kStrip + lane) * 4u),
                            __uint_as_float((uint32_t)(e.r1 * kStrip + lane) * 4u));
    }
    __syncthreads();  // barriers initialised, zcv in place

    // views staged for the run, in order: L0 .. L1 (copy c = v - L0 fills slot c % SLOTS)
    const int L0 = clamp_view(pfirst, P) - 1, L1 = clamp_view(plast, P) + 1;
    int next = L0;  // next view to copy in (the same in every thread)
    auto issue_upto = [&](int vmax) {
        vmax = vmax < L1 ? vmax : L1;
        for (; next <= vmax; ++next) {
            if (tid == 0) {
                const int s = (next - L0) % SLOTS;
                mbar_arrive_expect_tx(&full[s], k.box_bytes);
                tma_load_rows(tcu::smem_u32(ring + (size_t)s * k.slot_floats), &pmap, j0 - kHalo,
                              0, next - k.proj_view0, &full[s]);
            }
        }
    };
    issue_upto(L0 + SLOTS - 1);  // fill the ring

    const float2 cy = real ? __ldg(k.cuy + j) : make_float2(0.f, 0.f);
    // u stencil with the reference's edge rule (:63-78), as offsets into a staged row; columns
    // past YL read their own column (their samples are replaced by zero)
    int jl = j - 1, jr = j + 1;
    if (j < 2) { jl = 0; jr = 2; }
    else if (j > YL - 3) { jl = YL - 3; jr = YL - 1; }
    const int oc = lane + kHalo;
    const int ol = real ? jl - j0 + kHalo : oc, orr = real ? jr - j0 + kHalo : oc;
    // the first block of rows of this warp: its (zcv[k] * cy) factors for the whole run
    const int kb = warp * ROWS;
    float zcy[ROWS];
#pragma unroll
    for (int i = 0; i < ROWS; ++i) zcy[i] = kb + i < ZL ? zs[kb + i] * cy.y : 0.f;
    // kappa lines of this warp, and the 32-bit shared addresses the loop works with
    const int nl = AL > warp ? (AL - warp + kWarpsK1 - 1) / kWarpsK1 : 0;
    const size_t jx = (size_t)((j & 1) * (k.YLp >> 1) + (j >> 1));
    const size_t ostep = (size_t)kWarpsK1 * k.YLp;
    const uint32_t ring_s = tcu::smem_u32(ring);
    const uint32_t slot_b = (uint32_t)k.slot_floats * 4u;
    const uint32_t gf_s = tcu::smem_u32(gfb);
    const uint32_t gf_b = (uint32_t)(ZL * kStrip) * 4u;  // bytes per derivative buffer
    constexpr uint32_t kRowB = kRowW * 4;                  // bytes per staged row

    // the derivative of view q (:52-95) into the buffer at gcur
    auto derive = [&](int q, uint32_t gcur) {
        const int qc = clamp_view(q, P);
        const uint32_t Tm = ring_s + (uint32_t)((qc - 1 - L0) % SLOTS) * slot_b;
        const uint32_t Tp = ring_s + (uint32_t)((qc + 1 - L0) % SLOTS) * slot_b;
        const uint32_t Tv = ring_s + (uint32_t)((q - L0) % SLOTS) * slot_b;
        const uint32_t tv = Tv + (uint32_t)oc * 4u, tp = Tp + (uint32_t)oc * 4u;
        const uint32_t tm = Tm + (uint32_t)oc * 4u;
        const uint32_t tl = Tv + (uint32_t)ol * 4u, tq = Tv + (uint32_t)orr * 4u;
        const uint32_t gw = gcur + (uint32_t)lane * 4u;
        for (int k0 = kb; k0 < ZL; k0 += kWarpsK1 * ROWS) {
            if (k0 == kb && k0 >= 1 && k0 + ROWS + 1 <= ZL) {
                // no edge row: the v stencil is rows k - 1, k + 1; each half block loads all
                // its operands before it computes
#pragma unroll
                for (int h = 0; h < ROWS; h += 4) {
                    const uint32_t r0 = (uint32_t)(k0 + h) * kRowB;
                    float w[6], fp[4], fm[4], fl[4], fq[4];
#pragma unroll
                    for (int i = 0; i < 6; ++i) w[i] = lds_f32(tv + r0 - kRowB + i * kRowB);
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        fp[i] = lds_f32(tp + r0 + i * kRowB);
                        fm[i] = lds_f32(tm + r0 + i * kRowB);
                        fq[i] = lds_f32(tq + r0 + i * kRowB);
                        fl[i] = lds_f32(tl + r0 + i * kRowB);
                    }
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const float g = deriv_sample(fp[i], fm[i], fq[i], fl[i], cy.x, zcy[h + i],
                                                     w[i + 2], w[i], k.inv2dl);
                        sts_f32(gw + (uint32_t)((k0 + h + i) * kStrip) * 4u, real ? g : 0.f);
                    }
                }
            } else {
                // the first or the last row (edge rule, :85-95), rows past 128, or past ZL
                for (int i = 0; i < ROWS; ++i) {
                    const int kk = k0 + i;
                    if (kk >= ZL) break;
                    int kl = kk - 1, kr = kk + 1;
                    if (kk < 2) { kl = 0; kr = 2; }
                    else if (kk > ZL - 3) { kl = ZL - 3; kr = ZL - 1; }
                    const uint32_t r = (uint32_t)kk * kRowB;
                    const float g = deriv_sample(lds_f32(tp + r), lds_f32(tm + r), lds_f32(tq + r),
                                                 lds_f32(tl + r), cy.x, zs[kk] * cy.y,
                                                 lds_f32(tv + (uint32_t)kr * kRowB),
                                                 lds_f32(tv + (uint32_t)kl * kRowB), k.inv2dl);
                    sts_f32(gw + (uint32_t)(kk * kStrip) * 4u, real ? g : 0.f);
                }
            }
        }
    };
    // the forward rebin + pre-weight (:131-153) of view q from the buffer at gcur into the
    // chunk's kappa rows: every line's two derivative samples loaded first (lines past AL read
    // row 0 with zero weights), then the sums, then the stores
    auto rebin = [&](int q, uint32_t gcur) {
        float v[LINES];
        {
            float g0[LINES], g1[LINES];
#pragma unroll
            for (int i = 0; i < LINES; ++i) {
                g0[i] = lds_f32(gcur + __float_as_uint(te[i].z));
                g1[i] = lds_f32(gcur + __float_as_uint(te[i].w));
            }
#pragma unroll
            for (int i = 0; i < LINES; ++i) v[i] = fmaf(te[i].x, g0[i], te[i].y * g1[i]);
        }
        const size_t x0 = (size_t)(q - k.c0) * AL * k.YLp + (size_t)warp * k.YLp + jx;
        if constexpr (MODE == CTRECON_HILBERT_BF16X3) {
            // lanes l and l + 2 hold neighbouring elements of a de-interleaved row: lanes with
            // bit 1 clear store the two hi values at their own element, the others the two lo
            // values at the element before theirs (4-byte aligned: YLp and the plane offset are
            // even)
            const bool hi_lane = (lane & 2) == 0;
            __nv_bfloat16* o = static_cast<__nv_bfloat16*>(k.X) + x0 + (hi_lane ? 0 : k.plane - 1);
#pragma unroll
            for (int i = 0; i < LINES; ++i, o += ostep) {
                const __nv_bfloat16 hi = __float2bfloat16_rn(v[i]);
                const __nv_bfloat16 lo = __float2bfloat16_rn(v[i] - __bfloat162float(hi));
                const uint32_t u = (uint32_t)__bfloat16_as_ushort(hi) |
                                   ((uint32_t)__bfloat16_as_ushort(lo) << 16);
                const uint32_t dn = __shfl_down_sync(0xffffffffu, u, 2);
                const uint32_t up = __shfl_up_sync(0xffffffffu, u, 2);
                const uint32_t w = hi_lane ? __byte_perm(u, dn, 0x5410) : __byte_perm(up, u, 0x7632);
                if (i < nl) *reinterpret_cast<uint32_t*>(o) = w;
            }
        } else {
            float* o = static_cast<float*>(k.X) + x0;
#pragma unroll
            for (int i = 0; i < LINES; ++i, o += ostep) {
                float r = v[i];
                if constexpr (MODE == CTRECON_HILBERT_TF32) {
                    uint32_t t;
                    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t) : "f"(v[i]));
                    r = __uint_as_float(t);
                }
                if (i < nl) *o = r;
            }
        }
    };

    // VIEWS views a step: their derivatives into one set of VIEWS buffers, one barrier, the
    // copies the next step's window frees, their rebins; the next step's derivatives write the
    // other set, so the rebins need no barrier of their own
    int waited = 0;  // copies (c = v - L0) below this are known complete
    bool good = true;
    for (int p = pfirst; p <= plast; p += VIEWS) {
        const int pe = p + VIEWS - 1 < plast ? p + VIEWS - 1 : plast;  // the step's last view
        // views clamp(p) - 1 .. clamp(pe) + 1 have landed
        bool ok = true;
        while (ok && waited <= clamp_view(pe, P) + 1 - L0) {
            ok = tcu::mbar_wait(&full[waited % SLOTS], (uint32_t)(waited / SLOTS) & 1u, k.err, 31);
            if (ok) ++waited;
        }
        const uint32_t gset = gf_s + (uint32_t)(((p - pfirst) / VIEWS) & 1) * VIEWS * gf_b;
        if (ok) {
#pragma unroll
            for (int v = 0; v < VIEWS; ++v)
                if (p + v <= pe) derive(p + v, gset + v * gf_b);
        }
        // every thread's derivatives are in place and its reads of the ring are done
        if (!__syncthreads_and(ok)) { good = false; break; }
        if (pe < plast) issue_upto(clamp_view(pe + 1, P) - 1 + SLOTS - 1);
#pragma unroll
        for (int v = 0; v < VIEWS; ++v)
            if (p + v <= pe) rebin(p + v, gset + v * gf_b);
    }
    if (!good && tid == 0) {
        // no copy may still be writing shared memory when the CTA exits: wait (bounded) for
        // the copies not known complete
        for (int c = waited; c < next - L0; ++c)
            tcu::mbar_drain(&full[c % SLOTS], (uint32_t)(c / SLOTS) & 1u);
    }
}

// the kernel's shape for a detector of ZL rows and AL kappa lines
K1Shape staged_shape(int ZL, int AL) {
    return (ZL <= kWarpsK1 * kShort.rows && AL <= kWarpsK1 * kShort.lines) ? kShort : kTall;
}

// dynamic shared memory of the staged form, or 0 when it does not apply
size_t staged_smem(int ZL, int AL, int* slot_floats) {
    if (ZL < 3 || ZL > 256 || AL < 1) return 0;
    const K1Shape sh = staged_shape(ZL, AL);
    *slot_floats = (ZL * kRowW + 31) / 32 * 32;
    if (AL > sh.lines * kWarpsK1) return 0;
    const size_t bytes = (size_t)sh.slots * *slot_floats * 4 +
                         (size_t)2 * sh.views * ZL * kStrip * 4 +
                         (size_t)ZL * 4;
    return bytes <= kSmemBudget ? bytes + 128 : 0;
}

// Runs of views per strip. One CTA fits on an SM, so strips x runs CTAs take ceil(strips x runs
// / SMs) waves, each as long as a run (its views, plus about four views' worth of start-up: the
// two halo views copied in and the first copies' latency). The count that minimises waves x
// (views per run + 4): 32 strips of 2048 views take 9 runs in two waves of 148 SMs (288 CTAs)
// rather than 4 runs in one wave of 128.
int staged_runs(int nstrips, int n, int nsm) {
    int best = 1;
    long long best_cost = -1;
    const int gmax = std::min(n, 64);
    for (int g = 1; g <= gmax; ++g) {
        const long long waves = ((long long)nstrips * g + nsm - 1) / nsm;
        const long long cost = waves * ((n + g - 1) / g + 4);
        if (best_cost < 0 || cost < best_cost) {
            best_cost = cost;
            best = g;
        }
    }
    return best;
}

int k1_sm_count() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1)
        n = 148;
    return n;
}

Status make_proj_map(CUtensorMap* m, const float* base, int YL, int ZL, int nviews) {
    auto enc = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(tensor_map_encoder());
    if (!enc) return make_status(CTRECON_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    cuuint64_t dims[3] = {(cuuint64_t)YL, (cuuint64_t)ZL, (cuuint64_t)nviews};
    cuuint64_t strides[2] = {(cuuint64_t)YL * 4, (cuuint64_t)YL * ZL * 4};
    cuuint32_t box[3] = {(cuuint32_t)kRowW, (cuuint32_t)ZL, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides,
                     box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return make_status(CTRECON_ERR_CUDA,
                           "cuTensorMapEncodeTiled failed for the projections (" +
                               std::to_string((int)r) + ")");
    return Status::Ok();
}

template <int MODE, bool TALL>
Status run_staged(const CUtensorMap& map, const K1sParams& k, int grid, size_t smem,
                  cudaStream_t s) {
    constexpr K1Shape sh = TALL ? kTall : kShort;
    auto kern = k_deriv_rebin_staged<MODE, sh.rows, sh.lines, sh.slots, sh.views>;
    CTR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<grid, kThreadsK1, smem, s>>>(map, k);
    return Status::Ok();
}

}  // namespace

// Whether the staged K1 applies: rows of whole 16-byte units (YL a multiple of 4: the copies'
// row stride), at most 256 detector rows (one box), at most 176 kappa lines (11 per warp, their
// entries in registers; 96 for the short shape), two derivative buffers and the ring in shared memory, a 16-byte
// aligned buffer.
bool k1_staged_fits(int YL, int ZL, int AL, int YLp, const void* d_proj) {
    int sf = 0;
    return YL >= 3 && (YL % 4) == 0 && (YLp % kStrip) == 0 && ((uintptr_t)d_proj & 15u) == 0 &&
           staged_smem(ZL, AL, &sf) > 0;
}

Status launch_k1_staged(ctrecon_ctx* ctx, cudaStream_t s, const float* d_proj, int proj_view0,
                        int proj_nviews, int P, int YL, int ZL, int AL, int YLp, int c0, int n,
                        const FwEntry* fw, const float2* cuy, const float* zcv, float inv2dl,
                        void* X, size_t plane, int mode) {
    if (!k1_staged_fits(YL, ZL, AL, YLp, d_proj) || P < 3 || n < 1)
        return make_status(CTRECON_ERR_INTERNAL, "staged K1: unsupported shape");
    if (!ctx->ws_flag.ptr) return make_status(CTRECON_ERR_INTERNAL, "device error word not set up");
    // every view a chunk's windows read lies in the buffer (the caller's contract for K1)
    if (clamp_view(c0, P) - 1 < proj_view0 ||
        clamp_view(c0 + n - 1, P) + 1 >= proj_view0 + proj_nviews)
        return make_status(CTRECON_ERR_INTERNAL, "staged K1: views outside the projection buffer");
    K1sParams k;
    const size_t smem = staged_smem(ZL, AL, &k.slot_floats);
    CUtensorMap map;
    CTR_TRY(make_proj_map(&map, d_proj, YL, ZL, proj_nviews));
    k.P = P; k.YL = YL; k.ZL = ZL; k.AL = AL; k.YLp = YLp;
    k.proj_view0 = proj_view0;
    k.c0 = c0; k.n = n;
    k.nstrips = YLp / kStrip;
    k.ngroups = staged_runs(k.nstrips, n, k1_sm_count());
    k.box_bytes = (uint32_t)(kRowW * ZL * 4);
    k.inv2dl = inv2dl;
    k.plane = plane;
    k.fw = fw; k.cuy = cuy; k.zcv = zcv;
    k.X = X;
    k.err = ctx->ws_flag.as<int>();
    const int grid = k.nstrips * k.ngroups;
    const bool tall = staged_shape(ZL, AL).rows == kTall.rows;
    switch (mode) {
    case CTRECON_HILBERT_BF16X3:
        if (tall) CTR_TRY((run_staged<CTRECON_HILBERT_BF16X3, true>(map, k, grid, smem, s)));
        else CTR_TRY((run_staged<CTRECON_HILBERT_BF16X3, false>(map, k, grid, smem, s)));
        break;
    case CTRECON_HILBERT_TF32:
        if (tall) CTR_TRY((run_staged<CTRECON_HILBERT_TF32, true>(map, k, grid, smem, s)));
        else CTR_TRY((run_staged<CTRECON_HILBERT_TF32, false>(map, k, grid, smem, s)));
        break;
    default:
        if (tall) CTR_TRY((run_staged<CTRECON_HILBERT_FP32, true>(map, k, grid, smem, s)));
        else CTR_TRY((run_staged<CTRECON_HILBERT_FP32, false>(map, k, grid, smem, s)));
        break;
    }
    CTR_CUDA(cudaGetLastError());
    return Status::Ok();
}

}  // namespace ctr
