// filter.cu -- the Katsevich filter on the device (KatsevichFiltering.m:39-287).
//
// K1 k_deriv_rebin : per (view, column) the chain-rule derivative of KatsevichFiltering.m:52-95
//                    (view, u and v central differences with the reference's edge rules),
//                    kept in shared memory, then the forward height rebin onto the AL kappa
//                    lines with the pre-weight (:131-153). Writes one kappa-row chunk
//                    X[view][a][y] (rows padded to YLp, zero beyond YL).
// K2 k_hilbert_simt: the Hilbert filter as a direct Toeplitz sum over odd lags (h[m] = 0 for
//                    even m, :160-176), FP32 FMA with a register-rotated tap window, and the
//                    post-weight + backward rebin (:181-284) fused into its epilogue: the
//                    CTA holds all AL kappa rows of a 64-column tile, so every output
//                    FProj[view][z][y] = gb*H[b][y] + ge*H[e][y] is a shared-memory gather.
//                    (The tensor-core form of K2 lives in hilbert_tc.cu.)
//
// Views are processed in chunks so the kappa-row buffer stays small enough to live in L2
// between K1 and K2.
#include "internal.h"

#include <cuda_bf16.h>

#include <algorithm>
#include <vector>

namespace ctr {

// ---------------------------------------------------------------------------------------------
// K1
// ---------------------------------------------------------------------------------------------
constexpr int kRowGroups = 4;  // independent row walks per column in K1
// Output formats of the kappa rows: FP32 (SIMT Hilbert), BF16 hi and lo planes (BF16x3
// tensor-core Hilbert; the lo plane starts `plane` elements after the hi plane), or FP32
// rounded to TF32 (round to nearest) for the TF32 tensor-core Hilbert.
__device__ __forceinline__ void store_kappa(void* X, size_t idx, size_t plane, float v, int mode) {
    if (mode == CTRECON_HILBERT_BF16X3) {
        __nv_bfloat16 hi = __float2bfloat16_rn(v);
        __nv_bfloat16 lo = __float2bfloat16_rn(v - __bfloat162float(hi));
        static_cast<__nv_bfloat16*>(X)[idx] = hi;
        static_cast<__nv_bfloat16*>(X)[idx + plane] = lo;
    } else if (mode == CTRECON_HILBERT_TF32) {
        uint32_t r;
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
        static_cast<float*>(X)[idx] = __uint_as_float(r);
    } else {
        static_cast<float*>(X)[idx] = v;
    }
}

// Block (T columns) x (RG row groups): thread (tx, ry) owns column j = blockIdx.x * T + tx and
// computes the derivative rows k = ry, ry + RG, ... then the kappa rows a = ry, ry + RG, ...;
// the RG groups keep RG independent row walks in flight per column.
// dres != NULL selects the direct half-view derivative of KatsevichFiltering_T.m:50-101
// (entries [column][side], side 0 applied to the next view, side 1 to this one; dl = DeltaL):
// the resampled row position (k + 1 - HalfZ) * Dzc + HalfZ is formed here in FP32, the column
// position comes from the FP64 host table; indices clamped as CheckData.m.
__global__ void k_deriv_rebin(const float* __restrict__ proj, int proj_view0, int P, int YL,
                              int ZL, int AL, int YLp, int vbeg,
                              const FwEntry* __restrict__ fw, const float2* __restrict__ cuy,
                              const float* __restrict__ zcv, float inv2dl,
                              const DresCol* __restrict__ dres, float dl,
                              void* __restrict__ X, size_t plane, int mode) {
    extern __shared__ float gf[];  // ZL x blockDim.x: the derivative of the block's columns
    const int T = blockDim.x, tx = threadIdx.x, ry = threadIdx.y, RG = blockDim.y;
    const int j = blockIdx.x * T + tx;
    const int p = vbeg + blockIdx.y;
    const size_t xv = (size_t)blockIdx.y * AL * YLp;
    const bool real = j < YL;
    if (real && dres) {
        const size_t S = (size_t)YL * ZL;
        const int pc = p > P - 2 ? P - 2 : p;  // the last view repeats its neighbour (:101)
        const float* Pn = proj + (size_t)(pc + 1 - proj_view0) * S;
        const float* Pc = proj + (size_t)(pc - proj_view0) * S;
        const DresCol c1 = dres[(size_t)j * 2], c2 = dres[(size_t)j * 2 + 1];
        const float hz = 0.5f * (float)(ZL + 1);
        auto sample = [&](const float* Pv, const DresCol& c, int k) {
            const float zc = fmaf(c.dzc, (float)(k + 1) - hz, hz);
            const float fz = floorf(zc);
            const float b = zc - fz, a = c.alfa;
            const int iz = (int)fz;
            const int ZD = min(max(iz, 1), ZL) - 1, ZU = min(max(iz + 1, 1), ZL) - 1;
            const float* rd = Pv + (size_t)ZD * YL;
            const float* ru = Pv + (size_t)ZU * YL;
            return rd[c.yd] * (1.f - a) * (1.f - b) + ru[c.yd] * (1.f - a) * b +
                   rd[c.yu] * a * (1.f - b) + ru[c.yu] * a * b;
        };
        for (int k = ry; k < ZL; k += RG)
            gf[k * T + tx] = (sample(Pn, c1, k) - sample(Pc, c2, k)) / dl;
    } else if (real) {
        const size_t S = (size_t)YL * ZL;
        // view derivative: views 0 and P-1 reuse the derivative of views 1 and P-2 (:58-59)
        const int pc = p < 1 ? 1 : (p > P - 2 ? P - 2 : p);
        const float* Pm = proj + (size_t)(pc - 1 - proj_view0) * S;
        const float* Pp = proj + (size_t)(pc + 1 - proj_view0) * S;
        const float* Pv = proj + (size_t)(p - proj_view0) * S;
        // u stencil with the reference's edge rule (:63-78)
        int jl = j - 1, jr = j + 1;
        if (j < 2) { jl = 0; jr = 2; }
        else if (j > YL - 3) { jl = YL - 3; jr = YL - 1; }
        const float2 cy = cuy[j];  // (u coefficient, y coordinate)
        // sixteen rows' loads in flight per thread (the kernel is load-latency bound)
#pragma unroll 16
        for (int k = ry; k < ZL; k += RG) {
            int kl = k - 1, kr = k + 1;  // v stencil, same edge rule (:85-95)
            if (k < 2) { kl = 0; kr = 2; }
            else if (k > ZL - 3) { kl = ZL - 3; kr = ZL - 1; }
            const float* row = Pv + (size_t)k * YL;
            float g = (Pp[(size_t)k * YL + j] - Pm[(size_t)k * YL + j]) * inv2dl;
            g = fmaf(row[jr] - row[jl], cy.x, g);
            g = fmaf(zcv[k] * cy.y, Pv[(size_t)kr * YL + j] - Pv[(size_t)kl * YL + j], g);
            gf[k * T + tx] = g;
        }
    }
    __syncthreads();
    if (j >= YLp) return;
    // every Hilbert form reads the kappa rows de-interleaved: even columns, then odd ones
    const size_t jx = (size_t)((j & 1) * (YLp >> 1) + (j >> 1));
    if (!real) {  // zero padding of the kappa rows (the GEMM form reads K = YLp)
        for (int a = ry; a < AL; a += RG) store_kappa(X, xv + (size_t)a * YLp + jx, plane, 0.f, mode);
        return;
    }
#pragma unroll 8
    for (int a = ry; a < AL; a += RG) {
        const FwEntry f = fw[(size_t)a * YL + j];
        store_kappa(X, xv + (size_t)a * YLp + jx, plane,
                    fmaf(f.wa, gf[f.r0 * T + tx], f.wb * gf[f.r1 * T + tx]), mode);
    }
}


// K1 launch: one thread per column (blocks of up to 128 columns x kRowGroups row groups), ZL
// floats of shared memory per thread
static Status k1_shape(int ZL, int* tj, size_t* smem) {
    *tj = 128;
    while (*tj > 32 && (size_t)ZL * *tj * sizeof(float) > 96 * 1024) *tj /= 2;
    *smem = (size_t)ZL * *tj * sizeof(float);
    if (*smem > 200 * 1024)
        return make_status(CTRECON_ERR_UNSUPPORTED, "too many detector rows for K1");
    return Status::Ok();
}

static Status launch_k1(cudaStream_t s, const float* d_proj, int proj_view0, int P, int YL,
                        int ZL, int AL, int YLp, int c0, int n, const FwEntry* fw,
                        const float2* cuy, const float* zcv, float inv2dl, const DresCol* dres,
                        float dl, void* X, size_t plane, int mode) {
    int tj;
    size_t smem;
    CTR_TRY(k1_shape(ZL, &tj, &smem));
    CTR_CUDA(cudaFuncSetAttribute(k_deriv_rebin, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
    const dim3 g((YLp + tj - 1) / tj, n);
    const dim3 b(tj, kRowGroups);
    k_deriv_rebin<<<g, b, smem, s>>>(d_proj, proj_view0, P, YL, ZL, AL, YLp, c0, fw, cuy, zcv,
                                     inv2dl, dres, dl, X, plane, mode);
    CTR_CUDA(cudaGetLastError());
    return Status::Ok();
}

// ---------------------------------------------------------------------------------------------
// K2 (FP32 SIMT)
// ---------------------------------------------------------------------------------------------
constexpr int kTileI = 64;   // output columns per CTA (32 of each parity)
constexpr int kXS = 65;      // padded row stride of the output tile in shared memory
constexpr int kXP = 36;      // row stride (floats) of one parity's 32 staged inputs
// kappa rows per thread: 4 (at most 384 threads, two CTAs per SM), or 8 for views of more than
// 192 kappa rows (at most 512 threads)
inline int simt_rows_per_thread(int AL) { return AL > 192 ? 8 : 4; }

__device__ __forceinline__ void cp_async16(float* dst, const float* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Thread (ig, ag): ig in 0..7 selects output parity q = ig>>2 and column group s = ig&3; the
// thread owns columns i_m = i0 + q + 2(8s + m), m = 0..7, and kappa rows a0..a0+RA-1. Only
// inputs of the other parity contribute (odd lags): with j_n = jc + (1-q) + 2n the lag is
// 2K + 1, K = (i0 - jc)/2 + q - 1 + 8s + m - n, and hso[KOFF + K] = h(2K + 1) (odd-lag taps,
// contiguous). Eight input steps n use the 15 taps K = c - 7 .. c + 7 of a register window
// indexed statically (T[m - n + 7]), so the inner loop is FMAs and its loads only. The
// kappa rows are de-interleaved (even columns, then odd ones, as the derivative kernel writes
// them), so each parity's 32 inputs of a chunk are 128 contiguous bytes: they are staged with
// cp.async into a double-buffered ring, one chunk ahead of the arithmetic.
template <int RA>
__global__ void __launch_bounds__(RA == 4 ? 384 : 512, RA == 4 ? 2 : 1)
k_hilbert_simt(const float* __restrict__ X, int AL, int ALpad, int YL, int YLp, int ZL,
               const float* __restrict__ hso, const BkEntry* __restrict__ bk,
               float* __restrict__ fproj) {
    extern __shared__ __align__(16) float sm[];
    const int KOFF = simt_koff(YLp);
    // the odd-lag taps twice: hs0 = hso, and hs1 shifted by one element so that both output
    // parities' 15-tap windows start on a 16-byte boundary (four LDS.128); hs1 sits 4 words past
    // a bank-aligned offset so the two parities' windows fall in different banks
    float* hs0 = sm;
    float* hs1 = sm + 2 * KOFF + 4;
    float* xs = sm + 4 * KOFF + 8;  // two stages of ALpad x 2 parities x kXP; later the output tile
    const int stage_f = ALpad * 2 * kXP;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int ig = tid & 7, ag = tid >> 3;
    const int q = ig >> 2, s = ig & 3;
    const int i0 = blockIdx.x * kTileI;
    const int v = blockIdx.y;
    const int YLh = YLp >> 1;
    const float* Xv = X + (size_t)v * AL * YLp;
    const int nchunk = YLp / kTileI;
    // staging: 8 threads per staged row (2 AL rows: kappa row a, parity p at r = 2a + p), 16
    // bytes each; a thread keeps one parity and steps RS rows (RS even), so its addresses advance
    // by constants
    const int RS = (nt >> 3) & ~1;
    const int r0 = tid >> 3, piece = tid & 7;
    const bool stager = r0 < RS;
    const float* src0 = Xv + (size_t)(r0 >> 1) * YLp + (r0 & 1) * YLh + 4 * piece;
    const size_t src_step = (size_t)(RS >> 1) * YLp;
    auto stage_in = [&](int c, int st) {
        if (stager) {
            float* dst = xs + st * stage_f + r0 * kXP + 4 * piece;
            const float* src = src0 + 32 * c;
            for (int r = r0; r < 2 * AL; r += RS, dst += RS * kXP, src += src_step)
                cp_async16(dst, src);
        }
        cp_async_commit();
    };
    stage_in(0, 0);
    for (int t = tid; t < 2 * KOFF; t += nt) {
        hs0[t] = hso[t];
        hs1[t] = t + 1 < 2 * KOFF ? hso[t + 1] : 0.f;
    }
    for (int t = tid; t < (ALpad - AL) * 2 * kXP; t += nt) {  // padded rows stay zero
        xs[AL * 2 * kXP + t] = 0.f;
        xs[stage_f + AL * 2 * kXP + t] = 0.f;
    }
    const int a0 = ag * RA;
    float acc[RA][8];
#pragma unroll
    for (int r = 0; r < RA; ++r)
#pragma unroll
        for (int m = 0; m < 8; ++m) acc[r][m] = 0.f;

    for (int c = 0; c < nchunk; ++c) {
        if (c + 1 < nchunk) {
            stage_in(c + 1, (c + 1) & 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const float* xr = xs + (c & 1) * stage_f + (a0 * 2 + (1 - q)) * kXP;
        const int c0 = KOFF + ((i0 - c * kTileI) >> 1) + q - 1 + 8 * s;
        // window start c0 - 8t - 7 is q (mod 4): hs0 from it, or hs1 from one element before
        const float* hq = q ? hs1 + (c0 - 8) : hs0 + (c0 - 7);
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            float T[16];
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                const float4 h4 = *reinterpret_cast<const float4*>(hq - 8 * t + 4 * w);
                T[4 * w] = h4.x; T[4 * w + 1] = h4.y; T[4 * w + 2] = h4.z; T[4 * w + 3] = h4.w;
            }
#pragma unroll
            for (int r = 0; r < RA; ++r) {
                const float4 x0 = *reinterpret_cast<const float4*>(xr + r * 2 * kXP + 8 * t);
                const float4 x1 = *reinterpret_cast<const float4*>(xr + r * 2 * kXP + 8 * t + 4);
                const float xv[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
#pragma unroll
                for (int n = 0; n < 8; ++n)
#pragma unroll
                    for (int m = 0; m < 8; ++m) acc[r][m] = fmaf(T[m - n + 7], xv[n], acc[r][m]);
            }
        }
        __syncthreads();  // the stage is refilled two chunks on
    }
    float* ot = xs;  // [ALpad][kXS] output tile in natural column order
#pragma unroll
    for (int r = 0; r < RA; ++r)
#pragma unroll
        for (int m = 0; m < 8; ++m) ot[(a0 + r) * kXS + q + 2 * (8 * s + m)] = acc[r][m];
    __syncthreads();
    // post-weight + backward rebin (:181-284): a gather across the kappa rows of the tile; the
    // table entries of four outputs are loaded (read-only path) before their stores, so their
    // latencies overlap
    const int4* bk4 = reinterpret_cast<const int4*>(bk);
    for (int idx0 = tid; idx0 < ZL * kTileI; idx0 += 4 * nt) {
        int4 e[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int idx = idx0 + r * nt, k = idx >> 6, i = i0 + (idx & 63);
            e[r] = (idx < ZL * kTileI && i < YL) ? __ldg(bk4 + (size_t)k * YL + i)
                                                 : make_int4(0, 0, 0, 0);
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int idx = idx0 + r * nt, k = idx >> 6, t = idx & 63, i = i0 + t;
            if (idx >= ZL * kTileI || i >= YL) continue;
            fproj[((size_t)v * ZL + k) * YL + i] =
                fmaf(__int_as_float(e[r].z), ot[e[r].x * kXS + t],
                     __int_as_float(e[r].w) * ot[e[r].y * kXS + t]);
        }
    }
}

// shared memory of k_hilbert_simt: the taps, two input stages, or the output tile
size_t simt_smem_bytes(int ALpad, int YLp) {
    const size_t stages = (size_t)2 * ALpad * 2 * kXP;
    return (4 * (size_t)simt_koff(YLp) + 8 + std::max(stages, (size_t)ALpad * kXS)) * sizeof(float);
}

// Launches k_hilbert_simt over `n` views of kappa rows X into `out` (shape checked first).
static Status simt_shape(int AL, int YLp, int* RA, int* ALpad, int* nthreads, size_t* smem) {
    *RA = simt_rows_per_thread(AL);
    *ALpad = (AL + *RA - 1) / *RA * *RA;
    *nthreads = (*ALpad / *RA) * 8;
    if (*nthreads > 512)
        return make_status(CTRECON_ERR_UNSUPPORTED, "too many kappa lines for the FP32 filter");
    *smem = simt_smem_bytes(*ALpad, YLp);
    if (*smem > 227 * 1024)
        return make_status(CTRECON_ERR_UNSUPPORTED, "detector too wide for the FP32 filter");
    if (YLp % 64)
        return make_status(CTRECON_ERR_INTERNAL, "kappa rows must be padded to 64 columns");
    return Status::Ok();
}

static Status launch_simt(cudaStream_t s, const float* X, int AL, int YL, int YLp, int ZL,
                          const float* hso, const BkEntry* bk, float* out, int n) {
    int RA, ALpad, nthreads;
    size_t smem;
    CTR_TRY(simt_shape(AL, YLp, &RA, &ALpad, &nthreads, &smem));
    const dim3 g((YL + kTileI - 1) / kTileI, n);
    if (RA == 4) {
        CTR_CUDA(cudaFuncSetAttribute(k_hilbert_simt<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
        k_hilbert_simt<4><<<g, nthreads, smem, s>>>(X, AL, ALpad, YL, YLp, ZL, hso, bk, out);
    } else {
        CTR_CUDA(cudaFuncSetAttribute(k_hilbert_simt<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
        k_hilbert_simt<8><<<g, nthreads, smem, s>>>(X, AL, ALpad, YL, YLp, ZL, hso, bk, out);
    }
    CTR_CUDA(cudaGetLastError());
    return Status::Ok();
}

// ---------------------------------------------------------------------------------------------
// FP64 <-> FP32 conversion (host-call staging)
// ---------------------------------------------------------------------------------------------
__global__ void k_f64_to_f32(const double* __restrict__ in, float* __restrict__ out, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}
__global__ void k_f32_to_f64(const float* __restrict__ in, double* __restrict__ out, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        out[i] = (double)in[i];
}

static int grid_for(size_t n) {
    size_t b = (n + 255) / 256;
    return (int)std::min<size_t>(b, 148 * 32);
}

Status launch_convert_f64_to_f32(cudaStream_t s, const double* in, float* out, size_t n) {
    if (n == 0) return Status::Ok();
    k_f64_to_f32<<<grid_for(n), 256, 0, s>>>(in, out, n);
    CTR_CUDA(cudaGetLastError());
    return Status::Ok();
}
Status launch_convert_f32_to_f64(cudaStream_t s, const float* in, double* out, size_t n) {
    if (n == 0) return Status::Ok();
    k_f32_to_f64<<<grid_for(n), 256, 0, s>>>(in, out, n);
    CTR_CUDA(cudaGetLastError());
    return Status::Ok();
}

// FilteringMode 1 (FunctionKat_v6.m:86-90): FProj = (FProj + FProj1) / 2, in place in `a`
__global__ void k_average_into(float* __restrict__ a, const float* __restrict__ b, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        a[i] = (a[i] + b[i]) / 2.f;
}
Status launch_average_into(cudaStream_t s, float* a, const float* b, size_t n) {
    if (n == 0) return Status::Ok();
    k_average_into<<<grid_for(n), 256, 0, s>>>(a, b, n);
    CTR_CUDA(cudaGetLastError());
    return Status::Ok();
}

// implemented in hilbert_tc.cu
Status launch_hilbert_tc(ctrecon_ctx* ctx, cudaStream_t s, FilterPlan& plan, const void* X,
                         int nviews, float* d_fproj_chunk, int mode);

// ---------------------------------------------------------------------------------------------
// Orchestration: views [view_begin, view_end) of a projection buffer holding views
// [proj_view0, proj_view0 + proj_nviews) are filtered into d_fproj (which holds views from
// out_view0 on).
// ---------------------------------------------------------------------------------------------
Status launch_filter(ctrecon_ctx* ctx, cudaStream_t s, FilterPlan& plan, const float* d_proj,
                     int proj_view0, int proj_nviews, float* d_fproj, int out_view0,
                     int view_begin, int view_end) {
    const FilterTables& t = plan.t;
    const int YL = t.YL, ZL = t.ZL, AL = t.AL, YLp = plan.YLp, P = t.P;
    const int mode = ctx->opt_hilbert;
    const int chunk = std::max(1, ctx->opt_filter_chunk);
    // 4 bytes per kappa sample in every format (FP32, TF32, or BF16 hi + lo planes), for the
    // views of one chunk or of the whole call when it has fewer
    const int nbuf = std::max(1, std::min(chunk, view_end - view_begin));
    CTR_TRY(ctx->ws_kappa.ensure((size_t)nbuf * AL * YLp * sizeof(float), "filter kappa rows"));
    void* X = ctx->ws_kappa.ptr;
    const DresCol* dres = nullptr;  // DerMode 0 resampling columns
    if (ctx->opt_deriv == CTRECON_DERIV_DIRECT) {
        if (!plan.dres_ready) {
            std::vector<DresCol> h((size_t)YL * 2);
            for (int j = 0; j < YL; ++j)
                for (int side = 0; side < 2; ++side)
                    h[(size_t)j * 2 + side] =
                        DresCol{t.dres_yd[side][j], t.dres_yu[side][j],
                                (float)t.dres_alfa[side][j], (float)t.dres_dzc[side][j]};
            CTR_TRY(plan.dres.ensure(h.size() * sizeof(DresCol), "DerMode 0 resampling table"));
            CTR_TRY(upload_now(plan.dres.ptr, h.data(), h.size() * sizeof(DresCol)));
            plan.dres_ready = true;
        }
        dres = plan.dres.as<DresCol>();
    }

    // K1: the staged form where it applies (chain-rule derivative), else the per-view form,
    // whose launch shape is checked before any launch
    const bool staged = ctx->opt_k1_form == CTRECON_K1_STAGED && !dres &&
                        k1_staged_fits(YL, ZL, AL, YLp, d_proj);
    if (!staged) {
        int tj;
        size_t smem1;
        CTR_TRY(k1_shape(ZL, &tj, &smem1));
    }
    if (mode == CTRECON_HILBERT_FP32) {  // K2 launch shape, checked before any launch
        int RA, ALpad, nthreads2;
        size_t smem2;
        CTR_TRY(simt_shape(AL, YLp, &RA, &ALpad, &nthreads2, &smem2));
    }

    for (int c0 = view_begin; c0 < view_end; c0 += chunk) {
        const int n = std::min(chunk, view_end - c0);
        const size_t plane = (size_t)n * AL * YLp;
        {
            KernelTimer tm(ctx, s, kKDerivRebin);
            if (staged)
                CTR_TRY(launch_k1_staged(ctx, s, d_proj, proj_view0, proj_nviews, P, YL, ZL, AL,
                                         YLp, c0, n, plan.fw.as<FwEntry>(),
                                         plan.cuy.as<float2>(), plan.zcv.as<float>(),
                                         plan.inv2dl, X, plane, mode));
            else
                CTR_TRY(launch_k1(s, d_proj, proj_view0, P, YL, ZL, AL, YLp, c0, n,
                                  plan.fw.as<FwEntry>(), plan.cuy.as<float2>(),
                                  plan.zcv.as<float>(), plan.inv2dl, dres, (float)t.DeltaL, X,
                                  plane, mode));
        }
        float* out = d_fproj + (size_t)(c0 - out_view0) * YL * ZL;
        if (mode == CTRECON_HILBERT_FP32) {
            KernelTimer tm(ctx, s, kKHilbertSimt);
            CTR_TRY(launch_simt(s, static_cast<const float*>(X), AL, YL, YLp, ZL,
                                plan.h.as<float>(), plan.bk.as<BkEntry>(), out, n));
        } else {
            KernelTimer tm(ctx, s, kKHilbertTc);
            CTR_TRY(launch_hilbert_tc(ctx, s, plan, X, n, out, mode));
        }
    }
    return Status::Ok();
}

// The FP32 filter over all views with caller-placed device tables and kappa-row scratch
// (`chunk` views of AL*YLp floats), for the entry point that allocates nothing (noalloc.cu).
Status launch_filter_fp32_preplaced(cudaStream_t s, const FilterTables& t, int YLp,
                                    const FwEntry* fw, const BkEntry* bk, const float2* cuy,
                                    const float* zcv, const float* hso, float inv2dl,
                                    float* kappa, int chunk, const float* d_proj,
                                    float* d_fproj) {
    const int YL = t.YL, ZL = t.ZL, AL = t.AL, P = t.P;
    {
        int tj;
        size_t smem1;
        CTR_TRY(k1_shape(ZL, &tj, &smem1));
    }
    {
        int RA, ALpad, nthreads2;
        size_t smem2;
        CTR_TRY(simt_shape(AL, YLp, &RA, &ALpad, &nthreads2, &smem2));
    }
    for (int c0 = 0; c0 < P; c0 += chunk) {
        const int n = std::min(chunk, P - c0);
        CTR_TRY(launch_k1(s, d_proj, 0, P, YL, ZL, AL, YLp, c0, n, fw, cuy, zcv, inv2dl, nullptr,
                          0.f, kappa, 0, CTRECON_HILBERT_FP32));
        CTR_TRY(launch_simt(s, kappa, AL, YL, YLp, ZL, hso, bk, d_fproj + (size_t)c0 * YL * ZL, n));
    }
    return Status::Ok();
}

}  // namespace ctr
