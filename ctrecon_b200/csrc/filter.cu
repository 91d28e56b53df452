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
    // the tensor-core forms read each kappa row de-interleaved: even columns, then odd ones
    const size_t jx = mode == CTRECON_HILBERT_FP32 ? (size_t)j
                                                   : (size_t)((j & 1) * (YLp >> 1) + (j >> 1));
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

// ---------------------------------------------------------------------------------------------
// K2 (FP32 SIMT)
// ---------------------------------------------------------------------------------------------
constexpr int kTileI = 64;   // output columns per CTA
constexpr int kXS = 65;      // padded shared-memory row stride
constexpr int kRA = 4;       // kappa rows per thread

// thread (ig, ag): ig in 0..7 selects parity q = ig>>2 and column group s = ig&3; the thread
// owns columns i_m = i0 + q + 2(8s + m), m = 0..7, and kappa rows a0..a0+kRA-1. Only inputs
// j of the opposite parity contribute (odd lags), so the lag window advances by one tap
// per step of j and rotates through registers.
__global__ void k_hilbert_simt(const float* __restrict__ X, int AL, int ALpad, int YL, int YLp,
                               int ZL, const float* __restrict__ hpad, int HOFF,
                               const BkEntry* __restrict__ bk, float* __restrict__ fproj) {
    extern __shared__ float sm[];
    float* hs = sm;               // 2*HOFF taps, hs[HOFF + L] = h[L]
    float* xs = hs + 2 * HOFF;    // ALpad x kXS: kappa-row chunk, later the output tile
    const int tid = threadIdx.x, nt = blockDim.x;
    const int ig = tid & 7, ag = tid >> 3;
    const int q = ig >> 2, s = ig & 3;
    const int i0 = blockIdx.x * kTileI;
    const int v = blockIdx.y;
    const float* Xv = X + (size_t)v * AL * YLp;
    for (int t = tid; t < 2 * HOFF; t += nt) hs[t] = hpad[t];
    const int a0 = ag * kRA;
    float acc[kRA][8];
#pragma unroll
    for (int r = 0; r < kRA; ++r)
#pragma unroll
        for (int m = 0; m < 8; ++m) acc[r][m] = 0.f;

    for (int jc = 0; jc < YLp; jc += kTileI) {
        __syncthreads();
        for (int t = tid; t < ALpad * kTileI; t += nt) {
            const int a = t >> 6, jj = t & 63;
            xs[a * kXS + jj] = (a < AL) ? Xv[(size_t)a * YLp + jc + jj] : 0.f;
        }
        __syncthreads();
        if (a0 < ALpad) {
            // lag(m, n) = i_m - j_n with j_n = jc + (1-q) + 2n
            const int base = HOFF + i0 - jc + 2 * q - 1 + 16 * s;
            float w[8];
#pragma unroll
            for (int m = 0; m < 8; ++m) w[m] = hs[base + 2 * m];
            const float* xr = xs + a0 * kXS + (1 - q);
#pragma unroll
            for (int n = 0; n < 32; ++n) {
                if (n > 0) {
#pragma unroll
                    for (int m = 7; m > 0; --m) w[m] = w[m - 1];
                    w[0] = hs[base - 2 * n];
                }
#pragma unroll
                for (int r = 0; r < kRA; ++r) {
                    const float xv = xr[r * kXS + 2 * n];
#pragma unroll
                    for (int m = 0; m < 8; ++m) acc[r][m] = fmaf(w[m], xv, acc[r][m]);
                }
            }
        }
    }
    __syncthreads();
    if (a0 < ALpad) {
#pragma unroll
        for (int r = 0; r < kRA; ++r)
#pragma unroll
            for (int m = 0; m < 8; ++m) xs[(a0 + r) * kXS + q + 2 * (8 * s + m)] = acc[r][m];
    }
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
                fmaf(__int_as_float(e[r].z), xs[e[r].x * kXS + t],
                     __int_as_float(e[r].w) * xs[e[r].y * kXS + t]);
        }
    }
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
    (void)proj_nviews;
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

    // K1 launch shape: one thread per column, ZL floats of shared memory per thread
    int tj = 128;
    while (tj > 32 && (size_t)ZL * tj * sizeof(float) > 96 * 1024) tj /= 2;
    const size_t smem1 = (size_t)ZL * tj * sizeof(float);
    const dim3 b1(tj, kRowGroups);
    if (smem1 > 200 * 1024)
        return make_status(CTRECON_ERR_UNSUPPORTED, "too many detector rows for K1");
    CTR_CUDA(cudaFuncSetAttribute(k_deriv_rebin, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem1));
    // K2 launch shape
    const int ALpad = (AL + kRA - 1) / kRA * kRA;
    const int nthreads2 = std::max(32, (ALpad / kRA) * 8);
    if (nthreads2 > 1024)
        return make_status(CTRECON_ERR_UNSUPPORTED, "too many kappa lines for the FP32 filter");
    const int HOFF = YLp + 64;
    const size_t smem2 = (2 * (size_t)HOFF + (size_t)ALpad * kXS) * sizeof(float);
    if (smem2 > 227 * 1024)
        return make_status(CTRECON_ERR_UNSUPPORTED, "detector too wide for the FP32 filter");
    CTR_CUDA(cudaFuncSetAttribute(k_hilbert_simt, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem2));

    for (int c0 = view_begin; c0 < view_end; c0 += chunk) {
        const int n = std::min(chunk, view_end - c0);
        dim3 g1((YLp + tj - 1) / tj, n);
        const size_t plane = (size_t)n * AL * YLp;
        {
            KernelTimer tm(ctx, s, kKDerivRebin);
            k_deriv_rebin<<<g1, b1, smem1, s>>>(d_proj, proj_view0, P, YL, ZL, AL, YLp, c0,
                                                plan.fw.as<FwEntry>(), plan.cuy.as<float2>(),
                                                plan.zcv.as<float>(), plan.inv2dl, dres,
                                                (float)t.DeltaL, X, plane, mode);
            CTR_CUDA(cudaGetLastError());
        }
        float* out = d_fproj + (size_t)(c0 - out_view0) * YL * ZL;
        if (mode == CTRECON_HILBERT_FP32) {
            KernelTimer tm(ctx, s, kKHilbertSimt);
            dim3 g2((YL + kTileI - 1) / kTileI, n);
            k_hilbert_simt<<<g2, nthreads2, smem2, s>>>(static_cast<const float*>(X), AL, ALpad,
                                                        YL, YLp, ZL, plan.h.as<float>(), HOFF,
                                                        plan.bk.as<BkEntry>(), out);
            CTR_CUDA(cudaGetLastError());
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
                                    const float* zcv, const float* hpad, float inv2dl,
                                    float* kappa, int chunk, const float* d_proj,
                                    float* d_fproj) {
    const int YL = t.YL, ZL = t.ZL, AL = t.AL, P = t.P;
    int tj = 128;
    while (tj > 32 && (size_t)ZL * tj * sizeof(float) > 96 * 1024) tj /= 2;
    const size_t smem1 = (size_t)ZL * tj * sizeof(float);
    const dim3 b1(tj, kRowGroups);
    if (smem1 > 200 * 1024)
        return make_status(CTRECON_ERR_UNSUPPORTED, "too many detector rows for K1");
    CTR_CUDA(cudaFuncSetAttribute(k_deriv_rebin, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem1));
    const int ALpad = (AL + kRA - 1) / kRA * kRA;
    const int nthreads2 = std::max(32, (ALpad / kRA) * 8);
    if (nthreads2 > 1024)
        return make_status(CTRECON_ERR_UNSUPPORTED, "too many kappa lines for the FP32 filter");
    const int HOFF = YLp + 64;
    const size_t smem2 = (2 * (size_t)HOFF + (size_t)ALpad * kXS) * sizeof(float);
    if (smem2 > 227 * 1024)
        return make_status(CTRECON_ERR_UNSUPPORTED, "detector too wide for the FP32 filter");
    CTR_CUDA(cudaFuncSetAttribute(k_hilbert_simt, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem2));
    for (int c0 = 0; c0 < P; c0 += chunk) {
        const int n = std::min(chunk, P - c0);
        dim3 g1((YLp + tj - 1) / tj, n);
        k_deriv_rebin<<<g1, b1, smem1, s>>>(d_proj, 0, P, YL, ZL, AL, YLp, c0, fw, cuy, zcv,
                                            inv2dl, nullptr, 0.f, kappa, 0,
                                            CTRECON_HILBERT_FP32);
        CTR_CUDA(cudaGetLastError());
        dim3 g2((YL + kTileI - 1) / kTileI, n);
        k_hilbert_simt<<<g2, nthreads2, smem2, s>>>(kappa, AL, ALpad, YL, YLp, ZL, hpad, HOFF, bk,
                                                    d_fproj + (size_t)c0 * YL * ZL);
        CTR_CUDA(cudaGetLastError());
    }
    return Status::Ok();
}

}  // namespace ctr
