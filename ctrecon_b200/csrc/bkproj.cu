// bkproj.cu -- K4: voxel-driven backprojection over each voxel's PI interval
// (KatsevichBkProj.cpp:164-265), FP32 interpolation and accumulation.
//
// Work decomposition. A CTA owns a 16 x 16 tile of (x, y) columns and kTZ consecutive z
// voxels per column; thread t owns one column and its kTZ voxels. The CTA walks the union of
// its voxels' PI intervals in blocks of kNB views. For each view of a block one thread
// projects the tile's 8 corners to get the detector footprint (a convex bound of every tap
// the tile can read), and the CTA stages that footprint of FProj into shared memory. Per
// (column, view) the thread computes the z-invariant quantities once -- the column's detector
// u and its bilinear weight, 1/fenmu, |X-S|^2 in the xy plane -- so that per voxel only the
// detector v, one rsqrt and the v-interpolation remain (KatsevichBkProj.cpp:243-246: fenmu
// and YY do not depend on z).
//
// Endpoint weights. With the PI record (bi, bf, ti, tf), B = bi + bf and T = ti + tf, the
// reference's loop bounds are [max(1, bi), min(ti+1, P-2)] and its Coef values (:182-234)
// are F(T - p) on views p >= ti and F(p - B) on the others, F(s) the quadratic ramp
// 0 (s <= -1), (1+s)^2/2 (-1 < s <= 0), 1-(1-s)^2/2 (0 < s < 1), 1 (s >= 1); the "T side
// wins" rule reproduces the order in which the reference assigns Coef for short intervals.
#include "internal.h"

#include <climits>

namespace ctr {

constexpr int kTXY = 16;     // columns per tile edge
constexpr int kTZ = 8;       // z voxels per thread
constexpr int kNB = 4;       // views per staged block
constexpr int kCap = 2048;   // shared floats per staged view

struct Foot { int u0, v0, W, H; };

__device__ __forceinline__ float ramp(float s) {
    float c = fminf(fmaxf(s, -1.f), 1.f);
    return 0.5f + c - 0.5f * c * fabsf(c);
}

template <typename OutT>
__global__ void __launch_bounds__(256, 2)
k_bkproj(BPParams kp, const float* __restrict__ fproj, const PiRecord* __restrict__ pit,
         const float4* __restrict__ views, const float* __restrict__ xyz,
         OutT* __restrict__ image) {
    extern __shared__ float tile[];  // kNB x kCap
    __shared__ Foot foot[kNB];
    __shared__ float4 vg[kNB];
    __shared__ int s_pmin, s_pmax;

    const int tid = threadIdx.x;
    const int tx = tid & (kTXY - 1), ty = tid >> 4;
    const int x = blockIdx.x * kTXY + tx, y = blockIdx.y * kTXY + ty;
    const int zb = blockIdx.z * kTZ;
    const int NX = kp.NX, NY = kp.NY, NZ = kp.NZ, P = kp.P, YL = kp.YL, ZL = kp.ZL;
    const bool col_ok = (x < NX) && (y < NY);
    const float* xc = xyz;
    const float* yc = xyz + NX;
    const float* zc = xyz + NX + NY;
    const float X = col_ok ? xc[x] : 0.f, Y = col_ok ? yc[y] : 0.f;

    if (tid == 0) { s_pmin = INT_MAX; s_pmax = INT_MIN; }

    int bi[kTZ], ti[kTZ];
    float bf[kTZ], tf[kTZ], zv[kTZ], acc[kTZ];
    int tmin = INT_MAX, tmax = INT_MIN;
    const size_t colbase = ((size_t)x * NY + y) * NZ;
#pragma unroll
    for (int k = 0; k < kTZ; ++k) {
        const int z = zb + k;
        PiRecord r{kPiInvalid, 0.f, -10, 0.f};
        if (col_ok && z < NZ) r = pit[colbase + z];
        bi[k] = r.bi; bf[k] = r.bf; ti[k] = r.ti; tf[k] = r.tf;
        zv[k] = (z < NZ) ? zc[z] : 0.f;
        acc[k] = 0.f;
        if (r.bi != kPiInvalid) {
            tmin = min(tmin, max(max(1, r.bi), kp.win0));
            tmax = max(tmax, min(min(r.ti + 1, P - 2), kp.win1));
        }
    }
    // warp and CTA view ranges
    int wmin = tmin, wmax = tmax;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        wmin = min(wmin, __shfl_xor_sync(0xffffffffu, wmin, o));
        wmax = max(wmax, __shfl_xor_sync(0xffffffffu, wmax, o));
    }
    __syncthreads();
    if ((tid & 31) == 0 && wmin <= wmax) {
        atomicMin(&s_pmin, wmin);
        atomicMax(&s_pmax, wmax);
    }
    __syncthreads();
    const int pmin = s_pmin, pmax = s_pmax;
    if (pmin > pmax) return;  // no written voxel in this tile

    // the tile's bounding box (voxel centres) for the footprint
    const int x0 = blockIdx.x * kTXY, x1 = min(x0 + kTXY, NX) - 1;
    const int y0 = blockIdx.y * kTXY, y1 = min(y0 + kTXY, NY) - 1;
    const int z1 = min(zb + kTZ, NZ) - 1;
    const float bx0 = xc[x0], bx1 = xc[x1], by0 = yc[y0], by1 = yc[y1];
    const float bz0 = zc[zb], bz1 = zc[z1];
    const float R = kp.Rf, DdU = kp.DdU, DdV = kp.DdV, HalfY = kp.HalfY, HalfZ = kp.HalfZ;

    for (int pb = pmin; pb <= pmax; pb += kNB) {
        __syncthreads();  // previous block fully consumed
        if (tid < kNB) {
            const int p = pb + tid;
            Foot f{0, 0, -1, 0};
            if (p <= pmax) {
                const float4 g = views[p];
                vg[tid] = g;
                float umin = 1e30f, umax = -1e30f, vmin = 1e30f, vmax = -1e30f;
                bool ok = true;
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const float cx = (c & 1) ? bx1 : bx0, cy = (c & 2) ? by1 : by0;
                    const float fen = R - (cx * g.x + cy * g.y);
                    ok = ok && (fen > 1e-3f * R);
                    const float inv = 1.f / fen;
                    const float u = (cy * g.x - cx * g.y) * DdU * inv + HalfY;
                    const float va = (bz0 - g.z) * DdV * inv + HalfZ;
                    const float vb = (bz1 - g.z) * DdV * inv + HalfZ;
                    umin = fminf(umin, u); umax = fmaxf(umax, u);
                    vmin = fminf(vmin, fminf(va, vb)); vmax = fmaxf(vmax, fmaxf(va, vb));
                }
                if (ok) {
                    // taps use floor() clamped to [0, N-2] and the next cell; widen by one
                    const int u0 = max(0, min(YL - 2, (int)floorf(umin) - 1));
                    const int u1 = max(0, min(YL - 2, (int)floorf(umax) + 1)) + 1;
                    const int v0 = max(0, min(ZL - 2, (int)floorf(vmin) - 1));
                    const int v1 = max(0, min(ZL - 2, (int)floorf(vmax) + 1)) + 1;
                    const int W = u1 - u0 + 1, H = v1 - v0 + 1;
                    if (W * H <= kCap) f = Foot{u0, v0, W, H};
                    else f = Foot{0, 0, -2, 0};  // too large: read FProj directly
                } else {
                    f = Foot{0, 0, -2, 0};
                }
            }
            foot[tid] = f;
        }
        __syncthreads();
        // stage the footprints
#pragma unroll 1
        for (int j = 0; j < kNB; ++j) {
            const Foot f = foot[j];
            if (f.W <= 0) continue;
            const float* src = fproj + ((size_t)(pb + j) * ZL + f.v0) * YL + f.u0;
            float* dst = tile + j * kCap;
            const int n = f.W * f.H;
            for (int t = tid; t < n; t += blockDim.x) {
                const int r = t / f.W, c = t - r * f.W;
                dst[t] = __ldg(src + (size_t)r * YL + c);
            }
        }
        __syncthreads();
        if (!col_ok || wmin > wmax) continue;
#pragma unroll 1
        for (int j = 0; j < kNB; ++j) {
            const int p = pb + j;
            if (p > pmax) break;
            if (p < wmin || p > wmax) continue;  // warp-uniform
            if (p < tmin || p > tmax) continue;
            const Foot f = foot[j];
            const float4 g = vg[j];
            const float fen = R - (X * g.x + Y * g.y);
            const float YY = Y * g.x - X * g.y;
            const float inv = 1.f / fen;
            const float u = YY * DdU * inv + HalfY;
            const float kv = DdV * inv;
            const float r2 = fen * fen + YY * YY;
            const int ui = max(0, min(YL - 2, (int)floorf(u)));
            const float alfa = u - (float)ui;
            const bool smem = f.W > 0;
            const float* base;
            int stride;
            if (smem) {
                base = tile + j * kCap + (ui - f.u0) - f.v0 * f.W;
                stride = f.W;
            } else {
                base = fproj + (size_t)p * ZL * YL + ui;
                stride = YL;
            }
#pragma unroll
            for (int k = 0; k < kTZ; ++k) {
                const int d0 = p - bi[k];
                const int d1 = ti[k] + 1 - p;
                if ((d0 | d1) < 0) continue;
                float w = 1.f;
                if (d1 <= 1) w = ramp(tf[k] + (float)(d1 - 1));
                else if (d0 <= 1) w = ramp((float)d0 - bf[k]);
                const float dz = zv[k] - g.z;
                const float v = fmaf(dz, kv, HalfZ);
                const float rinv = rsqrtf(fmaf(dz, dz, r2));
                const int vi = max(0, min(ZL - 2, (int)floorf(v)));
                const float beta = v - (float)vi;
                const float* q = base + vi * stride;
                float t00, t01, t10, t11;
                if (smem) {
                    t00 = q[0]; t01 = q[1]; t10 = q[stride]; t11 = q[stride + 1];
                } else {
                    t00 = __ldg(q); t01 = __ldg(q + 1); t10 = __ldg(q + stride);
                    t11 = __ldg(q + stride + 1);
                }
                const float a0 = fmaf(alfa, t01 - t00, t00);
                const float a1 = fmaf(alfa, t11 - t10, t10);
                const float val = fmaf(beta, a1 - a0, a0);
                acc[k] = fmaf(w * val, rinv, acc[k]);
            }
        }
    }
    if (!col_ok) return;
#pragma unroll
    for (int k = 0; k < kTZ; ++k) {
        const int z = zb + k;
        if (z < NZ && bi[k] != kPiInvalid) {
            OutT* o = image + colbase + z;
            const OutT v = (OutT)(-acc[k] * kp.invPs);
            *o = kp.accum ? *o + v : v;
        }
    }
}

template <typename OutT>
static Status launch_bk(cudaStream_t s, BPPlan& plan, const float* d_fproj,
                        const PiRecord* d_pitab, OutT* d_image) {
    const BPParams& kp = plan.kp;
    dim3 grid((kp.NX + kTXY - 1) / kTXY, (kp.NY + kTXY - 1) / kTXY, (kp.NZ + kTZ - 1) / kTZ);
    const size_t smem = (size_t)kNB * kCap * sizeof(float);
    CTR_CUDA(cudaFuncSetAttribute(k_bkproj<OutT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
    k_bkproj<OutT><<<grid, 256, smem, s>>>(kp, d_fproj, d_pitab, plan.views.as<float4>(),
                                           plan.xyz.as<float>(), d_image);
    CTR_CUDA(cudaGetLastError());
    return Status::Ok();
}

// Valid voxels (those with a PI interval) set to 0 before view-window accumulation.
__global__ void k_zero_valid(const PiRecord* __restrict__ pit, double* __restrict__ image,
                             size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        if (pit[i].bi != kPiInvalid) image[i] = 0.0;
}

Status launch_zero_valid_f64(cudaStream_t s, const PiRecord* d_pitab, double* d_image, size_t n) {
    if (n == 0) return Status::Ok();
    const unsigned grid = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 32);
    k_zero_valid<<<grid, 256, 0, s>>>(d_pitab, d_image, n);
    CTR_CUDA(cudaGetLastError());
    return Status::Ok();
}

template <typename OutT>
Status launch_bkproj_v2(int variant, cudaStream_t s, BPPlan& plan, const float* d_fproj,
                        const PiRecord* d_pitab, OutT* d_image, int* err);

// CTRECON_OPT_BP_VARIANT: 0..12 select the tiled forms (bkproj2.cu), 100 the first form above,
// CTRECON_BP_AUTO the tuning table's choice. The fourth and fifth forms (5..12) report a
// bounded wait that gave up in the context's device word.
Status launch_bkproj_f32(ctrecon_ctx* ctx, cudaStream_t s, BPPlan& plan, const float* d_fproj,
                         const PiRecord* d_pitab, float* d_image) {
    const int variant = bp_variant_for(ctx, plan.g);
    if (variant >= 100) {
        KernelTimer tm(ctx, s, kKBackproject);
        return launch_bk<float>(s, plan, d_fproj, d_pitab, d_image);
    }
    if (!ctx->ws_flag.ptr) return make_status(CTRECON_ERR_INTERNAL, "device error word not set up");
    if (variant >= 10)
        return launch_bkproj_v5<float>(variant, s, plan, d_fproj, d_pitab, d_image,
                                       ctx->ws_flag.as<int>(), ctx->ws_rec, ctx->ws_boxmaps,
                                       ctx->boxmap_key, ctx->opt_bp_window, ctx);
    KernelTimer tm(ctx, s, kKBackproject);
    return launch_bkproj_v2<float>(variant, s, plan, d_fproj, d_pitab, d_image,
                                   ctx->ws_flag.as<int>());
}

Status launch_bkproj_f64out(ctrecon_ctx* ctx, cudaStream_t s, BPPlan& plan,
                            const float* d_fproj, const PiRecord* d_pitab, double* d_image) {
    const int variant = bp_variant_for(ctx, plan.g);
    if (variant >= 100) {
        KernelTimer tm(ctx, s, kKBackproject);
        return launch_bk<double>(s, plan, d_fproj, d_pitab, d_image);
    }
    if (!ctx->ws_flag.ptr) return make_status(CTRECON_ERR_INTERNAL, "device error word not set up");
    if (variant >= 10)
        return launch_bkproj_v5<double>(variant, s, plan, d_fproj, d_pitab, d_image,
                                        ctx->ws_flag.as<int>(), ctx->ws_rec, ctx->ws_boxmaps,
                                        ctx->boxmap_key, ctx->opt_bp_window, ctx);
    KernelTimer tm(ctx, s, kKBackproject);
    return launch_bkproj_v2<double>(variant, s, plan, d_fproj, d_pitab, d_image,
                                    ctx->ws_flag.as<int>());
}

}  // namespace ctr
