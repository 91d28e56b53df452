// pinet_infer.cu -- inference of the PI-line network, and the learned PI-line solve.
//
// A persistent CTA of 128 threads evaluates the network for 128 items at a time (voxels of the
// volume, or given feature triples), one item per thread and per TMEM lane:
//   layer 0 (3 -> 64)   FP32 FMA with BF16-rounded weights, SiLU, BF16 activations written
//                       into a 128 x 64 K-major tile in shared memory (128-byte swizzle);
//   layers 1..3 (64x64) one thread issues four tcgen05.mma (M = 128 items, N = 64, K = 16 each)
//                       from that tile and the layer's BF16 weight tile, FP32 accumulation in 64
//                       TMEM columns; every thread reads its row back (tcgen05.ld), adds the bias,
//                       applies SiLU and writes the next layer's input tile;
//   layer 4 (64 -> 2)   FP32 FMA.
// For the learned PI solve the kernel stores each voxel's predicted sb offset; the FP64 Newton
// kernel (pi.cu) then starts from 2 pi z - pi/2 + offset and writes the voxel's PI record
// exactly as the plain solver does.
//
// k_pinet_voxels is the per-voxel learned start in packed BF16 (CTRECON_PINET_VOXEL_BF16): the
// same network with FP32 features, every SiLU in packed BF16 arithmetic (the hidden
// pre-activations cut to BF16 by a byte permute) and the output layer as a fourth tensor-core
// product; its output only starts the FP64 Newton solve, which still decides every endpoint.
// Either per-voxel form is bounded by the MUFU pipe (one tanh per neuron: 256 per voxel, 16 per
// SM and clock in every precision).
//
// CTRECON_PINET_GRID (the default): the network's inputs depend on (r, psi = phi - 2 pi z)
// only, so k_pinet_infer evaluates it once per point of a 256 x 4096 grid of (r, psi), an FP64
// Newton solve refines each grid point from the network's output (k_grid_refine), and the Newton
// kernel (pi.cu) starts every voxel from the bilinear interpolation of the refined grid.
#include "internal.h"
#include "pi_device.cuh"
#include "pinet.h"
#include "tc_util.cuh"

#include <cuda_bf16.h>

#include <algorithm>

namespace ctr {

Status pinet_ensure(ctrecon_ctx* ctx);
Status launch_pi_guess(ctrecon_ctx* ctx, cudaStream_t s, BPPlan& plan, PiRecord* d_pitab,
                       unsigned long long* d_updates, unsigned long long* d_iters,
                       const float* d_guess, const void* d_grid, int nr, int np, double r_max);

namespace {

constexpr int kT = 128;
// shared-memory layout (offsets from a 1024-byte aligned base)
constexpr int kSmA = 0;                    // activation tile, 128 x 128 B
constexpr int kSmW = 16384;                // three weight tiles, 64 x 128 B each
constexpr int kSmF = 16384 + 3 * 8192;     // FP32 parameters (kNetF32 floats)
constexpr int kSmBar = kSmF + kNetF32 * 4; // mbarrier (8-byte aligned)
constexpr int kSmSlot = kSmBar + 8;        // TMEM address
constexpr int kSmBytes = kSmSlot + 8 + 1024;

// SiLU, x * sigmoid(x): accurate form for the FP32 features of the output layer, one-MUFU
// form 0.5 x (1 + tanh(x/2)) for activations that are rounded to BF16 anyway
__device__ __forceinline__ float silu_acc(float z) { return __fdividef(z, 1.f + __expf(-z)); }
__device__ __forceinline__ float silu_bf(float z) {
    const float h = 0.5f * z;
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(h));
    return fmaf(h, t, h);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);  // .x = a (low half)
    return *reinterpret_cast<uint32_t*>(&h);
}

__global__ void k_net_prep(const float* __restrict__ theta, unsigned char* __restrict__ net) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    __nv_bfloat16* wb = reinterpret_cast<__nv_bfloat16*>(net);
    float* f = reinterpret_cast<float*>(net + kNetBf16Bytes);
    if (i < 3 * 4096) wb[i] = __float2bfloat16_rn(theta[pinet_offW(1 + i / 4096) + i % 4096]);
    if (i < 192) f[kNetF32_W0 + i] = __bfloat162float(__float2bfloat16_rn(theta[pinet_offW(0) + i]));
    if (i < 256) f[kNetF32_B0 + i] = theta[pinet_offB(i / 64) + i % 64];
    if (i < 128) f[kNetF32_W4 + i] = __bfloat162float(__float2bfloat16_rn(theta[pinet_offW(4) + i]));
    if (i < 2) f[kNetF32_B4 + i] = theta[pinet_offB(4) + i];
}

// voxel mode (feat == nullptr): guess[idx] = predicted sb offset (radians) of each voxel inside
// the cylinder; feature mode: raw[idx] = the two network outputs
__global__ void __launch_bounds__(kT)
k_pinet_infer(BPParams kp, const unsigned char* __restrict__ net, long long n_items,
              const float* __restrict__ feat, float2* __restrict__ raw,
              float* __restrict__ guess, int* __restrict__ err) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* sm = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* A = sm + kSmA;
    uint8_t* Wt = sm + kSmW;
    float* F = reinterpret_cast<float*>(sm + kSmF);
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kSmBar);
    uint32_t* slot = reinterpret_cast<uint32_t*>(sm + kSmSlot);
    const int t = threadIdx.x, warp = t >> 5;

    // weights into 128-byte-swizzled K-major tiles (row = output neuron, 8 chunks of 8 inputs)
    const uint4* src = reinterpret_cast<const uint4*>(net);
    for (int q = t; q < 3 * 64 * 8; q += kT) {
        const int l = q >> 9, r = (q >> 3) & 63, c = q & 7;
        *reinterpret_cast<uint4*>(Wt + l * 8192 + tcu::sw128_offset(r, c)) = src[q];
    }
    const float* fsrc = reinterpret_cast<const float*>(net + kNetBf16Bytes);
    for (int q = t; q < kNetF32; q += kT) F[q] = fsrc[q];
    if (t == 0) {
        tcu::mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tcu::tmem_alloc(slot, 64);
    tcu::fence_proxy_async();
    tcu::fence_before();
    __syncthreads();
    tcu::fence_after();
    const uint32_t tmem = *slot;
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
    const uint32_t idesc = tcu::idesc_bf16_f32(128, 64);
    const uint32_t a_addr = tcu::smem_u32(A), w_addr = tcu::smem_u32(Wt);
    uint32_t phase = 0;
    const float* W0 = F + kNetF32_W0;
    const float* B0 = F + kNetF32_B0;
    const float* W4 = F + kNetF32_W4;
    const float* B4 = F + kNetF32_B4;
    const long long ntiles = (n_items + kT - 1) / kT;

    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long long idx = tile * kT + t;
        const bool valid = idx < n_items;
        float f0 = 0.f, f1 = 1.f, f2 = 0.f;
        bool inside = false;
        if (feat) {
            if (valid) { f0 = feat[3 * idx]; f1 = feat[3 * idx + 1]; f2 = feat[3 * idx + 2]; }
        } else if (valid) {
            int xi, yi, zi;
            double X, Y, Z;
            voxel_xyz(kp, idx, &xi, &yi, &zi, &X, &Y, &Z);
            inside = X * X + Y * Y < kp.ObjR2;  // KatsevichBkProj.cpp:168
            const double x = X / kp.ScanR, y = Y / kp.ScanR, z = Z / kp.HelicP;
            const double r = sqrt(x * x + y * y);
            double s2, c2;
            sincos(2 * kRefPi * z, &s2, &c2);
            const double cph = r > 0 ? x / r : 1.0, sph = r > 0 ? y / r : 0.0;
            f0 = (float)(r * kPinetRInv);
            f1 = (float)(cph * c2 + sph * s2);  // cos(phi - 2 pi z)
            f2 = (float)(sph * c2 - cph * s2);  // sin(phi - 2 pi z)
        }
        // layer 0 -> activation tile
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            uint32_t pk[4];
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                const int o = c * 8 + 2 * h;
                const float v0 = silu_bf(B0[o] + W0[3 * o] * f0 + W0[3 * o + 1] * f1 + W0[3 * o + 2] * f2);
                const float v1 = silu_bf(B0[o + 1] + W0[3 * o + 3] * f0 + W0[3 * o + 4] * f1 + W0[3 * o + 5] * f2);
                pk[h] = pack_bf16(v0, v1);
            }
            *reinterpret_cast<uint4*>(A + tcu::sw128_offset(t, c)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        }
        float o0 = B4[0], o1 = B4[1];
        bool ok = true;
#pragma unroll 1
        for (int l = 0; l < 3; ++l) {
            tcu::fence_proxy_async();
            tcu::fence_before();
            __syncthreads();
            tcu::fence_after();
            if (t == 0) {
#pragma unroll
                for (int ks = 0; ks < 4; ++ks)
                    tcu::mma_bf16(tmem, tcu::sw128_desc(a_addr + 32 * ks),
                                  tcu::sw128_desc(w_addr + l * 8192 + 32 * ks), idesc, ks > 0);
                tcu::mma_commit(bar);
            }
            __syncwarp();
            ok = __all_sync(0xffffffffu, tcu::mbar_wait_poll(bar, phase, err, 5)) && ok;
            phase ^= 1u;
            tcu::fence_after();
            const float* bl = B0 + 64 * (l + 1);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float h[16];
                if (ok) tcu::tmem_ld16(lane_addr + 16 * q, h);
                else {
#pragma unroll
                    for (int i = 0; i < 16; ++i) h[i] = 0.f;
                }
                if (l < 2) {
#pragma unroll
                    for (int cc = 0; cc < 2; ++cc) {
                        const int c = 2 * q + cc;
                        const float* hv = h + 8 * cc;
                        const float* bb = bl + 8 * c;
                        const uint4 v = make_uint4(
                            pack_bf16(silu_bf(hv[0] + bb[0]), silu_bf(hv[1] + bb[1])),
                            pack_bf16(silu_bf(hv[2] + bb[2]), silu_bf(hv[3] + bb[3])),
                            pack_bf16(silu_bf(hv[4] + bb[4]), silu_bf(hv[5] + bb[5])),
                            pack_bf16(silu_bf(hv[6] + bb[6]), silu_bf(hv[7] + bb[7])));
                        *reinterpret_cast<uint4*>(A + tcu::sw128_offset(t, c)) = v;
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < 16; ++i) {
                        const float a = silu_acc(h[i] + bl[16 * q + i]);
                        o0 = fmaf(W4[16 * q + i], a, o0);
                        o1 = fmaf(W4[64 + 16 * q + i], a, o1);
                    }
                }
            }
        }
        if (valid) {
            if (raw) raw[idx] = make_float2(o0, o1);
            if (guess) guess[idx] = inside ? (float)(o0 / kPinetOutScale) : 0.f;
        }
    }
    tcu::fence_before();
    __syncthreads();
    if (warp == 0) tcu::tmem_dealloc(tmem, 64);
}

// ---- fast voxel-mode inference ---------------------------------------------------------------
// shared memory (offsets from a 1024-byte aligned base)
constexpr int kVsA = 0;                 // activation tile 128 x 128 B
constexpr int kVsW = 16384;             // hidden weight tiles, 3 x 64 x 128 B
constexpr int kVsO = kVsW + 3 * 8192;   // output weight tile 16 x 128 B (rows 0, 1 = W4)
constexpr int kVsP0 = kVsO + 2048;      // layer 0: 64 x float4 {w0, w1, w2, b} / 2
constexpr int kVsPB = kVsP0 + 1024;     // hidden biases / 2 as BF16 pairs, 3 x 32 x 4 B
constexpr int kVsBar = kVsPB + 384;
constexpr int kVsSlot = kVsBar + 8;
constexpr int kVsBytes = kVsSlot + 8 + 1024;
constexpr int kVsPerSM = 233472 / (kVsBytes + 1024) < 8 ? 233472 / (kVsBytes + 1024) : 8;

__device__ __forceinline__ uint32_t bf16x2_cut(float a, float b) {  // upper halves of a, b
    uint32_t x;
    asm("prmt.b32 %0, %1, %2, 0x7632;" : "=r"(x) : "r"(__float_as_uint(a)), "r"(__float_as_uint(b)));
    return x;
}
// y = h tanh(h) + h = SiLU(2h) for a BF16 pair h
__device__ __forceinline__ uint32_t silu2_half(uint32_t h) {
    uint32_t t, y;
    asm("tanh.approx.bf16x2 %0, %1;" : "=r"(t) : "r"(h));
    asm("fma.rn.bf16x2 %0, %1, %2, %1;" : "=r"(y) : "r"(h), "r"(t));
    return y;
}
__device__ __forceinline__ uint32_t hfma2(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t d;
    asm("fma.rn.bf16x2 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}

__global__ void __launch_bounds__(kT)
k_pinet_voxels(BPParams kp, const unsigned char* __restrict__ net, long long n_items,
               float* __restrict__ guess, int* __restrict__ err) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* sm = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* A = sm + kVsA;
    uint8_t* Wt = sm + kVsW;
    uint8_t* Wo = sm + kVsO;
    float4* P0 = reinterpret_cast<float4*>(sm + kVsP0);
    uint32_t* PB = reinterpret_cast<uint32_t*>(sm + kVsPB);
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kVsBar);
    uint32_t* slot = reinterpret_cast<uint32_t*>(sm + kVsSlot);
    const int t = threadIdx.x, warp = t >> 5;

    const uint4* src = reinterpret_cast<const uint4*>(net);
    for (int q = t; q < 3 * 64 * 8; q += kT) {
        const int l = q >> 9, r = (q >> 3) & 63, c = q & 7;
        *reinterpret_cast<uint4*>(Wt + l * 8192 + tcu::sw128_offset(r, c)) = src[q];
    }
    const float* fsrc = reinterpret_cast<const float*>(net + kNetBf16Bytes);
    // output tile: row n < 2 = W4[n][0..63] in BF16, rows 2..15 zero
    for (int q = t; q < 16 * 8; q += kT) {
        const int r = q >> 3, c = q & 7;
        uint32_t w[4] = {0, 0, 0, 0};
        if (r < 2)
            for (int k = 0; k < 4; ++k)
                w[k] = pack_bf16(fsrc[kNetF32_W4 + 64 * r + 8 * c + 2 * k],
                                 fsrc[kNetF32_W4 + 64 * r + 8 * c + 2 * k + 1]);
        *reinterpret_cast<uint4*>(Wo + tcu::sw128_offset(r, c)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    // layer 0 halved and scaled by 1 + 2^-9, so that cutting its pre-activations to BF16
    // rounds to nearest on average
    constexpr float kHalfUp = 0.5f * (1.0f + 1.0f / 512.0f);
    for (int q = t; q < 64; q += kT) {
        const float* w = fsrc + kNetF32_W0 + 3 * q;
        P0[q] = make_float4(kHalfUp * w[0], kHalfUp * w[1], kHalfUp * w[2],
                            kHalfUp * fsrc[kNetF32_B0 + q]);
    }
    for (int q = t; q < 96; q += kT) {
        const float* b = fsrc + kNetF32_B0 + 64 + 2 * q;
        PB[q] = pack_bf16(0.5f * b[0], 0.5f * b[1]);
    }
    const float b4 = fsrc[kNetF32_B4];
    if (t == 0) {
        tcu::mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tcu::tmem_alloc(slot, 64);
    tcu::fence_proxy_async();
    tcu::fence_before();
    __syncthreads();
    tcu::fence_after();
    const uint32_t tmem = *slot;
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
    const uint32_t idesc = tcu::idesc_bf16_f32(128, 64), idesc_o = tcu::idesc_bf16_f32(128, 16);
    const uint32_t a_addr = tcu::smem_u32(A), w_addr = tcu::smem_u32(Wt), o_addr = tcu::smem_u32(Wo);
    const uint32_t half2 = 0x3F003F00u;  // (0.5, 0.5)
    uint32_t phase = 0;
    const long long ntiles = (n_items + kT - 1) / kT;
    const float XC = (float)kp.XC, YC = (float)kp.YC, ZC = (float)kp.ZC;
    const float dx = (float)kp.dx, dy = (float)kp.dy, dz = (float)kp.dz;
    const float iR = (float)(1.0 / kp.ScanR), iH = (float)(1.0 / kp.HelicP);
    bool ok = true;

    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long long idx = tile * kT + t;
        const bool valid = idx < n_items;
        float f0 = 0.f, f1 = 1.f, f2 = 0.f;
        bool inside = false;
        if (valid) {
            // the volume has fewer than 2^31 voxels (ctrecon_bp_geom checks)
            const int ii = (int)idx;
            const int zi = ii % kp.NZ, xy = ii / kp.NZ;
            const int yi = xy % kp.NY, xi = xy / kp.NY;
            const double Xd = (xi - kp.XC) * kp.dx, Yd = (yi - kp.YC) * kp.dy;
            inside = Xd * Xd + Yd * Yd < kp.ObjR2;  // KatsevichBkProj.cpp:168
            const float x = ((float)xi - XC) * dx * iR, y = ((float)yi - YC) * dy * iR;
            const float z = ((float)zi - ZC) * dz * iH;
            const float r = sqrtf(x * x + y * y);
            float s2, c2;
            sincospif(2.f * (z - rintf(z)), &s2, &c2);
            const float ir = r > 0.f ? 1.f / r : 0.f;
            const float cph = r > 0.f ? x * ir : 1.f, sph = y * ir;
            f0 = r * (float)kPinetRInv;
            f1 = cph * c2 + sph * s2;  // cos(phi - 2 pi z)
            f2 = sph * c2 - cph * s2;  // sin(phi - 2 pi z)
        }
        // layer 0 (FP32, halved): h = (w . f + b) / 2 cut to BF16, SiLU(2h)
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            uint32_t pk[4];
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                const float4 p = P0[c * 8 + 2 * h], q = P0[c * 8 + 2 * h + 1];
                pk[h] = silu2_half(bf16x2_cut(fmaf(p.z, f2, fmaf(p.y, f1, fmaf(p.x, f0, p.w))),
                                              fmaf(q.z, f2, fmaf(q.y, f1, fmaf(q.x, f0, q.w)))));
            }
            *reinterpret_cast<uint4*>(A + tcu::sw128_offset(t, c)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        }
        // hidden layers 1..3 on the tensor core, then the output layer (N = 16, column 0 = sb)
#pragma unroll 1
        for (int l = 0; l < 4; ++l) {
            tcu::fence_proxy_async();
            tcu::fence_before();
            __syncthreads();
            tcu::fence_after();
            if (t == 0) {
#pragma unroll
                for (int ks = 0; ks < 4; ++ks)
                    tcu::mma_bf16(tmem, tcu::sw128_desc(a_addr + 32 * ks),
                                  tcu::sw128_desc((l < 3 ? w_addr + l * 8192 : o_addr) + 32 * ks),
                                  l < 3 ? idesc : idesc_o, ks > 0);
                tcu::mma_commit(bar);
            }
            __syncwarp();
            ok = __all_sync(0xffffffffu, tcu::mbar_wait_poll(bar, phase, err, 5)) && ok;
            phase ^= 1u;
            tcu::fence_after();
            if (l == 3) {
                float h[16];
                if (ok) tcu::tmem_ld16(lane_addr, h);
                else h[0] = 0.f;
                if (valid) guess[idx] = inside ? (h[0] + b4) / (float)kPinetOutScale : 0.f;
                break;
            }
            const uint32_t* pb = PB + 32 * l;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float h[16];
                if (ok) tcu::tmem_ld16(lane_addr + 16 * q, h);
                else {
#pragma unroll
                    for (int i = 0; i < 16; ++i) h[i] = 0.f;
                }
#pragma unroll
                for (int cc = 0; cc < 2; ++cc) {
                    const int c = 2 * q + cc;
                    const float* hv = h + 8 * cc;
                    const uint4 bb = *reinterpret_cast<const uint4*>(pb + 4 * c);
                    const uint4 v = make_uint4(
                        silu2_half(hfma2(bf16x2_cut(hv[0], hv[1]), half2, bb.x)),
                        silu2_half(hfma2(bf16x2_cut(hv[2], hv[3]), half2, bb.y)),
                        silu2_half(hfma2(bf16x2_cut(hv[4], hv[5]), half2, bb.z)),
                        silu2_half(hfma2(bf16x2_cut(hv[6], hv[7]), half2, bb.w)));
                    *reinterpret_cast<uint4*>(A + tcu::sw128_offset(t, c)) = v;
                }
            }
        }
    }
    tcu::fence_before();
    __syncthreads();
    if (warp == 0) tcu::tmem_dealloc(tmem, 64);
}

// CTAs per SM of k_pinet_infer: as many as the shared memory holds (1 KB reserved per CTA), at
// most 8 (TMEM: 64 columns each)
int persistent_blocks() {
    constexpr int per_sm = 233472 / (kSmBytes + 1024) < 8 ? 233472 / (kSmBytes + 1024) : 8;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms * per_sm;
}

}  // namespace

Status pinet_prepare(ctrecon_ctx* ctx, cudaStream_t s) {
    PinetState& P = ctx->pinet;
    if (!P.trained)
        return make_status(CTRECON_ERR_INVALID_ARGUMENT,
                           "the PI-line network is not trained (ctrecon_pinet_train or "
                           "ctrecon_pinet_set_params first)");
    if (P.infer_version == P.version && P.infer.ptr) return Status::Ok();
    CTR_TRY(P.infer.ensure(kNetBytes, "network inference copy"));
    k_net_prep<<<(3 * 4096 + 255) / 256, 256, 0, s>>>(P.theta.as<float>(), P.infer.as<unsigned char>());
    CTR_CUDA(cudaGetLastError());
    P.infer_version = P.version;
    return Status::Ok();
}

static Status launch_infer(ctrecon_ctx* ctx, cudaStream_t s, const BPParams& kp, long long n,
                           const float* feat, float2* raw, float* guess) {
    CTR_TRY(pinet_prepare(ctx, s));
    if (!ctx->ws_flag.ptr) return make_status(CTRECON_ERR_INTERNAL, "device error word not set up");
    const long long ntiles = (n + kT - 1) / kT;
    if (!feat && ctx->opt_pinet_mode == CTRECON_PINET_VOXEL_BF16) {
        CTR_CUDA(cudaFuncSetAttribute(k_pinet_voxels, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      kVsBytes));
        int dev = 0, sms = 148;
        CTR_CUDA(cudaGetDevice(&dev));
        CTR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        const int grid = (int)std::min<long long>(ntiles, (long long)sms * kVsPerSM);
        if (grid <= 0) return Status::Ok();
        k_pinet_voxels<<<grid, kT, kVsBytes, s>>>(kp, ctx->pinet.infer.as<unsigned char>(), n,
                                                  guess, ctx->ws_flag.as<int>());
        CTR_CUDA(cudaGetLastError());
        return Status::Ok();
    }
    CTR_CUDA(cudaFuncSetAttribute(k_pinet_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmBytes));
    const int grid = (int)std::min<long long>(ntiles, persistent_blocks());
    if (grid <= 0) return Status::Ok();
    k_pinet_infer<<<grid, kT, kSmBytes, s>>>(kp, ctx->pinet.infer.as<unsigned char>(), n, feat,
                                             raw, guess, ctx->ws_flag.as<int>());
    CTR_CUDA(cudaGetLastError());
    return Status::Ok();
}

// features of the (r, psi) grid: r = i r_max / (nr - 1) (normalised by ScanR), psi = 2 pi j / np
__global__ void k_grid_feat(float* __restrict__ feat, int nr, int np, double r_max) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nr * np) return;
    const int i = q / np, j = q % np;
    double sp, cp;
    sincospi(2.0 * j / np, &sp, &cp);
    feat[3 * q] = (float)(r_max * i / (nr - 1) * kPinetRInv);
    feat[3 * q + 1] = (float)cp;
    feat[3 * q + 2] = (float)sp;
}

// The network's predictions at the grid points refined by the FP64 Newton solve (pi_device.cuh)
// of the grid point itself, (x, y, z) = r (cos psi, sin psi) / ScanR at z = 0, from the network's
// start: by the screw symmetry of the PI lines (a turn of the helix by psi lifts every chord by
// psi / 2 pi) each voxel's interpolated start is then within the grid's interpolation error of its
// root (~3e-7 rad on this grid), under the 1e-6 rad at which Newton accepts a step, so a voxel's
// solve takes one Newton evaluation before the replayed bisection; the grid points whose Newton
// solve does not converge keep the network's prediction.
__global__ void k_grid_refine(float2* __restrict__ out, int nr, int np, double r_max) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nr * np) return;
    const int i = q / np, j = q % np;
    double sp, cp;
    sincospi(2.0 * j / np, &sp, &cp);
    const double r = r_max * i / (nr - 1);
    const float2 o = out[q];
    double sb, st;
    int it = 0;
    bool conv = false;
    pi_newton(r * cp, r * sp, 0.0, (double)o.x / kPinetOutScale - 0.5 * kRefPi, &sb, &st, &it,
              nullptr, &conv);
    if (conv)
        out[q] = make_float2((float)((sb + 0.5 * kRefPi) * kPinetOutScale),
                             (float)((st - 0.5 * kRefPi) * kPinetOutScale));
}

constexpr int kGridNR = 256, kGridNP = 4096;

Status launch_pi_learned(ctrecon_ctx* ctx, cudaStream_t s, BPPlan& plan, PiRecord* d_pitab,
                         unsigned long long* d_updates, unsigned long long* d_iters) {
    const long long n = (long long)plan.kp.NX * plan.kp.NY * plan.kp.NZ;
    if (ctx->opt_pinet_mode == CTRECON_PINET_GRID) {
        // the network once per grid point (FP32 SiLU, feature mode), then the Newton solve
        // interpolates its outputs; r up to the cylinder's radius
        const int ng = kGridNR * kGridNP;
        const double r_max = plan.g.ObjR / plan.g.ScanR;
        CTR_TRY(ctx->pinet.grid_feat.ensure((size_t)ng * 3 * sizeof(float), "network grid features"));
        CTR_TRY(ctx->pinet.grid_out.ensure((size_t)ng * sizeof(float2), "network grid outputs"));
        k_grid_feat<<<(ng + 255) / 256, 256, 0, s>>>(ctx->pinet.grid_feat.as<float>(), kGridNR,
                                                     kGridNP, r_max);
        CTR_CUDA(cudaGetLastError());
        CTR_TRY(launch_infer(ctx, s, plan.kp, ng, ctx->pinet.grid_feat.as<float>(),
                             ctx->pinet.grid_out.as<float2>(), nullptr));
        k_grid_refine<<<(ng + 127) / 128, 128, 0, s>>>(ctx->pinet.grid_out.as<float2>(), kGridNR,
                                                       kGridNP, r_max);
        CTR_CUDA(cudaGetLastError());
        return launch_pi_guess(ctx, s, plan, d_pitab, d_updates, d_iters, nullptr,
                               ctx->pinet.grid_out.ptr, kGridNR, kGridNP, r_max);
    }
    CTR_TRY(ctx->pinet.guess.ensure((size_t)n * sizeof(float), "learned PI guesses"));
    float* g = ctx->pinet.guess.as<float>();
    CTR_TRY(launch_infer(ctx, s, plan.kp, n, nullptr, nullptr, g));
    return launch_pi_guess(ctx, s, plan, d_pitab, d_updates, d_iters, g, nullptr, 0, 0, 0.0);
}

Status pinet_predict(ctrecon_ctx* ctx, cudaStream_t s, const float* d_feat, long long n,
                     float* d_out) {
    BPParams kp{};
    return launch_infer(ctx, s, kp, n, d_feat, reinterpret_cast<float2*>(d_out), nullptr);
}

}  // namespace ctr
