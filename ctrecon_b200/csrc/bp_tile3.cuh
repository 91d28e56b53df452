// bp_tile3.cuh -- the third form of the voxel-driven backprojection tile
// (KatsevichBkProj.cpp:164-265; FP32 interpolation and accumulation, the reference's endpoint
// rule), built so that an update costs about a dozen instructions:
//
//  * Cell records. Every detector cell (r, c) of a view's footprint is stored once per tile as a
//    16-byte record {A, B, C, D} of its four corner taps t00 = F[r][c], t01 = F[r][c+1],
//    t10 = F[r+1][c], t11 = F[r+1][c+1]:
//        A = (t00 + t01 + t10 + t11) / 4,    B = ((t01 - t00) + (t11 - t10)) / 2,
//        C = ((t10 - t00) + (t11 - t01)) / 2, D = (t11 - t10) - (t01 - t00),
//    so that the bilinear value at fractions (alpha, beta) is, with a = alpha - 1/2 and
//    b = beta - 1/2, A + a B + b (C + a D): one 16-byte shared load and three FMAs.
//  * Floor by rounding. u - 1/2 + 1.5 * 2^23 rounds to floor(u) (exact integers may round to
//    u - 1 with a = +1/2, the same bilinear value), and the cell index comes straight from the
//    bits of that sum: no conversions, no clamps. This is valid because a view takes the cell
//    path only when the tile's whole footprint (one cell of margin) lies inside the detector,
//    where the reference's reads and the clamped reads agree.
//  * Staging: raw footprint rows are copied with cp.async into a double buffer while the
//    previous block of views is accumulated; the cell records of a block are built from the
//    raw rows in shared memory (a few instructions per cell against ~2000 updates per view).
//  * A warp whose voxels all lie strictly inside their PI intervals for a whole block of views
//    (unit weights) takes a branch-free loop; the others apply the endpoint rule per voxel. Views
//    whose footprint is too large or reaches the detector border read FProj directly with the
//    clamped indices of the first form.
#pragma once

#include "bp_common.cuh"

namespace ctr {
namespace bp {

constexpr int kCapR3 = 640;  // raw footprint floats per staged view
constexpr int kCapQ3 = 512;  // cell records per staged view
constexpr float kMagic = 12582912.0f;         // 1.5 * 2^23
constexpr int kMagicBits = 0x4B400000;        // its bit pattern

// Footprint of one view over a tile: cells [u0, u0 + W - 1) x [v0, v0 + H - 1).
// W > 0: cell path; W == -2: direct global reads; W == -1: empty slot (view past the range).
struct Foot3 { int u0, v0, W, H; };

template <int NB>
struct Shared3 {
    Foot3 foot[2][NB];
    float4 vg[2][NB];
    int cells[2];  // every view of the block takes the cell path
    int s_pmin, s_pmax, s_item;
};

template <int NB>
__host__ __device__ constexpr size_t tile3_smem_bytes() {
    return (size_t)NB * kCapQ3 * 16 + (size_t)2 * NB * kCapR3 * sizeof(float);
}

// One CTA tile: columns [16 bx, 16 bx + 16) x [16 by, 16 by + 16), slices [8 bz, 8 bz + 8).
// Called by all 256 threads; returns with no copies in flight.
template <int NB, typename OutT>
__device__ __forceinline__ void tile3(const BPParams& kp, const float* __restrict__ fproj,
                                      const PiRecord* __restrict__ pit,
                                      const float4* __restrict__ views,
                                      const float* __restrict__ xyz, OutT* __restrict__ image,
                                      int bx, int by, int bz, Shared3<NB>& sh,
                                      unsigned char* dyn) {
    constexpr int TZ = 8;
    float4* cellbuf = reinterpret_cast<float4*>(dyn);                 // NB * kCapQ3
    float* raw = reinterpret_cast<float*>(dyn + (size_t)NB * kCapQ3 * 16);  // 2 * NB * kCapR3
    const uint32_t cell_s = smem_addr(cellbuf);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int tx = tid & (kTXY - 1), ty = tid >> 4;
    const int x = bx * kTXY + tx, y = by * kTXY + ty;
    const int zb = bz * TZ;
    const int NX = kp.NX, NY = kp.NY, NZ = kp.NZ, P = kp.P, YL = kp.YL, ZL = kp.ZL;
    const bool col_ok = (x < NX) && (y < NY);
    const float* xc = xyz;
    const float* yc = xyz + NX;
    const float* zc = xyz + NX + NY;
    const float X = col_ok ? xc[x] : 0.f, Y = col_ok ? yc[y] : 0.f;
    const float z0 = zc[zb];
    const float dzf = kp.dzf;

    if (tid == 0) { sh.s_pmin = INT_MAX; sh.s_pmax = INT_MIN; }
    VoxelRanges<TZ> vr;
    const size_t colbase = ((size_t)x * NY + y) * NZ;
    load_ranges<TZ>(pit, colbase, zb, NZ, P, col_ok, kp.win0, kp.win1, vr);
    float acc[TZ];
#pragma unroll
    for (int k = 0; k < TZ; ++k) acc[k] = 0.f;
    int wmin = vr.tmin, wmax = vr.tmax;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        wmin = min(wmin, __shfl_xor_sync(0xffffffffu, wmin, o));
        wmax = max(wmax, __shfl_xor_sync(0xffffffffu, wmax, o));
    }
    __syncthreads();
    if (lane == 0 && wmin <= wmax) {
        atomicMin(&sh.s_pmin, wmin);
        atomicMax(&sh.s_pmax, wmax);
    }
    __syncthreads();
    const int pmin = sh.s_pmin, pmax = sh.s_pmax;
    if (pmin > pmax) return;

    const int x0 = bx * kTXY, x1 = min(x0 + kTXY, NX) - 1;
    const int y0 = by * kTXY, y1 = min(y0 + kTXY, NY) - 1;
    const int z1 = min(zb + TZ, NZ) - 1;
    const float bx0 = xc[x0], bx1 = xc[x1], by0 = yc[y0], by1 = yc[y1];
    const float bz0 = zc[zb], bz1 = zc[z1];
    const float R = kp.Rf, DdU = kp.DdU, DdV = kp.DdV, HalfY = kp.HalfY, HalfZ = kp.HalfZ;
    const float HalfYm = HalfY - 0.5f, HalfZm = HalfZ - 0.5f;

    // footprints of views [pb, pb + NB) into slot `buf`: warp 0, lane j -> view pb + j
    auto footprints = [&](int buf, int pb) {
        if (warp != 0) return;
        Foot3 f{0, 0, -1, 0};
        const int p = pb + lane;
        if (lane < NB && p <= pmax) {
            const float4 g = views[p];
            sh.vg[buf][lane] = g;
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
            f = Foot3{0, 0, -2, 0};
            // |u|, |v| < 2^20 keeps the integer conversions exact and the rounding trick valid
            if (ok && fabsf(umin) < 1048576.f && fabsf(umax) < 1048576.f &&
                fabsf(vmin) < 1048576.f && fabsf(vmax) < 1048576.f) {
                const int u0 = (int)floorf(umin) - 1, u1 = (int)floorf(umax) + 2;
                const int v0 = (int)floorf(vmin) - 1, v1 = (int)floorf(vmax) + 2;
                const int W = u1 - u0 + 1, H = v1 - v0 + 1;
                if (u0 >= 0 && u1 <= YL - 1 && v0 >= 0 && v1 <= ZL - 1 && W <= 64 &&
                    W * H <= kCapR3 && (W - 1) * (H - 1) <= kCapQ3)
                    f = Foot3{u0, v0, W, H};
            }
        }
        if (lane < NB) sh.foot[buf][lane] = f;
        const unsigned cellmask = __ballot_sync(0xffffffffu, lane >= NB || f.W > 0);
        if (lane == 0) sh.cells[buf] = (cellmask == 0xffffffffu);
    };
    // cp.async the raw footprint rows of slot `buf` (views from pb): warp per row
    auto stage = [&](int buf, int pb) {
#pragma unroll 1
        for (int j = 0; j < NB; ++j) {
            const Foot3 f = sh.foot[buf][j];
            if (f.W <= 0) continue;
            const float* src = fproj + ((size_t)(pb + j) * ZL + f.v0) * YL + f.u0;
            float* dst = raw + (buf * NB + j) * kCapR3;
            for (int r = warp; r < f.H; r += 8) {
                if (lane < f.W) cp_async4(dst + r * f.W + lane, src + (size_t)r * YL + lane);
                if (lane + 32 < f.W)
                    cp_async4(dst + r * f.W + lane + 32, src + (size_t)r * YL + lane + 32);
            }
        }
        cp_async_commit();
    };
    // cell records of slot `buf` from its raw rows
    auto build = [&](int buf) {
#pragma unroll 1
        for (int j = 0; j < NB; ++j) {
            const Foot3 f = sh.foot[buf][j];
            if (f.W <= 0) continue;
            const float* src = raw + (buf * NB + j) * kCapR3;
            float4* dst = cellbuf + j * kCapQ3;
            const int Wc = f.W - 1;
            for (int r = warp; r < f.H - 1; r += 8) {
                for (int c = lane; c < Wc; c += 32) {
                    const float* s0 = src + r * f.W + c;
                    const float t00 = s0[0], t01 = s0[1], t10 = s0[f.W], t11 = s0[f.W + 1];
                    const float h0 = t01 - t00, h1 = t11 - t10;
                    const float g0 = t10 - t00, g1 = t11 - t01;
                    dst[r * Wc + c] = make_float4(0.25f * ((t00 + t01) + (t10 + t11)),
                                                  0.5f * (h0 + h1), 0.5f * (g0 + g1), h1 - h0);
                }
            }
        }
    };

    footprints(0, pmin);
    __syncthreads();
    stage(0, pmin);
    int buf = 0;
#pragma unroll 1
    for (int pb = pmin; pb <= pmax; pb += NB, buf ^= 1) {
        const int pn = pb + NB;
        cp_async_wait<0>();
        __syncthreads();  // raw rows of this block landed; the previous block is finished
        footprints(buf ^ 1, pn);
        build(buf);
        __syncthreads();  // cell records and the next block's footprints are visible
        stage(buf ^ 1, pn);
        // warp-uniform: every lane's voxels are inside their intervals for the whole block
        // and every view takes the cell path
        const bool fast = __all_sync(0xffffffffu, vr.all_valid && pb >= vr.flo &&
                                                   pb + NB - 1 <= vr.fhi &&
                                                   pb + NB - 1 <= pmax && sh.cells[buf] != 0);
        if (!col_ok || wmin > wmax || pb + NB - 1 < wmin || pb > wmax) continue;
#pragma unroll 1
        for (int j = 0; j < NB; ++j) {
            const int p = pb + j;
            if (p > pmax) break;
            if (!fast && (p < vr.tmin || p > vr.tmax)) continue;
            const Foot3 f = sh.foot[buf][j];
            const float4 g = sh.vg[buf][j];
            const float fen = R - (X * g.x + Y * g.y);
            const float YY = Y * g.x - X * g.y;
            const float inv = rcp_approx(fen);
            const float kv = DdV * inv;
            const float r2 = fen * fen + YY * YY;
            const float dz0 = z0 - g.z;
            if (f.W > 0) {
                const float u = fmaf(YY * DdU, inv, HalfYm);  // u - 1/2
                const float tu = u + kMagic;
                const float a = u - (tu - kMagic);           // alpha - 1/2
                const uint32_t W16 = (uint32_t)(f.W - 1) * 16u;
                // byte address of cell (bits(tv) - kMagicBits - v0, bits(tu) - kMagicBits - u0)
                const uint32_t cbase =
                    cell_s + (uint32_t)(j * kCapQ3) * 16u +
                    ((uint32_t)__float_as_int(tu) - (uint32_t)(kMagicBits + f.u0)) * 16u -
                    (uint32_t)(kMagicBits + f.v0) * W16;
                if (fast) {
#pragma unroll
                    for (int k = 0; k < TZ; ++k) {
                        const float dz = fmaf((float)k, dzf, dz0);
                        const float v = fmaf(dz, kv, HalfZm);  // v - 1/2
                        const float rinv = rsqrt_approx(fmaf(dz, dz, r2));
                        const float tv = v + kMagic;
                        const float b = v - (tv - kMagic);
                        const float4 q = lds128((uint32_t)__float_as_int(tv) * W16 + cbase);
                        acc[k] = fmaf(fmaf(b, fmaf(a, q.w, q.z), fmaf(a, q.y, q.x)), rinv, acc[k]);
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < TZ; ++k) {
                        const int d0 = p - vr.bi[k];
                        const int d1 = vr.ti[k] + 1 - p;
                        if ((d0 | d1) < 0) continue;
                        float w = 1.f;
                        if (d1 <= 1) w = ramp(vr.tf[k] + (float)(d1 - 1));
                        else if (d0 <= 1) w = ramp((float)d0 - vr.bf[k]);
                        const float dz = fmaf((float)k, dzf, dz0);
                        const float v = fmaf(dz, kv, HalfZm);
                        const float rinv = rsqrt_approx(fmaf(dz, dz, r2));
                        const float tv = v + kMagic;
                        const float b = v - (tv - kMagic);
                        const float4 q = lds128((uint32_t)__float_as_int(tv) * W16 + cbase);
                        acc[k] = fmaf(w * fmaf(b, fmaf(a, q.w, q.z), fmaf(a, q.y, q.x)), rinv,
                                      acc[k]);
                    }
                }
            } else {
                // direct reads with the clamped indices of the first form
                const float u = YY * DdU * inv + HalfY;
                const int ui = max(0, min(YL - 2, __float2int_rd(u)));
                const float alfa = u - (float)ui;
                const float* base = fproj + (size_t)p * ZL * YL + ui;
#pragma unroll
                for (int k = 0; k < TZ; ++k) {
                    const int d0 = p - vr.bi[k];
                    const int d1 = vr.ti[k] + 1 - p;
                    if ((d0 | d1) < 0) continue;
                    float w = 1.f;
                    if (d1 <= 1) w = ramp(vr.tf[k] + (float)(d1 - 1));
                    else if (d0 <= 1) w = ramp((float)d0 - vr.bf[k]);
                    const float dz = fmaf((float)k, dzf, dz0);
                    const float v = fmaf(dz, kv, HalfZ);
                    const float rinv = rsqrt_approx(fmaf(dz, dz, r2));
                    const int vi = max(0, min(ZL - 2, __float2int_rd(v)));
                    const float beta = v - (float)vi;
                    const float* q = base + (size_t)vi * YL;
                    const float t00 = __ldg(q), t01 = __ldg(q + 1);
                    const float t10 = __ldg(q + YL), t11 = __ldg(q + YL + 1);
                    const float a0 = fmaf(alfa, t01 - t00, t00);
                    const float a1 = fmaf(alfa, t11 - t10, t10);
                    acc[k] = fmaf(w * fmaf(beta, a1 - a0, a0), rinv, acc[k]);
                }
            }
        }
    }
    cp_async_wait<0>();
    __syncthreads();  // no thread leaves while others may still read this tile's buffers
    if (!col_ok) return;
#pragma unroll
    for (int k = 0; k < TZ; ++k) {
        const int z = zb + k;
        if (z < NZ && vr.bi[k] != kPiInvalid) store_voxel(image + colbase + z, -acc[k] * kp.invPs, kp.accum);
    }
}

}  // namespace bp
}  // namespace ctr
