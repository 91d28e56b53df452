// bkproj2.cu -- K4, the tiled forms of the voxel-driven backprojection of bkproj.cu
// (KatsevichBkProj.cpp:164-265, FP32 interpolation and accumulation, identical endpoint rule).
//
// Second form (bp_tile below), reorganised for issue throughput:
//  * views are staged in blocks of NB with two shared-memory buffers: while block b is being
//    accumulated, block b+1's footprints are already in flight (cp.async, one warp per detector
//    row, no integer division), so each block costs three barriers instead of stalling on loads;
//  * a thread whose TZ voxels are all strictly inside their PI intervals (away from the two
//    ramp views at each end) for a whole block takes a branch-free path with unit weights --
//    the common case; the others take the checked path of bkproj.cu;
//  * voxel z coordinates are generated, not held in registers, and the launch is bounded to
//    three CTAs of 256 threads per SM.
// Third form (bp_tile3.cuh): per-cell bilinear records and a rounding floor that
// bring an update down to about a dozen instructions.
//
// Also the persistent batched kernel (either form) behind the batch API.
#include "bp_tile4.cuh"

#include <cudaTypedefs.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

namespace ctr {

namespace {

using namespace bp;
constexpr int kTXY2 = kTXY;
constexpr int kCap2 = 1024;  // shared floats per staged view

struct Foot2 { int u0, v0, W, H; };

}  // namespace

Caps4 caps_within(int cells, int raw, int NB, int S, size_t budget);
// dynamic shared memory per fourth-form CTA: three CTAs per SM with up to two producer warps,
// two with more
constexpr size_t smem4_budget(int PW) { return PW <= 2 ? 72 * 1024 : 104 * 1024; }

template <int NB>
struct BPShared {
    Foot2 foot[2][NB];
    float4 vg[2][NB];
    int s_pmin, s_pmax, s_item;
};

// One CTA tile: columns [16 bx, 16 bx + 16) x [16 by, 16 by + 16), slices [TZ bz, TZ bz + TZ).
// Called by all 256 threads of the CTA; returns with no copies in flight.
template <int TZ, int NB, typename OutT>
__device__ __forceinline__ void bp_tile(const BPParams& kp, const float* __restrict__ fproj,
                                        const PiRecord* __restrict__ pit,
                                        const float4* __restrict__ views,
                                        const float* __restrict__ xyz, OutT* __restrict__ image,
                                        int bx, int by, int bz, BPShared<NB>& sh, float* tile) {
    auto& foot = sh.foot;
    auto& vg = sh.vg;
    int& s_pmin = sh.s_pmin;
    int& s_pmax = sh.s_pmax;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int tx = tid & (kTXY2 - 1), ty = tid >> 4;
    const int x = bx * kTXY2 + tx, y = by * kTXY2 + ty;
    const int zb = bz * TZ;
    const int NX = kp.NX, NY = kp.NY, NZ = kp.NZ, P = kp.P, YL = kp.YL, ZL = kp.ZL;
    const bool col_ok = (x < NX) && (y < NY);
    const float* xc = xyz;
    const float* yc = xyz + NX;
    const float* zc = xyz + NX + NY;
    const float X = col_ok ? xc[x] : 0.f, Y = col_ok ? yc[y] : 0.f;
    const float z0 = zc[zb];
    const float dzf = kp.dzf;

    if (tid == 0) { s_pmin = INT_MAX; s_pmax = INT_MIN; }

    int bi[TZ], ti[TZ];
    float bf[TZ], tf[TZ], acc[TZ];
    int tmin = INT_MAX, tmax = INT_MIN, flo = INT_MIN, fhi = INT_MAX;
    bool all_valid = col_ok;
    const size_t colbase = ((size_t)x * NY + y) * NZ;
#pragma unroll
    for (int k = 0; k < TZ; ++k) {
        const int z = zb + k;
        PiRecord r{kPiInvalid, 0.f, -10, 0.f};
        if (col_ok && z < NZ) r = pit[colbase + z];
        bi[k] = r.bi; bf[k] = r.bf; ti[k] = r.ti; tf[k] = r.tf;
        acc[k] = 0.f;
        if (r.bi != kPiInvalid) {
            tmin = min(tmin, max(max(1, r.bi), kp.win0));
            tmax = max(tmax, min(min(r.ti + 1, P - 2), kp.win1));
            flo = max(flo, r.bi + 2);  // views past both B-side ramp views
            fhi = min(fhi, r.ti - 1);  // views before both T-side ramp views
        } else {
            all_valid = false;
        }
    }
    int wmin = tmin, wmax = tmax;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        wmin = min(wmin, __shfl_xor_sync(0xffffffffu, wmin, o));
        wmax = max(wmax, __shfl_xor_sync(0xffffffffu, wmax, o));
    }
    __syncthreads();
    if (lane == 0 && wmin <= wmax) {
        atomicMin(&s_pmin, wmin);
        atomicMax(&s_pmax, wmax);
    }
    __syncthreads();
    const int pmin = s_pmin, pmax = s_pmax;
    if (pmin > pmax) return;

    const int x0 = bx * kTXY2, x1 = min(x0 + kTXY2, NX) - 1;
    const int y0 = by * kTXY2, y1 = min(y0 + kTXY2, NY) - 1;
    const int z1 = min(zb + TZ, NZ) - 1;
    const float bx0 = xc[x0], bx1 = xc[x1], by0 = yc[y0], by1 = yc[y1];
    const float bz0 = zc[zb], bz1 = zc[z1];
    const float R = kp.Rf, DdU = kp.DdU, DdV = kp.DdV, HalfY = kp.HalfY, HalfZ = kp.HalfZ;

    // footprint of view p for buffer slot j (one thread per view)
    auto footprint = [&](int buf, int j, int p) {
        Foot2 f{0, 0, -1, 0};
        if (p <= pmax) {
            const float4 g = views[p];
            vg[buf][j] = g;
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
            f = Foot2{0, 0, -2, 0};  // direct global reads unless the footprint fits
            if (ok) {
                const int u0 = max(0, min(YL - 2, (int)floorf(umin) - 1));
                const int u1 = max(0, min(YL - 2, (int)floorf(umax) + 1)) + 1;
                const int v0 = max(0, min(ZL - 2, (int)floorf(vmin) - 1));
                const int v1 = max(0, min(ZL - 2, (int)floorf(vmax) + 1)) + 1;
                const int W = u1 - u0 + 1, H = v1 - v0 + 1;
                if (W * H <= kCap2 && W <= 64) f = Foot2{u0, v0, W, H};
            }
        }
        foot[buf][j] = f;
    };
    // cp.async the footprints of buffer `buf` (block starting at view pb): warp per row
    auto stage = [&](int buf, int pb) {
#pragma unroll 1
        for (int j = 0; j < NB; ++j) {
            const Foot2 f = foot[buf][j];
            if (f.W <= 0) continue;
            const float* src = fproj + ((size_t)(pb + j) * ZL + f.v0) * YL + f.u0;
            float* dst = tile + (buf * NB + j) * kCap2;
            for (int r = warp; r < f.H; r += 8) {
                if (lane < f.W) cp_async4(dst + r * f.W + lane, src + (size_t)r * YL + lane);
                if (lane + 32 < f.W) cp_async4(dst + r * f.W + lane + 32, src + (size_t)r * YL + lane + 32);
            }
        }
        cp_async_commit();
    };

    if (tid < NB) footprint(0, tid, pmin + tid);
    __syncthreads();
    stage(0, pmin);
    int buf = 0;
#pragma unroll 1
    for (int pb = pmin; pb <= pmax; pb += NB, buf ^= 1) {
        const int pn = pb + NB;
        if (tid < NB) footprint(buf ^ 1, tid, pn + tid);  // empty slots when pn > pmax
        __syncthreads();
        stage(buf ^ 1, pn);
        cp_async_wait<1>();
        __syncthreads();
        // warp-uniform: every lane's voxels are all inside their intervals for the block
        const bool fast = __all_sync(0xffffffffu, all_valid && pb >= flo &&
                                                   pb + NB - 1 <= fhi && pb + NB - 1 <= pmax);
        if (col_ok && wmin <= wmax && !(pb + NB - 1 < wmin || pb > wmax)) {
#pragma unroll 1
            for (int j = 0; j < NB; ++j) {
                const int p = pb + j;
                if (p > pmax) break;
                if (!fast && (p < tmin || p > tmax)) continue;
                const Foot2 f = foot[buf][j];
                const float4 g = vg[buf][j];
                const float fen = R - (X * g.x + Y * g.y);
                const float YY = Y * g.x - X * g.y;
                const float inv = rcp_approx(fen);
                const float u = YY * DdU * inv + HalfY;
                const float kv = DdV * inv;
                const float r2 = fen * fen + YY * YY;
                const int ui = max(0, min(YL - 2, __float2int_rd(u)));
                const float alfa = u - (float)ui;
                const bool smem = f.W > 0;
                // staged taps: 32-bit index into the shared tile (row stride W)
                const int W = f.W;
                const int tb = (buf * NB + j) * kCap2 + (ui - f.u0) - f.v0 * W;
                const float* base;
                int stride;
                if (smem) {
                    base = tile + tb;
                    stride = W;
                } else {
                    base = fproj + (size_t)p * ZL * YL + ui;
                    stride = YL;
                }
                const float dz0 = z0 - g.z;
                if (fast && smem) {
#pragma unroll
                    for (int k = 0; k < TZ; ++k) {
                        const float dz = fmaf((float)k, dzf, dz0);
                        const float v = fmaf(dz, kv, HalfZ);
                        const float rinv = rsqrt_approx(fmaf(dz, dz, r2));
                        const int vi = max(0, min(ZL - 2, __float2int_rd(v)));
                        const float beta = v - (float)vi;
                        const int i0 = tb + vi * W;
                        const int i1 = i0 + W;
                        const float t00 = tile[i0], t01 = tile[i0 + 1];
                        const float t10 = tile[i1], t11 = tile[i1 + 1];
                        const float a0 = fmaf(alfa, t01 - t00, t00);
                        const float a1 = fmaf(alfa, t11 - t10, t10);
                        acc[k] = fmaf(fmaf(beta, a1 - a0, a0), rinv, acc[k]);
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < TZ; ++k) {
                        const int d0 = p - bi[k];
                        const int d1 = ti[k] + 1 - p;
                        if ((d0 | d1) < 0) continue;
                        float w = 1.f;
                        if (d1 <= 1) w = ramp(tf[k] + (float)(d1 - 1));
                        else if (d0 <= 1) w = ramp((float)d0 - bf[k]);
                        const float dz = fmaf((float)k, dzf, dz0);
                        const float v = fmaf(dz, kv, HalfZ);
                        const float rinv = rsqrt_approx(fmaf(dz, dz, r2));
                        const int vi = max(0, min(ZL - 2, __float2int_rd(v)));
                        const float beta = v - (float)vi;
                        const float* q = base + vi * stride;
                        float t00, t01, t10, t11;
                        if (smem) {
                            const int i0 = tb + vi * W, i1 = i0 + W;
                            t00 = tile[i0]; t01 = tile[i0 + 1]; t10 = tile[i1]; t11 = tile[i1 + 1];
                        } else {
                            t00 = __ldg(q); t01 = __ldg(q + 1); t10 = __ldg(q + stride);
                            t11 = __ldg(q + stride + 1);
                        }
                        const float a0 = fmaf(alfa, t01 - t00, t00);
                        const float a1 = fmaf(alfa, t11 - t10, t10);
                        acc[k] = fmaf(w * fmaf(beta, a1 - a0, a0), rinv, acc[k]);
                    }
                }
            }
        }
        __syncthreads();  // buffer `buf` is free for the block after next
    }
    cp_async_wait<0>();
    if (!col_ok) return;
#pragma unroll
    for (int k = 0; k < TZ; ++k) {
        const int z = zb + k;
        if (z < NZ && bi[k] != kPiInvalid) {
            OutT* o = image + colbase + z;
            const OutT v = (OutT)(-acc[k] * kp.invPs);
            *o = kp.accum ? *o + v : v;
        }
    }
}

template <int TZ, int NB, typename OutT>
__global__ void __launch_bounds__(256, 3)
k_bkproj2(BPParams kp, const float* __restrict__ fproj, const PiRecord* __restrict__ pit,
          const float4* __restrict__ views, const float* __restrict__ xyz,
          OutT* __restrict__ image) {
    extern __shared__ float tile[];  // 2 x NB x kCap2
    __shared__ BPShared<NB> sh;
    bp_tile<TZ, NB, OutT>(kp, fproj, pit, views, xyz, image, blockIdx.x, blockIdx.y, blockIdx.z,
                          sh, tile);
}

template <int NB, typename OutT>
__global__ void __launch_bounds__(256, 3)
k_bkproj3(BPParams kp, const float* __restrict__ fproj, const PiRecord* __restrict__ pit,
          const float4* __restrict__ views, const float* __restrict__ xyz,
          OutT* __restrict__ image) {
    extern __shared__ __align__(16) unsigned char dyn3[];
    __shared__ Shared3<NB> sh;
    tile3<NB, OutT>(kp, fproj, pit, views, xyz, image, blockIdx.x, blockIdx.y, blockIdx.z, sh,
                    dyn3);
}

template <int NB, int S, int PW, typename OutT>
__global__ void __launch_bounds__(32 * (8 + PW), PW <= 2 ? 3 : 2)
k_bkproj4(BPParams kp, const float* __restrict__ fproj, const PiRecord* __restrict__ pit,
          const float4* __restrict__ views, const float* __restrict__ xyz,
          OutT* __restrict__ image, Caps4 caps, int* err) {
    extern __shared__ __align__(16) unsigned char dyn4[];
    __shared__ Shared4<NB, S, PW> sh;
    tile4_init(sh);
    tile4<NB, S, PW, false, OutT>(kp, fproj, pit, views, xyz, image, blockIdx.x, blockIdx.y,
                                  blockIdx.z, sh, dyn4, caps, err, 0u);
}

// Fifth form: the fourth form's consumers fed from the global cell records (k_cell_records) by
// one producer warp, one tensor copy per view (tmaps: the box table of bp_tile4.cuh).
// Paired (FP32x2) slice updates in the fifth form: measured 5% faster with blocks of 8 views
// and two CTAs per SM (96 registers); slower with 4-view blocks, and with three CTAs per SM
// (72 registers) the extra registers spill.
__host__ __device__ constexpr bool pair_slices5(int nb, int minb) { return nb >= 8 && minb < 3; }

template <int NB, int S, int MINB, typename OutT>
__global__ void __launch_bounds__(32 * 9, MINB)
k_bkproj5(BPParams kp, const float* __restrict__ fproj, const PiRecord* __restrict__ pit,
          const float4* __restrict__ views, const float* __restrict__ xyz,
          OutT* __restrict__ image, Caps4 caps, int* err, const CUtensorMap* __restrict__ tmaps,
          int rec_p0) {
    extern __shared__ __align__(128) unsigned char dyn5[];
    __shared__ Shared4<NB, S, 1> sh;
    tile4_init(sh);
    tile4<NB, S, 1, true, OutT, pair_slices5(NB, MINB)>(kp, fproj, pit, views, xyz, image,
                                                        blockIdx.x, blockIdx.y, blockIdx.z, sh,
                                                        dyn5, caps, err, 0u, tmaps, rec_p0);
}

// The cell records of views [p0, p0 + nviews): rec[v][r][c] = cell_record of the samples
// (r, c) .. (r + 1, c + 1) of view p0 + v, (ZL - 1) x (YL - 1) cells per view. A thread makes
// the records of kRecRows rows of one column: all its loads are in flight at once (one cell per
// thread was bound by the latency of its dependent loads), every sample row is read once, and
// each store of a warp is 512 contiguous bytes.
constexpr int kRecRows = 8;
__global__ void __launch_bounds__(128) k_cell_records(const float* __restrict__ fproj,
                                                      float4* __restrict__ rec, int p0,
                                                      int nviews, int YL, int ZL) {
    const int RW = YL - 1, RH = ZL - 1;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r0 = blockIdx.y * kRecRows;
    if (c >= RW) return;
    const int nr = min(kRecRows, RH - r0);  // rows of records here; samples r0 .. r0 + nr
    for (int v = blockIdx.z; v < nviews; v += gridDim.z) {
        const float* t = fproj + ((size_t)(p0 + v) * ZL + r0) * YL + c;
        float s0[kRecRows + 1], s1[kRecRows + 1];
#pragma unroll
        for (int i = 0; i <= kRecRows; ++i) {
            if (i <= nr) {
                s0[i] = __ldg(t + (size_t)i * YL);
                s1[i] = __ldg(t + (size_t)i * YL + 1);
            }
        }
        float4* o = rec + ((size_t)v * RH + r0) * RW + c;
#pragma unroll
        for (int i = 0; i < kRecRows; ++i)
            if (i < nr) o[(size_t)i * RW] = cell_record(s0[i], s1[i], s0[i + 1], s1[i + 1]);
    }
}

template <typename OutT>
__global__ void k_zero_valid_any(const PiRecord* __restrict__ pit, OutT* __restrict__ image,
                                 size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        if (pit[i].bi != kPiInvalid) image[i] = (OutT)0;
}

// Variants: 0, 1 = third form with blocks of 4 / 8 views; 2, 3, 4 = second form with
// (TZ, NB) = (8, 8), (4, 8), (8, 4); 5 .. 9 = fourth form with (NB, S, PW) = (4, 2, 1),
// (2, 4, 1), (4, 2, 2), (4, 2, 3), (4, 3, 4).
__host__ __device__ constexpr int variant_tz(int variant) { return variant == 3 ? 4 : 8; }

// The persistent batched kernel of the fourth form (its own block size).
template <int NB, int S, int PW>
__global__ void __launch_bounds__(32 * (8 + PW), PW <= 2 ? 3 : 2)
k_bkproj4_batch(const BatchScanDev* __restrict__ scans, int n_scans, long long total_tiles,
                unsigned long long* __restrict__ counter, Caps4 caps, int* err) {
    extern __shared__ __align__(16) unsigned char dynb4[];
    __shared__ Shared4<NB, S, PW> sh;
    __shared__ BatchScanDev sc;  // this tile's scan record, read from shared memory
    tile4_init(sh);
    uint32_t iter = 0;
    for (;;) {
        if (threadIdx.x == 0) {
            const long long item = (long long)atomicAdd(counter, 1ull);
            sh.s_item = item;
            if (item < total_tiles) {
                int s = 0;
                while (s + 1 < n_scans && scans[s + 1].first_tile <= item) ++s;
                sc = scans[s];
            }
        }
        __syncthreads();
        const long long item = sh.s_item;
        if (item >= total_tiles) break;
        const int nxt = (sc.kp.NX + kTXY2 - 1) / kTXY2, nyt = (sc.kp.NY + kTXY2 - 1) / kTXY2;
        const long long local = item - sc.first_tile;
        const int bx = (int)(local % nxt);
        const int by = (int)((local / nxt) % nyt);
        const int bz = (int)(local / ((long long)nxt * nyt));
        iter = tile4<NB, S, PW, false, float>(sc.kp, sc.fproj, sc.pit, sc.views, sc.xyz,
                                              sc.image, bx, by, bz, sh, dynb4, caps, err, iter);
        if (sh.s_abort) break;  // uniform: read after the tile's closing barrier
    }
}

// The persistent batched kernel of the fifth form: as k_bkproj4_batch, each scan's records
// brought in through its own box-map table.
template <int NB, int S, int MINB>
__global__ void __launch_bounds__(32 * 9, MINB)
k_bkproj5_batch(const BatchScanDev* __restrict__ scans, int n_scans, long long total_tiles,
                unsigned long long* __restrict__ counter, Caps4 caps, int* err) {
    extern __shared__ __align__(128) unsigned char dynb5[];
    __shared__ Shared4<NB, S, 1> sh;
    __shared__ BatchScanDev sc;
    tile4_init(sh);
    uint32_t iter = 0;
    for (;;) {
        if (threadIdx.x == 0) {
            const long long item = (long long)atomicAdd(counter, 1ull);
            sh.s_item = item;
            if (item < total_tiles) {
                int s = 0;
                while (s + 1 < n_scans && scans[s + 1].first_tile <= item) ++s;
                sc = scans[s];
            }
        }
        __syncthreads();
        const long long item = sh.s_item;
        if (item >= total_tiles) break;
        const int nxt = (sc.kp.NX + kTXY2 - 1) / kTXY2, nyt = (sc.kp.NY + kTXY2 - 1) / kTXY2;
        const long long local = item - sc.first_tile;
        const int bx = (int)(local % nxt);
        const int by = (int)((local / nxt) % nyt);
        const int bz = (int)(local / ((long long)nxt * nyt));
        iter = tile4<NB, S, 1, true, float, pair_slices5(NB, MINB)>(
            sc.kp, sc.fproj, sc.pit, sc.views, sc.xyz, sc.image, bx, by, bz, sh, dynb5, caps, err,
            iter, static_cast<const CUtensorMap*>(sc.tmaps), sc.rec_p0);
        if (sh.s_abort) break;  // uniform: read after the tile's closing barrier
    }
}

// Many scans in one persistent launch: the CTAs pull tiles of all scans from one atomic
// counter (largest-first order is the caller's choice of scan order), so uneven scans share
// the GPU without tails between them.
template <int FORM, int TZ, int NB>
__global__ void __launch_bounds__(256, 3)
k_bkproj_batch(const BatchScanDev* __restrict__ scans, int n_scans, long long total_tiles,
               unsigned long long* __restrict__ counter) {
    extern __shared__ __align__(16) unsigned char dynb[];
    __shared__ BPShared<NB> sh2;
    __shared__ Shared3<NB> sh3;
    __shared__ long long s_item;
    __shared__ BatchScanDev sc;  // this tile's scan record, read from shared memory
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) {
            const long long item = (long long)atomicAdd(counter, 1ull);
            s_item = item;
            if (item < total_tiles) {
                int s = 0;
                while (s + 1 < n_scans && scans[s + 1].first_tile <= item) ++s;
                sc = scans[s];
            }
        }
        __syncthreads();
        const long long item = s_item;
        if (item >= total_tiles) break;
        const int nxt = (sc.kp.NX + kTXY2 - 1) / kTXY2, nyt = (sc.kp.NY + kTXY2 - 1) / kTXY2;
        const long long local = item - sc.first_tile;
        const int bx = (int)(local % nxt);
        const int by = (int)((local / nxt) % nyt);
        const int bz = (int)(local / ((long long)nxt * nyt));
        if constexpr (FORM == 3)
            tile3<NB, float>(sc.kp, sc.fproj, sc.pit, sc.views, sc.xyz, sc.image, bx, by, bz, sh3,
                             dynb);
        else
            bp_tile<TZ, NB, float>(sc.kp, sc.fproj, sc.pit, sc.views, sc.xyz, sc.image, bx, by,
                                   bz, sh2, reinterpret_cast<float*>(dynb));
    }
}

long long bkproj_batch_tiles(const BPParams& kp, int variant) {
    const int TZ = variant_tz(variant);
    return (long long)((kp.NX + kTXY2 - 1) / kTXY2) * ((kp.NY + kTXY2 - 1) / kTXY2) *
           ((kp.NZ + TZ - 1) / TZ);
}

template <int FORM, int TZ, int NB>
static Status launch_batch(cudaStream_t s, const BatchScanDev* d_scans, int n,
                           long long total, unsigned long long* d_counter) {
    const size_t smem = FORM == 3 ? tile3_smem_bytes<NB>() : (size_t)2 * NB * kCap2 * sizeof(float);
    CTR_CUDA(cudaFuncSetAttribute(k_bkproj_batch<FORM, TZ, NB>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev = 0, sms = 148, per_sm = 1;
    CTR_CUDA(cudaGetDevice(&dev));
    CTR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CTR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bkproj_batch<FORM, TZ, NB>,
                                                           256, smem));
    const long long grid = std::min<long long>(total, (long long)std::max(1, per_sm) * sms);
    CTR_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(unsigned long long), s));
    if (grid > 0)
        k_bkproj_batch<FORM, TZ, NB><<<(unsigned)grid, 256, smem, s>>>(d_scans, n, total, d_counter);
    CTR_CUDA(cudaGetLastError());
    return Status::Ok();
}

template <int NB, int S, int PW>
static Status launch_batch4(cudaStream_t s, const BatchScanDev* d_scans, int n, long long total,
                            unsigned long long* d_counter, Caps4 caps, int* err) {
    const size_t smem = tile4_smem_bytes<NB, S, PW>(caps);
    const int threads = 32 * (8 + PW);
    CTR_CUDA(cudaFuncSetAttribute(k_bkproj4_batch<NB, S, PW>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev = 0, sms = 148, per_sm = 1;
    CTR_CUDA(cudaGetDevice(&dev));
    CTR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CTR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bkproj4_batch<NB, S, PW>,
                                                           threads, smem));
    const long long grid = std::min<long long>(total, (long long)std::max(1, per_sm) * sms);
    CTR_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(unsigned long long), s));
    if (grid > 0)
        k_bkproj4_batch<NB, S, PW><<<(unsigned)grid, threads, smem, s>>>(d_scans, n, total,
                                                                        d_counter, caps, err);
    CTR_CUDA(cudaGetLastError());
    return Status::Ok();
}

// Shared memory per fifth-form CTA: three CTAs per SM (MINB 3) or two.
constexpr size_t smem5_budget(int minb) { return minb >= 3 ? 72 * 1024 : 108 * 1024; }
template <int NB, int S, int MINB>
static Status launch_batch5(cudaStream_t s, const BatchScanDev* d_scans, int n, long long total,
                            unsigned long long* d_counter, int box_cap, int* err) {
    int cells = (box_cap + 7) / 8 * 8;
    const size_t budget = smem5_budget(MINB) - 128;
    if ((size_t)S * NB * cells * 16 > budget)
        cells = std::max(64, (int)(budget / ((size_t)S * NB * 16)) / 8 * 8);
    const Caps4 caps{cells, 0};
    const size_t smem = tile4_smem_bytes<NB, S, 1>(caps) + 128;
    const int threads = 32 * 9;
    CTR_CUDA(cudaFuncSetAttribute(k_bkproj5_batch<NB, S, MINB>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev = 0, sms = 148, per_sm = 1;
    CTR_CUDA(cudaGetDevice(&dev));
    CTR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CTR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bkproj5_batch<NB, S, MINB>,
                                                           threads, smem));
    const long long grid = std::min<long long>(total, (long long)std::max(1, per_sm) * sms);
    CTR_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(unsigned long long), s));
    if (grid > 0)
        k_bkproj5_batch<NB, S, MINB><<<(unsigned)grid, threads, smem, s>>>(d_scans, n, total,
                                                                         d_counter, caps, err);
    CTR_CUDA(cudaGetLastError());
    return Status::Ok();
}

// cells_cap: the group's fourth-form record capacity, or for 10..12 its box capacity
Status launch_bkproj_batch(int variant, cudaStream_t s, const BatchScanDev* d_scans, int n,
                           long long total, unsigned long long* d_counter, int cells_cap,
                           int raw_cap, int* err) {
    switch (variant) {
    case 10: return launch_batch5<4, 3, 3>(s, d_scans, n, total, d_counter, cells_cap, err);
    case 11: return launch_batch5<4, 4, 2>(s, d_scans, n, total, d_counter, cells_cap, err);
    case 12: return launch_batch5<8, 2, 2>(s, d_scans, n, total, d_counter, cells_cap, err);
    case 5: return launch_batch4<4, 2, 1>(s, d_scans, n, total, d_counter,
                                              caps_within(cells_cap, raw_cap, 4, 2, smem4_budget(1)), err);
    case 6: return launch_batch4<2, 4, 1>(s, d_scans, n, total, d_counter,
                                              caps_within(cells_cap, raw_cap, 2, 4, smem4_budget(1)), err);
    case 7: return launch_batch4<4, 2, 2>(s, d_scans, n, total, d_counter,
                                              caps_within(cells_cap, raw_cap, 4, 2, smem4_budget(2)), err);
    case 8: return launch_batch4<4, 2, 3>(s, d_scans, n, total, d_counter,
                                              caps_within(cells_cap, raw_cap, 4, 2, smem4_budget(3)), err);
    case 9: return launch_batch4<4, 3, 4>(s, d_scans, n, total, d_counter,
                                              caps_within(cells_cap, raw_cap, 4, 3, smem4_budget(4)), err);
    case 1: return launch_batch<3, 8, 8>(s, d_scans, n, total, d_counter);
    case 2: return launch_batch<2, 8, 8>(s, d_scans, n, total, d_counter);
    case 3: return launch_batch<2, 4, 8>(s, d_scans, n, total, d_counter);
    case 4: return launch_batch<2, 8, 4>(s, d_scans, n, total, d_counter);
    default: return launch_batch<3, 8, 4>(s, d_scans, n, total, d_counter);
    }
}

template <int TZ, int NB, typename OutT>
static Status launch_v2(cudaStream_t s, BPPlan& plan, const float* d_fproj,
                        const PiRecord* d_pitab, OutT* d_image) {
    const BPParams& kp = plan.kp;
    dim3 grid((kp.NX + kTXY2 - 1) / kTXY2, (kp.NY + kTXY2 - 1) / kTXY2, (kp.NZ + TZ - 1) / TZ);
    const size_t smem = (size_t)2 * NB * kCap2 * sizeof(float);
    CTR_CUDA(cudaFuncSetAttribute(k_bkproj2<TZ, NB, OutT>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_bkproj2<TZ, NB, OutT><<<grid, 256, smem, s>>>(kp, d_fproj, d_pitab, plan.views.as<float4>(),
                                                    plan.xyz.as<float>(), d_image);
    CTR_CUDA(cudaGetLastError());
    return Status::Ok();
}

template <int NB, typename OutT>
static Status launch_v3(cudaStream_t s, BPPlan& plan, const float* d_fproj,
                        const PiRecord* d_pitab, OutT* d_image) {
    const BPParams& kp = plan.kp;
    dim3 grid((kp.NX + kTXY2 - 1) / kTXY2, (kp.NY + kTXY2 - 1) / kTXY2, (kp.NZ + 7) / 8);
    const size_t smem = tile3_smem_bytes<NB>();
    CTR_CUDA(cudaFuncSetAttribute(k_bkproj3<NB, OutT>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_bkproj3<NB, OutT><<<grid, 256, smem, s>>>(kp, d_fproj, d_pitab, plan.views.as<float4>(),
                                                plan.xyz.as<float>(), d_image);
    CTR_CUDA(cudaGetLastError());
    return Status::Ok();
}

template <int NB, int S, int PW, typename OutT>
static Status launch_v4(cudaStream_t s, BPPlan& plan, const float* d_fproj,
                        const PiRecord* d_pitab, OutT* d_image, int* err) {
    const BPParams& kp = plan.kp;
    bp4_caps(plan);
    const Caps4 caps = caps_within(plan.caps_cells, plan.caps_raw, NB, S, smem4_budget(PW));
    dim3 grid((kp.NX + kTXY2 - 1) / kTXY2, (kp.NY + kTXY2 - 1) / kTXY2, (kp.NZ + 7) / 8);
    const size_t smem = tile4_smem_bytes<NB, S, PW>(caps);
    CTR_CUDA(cudaFuncSetAttribute(k_bkproj4<NB, S, PW, OutT>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_bkproj4<NB, S, PW, OutT><<<grid, 32 * (8 + PW), smem, s>>>(
        kp, d_fproj, d_pitab, plan.views.as<float4>(), plan.xyz.as<float>(), d_image, caps, err);
    CTR_CUDA(cudaGetLastError());
    return Status::Ok();
}

// Capacities of the fourth form's shared buffers for a geometry: the largest footprint (cell
// records and raw floats) over a sample of tiles and views, computed as the kernel does, with
// a margin. A view that still does not fit is read directly; the capacities only trade
// shared memory (occupancy) for the share of views that take the cell path.
void bp4_caps(BPPlan& plan) {
    if (plan.caps_cells > 0) return;
    const BPParams& kp = plan.kp;
    const BPGeom& g = plan.g;
    const int ntx = (kp.NX + 15) / 16, nty = (kp.NY + 15) / 16, ntz = (kp.NZ + 7) / 8;
    const int sx = std::max(1, ntx / 12), sy = std::max(1, nty / 12), sz = std::max(1, ntz / 8);
    const int sp = std::max(1, kp.P / 48);
    auto xc = [&](int i) { return (i - g.XC) * g.dx; };
    auto yc = [&](int i) { return (i - g.YC) * g.dy; };
    auto zc = [&](int i) { return (i - g.ZC) * g.dz; };
    const double R = g.ScanR, DdU = g.StdDis / g.DeltaU, DdV = g.StdDis / g.DeltaV;
    const double PI = kRefPi;
    int max_cells = 0, max_raw = 0, max_box = 0;
    for (int tx = 0; tx < ntx; tx += sx)
        for (int ty = 0; ty < nty; ty += sy)
            for (int tz = 0; tz < ntz; tz += sz) {
                const double bx0 = xc(tx * 16), bx1 = xc(std::min(tx * 16 + 15, kp.NX - 1));
                const double by0 = yc(ty * 16), by1 = yc(std::min(ty * 16 + 15, kp.NY - 1));
                const double bz0 = zc(tz * 8), bz1 = zc(std::min(tz * 8 + 7, kp.NZ - 1));
                if (std::min(bx0 * bx0, bx1 * bx1) + std::min(by0 * by0, by1 * by1) >
                    g.ObjR * g.ObjR * 1.05)
                    continue;  // tile outside the reconstruction cylinder
                for (int p = 0; p < kp.P; p += sp) {
                    const double th = (p + g.ProjBegin - g.ProjCtr) * g.DeltaL;
                    const double c = std::cos(th), sn = std::sin(th), szs = g.HelicP * th / (2 * PI);
                    double umin = 1e30, umax = -1e30, vmin = 1e30, vmax = -1e30;
                    bool ok = true;
                    for (int k = 0; k < 4; ++k) {
                        const double cx = (k & 1) ? bx1 : bx0, cy = (k & 2) ? by1 : by0;
                        const double fen = R - (cx * c + cy * sn);
                        ok = ok && fen > 1e-3 * R;
                        const double u = (cy * c - cx * sn) * DdU / fen + g.HalfY;
                        const double va = (bz0 - szs) * DdV / fen + g.HalfZ;
                        const double vb = (bz1 - szs) * DdV / fen + g.HalfZ;
                        umin = std::min(umin, u); umax = std::max(umax, u);
                        vmin = std::min(vmin, std::min(va, vb));
                        vmax = std::max(vmax, std::max(va, vb));
                    }
                    if (!ok) continue;
                    // the kernels' footprint (bp_tile4.cuh), a little wider
                    const int u0 = (int)std::floor(umin - 2 * kFootMargin);
                    const int u1 = (int)std::floor(umax + 2 * kFootMargin) + 1;
                    const int v0 = (int)std::floor(vmin - 2 * kFootMargin);
                    const int v1 = (int)std::floor(vmax + 2 * kFootMargin) + 1;
                    const int W = u1 - u0 + 1, H = v1 - v0 + 1;
                    if (u0 < 0 || u1 > g.YL - 1 || v0 < 0 || v1 > g.ZL - 1 || W > 64) continue;
                    max_cells = std::max(max_cells, (W - 1) * (H - 1));
                    max_raw = std::max(max_raw, W * H);
                    max_box = std::max(max_box, ((W - 1 + 3) & ~3) * ((H - 1 + 1) & ~1));
                }
            }
    auto cap = [](int v, int lo, int hi) {
        v = (int)(v * 1.15) + 8;
        v = (v + 3) / 4 * 4;
        return std::max(lo, std::min(hi, v));
    };
    plan.caps_cells = cap(max_cells, 64, 1024);
    plan.caps_raw = cap(max_raw, 96, 1536);
    plan.caps_box = cap(max_box, 64, kBoxMaxW * kBoxMaxH);
}

// Capacities that keep a fourth-form CTA within `budget` bytes of dynamic shared memory
// (occupancy): shrunk in proportion when the geometry's footprints would need more; larger
// footprints then take the direct path.
Caps4 caps_within(int cells, int raw, int NB, int S, size_t budget) {
    auto bytes = [&](int c, int r) { return (size_t)S * NB * c * 16 + (size_t)2 * NB * r * 4; };
    if (bytes(cells, raw) > budget) {
        const double f = (double)budget / (double)bytes(cells, raw);
        cells = std::max(64, (int)(cells * f) / 4 * 4);
        raw = std::max(96, (int)(raw * f) / 4 * 4);
    }
    return Caps4{cells, raw};
}

// variants 0 .. 9 of the tiled forms; 100 + k selects the first form (bkproj.cu)
template <typename OutT>
Status launch_bkproj_v2(int variant, cudaStream_t s, BPPlan& plan, const float* d_fproj,
                        const PiRecord* d_pitab, OutT* d_image, int* err) {
    switch (variant) {
    case 5: return launch_v4<4, 2, 1, OutT>(s, plan, d_fproj, d_pitab, d_image, err);
    case 6: return launch_v4<2, 4, 1, OutT>(s, plan, d_fproj, d_pitab, d_image, err);
    case 7: return launch_v4<4, 2, 2, OutT>(s, plan, d_fproj, d_pitab, d_image, err);
    case 8: return launch_v4<4, 2, 3, OutT>(s, plan, d_fproj, d_pitab, d_image, err);
    case 9: return launch_v4<4, 3, 4, OutT>(s, plan, d_fproj, d_pitab, d_image, err);
    case 1: return launch_v3<8, OutT>(s, plan, d_fproj, d_pitab, d_image);
    case 2: return launch_v2<8, 8, OutT>(s, plan, d_fproj, d_pitab, d_image);
    case 3: return launch_v2<4, 8, OutT>(s, plan, d_fproj, d_pitab, d_image);
    case 4: return launch_v2<8, 4, OutT>(s, plan, d_fproj, d_pitab, d_image);
    default: return launch_v3<4, OutT>(s, plan, d_fproj, d_pitab, d_image);
    }
}

// ---- fifth form ------------------------------------------------------------------------

template <int NB, int S, int MINB, typename OutT>
static Status launch_v5(cudaStream_t s, BPPlan& plan, const BPParams& kp, const float* d_fproj,
                        const PiRecord* d_pitab, OutT* d_image, int* err,
                        const CUtensorMap* tmaps, int rec_p0) {
    bp4_caps(plan);
    // slots of whole boxes, a multiple of 8 records (128-byte aligned slots)
    int cells = (plan.caps_box + 7) / 8 * 8;
    const size_t budget = smem5_budget(MINB) - 128;
    if ((size_t)S * NB * cells * 16 > budget)
        cells = std::max(64, (int)(budget / ((size_t)S * NB * 16)) / 8 * 8);
    const Caps4 caps{cells, 0};
    dim3 grid((kp.NX + kTXY2 - 1) / kTXY2, (kp.NY + kTXY2 - 1) / kTXY2, (kp.NZ + 7) / 8);
    const size_t smem = tile4_smem_bytes<NB, S, 1>(caps) + 128;
    CTR_CUDA(cudaFuncSetAttribute(k_bkproj5<NB, S, MINB, OutT>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_bkproj5<NB, S, MINB, OutT><<<grid, 32 * 9, smem, s>>>(
        kp, d_fproj, d_pitab, plan.views.as<float4>(), plan.xyz.as<float>(), d_image, caps, err,
        tmaps, rec_p0);
    CTR_CUDA(cudaGetLastError());
    return Status::Ok();
}

// Variants 10, 11, 12: (NB, S, CTAs per SM) = (4, 3, 3), (4, 4, 2), (8, 2, 2). The loop views
// [win0, win1] of the plan are backprojected in windows whose cell records fit kRecBudget and
// half of the free device memory (beside the records already held) (and
// of at most max_views views when that is > 0);
// with more than one window the valid voxels are zeroed first (or kept, when the plan
// accumulates) and every window adds its sum.
// The box table over records of `nviews` views at `rec`: a tensor map per (bw, bh) box with
// bw = 4, 8 .. kBoxMaxW and bh = 2, 4 .. kBoxMaxH cells, zeroed where the box exceeds the
// detector (the kernel never selects those). Uploaded to `maps` only when it changed.
Status encode_box_maps(void* out, const void* rec, int RW, int RH, int nviews) {
    static_assert(kBoxMaps == kBoxSteps * (kBoxMaxH / 2), "box table size");
    auto enc = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(tensor_map_encoder());
    if (!enc) return make_status(CTRECON_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    CUtensorMap* host = static_cast<CUtensorMap*>(out);
    std::memset(host, 0, sizeof(CUtensorMap) * kBoxMaps);
    cuuint64_t dims[4] = {4, (cuuint64_t)RW, (cuuint64_t)RH, (cuuint64_t)nviews};
    cuuint64_t strides[3] = {16, (cuuint64_t)RW * 16, (cuuint64_t)RW * RH * 16};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    for (int ih = 0; ih < kBoxMaxH / 2; ++ih)
        for (int iw = 0; iw < kBoxSteps; ++iw) {
            const int bw = 4 * (iw + 1), bh = 2 * (ih + 1);
            if (bw > RW || bh > RH) continue;
            cuuint32_t box[4] = {4, (cuuint32_t)bw, (cuuint32_t)bh, 1};
            CUresult r = enc(&host[iw + kBoxSteps * ih], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                             const_cast<void*>(rec), dims, strides, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS)
                return make_status(CTRECON_ERR_CUDA, "cuTensorMapEncodeTiled failed for the "
                                                     "cell records (" + std::to_string((int)r) + ")");
        }
    return Status::Ok();
}

Status launch_cell_records(cudaStream_t s, const float* d_fproj, void* rec, int p0, int nviews,
                           int YL, int ZL) {
    if (nviews <= 0) return Status::Ok();
    dim3 g((YL - 1 + 127) / 128, (ZL - 1 + kRecRows - 1) / kRecRows,
           (unsigned)std::min(nviews, 65535));
    k_cell_records<<<g, 128, 0, s>>>(d_fproj, static_cast<float4*>(rec), p0, nviews, YL, ZL);
    CTR_CUDA(cudaGetLastError());
    return Status::Ok();
}

static Status upload_box_maps(cudaStream_t s, DevBuf& maps, BoxMapKey& key, const float4* rec,
                              int RW, int RH, int nviews) {
    const BoxMapKey want{(const void*)rec, RW, RH, nviews};
    if (maps.ptr && key == want) return Status::Ok();
    constexpr int n = kBoxMaps;
    std::vector<CUtensorMap> host(n);
    CTR_TRY(encode_box_maps(host.data(), rec, RW, RH, nviews));
    CTR_TRY(maps.ensure(sizeof(CUtensorMap) * n, "cell-record box maps"));
    // pageable source: staged by the driver before the call returns, copied in stream order
    CTR_CUDA(cudaMemcpyAsync(maps.ptr, host.data(), sizeof(CUtensorMap) * n,
                             cudaMemcpyHostToDevice, s));
    key = want;
    return Status::Ok();
}

template <typename OutT>
Status launch_bkproj_v5(int variant, cudaStream_t s, BPPlan& plan, const float* d_fproj,
                        const PiRecord* d_pitab, OutT* d_image, int* err, DevBuf& recbuf,
                        DevBuf& maps, BoxMapKey& mkey, int max_views, ctrecon_ctx* tctx) {
    const BPParams& kp0 = plan.kp;
    const int RW = kp0.YL - 1, RH = kp0.ZL - 1;
    const size_t plane = (size_t)RW * RH * sizeof(float4);
    const int w0 = std::max(0, kp0.win0), w1 = std::min(kp0.P - 1, kp0.win1);
    if (w1 < w0) return Status::Ok();
    const int nv_all = w1 - w0 + 1;
    // record budget: whatever the buffer already holds when all views fit in it (the steady
    // state: no driver query per call, which can stall the host while other processes hold the
    // driver), else at most kRecBudget and half of the free device memory
    size_t budget = kRecBudget;
    if ((size_t)nv_all * plane > recbuf.bytes) {
        size_t free_b = 0, total_b = 0;
        CTR_CUDA(cudaMemGetInfo(&free_b, &total_b));
        budget = std::min(kRecBudget, (free_b + recbuf.bytes) / 2);
    }
    int per = (int)std::max<size_t>(1, std::min<size_t>(nv_all, budget / plane));
    if (max_views > 0) per = std::min(per, max_views);
    const int nwin = (nv_all + per - 1) / per;
    CTR_TRY(recbuf.ensure((size_t)std::min(per, nv_all) * plane, "cell records"));
    CTR_TRY(upload_box_maps(s, maps, mkey, recbuf.as<float4>(), RW, RH, std::min(per, nv_all)));
    const CUtensorMap* tmaps = maps.as<CUtensorMap>();
    BPParams kp = kp0;
    if (nwin > 1 && !kp0.accum) {
        const size_t n = (size_t)kp0.NX * kp0.NY * kp0.NZ;
        const unsigned g = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 32);
        k_zero_valid_any<OutT><<<g, 256, 0, s>>>(d_pitab, d_image, n);
        CTR_CUDA(cudaGetLastError());
        kp.accum = 1;
    }
    float4* rec = recbuf.as<float4>();
    for (int w = 0; w < nwin; ++w) {
        const int a = w0 + w * per, b = std::min(w1, a + per - 1);
        const int nv = b - a + 1;
        {
            KernelTimer tm(tctx, s, kKCellRecords);
            CTR_TRY(launch_cell_records(s, d_fproj, rec, a, nv, kp0.YL, kp0.ZL));
        }
        kp.win0 = a;
        kp.win1 = b;
        KernelTimer tm(tctx, s, kKBackproject);
        Status st;
        switch (variant) {
        case 11: st = launch_v5<4, 4, 2, OutT>(s, plan, kp, d_fproj, d_pitab, d_image, err, tmaps, a); break;
        case 12: st = launch_v5<8, 2, 2, OutT>(s, plan, kp, d_fproj, d_pitab, d_image, err, tmaps, a); break;
        default: st = launch_v5<4, 3, 3, OutT>(s, plan, kp, d_fproj, d_pitab, d_image, err, tmaps, a); break;
        }
        CTR_TRY(st);
    }
    return Status::Ok();
}

template Status launch_bkproj_v5<float>(int, cudaStream_t, BPPlan&, const float*, const PiRecord*, float*, int*, DevBuf&, DevBuf&, BoxMapKey&, int, ctrecon_ctx*);
template Status launch_bkproj_v5<double>(int, cudaStream_t, BPPlan&, const float*, const PiRecord*, double*, int*, DevBuf&, DevBuf&, BoxMapKey&, int, ctrecon_ctx*);

template Status launch_bkproj_v2<float>(int, cudaStream_t, BPPlan&, const float*, const PiRecord*, float*, int*);
template Status launch_bkproj_v2<double>(int, cudaStream_t, BPPlan&, const float*, const PiRecord*, double*, int*);

}  // namespace ctr
