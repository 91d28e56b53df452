// bp_tile4.cuh -- the fourth form of the voxel-driven backprojection tile
// (KatsevichBkProj.cpp:164-265; FP32 interpolation and accumulation, the reference's endpoint
// rule): the per-cell records and rounding floor of the third form (bp_tile3.cuh), with the
// staging taken off the compute warps.
//
//  * Warp roles. Warps 0-7 (the 16 x 16 voxel columns of the tile, 8 slices each) only
//    accumulate. PW producer warps compute the footprints of each block of NB views, copy the
//    raw footprint rows with cp.async two blocks ahead, and build the 16-byte cell records
//    {A, C, B, D} into a ring of S slots.
//  * Hand-off. Slot s has a `full` mbarrier (every producer thread arrives after writing its
//    records) and an `empty` one (every consumer thread arrives after its last read); phases
//    follow a per-CTA block counter, so the ring runs on across the tiles of the persistent
//    batched kernel. Every wait is bounded: a wait that gives up records an error code in the
//    device word and the CTA abandons the tile (no write) after draining its copies.
//  * Capacities (cell records and raw floats per staged view) are launch parameters sized on
//    the host from the geometry; a view whose footprint does not fit, or reaches the detector
//    border, is read directly from FProj with the first form's clamped indices.
//  * REC = true (the fifth form): the cell records of every view were written to global memory
//    beforehand (k_cell_records); a single producer warp computes the footprints and brings
//    each into the ring with ONE tensor copy of the smallest box of the box-map table that
//    holds it (complete_tx on `full`), so no thread builds records and no raw rows are staged.
//    One copy per view instead of one per footprint row: the copies were bound by their
//    request rate, not their bytes.
#pragma once

#include "bp_tile3.cuh"
#include "tc_util.cuh"

#include <cuda.h>

namespace ctr {
namespace bp {

__device__ __forceinline__ void mbar_init4(uint64_t* bar, uint32_t count) {
    tcu::mbar_init(bar, count);
}
__device__ __forceinline__ void mbar_arrive4(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
// bounded wait (suspend-hinted try_wait, time limit): tc_util.cuh
__device__ __forceinline__ bool mbar_wait4(uint64_t* bar, uint32_t parity, int* err, int code) {
    return tcu::mbar_wait(bar, parity, err, code);
}
__device__ __forceinline__ void mbar_expect_tx4(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;"
                 ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
// Fifth form: the footprint of a view is brought in by one tensor copy of a box of bw x bh cell
// records (bw a multiple of 4 up to kBoxMaxW, bh a multiple of 2 up to kBoxMaxH), from a table
// of tensor maps over the records [views][ZL - 1][YL - 1][4 floats] that differ only in the
// box: map index (bw / 4 - 1) + kBoxSteps * (bh / 2 - 1).
constexpr int kBoxMaxW = 64, kBoxMaxH = 32, kBoxSteps = 16;
__device__ __forceinline__ void tma_load_cells(uint32_t dst, const void* map, int u, int v,
                                               int view, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
        "l"((uint64_t)map), "r"(0), "r"(u), "r"(v), "r"(view), "r"(smem_addr(bar))
        : "memory");
}
// The bilinear record of the cell between detector samples (r, c) .. (r + 1, c + 1), for
// offsets alpha - 1/2, beta - 1/2 from the cell centre: value = A + a B + b (C + a D), stored
// {A, C, B, D} so that the two halves of the 16-byte record give (A + a B, C + a D) in one
// packed FP32x2 fma.
__device__ __forceinline__ float4 cell_record(float t00, float t01, float t10, float t11) {
    const float h0 = t01 - t00, h1 = t11 - t10;
    const float g0 = t10 - t00, g1 = t11 - t01;
    return make_float4(0.25f * ((t00 + t01) + (t10 + t11)), 0.5f * (g0 + g1), 0.5f * (h0 + h1),
                       h1 - h0);
}

// slack of the footprint bounds, in detector cells
constexpr float kFootMargin = 0.0625f;

// packed FP32 pairs (sm_100 f32x2 arithmetic): two slices' v coordinate, floor and distance
// in one instruction each; the halves are the two 32-bit registers of the pair
__device__ __forceinline__ uint64_t pk2(float lo, float hi) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void upk2(uint64_t v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ uint64_t ffma2(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ uint64_t fadd2(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t fsub2(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

// a cell record as its two 64-bit halves {A, C} and {B, D}
__device__ __forceinline__ void lds_record(uint32_t addr, uint64_t& ac, uint64_t& bd) {
    asm volatile("ld.shared.v2.b64 {%0, %1}, [%2];" : "=l"(ac), "=l"(bd) : "r"(addr));
}
// the record's value at cell offsets (a, b), a2 = (a, a): A + a B + b (C + a D), rounded as
// fma(b, fma(a, D, C), fma(a, B, A))
__device__ __forceinline__ float record_value(uint32_t addr, uint64_t a2, float b) {
    uint64_t ac, bd;
    lds_record(addr, ac, bd);
    float lo, hi;
    upk2(ffma2(a2, bd, ac), lo, hi);
    return fmaf(b, hi, lo);
}

struct Caps4 {
    int cells;  // cell records per staged view (multiple of 4)
    int raw;    // raw floats per staged view (multiple of 4)
};

template <int NB, int S, int PW>
struct Shared4 {
    uint64_t full[S], empty[S];
    Foot3 foot[S][NB];
    float4 vg[S][NB];
    // per staged view: {byte address of the cell records less (kMagicBits + u0) * 16 +
    // (kMagicBits + v0) * W16, W16 = row stride in bytes}, so that a consumer's cell base is
    // bits(u + kMagic) * 16 + kb
    int2 kw[S][NB];
    // per consumer warp and slice: warp-wide view ranges {lo, hi} (some lane's voxel has a PI
    // interval there) and {flo, fhi} (every lane's voxel has weight 1 there)
    int4 sr[8][8];
    Foot3 pfoot[2][NB];  // producer side: footprints of the blocks being staged
    float4 pvg[2][NB];
    int s_pmin, s_pmax, s_abort;
    long long s_item;
};

template <int NB, int S, int PW>
__host__ __device__ inline size_t tile4_smem_bytes(const Caps4& c) {
    return (size_t)S * NB * c.cells * 16 + (size_t)2 * NB * c.raw * sizeof(float);
}

template <int NB, int S, int PW>
__device__ __forceinline__ void tile4_init(Shared4<NB, S, PW>& sh) {
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init4(&sh.full[s], 32 * PW);
            mbar_init4(&sh.empty[s], 256);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
}

// One CTA tile: columns [16 bx, 16 bx + 16) x [16 by, 16 by + 16), slices [8 bz, 8 bz + 8).
// Called by all 32 * (8 + PW) threads with the same `iter` (blocks of views this CTA has
// processed before); returns the new count. Returns with no copies in flight. Sets
// sh.s_abort (and leaves the tile unwritten) when a wait gave up. PK2: unweighted updates of
// two slices share their packed FP32x2 arithmetic (needs about 8 more registers per thread).
template <int NB, int S, int PW, bool REC, typename OutT, bool PK2 = false>
__device__ __forceinline__ uint32_t tile4(const BPParams& kp, const float* __restrict__ fproj,
                                          const PiRecord* __restrict__ pit,
                                          const float4* __restrict__ views,
                                          const float* __restrict__ xyz, OutT* __restrict__ image,
                                          int bx, int by, int bz, Shared4<NB, S, PW>& sh,
                                          unsigned char* dyn, Caps4 caps, int* err,
                                          uint32_t iter, const CUtensorMap* __restrict__ tmaps = nullptr,
                                          int rec_p0 = 0) {
    constexpr int TZ = 8;
    const int ccap = caps.cells, rcap = caps.raw;
    // cell records S * NB * ccap (the fifth form's tensor copies want 128-byte aligned slots:
    // ccap is a multiple of 8 and the base rounded up), then 2 * NB * rcap raw floats
    if constexpr (REC) dyn += (128u - (smem_addr(dyn) & 127u)) & 127u;
    float4* cellbuf = reinterpret_cast<float4*>(dyn);
    float* raw = reinterpret_cast<float*>(dyn + (size_t)S * NB * ccap * 16);
    const uint32_t cell_s = smem_addr(cellbuf);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool consumer = warp < 8;
    const int NX = kp.NX, NY = kp.NY, NZ = kp.NZ, P = kp.P, YL = kp.YL, ZL = kp.ZL;
    const int zb = bz * TZ;
    const float* xc = xyz;
    const float* yc = xyz + NX;
    const float* zc = xyz + NX + NY;

    // consumer state
    // warp w holds the 8 x 4 columns x in 8 (w & 1) + [0, 8), y in 4 (w >> 1) + [0, 4) (compact,
    // so its voxels' PI intervals differ little); each quarter-warp of its 16-byte record loads is
    // a 2 x 4 patch (lane bit 0: x, bits 1-2: y, bits 3-4: x), whose cells on the detector lie closer
    // together than 8 columns of one row, so fewer of them share a bank group
    const int lane_ = tid & 31, w_ = (tid >> 5) & 7;
    const int tx = (w_ & 1) * 8 + (lane_ & 1) + ((lane_ >> 3) & 3) * 2;
    const int ty = (w_ >> 1) * 4 + ((lane_ >> 1) & 3);
    const int x = bx * kTXY + tx, y = by * kTXY + ty;
    const bool col_ok = consumer && (x < NX) && (y < NY);
    const size_t colbase = ((size_t)x * NY + y) * NZ;
    VoxelRanges<TZ> vr;
    load_ranges<TZ>(pit, colbase, zb, NZ, P, col_ok, kp.win0, kp.win1, vr);
    int wmin = vr.tmin, wmax = vr.tmax;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        wmin = min(wmin, __shfl_xor_sync(0xffffffffu, wmin, o));
        wmax = max(wmax, __shfl_xor_sync(0xffffffffu, wmax, o));
    }
    if (tid == 0) { sh.s_pmin = INT_MAX; sh.s_pmax = INT_MIN; sh.s_abort = 0; }
    __syncthreads();
    if (consumer && lane == 0 && wmin <= wmax) {
        atomicMin(&sh.s_pmin, wmin);
        atomicMax(&sh.s_pmax, wmax);
    }
    __syncthreads();
    const int pmin = sh.s_pmin, pmax = sh.s_pmax;
    if (pmin > pmax) return iter;
    const int nblk = (pmax - pmin) / NB + 1;

    const float R = kp.Rf, DdU = kp.DdU, DdV = kp.DdV, HalfY = kp.HalfY, HalfZ = kp.HalfZ;
    float acc[TZ];
#pragma unroll
    for (int k = 0; k < TZ; ++k) acc[k] = 0.f;
    int issued = 0;  // fifth form: blocks whose copies this producer thread has started

    if (!consumer) {
        // ------------------------------------------------------------------ producers
        const int pw = warp - 8;  // views j with j % PW == pw are this warp's
        const int x0 = bx * kTXY, x1 = min(x0 + kTXY, NX) - 1;
        const int y0 = by * kTXY, y1 = min(y0 + kTXY, NY) - 1;
        const int z1 = min(zb + TZ, NZ) - 1;
        const float bx0 = xc[x0], bx1 = xc[x1], by0 = yc[y0], by1 = yc[y1];
        const float bz0 = zc[zb], bz1 = zc[z1];
        // lane i < NB / PW owns view j = pw + i * PW of every block
        constexpr int VPW = (NB + PW - 1) / PW;
        const int jl = pw + lane * PW;
        const bool vlane = lane < VPW && jl < NB;
        // view geometry of this lane's view of block ib (zero past the range)
        auto view_of = [&](int ib) {
            const int p = pmin + ib * NB + jl;
            return (vlane && ib < nblk && p <= pmax) ? views[p] : make_float4(0.f, 0.f, 0.f, 0.f);
        };
        // footprints of this warp's views of block ib; g = view_of(ib), loaded a block ahead
        auto footprint = [&](int ib, float4 g) {
            if (vlane) {
                Foot3 f{0, 0, -1, 0};
                const int p = pmin + ib * NB + jl;
                if (p <= pmax) {
                    float umin = 1e30f, umax = -1e30f, vmin = 1e30f, vmax = -1e30f;
                    bool ok = true;
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        const float cx = (c & 1) ? bx1 : bx0, cy = (c & 2) ? by1 : by0;
                        const float fen = R - (cx * g.x + cy * g.y);
                        ok = ok && (fen > 1e-3f * R);
                        const float inv = rcp_approx(fen);  // within the +-1 cell margin
                        const float u = (cy * g.x - cx * g.y) * DdU * inv + HalfY;
                        const float va = (bz0 - g.z) * DdV * inv + HalfZ;
                        const float vb = (bz1 - g.z) * DdV * inv + HalfZ;
                        umin = fminf(umin, u); umax = fmaxf(umax, u);
                        vmin = fminf(vmin, fminf(va, vb)); vmax = fmaxf(vmax, fmaxf(va, vb));
                    }
                    f = Foot3{0, 0, -2, 0};
                    if (ok && fabsf(umin) < 1048576.f && fabsf(umax) < 1048576.f &&
                        fabsf(vmin) < 1048576.f && fabsf(vmax) < 1048576.f) {
                        // a voxel at detector position (u, v) reads the cell whose corner is
                        // (rint(u - 1/2), rint(v - 1/2)), i.e. (floor(u), floor(v)) or one less
                        // at integer positions; u and v are linear-fractional in the voxel
                        // coordinates, so their extremes over the tile are at the corners;
                        // kFootMargin covers the FP32 rounding between these corner values and
                        // the consumers' per-voxel ones (~1e-3 cells at most). Samples
                        // [u0, u1] x [v0, v1], cells [u0, u1) x [v0, v1).
                        const int u0 = (int)floorf(umin - kFootMargin);
                        const int u1 = (int)floorf(umax + kFootMargin) + 1;
                        const int v0 = (int)floorf(vmin - kFootMargin);
                        const int v1 = (int)floorf(vmax + kFootMargin) + 1;
                        const int W = u1 - u0 + 1, H = v1 - v0 + 1;
                        if (u0 >= 0 && u1 <= YL - 1 && v0 >= 0 && v1 <= ZL - 1 &&
                            (REC || (W <= 64 && W * H <= rcap)) && (W - 1) * (H - 1) <= ccap)
                            f = Foot3{u0, v0, W, H};
                    }
                }
                sh.pfoot[ib & 1][jl] = f;
                sh.pvg[ib & 1][jl] = g;
            }
            __syncwarp();
        };
        auto stage = [&](int ib) {  // raw rows of this warp's views of block ib
            for (int j = pw; j < NB; j += PW) {
                const Foot3 f = sh.pfoot[ib & 1][j];
                if (f.W <= 0) continue;
                const int p = pmin + ib * NB + j;
                const float* src = fproj + ((size_t)p * ZL + f.v0) * YL + f.u0;
                float* dst = raw + ((ib & 1) * NB + j) * rcap;
                for (int r = 0; r < f.H; ++r) {
                    if (lane < f.W) cp_async4(dst + r * f.W + lane, src + (size_t)r * YL + lane);
                    if (lane + 32 < f.W)
                        cp_async4(dst + r * f.W + lane + 32, src + (size_t)r * YL + lane + 32);
                }
            }
            cp_async_commit();
        };
        // the block's records: per-view constants, then the footprint (or nothing) in slot
        auto publish = [&](int ib, uint32_t slot, int j, const Foot3& f) {
            if (lane == 0) {
                sh.foot[slot][j] = f;
                sh.vg[slot][j] = sh.pvg[ib & 1][j];
                const uint32_t W16 = (uint32_t)(f.W - 1) * 16u;
                const uint32_t kb = cell_s + (uint32_t)((slot * NB + j) * ccap) * 16u -
                                    (uint32_t)(kMagicBits + f.u0) * 16u -
                                    (uint32_t)(kMagicBits + f.v0) * W16;
                sh.kw[slot][j] = make_int2((int)kb, (int)W16);
            }
        };
        if constexpr (REC) {
            // fifth form: one tensor copy per view from the global cell records; the footprint
            // is widened to the copied box (its origin moved in so that the box stays on the
            // detector), which the consumers then address like any footprint
            static_assert(PW == 1, "the fifth form has one producer warp");
            const int RW = YL - 1, RH = ZL - 1;
            float4 gnext = view_of(0);
            for (int ib = 0; ib < nblk; ++ib) {
                const float4 gv = gnext;
                gnext = view_of(ib + 1);
                footprint(ib, gv);
                const uint32_t g = iter + ib, slot = g % S, use = g / S;
                if (use >= 1 && !mbar_wait4(&sh.empty[slot], (use - 1) & 1, err, 11)) {
                    sh.s_abort = 1;
                    break;
                }
                if (vlane) {
                    Foot3 f = sh.pfoot[ib & 1][jl];
                    int box = -1, bw = 0, bh = 0;
                    if (f.W > 0) {
                        bw = (f.W - 1 + 3) & ~3;
                        bh = (f.H - 1 + 1) & ~1;
                        if (bw <= min(kBoxMaxW, RW) && bh <= min(kBoxMaxH, RH) && bw * bh <= ccap) {
                            f = Foot3{min(f.u0, RW - bw), min(f.v0, RH - bh), bw + 1, bh + 1};
                            box = (bw / 4 - 1) + kBoxSteps * (bh / 2 - 1);
                        } else {
                            f.W = -2;
                        }
                    }
                    sh.foot[slot][jl] = f;
                    sh.vg[slot][jl] = sh.pvg[ib & 1][jl];
                    const uint32_t W16 = (uint32_t)(f.W - 1) * 16u;
                    const uint32_t dst = cell_s + (uint32_t)((slot * NB + jl) * ccap) * 16u;
                    sh.kw[slot][jl] = make_int2((int)(dst - (uint32_t)(kMagicBits + f.u0) * 16u -
                                                      (uint32_t)(kMagicBits + f.v0) * W16),
                                                (int)W16);
                    if (box >= 0) {
                        mbar_expect_tx4(&sh.full[slot], (uint32_t)(bw * bh) * 16u);
                        tma_load_cells(dst, tmaps + box, f.u0, f.v0,
                                       pmin + ib * NB + jl - rec_p0, &sh.full[slot]);
                    }
                }
                mbar_arrive4(&sh.full[slot]);
                issued = ib + 1;
            }
        } else {
        footprint(0, view_of(0));
        stage(0);
        float4 gnext = view_of(1);
        for (int ib = 0; ib < nblk; ++ib) {
            if (ib + 1 < nblk) {
                const float4 g = gnext;
                gnext = view_of(ib + 2);  // in flight while this block is staged and built
                footprint(ib + 1, g);
                stage(ib + 1);
            } else {
                cp_async_commit();
            }
            cp_async_wait<1>();
            __syncwarp();  // this block's raw rows of all lanes have landed
            const uint32_t g = iter + ib, slot = g % S, use = g / S;
            if (use >= 1 && !mbar_wait4(&sh.empty[slot], (use - 1) & 1, err, 11)) {
                sh.s_abort = 1;
                break;
            }
            for (int j = pw; j < NB; j += PW) {
                const Foot3 f = sh.pfoot[ib & 1][j];
                publish(ib, slot, j, f);
                if (f.W <= 0) continue;
                const float* src = raw + ((ib & 1) * NB + j) * rcap;
                float4* dst = cellbuf + ((size_t)slot * NB + j) * ccap;
                const int Wc = f.W - 1;
                for (int r = 0; r < f.H - 1; ++r) {
                    for (int c = lane; c < Wc; c += 32) {
                        const float* s0 = src + r * f.W + c;
                        dst[r * Wc + c] = cell_record(s0[0], s0[1], s0[f.W], s0[f.W + 1]);
                    }
                }
            }
            __syncwarp();  // raw slot (ib & 1) is free for block ib + 2
            mbar_arrive4(&sh.full[slot]);
        }
        cp_async_wait<0>();
        }
    } else {
        // ------------------------------------------------------------------ consumers
        // a lane past the volume's edge takes the nearest column of the tile: its reads stay in
        // the staged footprint, and its voxels are never written
        const float X = xc[min(x, NX - 1)], Y = yc[min(y, NY - 1)];
        const float z0 = zc[zb];
        const float dzf = kp.dzf;
        const float HalfYm = HalfY - 0.5f, HalfZm = HalfZ - 0.5f;
        // Per slice k, warp-wide view ranges: [lo, hi] where some lane's voxel of the slice has
        // its PI interval (p in [bi, ti + 1]), [flo, fhi] where every lane's voxel has weight 1
        // (p in [bi + 2, ti - 1], both ramp views of each end excluded). Each block of views then gives every slice one of three warp-uniform
        // classes: no update, the unweighted update, or the checked (weighted) one. Deciding
        // per slice and per block keeps the blocks at the ends of the PI intervals close to the
        // unweighted blocks' cost: the PI ranges of a column's slices are shifted against each
        // other, so in those blocks most slices are wholly inside or wholly outside.
        // Only lanes whose voxel has an interval count: the others (outside the reconstructed
        // cylinder or the volume) are never written, so whatever they accumulate is dropped.
#pragma unroll
        for (int k = 0; k < TZ; ++k) {
            const bool v = col_ok && vr.bi[k] != kPiInvalid;
            int lo = v ? vr.bi[k] : INT_MAX, hi = v ? vr.ti[k] + 1 : INT_MIN;
            int flo = v ? vr.bi[k] + 2 : INT_MIN, fhi = v ? vr.ti[k] - 1 : INT_MAX;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
                hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
                flo = max(flo, __shfl_xor_sync(0xffffffffu, flo, o));
                fhi = min(fhi, __shfl_xor_sync(0xffffffffu, fhi, o));
            }
            if (lo > hi) { flo = INT_MAX; fhi = INT_MIN; }  // no lane with an interval
            if (lane == 0) sh.sr[warp][k] = make_int4(lo, hi, flo, fhi);
        }
        __syncwarp();
        // one voxel's update from cell records, weighted (w) or not
        auto cell_update = [&](int k, float dz0, float kv, float r2, uint64_t a2, uint32_t W16,
                               uint32_t cbase) {
            const float dz = fmaf((float)k, dzf, dz0);
            const float v = fmaf(dz, kv, HalfZm);  // v - 1/2
            const float rinv = rsqrt_approx(fmaf(dz, dz, r2));
            const float tv = v + kMagic;
            const float b = v - (tv - kMagic);
            const float val = record_value((uint32_t)__float_as_int(tv) * W16 + cbase, a2, b);
            acc[k] = fmaf(val, rinv, acc[k]);
        };
        // slices k and k + 1 (k even) with their v coordinate, rounding floor and squared
        // distance in packed pairs; the same operations as cell_update, rounded the same way
        const uint64_t dzf2 = pk2(dzf, dzf), hz2 = pk2(HalfZm, HalfZm), mag2 = pk2(kMagic, kMagic);
        auto cell_update2 = [&](int k, uint64_t dz02, uint64_t kv2, uint64_t r22, uint64_t a2,
                                uint32_t W16, uint32_t cbase) {
            const uint64_t dz = ffma2(pk2((float)k, (float)(k + 1)), dzf2, dz02);
            const uint64_t v = ffma2(dz, kv2, hz2);  // v - 1/2
            const uint64_t tv = fadd2(v, mag2);
            const uint64_t b = fsub2(v, fsub2(tv, mag2));
            float t0, t1, tv0, tv1, b0, b1;
            upk2(ffma2(dz, dz, r22), t0, t1);
            upk2(tv, tv0, tv1);
            upk2(b, b0, b1);
            const float val0 = record_value((uint32_t)__float_as_int(tv0) * W16 + cbase, a2, b0);
            const float val1 = record_value((uint32_t)__float_as_int(tv1) * W16 + cbase, a2, b1);
            acc[k] = fmaf(val0, rsqrt_approx(t0), acc[k]);
            acc[k + 1] = fmaf(val1, rsqrt_approx(t1), acc[k + 1]);
        };
        auto cell_update_w = [&](int k, int p, float dz0, float kv, float r2, uint64_t a2,
                                 uint32_t W16, uint32_t cbase) {
            const int d0 = p - vr.bi[k];
            const int d1 = vr.ti[k] + 1 - p;
            if ((d0 | d1) < 0) return;
            float w = 1.f;
            // the two views at each end of the interval (the fractions reread from the PI table,
            // which keeps them out of registers)
            if (d1 <= 1) w = ramp(__ldg(&pit[colbase + zb + k].tf) + (float)(d1 - 1));
            else if (d0 <= 1) w = ramp((float)d0 - __ldg(&pit[colbase + zb + k].bf));
            const float dz = fmaf((float)k, dzf, dz0);
            const float v = fmaf(dz, kv, HalfZm);
            const float rinv = rsqrt_approx(fmaf(dz, dz, r2));
            const float tv = v + kMagic;
            const float b = v - (tv - kMagic);
            const float val = record_value((uint32_t)__float_as_int(tv) * W16 + cbase, a2, b);
            acc[k] = fmaf(w * val, rinv, acc[k]);
        };
        for (int ib = 0; ib < nblk; ++ib) {
            const uint32_t g = iter + ib, slot = g % S, use = g / S;
            if (!mbar_wait4(&sh.full[slot], use & 1, err, 12)) {
                sh.s_abort = 1;
                break;
            }
            const int pb = pmin + ib * NB, pe = pb + NB - 1;
            bool blk = pe <= pmax;  // a whole block of views with cell records
#pragma unroll
            for (int j = 0; j < NB; ++j) blk = blk && (sh.foot[slot][j].W > 0);
            // 2 bits per slice: 0 no update in this block, 1 unweighted, 2 weighted
            uint32_t cls = 0;
            if (blk) {
#pragma unroll
                for (int k = 0; k < TZ; ++k) {
                    const int4 r = sh.sr[warp][k];
                    const uint32_t c = (pe < r.x || pb > r.y) ? 0u : ((pb >= r.z && pe <= r.w) ? 1u : 2u);
                    cls |= c << (2 * k);
                }
            }
            if (blk && cls == 0x5555u) {
                // every view of the block has cell records and weight 1 for all voxels of the
                // warp: no per-view tests
#pragma unroll
                for (int j = 0; j < NB; ++j) {
                    const float4 gv = sh.vg[slot][j];
                    const int2 kw = sh.kw[slot][j];
                    const float fen = R - (X * gv.x + Y * gv.y);
                    const float YY = Y * gv.x - X * gv.y;
                    const float inv = rcp_approx(fen);
                    const float kv = DdV * inv;
                    const float r2 = fen * fen + YY * YY;
                    const float dz0 = z0 - gv.z;
                    const float u = fmaf(YY * DdU, inv, HalfYm);  // u - 1/2
                    const float tu = u + kMagic;
                    const float a = u - (tu - kMagic);           // alpha - 1/2
                    const uint64_t a2 = pk2(a, a);
                    const uint32_t W16 = (uint32_t)kw.y;
                    const uint32_t cbase = (uint32_t)__float_as_int(tu) * 16u + (uint32_t)kw.x;
                    if constexpr (PK2) {
                        const uint64_t dz02 = pk2(dz0, dz0), kv2 = pk2(kv, kv), r22 = pk2(r2, r2);
#pragma unroll
                        for (int k = 0; k < TZ; k += 2)
                            cell_update2(k, dz02, kv2, r22, a2, W16, cbase);
                    } else {
#pragma unroll
                        for (int k = 0; k < TZ; ++k) cell_update(k, dz0, kv, r2, a2, W16, cbase);
                    }
                }
            } else if (blk) {
                // a block at an end of some slices' PI intervals: per slice its class
                if (cls != 0) {
#pragma unroll 1
                    for (int j = 0; j < NB; ++j) {
                        const int p = pb + j;
                        const float4 gv = sh.vg[slot][j];
                        const int2 kw = sh.kw[slot][j];
                        const float fen = R - (X * gv.x + Y * gv.y);
                        const float YY = Y * gv.x - X * gv.y;
                        const float inv = rcp_approx(fen);
                        const float kv = DdV * inv;
                        const float r2 = fen * fen + YY * YY;
                        const float dz0 = z0 - gv.z;
                        const float u = fmaf(YY * DdU, inv, HalfYm);  // u - 1/2
                        const float tu = u + kMagic;
                        const float a = u - (tu - kMagic);           // alpha - 1/2
                        const uint64_t a2 = pk2(a, a);
                        const uint32_t W16 = (uint32_t)kw.y;
                        const uint32_t cbase = (uint32_t)__float_as_int(tu) * 16u + (uint32_t)kw.x;
#pragma unroll
                        for (int k = 0; k < TZ; k += 2) {
                            const uint32_t c0 = (cls >> (2 * k)) & 3u, c1 = (cls >> (2 * k + 2)) & 3u;
                            if (PK2 && c0 == 1u && c1 == 1u) {
                                if constexpr (PK2)
                                    cell_update2(k, pk2(dz0, dz0), pk2(kv, kv), pk2(r2, r2), a2,
                                                 W16, cbase);
                            } else {
                                if (c0 == 1u) cell_update(k, dz0, kv, r2, a2, W16, cbase);
                                else if (c0 == 2u) cell_update_w(k, p, dz0, kv, r2, a2, W16, cbase);
                                if (c1 == 1u) cell_update(k + 1, dz0, kv, r2, a2, W16, cbase);
                                else if (c1 == 2u)
                                    cell_update_w(k + 1, p, dz0, kv, r2, a2, W16, cbase);
                            }
                        }
                    }
                }
            } else if (col_ok && wmin <= wmax && !(pb + NB - 1 < wmin || pb > wmax)) {
                // a partial block, or views without cell records: every update checked
#pragma unroll 1
                for (int j = 0; j < NB; ++j) {
                    const int p = pb + j;
                    if (p > pmax) break;
                    if (p < vr.tmin || p > vr.tmax) continue;
                    const Foot3 f = sh.foot[slot][j];
                    const float4 gv = sh.vg[slot][j];
                    const float fen = R - (X * gv.x + Y * gv.y);
                    const float YY = Y * gv.x - X * gv.y;
                    const float inv = rcp_approx(fen);
                    const float kv = DdV * inv;
                    const float r2 = fen * fen + YY * YY;
                    const float dz0 = z0 - gv.z;
                    if (f.W > 0) {
                        const float u = fmaf(YY * DdU, inv, HalfYm);  // u - 1/2
                        const float tu = u + kMagic;
                        const float a = u - (tu - kMagic);           // alpha - 1/2
                        const uint64_t a2 = pk2(a, a);
                        const int2 kw = sh.kw[slot][j];
                        const uint32_t W16 = (uint32_t)kw.y;
                        const uint32_t cbase =
                            (uint32_t)__float_as_int(tu) * 16u + (uint32_t)kw.x;
#pragma unroll
                        for (int k = 0; k < TZ; ++k)
                            cell_update_w(k, p, dz0, kv, r2, a2, W16, cbase);
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
                            if (d1 <= 1) w = ramp(__ldg(&pit[colbase + zb + k].tf) + (float)(d1 - 1));
                            else if (d0 <= 1) w = ramp((float)d0 - __ldg(&pit[colbase + zb + k].bf));
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
            mbar_arrive4(&sh.empty[slot]);
        }
    }
    __syncthreads();  // every role is done with the ring; an abort is visible
    if constexpr (REC) {
        if (sh.s_abort && !consumer) {
            // no copy may still be writing the ring when the CTA moves on or exits: wait
            // (bounded, whatever the error word says) for the blocks not known complete
            for (int ib = max(0, issued - S); ib < issued; ++ib) {
                const uint32_t g = iter + ib;
                tcu::mbar_drain(&sh.full[g % S], (g / S) & 1);
            }
        }
        __syncthreads();
    }
    if (col_ok && !sh.s_abort) {
#pragma unroll
        for (int k = 0; k < TZ; ++k) {
            const int z = zb + k;
            if (z < NZ && vr.bi[k] != kPiInvalid) store_voxel(image + colbase + z, -acc[k] * kp.invPs, kp.accum);
        }
    }
    __syncthreads();  // the caller may reuse the shared state for the next tile
    return iter + nblk;
}

}  // namespace bp
}  // namespace ctr
