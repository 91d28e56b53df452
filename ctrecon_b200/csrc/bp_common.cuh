// bp_common.cuh -- device helpers shared by the tiled backprojectors (bp_tile2.cuh,
// bp_tile3.cuh).
#pragma once

#include "internal.h"

#include <climits>
#include <cstdint>

namespace ctr {
namespace bp {

constexpr int kTXY = 16;  // a CTA tile is kTXY x kTXY voxel columns, one thread per column

// The endpoint ramp of KatsevichBkProj.cpp:182-234: F(s) = 0 below -1, (1+s)^2/2 on [-1,0],
// 1-(1-s)^2/2 on [0,1], 1 above 1.
__device__ __forceinline__ float ramp(float s) {
    float c = fminf(fmaxf(s, -1.f), 1.f);
    return 0.5f + c - 0.5f * c * fabsf(c);
}

// single-instruction reciprocal and reciprocal square root (relative error ~2^-23)
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float rsqrt_approx(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ float4 lds128(uint32_t addr) {
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "r"(addr));
    return v;
}

// The PI records of a thread's TZ voxels and the view ranges derived from them.
template <int TZ>
struct VoxelRanges {
    int bi[TZ], ti[TZ];
    float bf[TZ], tf[TZ];
    int tmin, tmax;  // views this thread updates at all
    int flo, fhi;    // views where every one of its voxels has weight 1
    bool all_valid;  // every voxel has a PI interval (and the column is in the volume)
};

// loop ranges clamped to the view window [win0, win1] (BPParams)
template <int TZ>
__device__ __forceinline__ void load_ranges(const PiRecord* __restrict__ pit, size_t colbase,
                                            int zb, int NZ, int P, bool col_ok, int win0,
                                            int win1, VoxelRanges<TZ>& r) {
    r.tmin = INT_MAX; r.tmax = INT_MIN; r.flo = INT_MIN; r.fhi = INT_MAX;
    r.all_valid = col_ok;
#pragma unroll
    for (int k = 0; k < TZ; ++k) {
        const int z = zb + k;
        PiRecord q{kPiInvalid, 0.f, -10, 0.f};
        if (col_ok && z < NZ) q = pit[colbase + z];
        r.bi[k] = q.bi; r.bf[k] = q.bf; r.ti[k] = q.ti; r.tf[k] = q.tf;
        if (q.bi != kPiInvalid) {
            // loop range of KatsevichBkProj.cpp:180-181: [max(1,Bindex), min(Tindex,P-2)]
            r.tmin = min(r.tmin, max(max(1, q.bi), win0));
            r.tmax = max(r.tmax, min(min(q.ti + 1, P - 2), win1));
            r.flo = max(r.flo, q.bi + 2);  // views past both B-side ramp views
            r.fhi = min(r.fhi, q.ti - 1);  // views before both T-side ramp views
        } else {
            r.all_valid = false;
        }
    }
}

// Endpoint weight of voxel k at view p (0 when p is outside its loop range): with F the ramp,
// the reference's Coef equals F(T-p) for p >= Tindex-1 and F(p-B) otherwise.
template <int TZ>
__device__ __forceinline__ float voxel_weight(const VoxelRanges<TZ>& r, int k, int p) {
    const int d0 = p - r.bi[k];
    const int d1 = r.ti[k] + 1 - p;
    if ((d0 | d1) < 0) return 0.f;
    if (d1 <= 1) return ramp(r.tf[k] + (float)(d1 - 1));
    if (d0 <= 1) return ramp((float)d0 - r.bf[k]);
    return 1.f;
}

// the voxel's result: assigned, or added in view-window accumulation
template <typename OutT>
__device__ __forceinline__ void store_voxel(OutT* o, float v, int accum) {
    *o = accum ? *o + (OutT)v : (OutT)v;
}

}  // namespace bp
}  // namespace ctr
