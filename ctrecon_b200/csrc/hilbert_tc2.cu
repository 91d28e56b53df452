// hilbert_tc2.cu -- the Hilbert filter of KatsevichFiltering.m:160-183 on the tensor cores, with
// the post-weight and backward rebin (:181-284) fused into the epilogue: the parity-split,
// persistent form used whenever one CTA tile holds whole views (AL <= 256 kappa rows).
//
// Parity split. The Hilbert taps h(m) vanish at even lags, so an output column i only sees inputs
// j of the other parity. With i = 2i' + p and j = 2j' + (1 - p):
//     D_p[i'][n] = sum_j' T_p[i'][j'] X[n][2j' + 1 - p],   T_p[i'][j'] = h(2(i' - j') + 2p - 1),
// two half-size Toeplitz products (every tap odd, none zero) instead of one full-size product
// half of whose taps are zero: half the MMAs and half the operand bytes. The derivative kernel
// writes each kappa row de-interleaved ([even columns | odd columns], filter.cu), so the inputs
// of one parity are a contiguous half-row for the tensor copies.
//
// Tiles: (view group, 128 outputs of one parity, parity); consecutive tiles alternate parity of
// the same columns and walk the column blocks of a view group before the next group, so the
// CTAs working at one time share the group's kappa rows in L2 and write whole sectors of FProj
// between them. M = 128 outputs (TMEM lanes), N = the group's vpt*AL kappa rows (<= 256),
// K = YLp/2 in blocks of 64 bytes for BF16x3 (64-byte swizzle; five stages of the four operand
// tiles fit shared memory) or 128 bytes for TF32 (128-byte swizzle), no multicast.
//
// Persistent and warp-specialised: one CTA per SM walks tiles blockIdx.x, + gridDim.x, ...;
// warp 0 issues the tensor copies into an S-stage ring, warp 1 the MMAs into one of two TMEM
// accumulators (columns [0,256) and [256,512)), warps 2..17 drain the other accumulator, so a
// tile's epilogue overlaps the next tile's MMAs.
//
// Epilogue straight from TMEM: FProj[v][z][i] = gb*D[i][b] + ge*D[i][e] with (b, e, gb, ge) the
// backward-rebin entry of (z, i). Over the 32 outputs of a warp the rows b..e span at most a few
// kappa rows (4 at 128 x 1024, measured on the tables), so each warp reads one 4-column window
// at the warp's smallest row (tcgen05.ld 32x32b.x4, a warp-uniform address) and every lane picks
// its two values from registers; wider spans take more windows. No shared-memory transpose.
//
// Every mbarrier wait is bounded (tc_util.cuh); a wait that gives up records an error code in
// the device word and its warp stops; all warps meet before TMEM is freed.
#include "internal.h"
#include "tc_util.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstring>
#include <vector>

namespace ctr {

namespace {

using tcu::smem_u32;

constexpr int kM2 = 128;
constexpr int kEpiWarps = 16;               // four per TMEM lane quarter
constexpr int kThreads2 = 32 * (2 + kEpiWarps);
constexpr int kAccCols = 256;               // one accumulator buffer
constexpr int kRowsAhead = 4;               // backward-rebin entries loaded ahead per warp

struct Tc2Params {
    int AL, YL, ZL, nviews, vpt, ntile, YLh, YLhA, nk, ncb, ntiles, S;
    int kin;  // K elements per block (the 64- or 128-byte swizzle row)
    int stage_bytes, a_bytes, b_bytes, bar_off;
    const BkEntry* bkp;  // [ZL][2][YLhA], entry (z, p, i') of output column 2 i' + p
    float* out;
    int* err;
};

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint64_t* bar,
                                            int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
        "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

template <int MODE>
__device__ __forceinline__ void mma2(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                     uint32_t accum) {
    if constexpr (MODE == CTRECON_HILBERT_BF16X3) {
        tcu::mma_bf16(tmem_d, a, b, idesc, accum);
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(a), "l"(b), "r"(idesc), "r"(accum));
    }
}

__device__ __forceinline__ void tmem_ld4(uint32_t taddr, float& v0, float& v1, float& v2,
                                         float& v3) {
    uint32_t r0, r1, r2, r3;
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    v0 = __uint_as_float(r0);
    v1 = __uint_as_float(r1);
    v2 = __uint_as_float(r2);
    v3 = __uint_as_float(r3);
}

// K-major operand with 64-byte rows and the 64-byte swizzle: SBO = 8 rows * 64 B = 512 B,
// version 1 (sm_100), layout type 4 (SWIZZLE_64B)
__device__ __forceinline__ uint64_t sw64_desc(uint32_t saddr) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)(512u >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)4 << 61;
    return d;
}

template <int RB>
__device__ __forceinline__ uint64_t swz_desc(uint32_t saddr) {
    if constexpr (RB == 128) return tcu::sw128_desc(saddr);
    else return sw64_desc(saddr);
}

// four rows' 4-column windows in flight behind one wait (the loaded registers pass through the
// wait, so no use of them can be scheduled before it)
__device__ __forceinline__ void tmem_ld4_nowait(uint32_t taddr, uint32_t* r) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld16(uint32_t* r) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                   "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                   "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
                 :
                 : "memory");
}

__device__ __forceinline__ float pick4(int d, float v0, float v1, float v2, float v3) {
    return d == 0 ? v0 : d == 1 ? v1 : d == 2 ? v2 : v3;
}
// the same for d in [0, 3] known: two levels of selects on its bits
__device__ __forceinline__ float sel4(int d, float v0, float v1, float v2, float v3) {
    const float a = (d & 1) ? v1 : v0;
    const float b = (d & 1) ? v3 : v2;
    return (d & 2) ? b : a;
}

template <int MODE>
__host__ __device__ constexpr int planes2() { return MODE == CTRECON_HILBERT_BF16X3 ? 2 : 1; }

// tile index -> (view group, column block of one parity, parity)
__device__ __forceinline__ void tile_coords(const Tc2Params& p, int t, int& vg, int& cb, int& par) {
    par = t & 1;
    const int r = t >> 1;
    cb = r % p.ncb;
    vg = r / p.ncb;
}

template <int MODE, int RB>
__global__ void __launch_bounds__(kThreads2, 1)
k_hilbert_tc2(const __grid_constant__ CUtensorMap tA0, const __grid_constant__ CUtensorMap tA1,
              const __grid_constant__ CUtensorMap tB0, const __grid_constant__ CUtensorMap tB1,
              Tc2Params p) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    constexpr int PL = planes2<MODE>();
    const int S = p.S;
    uint64_t* full = (uint64_t*)(smem + p.bar_off);
    uint64_t* empty = full + S;
    uint64_t* accf = empty + S;   // accumulator b complete (tcgen05.commit)
    uint64_t* acce = accf + 2;    // accumulator b drained (one arrive per epilogue warp)
    uint32_t* tslot = (uint32_t*)(acce + 2);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            tcu::mbar_init(&full[s], 1);
            tcu::mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            tcu::mbar_init(&accf[b], 1);
            tcu::mbar_init(&acce[b], kEpiWarps);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tcu::tmem_alloc(tslot, 2 * kAccCols);
    tcu::fence_before();
    __syncthreads();
    tcu::fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t kin = (uint32_t)p.kin;  // K elements per block of RB bytes

    if (warp == 0) {
        // ---- tensor copies -------------------------------------------------------------------
        if (lane == 0) {
            int it = 0;
            bool ok = true;
            for (int t = blockIdx.x; ok && t < p.ntiles; t += gridDim.x) {
                int vg, cb, par;
                tile_coords(p, t, vg, cb, par);
                const int arow = par * p.YLhA + cb * kM2;      // rows of T_par
                const int brow = vg * p.vpt * p.AL;             // first kappa row of the group
                const int bx0 = (1 - par) * p.YLh;              // inputs of the other parity
                for (int kb = 0; kb < p.nk; ++kb, ++it) {
                    const int s = it % S;
                    if (it >= S && !tcu::mbar_wait(&empty[s], ((it / S) - 1) & 1, p.err, 21)) {
                        ok = false;
                        break;
                    }
                    const uint32_t st = smem_u32(smem + (size_t)s * p.stage_bytes);
                    expect_tx(&full[s], (uint32_t)p.stage_bytes);
                    const int x = kb * (int)kin;
                    tma_load_2d(st, &tA0, &full[s], x, arow);
                    if (PL == 2) tma_load_2d(st + p.a_bytes, &tA1, &full[s], x, arow);
                    tma_load_2d(st + PL * p.a_bytes, &tB0, &full[s], bx0 + x, brow);
                    if (PL == 2)
                        tma_load_2d(st + PL * p.a_bytes + p.b_bytes, &tB1, &full[s], bx0 + x, brow);
                }
            }
            if (!ok)  // a wait gave up: let the copies still in flight land before the CTA exits
                for (int j = (it > S ? it - S : 0); j < it; ++j)
                    tcu::mbar_drain(&full[j % S], (j / S) & 1);
        }
    } else if (warp == 1) {
        // ---- MMA issue -------------------------------------------------------------------------
        if (lane == 0) {
            const uint32_t fmt = (MODE == CTRECON_HILBERT_BF16X3) ? 1u : 2u;
            const uint32_t idesc = (1u << 4) | (fmt << 7) | (fmt << 10) |
                                   ((uint32_t)(p.ntile >> 3) << 17) |
                                   ((uint32_t)(kM2 >> 4) << 24);
            int it = 0, u = 0;
            bool ok = true;
            for (int t = blockIdx.x; ok && t < p.ntiles; t += gridDim.x, ++u) {
                const int b = u & 1;
                if (u >= 2 && !tcu::mbar_wait(&acce[b], ((u >> 1) - 1) & 1, p.err, 22)) break;
                tcu::fence_after();
                const uint32_t td = tmem + (uint32_t)(b * kAccCols);
                for (int kb = 0; kb < p.nk; ++kb, ++it) {
                    const int s = it % S;
                    if (!tcu::mbar_wait_poll(&full[s], (it / S) & 1, p.err, 23)) {
                        ok = false;
                        break;
                    }
                    tcu::fence_after();
                    const uint32_t a0 = smem_u32(smem + (size_t)s * p.stage_bytes);
                    const uint32_t a1 = a0 + p.a_bytes;
                    const uint32_t b0 = a0 + PL * p.a_bytes;
                    const uint32_t b1 = b0 + p.b_bytes;
#pragma unroll
                    for (int ks = 0; ks < RB / 32; ++ks) {  // 32 bytes of K per MMA
                        const uint32_t off = 32u * ks;
                        const uint32_t acc = (kb > 0 || ks > 0) ? 1u : 0u;
                        mma2<MODE>(td, swz_desc<RB>(a0 + off), swz_desc<RB>(b0 + off), idesc, acc);
                        if (MODE == CTRECON_HILBERT_BF16X3) {
                            mma2<MODE>(td, swz_desc<RB>(a0 + off), swz_desc<RB>(b1 + off), idesc, 1u);
                            mma2<MODE>(td, swz_desc<RB>(a1 + off), swz_desc<RB>(b0 + off), idesc, 1u);
                        }
                    }
                    tcu::mma_commit(&empty[s]);
                }
                if (ok) tcu::mma_commit(&accf[b]);
            }
        }
    } else {
        // ---- epilogue: backward rebin straight from TMEM -----------------------------------
        const int q = warp & 3;             // TMEM lane quarter this warp may read
        const int h = (warp - 2) >> 2;      // which quarter of the detector rows
        const uint32_t lane_base = tmem + ((uint32_t)(q * 32) << 16);
        const size_t vstride = (size_t)p.ZL * p.YL;
        const int4* bk4 = reinterpret_cast<const int4*>(p.bkp);
        int u = 0;
        for (int t = blockIdx.x; t < p.ntiles; t += gridDim.x, ++u) {
            const int b = u & 1;
            if (!tcu::mbar_wait(&accf[b], (u >> 1) & 1, p.err, 24)) break;
            tcu::fence_after();
            int vg, cb, par;
            tile_coords(p, t, vg, cb, par);
            const int ip = cb * kM2 + q * 32 + lane;      // output index within the parity
            const int i = 2 * ip + par;                   // detector column
            const bool valid = ip < p.YLh && i < p.YL;
            const int nv = min(p.vpt, p.nviews - vg * p.vpt);
            const int4* bkrow = bk4 + (size_t)par * p.YLhA + ip;
            const size_t zstride = (size_t)2 * p.YLhA;
            const uint32_t acc_base = lane_base + (uint32_t)(b * kAccCols);
            // the entries of the next kRowsAhead rows are loaded while this batch is processed
            int4 enext[kRowsAhead];
#pragma unroll
            for (int r = 0; r < kRowsAhead; ++r) {
                const int k = h + 4 * r;
                enext[r] = k < p.ZL ? __ldg(bkrow + (size_t)k * zstride) : make_int4(0, 0, 0, 0);
            }
            for (int k0 = h; k0 < p.ZL; k0 += 4 * kRowsAhead) {
                int4 e[kRowsAhead];
#pragma unroll
                for (int r = 0; r < kRowsAhead; ++r) {
                    e[r] = enext[r];
                    const int k = k0 + 4 * kRowsAhead + 4 * r;
                    enext[r] = k < p.ZL ? __ldg(bkrow + (size_t)k * zstride) : make_int4(0, 0, 0, 0);
                }
                // rows past ZL (warp-uniform) read a harmless window and store nothing
                int lo[kRowsAhead], hi[kRowsAhead];
#pragma unroll
                for (int r = 0; r < kRowsAhead; ++r) {
                    lo[r] = (int)__reduce_min_sync(0xffffffffu, (unsigned)min(e[r].x, e[r].y));
                    hi[r] = (int)__reduce_max_sync(0xffffffffu, (unsigned)max(e[r].x, e[r].y));
                }
                // every row of the batch spans at most four kappa rows over the warp (the usual
                // case): one window per row, selects without range checks
                bool narrow = true;
#pragma unroll
                for (int r = 0; r < kRowsAhead; ++r) narrow = narrow && hi[r] - lo[r] < 4;
                for (int vl = 0; vl < nv && narrow; ++vl) {
                    const int cbase = vl * p.AL;  // this view's first accumulator column
                    float* ov = p.out + (size_t)(vg * p.vpt + vl) * vstride + (size_t)k0 * p.YL + i;
                    const size_t rstep = (size_t)4 * p.YL;  // rows k0, k0 + 4, ... of this warp
#pragma unroll
                    for (int r4 = 0; r4 < kRowsAhead; r4 += 4) {
                        uint32_t w[16];
                        int c0[4];
#pragma unroll
                        for (int r = 0; r < 4; ++r) {
                            c0[r] = min(cbase + lo[r4 + r], kAccCols - 4);
                            tmem_ld4_nowait(acc_base + (uint32_t)c0[r], w + 4 * r);
                        }
                        tmem_wait_ld16(w);
#pragma unroll
                        for (int r = 0; r < 4; ++r) {
                            const int k = k0 + 4 * (r4 + r);
                            const int4 er = e[r4 + r];
                            const int db = cbase + er.x - c0[r], de = cbase + er.y - c0[r];
                            const float v0 = __uint_as_float(w[4 * r]);
                            const float v1 = __uint_as_float(w[4 * r + 1]);
                            const float v2 = __uint_as_float(w[4 * r + 2]);
                            const float v3 = __uint_as_float(w[4 * r + 3]);
                            const float vb = sel4(db, v0, v1, v2, v3);
                            const float ve = sel4(de, v0, v1, v2, v3);
                            if (valid && k < p.ZL)
                                ov[(size_t)(r4 + r) * rstep] =
                                    fmaf(__int_as_float(er.z), vb, __int_as_float(er.w) * ve);
                        }
                    }
                }
                for (int vl = 0; vl < nv && !narrow; ++vl) {
                    const int cbase = vl * p.AL;  // this view's first accumulator column
#pragma unroll
                    for (int r4 = 0; r4 < kRowsAhead; r4 += 4) {
                        // the first 4-column window of four rows (kept inside the 256-column
                        // buffer), one wait for all four
                        uint32_t w[16];
                        int c0[4];
#pragma unroll
                        for (int r = 0; r < 4; ++r) {
                            c0[r] = min(cbase + lo[r4 + r], kAccCols - 4);
                            tmem_ld4_nowait(acc_base + (uint32_t)c0[r], w + 4 * r);
                        }
                        tmem_wait_ld16(w);
#pragma unroll
                        for (int r = 0; r < 4; ++r) {
                            const int k = k0 + 4 * (r4 + r);
                            const int4 er = e[r4 + r];
                            const int db = cbase + er.x - c0[r], de = cbase + er.y - c0[r];
                            const float v0 = __uint_as_float(w[4 * r]);
                            const float v1 = __uint_as_float(w[4 * r + 1]);
                            const float v2 = __uint_as_float(w[4 * r + 2]);
                            const float v3 = __uint_as_float(w[4 * r + 3]);
                            float vb = (db >= 0 && db < 4) ? pick4(db, v0, v1, v2, v3) : 0.f;
                            float ve = (de >= 0 && de < 4) ? pick4(de, v0, v1, v2, v3) : 0.f;
                            // rows spanning more than four kappa rows (warp-uniform): more windows
                            for (int ww = lo[r4 + r] + 4; ww <= hi[r4 + r]; ww += 4) {
                                const int cw = min(cbase + ww, kAccCols - 4);
                                float u0, u1, u2, u3;
                                tmem_ld4(acc_base + (uint32_t)cw, u0, u1, u2, u3);
                                const int db2 = cbase + er.x - cw, de2 = cbase + er.y - cw;
                                if (db2 >= 0 && db2 < 4) vb = pick4(db2, u0, u1, u2, u3);
                                if (de2 >= 0 && de2 < 4) ve = pick4(de2, u0, u1, u2, u3);
                            }
                            if (valid && k < p.ZL)
                                p.out[(size_t)(vg * p.vpt + vl) * vstride + (size_t)k * p.YL + i] =
                                    fmaf(__int_as_float(er.z), vb, __int_as_float(er.w) * ve);
                        }
                    }
                }
            }
            tcu::fence_before();
            __syncwarp();
            if (lane == 0) arrive(&acce[b]);
        }
    }
    tcu::fence_before();
    __syncthreads();
    if (warp == 0) tcu::tmem_dealloc(tmem, 2 * kAccCols);
}

Status make_map2(CUtensorMap* m, const void* base, bool bf16, uint64_t inner, uint64_t rows,
                 uint64_t row_stride_elems, uint32_t box_inner, uint32_t box_rows, int row_bytes) {
    auto enc = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(tensor_map_encoder());
    if (!enc) return make_status(CTRECON_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    const uint64_t esz = bf16 ? 2 : 4;
    cuuint64_t dims[2] = {inner, rows};
    cuuint64_t strides[1] = {row_stride_elems * esz};
    cuuint32_t box[2] = {box_inner, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(m, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                     2, const_cast<void*>(base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE,
                     row_bytes == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return make_status(CTRECON_ERR_CUDA,
                           "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return Status::Ok();
}

inline uint16_t bf16_rn_bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}
inline float bf16_bits_to_float(uint16_t b) {
    uint32_t u = (uint32_t)b << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
inline float tf32_round(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u += 0xFFFu + ((u >> 13) & 1u);
    u &= 0xFFFFE000u;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}

int sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1)
            n = 148;
    }
    return n;
}

}  // namespace

// The parity-split Toeplitz operands T_0, T_1 stacked as [2 * YLhA][YLh] (rows of T_p start at
// p * YLhA; rows beyond YLh are zero) and the backward-rebin table by parity, [ZL][2][YLhA]
// (columns past the detector repeat the last real column's rows with zero weights, so that a
// warp's row window stays narrow).
static Status ensure_tc2_operands(FilterPlan& plan, int mode) {
    if (plan.tc2_mode == mode) return Status::Ok();
    const FilterTables& t = plan.t;
    const int YL = t.YL, ZL = t.ZL, YLh = plan.YLp / 2;
    const int YLhA = (YLh + kM2 - 1) / kM2 * kM2;
    const size_t n = (size_t)2 * YLhA * YLh;
    auto tap = [&](int p, int ip, int jp) -> float {
        const int i = 2 * ip + p, j = 2 * jp + 1 - p;
        if (ip >= YLh || i >= YL || j >= YL) return 0.f;
        return (float)t.h[(size_t)(i - j + YL - 1)];
    };
    if (mode == CTRECON_HILBERT_BF16X3) {
        std::vector<uint16_t> hi(n, 0), lo(n, 0);
        for (int p = 0; p < 2; ++p)
            for (int ip = 0; ip < YLhA; ++ip)
                for (int jp = 0; jp < YLh; ++jp) {
                    const float v = tap(p, ip, jp);
                    const size_t k = ((size_t)p * YLhA + ip) * YLh + jp;
                    const uint16_t hb = bf16_rn_bits(v);
                    hi[k] = hb;
                    lo[k] = bf16_rn_bits(v - bf16_bits_to_float(hb));
                }
        CTR_TRY(plan.tc2T0.ensure(n * 2, "Toeplitz halves hi"));
        CTR_TRY(plan.tc2T1.ensure(n * 2, "Toeplitz halves lo"));
        CTR_TRY(upload_now(plan.tc2T0.ptr, hi.data(), n * 2));
        CTR_TRY(upload_now(plan.tc2T1.ptr, lo.data(), n * 2));
    } else {
        std::vector<float> tv(n, 0.f);
        for (int p = 0; p < 2; ++p)
            for (int ip = 0; ip < YLhA; ++ip)
                for (int jp = 0; jp < YLh; ++jp)
                    tv[((size_t)p * YLhA + ip) * YLh + jp] = tf32_round(tap(p, ip, jp));
        CTR_TRY(plan.tc2T0.ensure(n * 4, "Toeplitz halves tf32"));
        CTR_TRY(upload_now(plan.tc2T0.ptr, tv.data(), n * 4));
    }
    if (!plan.bkp_ready) {
        std::vector<BkEntry> bkp((size_t)ZL * 2 * YLhA);
        for (int z = 0; z < ZL; ++z)
            for (int p = 0; p < 2; ++p) {
                const int last = ((YL - 1 - p) / 2) * 2 + p;  // last real column of parity p
                for (int ip = 0; ip < YLhA; ++ip) {
                    const int i = 2 * ip + p;
                    const size_t src = (size_t)z * YL + (i < YL ? i : last);
                    BkEntry e{t.b[src], t.e[src], (float)t.gb[src], (float)t.ge[src]};
                    if (i >= YL) e.gb = e.ge = 0.f;
                    bkp[((size_t)z * 2 + p) * YLhA + ip] = e;
                }
            }
        CTR_TRY(plan.bkp.ensure(bkp.size() * sizeof(BkEntry), "backward-rebin table by parity"));
        CTR_TRY(upload_now(plan.bkp.ptr, bkp.data(), bkp.size() * sizeof(BkEntry)));
        plan.bkp_ready = true;
    }
    plan.tc2_mode = mode;
    return Status::Ok();
}

// Whether launch_hilbert_tc2 handles the plan: whole views per tile (AL <= 256), two rows of
// columns per parity fit its shared memory.
bool hilbert_tc2_fits(const FilterPlan& plan) { return plan.t.AL <= 256 && plan.t.YL >= 2; }

Status launch_hilbert_tc2(ctrecon_ctx* ctx, cudaStream_t s, FilterPlan& plan, const void* X,
                          int nviews, float* d_fproj_chunk, int mode) {
    const int AL = plan.t.AL, YL = plan.t.YL, ZL = plan.t.ZL, YLp = plan.YLp;
    if (!hilbert_tc2_fits(plan) || (YLp % 128) != 0)
        return make_status(CTRECON_ERR_INTERNAL, "parity-split Hilbert: unsupported shape");
    CTR_TRY(ensure_tc2_operands(plan, mode));
    if (!ctx->ws_flag.ptr) return make_status(CTRECON_ERR_INTERNAL, "device error word not set up");
    const bool bf = (mode == CTRECON_HILBERT_BF16X3);
    const int vpt = hilbert_tc_views_per_tile(AL);
    const int ntile = (vpt * AL + 15) / 16 * 16;
    const int YLh = YLp / 2, YLhA = (YLh + kM2 - 1) / kM2 * kM2;
    // BF16x3 stages hold four operand tiles: 64-byte rows (32 elements of K) let five stages fit
    // where 128-byte rows let two; TF32 keeps 128-byte rows (32 elements, one plane)
    const int RB = bf ? 64 : 128;
    const uint32_t kin = (uint32_t)RB / (bf ? 2 : 4);
    const uint64_t rows = (uint64_t)nviews * AL;
    const size_t plane = (size_t)rows * YLp * (bf ? 2 : 4);
    CUtensorMap tA0, tA1, tB0, tB1;
    CTR_TRY(make_map2(&tA0, plan.tc2T0.ptr, bf, YLh, (uint64_t)2 * YLhA, YLh, kin, kM2, RB));
    CTR_TRY(make_map2(&tA1, bf ? plan.tc2T1.ptr : plan.tc2T0.ptr, bf, YLh, (uint64_t)2 * YLhA, YLh,
                      kin, kM2, RB));
    CTR_TRY(make_map2(&tB0, X, bf, YLp, rows, YLp, kin, ntile, RB));
    CTR_TRY(make_map2(&tB1, bf ? (const void*)((const char*)X + plane) : X, bf, YLp, rows, YLp,
                      kin, ntile, RB));
    Tc2Params p;
    p.AL = AL; p.YL = YL; p.ZL = ZL; p.nviews = nviews; p.vpt = vpt; p.ntile = ntile;
    p.YLh = YLh; p.YLhA = YLhA;
    p.nk = YLh / (int)kin;
    p.kin = (int)kin;
    p.ncb = YLhA / kM2;
    const int nvg = (nviews + vpt - 1) / vpt;
    p.ntiles = nvg * p.ncb * 2;
    const int PL = bf ? 2 : 1;
    p.a_bytes = kM2 * RB;
    p.b_bytes = ntile * RB;
    p.stage_bytes = PL * (p.a_bytes + p.b_bytes);
    const size_t budget = 227 * 1024 - 1024 - 256;  // alignment slack and barriers
    p.S = (int)std::min<size_t>(6, budget / (size_t)p.stage_bytes);
    if (p.S < 2)
        return make_status(CTRECON_ERR_UNSUPPORTED, "parity-split Hilbert stage exceeds shared memory");
    p.bar_off = p.S * p.stage_bytes;
    p.bkp = plan.bkp.as<BkEntry>();
    p.out = d_fproj_chunk;
    p.err = ctx->ws_flag.as<int>();
    const size_t smem = (size_t)p.bar_off + 256 + 1024;
    const int grid = std::min(p.ntiles, sm_count());
    if (bf) {
        CTR_CUDA(cudaFuncSetAttribute(k_hilbert_tc2<CTRECON_HILBERT_BF16X3, 64>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_hilbert_tc2<CTRECON_HILBERT_BF16X3, 64><<<grid, kThreads2, smem, s>>>(tA0, tA1, tB0, tB1, p);
    } else {
        CTR_CUDA(cudaFuncSetAttribute(k_hilbert_tc2<CTRECON_HILBERT_TF32, 128>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_hilbert_tc2<CTRECON_HILBERT_TF32, 128><<<grid, kThreads2, smem, s>>>(tA0, tA1, tB0, tB1, p);
    }
    CTR_CUDA(cudaGetLastError());
    return Status::Ok();
}

}  // namespace ctr
