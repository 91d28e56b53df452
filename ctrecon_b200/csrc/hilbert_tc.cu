// hilbert_tc.cu -- the Hilbert filter of KatsevichFiltering.m:160-183 as a Toeplitz GEMM on the
// 5th-generation tensor cores (tcgen05, accumulators in TMEM), with the post-weight and the
// backward rebin (:191-284) fused into the epilogue.
//
//   D[i][n] = sum_j T[i][j] * X[n][j],  T[i][j] = h(i - j) (the Hilbert taps, zero for even
//   lags), n = (view, kappa line) rows of the chunk, i/j detector columns (padded to YLp).
//
// Tile: M = 128 output columns (TMEM lanes), N = as many whole views' kappa rows as fit in
// 256 (so every view's AL rows are in one CTA), K = YLp in blocks of 128 bytes. Operands are
// K-major, loaded by TMA with the 128-byte swizzle; one thread issues the MMAs, one thread
// the TMA loads, mbarriers chain the stages. Precision modes:
//   BF16X3: T and X split into BF16 hi + lo; D = Thi*Xhi + Thi*Xlo + Tlo*Xhi (kind::f16,
//           FP32 accumulation) -- the dropped Tlo*Xlo term is ~2^-16 relative;
//   TF32:   one kind::tf32 product of RN-rounded operands (about 2^-11 relative per term).
// Epilogue (kEpiGroups warps per TMEM lane quarter): the tile's accumulators go through a shared
// transpose buffer, then FProj[v][z][i] = gb*D[i][b] + ge*D[i][e] (the backward-rebin rows b, e
// and weights gb, ge of the host table) is gathered for all views of the tile per table entry,
// storing coalesced rows.
//
// Every mbarrier wait is bounded; a wait that gives up records an error code in a device word
// (read by the host after the call) and the CTA skips ahead, frees its TMEM and returns.
#include "internal.h"
#include "tc_util.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <vector>

namespace ctr {

namespace {

constexpr int kM = 128;
// Epilogue warps per TMEM lane quarter: the CTA has 4 * kEpiGroups warps (warps 0 and 1 also
// issue the TMA loads and the MMAs). A warp may only read the TMEM lanes of its quarter (warp % 4).
constexpr int kEpiGroups = 4;
constexpr int kThreads = 128 * kEpiGroups;

struct TcParams {
    int AL, YL, ZL, nviews, vpt, ntile, nk, ALt;  // ALt: odd row stride >= vpt * AL
    int nh;       // N halves: 1, or 2 when one view's kappa rows exceed 256 (vpt = 1)
    int bar_off;  // byte offset of the mbarriers (past the stages and the epilogue buffer)
    const BkEntry* bk;
    float* out;
    int* err;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// bounded wait (suspend-hinted try_wait, time limit): tc_util.cuh
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, int code) {
    return tcu::mbar_wait(bar, parity, err, code);
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
        "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// K-major operand tile, 128-byte rows, 128-byte swizzle: SBO = 8 rows * 128 B = 1024 B,
// LBO unused, version 1 (sm_100), layout type 2 (SWIZZLE_128B)
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)(1024u >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

template <int MODE>
__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                    uint32_t accum) {
    if constexpr (MODE == CTRECON_HILBERT_BF16X3) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(a), "l"(b), "r"(idesc), "r"(accum));
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(a), "l"(b), "r"(idesc), "r"(accum));
    }
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

__device__ __forceinline__ float tmem_ld1(uint32_t taddr) {
    uint32_t r;
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r) : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    return __uint_as_float(r);
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

template <int MODE>
__host__ __device__ constexpr int planes() { return MODE == CTRECON_HILBERT_BF16X3 ? 2 : 1; }
template <int MODE>
__host__ __device__ constexpr int stages() { return MODE == CTRECON_HILBERT_BF16X3 ? 2 : 4; }

__host__ __device__ inline uint32_t tmem_cols_for(int ntile) {
    return ntile <= 32 ? 32u : ntile <= 64 ? 64u : ntile <= 128 ? 128u : 256u;
}

template <int MODE>
__global__ void __launch_bounds__(kThreads, 1)
k_hilbert_tc(const __grid_constant__ CUtensorMap tA0, const __grid_constant__ CUtensorMap tA1,
             const __grid_constant__ CUtensorMap tB0, const __grid_constant__ CUtensorMap tB1,
             TcParams p) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    constexpr int PL = planes<MODE>();
    constexpr int S = stages<MODE>();
    const int abytes = kM * 128;
    const int bbytes = p.ntile * 128;
    const int stage_bytes = PL * (abytes + bbytes);
    uint64_t* full = (uint64_t*)(smem + p.bar_off);
    uint64_t* empty = full + S;
    uint64_t* done = empty + S;
    uint32_t* tslot = (uint32_t*)(done + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i0 = blockIdx.x * kM;
    const int vg0 = blockIdx.y * p.vpt;
    const int n0 = vg0 * p.AL;
    // with two halves, half h accumulates in TMEM columns [256 h, 256 h + ntile)
    const uint32_t ncols = p.nh == 2 ? 512u : tmem_cols_for(p.ntile);
    const int nit = p.nk * p.nh;  // pipeline steps: (K block, half)

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tslot)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    if (warp == 0 && lane == 0) {
        // TMA producer
        for (int it = 0; it < nit; ++it) {
            const int s = it % S, kb = it / p.nh, hf = it % p.nh;
            if (it >= S && !mbar_wait(&empty[s], ((it / S) - 1) & 1, p.err, 1)) break;
            uint8_t* st = smem + s * stage_bytes;
            mbar_expect_tx(&full[s], (uint32_t)stage_bytes);
            const int x = kb * (MODE == CTRECON_HILBERT_BF16X3 ? 64 : 32);
            const int nb = n0 + hf * p.ntile;
            tma_load_2d(st, &tA0, &full[s], x, i0);
            if (PL == 2) tma_load_2d(st + abytes, &tA1, &full[s], x, i0);
            tma_load_2d(st + PL * abytes, &tB0, &full[s], x, nb);
            if (PL == 2) tma_load_2d(st + PL * abytes + bbytes, &tB1, &full[s], x, nb);
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer: c = F32; a, b = BF16 (1) or TF32 (2); both K-major; N, M
        const uint32_t fmt = (MODE == CTRECON_HILBERT_BF16X3) ? 1u : 2u;
        const uint32_t idesc = (1u << 4) | (fmt << 7) | (fmt << 10) |
                               ((uint32_t)(p.ntile >> 3) << 17) | ((uint32_t)(kM >> 4) << 24);
        bool ok = true;
        for (int it = 0; it < nit; ++it) {
            const int s = it % S, kb = it / p.nh, hf = it % p.nh;
            const uint32_t td = tmem + (uint32_t)(hf * 256);
            if (!mbar_wait(&full[s], (it / S) & 1, p.err, 2)) { ok = false; break; }
            tc_fence_after();
            const uint32_t a0 = smem_u32(smem + s * stage_bytes);
            const uint32_t a1 = a0 + abytes;
            const uint32_t b0 = a0 + PL * abytes;
            const uint32_t b1 = b0 + bbytes;
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {  // four MMAs of 32 bytes of K per 128-byte block
                const uint32_t off = 32u * ks;
                const uint32_t acc = (kb > 0 || ks > 0) ? 1u : 0u;
                mma<MODE>(td, sw128_desc(a0 + off), sw128_desc(b0 + off), idesc, acc);
                if (MODE == CTRECON_HILBERT_BF16X3) {
                    mma<MODE>(td, sw128_desc(a0 + off), sw128_desc(b1 + off), idesc, 1u);
                    mma<MODE>(td, sw128_desc(a1 + off), sw128_desc(b0 + off), idesc, 1u);
                }
            }
            mma_commit(&empty[s]);
        }
        if (ok) mma_commit(done);
    }
    __syncwarp();

    // epilogue: all 4 * kEpiGroups warps. Warp w reads TMEM lanes [32 (w & 3), +32) (= output
    // columns) of its share of the tile's accumulator columns into the shared transpose buffer
    // of its lane quarter; after a barrier, each warp gathers rows z = (w >> 2), + kEpiGroups, ...
    // of every view of the tile, so each backward-rebin table entry is loaded once per tile.
    const bool have = __all_sync(0xffffffffu, mbar_wait(done, 0, p.err, 3));
    tc_fence_after();
    const int q = warp & 3, h = warp >> 2;
    const int nv = min(p.vpt, p.nviews - vg0);
    float* trq = reinterpret_cast<float*>(smem) + (size_t)q * 32 * p.ALt;
    const int i = i0 + q * 32 + lane;
    if (have) {
        const uint32_t lane_addr = tmem + ((uint32_t)(q * 32) << 16);
        // (view, column range) pieces this warp moves: per view when the tile holds several
        // views, per TMEM half when one view spans both halves
        const int npiece = p.nh == 2 ? 2 : nv;
        // work units: the 16-column chunks of every piece, then its remaining single columns,
        // dealt round-robin to the kEpiGroups warps of the lane quarter (warp-uniform test)
        int u = 0;
        for (int pc = 0; pc < npiece; ++pc) {
            const int c0 = p.nh == 2 ? pc * p.ntile : pc * p.AL;             // logical column
            const int c1 = p.nh == 2 ? min(p.AL, c0 + p.ntile) : c0 + p.AL;
            const int t0 = p.nh == 2 ? pc * 256 : c0;                        // TMEM column
            const int nfull = (c1 - c0) / 16;
            for (int m = 0; m < nfull; ++m, ++u) {
                if (u % kEpiGroups != h) continue;
                const int c = c0 + 16 * m;
                float r[16];
                tmem_ld16(lane_addr + (uint32_t)(t0 + c - c0), r);
#pragma unroll
                for (int k = 0; k < 16; ++k) trq[lane * p.ALt + c + k] = r[k];
            }
            for (int c = c0 + 16 * nfull; c < c1; ++c, ++u)
                if (u % kEpiGroups == h)
                    trq[lane * p.ALt + c] = tmem_ld1(lane_addr + (uint32_t)(t0 + c - c0));
        }
    }
    __syncthreads();
    if (have && i < p.YL) {
        const float* row = trq + lane * p.ALt;
        float* o = p.out + (size_t)vg0 * p.ZL * p.YL + i;
        const size_t vstride = (size_t)p.ZL * p.YL;
        // the table entries of kEpiRows rows are loaded (read-only path) before any of their
        // stores, so their latencies overlap instead of queueing behind the previous row's
        constexpr int kEpiRows = 8;
        const int4* bk4 = reinterpret_cast<const int4*>(p.bk);
        for (int k0 = h; k0 < p.ZL; k0 += kEpiGroups * kEpiRows) {
            int4 e[kEpiRows];
#pragma unroll
            for (int r = 0; r < kEpiRows; ++r) {
                const int k = k0 + kEpiGroups * r;
                e[r] = k < p.ZL ? __ldg(bk4 + (size_t)k * p.YL + i) : make_int4(0, 0, 0, 0);
            }
#pragma unroll
            for (int r = 0; r < kEpiRows; ++r) {
                const int k = k0 + kEpiGroups * r;
                if (k >= p.ZL) break;
                const float gb = __int_as_float(e[r].z), ge = __int_as_float(e[r].w);
                float* ok = o + (size_t)k * p.YL;
                for (int vl = 0; vl < nv; ++vl)
                    ok[vl * vstride] =
                        fmaf(gb, row[vl * p.AL + e[r].x], ge * row[vl * p.AL + e[r].y]);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(ncols)
                     : "memory");
    }
}

// ---- host side -------------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(tensor_map_encoder());
}

Status make_map(CUtensorMap* m, const void* base, bool bf16, uint64_t inner, uint64_t rows,
                uint32_t box_inner, uint32_t box_rows) {
    auto enc = get_encode();
    if (!enc) return make_status(CTRECON_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    const uint64_t esz = bf16 ? 2 : 4;
    cuuint64_t dims[2] = {inner, rows};
    cuuint64_t strides[1] = {inner * esz};
    cuuint32_t box[2] = {box_inner, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(m, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                     2, const_cast<void*>(base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return make_status(CTRECON_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return Status::Ok();
}

inline uint16_t bf16_bits_rn(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}
inline float bf16_to_float(uint16_t b) {
    uint32_t u = (uint32_t)b << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
inline float tf32_rn(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u += 0xFFFu + ((u >> 13) & 1u);
    u &= 0xFFFFE000u;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}

}  // namespace

// Toeplitz operand(s) for a plan, built on the host (FP64 taps -> BF16 hi/lo or TF32), with
// the columns in the kappa rows' de-interleaved order (the sum is over all j either way).
static Status ensure_toeplitz(FilterPlan& plan, int mode, DevBuf& T0, DevBuf& T1, int& have_mode) {
    if (have_mode == mode) return Status::Ok();
    const int YL = plan.t.YL, YLp = plan.YLp;
    const size_t n = (size_t)YLp * YLp;
    if (mode == CTRECON_HILBERT_BF16X3) {
        // columns in the kappa rows' de-interleaved order: input j sits at jd(j)
        auto jd = [&](int j) { return (size_t)((j & 1) * (YLp / 2) + (j >> 1)); };
        std::vector<uint16_t> hi(n, 0), lo(n, 0);
        for (int i = 0; i < YL; ++i)
            for (int j = 0; j < YL; ++j) {
                int m = i - j;
                if (!(m & 1)) continue;
                float v = (float)plan.t.h[(size_t)(m + YL - 1)];
                uint16_t h = bf16_bits_rn(v);
                hi[(size_t)i * YLp + jd(j)] = h;
                lo[(size_t)i * YLp + jd(j)] = bf16_bits_rn(v - bf16_to_float(h));
            }
        CTR_TRY(T0.ensure(n * 2, "Toeplitz hi"));
        CTR_TRY(T1.ensure(n * 2, "Toeplitz lo"));
        CTR_TRY(upload_now(T0.ptr, hi.data(), n * 2));
        CTR_TRY(upload_now(T1.ptr, lo.data(), n * 2));
    } else {
        auto jd = [&](int j) { return (size_t)((j & 1) * (YLp / 2) + (j >> 1)); };
        std::vector<float> t(n, 0.f);
        for (int i = 0; i < YL; ++i)
            for (int j = 0; j < YL; ++j) {
                int m = i - j;
                if (m & 1) t[(size_t)i * YLp + jd(j)] = tf32_rn((float)plan.t.h[(size_t)(m + YL - 1)]);
            }
        CTR_TRY(T0.ensure(n * 4, "Toeplitz tf32"));
        CTR_TRY(upload_now(T0.ptr, t.data(), n * 4));
    }
    have_mode = mode;
    return Status::Ok();
}

// Views per CTA tile: as many whole views' kappa rows as fit in N = 256; one view (in two
// N-halves) when a view has more than 256 kappa rows.
int hilbert_tc_views_per_tile(int AL) { return AL > 256 ? 1 : std::max(1, 256 / AL); }

Status launch_hilbert_tc(ctrecon_ctx* ctx, cudaStream_t s, FilterPlan& plan, const void* X,
                         int nviews, float* d_fproj_chunk, int mode) {
    if (ctx->opt_tc_form == CTRECON_TC_PARITY_SPLIT && hilbert_tc2_fits(plan))
        return launch_hilbert_tc2(ctx, s, plan, X, nviews, d_fproj_chunk, mode);
    const int AL = plan.t.AL, YL = plan.t.YL, ZL = plan.t.ZL, YLp = plan.YLp;
    if (AL > 512)
        return make_status(CTRECON_ERR_UNSUPPORTED,
                           "tensor-core Hilbert needs AL <= 512 kappa lines (ZL <= 392)");
    CTR_TRY(ensure_toeplitz(plan, mode, plan.tcT0, plan.tcT1, plan.tc_mode));
    if (!ctx->ws_flag.ptr) return make_status(CTRECON_ERR_INTERNAL, "device error word not set up");
    const bool bf = (mode == CTRECON_HILBERT_BF16X3);
    const int vpt = hilbert_tc_views_per_tile(AL);
    const int nh = AL > 256 ? 2 : 1;
    const int ntile = nh == 2 ? ((AL + 1) / 2 + 15) / 16 * 16 : (vpt * AL + 15) / 16 * 16;
    const uint64_t rows = (uint64_t)nviews * AL;
    const uint32_t kin = bf ? 64 : 32;
    CUtensorMap tA0, tA1, tB0, tB1;
    const size_t plane = (size_t)rows * YLp * (bf ? 2 : 4);
    CTR_TRY(make_map(&tA0, plan.tcT0.ptr, bf, YLp, YLp, kin, kM));
    CTR_TRY(make_map(&tA1, bf ? plan.tcT1.ptr : plan.tcT0.ptr, bf, YLp, YLp, kin, kM));
    CTR_TRY(make_map(&tB0, X, bf, YLp, rows, kin, ntile));
    CTR_TRY(make_map(&tB1, bf ? (const void*)((const char*)X + plane) : X, bf, YLp, rows, kin, ntile));
    TcParams p;
    p.AL = AL; p.YL = YL; p.ZL = ZL; p.nviews = nviews; p.vpt = vpt; p.ntile = ntile;
    p.nk = YLp / (int)kin;
    p.ALt = (vpt * AL) | 1;
    p.nh = nh;
    p.bk = plan.bk.as<BkEntry>();
    p.out = d_fproj_chunk;
    p.err = ctx->ws_flag.as<int>();
    const int PL = bf ? 2 : 1, S = bf ? 2 : 4;
    const size_t stage = (size_t)PL * (kM * 128 + (size_t)ntile * 128);
    const size_t epi = (size_t)4 * 32 * p.ALt * sizeof(float);
    // stages and the epilogue's transpose buffer share [0, bar_off); the mbarriers follow
    p.bar_off = (int)((std::max(S * stage, epi) + 7) / 8 * 8);
    const size_t smem = (size_t)p.bar_off + 256 + 1024;
    if (smem > 227 * 1024)
        return make_status(CTRECON_ERR_UNSUPPORTED, "tensor-core Hilbert tile exceeds shared memory");
    dim3 grid((YL + kM - 1) / kM, (nviews + vpt - 1) / vpt);
    if (bf) {
        CTR_CUDA(cudaFuncSetAttribute(k_hilbert_tc<CTRECON_HILBERT_BF16X3>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_hilbert_tc<CTRECON_HILBERT_BF16X3><<<grid, kThreads, smem, s>>>(tA0, tA1, tB0, tB1, p);
    } else {
        CTR_CUDA(cudaFuncSetAttribute(k_hilbert_tc<CTRECON_HILBERT_TF32>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_hilbert_tc<CTRECON_HILBERT_TF32><<<grid, kThreads, smem, s>>>(tA0, tA1, tB0, tB1, p);
    }
    CTR_CUDA(cudaGetLastError());
    return Status::Ok();
}

void* tensor_map_encoder() {
    static void* fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void* ptr = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = ptr;
    }
    return fn;
}

}  // namespace ctr
