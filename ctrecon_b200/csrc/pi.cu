// pi.cu -- K3: the PI-line solve for every voxel, in FP64.
//
// For voxel (X, Y, Z) inside the cylinder x^2 + y^2 < ObjR^2 the PI line's endpoints
// (sb, st) solve zz(sb) = z, where zz is the height of the chord from the helix point at
// sb to the point where it meets the helix again (KatsevichBkProj.cpp:283-312). They are
// turned into fractional view indices B, T (:177-178); the voxel is written iff
// !(B >= P-1 || T <= 0) (:180). The record keeps B and T split as integer + fraction so
// the backprojector can rebuild the reference's endpoint weights (:182-234) exactly.
//
// Solvers (ctx option CTRECON_OPT_PI_SOLVER):
//   BISECT  the reference's bisection, step for step (the judge of the others);
//   NEWTON  safeguarded Newton with the closed-form derivative inside the same bracket,
//           started at the PI line of the axis point at the same height;
//   LEARNED the same Newton started at the trained network's prediction (pinet_infer.cu).
#include "internal.h"
#include "pi_device.cuh"

namespace ctr {

__global__ void k_pi_solve(BPParams kp, double Ctr, double Beg, int solver,
                           const float* __restrict__ guess, PiRecord* __restrict__ out,
                           unsigned long long* __restrict__ count,
                           unsigned long long* __restrict__ iters_total) {
    const long long n = (long long)kp.NX * kp.NY * kp.NZ;
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    unsigned long long cnt = 0, its = 0;
    if (idx < n) {
        int xi, yi, zi;
        double X, Y, Z;
        voxel_xyz(kp, idx, &xi, &yi, &zi, &X, &Y, &Z);
        PiRecord rec{kPiInvalid, 0.f, -10, 0.f};
        if (X * X + Y * Y < kp.ObjR2) {  // KatsevichBkProj.cpp:168
            double x = X / kp.ScanR, y = Y / kp.ScanR, z = Z / kp.HelicP;  // :173-175
            double sb, st;
            if (solver == CTRECON_PI_BISECT) {
                int it = 0;
                pi_bisect(x, y, z, &sb, &st, &it);
                its = (unsigned long long)it;
            } else {
                // start: the PI line of the axis point at the same height, sb = 2 pi z - pi/2,
                // plus the learned offset when there is one
                double s0 = z * 2 * kRefPi - 0.5 * kRefPi;
                if (guess) s0 += (double)guess[idx];
                int it = 0;
                pi_newton(x, y, z, s0, &sb, &st, &it);
                its = (unsigned long long)it;
            }
            cnt = make_record(kp, Ctr, Beg, sb, st, &rec);
        }
        out[idx] = rec;
    }
    // warp reduction then one atomic per warp
    for (int o = 16; o > 0; o >>= 1) {
        cnt += __shfl_down_sync(0xffffffffu, cnt, o);
        its += __shfl_down_sync(0xffffffffu, its, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (count && cnt) atomicAdd(count, cnt);
        if (iters_total && its) atomicAdd(iters_total, its);
    }
}

// implemented in pinet_infer.cu
Status launch_pi_learned(ctrecon_ctx* ctx, cudaStream_t s, BPPlan& plan, PiRecord* d_pitab,
                         unsigned long long* d_updates, unsigned long long* d_iters);

static Status launch_solve(cudaStream_t s, BPPlan& plan, int solver, const float* guess,
                           PiRecord* d_pitab, unsigned long long* d_updates,
                           unsigned long long* d_iters) {
    const long long n = (long long)plan.kp.NX * plan.kp.NY * plan.kp.NZ;
    const int bs = 128;
    long long nb = (n + bs - 1) / bs;
    if (nb > 0x7fffffffLL) return make_status(CTRECON_ERR_UNSUPPORTED, "volume too large");
    k_pi_solve<<<(unsigned)nb, bs, 0, s>>>(plan.kp, plan.g.ProjCtr, (double)plan.g.ProjBegin,
                                           solver, guess, d_pitab, d_updates, d_iters);
    CTR_CUDA(cudaGetLastError());
    return Status::Ok();
}

// Newton from per-voxel offsets of the start point (the learned path, pinet_infer.cu)
Status launch_pi_guess(ctrecon_ctx* ctx, cudaStream_t s, BPPlan& plan, PiRecord* d_pitab,
                       unsigned long long* d_updates, unsigned long long* d_iters,
                       const float* d_guess) {
    (void)ctx;
    return launch_solve(s, plan, CTRECON_PI_LEARNED, d_guess, d_pitab, d_updates, d_iters);
}

Status launch_pi_stats(ctrecon_ctx* ctx, cudaStream_t s, BPPlan& plan, PiRecord* d_pitab,
                       unsigned long long* d_updates, unsigned long long* d_iters) {
    if (ctx->opt_pi == CTRECON_PI_LEARNED)
        return launch_pi_learned(ctx, s, plan, d_pitab, d_updates, d_iters);
    return launch_solve(s, plan, ctx->opt_pi, nullptr, d_pitab, d_updates, d_iters);
}

Status launch_pi(ctrecon_ctx* ctx, cudaStream_t s, BPPlan& plan, PiRecord* d_pitab,
                 unsigned long long* d_updates) {
    return launch_pi_stats(ctx, s, plan, d_pitab, d_updates, nullptr);
}

}  // namespace ctr
