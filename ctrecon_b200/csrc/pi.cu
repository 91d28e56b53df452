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
//   BISECT  the reference's bisection, step for step (the arbiter of the others);
//   NEWTON  safeguarded Newton with the closed-form derivative inside the same bracket,
//           started at the PI line of the axis point at the same height, then the bisection
//           replayed from Newton's root (pi_bisect_replay): the endpoints are BISECT's bit for
//           bit, for about one chord evaluation more;
//   LEARNED the same Newton started at the trained network's prediction (pinet_infer.cu).
#include "internal.h"
#include "pi_device.cuh"
#include "pinet.h"

namespace ctr {

// The learned start from the network's predictions on the (r, psi) grid (CTRECON_PINET_GRID):
// gtab[i * np + j].x = network output at r = i / rinv_step (r normalised by ScanR),
// psi = 2 pi j / np; bilinear in r and (periodic) psi.
struct PiGrid {
    const float2* tab;
    int nr, np;
    float rinv_step;
};

__global__ void k_pi_solve(BPParams kp, double Ctr, double Beg, int solver,
                           const float* __restrict__ guess, PiGrid grid,
                           PiRecord* __restrict__ out, unsigned long long* __restrict__ count,
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
                if (grid.tab) {
                    // psi = phi - 2 pi z in turns, reduced to [0, 1)
                    const float t = atan2f((float)y, (float)x) * (float)(0.5 / kRefPi) -
                                    (float)(z - floor(z));
                    const float fp = (t - floorf(t)) * (float)grid.np;
                    const float fr = fminf(sqrtf((float)(x * x + y * y)) * grid.rinv_step,
                                           (float)(grid.nr - 1) - 1e-3f);
                    const int i0 = (int)fr, j0 = min((int)fp, grid.np - 1);
                    const int j1 = j0 + 1 == grid.np ? 0 : j0 + 1;
                    const float a = fr - (float)i0, b = fp - (float)j0;
                    const float2* r0 = grid.tab + (size_t)i0 * grid.np;
                    const float2* r1 = r0 + grid.np;
                    const float o = (1.f - a) * ((1.f - b) * __ldg(&r0[j0].x) + b * __ldg(&r0[j1].x)) +
                                    a * ((1.f - b) * __ldg(&r1[j0].x) + b * __ldg(&r1[j1].x));
                    s0 += (double)(o / (float)kPinetOutScale);
                }
                // Newton finds the root; the bisection, replayed from it, decides the endpoints
                // (bit for bit those of CTRECON_PI_BISECT). Should Newton not converge, the plain
                // bisection runs instead.
                int it = 0;
                double dz = 0;
                bool conv = false;
                pi_newton(x, y, z, s0, &sb, &st, &it, &dz, &conv);
                if (conv && dz > 0) {
                    it += pi_bisect_replay(x, y, z, sb, dz, &sb, &st);
                } else {
                    int ib = 0;
                    pi_bisect(x, y, z, &sb, &st, &ib);
                    it += ib;
                }
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
                           unsigned long long* d_iters, PiGrid grid = PiGrid{nullptr, 0, 0, 0.f}) {
    const long long n = (long long)plan.kp.NX * plan.kp.NY * plan.kp.NZ;
    const int bs = 128;
    long long nb = (n + bs - 1) / bs;
    if (nb > 0x7fffffffLL) return make_status(CTRECON_ERR_UNSUPPORTED, "volume too large");
    k_pi_solve<<<(unsigned)nb, bs, 0, s>>>(plan.kp, plan.g.ProjCtr, (double)plan.g.ProjBegin,
                                           solver, guess, grid, d_pitab, d_updates, d_iters);
    CTR_CUDA(cudaGetLastError());
    return Status::Ok();
}

// Newton from per-voxel offsets of the start point (the learned path, pinet_infer.cu), or from
// the network's (r, psi) grid (d_grid: nr x np float2 outputs, r from 0 to r_max)
Status launch_pi_guess(ctrecon_ctx* ctx, cudaStream_t s, BPPlan& plan, PiRecord* d_pitab,
                       unsigned long long* d_updates, unsigned long long* d_iters,
                       const float* d_guess, const void* d_grid, int nr, int np, double r_max) {
    (void)ctx;
    PiGrid grid{static_cast<const float2*>(d_grid), nr, np,
                d_grid ? (float)((nr - 1) / r_max) : 0.f};
    return launch_solve(s, plan, CTRECON_PI_LEARNED, d_guess, d_pitab, d_updates, d_iters, grid);
}

Status launch_pi_stats(ctrecon_ctx* ctx, cudaStream_t s, BPPlan& plan, PiRecord* d_pitab,
                       unsigned long long* d_updates, unsigned long long* d_iters) {
    KernelTimer tm(ctx, s, kKPiSolve);
    if (ctx->opt_pi == CTRECON_PI_LEARNED)
        return launch_pi_learned(ctx, s, plan, d_pitab, d_updates, d_iters);
    return launch_solve(s, plan, ctx->opt_pi, nullptr, d_pitab, d_updates, d_iters);
}

Status launch_pi(ctrecon_ctx* ctx, cudaStream_t s, BPPlan& plan, PiRecord* d_pitab,
                 unsigned long long* d_updates) {
    return launch_pi_stats(ctx, s, plan, d_pitab, d_updates, nullptr);
}

}  // namespace ctr
