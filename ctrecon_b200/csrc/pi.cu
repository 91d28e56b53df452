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
//   NEWTON  safeguarded Newton on g(sb) = zz(sb) - z inside the same bracket, started at
//           the bracket midpoint (or at the learned initial guess, pinet.cu), stopped at
//           the same tolerances.
#include "internal.h"

namespace ctr {

constexpr double kPiTol = 0.0000001;  // DeltaMax, KatsevichBkProj.cpp:26

// chord of the PI line starting at sb: returns zz(sb) and st(sb)
__device__ __forceinline__ double pi_chord(double x, double y, double r2, double sb,
                                           double* st_out) {
    const double PI = kRefPi;
    double ssb, csb;
    sincos(sb, &ssb, &csb);
    double tempcos = 2 * (1 - y * ssb - x * csb);
    double t = (1 - r2) / tempcos;
    double templan = acos((y * csb - x * ssb) / sqrt(tempcos + r2 - 1));
    double st = 2 * templan + sb;
    *st_out = st;
    return (sb * t + (1 - t) * st) / (2 * PI);
}

__device__ void pi_bisect(double x, double y, double z, double* B, double* T) {
    const double PI = kRefPi;
    double delta = 1, bmax = z * 2 * PI, bmin, r2 = x * x + y * y;
    bmin = bmax - 2 * PI;
    double sb = 0, st = 0;
    while (((bmax - bmin) > kPiTol) && (delta > kPiTol)) {
        sb = (bmax + bmin) * 0.5;
        double zz = pi_chord(x, y, r2, sb, &st);
        if (zz < z) bmin = sb;
        else bmax = sb;
        delta = fabs(zz - z);
    }
    *B = sb;
    *T = st;
}

// Newton with a bisection safeguard: the iterate stays inside [bmin, bmax], which shrinks
// with the sign of g; the derivative is a central difference (g is smooth and monotone).
__device__ void pi_newton(double x, double y, double z, double s0, double* B, double* T,
                          int* iters) {
    const double PI = kRefPi;
    double bmax = z * 2 * PI, bmin = bmax - 2 * PI, r2 = x * x + y * y;
    double sb = (s0 > bmin && s0 < bmax) ? s0 : 0.5 * (bmin + bmax);
    double st = 0;
    int it = 0;
    for (; it < 60; ++it) {
        double zz = pi_chord(x, y, r2, sb, &st);
        double g = zz - z;
        if (fabs(g) <= kPiTol) break;
        if (g < 0) bmin = sb;
        else bmax = sb;
        if (bmax - bmin <= kPiTol) break;
        const double h = 1e-6;
        double stp, stm;
        double gp = pi_chord(x, y, r2, sb + h, &stp);
        double gm = pi_chord(x, y, r2, sb - h, &stm);
        double d = (gp - gm) / (2 * h);
        double nx = sb - g / d;
        if (!(d > 0) || !(nx > bmin && nx < bmax)) nx = 0.5 * (bmin + bmax);
        sb = nx;
    }
    *B = sb;
    *T = st;
    if (iters) *iters = it + 1;
}

__device__ __forceinline__ void voxel_xyz(const BPParams& kp, long long idx, int* xi, int* yi,
                                          int* zi, double* X, double* Y, double* Z) {
    int z = (int)(idx % kp.NZ);
    long long r = idx / kp.NZ;
    int y = (int)(r % kp.NY);
    int x = (int)(r / kp.NY);
    *xi = x; *yi = y; *zi = z;
    *X = (x - kp.XC) * kp.dx;  // KatsevichBkProj.cpp:142-147
    *Y = (y - kp.YC) * kp.dy;
    *Z = (z - kp.ZC) * kp.dz;
}

// record + loop count from (sb, st), KatsevichBkProj.cpp:177-234
__device__ __forceinline__ unsigned long long make_record(const BPParams& kp, double Ctr,
                                                          double Beg, double sb, double st,
                                                          PiRecord* rec) {
    double Bv = sb / kp.DeltaL + Ctr - Beg;
    double Tv = st / kp.DeltaL + Ctr - Beg;
    const int P = kp.P;
    if ((Bv >= P - 1) || (Tv <= 0)) {
        rec->bi = kPiInvalid; rec->bf = 0.f; rec->ti = -10; rec->tf = 0.f;
        return 0ull;
    }
    int Bindex = (int)(Bv + 10) - 10;
    int Tindex = (int)(Tv + 10) - 9;
    int LB = Bindex < 1 ? 1 : Bindex;
    int LE = Tindex > P - 2 ? P - 2 : Tindex;
    rec->bi = Bindex;
    rec->bf = (float)(Bv - Bindex);
    rec->ti = Tindex - 1;
    rec->tf = (float)(Tv - (Tindex - 1));
    return (unsigned long long)(LE - LB + 1);
}

__global__ void k_pi_solve(BPParams kp, double Ctr, double Beg, int solver,
                           const float2* __restrict__ guess, PiRecord* __restrict__ out,
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
                pi_bisect(x, y, z, &sb, &st);
                its = 27;
            } else {
                double s0 = -1e300;
                if (guess) s0 = (double)guess[idx].x + z * 2 * kRefPi;
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

Status launch_pi_solver(ctrecon_ctx* ctx, cudaStream_t s, BPPlan& plan, PiRecord* d_pitab,
                        unsigned long long* d_updates, int solver, const float2* d_guess,
                        unsigned long long* d_iters) {
    (void)ctx;
    const long long n = (long long)plan.kp.NX * plan.kp.NY * plan.kp.NZ;
    const int bs = 128;
    long long nb = (n + bs - 1) / bs;
    if (nb > 0x7fffffffLL) return make_status(CTRECON_ERR_UNSUPPORTED, "volume too large");
    k_pi_solve<<<(unsigned)nb, bs, 0, s>>>(plan.kp, plan.g.ProjCtr, (double)plan.g.ProjBegin,
                                           solver, d_guess, d_pitab, d_updates, d_iters);
    CTR_CUDA(cudaGetLastError());
    return Status::Ok();
}

Status launch_pi(ctrecon_ctx* ctx, cudaStream_t s, BPPlan& plan, PiRecord* d_pitab,
                 unsigned long long* d_updates) {
    int solver = ctx->opt_pi;
    if (solver == CTRECON_PI_LEARNED) solver = CTRECON_PI_NEWTON;  // guess wired in pinet.cu
    return launch_pi_solver(ctx, s, plan, d_pitab, d_updates, solver, nullptr, nullptr);
}

}  // namespace ctr
