// pi_device.cuh -- FP64 device functions of the PI-line solve (KatsevichBkProj.cpp:283-312),
// shared by the plain solver (pi.cu), the training-pair generator (pinet.cu) and the learned
// solver (pinet_infer.cu).
#pragma once

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

__device__ __forceinline__ void pi_bisect(double x, double y, double z, double* B, double* T,
                                          int* iters) {
    const double PI = kRefPi;
    double delta = 1, bmax = z * 2 * PI, bmin, r2 = x * x + y * y;
    bmin = bmax - 2 * PI;
    double sb = 0, st = 0;
    int it = 0;
    // the reference's loop test ((bmax - bmin) > DeltaMax) && (delta > DeltaMax): the bracket
    // starts 2 pi wide and halves each step, so its width test holds for the first 25 steps
    // (2 pi / 2^25 > 1e-7) and is only evaluated from then on
    while ((it < 25 || (bmax - bmin) > kPiTol) && (delta > kPiTol)) {
        sb = (bmax + bmin) * 0.5;
        double zz = pi_chord(x, y, r2, sb, &st);
        if (zz < z) bmin = sb;
        else bmax = sb;
        delta = fabs(zz - z);
        ++it;
    }
    *B = sb;
    *T = st;
    *iters = it;
}

// zz(sb), st(sb) and d zz / d sb in closed form. With s = sin sb, c = cos sb:
//   tempcos = 2(1 - y s - x c), t = (1 - r^2)/tempcos, n = y c - x s, q = tempcos + r^2 - 1,
//   w = n / sqrt(q), st = sb + 2 acos(w), zz = (sb t + (1 - t) st) / 2pi;
//   d tempcos = -2n, dt = 2(1 - r^2) n / tempcos^2, dn = tempcos/2 - 1,
//   dw = (dn q + n^2) / q^(3/2), dst = 1 - 2 dw / sqrt(1 - w^2),
//   dzz = (t + (1 - t) dst + dt (sb - st)) / 2pi.
// One reciprocal and two reciprocal square roots per evaluation (each FP64 division or
// square root costs a quarter-rate seed instruction plus refinement).
__device__ __forceinline__ double pi_chord_d(double x, double y, double r2, double sb,
                                             double* st_out, double* dst_out, double* dzz) {
    const double inv2pi = 1.0 / (2 * kRefPi);
    double s, c;
    sincos(sb, &s, &c);
    const double tempcos = 2 * (1 - y * s - x * c);
    const double itc = 1.0 / tempcos;
    const double t = (1 - r2) * itc;
    const double n = y * c - x * s;
    const double q = tempcos + r2 - 1;
    const double rq = rsqrt(q);
    const double w = n * rq;
    const double st = 2 * acos(w) + sb;
    const double dt = 2 * (1 - r2) * n * itc * itc;
    const double dn = 0.5 * tempcos - 1;
    const double dw = (dn * q + n * n) * (rq * rq * rq);
    const double dst = 1 - 2 * dw * rsqrt(fmax(1 - w * w, 1e-300));
    *st_out = st;
    *dst_out = dst;
    *dzz = (t + (1 - t) * dst + dt * (sb - st)) * inv2pi;
    return (sb * t + (1 - t) * st) * inv2pi;
}

// Newton with a bisection safeguard: the iterate stays inside the reference's bracket
// [2 pi z - 2 pi, 2 pi z], which shrinks with the sign of g = zz - z (zz increases with sb);
// a step leaving the bracket is replaced by its midpoint. Once a step is below 1e-6 rad the
// stepped point is accepted without another evaluation (its error is ~step^2 < 1e-12 rad) and
// st follows it along dst; both are then well inside the reference's 1e-7 bisection tolerance.
__device__ __forceinline__ void pi_newton(double x, double y, double z, double s0, double* B,
                                          double* T, int* iters, double* dz_out = nullptr,
                                          bool* converged = nullptr) {
    const double PI = kRefPi;
    double bmax = z * 2 * PI, bmin = bmax - 2 * PI;
    const double r2 = x * x + y * y;
    double sb = (s0 > bmin && s0 < bmax) ? s0 : 0.5 * (bmin + bmax);
    double st = 0, dst = 0, d = 0;
    int it = 0;
    for (; it < 60; ++it) {
        const double g = pi_chord_d(x, y, r2, sb, &st, &dst, &d) - z;
        if (g < 0) bmin = sb;
        else bmax = sb;
        double nx = sb - g / d;
        const bool newton = (d > 0) && (nx > bmin && nx < bmax);
        if (!newton) nx = 0.5 * (bmin + bmax);
        const double step = nx - sb;
        if (newton && fabs(step) < 1e-6) {
            st += dst * step;
            sb = nx;
            if (converged) *converged = true;
            break;
        }
        sb = nx;
    }
    *B = sb;
    *T = st;
    if (dz_out) *dz_out = d;
    if (iters) *iters = it + 1;
}

// The reference's bisection (pi_bisect, KatsevichBkProj.cpp:291-309) replayed from a root.
// Given tau, a root of zz(sb) = z accurate to ~1e-12 rad (Newton's), and dz = dzz/dsb near it,
// every midpoint's decisions follow from sb - tau: zz(sb) < z iff sb < tau (zz increases with
// sb), and the stop test |zz(sb) - z| <= 1e-7 is that of |dz (sb - tau)| (the linear model's
// error there is ~1e-12, far below the bisection's 1e-7). The chord is evaluated exactly -- the
// same pi_chord call as the bisection's -- only where either decision lies within 1e-10 of its
// threshold, and once at the final midpoint for st. The midpoints are the bisection's own
// arithmetic, so (sb, st) equal pi_bisect's bit for bit: the bisection still decides the
// endpoints, Newton only finds where it will end. Returns the chord evaluations made (~1).
__device__ __forceinline__ int pi_bisect_replay(double x, double y, double z, double tau,
                                                double dz, double* B, double* T) {
    const double PI = kRefPi;
    constexpr double kMargin = 1e-10;
    double delta = 1, bmax = z * 2 * PI, bmin, r2 = x * x + y * y;
    bmin = bmax - 2 * PI;
    double sb = 0, st = 0;
    bool have_st = false;
    int ev = 0;
    // the width test holds for the first 25 steps (as in pi_bisect)
    for (int it = 0; (it < 25 || (bmax - bmin) > kPiTol) && (delta > kPiTol); ++it) {
        sb = (bmax + bmin) * 0.5;
        const double dl = sb - tau;
        double g = dz * dl;  // ~ zz(sb) - z
        have_st = false;
        if (fabs(dl) < kMargin || fabs(fabs(g) - kPiTol) < kMargin) {
            g = pi_chord(x, y, r2, sb, &st) - z;
            have_st = true;
            ++ev;
        }
        if (g < 0) bmin = sb;
        else bmax = sb;
        delta = fabs(g);
    }
    if (!have_st) {
        pi_chord(x, y, r2, sb, &st);
        ++ev;
    }
    *B = sb;
    *T = st;
    return ev;
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

}  // namespace ctr
