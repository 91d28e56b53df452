// phantom.cu -- analytic cone-beam projections of a set of ellipsoids, FP64 on the device.
//
// The chord length of the ray from the source S through a detector cell inside an
// ellipsoid is 2*sqrt(B^2 - A*C)/A with A, B, C the coefficients of the quadratic of the
// ray in the ellipsoid's body frame (CreateProjSlice.cpp:98-134). Here the ellipsoids have
// general ZXZ orientations and the detector is flat at distance StdDis, cells centred on
// ((y-(YL-1)/2)*DecWidth/YL, (z-(ZL-1)/2)*DecHeigh/ZL); source angle of view p is
// (p + ProjBeginIndex - ProjCtr)*2*pi/ProjScale as in FunctionKat_v6.m:71.
//
// Optional Poisson noise: counts I ~ Poisson(N0 exp(-mu p)) with mu = 8 / max(p), then
// p~ = -ln(max(I,1)/N0)/mu. Counts are drawn from a counter-based generator keyed by
// (seed, ray index): exact inversion for means below 64, the normal approximation above.
#include "internal.h"

namespace ctr {

struct EllDev {
    double c[3];      // centre
    double m[9];      // rotation, row-major (body = m^T (p - c))
    double ia2[3];    // 1/a^2, 1/b^2, 1/c^2
    double rho;
};

__global__ void k_phantom(int P, int YL, int ZL, double R, double D, double H, double dL,
                          double ctr_minus_beg, double dU, double dV, double hY, double hZ,
                          const EllDev* __restrict__ ell, int n_ell, float* __restrict__ proj,
                          unsigned int* __restrict__ maxbits) {
    extern __shared__ EllDev se[];
    for (int i = threadIdx.x; i < n_ell; i += blockDim.x) se[i] = ell[i];
    __syncthreads();
    const long long n = (long long)P * YL * ZL;
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    float val = 0.f;
    if (idx < n) {
        const int j = (int)(idx % YL);
        const int k = (int)((idx / YL) % ZL);
        const int p = (int)(idx / ((long long)YL * ZL));
        const double PI = kRefPi;
        const double th = (p + ctr_minus_beg) * dL;
        double s, c;
        sincos(th, &s, &c);
        const double S0 = R * c, S1 = R * s, S2 = H * th / (2 * PI);
        const double u = (j - hY) * dU, v = (k - hZ) * dV;
        double d0 = -D * c - u * s, d1 = -D * s + u * c, d2 = v;
        const double nn = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        d0 /= nn; d1 /= nn; d2 /= nn;
        double acc = 0;
        for (int e = 0; e < n_ell; ++e) {
            const EllDev& E = se[e];
            const double w0 = S0 - E.c[0], w1 = S1 - E.c[1], w2 = S2 - E.c[2];
            double q[3], r[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                q[i] = E.m[i] * w0 + E.m[3 + i] * w1 + E.m[6 + i] * w2;
                r[i] = E.m[i] * d0 + E.m[3 + i] * d1 + E.m[6 + i] * d2;
            }
            const double A = r[0] * r[0] * E.ia2[0] + r[1] * r[1] * E.ia2[1] + r[2] * r[2] * E.ia2[2];
            const double B = r[0] * q[0] * E.ia2[0] + r[1] * q[1] * E.ia2[1] + r[2] * q[2] * E.ia2[2];
            const double C = q[0] * q[0] * E.ia2[0] + q[1] * q[1] * E.ia2[1] + q[2] * q[2] * E.ia2[2] - 1;
            const double disc = B * B - A * C;
            if (disc >= 0) acc += 2 * sqrt(disc) * E.rho / A;
        }
        val = (float)acc;
        proj[idx] = val;
    }
    if (maxbits) {
        float m = fmaxf(val, 0.f);
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
        if ((threadIdx.x & 31) == 0) atomicMax(maxbits, __float_as_uint(m));
    }
}

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
__device__ __forceinline__ double u01(unsigned long long x) {
    return ((x >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

__global__ void k_noise(float* __restrict__ proj, long long n, double photons,
                        const unsigned int* __restrict__ maxbits, unsigned long long seed) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= n) return;
    const double pmax = (double)__uint_as_float(*maxbits);
    if (!(pmax > 0)) return;
    const double mu = 8.0 / pmax;
    const double lam = photons * exp(-mu * (double)proj[idx]);
    unsigned long long key = splitmix64(seed ^ splitmix64((unsigned long long)idx));
    double cnt;
    if (lam < 64.0) {
        // inversion of the Poisson CDF
        double uu = u01(key), pk = exp(-lam), cdf = pk;
        int kk = 0;
        while (uu > cdf && kk < 1000) {
            ++kk;
            pk *= lam / kk;
            cdf += pk;
        }
        cnt = kk;
    } else {
        double a = u01(key), b = u01(splitmix64(key));
        double g = sqrt(-2.0 * log(a)) * cos(2.0 * kRefPi * b);
        cnt = floor(lam + sqrt(lam) * g + 0.5);
    }
    if (cnt < 1) cnt = 1;
    proj[idx] = (float)(-log(cnt / photons) / mu);
}

Status launch_phantom(cudaStream_t s, const BPGeom& g, const double* d_ell, int n_ell,
                      double photons, uint64_t seed, float* d_proj, float* d_max) {
    const long long n = (long long)g.ProjNum * g.YL * g.ZL;
    if (n == 0) return Status::Ok();
    const int bs = 128;
    const long long nb = (n + bs - 1) / bs;
    if (nb > 0x7fffffffLL) return make_status(CTRECON_ERR_UNSUPPORTED, "too many rays");
    unsigned int* mb = reinterpret_cast<unsigned int*>(d_max);
    if (mb) CTR_CUDA(cudaMemsetAsync(mb, 0, sizeof(unsigned int), s));
    const size_t smem = sizeof(EllDev) * (size_t)(n_ell > 0 ? n_ell : 1);
    if (smem > 48 * 1024) return make_status(CTRECON_ERR_UNSUPPORTED, "too many ellipsoids");
    k_phantom<<<(unsigned)nb, bs, smem, s>>>(
        g.ProjNum, g.YL, g.ZL, g.ScanR, g.StdDis, g.HelicP, g.DeltaL,
        (double)g.ProjBegin - g.ProjCtr, g.DeltaU, g.DeltaV, (g.YL - 1) * 0.5, (g.ZL - 1) * 0.5,
        reinterpret_cast<const EllDev*>(d_ell), n_ell, d_proj, (photons > 0) ? mb : nullptr);
    CTR_CUDA(cudaGetLastError());
    if (photons > 0 && mb) {
        k_noise<<<(unsigned)nb, bs, 0, s>>>(d_proj, n, photons, mb, (unsigned long long)seed);
        CTR_CUDA(cudaGetLastError());
    }
    return Status::Ok();
}

size_t phantom_ell_bytes(int n_ell) { return sizeof(EllDev) * (size_t)(n_ell > 0 ? n_ell : 1); }

// host: raw rows (cx cy cz a b c phi theta psi rho) -> device layout
void phantom_pack(const double* ell, int n_ell, void* out) {
    EllDev* o = static_cast<EllDev*>(out);
    for (int e = 0; e < n_ell; ++e) {
        const double* E = ell + 10 * e;
        double cf = cos(E[6]), sf = sin(E[6]), ct = cos(E[7]), st = sin(E[7]), cp = cos(E[8]),
               sp = sin(E[8]);
        EllDev d;
        d.c[0] = E[0]; d.c[1] = E[1]; d.c[2] = E[2];
        d.m[0] = cf * cp - sf * ct * sp; d.m[1] = -cf * sp - sf * ct * cp; d.m[2] = sf * st;
        d.m[3] = sf * cp + cf * ct * sp; d.m[4] = -sf * sp + cf * ct * cp; d.m[5] = -cf * st;
        d.m[6] = st * sp;                d.m[7] = st * cp;                 d.m[8] = ct;
        d.ia2[0] = 1.0 / (E[3] * E[3]);
        d.ia2[1] = 1.0 / (E[4] * E[4]);
        d.ia2[2] = 1.0 / (E[5] * E[5]);
        d.rho = E[9];
        o[e] = d;
    }
}

}  // namespace ctr
