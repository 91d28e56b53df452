// geometry.cpp -- FP64 host set-up of the filter tables and the backprojection geometry.
//
// Everything here runs once per parameter set on the host in FP64 (the per-scan geometry
// the design keeps in double precision); the kernels only read the FP32-rounded tables.
// The arithmetic follows the reference line by line so that every discrete decision
// (rebin rows, clamps, crossing fix-ups) is the reference's own.
#include "internal.h"

#include <cmath>
#include <cstdio>

namespace ctr {

Status make_status(ctrecon_status c, const std::string& m) {
    Status s;
    s.code = c;
    s.msg = m;
    return s;
}

Status cuda_status(cudaError_t e, const char* what) {
    ctrecon_status c = (e == cudaErrorMemoryAllocation) ? CTRECON_ERR_OUT_OF_MEMORY
                       : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
                           ? CTRECON_ERR_NO_DEVICE
                           : CTRECON_ERR_CUDA;
    return make_status(c, std::string(what) + ": " + cudaGetErrorString(e));
}

static const double kRebinFactor = 1.3;  // KatsevichFiltering.m:20

Status build_filter_tables(const ctrecon_filter_params& p, FilterTables& t) {
    const double PI = kRefPi;
    t = FilterTables();
    const int YL = p.yl, ZL = p.zl, P = p.proj_number;
    if (YL < 4 || ZL < 4)
        return make_status(CTRECON_ERR_INVALID_ARGUMENT,
                           "detector must have at least 4 columns and 4 rows");
    if (P < 3)
        return make_status(CTRECON_ERR_INVALID_ARGUMENT,
                           "at least 3 views are needed (KatsevichFiltering.m:53-59 takes "
                           "the view derivative from the neighbours of views 2..P-1)");
    if (!(p.proj_scale >= 1) || !(p.dec_width > 0) || !(p.dec_height > 0) || !(p.std_dis > 0) ||
        !(p.scan_r > 0) || !std::isfinite(p.helic_p) || !std::isfinite(p.delta_angle) ||
        !std::isfinite(p.filter_coeff))
        return make_status(CTRECON_ERR_INVALID_ARGUMENT, "non-finite or non-positive geometry");
    const int QQ = (int)std::ceil(ZL * kRebinFactor * 0.5);  // :103
    const int AL = 2 * QQ + 1;                                 // :104
    t.YL = YL; t.ZL = ZL; t.AL = AL; t.QQ = QQ; t.P = P;
    t.DeltaL = 2 * PI / p.proj_scale;   // :40
    t.DeltaU = p.dec_width / YL;        // :41
    t.DeltaV = p.dec_height / ZL;       // :42
    const double HalfZ1 = (ZL + 1) / 2.0, HalfY1 = (YL + 1) / 2.0;  // :43-44 (one-based)
    t.y.resize(YL);
    t.z.resize(ZL);
    for (int j = 0; j < YL; ++j) t.y[j] = ((j + 1) - HalfY1) * t.DeltaU;  // :46
    for (int k = 0; k < ZL; ++k) t.z[k] = ((k + 1) - HalfZ1) * t.DeltaV;  // :47

    // derivative coefficients (:64, :84)
    const double D = p.std_dis;
    t.cu.resize(YL);
    for (int j = 0; j < YL; ++j) t.cu[j] = (D * D + t.y[j] * t.y[j]) / (2 * t.DeltaU * D);
    t.cv = 1.0 / (2 * t.DeltaV * D);

    // kappa lines (:102-126)
    std::vector<double> Nata(AL), FC(AL), InDs(AL);
    t.Rato.assign(AL, 0.0);
    const double AngleRange = 2 * PI - p.delta_angle;
    for (int i = 1; i <= QQ; ++i) {
        double n = (double)i * AngleRange / (QQ - 1);
        Nata[QQ + i] = n;
        Nata[QQ - i] = -n;
    }
    Nata[QQ] = 0;
    for (int a = 0; a < AL; ++a) {
        if (a == QQ) FC[a] = 0;
        else if (p.filtering_mode == 2) FC[a] = p.filter_coeff;
        else FC[a] = (a < QQ) ? 1 - p.filter_coeff : p.filter_coeff;
    }
    for (int a = 0; a < AL; ++a) {
        double f = FC[a], n = Nata[a];
        double AA = std::sin(f * n) - f * std::sin(n);
        double BB = f - 1 + std::cos(f * n) - f * std::cos(n);
        double CC = std::sin((1 - f) * n) - std::sin(n) + std::sin(f * n);
        if (a == QQ) CC = 1;
        InDs[a] = n * p.helic_p * p.std_dis * AA / (2 * PI * p.scan_r * CC);
        t.Rato[a] = n * p.helic_p * BB / (2 * PI * p.scan_r * CC);
    }
    t.Rato[QQ] = p.helic_p / (2 * PI * p.scan_r);

    // forward rebin + pre-weight (:131-153)
    const size_t ay = (size_t)AL * YL;
    t.AZCor.resize(ay); t.coef.resize(ay);
    t.r0.resize(ay); t.r1.resize(ay); t.wa.resize(ay); t.wb.resize(ay);
    for (int a = 0; a < AL; ++a) {
        for (int j = 0; j < YL; ++j) {
            size_t i = (size_t)a * YL + j;
            double az = InDs[a] + t.Rato[a] * t.y[j];
            double c = p.std_dis / std::sqrt(D * D + t.y[j] * t.y[j] + az * az);
            t.AZCor[i] = az;
            t.coef[i] = c;
            double tempV = az / t.DeltaV + HalfZ1;
            if (tempV < 1.01) {
                t.r0[i] = 0; t.r1[i] = 0; t.wa[i] = c; t.wb[i] = 0;
            } else if (tempV > ZL) {
                t.r0[i] = ZL - 1; t.r1[i] = ZL - 1; t.wa[i] = c; t.wb[i] = 0;
            } else {
                double up = std::ceil(tempV), lw = up - 1;
                t.r0[i] = (int)lw - 1;       // zero-based lower row
                t.r1[i] = (int)up - 1;       // zero-based upper row
                t.wa[i] = (up - tempV) * c;  // weight of the lower row
                t.wb[i] = (tempV - lw) * c;  // weight of the upper row
            }
        }
    }

    // backward rebin (:191-287), one-based row numbers as in MATLAB
    const size_t zy = (size_t)ZL * YL;
    t.b.resize(zy); t.e.resize(zy); t.gb.resize(zy); t.ge.resize(zy);
    const double DecHeigh = p.dec_height;
    for (int j = 0; j < YL; ++j) {
        double zmax = -DecHeigh, zmin = DecHeigh;
        int MAXI = 1, MINI = AL;
        for (int tp = 1; tp <= AL; ++tp) {
            double az = t.AZCor[(size_t)(tp - 1) * YL + j];
            if (az > zmax) { zmax = az; MAXI = tp; }
            if (az < zmin) { zmin = az; MINI = tp; }
        }
        int BeginAL = 0, EndAL = 0;  // carried across rows, :211-212
        double BeginCoef = 0, EndCoef = 0;
        for (int k = 1; k <= ZL; ++k) {
            double CurrZ = (k - HalfZ1) * t.DeltaV;
            if (CurrZ < zmin) {
                BeginAL = MINI; EndAL = MINI; BeginCoef = 0.5; EndCoef = 0.5;
            } else if (CurrZ > zmax) {
                BeginAL = MAXI; EndAL = MAXI; BeginCoef = 0.5; EndCoef = 0.5;
            } else {
                double dB = DecHeigh, dE = DecHeigh;
                for (int tp = 1; tp <= AL; ++tp) {
                    double az = t.AZCor[(size_t)(tp - 1) * YL + j];
                    if (az > CurrZ && az - CurrZ < dE) { dE = az - CurrZ; EndAL = tp; }
                    if (az < CurrZ && CurrZ - az < dB) { dB = CurrZ - az; BeginAL = tp; }
                }
                if (!((EndAL == BeginAL + 1) || (EndAL == BeginAL))) {  // :243-276
                    double Sign_Dis = CurrZ - t.Rato[QQ] * t.y[j];      // Rato(QQ+1)
                    bool fixB;
                    if (Sign_Dis > 0) {
                        if (BeginAL < QQ + 1) fixB = true;
                        else if (EndAL < QQ + 1) fixB = false;
                        else if (EndAL < BeginAL) fixB = true;
                        else fixB = false;
                    } else {
                        if (BeginAL > QQ + 1) fixB = true;
                        else if (EndAL > QQ + 1) fixB = false;
                        else if (EndAL > BeginAL) fixB = true;
                        else fixB = false;
                    }
                    if (fixB) {
                        BeginAL = EndAL - 1;
                        if (BeginAL < 1 || BeginAL > AL) goto bad;
                        dB = CurrZ - t.AZCor[(size_t)(BeginAL - 1) * YL + j];
                    } else {
                        EndAL = BeginAL + 1;
                        if (EndAL < 1 || EndAL > AL) goto bad;
                        dE = t.AZCor[(size_t)(EndAL - 1) * YL + j] - CurrZ;
                    }
                }
                BeginCoef = dE / (dE + dB);
                EndCoef = dB / (dE + dB);
            }
            if (BeginAL < 1 || BeginAL > AL || EndAL < 1 || EndAL > AL) goto bad;
            {
                size_t o = (size_t)(k - 1) * YL + j;
                int b0 = BeginAL - 1, e0 = EndAL - 1;
                t.b[o] = b0;
                t.e[o] = e0;
                // ConvRes = -Hilbert/coef (:175, :182), then the two-row blend (:283-284)
                t.gb[o] = -BeginCoef / t.coef[(size_t)b0 * YL + j];
                t.ge[o] = -EndCoef / t.coef[(size_t)e0 * YL + j];
            }
        }
    }

    // DerMode 0 resampling (KatsevichFiltering_T.m:50-94): sample positions in one-based
    // detector coordinates; fractions from the unclamped indices, indices clamped (CheckData.m)
    {
        const double h2 = t.DeltaL / 2, D = p.std_dis;
        auto clampi = [](double v, int hi) { return (int)(v < 1 ? 1 : (v > hi ? hi : v)) - 1; };
        for (int side = 0; side < 2; ++side) {
            t.dres_yd[side].assign(YL, 0);
            t.dres_yu[side].assign(YL, 0);
            t.dres_alfa[side].assign(YL, 0.0);
            t.dres_dzc[side].assign(YL, 0.0);
            for (int j = 0; j < YL; ++j) {
                const double y = t.y[j];
                const double Dzc = side == 0 ? D / (D * std::cos(h2) - y * std::sin(h2))
                                             : D / (D * std::cos(h2) + y * std::sin(h2));
                const double Uy = side == 0 ? (y * std::cos(h2) + D * std::sin(h2)) * Dzc
                                            : (y * std::cos(h2) - D * std::sin(h2)) * Dzc;
                const double ycor = Uy / t.DeltaU + (YL + 1) / 2.0;
                const double fy = std::floor(ycor);
                t.dres_yd[side][j] = clampi(fy, YL);
                t.dres_yu[side][j] = clampi(fy + 1, YL);
                t.dres_alfa[side][j] = ycor - fy;
                t.dres_dzc[side][j] = Dzc;  // (Dzc * z) / DeltaV = Dzc * (k + 1 - HalfZ)
            }
        }
    }

    // Hilbert taps (CreateHSP.m:11-23 laid out as in KatsevichFiltering.m:160-166)
    t.h.assign(2 * (size_t)YL - 1, 0.0);
    for (int m = -(YL - 1); m <= YL - 1; ++m) {
        double v = 0;
        if (m != 0) {
            double s = std::sin(PI * (double)m / 2);
            v = 2 * (s * s) / (PI * (double)m);
        }
        t.h[(size_t)(m + YL - 1)] = v;
    }
    return Status::Ok();
bad:
    return make_status(CTRECON_ERR_GEOMETRY,
                       "backward rebin: the reference would index a kappa row outside 1..AL "
                       "(KatsevichFiltering.m:243-284); check DecHeigh/HelicP/DeltaAngle");
}

Status parse_bp_geom(const ctrecon_bp_geom& in, BPGeom& g) {
    const double PI = kRefPi;
    g.ScanR = in.locus[0];               // KatsevichBkProj.cpp:80-95
    g.StdDis = in.locus[1];
    g.HelicP = in.locus[2];
    g.ProjScale = (int)in.locus[3];
    g.ProjBegin = (int)in.locus[4];
    int ProjEnd = (int)in.locus[5];
    g.ProjCtr = in.locus[6];
    g.ProjNum = ProjEnd - g.ProjBegin + 1;
    g.DecWidth = in.detector[0];
    g.YL = (int)in.detector[1];
    g.DecHeigh = in.detector[2];
    g.ZL = (int)in.detector[3];
    g.ObjR = in.object[0];
    g.NX = (int)in.object[1];
    g.NY = (int)in.object[2];
    g.NZ = (int)in.object[3];
    if (g.ProjNum < 3 || g.YL < 2 || g.ZL < 2 || g.NX < 1 || g.NY < 1 || g.NZ < 1)
        return make_status(CTRECON_ERR_INVALID_ARGUMENT,
                           "geom: need >= 3 views, >= 2x2 detector cells, >= 1 voxel per axis");
    if (g.ProjScale < 1 || !(g.ScanR > 0) || !(g.StdDis > 0) || !(g.ObjR > 0) ||
        !(g.ObjR < g.ScanR) || !(g.DecWidth > 0) || !(g.DecHeigh > 0) ||
        !std::isfinite(g.HelicP) || g.HelicP == 0 || !std::isfinite(g.ProjCtr))
        return make_status(CTRECON_ERR_INVALID_ARGUMENT,
                           "geom: need ProjScale >= 1, 0 < ObjR < ScanR, positive detector "
                           "and a finite non-zero helical pitch");
    if ((long long)g.NX * g.NY * g.NZ > (1LL << 31) - 1 ||
        (long long)g.ProjNum * g.YL * g.ZL > (1LL << 40))
        return make_status(CTRECON_ERR_UNSUPPORTED, "geom: volume above 2^31 voxels");
    g.DeltaL = 2 * PI / g.ProjScale;  // :104-114
    g.DeltaU = g.DecWidth / g.YL;
    g.DeltaV = g.DecHeigh / g.ZL;
    g.HalfY = (g.YL - 1) * 0.5;
    g.HalfZ = (g.ZL - 1) * 0.5;
    g.dx = 2 * g.ObjR / g.NX;
    g.dy = 2 * g.ObjR / g.NY;
    g.dz = 2 * g.ObjR / g.NZ;
    // Detector(5:6) and Object(5:7) when present (KatsevichBkProj_GPU.cu:383-384 reads
    // the detector centres; every reference caller passes exactly the defaults)
    if (in.n_detector >= 6) { g.HalfY = in.detector[4]; g.HalfZ = in.detector[5]; }
    if (in.n_object >= 7) {
        if (!(in.object[4] > 0) || !(in.object[5] > 0) || !(in.object[6] > 0))
            return make_status(CTRECON_ERR_INVALID_ARGUMENT, "geom: voxel sizes must be > 0");
        g.dx = in.object[4]; g.dy = in.object[5]; g.dz = in.object[6];
    }
    g.XC = (g.NX - 1) * 0.5;
    g.YC = (g.NY - 1) * 0.5;
    g.ZC = (g.NZ - 1) * 0.5;
    return Status::Ok();
}

BPParams make_bp_params(const BPGeom& g) {
    BPParams k{};
    k.NX = g.NX; k.NY = g.NY; k.NZ = g.NZ; k.P = g.ProjNum; k.YL = g.YL; k.ZL = g.ZL;
    k.ScanR = g.ScanR; k.HelicP = g.HelicP; k.DeltaL = g.DeltaL;
    k.CtrMinusBeg = g.ProjCtr - g.ProjBegin;
    k.ObjR2 = g.ObjR * g.ObjR;
    k.XC = g.XC; k.YC = g.YC; k.ZC = g.ZC; k.dx = g.dx; k.dy = g.dy; k.dz = g.dz;
    k.Rf = (float)g.ScanR;
    k.DdU = (float)(g.StdDis / g.DeltaU);
    k.DdV = (float)(g.StdDis / g.DeltaV);
    k.HalfY = (float)g.HalfY;
    k.HalfZ = (float)g.HalfZ;
    k.invPs = (float)(1.0 / g.ProjScale);
    k.dzf = (float)g.dz;
    k.win0 = 0;
    k.win1 = g.ProjNum - 1;
    k.accum = 0;
    return k;
}

void build_simt_taps(const FilterTables& t, int YLp, std::vector<float>& hso) {
    const int KOFF = simt_koff(YLp);
    hso.assign(2 * (size_t)KOFF, 0.f);
    for (int K = -KOFF; K < KOFF; ++K) {
        const int L = 2 * K + 1;  // odd lag
        if (L >= -(t.YL - 1) && L <= t.YL - 1) hso[(size_t)(K + KOFF)] = (float)t.h[(size_t)(L + t.YL - 1)];
    }
}

}  // namespace ctr
