/*
 * katsevich_oracle.c -- FP64 CPU oracle of the Katsevich helical cone-beam chain.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker for the CUDA product in
 * ctrecon_b200/: tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg are
 * the only code that may load it, and never as the thing measured or shipped.
 *
 * Each function restates the reference algorithm (CTRecon) in plain C with the same
 * FP64 operation order; the reference file:line each block follows is cited inline.
 * See katsevich_oracle.h for the layouts and for how the oracle is pinned.
 */
#include "katsevich_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define REBIN_FACTOR 1.3 /* KatsevichFiltering.m:20 */

static void set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}

/* ------------------------------------------------------------------------------ */
/* Geometry sizing: FunctionKat_v6.m:49-57                                          */
/* ------------------------------------------------------------------------------ */
void orc_geometry_sizing(double ScanR, double StdDis, double HelicP, double ObjR, int YL,
                         int ZL, double* DecWidth, double* DecHeigh, double* delta) {
    const double PI = 3.1415926; /* FunctionKat_v6.m:49 */
    double U_HelicP = HelicP / ObjR;
    double U_ScanR = ScanR / ObjR;
    double U_DW = 2 * (U_ScanR / pow(U_ScanR * U_ScanR - 1, 0.5)) * YL / (YL - 2);
    double d = 2 * acos(ObjR / ScanR);
    double coef = (2 * PI - d) / (2 * PI * (1 - cos(d)));
    double U_DH = 2 * coef * U_HelicP * ZL / (ZL - 2);
    if (DecWidth) *DecWidth = U_DW * StdDis / U_ScanR;
    if (DecHeigh) *DecHeigh = U_DH * StdDis / U_ScanR;
    if (delta) *delta = d;
}

/* ------------------------------------------------------------------------------ */
/* Filter tables: KatsevichFiltering.m:102-153 and :191-280                          */
/* ------------------------------------------------------------------------------ */
int orc_num_kappa(int ZL, int* QQ) {
    int q = (int)ceil(ZL * REBIN_FACTOR * 0.5); /* :103 */
    if (QQ) *QQ = q;
    return 2 * q + 1; /* :104 */
}

typedef struct {
    int YL, ZL, AL, QQ, P;
    double DeltaL, DeltaU, DeltaV, HalfY1, HalfZ1; /* one-based halves (:43-44) */
    double *y, *z, *AZCor, *coef, *Rato;
    int* fw_mode; /* 0 interpolate, 1 clamp to row 1, 2 clamp to row ZL (:135-145) */
    int* fw_lw;   /* zero-based lower row */
    double *fw_wlw, *fw_wup;
    int *bAL, *eAL; /* zero-based, index z*YL + y */
    double *bC, *eC;
    double* h; /* h[m + YL - 1] */
} orc_tables;

static void free_tables(orc_tables* t) {
    free(t->y); free(t->z); free(t->AZCor); free(t->coef); free(t->Rato);
    free(t->fw_mode); free(t->fw_lw); free(t->fw_wlw); free(t->fw_wup);
    free(t->bAL); free(t->eAL); free(t->bC); free(t->eC); free(t->h);
    memset(t, 0, sizeof *t);
}

/* nextpow2 of MATLAB: smallest e with 2^e >= n */
static int nextpow2_exp(int n) {
    int e = 0;
    while ((1LL << e) < (long long)n) ++e;
    return e;
}

int orc_hilbert_taps(int YL, double* h) {
    /* nn = 2^(nextpow2(YL)+1), nn2 = 2*nn (:160-161); HS = CreateHSP(nn, 1)
     * (CreateHSP.m:11-23), laid circularly into nn2 (:163-166). Because nn/2 >= YL,
     * every lag |i-j| <= YL-1 of the length-nn2 circular convolution (:170-176) reads
     * HS(i - Center) with Center = nn/2 + 1 and i - Center = lag; the wrapped entry
     * HS(1) (lag -nn/2) is never reached. */
    const double PI = ORC_PI; /* CreateHSP.m:15 */
    if (YL < 1 || !h) return -2;
    int nn = 1 << (nextpow2_exp(YL) + 1);
    (void)nn;
    for (int m = -(YL - 1); m <= YL - 1; ++m) {
        double v;
        if (m == 0) {
            v = 0; /* HS(Center) = 0, CreateHSP.m:20 */
        } else {
            double s = sin(PI * (double)m / 2);
            v = 2 * (s * s) / (PI * (double)m); /* CreateHSP.m:18,22 */
        }
        h[m + YL - 1] = v;
    }
    return 0;
}

static int build_tables(const orc_filter_params* fp, orc_tables* t) {
    const double PI = ORC_PI; /* KatsevichFiltering.m:32 */
    memset(t, 0, sizeof *t);
    int YL = fp->YL, ZL = fp->ZL;
    if (YL < 3 || ZL < 3 || fp->ProjNumber < 3) return -2;
    int QQ, AL = orc_num_kappa(ZL, &QQ);
    if (QQ < 2) return -2;
    t->YL = YL; t->ZL = ZL; t->AL = AL; t->QQ = QQ; t->P = fp->ProjNumber;
    t->DeltaL = 2 * PI / fp->ProjScale;      /* :40 */
    t->DeltaU = fp->DecWidth / YL;           /* :41 */
    t->DeltaV = fp->DecHeigh / ZL;           /* :42 */
    t->HalfZ1 = (ZL + 1) / 2.0;              /* :43 */
    t->HalfY1 = (YL + 1) / 2.0;              /* :44 */
    size_t ay = (size_t)AL * YL, zy = (size_t)ZL * YL;
    t->y = malloc(sizeof(double) * YL);
    t->z = malloc(sizeof(double) * ZL);
    t->AZCor = malloc(sizeof(double) * ay);
    t->coef = malloc(sizeof(double) * ay);
    t->Rato = malloc(sizeof(double) * AL);
    t->fw_mode = malloc(sizeof(int) * ay);
    t->fw_lw = malloc(sizeof(int) * ay);
    t->fw_wlw = malloc(sizeof(double) * ay);
    t->fw_wup = malloc(sizeof(double) * ay);
    t->bAL = malloc(sizeof(int) * zy);
    t->eAL = malloc(sizeof(int) * zy);
    t->bC = malloc(sizeof(double) * zy);
    t->eC = malloc(sizeof(double) * zy);
    t->h = malloc(sizeof(double) * (2 * (size_t)YL - 1));
    double* Nata = malloc(sizeof(double) * AL);
    double* FC = malloc(sizeof(double) * AL);
    double* InDs = malloc(sizeof(double) * AL);
    for (int j = 0; j < YL; ++j) t->y[j] = ((j + 1) - t->HalfY1) * t->DeltaU; /* :46 */
    for (int k = 0; k < ZL; ++k) t->z[k] = ((k + 1) - t->HalfZ1) * t->DeltaV; /* :47 */

    double AngleRange = 2 * PI - fp->DeltaAngle; /* :102 */
    for (int i = 1; i <= QQ; ++i) {              /* :107-109 */
        double n = (double)i * AngleRange / (QQ - 1);
        Nata[QQ + i] = n;
        Nata[QQ - i] = -n;
    }
    Nata[QQ] = 0;
    for (int a = 0; a < AL; ++a) { /* :110-115 */
        if (a == QQ) FC[a] = 0;
        else if (fp->FilteringMode == 2) FC[a] = fp->FilterCoeFF;
        else FC[a] = (a < QQ) ? 1 - fp->FilterCoeFF : fp->FilterCoeFF;
    }
    for (int a = 0; a < AL; ++a) { /* :116-124 */
        double f = FC[a], n = Nata[a];
        double AA = sin(f * n) - f * sin(n);
        double BB = f - 1 + cos(f * n) - f * cos(n);
        double CC = sin((1 - f) * n) - sin(n) + sin(f * n);
        if (a == QQ) CC = 1;
        InDs[a] = n * fp->HelicP * fp->StdDis * AA / (2 * PI * fp->ScanR * CC);
        t->Rato[a] = n * fp->HelicP * BB / (2 * PI * fp->ScanR * CC);
    }
    t->Rato[QQ] = fp->HelicP / (2 * PI * fp->ScanR);
    double D2 = fp->StdDis * fp->StdDis;
    for (int a = 0; a < AL; ++a) {
        for (int j = 0; j < YL; ++j) {
            size_t i = (size_t)a * YL + j;
            double az = InDs[a] + t->Rato[a] * t->y[j]; /* :126 */
            t->AZCor[i] = az;
            t->coef[i] = fp->StdDis / sqrt(D2 + t->y[j] * t->y[j] + az * az); /* :150 */
            double tempV = az / t->DeltaV + t->HalfZ1;                        /* :134 */
            if (tempV < 1.01) {                                               /* :135 */
                t->fw_mode[i] = 1; t->fw_lw[i] = 0; t->fw_wlw[i] = 1; t->fw_wup[i] = 0;
            } else if (tempV > ZL) {                                          /* :137 */
                t->fw_mode[i] = 2; t->fw_lw[i] = ZL - 1; t->fw_wlw[i] = 1; t->fw_wup[i] = 0;
            } else {                                                          /* :139-144 */
                double up = ceil(tempV), lw = up - 1;
                t->fw_mode[i] = 0;
                t->fw_lw[i] = (int)lw - 1;
                t->fw_wup[i] = tempV - lw;
                t->fw_wlw[i] = up - tempV;
            }
        }
    }
    free(Nata); free(FC); free(InDs);

    /* backward rebin decisions, :192-286 (one-based indices as in MATLAB) */
    const double DecHeigh = fp->DecHeigh;
    for (int j = 0; j < YL; ++j) {
        double zmax = -DecHeigh, zmin = DecHeigh;
        int MAXI = 1, MINI = AL;
        for (int tp = 1; tp <= AL; ++tp) { /* :199-208 */
            double az = t->AZCor[(size_t)(tp - 1) * YL + j];
            if (az > zmax) { zmax = az; MAXI = tp; }
            if (az < zmin) { zmin = az; MINI = tp; }
        }
        int BeginAL = 0, EndAL = 0; /* :211-214, carried across Zindex */
        double BeginCoef = 0, EndCoef = 0;
        for (int k = 1; k <= ZL; ++k) {
            double CurrZ = (k - t->HalfZ1) * t->DeltaV; /* :216 */
            if (CurrZ < zmin) {
                BeginAL = MINI; EndAL = MINI; BeginCoef = 0.5; EndCoef = 0.5;
            } else if (CurrZ > zmax) {
                BeginAL = MAXI; EndAL = MAXI; BeginCoef = 0.5; EndCoef = 0.5;
            } else {
                double dB = DecHeigh, dE = DecHeigh; /* :228-229 */
                for (int tp = 1; tp <= AL; ++tp) {   /* :230-241 */
                    double az = t->AZCor[(size_t)(tp - 1) * YL + j];
                    if (az > CurrZ && az - CurrZ < dE) { dE = az - CurrZ; EndAL = tp; }
                    if (az < CurrZ && CurrZ - az < dB) { dB = CurrZ - az; BeginAL = tp; }
                }
                if (!((EndAL == BeginAL + 1) || (EndAL == BeginAL))) { /* :243-276 */
                    double Sign_Dis = CurrZ - t->Rato[QQ] * t->y[j];   /* Rato(QQ+1) */
                    int fixB;
                    if (Sign_Dis > 0) {
                        if (BeginAL < QQ + 1) fixB = 1;
                        else if (EndAL < QQ + 1) fixB = 0;
                        else if (EndAL < BeginAL) fixB = 1;
                        else fixB = 0;
                    } else {
                        if (BeginAL > QQ + 1) fixB = 1;
                        else if (EndAL > QQ + 1) fixB = 0;
                        else if (EndAL > BeginAL) fixB = 1;
                        else fixB = 0;
                    }
                    if (fixB) {
                        BeginAL = EndAL - 1;
                        if (BeginAL < 1 || BeginAL > AL) goto bad;
                        dB = CurrZ - t->AZCor[(size_t)(BeginAL - 1) * YL + j];
                    } else {
                        EndAL = BeginAL + 1;
                        if (EndAL < 1 || EndAL > AL) goto bad;
                        dE = t->AZCor[(size_t)(EndAL - 1) * YL + j] - CurrZ;
                    }
                }
                BeginCoef = dE / (dE + dB); /* :278-279 */
                EndCoef = dB / (dE + dB);
            }
            if (BeginAL < 1 || BeginAL > AL || EndAL < 1 || EndAL > AL) goto bad;
            size_t o = (size_t)(k - 1) * YL + j;
            t->bAL[o] = BeginAL - 1;
            t->eAL[o] = EndAL - 1;
            t->bC[o] = BeginCoef;
            t->eC[o] = EndCoef;
        }
    }
    orc_hilbert_taps(YL, t->h);
    return 0;
bad:
    free_tables(t);
    return -1;
}

int orc_filter_tables(const orc_filter_params* fp, double* AZCor, double* coef,
                      double* Rato, int* lw, double* w_lw, double* w_up, int* bAL,
                      int* eAL, double* bC, double* eC) {
    orc_tables t;
    int rc = build_tables(fp, &t);
    if (rc) return rc;
    size_t ay = (size_t)t.AL * t.YL, zy = (size_t)t.ZL * t.YL;
    if (AZCor) memcpy(AZCor, t.AZCor, sizeof(double) * ay);
    if (coef) memcpy(coef, t.coef, sizeof(double) * ay);
    if (Rato) memcpy(Rato, t.Rato, sizeof(double) * t.AL);
    if (lw) memcpy(lw, t.fw_lw, sizeof(int) * ay);
    if (w_lw) memcpy(w_lw, t.fw_wlw, sizeof(double) * ay);
    if (w_up) memcpy(w_up, t.fw_wup, sizeof(double) * ay);
    if (bAL) memcpy(bAL, t.bAL, sizeof(int) * zy);
    if (eAL) memcpy(eAL, t.eAL, sizeof(int) * zy);
    if (bC) memcpy(bC, t.bC, sizeof(double) * zy);
    if (eC) memcpy(eC, t.eC, sizeof(double) * zy);
    free_tables(&t);
    return 0;
}

/* ------------------------------------------------------------------------------ */
/* Filter, one view at a time (the MATLAB code vectorises over views; every element */
/* sees the same FP64 operations in the same order).                                */
/* ------------------------------------------------------------------------------ */

/* Step 1, derivative (:52-95), for view p into GF[ZL*YL] (index z*YL + y). */
static void view_derivative(const orc_filter_params* fp, const orc_tables* t,
                            const double* Proj, int p, double* GF) {
    const int YL = t->YL, ZL = t->ZL, P = t->P;
    const size_t S = (size_t)YL * ZL;
    /* view derivative (:53-59): views 1 and P copy views 2 and P-1 */
    int pc = p;
    if (pc == 0) pc = 1;
    if (pc == P - 1) pc = P - 2;
    const double* Pl = Proj + (size_t)(pc - 1) * S;
    const double* Pr = Proj + (size_t)(pc + 1) * S;
    for (size_t i = 0; i < S; ++i) GF[i] = (Pr[i] - Pl[i]) / (2 * t->DeltaL);

    const double* Pv = Proj + (size_t)p * S;
    const double D = fp->StdDis;
    /* u derivative (:63-78) */
    for (int k = 0; k < ZL; ++k) {
        const double* row = Pv + (size_t)k * YL;
        double* g = GF + (size_t)k * YL;
        for (int j = 2; j <= YL - 3; ++j) {
            double c = (D * D + t->y[j] * t->y[j]) / (2 * t->DeltaU * D);
            g[j] = g[j] + (row[j + 1] - row[j - 1]) * c;
        }
        double temp = row[2] - row[0];
        for (int j = 0; j <= 1; ++j) {
            double c = (D * D + t->y[j] * t->y[j]) / (2 * t->DeltaU * D);
            g[j] = g[j] + temp * c;
        }
        temp = row[YL - 1] - row[YL - 3];
        for (int j = YL - 2; j <= YL - 1; ++j) {
            double c = (D * D + t->y[j] * t->y[j]) / (2 * t->DeltaU * D);
            g[j] = g[j] + temp * c;
        }
    }
    /* v derivative (:82-95) */
    const double cv = 1.0 / (2 * t->DeltaV * D);
    for (int k = 2; k <= ZL - 3; ++k) {
        for (int j = 0; j < YL; ++j) {
            double temp = t->y[j] * (Pv[(size_t)(k + 1) * YL + j] - Pv[(size_t)(k - 1) * YL + j]);
            GF[(size_t)k * YL + j] = GF[(size_t)k * YL + j] + t->z[k] * temp * cv;
        }
    }
    for (int j = 0; j < YL; ++j) {
        double temp = t->y[j] * (Pv[(size_t)2 * YL + j] - Pv[j]);
        GF[j] = GF[j] + t->z[0] * cv * temp;
        GF[(size_t)YL + j] = GF[(size_t)YL + j] + t->z[1] * cv * temp;
    }
    for (int j = 0; j < YL; ++j) {
        double temp =
            t->y[j] * (Pv[(size_t)(ZL - 1) * YL + j] - Pv[(size_t)(ZL - 3) * YL + j]);
        GF[(size_t)(ZL - 2) * YL + j] = GF[(size_t)(ZL - 2) * YL + j] + t->z[ZL - 2] * cv * temp;
        GF[(size_t)(ZL - 1) * YL + j] = GF[(size_t)(ZL - 1) * YL + j] + t->z[ZL - 1] * cv * temp;
    }
}

/* The direct derivative of KatsevichFiltering_T.m:50-94 (DerMode 0 of FunctionKat_v6.m:95-102):
 * the projections bilinearly resampled onto the detector coordinates of the source rotated by
 * -dL/2 (GF1, :51-71) and +dL/2 (GF2, :73-93), then GF(p) = (GF1(p+1) - GF2(p)) / dL (:95-99),
 * the last view repeating its neighbour (:101). Sample positions use one-based coordinates; the
 * fractions come from the unclamped indices, the indices are clamped to the detector
 * (CheckData.m). */
static double resample_half(const orc_filter_params* fp, const orc_tables* t, const double* Pv,
                            int j, int k, int sign) {
    const int YL = t->YL, ZL = t->ZL;
    const double D = fp->StdDis, h = t->DeltaL / 2;
    const double Dzc = sign < 0 ? D / (D * cos(h) - t->y[j] * sin(h))
                                : D / (D * cos(h) + t->y[j] * sin(h));
    const double Uy = sign < 0 ? (t->y[j] * cos(h) + D * sin(h)) * Dzc
                               : (t->y[j] * cos(h) - D * sin(h)) * Dzc;
    const double ycor = Uy / t->DeltaU + t->HalfY1;
    const double zcor = (Dzc * t->z[k]) / t->DeltaV + t->HalfZ1;
    int YD = (int)floor(ycor), ZD = (int)floor(zcor);
    int YU = YD + 1, ZU = ZD + 1;
    const double alfa = ycor - YD, beta = zcor - ZD;
    YD = YD < 1 ? 1 : (YD > YL ? YL : YD);
    YU = YU < 1 ? 1 : (YU > YL ? YL : YU);
    ZD = ZD < 1 ? 1 : (ZD > ZL ? ZL : ZD);
    ZU = ZU < 1 ? 1 : (ZU > ZL ? ZL : ZU);
#define P1(yy, zz) Pv[(size_t)((zz) - 1) * YL + ((yy) - 1)]
    return P1(YD, ZD) * (1 - alfa) * (1 - beta) + P1(YD, ZU) * (1 - alfa) * beta +
           P1(YU, ZD) * alfa * (1 - beta) + P1(YU, ZU) * alfa * beta;
#undef P1
}

static void view_derivative_direct(const orc_filter_params* fp, const orc_tables* t,
                                   const double* Proj, int p, double* GF) {
    const int YL = t->YL, ZL = t->ZL, P = t->P;
    const size_t S = (size_t)YL * ZL;
    const int pc = p == P - 1 ? P - 2 : p;
    const double* Pn = Proj + (size_t)(pc + 1) * S;
    const double* Pc = Proj + (size_t)pc * S;
    for (int k = 0; k < ZL; ++k)
        for (int j = 0; j < YL; ++j)
            GF[(size_t)k * YL + j] = (resample_half(fp, t, Pn, j, k, -1) -
                                      resample_half(fp, t, Pc, j, k, +1)) / t->DeltaL;
}

/* Step 2, forward height rebin + pre-weight (:131-153) into X[AL*YL]. */
static void view_rebin(const orc_tables* t, const double* GF, double* X) {
    const int YL = t->YL;
    for (int a = 0; a < t->AL; ++a) {
        for (int j = 0; j < YL; ++j) {
            size_t i = (size_t)a * YL + j;
            double v;
            int lw = t->fw_lw[i];
            if (t->fw_mode[i] != 0) v = GF[(size_t)lw * YL + j];
            else v = GF[(size_t)(lw + 1) * YL + j] * t->fw_wup[i] + GF[(size_t)lw * YL + j] * t->fw_wlw[i];
            X[i] = v * t->coef[i];
        }
    }
}

/* Step 3, Hilbert filter + post-weight (:160-183): the circular FFT convolution of
 * :170-176 equals the direct Toeplitz sum over lags |i-j| <= YL-1 (see
 * orc_hilbert_taps); its result is negated and divided by coef. */
static void view_hilbert(const orc_tables* t, const double* X, double* C) {
    const int YL = t->YL;
    const double* h = t->h + (YL - 1);
    for (int a = 0; a < t->AL; ++a) {
        const double* x = X + (size_t)a * YL;
        double* c = C + (size_t)a * YL;
        for (int i = 0; i < YL; ++i) {
            double s = 0;
            for (int j = 0; j < YL; ++j) s += h[i - j] * x[j];
            c[i] = -s / t->coef[(size_t)a * YL + i];
        }
    }
}

/* Step 4, backward rebin (:283-284) of one view into FProj view p. */
static void view_backrebin(const orc_tables* t, const double* C, double* Fv) {
    const int YL = t->YL;
    for (int k = 0; k < t->ZL; ++k) {
        for (int j = 0; j < YL; ++j) {
            size_t o = (size_t)k * YL + j;
            Fv[o] = C[(size_t)t->bAL[o] * YL + j] * t->bC[o] +
                    C[(size_t)t->eAL[o] * YL + j] * t->eC[o];
        }
    }
}

int orc_filter(const orc_filter_params* fp, const double* Proj, double* FProj, int p_begin,
               int p_end, int nthreads) {
    orc_tables t;
    int rc = build_tables(fp, &t);
    if (rc) return rc;
    if (p_begin < 0) p_begin = 0;
    if (p_end <= 0 || p_end > t.P) p_end = t.P;
    set_threads(nthreads);
    const size_t S = (size_t)t.YL * t.ZL, A = (size_t)t.AL * t.YL;
#pragma omp parallel
    {
        double* GF = malloc(sizeof(double) * S);
        double* X = malloc(sizeof(double) * A);
        double* C = malloc(sizeof(double) * A);
#pragma omp for schedule(dynamic, 1)
        for (int p = p_begin; p < p_end; ++p) {
            view_derivative(fp, &t, Proj, p, GF);
            view_rebin(&t, GF, X);
            view_hilbert(&t, X, C);
            view_backrebin(&t, C, FProj + (size_t)p * S);
        }
        free(GF); free(X); free(C);
    }
    free_tables(&t);
    return 0;
}

int orc_filter_direct(const orc_filter_params* fp, const double* Proj, double* FProj,
                      int p_begin, int p_end, int nthreads) {
    orc_tables t;
    int rc = build_tables(fp, &t);
    if (rc) return rc;
    if (p_begin < 0) p_begin = 0;
    if (p_end <= 0 || p_end > t.P) p_end = t.P;
    set_threads(nthreads);
    const size_t S = (size_t)t.YL * t.ZL, A = (size_t)t.AL * t.YL;
#pragma omp parallel
    {
        double* GF = malloc(sizeof(double) * S);
        double* X = malloc(sizeof(double) * A);
        double* C = malloc(sizeof(double) * A);
#pragma omp for schedule(dynamic, 1)
        for (int p = p_begin; p < p_end; ++p) {
            view_derivative_direct(fp, &t, Proj, p, GF);
            view_rebin(&t, GF, X);
            view_hilbert(&t, X, C);
            view_backrebin(&t, C, FProj + (size_t)p * S);
        }
        free(GF); free(X); free(C);
    }
    free_tables(&t);
    return 0;
}

int orc_derivative_direct(const orc_filter_params* fp, const double* Proj, int p, double* GF) {
    orc_tables t;
    int rc = build_tables(fp, &t);
    if (rc) return rc;
    if (p < 0 || p >= t.P || t.P < 2) { free_tables(&t); return -2; }
    view_derivative_direct(fp, &t, Proj, p, GF);
    free_tables(&t);
    return 0;
}

int orc_filter_view_stages(const orc_filter_params* fp, const double* Proj, int p,
                           double* GF, double* conv_in, double* conv_out) {
    orc_tables t;
    int rc = build_tables(fp, &t);
    if (rc) return rc;
    if (p < 0 || p >= t.P) { free_tables(&t); return -2; }
    const size_t S = (size_t)t.YL * t.ZL, A = (size_t)t.AL * t.YL;
    double* g = malloc(sizeof(double) * S);
    double* x = malloc(sizeof(double) * A);
    double* c = malloc(sizeof(double) * A);
    view_derivative(fp, &t, Proj, p, g);
    view_rebin(&t, g, x);
    view_hilbert(&t, x, c);
    if (GF) memcpy(GF, g, sizeof(double) * S);
    if (conv_in) memcpy(conv_in, x, sizeof(double) * A);
    if (conv_out) memcpy(conv_out, c, sizeof(double) * A);
    free(g); free(x); free(c);
    free_tables(&t);
    return 0;
}

/* ------------------------------------------------------------------------------ */
/* Filtering coefficient: FindTau.m:6-22 (MATLAB's built-in pi)                       */
/* ------------------------------------------------------------------------------ */
double orc_find_tau(double ratio, double tol) {
    const double pi = 3.141592653589793;
    double am = 2 * pi - 2 * acos(ratio); /* :7 */
    double tu = 0.5, td = 0, delta = 1, t = 0;
    while (delta > tol) { /* :13-22 */
        t = (td + tu) / 2;
        double f = t * cos(am) - cos(t * am) + 1 - t;
        delta = fabs(f);
        if (f > 0) tu = t;
        else td = t;
    }
    return t;
}

/* ------------------------------------------------------------------------------ */
/* PI segment: KatsevichBkProj.cpp:283-312                                           */
/* ------------------------------------------------------------------------------ */
void orc_pisegment(double x, double y, double z, double* BAngle, double* TAngle) {
    const double PI = ORC_PI;
    const double dm = 0.0000001; /* DeltaMax, :26 */
    double delta = 1, bmin, bmax, r2, LanbudaInital;
    double sb = 0, st = 0, t, tempcos, templan, zz;
    LanbudaInital = z * 2 * PI;
    bmin = LanbudaInital - 2 * PI;
    bmax = LanbudaInital;
    r2 = x * x + y * y;
    while (((bmax - bmin) > dm) && (delta > dm)) {
        sb = (bmax + bmin) * 0.5;
        tempcos = 2 * (1 - y * sin(sb) - x * cos(sb));
        t = (1 - r2) / tempcos;
        templan = acos((y * cos(sb) - x * sin(sb)) / sqrt(tempcos + r2 - 1));
        st = 2 * templan + sb;
        zz = (sb * t + (1 - t) * st) / (2 * PI);
        if (zz < z) bmin = sb;
        else bmax = sb;
        delta = fabs(zz - z);
    }
    *BAngle = sb;
    *TAngle = st;
}

/* ------------------------------------------------------------------------------ */
/* Backprojection: KatsevichBkProj.cpp:71-281                                        */
/* ------------------------------------------------------------------------------ */
typedef struct {
    double ScanR, ObjR, StdDis, HelicP, ProjCtr;
    int ProjScale, ProjBeginIndex, ProjNum, YL, ZL, RecMX, RecMY, RecMZ;
    double DeltaL, DeltaU, DeltaV, HalfY, HalfZ;
    double *VectorS, *VectorE1, *VectorE2, *xCor, *yCor, *zCor;
} bp_setup;

static int bp_prepare(const orc_bp_geom* g, bp_setup* s) {
    const double PI = ORC_PI;
    memset(s, 0, sizeof *s);
    s->ScanR = g->locus[0];     /* :80-95 */
    s->ObjR = g->object[0];
    s->StdDis = g->locus[1];
    s->HelicP = g->locus[2];
    double DecWidth = g->detector[0], DecHeigh = g->detector[2];
    s->ProjCtr = g->locus[6];
    s->ProjScale = (int)g->locus[3];
    s->ProjBeginIndex = (int)g->locus[4];
    int ProjEndIndex = (int)g->locus[5];
    s->ProjNum = ProjEndIndex - s->ProjBeginIndex + 1;
    s->YL = (int)g->detector[1];
    s->ZL = (int)g->detector[3];
    s->RecMX = (int)g->object[1];
    s->RecMY = (int)g->object[2];
    s->RecMZ = (int)g->object[3];
    if (s->ProjNum < 1 || s->YL < 2 || s->ZL < 2 || s->RecMX < 1 || s->RecMY < 1 ||
        s->RecMZ < 1 || s->ProjScale == 0)
        return -2;
    s->DeltaL = 2 * PI / s->ProjScale; /* :104-114 */
    s->DeltaU = DecWidth / s->YL;
    s->DeltaV = DecHeigh / s->ZL;
    s->HalfY = (s->YL - 1) * 0.5;
    s->HalfZ = (s->ZL - 1) * 0.5;
    double DeltaX = 2 * s->ObjR / s->RecMX;
    double DeltaY = 2 * s->ObjR / s->RecMY;
    double DeltaZ = 2 * s->ObjR / s->RecMZ;
    if (g->honour_extras) {
        if (g->n_object >= 7) { DeltaX = g->object[4]; DeltaY = g->object[5]; DeltaZ = g->object[6]; }
        if (g->n_detector >= 6) { s->HalfY = g->detector[4]; s->HalfZ = g->detector[5]; }
    }
    double XCenter = (s->RecMX - 1) * 0.5, YCenter = (s->RecMY - 1) * 0.5,
           ZCenter = (s->RecMZ - 1) * 0.5;
    s->VectorS = malloc(sizeof(double) * 3 * s->ProjNum);
    s->VectorE1 = malloc(sizeof(double) * 2 * s->ProjNum);
    s->VectorE2 = malloc(sizeof(double) * 2 * s->ProjNum);
    s->xCor = malloc(sizeof(double) * s->RecMX);
    s->yCor = malloc(sizeof(double) * s->RecMY);
    s->zCor = malloc(sizeof(double) * s->RecMZ);
    for (int loop = 0; loop < s->ProjNum; loop++) { /* :130-140 */
        double temp = (loop + s->ProjBeginIndex - s->ProjCtr) * s->DeltaL;
        s->VectorS[loop * 3] = s->ScanR * cos(temp);
        s->VectorS[loop * 3 + 1] = s->ScanR * sin(temp);
        s->VectorS[loop * 3 + 2] = s->HelicP * temp / (2 * PI);
        s->VectorE1[loop * 2] = -cos(temp);
        s->VectorE1[loop * 2 + 1] = -sin(temp);
        s->VectorE2[loop * 2] = -sin(temp);
        s->VectorE2[loop * 2 + 1] = cos(temp);
    }
    for (int loop = 0; loop < s->RecMX; loop++) s->xCor[loop] = (loop - XCenter) * DeltaX;
    for (int loop = 0; loop < s->RecMY; loop++) s->yCor[loop] = (loop - YCenter) * DeltaY;
    for (int loop = 0; loop < s->RecMZ; loop++) s->zCor[loop] = (loop - ZCenter) * DeltaZ;
    return 0;
}

static void bp_release(bp_setup* s) {
    free(s->VectorS); free(s->VectorE1); free(s->VectorE2);
    free(s->xCor); free(s->yCor); free(s->zCor);
}

/* PI interval of one voxel (:173-234). Returns 1 if the voxel is written, with the
 * loop bounds and the endpoint weights written into Coef (length ProjNum, reset to 1
 * at the entries this voxel touches and restored by the caller's reset loop). */
static int voxel_interval(const bp_setup* s, int X, int Y, int Z, double* Bout,
                          double* Tout, int* LoopBegin, int* LoopEnd, double* Coef) {
    double BAngle, TAngle, temp;
    double x = s->xCor[X] / s->ScanR, y = s->yCor[Y] / s->ScanR, z = s->zCor[Z] / s->HelicP;
    orc_pisegment(x, y, z, &BAngle, &TAngle);
    BAngle = BAngle / s->DeltaL + s->ProjCtr - s->ProjBeginIndex;
    TAngle = TAngle / s->DeltaL + s->ProjCtr - s->ProjBeginIndex;
    if (Bout) *Bout = BAngle;
    if (Tout) *Tout = TAngle;
    const int ProjNum = s->ProjNum;
    if ((BAngle >= ProjNum - 1) || (TAngle <= 0)) return 0;
    int Bindex = (int)(BAngle + 10) - 10;
    int Tindex = (int)(TAngle + 10) - 9;
    if (Coef)
        for (int loop = 0; loop < ProjNum; loop++) Coef[loop] = 1; /* :184-185 */
    if (Bindex < 0) {
        *LoopBegin = 1;
    } else if (Bindex == 0) {
        temp = 1 - BAngle + Bindex;
        if (Coef) Coef[1] = 0.5 + (1 - temp * 0.5) * temp;
        *LoopBegin = 1;
    } else if (Bindex == ProjNum - 2) {
        temp = 1 - BAngle + Bindex;
        if (Coef) Coef[ProjNum - 2] = pow(temp, 2) * 0.5;
        *LoopBegin = ProjNum - 2;
    } else {
        temp = 1 - BAngle + Bindex;
        if (Coef) {
            Coef[Bindex] = pow(temp, 2) * 0.5;
            Coef[Bindex + 1] = 0.5 + (1 - temp * 0.5) * temp;
        }
        *LoopBegin = Bindex;
    }
    if (Tindex > ProjNum - 1) {
        *LoopEnd = ProjNum - 2;
    } else if (Tindex == ProjNum - 1) {
        temp = 1 + TAngle - Tindex;
        if (Coef) Coef[ProjNum - 2] = 0.5 + (1 - temp * 0.5) * temp;
        *LoopEnd = ProjNum - 2;
    } else if (Tindex == 1) {
        *LoopEnd = 1;
        temp = 1 + TAngle - Tindex;
        if (Coef) Coef[1] = pow(temp, 2) * 0.5;
    } else {
        *LoopEnd = Tindex;
        temp = 1 + TAngle - Tindex;
        if (Coef) {
            Coef[Tindex - 1] = 0.5 + (1 - temp * 0.5) * temp;
            Coef[Tindex] = pow(temp, 2) * 0.5;
        }
    }
    return 1;
}

int orc_bkproj(const orc_bp_geom* g, const double* proj, double* image, int x_begin,
               int x_end, int z_begin, int z_end, int nthreads, long long* n_updates,
               unsigned char* touched) {
    bp_setup s;
    int rc = bp_prepare(g, &s);
    if (rc) return rc;
    if (x_end <= 0 || x_end > s.RecMX) x_end = s.RecMX;
    if (x_begin < 0) x_begin = 0;
    if (z_end <= 0 || z_end > s.RecMZ) z_end = s.RecMZ;
    if (z_begin < 0) z_begin = 0;
    set_threads(nthreads);
    const int YL = s.YL, YLZL = s.YL * s.ZL, RecMY = s.RecMY, RecMZ = s.RecMZ;
    const long long proj_len = (long long)s.ProjNum * YLZL;
    const double ObjRSquare = pow(s.ObjR, 2);
    long long total = 0;
#pragma omp parallel reduction(+ : total)
    {
        double* Coef = malloc(sizeof(double) * s.ProjNum);
#pragma omp for schedule(dynamic, 1)
        for (int Xindex = x_begin; Xindex < x_end; Xindex++) {
            for (int Yindex = 0; Yindex < RecMY; Yindex++) {
                if (!(pow(s.xCor[Xindex], 2) + pow(s.yCor[Yindex], 2) < ObjRSquare)) continue;
                for (int Zindex = z_begin; Zindex < z_end; Zindex++) {
                    int LoopBegin, LoopEnd;
                    if (!voxel_interval(&s, Xindex, Yindex, Zindex, NULL, NULL, &LoopBegin,
                                        &LoopEnd, Coef))
                        continue;
                    double tpdata = 0; /* :236-262 */
                    for (int ProjIndex = LoopBegin; ProjIndex <= LoopEnd; ProjIndex++) {
                        double DPSx = s.xCor[Xindex] - s.VectorS[ProjIndex * 3];
                        double DPSy = s.yCor[Yindex] - s.VectorS[ProjIndex * 3 + 1];
                        double DPSz = s.zCor[Zindex] - s.VectorS[ProjIndex * 3 + 2];
                        double factor = sqrt(DPSx * DPSx + DPSy * DPSy + DPSz * DPSz);
                        double fenmu = DPSx * s.VectorE1[ProjIndex * 2] +
                                       DPSy * s.VectorE1[ProjIndex * 2 + 1];
                        double YY = DPSx * s.VectorE2[ProjIndex * 2] +
                                    DPSy * s.VectorE2[ProjIndex * 2 + 1];
                        YY = YY * s.StdDis / (fenmu * s.DeltaU) + s.HalfY;
                        double ZZ = DPSz * s.StdDis / (fenmu * s.DeltaV) + s.HalfZ;
                        int YYD = (int)YY, YYU = YYD + 1, ZZD = (int)ZZ, ZZU = ZZD + 1;
                        double alfa = YY - YYD, beta = ZZ - ZZD;
                        long long base = (long long)ProjIndex * YLZL;
                        long long i00 = base + (long long)ZZD * YL + YYD;
                        long long i01 = base + (long long)ZZD * YL + YYU;
                        long long i10 = base + (long long)ZZU * YL + YYD;
                        long long i11 = base + (long long)ZZU * YL + YYU;
                        /* the reference reads without bounds checks; the oracle reads the
                         * same element whenever it lies inside the array, else 0 */
                        double p00 = (i00 >= 0 && i00 < proj_len) ? proj[i00] : 0;
                        double p01 = (i01 >= 0 && i01 < proj_len) ? proj[i01] : 0;
                        double p10 = (i10 >= 0 && i10 < proj_len) ? proj[i10] : 0;
                        double p11 = (i11 >= 0 && i11 < proj_len) ? proj[i11] : 0;
                        double temp = p00 * (1 - alfa) * (1 - beta) + p01 * alfa * (1 - beta) +
                                      p10 * (1 - alfa) * beta + p11 * alfa * beta;
                        temp = temp * Coef[ProjIndex];
                        tpdata = tpdata + temp / factor;
                    }
                    tpdata = -tpdata / s.ProjScale;
                    long long idx = ((long long)Xindex * RecMY + Yindex) * RecMZ + Zindex;
                    image[idx] = tpdata;
                    if (touched) touched[idx] = 1;
                    total += (long long)(LoopEnd - LoopBegin + 1);
                }
            }
        }
        free(Coef);
    }
    if (n_updates) *n_updates = total;
    bp_release(&s);
    return 0;
}

int orc_pi_table(const orc_bp_geom* g, double* B, double* T, int* loop_begin,
                 int* loop_end, unsigned char* valid, int nthreads) {
    bp_setup s;
    int rc = bp_prepare(g, &s);
    if (rc) return rc;
    set_threads(nthreads);
    const double ObjRSquare = pow(s.ObjR, 2);
#pragma omp parallel for schedule(dynamic, 1)
    for (int X = 0; X < s.RecMX; X++) {
        for (int Y = 0; Y < s.RecMY; Y++) {
            int inside = pow(s.xCor[X], 2) + pow(s.yCor[Y], 2) < ObjRSquare;
            for (int Z = 0; Z < s.RecMZ; Z++) {
                long long idx = ((long long)X * s.RecMY + Y) * s.RecMZ + Z;
                double b = 0, t = 0;
                int lb = 0, le = -1, ok = 0;
                if (inside) ok = voxel_interval(&s, X, Y, Z, &b, &t, &lb, &le, NULL);
                if (B) B[idx] = b;
                if (T) T[idx] = t;
                if (loop_begin) loop_begin[idx] = ok ? lb : 0;
                if (loop_end) loop_end[idx] = ok ? le : -1;
                if (valid) valid[idx] = (unsigned char)ok;
            }
        }
    }
    bp_release(&s);
    return 0;
}

/* ------------------------------------------------------------------------------ */
/* Analytic ellipsoid projections: chord formula of CreateProjSlice.cpp:98-134,      */
/* with a general ZXZ rotation and a flat detector in mm (the reference uses one     */
/* z-axis rotation and a virtual detector through the isocentre in ObjR units).      */
/* ------------------------------------------------------------------------------ */
int orc_project_ellipsoids(const orc_bp_geom* g, const double* ell, int n_ell,
                           double* proj, int p_begin, int p_end, int nthreads) {
    const double PI = ORC_PI;
    const double R = g->locus[0], D = g->locus[1], H = g->locus[2];
    const int Ps = (int)g->locus[3];
    const int Beg = (int)g->locus[4], End = (int)g->locus[5];
    const double Ctr = g->locus[6];
    const int YL = (int)g->detector[1], ZL = (int)g->detector[3];
    const int P = End - Beg + 1;
    if (P < 1 || YL < 1 || ZL < 1 || Ps == 0) return -2;
    if (p_begin < 0) p_begin = 0;
    if (p_end <= 0 || p_end > P) p_end = P;
    const double dU = g->detector[0] / YL, dV = g->detector[2] / ZL;
    const double hY = (YL - 1) * 0.5, hZ = (ZL - 1) * 0.5;
    const double dL = 2 * PI / Ps;
    /* rotation matrices, R = Rz(phi) Rx(theta) Rz(psi), row-major */
    double* rot = malloc(sizeof(double) * 9 * (n_ell > 0 ? n_ell : 1));
    for (int e = 0; e < n_ell; ++e) {
        double cf = cos(ell[e * 10 + 6]), sf = sin(ell[e * 10 + 6]);
        double ct = cos(ell[e * 10 + 7]), st = sin(ell[e * 10 + 7]);
        double cp = cos(ell[e * 10 + 8]), sp = sin(ell[e * 10 + 8]);
        double* m = rot + 9 * e;
        m[0] = cf * cp - sf * ct * sp; m[1] = -cf * sp - sf * ct * cp; m[2] = sf * st;
        m[3] = sf * cp + cf * ct * sp; m[4] = -sf * sp + cf * ct * cp; m[5] = -cf * st;
        m[6] = st * sp;                m[7] = st * cp;                 m[8] = ct;
    }
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
    for (int p = p_begin; p < p_end; ++p) {
        double th = (p + Beg - Ctr) * dL;
        double c = cos(th), s = sin(th);
        double S[3] = {R * c, R * s, H * th / (2 * PI)};
        for (int k = 0; k < ZL; ++k) {
            double v = (k - hZ) * dV;
            for (int j = 0; j < YL; ++j) {
                double u = (j - hY) * dU;
                double d[3] = {-D * c - u * s, -D * s + u * c, v};
                double n = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                d[0] /= n; d[1] /= n; d[2] /= n;
                double acc = 0;
                for (int e = 0; e < n_ell; ++e) {
                    const double* E = ell + e * 10;
                    const double* m = rot + 9 * e;
                    double w[3] = {S[0] - E[0], S[1] - E[1], S[2] - E[2]};
                    double q[3], r[3];
                    for (int i = 0; i < 3; ++i) {
                        q[i] = m[i] * w[0] + m[3 + i] * w[1] + m[6 + i] * w[2];
                        r[i] = m[i] * d[0] + m[3 + i] * d[1] + m[6 + i] * d[2];
                    }
                    double a2[3] = {E[3] * E[3], E[4] * E[4], E[5] * E[5]};
                    double AA = r[0] * r[0] / a2[0] + r[1] * r[1] / a2[1] + r[2] * r[2] / a2[2];
                    double BB = r[0] * q[0] / a2[0] + r[1] * q[1] / a2[1] + r[2] * q[2] / a2[2];
                    double CC = q[0] * q[0] / a2[0] + q[1] * q[1] / a2[1] + q[2] * q[2] / a2[2] - 1;
                    double disc = BB * BB - AA * CC;
                    if (disc >= 0) acc += 2 * sqrt(disc) * E[9] / AA;
                }
                proj[((size_t)p * ZL + k) * YL + j] = acc;
            }
        }
    }
    free(rot);
    return 0;
}

/* rebinToPanel.m:1-36, line for line: the panel column ii (1-based) sits at fan angle
 * atan((ii - (N+1)/2) * newW / D) (:14), i.e. at fractional arc index idx (:15); the two arc
 * cells floor/ceil(idx) (:16-17) are clamped as at :18-29 (a column whose ceil is below 1 or
 * whose floor is beyond N stays zero) and blended with the weights of :33, which use the
 * clamped indices -- so an idx that is exactly a cell centre gives weight 0 to both cells. */
double orc_rebin_to_panel(const double* proj, int det_num, int det_hei, int prj_num,
                          double c, double w, double D, double* out) {
    const double oneFanAngle = atan(w / 2 / D) * 2.0;                                /* :6 */
    const double a1 = (c + 0.5) * oneFanAngle, a2 = (det_num - 1 - c + 0.5) * oneFanAngle;
    const double largerAngle = a1 > a2 ? a1 : a2;                                   /* :7 */
    const double detWidth = tan(largerAngle) * D * 2;                               /* :9 */
    const double newW = detWidth / det_num;                                         /* :10 */
    const size_t rows = (size_t)det_hei * prj_num;
    for (size_t r = 0; r < rows; ++r)
        for (int i = 0; i < det_num; ++i) out[r * det_num + i] = 0.0;               /* :11 */
    for (int ii = 1; ii <= det_num; ++ii) {
        const double fanAngle = atan((ii - (det_num + 1) / 2.0) * newW / D);         /* :15 */
        const double idx = fanAngle / oneFanAngle + c + 1;                          /* :16 */
        double lowIdx = floor(idx), higIdx = ceil(idx);
        if (lowIdx < 1) lowIdx = 1;
        if (higIdx < 1) continue;
        if (lowIdx > det_num) continue;
        if (higIdx > det_num) higIdx = det_num;
        const double wl = higIdx - idx, wh = idx - lowIdx;
        const int lo = (int)lowIdx - 1, hi = (int)higIdx - 1;
        for (size_t r = 0; r < rows; ++r) {                                         /* :30-33 */
            const double* src = proj + r * det_num;
            out[r * det_num + ii - 1] = src[lo] * wl + src[hi] * wh;
        }
    }
    return detWidth;
}
