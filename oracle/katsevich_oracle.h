/*
 * katsevich_oracle.h -- FP64 CPU oracle of the Katsevich chain (TEST INFRASTRUCTURE).
 *
 * This is the checker, never the product: only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load it. Every function restates the reference's
 * algorithm in plain C, in the reference's own FP64 arithmetic order, and cites the
 * reference lines it follows (paths relative to the CTRecon source tree).
 *
 * Pinning: the backprojector restatement is checked bit-for-bit against
 * KatsevichBkProj.cpp itself, compiled unchanged into oracle/_ref/ by
 * oracle/Makefile; the geometry sizing is checked against the constants recorded in
 * KatsevichFiltering_GPU.cu:997 and KatsevichBkProj_GPU.cu:465-479. The filter
 * restatement (KatsevichFiltering.m needs MATLAB or Octave, absent here) is pinned by
 * its stage identities (Toeplitz == FFT convolution, derivative stencils) and by the
 * golden vectors under tests/golden/.
 *
 * Arrays use the reference's MATLAB column-major layouts:
 *   Proj/FProj  (YL, ZL, P)  -> linear index (p*ZL + z)*YL + y
 *   image       z fastest    -> linear index (x*NY + y)*NZ + z   (KatsevichBkProj.cpp:264)
 */
#ifndef KATSEVICH_ORACLE_H
#define KATSEVICH_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* The reference's pi for the filter and backprojector (KatsevichFiltering.m:32,
 * KatsevichBkProj.cpp:25). */
#define ORC_PI 3.14159265358979

/* Inputs 2..13 of KatsevichFiltering_GPU / arguments of KatsevichFiltering.m:1. */
typedef struct {
    double ProjScale, DecWidth, DecHeigh, ScanR, StdDis, HelicP, FilterCoeFF, DeltaAngle;
    int FilteringMode, YL, ZL, ProjNumber;
} orc_filter_params;

/* The geom struct of KatsevichBkProj (FunctionKat_v6.m:110-112), by position. */
typedef struct {
    double locus[7];    /* ScanR StdDis HelicP ProjScale ProjBeginIndex ProjEndIndex ProjCtr */
    double detector[6]; /* DecWidth YL DecHeigh ZL DetCtrU DetCtrV */
    double object[7];   /* ObjR RecSX RecSY RecSZ DX DY DZ */
    int n_detector;     /* entries present in detector[] (4 or 6) */
    int n_object;       /* entries present in object[]   (4 or 7) */
    int honour_extras;  /* 0: exactly KatsevichBkProj.cpp (ignores DX.. and DetCtr..);
                           1: use DX/DY/DZ and DetCtrU/V when present */
} orc_bp_geom;

/* ---- geometry sizing: FunctionKat_v6.m:49-57 (with the driver's PI = 3.1415926) ---- */
void orc_geometry_sizing(double ScanR, double StdDis, double HelicP, double ObjR, int YL,
                         int ZL, double* DecWidth, double* DecHeigh, double* delta);

/* ---- filter (KatsevichFiltering.m:39-287) ---- */
int orc_num_kappa(int ZL, int* QQ); /* returns AL; QQ = ceil(ZL*1.3*0.5) (:103-104) */

/* Kappa-line geometry (:102-126,150) and backward-rebin decisions (:191-280).
 * Outputs (each may be NULL): AZCor[AL*YL], coef[AL*YL] (index a*YL + y), Rato[AL],
 * forward-rebin rows/weights lw[AL*YL] (zero-based lower row), w_lw, w_up (:134-145),
 * backward-rebin zero-based rows bAL/eAL[ZL*YL] and weights bC/eC (index z*YL + y).
 * Returns 0, or -1 when the reference would index a kappa row outside 1..AL (a MATLAB
 * index error in :283-284), or -2 for arguments the reference cannot run. */
int orc_filter_tables(const orc_filter_params* fp, double* AZCor, double* coef,
                      double* Rato, int* lw, double* w_lw, double* w_up, int* bAL,
                      int* eAL, double* bC, double* eC);

/* Hilbert impulse response h[m], m = -(YL-1)..YL-1 at h[m + YL - 1], exactly as the
 * circular kernel of :160-166 built by CreateHSP.m:11-23 (rectangle window). */
int orc_hilbert_taps(int YL, double* h);

/* Full filter for views [p_begin, p_end) of Proj (all P views must be readable, the
 * derivative needs view neighbours). FProj gets the same views. nthreads <= 0: all. */
int orc_filter(const orc_filter_params* fp, const double* Proj, double* FProj, int p_begin,
               int p_end, int nthreads);
/* KatsevichFiltering_T.m (DerMode 0): the same filter with the direct half-view derivative. */
int orc_filter_direct(const orc_filter_params* fp, const double* Proj, double* FProj,
                      int p_begin, int p_end, int nthreads);
/* Its derivative stage alone (KatsevichFiltering_T.m:50-101) for view p into GF[ZL*YL]. */
int orc_derivative_direct(const orc_filter_params* fp, const double* Proj, int p, double* GF);

/* Stage outputs for one view (for stage-level tests): GF (ZL*YL) after step 1,
 * ConvRes before the Hilbert (AL*YL, pre-weighted, index a*YL + y), and after the
 * Hilbert and post-weight. Any output may be NULL. */
int orc_filter_view_stages(const orc_filter_params* fp, const double* Proj, int p,
                           double* GF, double* conv_in, double* conv_out);

/* ---- filtering coefficient: FindTau.m:6-22 ----
 * Bisection on [0, 0.5] for t*cos(am) - cos(t*am) + 1 - t = 0 with am = 2*pi - 2*acos(ratio)
 * (ratio = ObjR/ScanR; the script uses 2/3), stopping when |f| <= tol (the script: 1e-4). */
double orc_find_tau(double ratio, double tol);

/* ---- PI line: KatsevichBkProj.cpp:283-312 ---- */
void orc_pisegment(double x, double y, double z, double* BAngle, double* TAngle);

/* ---- backprojection: KatsevichBkProj.cpp:71-281 ----
 * Writes image voxels with x in [x_begin, x_end) and z in [z_begin, z_end) (pass
 * 0, 0 for "all"); untouched voxels keep their value. n_updates (may be NULL) gets
 * sum(LoopEnd-LoopBegin+1) over written voxels; touched (may be NULL, one byte per
 * voxel of the full volume) is set to 1 for written voxels. */
int orc_bkproj(const orc_bp_geom* g, const double* proj, double* image, int x_begin,
               int x_end, int z_begin, int z_end, int nthreads, long long* n_updates,
               unsigned char* touched);

/* Per-voxel PI-interval record (the quantities of KatsevichBkProj.cpp:176-234):
 * B and T as fractional view indices (BAngle, TAngle after :177-178), LoopBegin and
 * LoopEnd, valid = 1 if the voxel is written. Arrays have NX*NY*NZ entries. */
int orc_pi_table(const orc_bp_geom* g, double* B, double* T, int* loop_begin,
                 int* loop_end, unsigned char* valid, int nthreads);

/* ---- analytic ellipsoid phantom: CreateProjSlice.cpp:62-138, generalised ----
 * ell: n rows of (cx, cy, cz, a, b, c, phi, theta, psi, density), mm and radians,
 * ZXZ Euler angles; body-frame coordinates are R^T (p - c) with R = Rz(phi) Rx(theta)
 * Rz(psi). Flat detector at distance StdDis from the source, cells centred on
 * ((y-(YL-1)/2)*DecWidth/YL, (z-(ZL-1)/2)*DecHeigh/ZL). Views [p_begin, p_end),
 * source angle (p + ProjBeginIndex - ProjCtr)*2*pi/ProjScale. */
int orc_project_ellipsoids(const orc_bp_geom* g, const double* ell, int n_ell,
                           double* proj, int p_begin, int p_end, int nthreads);

/* rebinToPanel.m:1-36: arc detector (det_num columns, centre index c 0-based, cell width w at
 * source distance D) to a flat panel of the same column count; proj is [views][rows][det_num]
 * (MATLAB det_num x det_hei x prj_num). Columns the reference skips stay 0. Returns the panel
 * width detWidth. */
double orc_rebin_to_panel(const double* proj, int det_num, int det_hei, int prj_num,
                          double c, double w, double D, double* out);

#ifdef __cplusplus
}
#endif
#endif
