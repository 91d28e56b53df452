/*
 * ctrecon.h -- C ABI of ctrecon-b200, a single-GPU (NVIDIA B200, sm_100a) implementation of
 * CTRecon's Katsevich exact helical cone-beam reconstruction chain:
 *
 *   derivative -> forward height rebin -> Hilbert filter -> backward rebin   (filter)
 *   PI-line solve -> voxel-driven backprojection                             (backprojection)
 *
 * Plain C types only (no CUDA or torch types): streams are passed as `void*` (a
 * cudaStream_t, NULL = the legacy default stream) and device buffers as plain pointers.
 * Every call returns a ctrecon_status; on failure ctrecon_last_error() describes it. No C++
 * exception crosses this boundary.
 *
 * Layouts are the reference's MATLAB column-major arrays:
 *   projections  Proj(YL, ZL, P)   linear index (p*ZL + z)*YL + y
 *                                  (KatsevichFiltering_GPU.cu:63, KatsevichFiltering.m:33)
 *   image        z fastest         linear index (x*NY + y)*NZ + z   (KatsevichBkProj.cpp:264)
 *
 * Threading: one context per host thread; a context is not thread-safe. Host (`_host_f64`)
 * calls are synchronous, like the reference's MEX functions; device (`_dev`) calls are
 * ordered on the given stream and return once the work is enqueued.
 */
#ifndef CTRECON_H
#define CTRECON_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CTRECON_ABI_VERSION 1

typedef enum ctrecon_status {
    CTRECON_OK = 0,
    CTRECON_ERR_INVALID_ARGUMENT = 1, /* sizes or parameters the chain cannot run */
    CTRECON_ERR_GEOMETRY = 2,         /* the reference would index outside an array */
    CTRECON_ERR_CUDA = 3,             /* a CUDA runtime call or kernel failed */
    CTRECON_ERR_OUT_OF_MEMORY = 4,    /* device or pinned-host allocation failed */
    CTRECON_ERR_NO_DEVICE = 5,        /* no usable sm_100 device */
    CTRECON_ERR_TIMEOUT = 6,          /* a bounded device-side wait gave up */
    CTRECON_ERR_UNSUPPORTED = 7,      /* option or size outside what this build supports */
    CTRECON_ERR_INTERNAL = 8
} ctrecon_status;

typedef struct ctrecon_ctx ctrecon_ctx;

/* Inputs 2..13 of KatsevichFiltering_GPU (KatsevichFiltering_GPU.cu:941-959), in order. */
typedef struct ctrecon_filter_params {
    double proj_scale;   /* ProjScale: views per turn */
    double dec_width;    /* DecWidth: detector width (mm) */
    double dec_height;   /* DecHeigh: detector height (mm) */
    double scan_r;       /* ScanR: source-to-axis distance */
    double std_dis;      /* StdDis: source-to-detector distance */
    double helic_p;      /* HelicP: helical pitch (table travel per turn) */
    double filter_coeff; /* FilterCoeFF: filtering coefficient tau */
    double delta_angle;  /* DeltaAngle: 2*acos(ObjR/ScanR) */
    int filtering_mode;  /* FilteringMode: 2 = dual symmetric operators, else single */
    int yl;              /* YL: detector columns */
    int zl;              /* ZL: detector rows */
    int proj_number;     /* ProjNumber: views */
} ctrecon_filter_params;

/* The geom struct of KatsevichBkProj (FunctionKat_v6.m:110-112, read at
 * KatsevichBkProj.cpp:80-95 and KatsevichBkProj_GPU.cu:353-374), field by position:
 *   locus    = [ScanR StdDis HelicP ProjScale ProjBeginIndex ProjEndIndex ProjCtr]
 *   detector = [DecWidth YL DecHeigh ZL DetCtrU DetCtrV]      (n_detector = 4 or 6)
 *   object   = [ObjR RecSX RecSY RecSZ DX DY DZ]              (n_object   = 4 or 7)
 * When present, DetCtrU/V and DX/DY/DZ are honoured (every reference caller passes
 * exactly (N-1)/2 and 2*ObjR/N, where this equals KatsevichBkProj.cpp). */
typedef struct ctrecon_bp_geom {
    double locus[7];
    double detector[6];
    double object[7];
    int n_detector;
    int n_object;
} ctrecon_bp_geom;

/* Hilbert-filter arithmetic (CTRECON_OPT_HILBERT). */
enum {
    CTRECON_HILBERT_FP32 = 0,   /* FP32 SIMT direct Toeplitz sum (the plain form) */
    CTRECON_HILBERT_BF16X3 = 1, /* tcgen05 Toeplitz GEMM, BF16 hi/lo split, 3 products */
    CTRECON_HILBERT_TF32 = 2    /* tcgen05 Toeplitz GEMM in TF32 */
};

/* PI-line solver (CTRECON_OPT_PI_SOLVER). All are FP64 and give the same endpoints bit for bit:
 * Newton finds the root, then the bisection is replayed from it (its midpoint decisions follow
 * from the root; the chord is evaluated where a decision is close to its threshold and at the
 * final midpoint), so the bisection decides every endpoint. */
enum {
    CTRECON_PI_BISECT = 0,  /* bisection of KatsevichBkProj.cpp:283-312 (the arbiter) */
    CTRECON_PI_NEWTON = 1,  /* safeguarded Newton from the axis point's PI line, then the
                               bisection replayed from its root */
    CTRECON_PI_LEARNED = 2  /* the same, Newton seeded by the trained PI-line network */
};

/* Derivative of the filter (CTRECON_OPT_DERIVATIVE). */
enum {
    CTRECON_DERIV_DIRECT = 0,  /* DerMode 0: KatsevichFiltering_T.m:50-101, the projections
                                  resampled for the source rotated by -/+ dL/2 and differenced:
                                  the derivative sits half a view later (its backprojection takes
                                  ProjCtr - 0.5, FunctionKat_v6.m:102) */
    CTRECON_DERIV_CHAIN = 1    /* DerMode 1: KatsevichFiltering.m:52-95, chain rule (default) */
};

/* CTRECON_OPT_PINET_MODE. The network's inputs are (r, cos psi, sin psi) with
 * psi = phi - 2 pi z / pitch (the helix's screw symmetry), so its prediction is a function of
 * (r, psi) alone. Whatever the mode, the FP64 solve decides every endpoint. */
enum {
    CTRECON_PINET_VOXEL_FP32 = 0, /* per voxel, FP32 SiLU (as ctrecon_pinet_predict) */
    CTRECON_PINET_VOXEL_BF16 = 1, /* per voxel, packed BF16 SiLU */
    CTRECON_PINET_GRID = 2        /* default: the network (FP32 SiLU) on a 256 x 4096 grid of
                                     (r, psi) each solve, each grid point refined by the FP64
                                     Newton solve from the network's output, bilinear in
                                     (r, psi) per voxel */
};

typedef enum ctrecon_option {
    CTRECON_OPT_HILBERT = 1,          /* CTRECON_HILBERT_*; default FP32 */
    CTRECON_OPT_PI_SOLVER = 2,        /* CTRECON_PI_*; default BISECT */
    CTRECON_OPT_FILTER_CHUNK = 3,     /* views per filter work chunk; default 2048 */
    CTRECON_OPT_BP_VARIANT = 4,       /* backprojector variant, default CTRECON_BP_AUTO (the
                                         tuning table's form for the geometry, else 12): 0, 1 = per-cell
                                         records, blocks of 4 / 8 views; 2, 3, 4 = second
                                         form (slices x views) 8x8, 4x8, 8x4; 5, 6, 7 = per-cell
                                         records staged by producer warps (views per block x
                                         ring slots x producer warps) 4x2x1, 2x4x1, 4x2x2;
                                         8, 9 = the same with 4x2x3, 4x3x4; 10, 11, 12 =
                                         per-cell records written to device memory first and
                                         copied in by one producer warp (views per block x
                                         ring slots x CTAs per SM) 4x3x3, 4x4x2, 8x2x2;
                                         100 = first form; CTRECON_BP_AUTO = the tuning
                                         table's choice */
    CTRECON_OPT_VERBOSE = 5,
    CTRECON_OPT_DERIVATIVE = 6,       /* CTRECON_DERIV_*; default CHAIN (the MEX filter's) */
    CTRECON_OPT_BP_WINDOW = 7,        /* views per cell-record window of variants 10..12;
                                         0 (default) = as many as 32 GiB of records hold,
                                         and at most half of the free device memory */
    CTRECON_OPT_PINET_MODE = 8,       /* how the learned PI solve evaluates the network:
                                         CTRECON_PINET_* below */
    CTRECON_OPT_KERNEL_TIMING = 9,    /* 1: time every kernel launch of the single-scan entry
                                         points with CUDA events on its stream (read with
                                         ctrecon_kernel_times); default 0 */
    CTRECON_OPT_TC_FORM = 10,         /* form of the tensor-core Hilbert: CTRECON_TC_* below */
    CTRECON_OPT_K1_FORM = 11,         /* form of the derivative + forward rebin: CTRECON_K1_* */
    CTRECON_OPT_HOST_THREADS = 12     /* host threads with which the host (FP64) calls convert
                                         their input views to FP32 before they cross to the
                                         device (half the bytes over the host link), each slot of
                                         views copied up as soon as it is converted, and widen
                                         ctrecon_filter_host_f64's FP32 results on the host when
                                         FProj is pageable; 0: copy FP64 and convert on the
                                         device; default -1: as many as the host has, at most
                                         16. The results are the same bit for bit. */
} ctrecon_option;

/* CTRECON_OPT_TC_FORM. Both forms compute the same sums to FP32 rounding. */
enum {
    CTRECON_TC_PARITY_SPLIT = 0, /* default: odd and even output columns as two half-size
                                    Toeplitz products (the taps vanish at even lags), one
                                    persistent CTA per SM overlapping each tile's backward rebin
                                    with the next tile's MMAs; views of up to 256 kappa rows */
    CTRECON_TC_SINGLE_PASS = 1   /* one full-size product per tile, then its backward rebin; also
                                    the form used for views of more than 256 kappa rows */
};

/* CTRECON_OPT_K1_FORM. Both forms write the same kappa rows bit for bit. */
enum {
    CTRECON_K1_STAGED = 0,  /* default: a CTA per (32-column strip, run of views) walks its
                               views in order, each view's rows copied in once by a tensor
                               copy, the strip's rebin entries held in shared memory; used
                               where it applies (chain-rule derivative, YL a multiple of 4, at
                               most 256 detector rows), else the per-view form */
    CTRECON_K1_PER_VIEW = 1 /* a CTA per (view, 128 columns), rows read from device memory */
};

/* ---- context ---------------------------------------------------------------------- */
ctrecon_status ctrecon_ctx_create(int device, ctrecon_ctx** out);
void ctrecon_ctx_destroy(ctrecon_ctx* ctx);
const char* ctrecon_last_error(const ctrecon_ctx* ctx);
const char* ctrecon_status_string(ctrecon_status s);
int ctrecon_abi_version(void);
ctrecon_status ctrecon_set_option(ctrecon_ctx* ctx, ctrecon_option opt, int value);
ctrecon_status ctrecon_get_option(const ctrecon_ctx* ctx, ctrecon_option opt, int* value);

/* ---- host, FP64, MEX-equivalent (synchronous) ------------------------------------------ */

/* Replaces the KatsevichFiltering_GPU MEX function (KatsevichFiltering_GPU.cu:939-978,
 * caller KatsevichFiltering.m:37-38): filters `proj` (YL x ZL x P doubles) and writes the
 * result into `fproj` (same shape; may alias `proj`, as the MATLAB caller's lazy copy
 * makes it). Computes KatsevichFiltering.m:39-287. */
ctrecon_status ctrecon_filter_host_f64(ctrecon_ctx* ctx, const ctrecon_filter_params* p,
                                       const double* proj, double* fproj);

/* Replaces the KatsevichBkProj / KatsevichBkProj_GPU MEX functions
 * (KatsevichBkProj.cpp:314-352, KatsevichBkProj_GPU.cu:332-429; callers
 * FunctionKat_v6.m:113, katsevichReconForGUI.m:107-109): backprojects `fproj` into
 * `image` in place. Voxels outside the cylinder of radius ObjR or without a PI interval
 * inside the scan keep their value, as in KatsevichBkProj.cpp. */
ctrecon_status ctrecon_bkproj_host_f64(ctrecon_ctx* ctx, const ctrecon_bp_geom* g,
                                       const double* fproj, double* image);

/* Filter + backprojection in one call with the filtered projections kept on the device
 * (FunctionKat_v6.m:85-113 without the intermediate FProj round trip). */
ctrecon_status ctrecon_recon_host_f64(ctrecon_ctx* ctx, const ctrecon_filter_params* p,
                                      const ctrecon_bp_geom* g, const double* proj,
                                      double* image);

/* ---- device, FP32, stream-ordered ------------------------------------------------------ */

/* Filter of device-resident FP32 projections (KatsevichFiltering_GPU<T>,
 * KatsevichFiltering_GPU.cu:858-935). d_fproj must not alias d_proj. */
ctrecon_status ctrecon_filter_dev_f32(ctrecon_ctx* ctx, void* stream,
                                      const ctrecon_filter_params* p, const float* d_proj,
                                      float* d_fproj);

/* FilteringMode 1 of the reference's driver (FunctionKat_v6.m:86-90): the average of the
 * filters with FilterCoeFF and 1 - FilterCoeFF, (FProj + FProj1) / 2, into d_fproj. Holds a
 * second filtered copy in the context (4 bytes per projection sample) while it runs. */
ctrecon_status ctrecon_filter_mode1_dev_f32(ctrecon_ctx* ctx, void* stream,
                                            const ctrecon_filter_params* p, const float* d_proj,
                                            float* d_fproj);

/* Bytes of the per-voxel PI-interval table written by ctrecon_pi_dev. The table holds 16-byte
 * records: every d_pitab argument must be 16-byte aligned (device allocations are), else the
 * call returns CTRECON_ERR_INVALID_ARGUMENT before any work. */
ctrecon_status ctrecon_pi_table_bytes(const ctrecon_bp_geom* g, size_t* bytes);

/* PI-line solve for every voxel (PISegment, KatsevichBkProj.cpp:283-312 and the interval
 * and endpoint rules of :177-234) into d_pitab. If d_updates is not NULL it receives (on
 * the device, as one unsigned long long) sum(LoopEnd-LoopBegin+1) over written voxels. */
ctrecon_status ctrecon_pi_dev(ctrecon_ctx* ctx, void* stream, const ctrecon_bp_geom* g,
                              void* d_pitab, unsigned long long* d_updates);

/* Voxel-driven backprojection (KatsevichBkProj.cpp:164-265) of device-resident FP32
 * filtered projections into the device FP32 image (in place: unwritten voxels keep their
 * value). d_pitab from ctrecon_pi_dev, or NULL to solve the PI lines internally. */
ctrecon_status ctrecon_bkproj_dev_f32(ctrecon_ctx* ctx, void* stream,
                                      const ctrecon_bp_geom* g, const float* d_fproj,
                                      const void* d_pitab, float* d_image);

/* The plain FP32 filter (same result as ctrecon_filter_dev_f32 with CTRECON_HILBERT_FP32) for
 * callers that cannot allocate GPU memory -- e.g. a plug-in inside an application that owns all
 * device allocations, or a real-time loop that forbids cudaMalloc after start-up. No
 * counterpart in the reference: it is an addition of this library. It allocates nothing and
 * needs no context: its tables and kappa-row scratch live in one fixed 16 MiB device array of
 * the library (held by every GPU that loads the library, until exit); sizes that do not fit
 * (tables + one view of kappa rows > 16 MiB) return CTRECON_ERR_UNSUPPORTED with the sizes
 * in ctrecon_last_error(NULL). The caller passes the input and output buffers (distinct) and
 * a stream; the call is stream-ordered. The first call on a device looks up the array's
 * device address (cudaGetSymbolAddress) with that device current and keeps it for the life of
 * the process (it assumes the device's primary context is not reset); make that first call
 * before any stream capture. Every call copies its tables into the array from a temporary host
 * buffer, so it must not be called while its stream is being captured: it then returns
 * CTRECON_ERR_UNSUPPORTED and enqueues nothing. Every call shares the array and leaves its
 * contents behind, so calls that overlap on the GPU (concurrent streams, or several host
 * threads) race; serialise them. A successful call clears ctrecon_last_error(NULL). */
ctrecon_status ctrecon_filter_noalloc_dev_f32(void* stream, const ctrecon_filter_params* p,
                                              const float* d_proj, float* d_fproj);

/* Device time per kernel kind of the launches made since the last call while
 * CTRECON_OPT_KERNEL_TIMING was on, in milliseconds, with the launch counts; the kinds are
 * 0 derivative + forward rebin (k_deriv_rebin), 1 FP32 Hilbert + backward rebin
 * (k_hilbert_simt), 2 tensor-core Hilbert + backward rebin (k_hilbert_tc), 3 PI-line solve
 * (with the learned start's network), 4 cell records of the fifth backprojector form,
 * 5 backprojection (any form). Arrays of n entries; waits for the timed work. No counterpart in
 * the reference (a profiling aid). */
#define CTRECON_KERNEL_KINDS 6
ctrecon_status ctrecon_kernel_times(ctrecon_ctx* ctx, double* ms, unsigned long long* launches,
                                    int n);

/* Waits for the work enqueued on `stream` and reports device-side failures: a CUDA error,
 * or CTRECON_ERR_TIMEOUT when a bounded wait inside a kernel gave up. */
ctrecon_status ctrecon_sync(ctrecon_ctx* ctx, void* stream);

/* PI-line solve as ctrecon_pi_dev, also counting the solver's chord evaluations (device
 * unsigned long long, summed over solved voxels): bisection steps for CTRECON_PI_BISECT, Newton
 * steps plus the replay's evaluations for CTRECON_PI_NEWTON / CTRECON_PI_LEARNED. */
ctrecon_status ctrecon_pi_dev_stats(ctrecon_ctx* ctx, void* stream, const ctrecon_bp_geom* g,
                                    void* d_pitab, unsigned long long* d_updates,
                                    unsigned long long* d_iters);

/* ---- batches of uneven scans (no counterpart in the reference) ----------------------------
 * A batch reconstructs n scans with their own geometries. Each run enqueues every scan's filter
 * and PI solve, then ONE persistent backprojection launch over the tiles of all scans (largest
 * scans first, CTAs pulling tiles from a shared counter). With use_graph != 0 the first run is
 * eager and the second is captured into a CUDA graph that later runs replay (re-captured when
 * the buffer pointers change); graph mode needs a created stream. The batch uses the context's
 * options (Hilbert mode, PI solver, backprojector variant) and its work buffers: one batch run
 * at a time per context. */
typedef struct ctrecon_batch ctrecon_batch;
ctrecon_status ctrecon_batch_create(ctrecon_ctx* ctx, int n_scans,
                                    const ctrecon_filter_params* params,
                                    const ctrecon_bp_geom* geoms, ctrecon_batch** out);
void ctrecon_batch_destroy(ctrecon_batch* batch);
/* backprojector form of every scan of the batch: 0 .. 12 as CTRECON_OPT_BP_VARIANT (default:
 * the context's when it names a form 0 .. 12, else 2); scans that share a form share one
 * persistent launch. The fifth form
 * (10 .. 12) holds the cell records of all its scans at once (16 bytes per detector cell and
 * view) and writes them right before the launch. */
ctrecon_status ctrecon_batch_set_variant(ctrecon_batch* batch, int variant);
/* per-scan forms (n = the batch's scan count) */
ctrecon_status ctrecon_batch_set_variants(ctrecon_batch* batch, const int* variants, int n);
/* the form of each scan (n >= the batch's scan count) */
ctrecon_status ctrecon_batch_get_variants(const ctrecon_batch* batch, int* variants, int n);
/* d_proj[i] (input), d_fproj[i] (work), d_image[i] (output, in place) for scan i */
ctrecon_status ctrecon_batch_run_dev(ctrecon_batch* batch, void* stream,
                                     const float* const* d_proj, float* const* d_fproj,
                                     float* const* d_image, int use_graph);
/* sum(LoopEnd-LoopBegin+1) of each scan (bisection PI solve, synchronous) */
ctrecon_status ctrecon_batch_updates(ctrecon_batch* batch, unsigned long long* host_updates);

/* ---- autotuner (no counterpart in the reference) -----------------------------------------
 * Times candidate backprojector forms -- tile shapes (slices per thread) and view-block
 * depths / staging rings, the CTRECON_OPT_BP_VARIANT values -- on the caller's own data and
 * keeps the fastest. Timing uses CUDA events on `stream` and is synchronous. The
 * backprojection assigns voxel values (it does not accumulate), so tuning on the caller's
 * image leaves it as one backprojection would. */
#define CTRECON_BP_AUTO (-1) /* CTRECON_OPT_BP_VARIANT value: use the tuning table */
#define CTRECON_TUNE_MAX 16
typedef struct ctrecon_tune_result {
    int best_variant;
    float best_ms;                      /* mean device time per launch of the best form */
    int n;                              /* candidates tried */
    int variants[CTRECON_TUNE_MAX];
    float ms[CTRECON_TUNE_MAX];         /* mean time per launch; -1 = does not fit */
} ctrecon_tune_result;
/* Single scan: tunes the backprojection of d_fproj with the PI table d_pitab (NULL: solved
 * first) into d_image, records the winner for this geometry in the context's tuning table
 * (used when CTRECON_OPT_BP_VARIANT is CTRECON_BP_AUTO) and returns the timings. */
ctrecon_status ctrecon_tune_bkproj(ctrecon_ctx* ctx, void* stream, const ctrecon_bp_geom* g,
                                   const float* d_fproj, const void* d_pitab, float* d_image,
                                   ctrecon_tune_result* out);
/* Batch: runs the batch once (filters and PI solves included), then times every candidate form
 * on each scan and keeps each scan's fastest (ctrecon_batch_get_variants); scans are grouped by
 * form, one persistent launch per group. `out` gives, per candidate, the summed time over the
 * scans, best_ms the sum of the scans' best times and best_variant the most chosen form. */
ctrecon_status ctrecon_batch_tune(ctrecon_batch* batch, void* stream, const float* const* d_proj,
                                  float* const* d_fproj, float* const* d_image,
                                  ctrecon_tune_result* out);
/* The tuning table as text (one geometry per line); load merges into the context's table. */
ctrecon_status ctrecon_tune_save(const ctrecon_ctx* ctx, const char* path);
ctrecon_status ctrecon_tune_load(ctrecon_ctx* ctx, const char* path);

/* ---- learned PI-line initialiser (no counterpart in the reference) -----------------------
 * A 3 -> 64 -> 64 -> 64 -> 64 -> 2 SiLU network mapping (r/0.25, cos psi, sin psi), with r and
 * psi = phi - 2 pi z the voxel's normalised radius and helix-relative angle, to 4x the offsets
 * of the PI-line endpoints from the on-axis solution (sb = 2 pi z - pi/2, st = 2 pi z + pi/2).
 * The network lives in the context; CTRECON_PI_LEARNED uses it as the start of the FP64 Newton
 * solve. Parameters: per layer W[out][in] row-major then b[out], FP32 (inference in BF16). */
int ctrecon_pinet_num_params(void);
/* Trains from scratch on n_pairs FP64-solved (point, endpoint) pairs, area-uniform in the disc
 * of normalised radius r_max (ObjR/ScanR or more), with Adam; synchronous. */
ctrecon_status ctrecon_pinet_train(ctrecon_ctx* ctx, void* stream, int n_pairs, int batch,
                                   int epochs, double r_max, uint64_t seed, float* final_loss);
ctrecon_status ctrecon_pinet_get_params(ctrecon_ctx* ctx, float* host_params, int n);
ctrecon_status ctrecon_pinet_set_params(ctrecon_ctx* ctx, const float* host_params, int n,
                                        double r_max);
/* Mean (over n samples) squared error of the current parameters and its gradient (device
 * buffers: d_feat n x 3, d_targ n x 2, d_grad ctrecon_pinet_num_params(), d_loss 1). */
ctrecon_status ctrecon_pinet_loss_grad(ctrecon_ctx* ctx, void* stream, const float* d_feat,
                                       const float* d_targ, int n, float* d_grad,
                                       float* d_loss);
/* Network outputs (n x 2) of the BF16 inference kernel for n feature triples. */
ctrecon_status ctrecon_pinet_predict(ctrecon_ctx* ctx, void* stream, const float* d_feat, int n,
                                     float* d_out);

/* ---- tables and helpers (host only, no GPU needed) --------------------------------------- */

/* Number of kappa lines AL = 2*ceil(0.65*ZL)+1 (KatsevichFiltering.m:103-104). */
int ctrecon_num_kappa(int zl);

/* The filter's FP64 host tables, as the device uses them (rounded to FP32 there):
 * forward rebin (KatsevichFiltering.m:131-153): per (a, y) rows r0/r1 and weights
 *   wa/wb including the pre-weight, X[a][y] = wa*GF[r0][y] + wb*GF[r1][y];
 * backward rebin (:191-287): per (z, y) kappa rows b/e and weights gb/ge including the
 *   Hilbert sign and the post-weight, FProj[z][y] = gb*H[b][y] + ge*H[e][y] where H is
 *   the unsigned Hilbert sum. Arrays are [AL*YL] (index a*YL+y) and [ZL*YL] (z*YL+y);
 *   any may be NULL. */
ctrecon_status ctrecon_filter_tables(const ctrecon_filter_params* p, int* r0, int* r1,
                                     double* wa, double* wb, int* b, int* e, double* gb,
                                     double* ge);

/* Filtering coefficient tau of FindTau.m:6-22: the root in [0, 0.5] of
 * t*cos(am) - cos(t*am) + 1 - t with am = 2*pi - 2*acos(ratio), ratio = ObjR/ScanR, found by
 * the script's bisection until |f| <= tol (the script uses ratio 2/3 and tol 1e-4). */
ctrecon_status ctrecon_find_tau(double ratio, double tol, double* tau);

/* Detector sizing of FunctionKat_v6.m:49-57 (with its PI = 3.1415926). */
void ctrecon_geometry_sizing(double scan_r, double std_dis, double helic_p, double obj_r,
                             int yl, int zl, double* dec_width, double* dec_height,
                             double* delta);

/* ---- analytic ellipsoid phantom (input generator; FP64 on the device) ------------------- */

/* Line integrals of n_ell ellipsoids (rows of 10 doubles: cx cy cz a b c phi theta psi
 * density; ZXZ Euler angles) for all views of geometry g into d_proj (FP32, layout
 * above), the chord formula of CreateProjSlice.cpp:98-134 on a flat detector. If
 * photons > 0, Poisson noise with `photons` incident photons per ray is applied with the
 * attenuation scale mu = 8/max(line integral) (seeded, reproducible). */
ctrecon_status ctrecon_phantom_project_dev(ctrecon_ctx* ctx, void* stream,
                                           const ctrecon_bp_geom* g, const double* ell,
                                           int n_ell, double photons, uint64_t seed,
                                           float* d_proj);

/* ---- arc detector to flat panel (rebinToPanel.m:1-36) -------------------------------------
 * Resamples projections from an arc detector (det_num columns of arc length det_cell_width at
 * distance sour_to_det, centre index det_center_idx 0-based) onto a flat panel with the same
 * column count and width 2 D tan(largest half fan) (returned in *det_width, may be NULL).
 * d_proj / d_out: [prj_num][det_hei][det_num] (MATLAB det_num x det_hei x prj_num), distinct.
 * The reference's edge rules are kept: columns it skips are 0, and a panel column whose fan
 * angle falls exactly on an arc-cell centre is 0 as well (its weights use clamped indices).
 * The FP64 variant reproduces the reference's arithmetic exactly; stream-ordered. */
ctrecon_status ctrecon_rebin_to_panel_dev_f32(ctrecon_ctx* ctx, void* stream, const float* d_proj,
                                              int det_num, int det_hei, int prj_num,
                                              double det_center_idx, double det_cell_width,
                                              double sour_to_det, float* d_out,
                                              double* det_width);
ctrecon_status ctrecon_rebin_to_panel_dev_f64(ctrecon_ctx* ctx, void* stream, const double* d_proj,
                                              int det_num, int det_hei, int prj_num,
                                              double det_center_idx, double det_cell_width,
                                              double sour_to_det, double* d_out,
                                              double* det_width);

/* ---- the reference's data files (host only, no GPU) ---------------------------------------
 * ProjectionData.m:113-176 and ReconImage.m:60-117 store little-endian doubles: a header of
 * scalars, the data array, then a 3-entry storage order ([1 2 3] = U V P for projections,
 * X Y Z for images; the data's MATLAB dimensions are those axes in that order). The readers
 * validate the file size against the header; `data` may be NULL to read the header alone. */
typedef struct ctrecon_projfile_header {
    double source_to_center, source_to_detector;  /* SourceToCenterDistance, ...DetectorDistance */
    double det_reso_u, det_reso_v;                /* DetResoU, DetResoV (cells) */
    double det_pixel_u, det_pixel_v;              /* DetPixelSizeU, DetPixelSizeV */
    double det_center_u, det_center_v;            /* DetCntIdxU, DetCntIdxV (0-based) */
    double is_arc;                                /* IsArcDetector (1 arc, 0 flat) */
    double start_angle_deg, start_z, pitch;       /* StartSourceAngle, StartSourceZPos, Pitch */
    double total_views, views_per_turn;           /* TotalProjectionNumber, ...PerTurn */
    double storage_order[3];                      /* StorageOrder */
} ctrecon_projfile_header;
ctrecon_status ctrecon_projfile_read(const char* path, ctrecon_projfile_header* h, double* data,
                                     size_t capacity);
ctrecon_status ctrecon_projfile_write(const char* path, const ctrecon_projfile_header* h,
                                      const double* data);

typedef struct ctrecon_imgfile_header {
    double reso[3];          /* resoX, resoY, resoZ */
    double pixel[3];         /* pixelSizeX, ... */
    double ctr_idx[3];       /* ctrIdxX, ... */
    double center[3];        /* imgCenterX, ... */
    double storage_order[3]; /* storageOrder */
} ctrecon_imgfile_header;
ctrecon_status ctrecon_imgfile_read(const char* path, ctrecon_imgfile_header* h, double* data,
                                    size_t capacity);
ctrecon_status ctrecon_imgfile_write(const char* path, const ctrecon_imgfile_header* h,
                                     const double* data);

/* ---- failure detection ------------------------------------------------------------------ */
/* Every pipelined kernel of the library bounds its waits (2 s of %globaltimer): a wait that
 * gives up records a code in the context's device error word, the kernel returns, and the call
 * reports CTRECON_ERR_TIMEOUT. This self-test runs that mechanism on a wait that nothing ever
 * completes (limit_ms, 1..10000): it returns CTRECON_ERR_TIMEOUT when the wait gave up and was
 * reported, CTRECON_ERR_INTERNAL otherwise; the context stays usable. */
ctrecon_status ctrecon_selftest_bounded_wait(ctrecon_ctx* ctx, void* stream, int limit_ms);

#ifdef __cplusplus
}
#endif
#endif /* CTRECON_H */
