"""Benchmark: Katsevich helical cone-beam reconstruction of a 512^3 volume on B200.

Workload (default, c3): flat detector 128 rows x 1024 columns at 0.8 mm, source radius 600 mm,
source-detector 1200 mm, 2304 views/turn over 6 turns (13824 views), pitch 0.9x the
Tam-Danielson window, 40 seeded random ellipsoids, 512^3 FP32 volume at 2*ObjR/512 = 0.469 mm.
Synthetic data made on the device by the analytic FP64 projector (not timed). `--config c2`
runs the 512x512x256 plain-FP32 scan (64 x 736 detector, 9280 views, Poisson noise) instead.

One step = the whole hot path over one scan: filter (derivative, forward height rebin,
Hilbert, backward rebin) -> PI-line solve -> voxel-driven backprojection.

Metric: GUPS = voxel-view updates per second, the update count being the reference's own
loop count sum(LoopEnd - LoopBegin + 1) over written voxels (KatsevichBkProj.cpp:237), taken
from the bisection PI solve and used for every form. `value` is the plain FP32 form (FP32
Hilbert, bisection PI solve) with inputs resident in HBM (all ranks' updates / max-over-ranks
time). Beside it, on the same resident inputs: `forms.mixed_learned` (BF16x3 tensor-core
Hilbert, the learned PI start) and `forms.mixed_learned_batched` (the same for two copies of the
scan in one batch: one persistent backprojection launch over both, replayed as a CUDA graph),
each with `vs_plain`; `accuracy` gives every form's relative RMSE and max-abs against the FP64
oracle of the whole chain on a central 48^3 block. `e2e` is the plain form end to end through
the C ABI's whole-chain call `ctrecon_recon_host_f64` (FP64 pinned host buffers, copies in the
timed region); `e2e_mex_pinned` through the two MEX-equivalent calls (FProj comes down and goes
back up in between) and `e2e_pageable` through the MEX modules themselves with pageable FP64
arrays, as MATLAB calls them.
`roofline` is the backprojection kernel's (the dominant one) against its issue limit;
`kernels` gives every kernel's time and roofline fraction, from CUDA events around each launch.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config c3|c2]
                    [--hilbert fp32|bf16x3|tf32] [--pi bisect|newton|learned]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from ctrecon_b200.geometry import config  # noqa: E402

def workload_name(s):
    """e.g. katsevich_helical_512x512x256_det64x736_9280views_40ellipsoids_poisson1e5"""
    noise = f"_poisson{s.photons:.0e}".replace("+0", "").replace("+", "") if s.photons else ""
    return (f"katsevich_helical_{s.NX}x{s.NY}x{s.NZ}_det{s.ZL}x{s.YL}_{s.P}views_"
            f"{s.n_ellipsoids}ellipsoids{noise}")
METRIC = "Katsevich 512^3 recon GUPS & s/vol: plain FP32 vs mixed+learned @ equal RMSE"
BYTES_PER_UPDATE = 16  # four FP32 bilinear taps (KatsevichBkProj.cpp:253-256)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c3")
    ap.add_argument("--hilbert", default="fp32", choices=["fp32", "bf16x3", "tf32"])
    ap.add_argument("--pi", default="bisect", choices=["bisect", "newton", "learned"])
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip the mixed + learned measurement beside the plain line")
    ap.add_argument("--pinet-mode", default="grid", choices=["voxel-fp32", "voxel-bf16", "grid"],
                    help="learned PI solve: the network per voxel (FP32 or packed BF16 SiLU) or "
                         "on the (r, psi) screw-symmetry grid, interpolated (default)")
    ap.add_argument("--bp-variant", type=int, default=-1,
                    help="backprojector form: -1 autotuned on the workload before timing "
                         "(default), 0, 1 per-cell records (4 / 8 views per block), 2-4 second "
                         "form tile shapes, 5-9 per-cell records staged by producer warps, "
                         "10-12 cell records written to HBM first and brought in by tensor "
                         "copies, 100 first form")
    ap.add_argument("--bp-window", type=int, default=0,
                    help="views per cell-record window of the fifth backprojector form (0: as "
                         "many as fit); smaller windows hold less device memory")
    ap.add_argument("--batched", action="store_true",
                    help="16 uneven scans (c4): one-at-a-time vs one batched graph replay")
    ap.add_argument("--report", choices=["c3", "c5", "extras", "refgpu"],
                    help="c3: error of each Hilbert variant vs the FP64 oracle and their times; "
                         "c5: the learned PI initialiser at 1024^3 (iterations saved, endpoint "
                         "agreement, time vs the plain form); extras: the panel rebin, "
                         "DerMode 0, FilteringMode 1 and the file formats on the c2 scan; "
                         "refgpu: the reference's own GPU MEX files recompiled for sm_100a "
                         "(baseline/_ref) timed and checked beside this library on the c2 scan")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the FP64 oracle check of each form on the central block")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the mixed + learned + batched form (two scans, one graph)")
    return ap.parse_args()


def load_peaks():
    """Roofline denominators: MEASURED_PEAKS.json (copy bandwidth, cuBLAS BF16 burst and
    sustained), else the pool's earlier measurement ("fallback")."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"]),
                "bf16_tflops_sustained": float(d.get("bf16_tflops_sustained", d["bf16_tflops"])),
                "source": "measured"}
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0,
                "source": "fallback"}


def load_profile_table(name):
    """Rows `kernel workload value` of a committed ncu summary table under profiles/."""
    out = {}
    try:
        for line in open(os.path.join(ROOT, "profiles", name)):
            parts = line.split()
            if len(parts) >= 3 and not line.startswith("#"):
                out[(parts[0], parts[1])] = float(parts[2])
    except OSError:
        pass
    return out


def load_traffic(kernel, workload):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary, if any."""
    return load_profile_table("traffic.txt").get((kernel, workload))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if not self.proc:
            return out
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sms, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sms.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        if sms:
            out = {"sm_mhz": statistics.median(sms), "sm_max_mhz": mx,
                   "reasons": sorted(reasons), "samples": len(sms)}
        return out


def dist_setup(n, backend=None):
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE). The ranks are
    replicas: each reconstructs its own scan and only the timing is reduced. NCCL on GPUs,
    gloo without them (the CPU tests of this plumbing)."""
    import torch
    import torch.distributed as dist
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        from datetime import timedelta
        backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        extra = {"device_id": torch.device("cuda", local)} if backend == "nccl" else {}
        dist.init_process_group(backend, timeout=timedelta(seconds=300), **extra)
    if torch.cuda.is_available():
        torch.cuda.set_device(local)
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, ws):
    """The largest of the ranks' x (every rank gets it): step times are the slowest rank's."""
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_gups(updates, ms_step, ws):
    """Whole-job throughput of ws replicas, each doing `updates` per step, timed by the
    slowest (ms_step = max over ranks)."""
    return ws * updates / (ms_step / 1e3) / 1e9


# ---------------------------------------------------------------------------------------------
# CPU baselines (the oracle restatement, or the reference's own compiled backprojector)
# ---------------------------------------------------------------------------------------------
def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    return oracle


def block_problem(O, s, n=48):
    """A central n^3 block of the volume at the workload's voxel pitch, posed as a geom the
    reference's MEX accepts (it derives the pitch from ObjR as 2*ObjR/N), restricted to the
    views [lo, hi) its PI intervals need (with a 2-view margin, so the loop bounds and
    endpoint weights are those of the full scan)."""
    dx = s.voxel_size[0]
    obj = [dx * n / 2.0, float(n), float(n), float(n), dx, dx, dx]
    g = O.bp_geom(s.locus(), s.detector(), obj, honour_extras=True)
    pit = O.pi_table(g)
    v = pit["valid"]
    lo = max(0, int(np.floor(pit["B"][v].min())) - 3)
    hi = min(s.P, int(np.ceil(pit["T"][v].max())) + 4)
    locus = s.locus()
    locus[4] = float(lo + 1)          # ProjBeginIndex (one-based)
    locus[5] = float(hi)              # ProjEndIndex
    return locus, s.detector(), obj, lo, hi


def cpu_filter_views(O, s, proj_sub):
    """FP64 filter restatement of a contiguous view range; the first and last view only
    serve as derivative neighbours and are not valid outputs."""
    fp = O.filter_params(ProjScale=float(s.views_per_turn), DecWidth=s.DecWidth,
                         DecHeigh=s.DecHeigh, ScanR=s.ScanR, StdDis=s.StdDis, HelicP=s.HelicP,
                         FilterCoeFF=s.filter_coeff, DeltaAngle=s.delta,
                         FilteringMode=s.filtering_mode, YL=s.YL, ZL=s.ZL,
                         ProjNumber=proj_sub.shape[0])
    return O.katsevich_filter(fp, proj_sub)


def workload_config(s, ws):
    """The `config` of both arms' lines: the workload, nothing of the implementation."""
    gb = 4 * s.P * s.ZL * s.YL / 1e9
    return {"workload": workload_name(s), "volume": list(s.vol_shape),
            "voxel_mm": [round(v, 6) for v in s.voxel_size], "detector": [s.ZL, s.YL],
            "views": s.P, "views_per_turn": s.views_per_turn, "parallelism": f"replicas{ws}",
            "l2": (f"inputs larger than L2 (FP32 projections {gb:.2f} GB)" if gb > 0.126 else
                   f"inputs smaller than L2 (FP32 projections {gb:.3f} GB): a test size")}


def _ref_worker(args):
    locus, det, obj, fproj_path = args
    O = _oracle()
    fproj = np.ascontiguousarray(np.load(fproj_path))
    n = int(obj[1])
    img = np.zeros((n, n, n))
    geom = {"Locus": np.array(locus), "Detector": np.array(det), "Object": np.array(obj)}
    t = time.perf_counter()
    O.ref_bkproj(geom, fproj, img)
    return time.perf_counter() - t


class CpuChainSample:
    """A bounded sample of the whole chain on the host cores, sized so that its own throughput
    is the full scan's: the backprojection of a central n^3 block (one copy per process, or
    OpenMP threads) and the filter of the same fraction of the scan's views as the block's
    updates are of the scan's updates. Then GUPS = sample updates / sample time, with
    full-scan time = full updates / GUPS."""

    def __init__(self, O, s, d_proj_views, full_updates, n=32, copies=1):
        self.O, self.s, self.n, self.copies = O, s, n, copies
        self.locus, self.det, self.obj, lo, hi = block_problem(O, s, n)
        self.gb = O.bp_geom(self.locus, self.det, self.obj, honour_extras=True)
        proj_b = d_proj_views(max(0, lo - 1), min(s.P, hi + 1))
        a = max(0, lo - 1)
        self.fproj = np.ascontiguousarray(cpu_filter_views(O, s, proj_b)[lo - a:hi - a])
        _, self.block_updates = O.bkproj(self.gb, self.fproj, np.zeros((n, n, n)))
        self.updates = copies * self.block_updates
        # filtered views in the same proportion to the scan's views as the updates
        self.nview = max(1, int(round(s.P * self.updates / full_updates)))
        self.filter_in = proj_b[:min(len(proj_b), self.nview + 2)]
        while len(self.filter_in) < self.nview + 2:
            self.filter_in = np.concatenate([self.filter_in, proj_b[:self.nview + 2 -
                                                                     len(self.filter_in)]])
        self.full_updates = full_updates

    def filter_once(self):
        t = time.perf_counter()
        cpu_filter_views(self.O, self.s, self.filter_in)
        return time.perf_counter() - t

    def describe(self, who, workers):
        return (f"per step: the filter of {self.nview} views ({who} filter restatement, "
                f"OpenMP) and the backprojection of {self.copies} x a central {self.n}^3 block "
                f"at the workload's voxel pitch ({self.updates} updates) by {workers}; "
                f"views / {self.s.P} = updates / {self.full_updates}, so the sample's rate is "
                f"the full chain's")


# ---------------------------------------------------------------------------------------------
def run_reference(args):
    """The reference's CPU path, timed on the host cores: KatsevichBkProj.cpp compiled
    unchanged (oracle/_ref; single-threaded code, one process per core, each on the same
    central block) for the backprojection, and the FP64 restatement of KatsevichFiltering.m
    (MATLAB is unavailable; OpenMP over views) for the filter. Each step is a bounded sample
    whose views and updates are the same fraction of the scan's (CpuChainSample), so the
    step's own rate is the chain's GUPS."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    O = _oracle()
    s = config(args.config)
    cores = os.cpu_count() or 1
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref (KatsevichBkProj.cpp built from the CTRecon sources) "
                          "is missing"}))
        return
    full_updates = _full_update_count(s)
    gsub_cache = {}

    def proj_views(a, b):
        locus = s.locus()
        locus[4], locus[5] = float(a + 1), float(b)
        g = O.bp_geom(locus, s.detector(), s.object())
        gsub_cache["g"] = g
        return O.project_ellipsoids(g, s.ellipsoids())

    smp = CpuChainSample(O, s, proj_views, full_updates, n=32, copies=cores)
    tmpdir = tempfile.mkdtemp()
    fpath = os.path.join(tmpdir, "fproj.npy")
    np.save(fpath, smp.fproj)
    import multiprocessing as mp
    per_step = []
    with mp.get_context("spawn").Pool(cores) as pool:
        pool.map(_ref_worker, [(smp.locus, smp.det, smp.obj, fpath)] * cores)  # load + page in
        for it in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            smp.filter_once()
            pool.map(_ref_worker, [(smp.locus, smp.det, smp.obj, fpath)] * cores)
            if it >= args.warmup:
                per_step.append(time.perf_counter() - t0)
    os.unlink(fpath)
    os.rmdir(tmpdir)
    t_step = statistics.mean(per_step)
    gups = smp.updates / t_step / 1e9
    sample = smp.describe("the FP64", f"KatsevichBkProj.cpp (oracle/_ref) in {cores} processes")
    line = {"impl": "reference", "metric": METRIC, "value": gups, "unit": "GUPS",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(s, ws),
            "cpu_baseline": {"value": gups, "unit": "GUPS", "cores": cores,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": gups, "unit": "GUPS", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "updates_per_step": smp.updates, "s_per_vol": full_updates / (gups * 1e9)}
    print(json.dumps(line))


def _full_update_count(s):
    """sum(LoopEnd-LoopBegin+1) of the whole volume; on the GPU when there is one."""
    try:
        import torch
        if torch.cuda.is_available():
            import ctrecon_b200 as ct
            c = ct.Context(torch.cuda.current_device())
            d_tab = torch.empty(c.pi_table_bytes(s.geom_struct()), dtype=torch.uint8,
                                device="cuda")
            d_cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
            c.pi_dev(s.geom_struct(), d_tab, d_cnt)
            torch.cuda.synchronize()
            n = int(d_cnt.item())
            c.close()
            del d_tab
            return n
    except Exception:
        pass
    O = _oracle()
    t = O.pi_table(O.bp_geom(s.locus(), s.detector(), s.object()))
    v = t["valid"]
    return int(np.sum(t["loop_end"][v] - t["loop_begin"][v] + 1))


def run_batched(args):
    """c4: 16 helical scans of uneven size. Times the one-at-a-time chain (filter, PI solve,
    backprojection per scan) and the batched form (one persistent backprojection launch over
    all scans, replayed as a CUDA graph); value = aggregate GUPS of the batched form."""
    import torch
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    from ctrecon_b200.geometry import batch_configs
    scans = batch_configs()
    hil = {"fp32": _lib.HILBERT_FP32, "bf16x3": _lib.HILBERT_BF16X3,
           "tf32": _lib.HILBERT_TF32}[args.hilbert]
    pis = {"bisect": _lib.PI_BISECT, "newton": _lib.PI_NEWTON, "learned": _lib.PI_LEARNED}[args.pi]
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        ctx = ct.Context(0, hilbert=hil, pi_solver=_lib.PI_BISECT)
        if pis == _lib.PI_LEARNED:
            import ctypes
            loss = ctypes.c_float()
            _lib.check(_lib.lib().ctrecon_pinet_train(ctx.handle, stream.cuda_stream, 1 << 22, 8192, 8,
                                                      0.21, 2024, ctypes.byref(loss)), ctx.handle)
        projs, fprojs, imgs = [], [], []
        for s in scans:
            d = torch.empty(s.proj_shape, dtype=torch.float32, device="cuda")
            ctx.phantom_dev(s.geom_struct(), s.ellipsoids(), d, photons=s.photons or 0.0, seed=s.seed)
            projs.append(d)
            fprojs.append(torch.empty_like(d))
            imgs.append(torch.zeros(s.vol_shape, dtype=torch.float32, device="cuda"))
        b = ct.Batch(ctx, scans)
        updates = b.updates()
        ctx.set_option(_lib.OPT_PI_SOLVER, pis)
        total = sum(updates)
        tune = None
        if args.bp_variant == -1:
            # the autotuner picks the batch's backprojector form (tile shape, view-block
            # depth, staging) on these scans, and each scan's own form for the one-at-a-time
            # runs (the table behind CTRECON_BP_AUTO), untimed
            tune = b.tune(projs, fprojs, imgs, stream=stream)
            single = []
            for s_, d, f, im in zip(scans, projs, fprojs, imgs):
                ctx.filter_dev(ct.scan_filter_params(s_), d, f)
                single.append(ctx.tune_bkproj(s_.geom_struct(), f, im)["best_variant"])
            ctx.set_option(_lib.OPT_BP_VARIANT, _lib.BP_AUTO)
            tune["single_scan_best"] = single
        else:
            b.set_variant(args.bp_variant if args.bp_variant < 100 else 2)
            ctx.set_option(_lib.OPT_BP_VARIANT, args.bp_variant)

        def one_at_a_time():
            for s, d, f, im in zip(scans, projs, fprojs, imgs):
                ctx.filter_dev(ct.scan_filter_params(s), d, f)
                ctx.bkproj_dev(s.geom_struct(), f, im)  # PI solved inside (context table)

        def timed(fn, k):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            stream.synchronize()
            e0.record(stream)
            for _ in range(k):
                fn()
            e1.record(stream)
            stream.synchronize()
            return e0.elapsed_time(e1) / k

        for _ in range(max(3, args.warmup)):
            one_at_a_time()
            b.run(projs, fprojs, imgs, use_graph=True)
        sampler = ClockSampler(0)
        sampler.start()
        ms_seq = timed(one_at_a_time, args.steps)
        ms_bat = timed(lambda: b.run(projs, fprojs, imgs, use_graph=True), args.steps)
        clocks = sampler.stop()
        b.close()
        ctx.close()
    line = {"metric": METRIC, "value": total / (ms_bat / 1e3) / 1e9, "unit": "GUPS",
            "n_gpus": 1, "steps": args.steps, "warmup": max(3, args.warmup),
            "ms_per_step": ms_bat, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "c4_batch_16_uneven_helical_scans", "scans": len(scans),
                       "volumes": [list(s.vol_shape) for s in scans],
                       "detectors": [[s.ZL, s.YL] for s in scans], "views": [s.P for s in scans],
                       "hilbert": args.hilbert, "pi_solver": args.pi, "graph": True,
                       "l2": "inputs larger than L2 (40 GB of projections and volumes)"},
            "updates_per_step": total,
            "one_at_a_time": {"ms_per_step": ms_seq, "gups": total / (ms_seq / 1e3) / 1e9},
            "batched_speedup": ms_seq / ms_bat, "bp_tune": tune, "clocks": clocks}
    print(json.dumps(line))


# ---------------------------------------------------------------------------------------------
def _pi_stats(ctx, torch, geom, d_tab):
    """PI solve with the context's solver: (update count, solver iterations)."""
    import ctypes
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    g = ct.bp_geom(geom)
    d_cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    d_its = torch.zeros(1, dtype=torch.int64, device="cuda")
    _lib.check(_lib.lib().ctrecon_pi_dev_stats(ctx.handle, torch.cuda.current_stream().cuda_stream,
                                               ctypes.byref(g), d_tab.data_ptr(),
                                               d_cnt.data_ptr(), d_its.data_ptr()), ctx.handle)
    torch.cuda.synchronize()
    return int(d_cnt.item()), int(d_its.item())


def _compare_pi_tables(torch, a, b, chunk=1 << 26):
    """Endpoint agreement of two PI tables on the device: max |dB|, |dT| (views) over voxels
    valid in both, voxels whose validity or loop range [Bindex, Tindex] differ."""
    ra, rb = a.view(torch.int32).view(-1, 4), b.view(torch.int32).view(-1, 4)
    fa, fb = a.view(torch.float32).view(-1, 4), b.view(torch.float32).view(-1, 4)
    dB = dT = 0.0
    bad_valid = bad_range = 0
    for i in range(0, ra.shape[0], chunk):
        sa, sb = ra[i:i + chunk], rb[i:i + chunk]
        va, vb = sa[:, 0] != 0x7FFFFFFF, sb[:, 0] != 0x7FFFFFFF
        bad_valid += int((va != vb).sum())
        v = va & vb
        if not bool(v.any()):
            continue
        Ba = sa[v, 0].double() + fa[i:i + chunk][v, 1].double()
        Bb = sb[v, 0].double() + fb[i:i + chunk][v, 1].double()
        Ta = sa[v, 2].double() + fa[i:i + chunk][v, 3].double()
        Tb = sb[v, 2].double() + fb[i:i + chunk][v, 3].double()
        dB = max(dB, float((Ba - Bb).abs().max()))
        dT = max(dT, float((Ta - Tb).abs().max()))
        bad_range += int(((sa[v, 0] != sb[v, 0]) | (sa[v, 2] != sb[v, 2])).sum())
    return {"max_abs_dB_views": dB, "max_abs_dT_views": dT, "voxels_validity_differs": bad_valid,
            "voxels_loop_range_differs": bad_range}


def run_report_extras(args):
    """The rows next to the path on the c2 scan: arc-to-flat panel rebin (HBM roofline),
    DerMode 0 and FilteringMode 1 filters against the chain-rule filter, file read/write."""
    import torch
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    from ctrecon_b200.formats import ProjectionData
    s = config(args.config)
    geom = s.geom_struct()
    fpar = ct.scan_filter_params(s)
    ctx = ct.Context(0)
    d_proj = torch.empty(s.proj_shape, dtype=torch.float32, device="cuda")
    ctx.phantom_dev(geom, s.ellipsoids(), d_proj, photons=s.photons or 0.0, seed=s.seed)
    d_out = torch.empty_like(d_proj)
    peak, peak_kind = load_peaks()
    stream = torch.cuda.current_stream()

    def timed(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    out = {"report": "extras", "workload": workload_name(s)}
    n = d_proj.numel()
    # panel rebin: arc detector of the same size (pitch = arc length 0.8 mm at D)
    c_idx = (s.YL - 1) / 2 + 0.25
    rb = {}
    for name, t in (("f32", d_proj), ("f64", d_proj.double())):
        o = torch.empty_like(t)
        ms = timed(lambda: ctx.rebin_to_panel_dev(t, c_idx, 0.8, s.StdDis, o))
        b = 2 * n * t.element_size()  # one read and one write of each sample
        rb[name] = {"ms": ms, "bytes": b, "achieved_gbs": b / ms / 1e6,
                    "frac_of_hbm": b / ms / 1e6 / peak}
        del o
    out["panel_rebin"] = dict(rb, peak_gbs=peak, peak_source=peak_kind,
                              model="one read + one write per sample")
    # filters
    flt = {}
    for name, hil in (("fp32", _lib.HILBERT_FP32), ("bf16x3", _lib.HILBERT_BF16X3)):
        ctx.set_option(_lib.OPT_HILBERT, hil)
        ctx.set_option(_lib.OPT_DERIVATIVE, _lib.DERIV_CHAIN)
        chain = timed(lambda: ctx.filter_dev(fpar, d_proj, d_out), 3)
        mode1 = timed(lambda: ctx.filter_mode1_dev(fpar, d_proj, d_out), 3)
        ctx.set_option(_lib.OPT_DERIVATIVE, _lib.DERIV_DIRECT)
        direct = timed(lambda: ctx.filter_dev(fpar, d_proj, d_out), 3)
        ctx.set_option(_lib.OPT_DERIVATIVE, _lib.DERIV_CHAIN)
        flt[name] = {"chain_rule_ms": chain, "dermode0_ms": direct, "filtering_mode1_ms": mode1}
    out["filter"] = flt
    # files (host): one c2 projection file, 3.5 GB of doubles
    h = ProjectionData(source_to_center=s.ScanR, source_to_detector=s.StdDis, det_reso_u=s.YL,
                       det_reso_v=s.ZL, det_pixel_u=0.8, det_pixel_v=0.8,
                       det_center_u=(s.YL - 1) / 2, det_center_v=(s.ZL - 1) / 2, is_arc=False,
                       total_views=s.P, views_per_turn=s.views_per_turn,
                       projection=d_proj.cpu().numpy().astype(np.float64))
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "c2.prj")
        t0 = time.perf_counter()
        h.write(path)
        tw = time.perf_counter() - t0
        t0 = time.perf_counter()
        q = ProjectionData.read(path)
        tr = time.perf_counter() - t0
        size = os.path.getsize(path)
        ok = bool(np.array_equal(q.projection, h.projection))
    out["projection_file"] = {"bytes": size, "write_gbs": size / tw / 1e9,
                              "read_gbs": size / tr / 1e9, "round_trip_equal": ok,
                              "note": "page-cache bound (tmpfs or disk of the host)"}
    print(json.dumps(out))
    ctx.close()


def _refgpu_guard(s, AL, n_vox):
    """(filter, backprojection) reasons the reference GPU MEX files cannot run scan s (None when
    they can), found by reading them. Filter: int32 element indices
    (KatsevichFiltering_GPU.cu:294 (pIdx*AL + AIndex)*YL, :71, :820); the complex buffer of a
    Hilbert batch, YL*nn2*ProjNumber elements computed in int (:637, batches of 1024 views, the
    last of up to 2047); at least one batch of 1024 views (:685: fewer make its batch loop run
    past the data). Backprojection: a 3-D texture of depth ProjNum (KatsevichBkProj_GPU.cu:262,
    at most 16384) and coordinate vectors sized ProjNum that receive RecMX/RecMY/RecMZ entries
    (KatsevichBkProj_GPU.cu:300-309)."""
    P = s.P
    lim = 2 ** 31 - 1
    nn2 = 2 * 2 ** (int(np.ceil(np.log2(s.YL))) + 1)
    last = P - (P // 1024 - 1) * 1024 if P >= 1024 else P
    f = None
    if P < 1024:
        f = "fewer than 1024 views: the reference's Hilbert batching needs one whole batch"
    elif P * AL * s.YL > lim or P * s.ZL * s.YL > lim:
        f = "element indices exceed int32 in the reference GPU filter"
    elif s.YL * nn2 * last > lim:
        f = (f"its Hilbert buffer of YL*nn2*views = {s.YL}*{nn2}*{last} elements overflows the "
             f"int it is sized with (KatsevichFiltering_GPU.cu:637)")
    b = None
    if P > 16384:
        b = "more than 16384 views: beyond a 3-D texture's depth"
    elif max(n_vox) > P:
        b = "a volume side larger than the view count overruns the reference's vectors"
    elif int(np.prod(n_vox)) > lim:
        b = "image indices exceed int32"
    return f, b


def run_report_refgpu(args):
    """The reference's own GPU MEX functions (KatsevichFiltering_GPU.cu, KatsevichBkProj_GPU.cu)
    recompiled for sm_100a against the mex.h shim (baseline/Makefile), beside this library's MEX
    modules on the same FP64 host arrays (synchronous calls, as MATLAB makes them): their time
    through the MEX interface, the device span of their work (CUDA events on the legacy stream
    they use), and their error against the FP64 oracle on a central block. The reference GPU
    filter runs where its int-sized buffers allow (c1; at c2 and above its Hilbert buffer size
    overflows), its backprojector on c1 and c2. Not a parity target: the reference GPU path has
    no endpoint weights, FP32 cuFFT and 9-bit texture interpolation weights."""
    import torch
    import ctrecon_b200 as ct
    from ctrecon_b200.mexharness import MexModule
    refdir = os.path.join(ROOT, "baseline", "_ref")
    fpath = os.path.join(refdir, "KatsevichFiltering_GPU_ref.so")
    bpath = os.path.join(refdir, "KatsevichBkProj_GPU_ref.so")
    if not (os.path.exists(fpath) and os.path.exists(bpath)):
        print(json.dumps({"report": "refgpu", "unavailable": "baseline/_ref (the reference GPU "
                          "MEX files built by baseline/Makefile) is missing"}))
        return
    O = _oracle()
    names = [args.config] if args.config not in ("c3",) else ["c1", "c2"]
    result = {"report": "refgpu",
              "arrays": "FP64 pageable host arrays through the MEX interface (mex.h shim)",
              "scans": {}}
    leg = torch.cuda.default_stream()  # the legacy stream the reference's thrust and kernels use

    def timed(fn, reps=2):
        fn()
        torch.cuda.synchronize()
        walls, devs = [], []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(leg)
            t0 = time.perf_counter()
            fn()
            e1.record(leg)
            torch.cuda.synchronize()
            walls.append(time.perf_counter() - t0)
            devs.append(e0.elapsed_time(e1) / 1e3)
        return {"wall_s": min(walls), "device_span_s": min(devs)}

    def err(x, r, m=None):
        x, r = (x[m], r[m]) if m is not None else (x, r)
        return {"rel_rmse": float(np.linalg.norm(x - r) / np.linalg.norm(r)),
                "max_abs": float(np.abs(x - r).max())}

    ref_f, ref_b = MexModule(fpath), MexModule(bpath)
    ours_f = MexModule(os.path.join(ROOT, "ctrecon_b200", "lib", "mex", "KatsevichFiltering_GPU.so"))
    ours_b = MexModule(os.path.join(ROOT, "ctrecon_b200", "lib", "mex", "KatsevichBkProj_GPU.so"))
    for m in (ref_f, ref_b, ours_f, ours_b):
        m.set_print(False)
    for name in names:
        s = config(name)
        AL = 2 * int(np.ceil(s.ZL * 1.3 * 0.5)) + 1
        why_f, why_b = _refgpu_guard(s, AL, s.vol_shape)
        out = {"workload": workload_name(s)}
        ctx = ct.Context(0)
        geom = s.geom_struct()
        d_proj = torch.empty(s.proj_shape, dtype=torch.float32, device="cuda")
        ctx.phantom_dev(geom, s.ellipsoids(), d_proj, photons=s.photons or 0.0, seed=s.seed)
        d_tab = torch.empty(ctx.pi_table_bytes(geom), dtype=torch.uint8, device="cuda")
        d_cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
        ctx.pi_dev(geom, d_tab, d_cnt)
        torch.cuda.synchronize()
        updates = int(d_cnt.item())
        out["updates"] = updates
        proj64 = d_proj.cpu().numpy().astype(np.float64)   # pageable, as MATLAB's arrays
        del d_proj, d_tab
        ctx.close()
        torch.cuda.empty_cache()
        fargs = list(s.filter_args())
        f_ours = np.empty_like(proj64)
        out["filter_ours_mex"] = timed(lambda: ours_f.call([proj64] + fargs + [f_ours]))
        if why_f is None:
            f_ref = np.empty_like(proj64)
            out["filter_reference_gpu"] = timed(lambda: ref_f.call([proj64] + fargs + [f_ref]))
        else:
            out["filter_reference_gpu"] = {"unavailable": why_f}
        img_ours = np.zeros(s.vol_shape)
        out["bkproj_ours_mex"] = timed(lambda: ours_b.call([geom, f_ours, img_ours]))
        if why_b is None:
            img_ref = np.zeros(s.vol_shape)
            out["bkproj_reference_gpu"] = timed(lambda: ref_b.call([geom, f_ours, img_ref]))
        else:
            out["bkproj_reference_gpu"] = {"unavailable": why_b}
        # accuracy on the central block: the reference GPU filter's views and its
        # backprojection (of the oracle's filtered views) against the FP64 oracle
        n = 48
        locus, det, obj, lo, hi = block_problem(O, s, n)
        a0, a1 = max(0, lo - 1), min(s.P, hi + 1)
        orc_f = np.ascontiguousarray(cpu_filter_views(O, s, proj64[a0:a1])[lo - a0:hi - a0])
        gb = O.bp_geom(locus, det, obj, honour_extras=True)
        orc_img, _, touched = O.bkproj(gb, orc_f, np.zeros((n, n, n)), want_touched=True)
        t = touched.astype(bool)
        block = {"Locus": np.array(locus), "Detector": np.array(det), "Object": np.array(obj)}
        acc = {"block": {"voxels": n ** 3, "written": int(t.sum()), "views": [lo, hi]},
               "filter_ours": err(f_ours[lo:hi], orc_f)}
        bimg_ours = np.zeros((n, n, n))
        ours_b.call([block, orc_f, bimg_ours])
        acc["bkproj_ours"] = err(bimg_ours, orc_img, t)
        if why_f is None:
            acc["filter_reference_gpu"] = err(f_ref[lo:hi], orc_f)
        if why_b is None:
            bimg_ref = np.zeros((n, n, n))
            ref_b.call([block, orc_f, bimg_ref])
            acc["bkproj_reference_gpu"] = err(bimg_ref, orc_img, t)
        out["accuracy_vs_fp64_oracle"] = acc
        sp = {}
        if why_f is None:
            sp["filter"] = out["filter_reference_gpu"]["wall_s"] / out["filter_ours_mex"]["wall_s"]
        if why_b is None:
            sp["bkproj"] = out["bkproj_reference_gpu"]["wall_s"] / out["bkproj_ours_mex"]["wall_s"]
        if why_f is None and why_b is None:
            rt = out["filter_reference_gpu"]["wall_s"] + out["bkproj_reference_gpu"]["wall_s"]
            ot = out["filter_ours_mex"]["wall_s"] + out["bkproj_ours_mex"]["wall_s"]
            sp["chain"] = rt / ot
            out["gups_mex"] = {"reference_gpu": updates / rt / 1e9, "ours": updates / ot / 1e9}
        out["speedup_mex"] = sp
        result["scans"][name] = out
        del proj64, f_ours, img_ours
    print(json.dumps(result))


def _train_pinet(ctx, s, out, stream, torch):
    """Trains the learned PI-line initialiser on the GPU (2^22 FP64 Newton pairs, 8 epochs)."""
    import ctypes
    from ctrecon_b200 import _lib
    loss = ctypes.c_float()
    t0 = time.perf_counter()
    _lib.check(_lib.lib().ctrecon_pinet_train(
        ctx.handle, stream.cuda_stream, 1 << 22, 8192, 8, s.ObjR / s.ScanR * 1.05, 2024,
        ctypes.byref(loss)), ctx.handle)
    torch.cuda.synchronize()
    out["pinet"] = {"train_pairs": 1 << 22, "epochs": 8, "train_s": time.perf_counter() - t0,
                    "final_loss": loss.value}


def run_report(args):
    """Reports of the c3 and c5 configurations (not the headline line)."""
    if args.report == "extras":
        run_report_extras(args)
        return
    if args.report == "refgpu":
        run_report_refgpu(args)
        return
    import torch
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib
    s = config(args.config if args.config != "c2" else args.report)  # c3 / c5 by default
    geom = s.geom_struct()
    fpar = ct.scan_filter_params(s)
    ctx = ct.Context(0)
    d_proj = torch.empty(s.proj_shape, dtype=torch.float32, device="cuda")
    ctx.phantom_dev(geom, s.ellipsoids(), d_proj, photons=s.photons or 0.0, seed=s.seed)
    d_fproj = torch.empty_like(d_proj)
    d_img = torch.zeros(s.vol_shape, dtype=torch.float32, device="cuda")
    d_tab = torch.empty(ctx.pi_table_bytes(geom), dtype=torch.uint8, device="cuda")
    ctx.set_option(_lib.OPT_PI_SOLVER, _lib.PI_BISECT)
    updates, iters_bisect = _pi_stats(ctx, torch, geom, d_tab)
    stream = torch.cuda.current_stream()

    def chain_ms(steps=2):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ctx.filter_dev(fpar, d_proj, d_fproj)
        ctx.pi_dev(geom, d_tab)
        ctx.bkproj_dev(geom, d_fproj, d_img, d_pitab=d_tab)
        ph = [0.0, 0.0, 0.0]
        for _ in range(steps):
            e[0].record(stream)
            ctx.filter_dev(fpar, d_proj, d_fproj)
            e[1].record(stream)
            ctx.pi_dev(geom, d_tab)
            e[2].record(stream)
            ctx.bkproj_dev(geom, d_fproj, d_img, d_pitab=d_tab)
            e[3].record(stream)
            torch.cuda.synchronize()
            for k in range(3):
                ph[k] += e[k].elapsed_time(e[k + 1]) / steps
        return {"filter": ph[0], "pi": ph[1], "bkproj": ph[2], "step": sum(ph)}

    out = {"report": args.report, "workload": workload_name(s), "volume": list(s.vol_shape),
           "detector": [s.ZL, s.YL], "views": s.P, "updates_per_step": updates}
    if args.bp_variant == -1:
        ctx.filter_dev(fpar, d_proj, d_fproj)
        out["bp_tune"] = ctx.tune_bkproj(geom, d_fproj, d_img, d_pitab=d_tab)
        ctx.set_option(_lib.OPT_BP_VARIANT, _lib.BP_AUTO)
    else:
        ctx.set_option(_lib.OPT_BP_VARIANT, args.bp_variant)

    if args.report == "c3":
        O = _oracle()
        cores = os.cpu_count() or 1
        m = s.P // 2
        proj_v = d_proj[m - 1:m + 17].cpu().numpy().astype(np.float64)
        ref_views = cpu_filter_views(O, s, proj_v)[1:-1]          # views m .. m+15
        n = 48
        locus, det, obj, lo, hi = block_problem(O, s, n)
        proj_b = d_proj[lo - 1:hi + 1].cpu().numpy().astype(np.float64)
        t0 = time.perf_counter()
        ref_fb = np.ascontiguousarray(cpu_filter_views(O, s, proj_b)[1:-1])
        gb = O.bp_geom(locus, det, obj, honour_extras=True)
        ref_img, _, touched = O.bkproj(gb, ref_fb, np.zeros((n, n, n)), nthreads=cores,
                                       want_touched=True)
        t_oracle = time.perf_counter() - t0
        touched = touched.astype(bool)
        block = {"Locus": locus, "Detector": det, "Object": obj}
        modes = {}
        for name, mode in (("fp32", _lib.HILBERT_FP32), ("bf16x3", _lib.HILBERT_BF16X3),
                           ("tf32", _lib.HILBERT_TF32)):
            ctx.set_option(_lib.OPT_HILBERT, mode)
            ctx.set_option(_lib.OPT_PI_SOLVER, _lib.PI_NEWTON)
            ph = chain_ms()
            got_v = d_fproj[m:m + 16].cpu().numpy().astype(np.float64)
            d_blk = torch.zeros((n, n, n), dtype=torch.float32, device="cuda")
            ctx.set_option(_lib.OPT_PI_SOLVER, _lib.PI_BISECT)
            ctx.bkproj_dev(block, d_fproj[lo:hi].contiguous(), d_blk)
            torch.cuda.synchronize()
            got_b = d_blk.cpu().numpy().astype(np.float64)
            dv, db = got_v - ref_views, (got_b - ref_img)[touched]
            modes[name] = {
                "filter_rel_rmse": float(np.linalg.norm(dv) / np.linalg.norm(ref_views)),
                "filter_max_abs": float(np.abs(dv).max()),
                "filter_ref_max_abs": float(np.abs(ref_views).max()),
                "chain_block_rel_rmse": float(np.linalg.norm(db) /
                                              np.linalg.norm(ref_img[touched])),
                "chain_block_max_abs": float(np.abs(db).max()),
                "chain_block_ref_max_abs": float(np.abs(ref_img[touched]).max()),
                "phase_ms": ph, "gups": updates / (ph["step"] / 1e3) / 1e9,
                "s_per_vol": ph["step"] / 1e3}
        out.update({"modes": modes, "filter_views_compared": [m, m + 16],
                    "chain_block": {"voxels": n ** 3, "written": int(touched.sum()),
                                    "views": [lo, hi], "oracle_s": t_oracle,
                                    "pi_solver": "bisection (the reference's) for the block"},
                    "pi_solver_in_timing": "newton"})
    else:  # c5: the learned PI-line initialiser at scale
        _train_pinet(ctx, s, out, stream, torch)
        d_tab_b = d_tab.clone()  # the bisection table (the arbiter)
        res = {}
        for name, solver, nmode in (("bisect", _lib.PI_BISECT, None),
                                    ("newton", _lib.PI_NEWTON, None),
                                    ("learned_voxel_fp32", _lib.PI_LEARNED, _lib.PINET_VOXEL_FP32),
                                    ("learned_voxel_bf16", _lib.PI_LEARNED, _lib.PINET_VOXEL_BF16),
                                    ("learned", _lib.PI_LEARNED, _lib.PINET_GRID)):
            ctx.set_option(_lib.OPT_PI_SOLVER, solver)
            if nmode is not None:
                ctx.set_option(_lib.OPT_PINET_MODE, nmode)
            cnt, its = _pi_stats(ctx, torch, geom, d_tab)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            ev[0].record(stream)
            ctx.pi_dev(geom, d_tab)
            ev[1].record(stream)
            torch.cuda.synchronize()
            r = {"updates": cnt, "iterations": its, "pi_ms": ev[0].elapsed_time(ev[1])}
            if name != "bisect" and not name.startswith("learned_voxel"):
                r["vs_bisection"] = _compare_pi_tables(torch, d_tab, d_tab_b)
            if name == "newton":
                d_tab_n = d_tab.clone()
            if name == "learned":  # converged endpoints of the two Newton starts
                r["vs_newton"] = _compare_pi_tables(torch, d_tab, d_tab_n)
                del d_tab_n
            res[name] = r
        out["pi"] = res
        out["newton_iterations_saved_per_voxel"] = (
            (res["newton"]["iterations"] - res["learned"]["iterations"]) /
            max(1, int((d_tab_b.view(torch.int32).view(-1, 4)[:, 0] != 0x7FFFFFFF).sum())))
        del d_tab_b
    # the forms of the headline comparison on this workload: plain (FP32 Hilbert, bisection)
    # against the mixed forms, device-resident chain, CUDA events
    if "pinet" not in out:
        _train_pinet(ctx, s, out, stream, torch)
    forms = {"plain_fp32_bisect": (_lib.HILBERT_FP32, _lib.PI_BISECT),
             "fp32_newton": (_lib.HILBERT_FP32, _lib.PI_NEWTON),
             "fp32_learned": (_lib.HILBERT_FP32, _lib.PI_LEARNED),
             "bf16x3_newton": (_lib.HILBERT_BF16X3, _lib.PI_NEWTON),
             "bf16x3_learned": (_lib.HILBERT_BF16X3, _lib.PI_LEARNED)}
    out["chain_ms"] = {}
    for name, (hil, pis) in forms.items():
        ctx.set_option(_lib.OPT_HILBERT, hil)
        ctx.set_option(_lib.OPT_PI_SOLVER, pis)
        ph = chain_ms(1 if args.report == "c5" else 2)
        ph["gups"] = updates / (ph["step"] / 1e3) / 1e9
        out["chain_ms"][name] = ph
    if args.report == "c3":
        # mixed + learned + batched: two copies of the scan through the batch API (filters, PI
        # solves, one persistent backprojection launch over both volumes), replayed as a graph
        ctx.set_option(_lib.OPT_HILBERT, _lib.HILBERT_BF16X3)
        ctx.set_option(_lib.OPT_PI_SOLVER, _lib.PI_LEARNED)
        del d_tab
        b = ct.Batch(ctx, [s, s])
        bform = out.get("bp_tune", {}).get("best_variant", args.bp_variant)
        b.set_variant(bform if 0 <= bform < 100 else 10)
        d_fproj2, d_img2 = torch.empty_like(d_proj), torch.zeros_like(d_img)
        bargs = ([d_proj, d_proj], [d_fproj, d_fproj2], [d_img, d_img2])
        sb = torch.cuda.Stream()
        with torch.cuda.stream(sb):
            for _ in range(3):
                b.run(*bargs, stream=sb, use_graph=True)
            sb.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(sb)
            for _ in range(2):
                b.run(*bargs, stream=sb, use_graph=True)
            e1.record(sb)
            sb.synchronize()
        ms = e0.elapsed_time(e1) / 2
        out["chain_ms"]["bf16x3_learned_batched_x2"] = {
            "step": ms, "scans": 2, "bp_variant": b.variants()[0],
            "gups": 2 * updates / (ms / 1e3) / 1e9}
        b.close()
    plain = out["chain_ms"]["plain_fp32_bisect"]["gups"]
    out["vs_plain"] = {k: v["gups"] / plain for k, v in out["chain_ms"].items()}
    print(json.dumps(out))
    ctx.close()


# ---------------------------------------------------------------------------------------------
FP32_LANES_PER_SM = 128  # FP32 FMA per SM and clock (sm_100)
SMS = 148


def kernel_rooflines(s, kt, steps, updates, peaks, sm_mhz, hil):
    """Per-kernel time and roofline fraction from the CUDA-event kernel times `kt` ({kind:
    (ms, launches)}) of `steps` steps. Algorithmic work per view / per update:
      K1 deriv_rebin   HBM: 4*YL*ZL bytes read + 4*AL*YLp written (FP32, or BF16 hi + lo)
      K2 hilbert_tc    tensor: 2*YL^2*AL flop per view (the dense Toeplitz product); the kernel
                       executes two half-size products per view group (odd lags only, padded
                       rows and kappa rows), three of them for BF16x3: `executed`
      K2 hilbert_simt  FP32 FMA pipe: AL*YL*YL/2 FMA per view (odd lags only) at
                       128 FMA/SM/clock
      cell_records     HBM: 4 bytes read + 16 written per detector cell and view
      backproject      issue: warp instructions per update (ncu, profiles/inst_per_update.txt)
                       over 148 SMs x 4 schedulers x the SM clock."""
    YL, ZL, P = s.YL, s.ZL, s.P
    AL = 2 * int(np.ceil(ZL * 1.3 * 0.5)) + 1
    YLp = (YL + 127) // 128 * 128
    clk = (sm_mhz or 1965.0) * 1e6
    out = {}
    for kind, (ms, n) in kt.items():
        if n == 0:
            continue
        t = ms / 1e3 / steps  # seconds per step
        r = {"ms_per_step": ms / steps, "launches_per_step": n / steps}
        if kind == "deriv_rebin":
            b = P * (4 * YL * ZL + 4 * AL * YLp)
            r.update(bound="hbm", achieved_gbs=b / t / 1e9, peak_gbs=peaks["hbm_gbs"],
                     frac=b / t / 1e9 / peaks["hbm_gbs"], algorithmic_bytes=b,
                     peak_source=peaks["source"])
        elif kind == "hilbert_tc":
            f = 2.0 * YL * YL * AL * P
            # the parity-split form: two products of (YLp/2 rows padded to 128) x YLp/2 per
            # parity on each view group's kappa rows padded to 16
            vpt = max(1, 256 // AL)
            ntile = (vpt * AL + 15) // 16 * 16
            YLh = YLp // 2
            YLhA = (YLh + 127) // 128 * 128
            ex = ((3 if hil == "bf16x3" else 1) * 2.0 * (2 * YLhA) * YLh * ntile *
                  np.ceil(P / vpt))
            if AL > 256:  # the single-pass form: one full product per view
                ex = (3 if hil == "bf16x3" else 1) * 2.0 * YLp * YLp * AL * P
            pk = peaks["bf16_tflops"] * (1 if hil == "bf16x3" else 0.5)
            r.update(bound="tensor", achieved_tflops=f / t / 1e12, peak_tflops=pk,
                     frac=f / t / 1e12 / pk, executed_tflops=ex / t / 1e12,
                     executed_frac=ex / t / 1e12 / pk, algorithmic_flop=f,
                     peak_note=(f"BF16 burst of {peaks['source']}" if hil == "bf16x3" else
                                f"half the BF16 burst of {peaks['source']} (TF32 rate)"))
        elif kind == "hilbert_simt":
            fma = AL * YL * (YL / 2.0) * P
            pk = SMS * FP32_LANES_PER_SM * clk
            r.update(bound="fp32_fma", achieved_tflops=2 * fma / t / 1e12,
                     peak_tflops=2 * pk / 1e12, frac=fma / t / pk, algorithmic_fma=fma)
        elif kind == "cell_records":
            b = P * (YL - 1) * (ZL - 1) * 20
            r.update(bound="hbm", achieved_gbs=b / t / 1e9, peak_gbs=peaks["hbm_gbs"],
                     frac=b / t / 1e9 / peaks["hbm_gbs"], algorithmic_bytes=b,
                     peak_source=peaks["source"])
        elif kind == "backproject":
            r.update(gups=updates / t / 1e9,
                     gather_equivalent_gbs=BYTES_PER_UPDATE * updates / t / 1e9)
        elif kind == "pi_solve":
            r.update(voxels_per_s=float(np.prod(s.vol_shape)) / t)
        out[kind] = r
    return out


def run_headline(args):
    import torch
    import ctrecon_b200 as ct
    from ctrecon_b200 import _lib

    ws, rank, local = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    s = config(args.config)
    hil_of = {"fp32": _lib.HILBERT_FP32, "bf16x3": _lib.HILBERT_BF16X3,
              "tf32": _lib.HILBERT_TF32}
    pi_of = {"bisect": _lib.PI_BISECT, "newton": _lib.PI_NEWTON, "learned": _lib.PI_LEARNED}
    ctx = ct.Context(local)
    if args.bp_window:
        ctx.set_option(_lib.OPT_BP_WINDOW, args.bp_window)
    ctx.set_option(_lib.OPT_PINET_MODE, {"voxel-fp32": _lib.PINET_VOXEL_FP32,
                                         "voxel-bf16": _lib.PINET_VOXEL_BF16,
                                         "grid": _lib.PINET_GRID}[args.pinet_mode])
    geom = s.geom_struct()
    fpar = ct.scan_filter_params(s)
    stream = torch.cuda.current_stream()
    peaks = load_peaks()

    # ---- inputs, resident in HBM before timing --------------------------------------------------
    d_proj = torch.empty(s.proj_shape, dtype=torch.float32, device=dev)
    ctx.phantom_dev(geom, s.ellipsoids(), d_proj, photons=s.photons or 0.0, seed=s.seed + rank)
    d_fproj = torch.empty_like(d_proj)
    d_img = torch.zeros(s.vol_shape, dtype=torch.float32, device=dev)
    d_tab = torch.empty(ctx.pi_table_bytes(geom), dtype=torch.uint8, device=dev)
    d_cnt = torch.zeros(1, dtype=torch.int64, device=dev)
    # exact update count: the reference's loop count from the bisection PI solve
    ctx.set_option(_lib.OPT_PI_SOLVER, _lib.PI_BISECT)
    ctx.pi_dev(geom, d_tab, d_cnt)
    torch.cuda.synchronize()
    updates = int(d_cnt.item())

    pinet_info = None

    def train_pinet():
        nonlocal pinet_info
        if pinet_info is not None:
            return
        import ctypes
        loss = ctypes.c_float()
        t0 = time.perf_counter()
        _lib.check(_lib.lib().ctrecon_pinet_train(
            ctx.handle, stream.cuda_stream, 1 << 22, 8192, 8, s.ObjR / s.ScanR * 1.05, 2024,
            ctypes.byref(loss)), ctx.handle)
        torch.cuda.synchronize()
        pinet_info = {"train_pairs": 1 << 22, "epochs": 8,
                      "train_s": time.perf_counter() - t0, "final_loss": loss.value}

    # ---- the backprojector form: the autotuner's choice on this workload (untimed) ------------
    tune = None
    if args.bp_variant == -1:
        ctx.set_option(_lib.OPT_HILBERT, _lib.HILBERT_FP32)
        ctx.filter_dev(fpar, d_proj, d_fproj)
        tune = ctx.tune_bkproj(geom, d_fproj, d_img, d_pitab=d_tab)
        ctx.set_option(_lib.OPT_BP_VARIANT, _lib.BP_AUTO)
        bp_form = tune["best_variant"]
    else:
        ctx.set_option(_lib.OPT_BP_VARIANT, args.bp_variant)
        bp_form = args.bp_variant

    ev = {k: [] for k in ("f0", "f1", "p1", "b1")}

    def step(record):
        if record:
            e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            e[0].record(stream)
        ctx.filter_dev(fpar, d_proj, d_fproj)
        if record:
            e[1].record(stream)
        ctx.pi_dev(geom, d_tab)
        if record:
            e[2].record(stream)
        ctx.bkproj_dev(geom, d_fproj, d_img, d_pitab=d_tab)
        if record:
            e[3].record(stream)
            for k, x in zip(("f0", "f1", "p1", "b1"), e):
                ev[k].append(x)

    def time_form(hil, pis):
        """K device-resident steps of one form; CUDA events on the launching stream, the
        slowest rank's time, per-phase means and per-kernel times."""
        ctx.set_option(_lib.OPT_HILBERT, hil_of[hil])
        ctx.set_option(_lib.OPT_PI_SOLVER, pi_of[pis])
        if pis == "learned":
            train_pinet()
        for k in ev:
            ev[k].clear()
        ctx.set_option(_lib.OPT_KERNEL_TIMING, 0)
        for _ in range(max(3, args.warmup)):
            step(False)
        torch.cuda.synchronize()
        barrier(ws)
        ctx.kernel_times()  # drop anything recorded before
        ctx.set_option(_lib.OPT_KERNEL_TIMING, 1)
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(args.steps):
            step(True)
        t1.record(stream)
        torch.cuda.synchronize()
        barrier(ws)
        ctx.set_option(_lib.OPT_KERNEL_TIMING, 0)
        kt = ctx.kernel_times()
        ms = max_over_ranks(t0.elapsed_time(t1) / args.steps, ws)
        ph = {"filter": statistics.mean(a.elapsed_time(b) for a, b in zip(ev["f0"], ev["f1"])),
              "pi": statistics.mean(a.elapsed_time(b) for a, b in zip(ev["f1"], ev["p1"])),
              "bkproj": statistics.mean(a.elapsed_time(b) for a, b in zip(ev["p1"], ev["b1"]))}
        return {"value": replica_gups(updates, ms, ws), "unit": "GUPS", "ms_per_step": ms,
                "s_per_vol": ms / 1e3, "hilbert": hil, "pi_solver": pis, "bp_variant": bp_form,
                "phase_ms": ph, "kernel_times": kt}

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    plain = time_form(args.hilbert, args.pi)
    plain_form = (args.hilbert, args.pi) == ("fp32", "bisect")
    forms = {}
    batched_equal = None
    if plain_form and not args.no_mixed:
        forms["mixed_learned"] = time_form("bf16x3", "learned")
        forms["mixed_learned"]["vs_plain"] = plain["ms_per_step"] / forms["mixed_learned"]["ms_per_step"]
        mixed_img = d_img.clone()
        if not args.no_batched:
            # two copies of the scan through the batch API: both filters and PI solves, then ONE
            # persistent backprojection launch over the tiles of both volumes; captured into a
            # CUDA graph on the second run and replayed
            b = ct.Batch(ctx, [s, s])
            b.set_variant(bp_form if 0 <= bp_form < 100 else 12)
            d_fproj2, d_img2 = torch.empty_like(d_proj), torch.zeros_like(d_img)
            bargs = ([d_proj, d_proj], [d_fproj, d_fproj2], [d_img, d_img2])
            sb = torch.cuda.Stream()
            with torch.cuda.stream(sb):
                for _ in range(max(3, args.warmup)):
                    b.run(*bargs, stream=sb, use_graph=True)
                sb.synchronize()
                barrier(ws)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(sb)
                for _ in range(args.steps):
                    b.run(*bargs, stream=sb, use_graph=True)
                e1.record(sb)
                sb.synchronize()
                barrier(ws)
            ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, ws)
            # the batch's volumes against the single-scan mixed + learned volume (same options)
            batched_equal = bool(torch.equal(d_img, mixed_img) and torch.equal(d_img2, mixed_img))
            forms["mixed_learned_batched"] = {
                "value": replica_gups(2 * updates, ms, ws), "unit": "GUPS", "ms_per_step": ms,
                "scans_per_step": 2, "s_per_vol": ms / 2e3, "hilbert": "bf16x3",
                "pi_solver": "learned", "bp_variant": b.variants()[0], "graph": True,
                "vs_plain": plain["ms_per_step"] / (ms / 2),
                "volumes_equal_single_scan_form": batched_equal}
            b.close()
            del d_fproj2, d_img2
        del mixed_img
    clocks = sampler.stop()
    value = plain["value"]
    ms_step = plain["ms_per_step"]

    # ---- accuracy: every form's whole chain against the FP64 oracle on a central block --------
    accuracy = None
    if rank == 0 and not args.no_accuracy:
        O = _oracle()
        n = 48
        locus, det, obj, lo, hi = block_problem(O, s, n)
        a0, a1 = max(0, lo - 1), min(s.P, hi + 1)
        t0 = time.perf_counter()
        ref_f = np.ascontiguousarray(cpu_filter_views(
            O, s, d_proj[a0:a1].cpu().numpy().astype(np.float64))[lo - a0:hi - a0])
        gb = O.bp_geom(locus, det, obj, honour_extras=True)
        sentinel = -5.5
        ref_img, _, touched = O.bkproj(gb, ref_f, np.full((n, n, n), sentinel),
                                       want_touched=True)
        t_oracle = time.perf_counter() - t0
        t = touched.astype(bool)
        block = {"Locus": locus, "Detector": det, "Object": obj}
        accuracy = {"block": {"voxels": n ** 3, "written": int(t.sum()), "views": [lo, hi],
                              "oracle_s": t_oracle,
                              "oracle": "FP64 filter restatement + orc_bkproj (= "
                                        "KatsevichBkProj.cpp bit for bit)"}}
        for name, (hil, pis) in (("plain", (args.hilbert, args.pi)),
                                 ("mixed_learned", ("bf16x3", "learned"))):
            if name != "plain" and name not in forms:
                continue
            ctx.set_option(_lib.OPT_HILBERT, hil_of[hil])
            ctx.set_option(_lib.OPT_PI_SOLVER, pi_of[pis])
            ctx.filter_dev(fpar, d_proj, d_fproj)
            d_blk = torch.full((n, n, n), sentinel, dtype=torch.float32, device=dev)
            ctx.bkproj_dev(block, d_fproj[lo:hi].contiguous(), d_blk)
            torch.cuda.synchronize()
            got = d_blk.cpu().numpy().astype(np.float64)
            d = (got - ref_img)[t]
            accuracy[name] = {
                "rel_rmse": float(np.linalg.norm(d) / np.linalg.norm(ref_img[t])),
                "max_abs": float(np.abs(d).max()),
                "ref_max_abs": float(np.abs(ref_img[t]).max()),
                "untouched_kept": bool(np.array_equal(got[~t], ref_img[~t]))}
        if "mixed_learned_batched" in forms:
            accuracy["mixed_learned_batched"] = dict(
                accuracy["mixed_learned"],
                note="its volumes are bit-identical to the single-scan mixed_learned form's "
                     "(checked in this run)" if batched_equal else
                     "its volumes DIFFER from the single-scan form's")
    ctx.set_option(_lib.OPT_HILBERT, hil_of[args.hilbert])
    ctx.set_option(_lib.OPT_PI_SOLVER, pi_of[args.pi])

    # ---- e2e through the MEX-equivalent host calls (FP64 pinned host buffers) -----------------
    e2e = e2e_mex = e2e_pageable = None
    nproj, nvox = int(np.prod(s.proj_shape)), int(np.prod(s.vol_shape))
    if not args.no_e2e:
        h_proj = torch.empty(s.proj_shape, dtype=torch.float64, pin_memory=True)
        h_proj.copy_(d_proj.cpu().to(torch.float64))
        h_fproj = torch.empty_like(h_proj).pin_memory()
        h_img = torch.zeros(s.vol_shape, dtype=torch.float64).pin_memory()
        np_proj, np_fproj, np_img = h_proj.numpy(), h_fproj.numpy(), h_img.numpy()
        e2e_steps = max(1, min(args.steps, 3))
        # the whole chain in one call: FP64 projections up (pipelined with the filter), FProj
        # kept on the device, the FP64 image up (untouched voxels keep their values) and down
        ctx.recon_host(fpar, geom, np_proj, np_img)
        barrier(ws)
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            ctx.recon_host(fpar, geom, np_proj, np_img)
        t_e2e = max_over_ranks((time.perf_counter() - t0) / e2e_steps, ws)
        # the FP64 projections cross to the device as FP32 when host threads convert them
        # (CTRECON_OPT_HOST_THREADS, default: the host's threads, at most 16)
        host_threads = ctx.get_option(_lib.OPT_HOST_THREADS)
        if host_threads < 0:
            host_threads = min(16, os.cpu_count() or 4)
        proj_bytes = (4 if host_threads > 0 else 8) * nproj
        e2e = {"value": ws * updates / t_e2e / 1e9, "unit": "GUPS",
               "h2d_bytes_per_step": proj_bytes + 8 * nvox, "d2h_bytes_per_step": 8 * nvox,
               "s_per_vol": t_e2e, "steps": e2e_steps, "host_threads": host_threads,
               "path": "ctrecon_recon_host_f64 (filter + backprojection in one call, "
                       "FunctionKat_v6.m:85-113 without the FProj round trip), pinned FP64 host "
                       "buffers, the projections converted to FP32 by host threads slot by slot "
                       "as they go up (FP64 copies converted on the device when host_threads "
                       "is 0)"}
        # the two MEX-equivalent calls, FProj through the host in between
        ctx.filter_host(fpar, np_proj, np_fproj)
        ctx.bkproj_host(geom, np_fproj, np_img)
        barrier(ws)
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            ctx.filter_host(fpar, np_proj, np_fproj)       # KatsevichFiltering_GPU
            ctx.bkproj_host(geom, np_fproj, np_img)        # KatsevichBkProj_GPU
        t_mex = max_over_ranks((time.perf_counter() - t0) / e2e_steps, ws)
        # inputs cross as FP32 when host threads convert them; the pinned FProj comes down
        # in FP64
        in_b = 4 if host_threads > 0 else 8
        e2e_mex = {"value": ws * updates / t_mex / 1e9, "unit": "GUPS",
                   "h2d_bytes_per_step": 2 * in_b * nproj + 8 * nvox,
                   "d2h_bytes_per_step": 8 * (nproj + nvox), "s_per_vol": t_mex,
                   "steps": e2e_steps,
                   "path": "ctrecon_filter_host_f64 + ctrecon_bkproj_host_f64 (the two MEX "
                           "calls' C ABI), pinned FP64 host buffers"}
        del h_fproj, h_img
        # the MEX modules themselves, with pageable FP64 arrays as MATLAB passes them
        # (FunctionKat_v6.m:85-113: FProj = Proj then KatsevichFiltering_GPU writes in place)
        from ctrecon_b200.mexharness import MexModule
        os.environ["CTRECON_DEVICE"] = str(local)  # the MEX modules' own contexts
        libdir = os.path.join(ROOT, "ctrecon_b200", "lib", "mex")
        mf = MexModule(os.path.join(libdir, "KatsevichFiltering_GPU.so"))
        mb = MexModule(os.path.join(libdir, "KatsevichBkProj_GPU.so"))
        p_proj = np.array(np_proj)          # pageable copies
        del h_proj, np_proj
        p_fproj = np.empty_like(p_proj)
        p_img = np.zeros(s.vol_shape)
        fargs = list(s.filter_args())

        def mex_step():
            mf.call([p_proj] + fargs + [p_fproj])
            mb.call([geom, p_fproj, p_img])

        mex_step()
        pg_steps = max(1, min(args.steps, 2))
        barrier(ws)
        t0 = time.perf_counter()
        for _ in range(pg_steps):
            mex_step()
        t_pg = max_over_ranks((time.perf_counter() - t0) / pg_steps, ws)
        # the pageable FProj comes down in FP32 and is widened by host threads
        e2e_pageable = {"value": ws * updates / t_pg / 1e9, "unit": "GUPS",
                        "h2d_bytes_per_step": 2 * in_b * nproj + 8 * nvox,
                        "d2h_bytes_per_step": in_b * nproj + 8 * nvox, "s_per_vol": t_pg,
                        "steps": pg_steps,
                        "path": "KatsevichFiltering_GPU + KatsevichBkProj_GPU MEX modules "
                                "(mex.h shim), pageable FP64 arrays"}
        del p_proj, p_fproj, p_img

    # ---- rooflines --------------------------------------------------------------------------------
    kern = kernel_rooflines(s, plain["kernel_times"], args.steps, updates, peaks,
                            clocks.get("sm_mhz"), args.hilbert)
    if "mixed_learned" in forms:
        forms["mixed_learned"]["kernels"] = kernel_rooflines(
            s, forms["mixed_learned"]["kernel_times"], args.steps, updates, peaks,
            clocks.get("sm_mhz"), "bf16x3")
    bp_kernel = ("k_bkproj" if bp_form >= 100 else "k_bkproj3" if bp_form in (0, 1)
                 else "k_bkproj2" if bp_form in (2, 3, 4) else "k_bkproj5" if bp_form >= 10
                 else "k_bkproj4")
    wl = workload_name(s)
    ipu = load_profile_table("inst_per_update.txt").get((bp_kernel, wl))
    roofline = None
    bpk = kern.get("backproject")
    if bpk:
        t_bp = bpk["ms_per_step"] / 1e3
        clk = (clocks.get("sm_mhz") or 1965.0) * 1e6
        issue_peak = SMS * 4 * clk  # warp instructions per second
        roofline = {"kernel": bp_kernel, "bound": "issue",
                    "model": "warp instructions per update (ncu smsp__inst_executed.sum / "
                             "updates, profiles/inst_per_update.txt) x updates / kernel time, "
                             "over 148 SMs x 4 schedulers x the SM clock sampled in the run",
                    "inst_per_update": ipu, "unit": "Ginst/s",
                    "peak": issue_peak / 1e9, "peak_source": "148 x 4 x median SM clock",
                    "achieved": ipu * updates / t_bp / 1e9 if ipu else None,
                    "frac": ipu * updates / t_bp / issue_peak if ipu else None,
                    "traffic": load_traffic(bp_kernel, wl),
                    "hbm_gather_equivalent": {
                        "model": "16 B per update (the four FP32 taps the reference reads, "
                                 "KatsevichBkProj.cpp:253-256); the taps come from shared "
                                 "memory, so this is not an HBM bound",
                        "achieved_gbs": BYTES_PER_UPDATE * updates / t_bp / 1e9,
                        "hbm_peak_gbs": peaks["hbm_gbs"], "hbm_peak_source": peaks["source"]}}

    # ---- CPU baseline (rank 0, N = 1): the FP64 oracle restatement on a bounded sample -----------
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        try:
            O = _oracle()
            cores = os.cpu_count() or 1
            smp = CpuChainSample(O, s, lambda a, b: d_proj[a:b].cpu().numpy().astype(np.float64),
                                 updates, n=32, copies=1)
            # the sample repeated until 10 s of CPU time have passed
            reps = 0
            t0 = time.perf_counter()
            while reps == 0 or time.perf_counter() - t0 < 10.0:
                smp.filter_once()
                O.bkproj(smp.gb, smp.fproj, np.zeros((smp.n,) * 3), nthreads=cores)
                reps += 1
            t_smp = time.perf_counter() - t0
            g = reps * smp.updates / t_smp / 1e9
            cpu = {"value": g, "unit": "GUPS", "cores": cores, "kind": "port",
                   "s_per_vol": updates / (g * 1e9), "sample_s": t_smp, "repeats": reps,
                   "sample": smp.describe("the FP64 oracle's",
                                          f"the FP64 oracle with {cores} OpenMP threads") +
                   f"; repeated {reps} times ({t_smp:.1f} s)"}
        except Exception as exc:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "GUPS", "cores": 0, "kind": "port",
                   "sample": f"failed: {exc}"}

    if rank == 0:
        launches = sum(n for _, n in plain["kernel_times"].values())
        line = {"metric": METRIC, "value": value, "unit": "GUPS", "n_gpus": ws,
                "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic", "config": workload_config(s, ws),
                "form": {k: plain[k] for k in ("hilbert", "pi_solver", "bp_variant")},
                "updates_per_step": updates, "s_per_vol": ms_step / 1e3,
                "phase_ms": plain["phase_ms"],
                "bkproj_gups": updates / (plain["phase_ms"]["bkproj"] / 1e3) / 1e9,
                "gpu_launches": launches,
                "e2e": e2e, "e2e_mex_pinned": e2e_mex, "e2e_pageable": e2e_pageable,
                "roofline": roofline,
                "kernels": kern, "cpu_baseline": cpu, "clocks": clocks,
                "forms": {k: {kk: vv for kk, vv in v.items() if kk != "kernel_times"}
                          for k, v in forms.items()},
                "accuracy": accuracy, "pinet": pinet_info, "bp_tune": tune,
                "peaks": peaks}
        print(json.dumps(line))
    ctx.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.batched:
        run_batched(args)
        return
    if args.report:
        run_report(args)
        return
    run_headline(args)


if __name__ == "__main__":
    main()
