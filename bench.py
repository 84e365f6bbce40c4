"""Benchmark: BEM operator applies (matvecs) per second on one B200 per rank.

Workload (N = 1 line): the 60k-triangle direct-farfield configuration --
a 174 x 174 vertex grid over [-10, 10]^2 with topography
z = 0.5 exp(-(x^2 + y^2)/8) + 0.02 N(0, 1) (seed 2), 59,858 triangles,
538,722 DOF -- with the production elastic hypersingular operator
RegularizedSparseIntegralOp(6, 6, 6, 1, 5, 2.5, 'elasticRH3', 'elasticRH3',
[1, 0.25], ..., float32, TriToTriDirectFarfieldOp): 3-point farfield rule on
all 3.58e9 triangle pairs plus the corrected nearfield (BSR).
A step is one apply y = H x on a seeded N(0, 1) x (seed 3 + rank).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 runs under torchrun, one rank per GPU; every rank applies its own
operator to its own inputs (independent units, no collective on the data
path: weak scaling); time = max over ranks.  --impl reference times the
reference's algorithm on the host cores (the oracle restatement: the
reference's PyOpenCL CPU path cannot run here) on a bounded sample of the
same apply, extrapolated to one full apply.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

PARAMS = [1.0, 0.25]
NQ = dict(nq_co=6, nq_ea=6, nq_va=6, nq_far=1, nq_near=5, thr=2.5)
K_NAME = "elasticRH3"
# Algorithmic FP32 flops per farfield point pair of the hoisted elasticRH3
# kernel (FMA = 2): D 3, r^2 5, rsqrt 1, weights 4, S0 1, g*D 3, T 12 = 29,
# plus the per-triangle-pair W update 63 flops / 9 point pairs = 7.
FLOPS_PER_POINT_PAIR_RH = 36.0
# DRAM bytes of one far_main_rh2 launch on the 59,858-triangle surface (ncu
# dram__bytes_read.sum + dram__bytes_write.sum, one full-size capture): the
# kernel reads its source records through L2 and is compute-bound
FAR_TRAFFIC_BYTES = 14.856e6
# DRAM bytes of one bsr9_kernel launch on the same surface's nearfield matrix
# (5,477,848 blocks, rows aligned to 32 slots; one full-size capture):
# 1.05x the algorithmic 1.801e9 bytes
NEAR_TRAFFIC_BYTES = 1.8995e9


def c2_mesh(n=174, seed=2):
    from tectosaur_b200.mesh.mesh_gen import make_rect
    pts, tris = make_rect(n, n, [[-10, -10, 0], [10, -10, 0], [10, 10, 0], [-10, 10, 0]])
    rng = np.random.default_rng(seed)
    pts = pts.copy()
    pts[:, 2] = 0.5 * np.exp(-(pts[:, 0] ** 2 + pts[:, 1] ** 2) / 8.0) + \
        0.02 * rng.standard_normal(pts.shape[0])
    return pts, tris


def c4_mesh(n=707, seed=5):
    """The 1M-triangle FMM configuration: an n x n vertex grid over [-50, 50]^2
    with three seeded Gaussian hills (amplitude U[0.5, 2], width U[3, 10],
    centres U[-30, 30]^2) plus a 20 x 10 planar thrust fault dipping 30 degrees
    (top edge at z = -0.5, strike along x) meshed at the surface's spacing;
    surface and fault concatenated without merging vertices."""
    from tectosaur_b200.mesh.mesh_gen import concat_no_dedupe, make_rect
    rng = np.random.default_rng(seed)
    pts, tris = make_rect(n, n, [[-50, -50, 0], [50, -50, 0], [50, 50, 0], [-50, 50, 0]])
    pts = pts.copy()
    for _ in range(3):
        amp, width = rng.uniform(0.5, 2.0), rng.uniform(3.0, 10.0)
        cx, cy = rng.uniform(-30.0, 30.0, 2)
        pts[:, 2] += amp * np.exp(-((pts[:, 0] - cx) ** 2 + (pts[:, 1] - cy) ** 2) /
                                  (2.0 * width * width))
    h = 100.0 / (n - 1)
    dip = np.radians(30.0)
    y1, z1 = 10.0 * np.cos(dip), -0.5 - 10.0 * np.sin(dip)
    fault = make_rect(int(round(20.0 / h)) + 1, int(round(10.0 / h)) + 1,
                      [[-10, 0, -0.5], [10, 0, -0.5], [10, y1, z1], [-10, y1, z1]])
    return concat_no_dedupe((pts, tris), fault)


def build_op(pts, tris):
    import tectosaur_b200 as tct
    from tectosaur_b200.ops.sparse_farfield_op import TriToTriDirectFarfieldOp
    return tct.RegularizedSparseIntegralOp(
        NQ["nq_co"], NQ["nq_ea"], NQ["nq_va"], NQ["nq_far"], NQ["nq_near"], NQ["thr"],
        K_NAME, K_NAME, PARAMS, pts, tris, np.float32, TriToTriDirectFarfieldOp,
        keep_uncorrected=False)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu_index = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu_index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
            return
        # nvidia-smi's start-up (NVML initialisation) stalls the driver for
        # up to a second: a timed region that overlapped it measured a C4
        # near search at 0.93 s instead of 0.22 s; timing starts after the
        # first sample
        t0 = time.perf_counter()
        while not self.lines and self.proc.poll() is None and time.perf_counter() - t0 < 10.0:
            time.sleep(0.02)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, power = [], [], []
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "power_w_max": max(power) if power else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def measured_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return None


def fp32_peak_tflops(torch, lib):
    """Measured FP32 FMA throughput of this GPU (TFLOP/s, CUDA events):
    (scalar FFMA probe, packed fma.rn.f32x2 probe)."""
    from tectosaur_b200 import _lib
    out = torch.empty(256, dtype=torch.float32, device="cuda")
    n_blocks = 148 * 16
    iters = 8192
    res = []
    for fn, per_iter in [(lib.tct_fp32_fma_probe, 16), (lib.tct_fp32x2_fma_probe, 32)]:
        for _ in range(2):
            _lib.check(fn(_lib.tptr(out), n_blocks, iters, _lib.stream_ptr()), "fma probe")
        torch.cuda.synchronize()
        best = 0.0
        for _ in range(5):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            _lib.check(fn(_lib.tptr(out), n_blocks, iters, _lib.stream_ptr()), "fma probe")
            b.record()
            b.synchronize()
            ms = a.elapsed_time(b)
            best = max(best, n_blocks * 256.0 * iters * per_iter / (ms * 1e-3) / 1e12)
        res.append(best)
    return tuple(res)


# ---- CPU baseline: the reference's algorithm on the host cores ---------------
# These legs import nothing from tectosaur_b200 (no libtct_b200.so): meshes,
# near pairs (the reference's own compiled finder), rules (the reference's own
# arrays) and kernels (liboracle) all come from oracle/ref_pipeline.py.
def c2_mesh_ref(n=174, seed=2):
    """c2_mesh built without the product package (same arrays)."""
    from oracle import ref_pipeline as rp
    pts, tris = rp.make_rect(n, n, [[-10, -10, 0], [10, -10, 0], [10, 10, 0], [-10, 10, 0]])
    rng = np.random.default_rng(seed)
    pts = pts.copy()
    pts[:, 2] = 0.5 * np.exp(-(pts[:, 0] ** 2 + pts[:, 1] ** 2) / 8.0) + \
        0.02 * rng.standard_normal(pts.shape[0])
    return pts, tris


def c2_sample(pts, tris, classes, n_rows, seed, float_type, fast, n_threads=None):
    """Seeded observation rows of the C2 operator (oracle/ref_pipeline), their
    nearfield blocks integrated (setup)."""
    from oracle import ref_pipeline as rp
    n = tris.shape[0]
    rows = np.sort(np.random.default_rng(seed).choice(n, size=min(n_rows, n), replace=False))
    return rp.SampledRows(pts, tris, rows, NQ["nq_co"], NQ["nq_ea"], NQ["nq_va"], NQ["nq_far"],
                          NQ["nq_near"], NQ["thr"], K_NAME, PARAMS, float_type,
                          classes=classes, n_threads=n_threads, fast=fast)


def c2_classes(pts, tris):
    from oracle import ref_pipeline as rp
    return rp.classify(tris, rp.near_pairs(pts, tris, NQ["thr"]))


def cpu_step_rows(pts, tris, classes, target_s):
    """Rows per timed CPU step so that one step takes about target_s (timed
    build, all host threads)."""
    n = tris.shape[0]
    probe = c2_sample(pts, tris, classes, 32, 99, np.float32, True)
    x = np.random.default_rng(98).standard_normal(9 * n)
    probe.apply(x)
    t0 = time.perf_counter()
    probe.apply(x)
    per_row = max((time.perf_counter() - t0) / 32, 1e-6)
    return int(min(max(32, target_s / per_row), n // 4))


def cpu_baseline(pts, tris, classes=None, target_s=3.0, reps=3):
    """The reference operator's apply on the host cores: FP32 (the reference's
    default precision), the timed build of the oracle restatement (-O3
    -march=native, OpenMP on every host thread) on a seeded sample of
    observation rows -- farfield against all sources plus their nearfield
    BCOO rows; value = the fraction of an apply per second."""
    n = tris.shape[0]
    threads = os.cpu_count() or 1
    if classes is None:
        classes = c2_classes(pts, tris)
    n_s = cpu_step_rows(pts, tris, classes, target_s)
    s = c2_sample(pts, tris, classes, n_s, 3, np.float32, True)
    x = np.random.default_rng(3).standard_normal(9 * n)
    s.apply(x)
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        s.apply(x)
        ts.append(time.perf_counter() - t0)
    t = statistics.median(ts)
    return {
        "value": (n_s / n) / t, "unit": "matvecs/s", "cores": threads, "kind": "port",
        "sample": ("oracle restatement of the reference kernels, FP32, -O3 -march=native, "
                   "OpenMP %d threads: rows of %d seeded observation triangles of %d (farfield "
                   "against all sources + their %d nearfield blocks), median of %d applies "
                   "%.2f s; value = (%d / %d of an apply) / time"
                   % (threads, n_s, n, s.n_blocks, reps, t, n_s, n)),
    }


def c2_parity(pts, tris, y_dev, x, classes=None, n_rows=512, seed=17):
    """Relative 2-norm error of the timed FP32 apply y_dev on n_rows seeded
    observation rows against the FP64 oracle (checker build) of the same
    rows: farfield against all sources + corrected nearfield rows."""
    if classes is None:
        classes = c2_classes(pts, tris)
    s = c2_sample(pts, tris, classes, n_rows, seed, np.float64, False)
    want = s.apply(np.asarray(x, dtype=np.float64))
    got = np.asarray(y_dev, dtype=np.float64).reshape(-1, 9)[s.rows].reshape(-1)
    err = float(np.linalg.norm(got - want) / np.linalg.norm(want))
    far = s.farfield(np.asarray(x, dtype=np.float64))
    return {"rel_err_fp64": err, "rows": int(s.rows.shape[0]), "seed": seed,
            "oracle": "FP64 oracle restatement (no FMA contraction) of the reference operator "
                      "on the sampled rows; near pairs from the reference's compiled finder, "
                      "rules from the reference's arrays",
            "far_share_of_norm": float(np.linalg.norm(far) / np.linalg.norm(want))}


def run_reference(args, rank, world):
    """The reference arm: the reference operator's apply on the host cores
    (see cpu_baseline), one sampled partial apply per step."""
    if rank != 0:
        return
    pts, tris = c2_mesh_ref()
    n = tris.shape[0]
    classes = c2_classes(pts, tris)
    nnzb = int(sum(v.shape[0] for v in classes.values()))
    threads = os.cpu_count() or 1
    n_s = cpu_step_rows(pts, tris, classes, 1.0)
    s = c2_sample(pts, tris, classes, n_s, 3, np.float32, True)
    x = np.random.default_rng(3).standard_normal(9 * n)
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        s.apply(x)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    t = float(np.sum(times))
    frac = n_s / n
    value = args.steps * frac / t
    line = {
        "metric": "BEM matvecs/s", "value": value, "unit": "matvecs/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "impl": "reference",
        "config": dict(config_block(n, nnzb), step=(
            "one partial apply: the %d seeded observation rows of %d (%.4f of an apply); "
            "value = steps x %.4f / time" % (n_s, n, frac, frac))),
        "cpu_baseline": {"value": value, "unit": "matvecs/s", "cores": threads, "kind": "port",
                         "sample": "each step: farfield of %d of %d observation triangles "
                                   "against all sources + their %d nearfield BCOO blocks, "
                                   "oracle restatement FP32, -O3 -march=native, OpenMP %d "
                                   "threads (the reference's PyOpenCL CPU path cannot run: "
                                   "no pyopencl, no CPU OpenCL platform)"
                                   % (n_s, n, s.n_blocks, threads)},
        "e2e": {"value": value, "unit": "matvecs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


FMM_CFG = dict(mac=3.0, pts_per_cell=128, order=8, mode="fmm")


def fmm_algorithmic_flops(fmm, n_q):
    """FP32 flops of one FMM apply counted from the interaction lists: P2P
    point pairs x 36 (the hoisted elasticRH3 pair loop) + M2L pairs x
    C(p+6, 6) (a, b) products x 21 channels x 2."""
    st, ot = fmm.src_tree, fmm.obs_tree
    l = fmm.p2p
    n_o = (ot.end - ot.start)[l.obs_n_idxs]
    lens = np.diff(l.obs_src_starts)
    n_s = (st.end - st.start)[l.src_n_idxs]
    src_per_obs = np.add.reduceat(n_s, l.obs_src_starts[:-1]) if lens.size else np.zeros(0)
    p2p_pairs = float(np.sum(n_o * src_per_obs)) * n_q * n_q
    p = fmm.order
    ab = (p + 1) * (p + 2) * (p + 3) * (p + 4) * (p + 5) * (p + 6) / 720.0
    m2l = float(fmm.m2l.src_n_idxs.shape[0]) * ab * 21 * 2
    return p2p_pairs * FLOPS_PER_POINT_PAIR_RH + m2l, p2p_pairs, m2l


def cpu_direct_far_baseline(pts, tris, target_s=10.0, K=None):
    """The direct farfield on the host cores (oracle restatement, FP32, all
    threads) for a sample of observation triangles against all sources,
    extrapolated to one full apply (the reference's FMM has no CPU path)."""
    from oracle import oracle as orc
    from tectosaur_b200.util.quadrature import gauss2d_tri
    n = tris.shape[0]
    rng = np.random.default_rng(11)
    x = rng.standard_normal(n * 9)
    q = gauss2d_tri(1)
    def t_sample(m):
        obs = np.sort(rng.choice(n, size=m, replace=False))
        t0 = time.perf_counter()
        orc.farfield_tris(K or K_NAME, np.float32, q, pts, tris[obs], tris, x, PARAMS)
        return time.perf_counter() - t0
    probe = 16
    per = max(t_sample(probe) / probe, 1e-6)
    m = int(min(max(probe, target_s / per), n // 4))
    t = t_sample(m)
    t_full = t * n / m
    return {"value": 1.0 / t_full, "unit": "matvecs/s", "cores": os.cpu_count() or 1,
            "kind": "port",
            "sample": ("direct farfield (the reference's CPU-runnable algorithm; its treecode "
                       "has no CPU path) of %d of %d observation triangles against all "
                       "sources, oracle restatement FP32 on %d threads, %.1f s, extrapolated "
                       "to one apply (%.0f s)" % (m, n, os.cpu_count() or 1, t, t_full))}


def run_fmm_workload(args, rank, world, torch, dist):
    from tectosaur_b200 import _lib
    from tectosaur_b200.fmm.tsfmm import FMMFarfieldOpImpl
    from tectosaur_b200.ops.sparse_farfield_op import TriToTriDirectFarfieldOp
    pts, tris = c4_mesh(args.grid or 707)
    n = tris.shape[0]
    idx = np.arange(n)
    cfg = dict(FMM_CFG)
    if args.fmm_order is not None:
        cfg["order"] = args.fmm_order
    if args.fmm_ppc is not None:
        cfg["pts_per_cell"] = args.fmm_ppc
    if args.fmm_mode is not None:
        cfg["mode"] = args.fmm_mode
    t0 = time.perf_counter()
    op = FMMFarfieldOpImpl(1, K_NAME, PARAMS, pts, tris, np.float32, idx, idx, cfg["mac"],
                           cfg["pts_per_cell"], cfg["order"], cfg["mode"])
    torch.cuda.synchronize()
    t_build = time.perf_counter() - t0
    x = torch.from_numpy(np.random.default_rng(3 + rank).standard_normal(9 * n)
                         .astype(np.float32)).cuda()
    y = torch.empty_like(x)
    for _ in range(args.warmup):
        op.dot_device(x, y)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    sampler.start()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    for _ in range(args.steps):
        op.dot_device(x, y)
    b.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    total_ms = a.elapsed_time(b)
    if dist is not None:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms = total_ms / args.steps
    # accuracy on sampled rows against the direct farfield
    sample = np.sort(np.random.default_rng(7).choice(n, 2048, replace=False))
    d = TriToTriDirectFarfieldOp(1, K_NAME, PARAMS, pts, tris, np.float32, sample, idx)
    yd = torch.empty(9 * sample.shape[0], dtype=torch.float32, device="cuda")
    d.dot_device(x, yd)
    rows = (sample[:, None] * 9 + np.arange(9)).reshape(-1)
    ref = yd.double().cpu().numpy()
    err = float(np.linalg.norm(y.double().cpu().numpy()[rows] - ref) / np.linalg.norm(ref))
    del d
    # e2e through the public API with host arrays
    xh = x.cpu().numpy()
    op.dot(xh)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        yh = op.dot(xh)
    t_e2e = time.perf_counter() - t0
    if dist is not None:
        t = torch.tensor([t_e2e], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_e2e = float(t.item())
    if rank != 0:
        return
    flops, p2p_pairs, m2l_flops = fmm_algorithmic_flops(op.fmm, op.fmm.nq)
    peak_ffma, peak_ffma2 = fp32_peak_tflops(torch, _lib.lib)
    peak = max(peak_ffma, peak_ffma2)
    achieved = flops / (ms * 1e-3) / 1e12
    n_launch = 8 + op.fmm.src_desc.n_levels + op.fmm.obs_desc.n_levels
    line = {
        "metric": "BEM farfield matvecs/s (FMM)", "value": world * args.steps / (total_ms * 1e-3),
        "unit": "matvecs/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded mesh and inputs)",
        "config": {"workload": ("FMM farfield of the 1M-triangle topographic surface + "
                                "dipping thrust fault (%d triangles), elasticRH3, 3-point "
                                "rule, FMMFarfieldOp(mac=%g, pts_per_cell=%d, order=%d, "
                                "mode=%s)" % (n, cfg["mac"], cfg["pts_per_cell"],
                                              cfg["order"], cfg["mode"])),
                   "n_tris": int(n), "dof": int(9 * n), "p2p_leaf_pairs":
                   int(op.fmm.p2p.src_n_idxs.shape[0]), "m2l_pairs":
                   int(op.fmm.m2l.src_n_idxs.shape[0]), "m2p_pairs":
                   int(op.fmm.m2p.src_n_idxs.shape[0]), "tree_nodes": int(op.fmm.src_tree.n_nodes),
                   "setup_s": t_build, "rel_err_vs_direct_2048_rows": err,
                   "l2": "inputs larger than L2 (workspace %.0f MB per apply)"
                         % (op.fmm.ws_bytes / 1e6), "parallelism": "replicas"},
        "roofline": {"kernel": "whole FMM apply (P2P + M2L dominate)", "bound": "fp32",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": None,
                     "peak_source": "measured live: best FP32 FMA probe (scalar %.1f, packed "
                                    "%.1f TFLOP/s)" % (peak_ffma, peak_ffma2),
                     "algorithmic": "%.3e flops per apply: %.3e P2P point pairs x 36 + M2L "
                                    "%.3e" % (flops, p2p_pairs, m2l_flops)},
        "e2e": {"value": world * args.steps / t_e2e, "unit": "matvecs/s",
                "h2d_bytes_per_step": int(xh.nbytes), "d2h_bytes_per_step": int(yh.nbytes),
                "api": "FMMFarfieldOpImpl.dot(numpy float32) -> numpy"},
        "gpu_launches": args.steps * n_launch,
        "clocks": clocks,
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_direct_far_baseline(pts, tris)
    print(json.dumps(line), flush=True)


def c1_mesh():
    """The small plain-method configuration: make_rect(20, 20) over [-1, 1]^2
    (722 triangles, 6,498 DOF)."""
    from tectosaur_b200.mesh.mesh_gen import make_rect
    return make_rect(20, 20, [[-1, -1, 0], [-1, 1, 0], [1, 1, 0], [1, -1, 0]])


C1_NQ = (6, 6, 6, 2, 5, 2.5)


def cpu_solve_baseline(pts, tris, cm, rhs, tol):
    """scipy GMRES (restart 200) on the host driving the oracle restatement
    of the FP64 operator (nearfield blocks assembled once, untimed; farfield
    recomputed per matvec on all host threads): the reference's
    examples/solve.py:25-61 algorithm on the host cores."""
    import scipy.sparse
    import scipy.sparse.linalg
    from oracle import oracle as orc
    from tectosaur_b200.nearfield import triangle_rules as trr
    from tectosaur_b200.nearfield.nearfield_op import nearfield_pairs
    from tectosaur_b200.util.quadrature import gauss2d_tri, gauss4d_tri
    nq_co, nq_ea, nq_va, nq_far, nq_near, thr = C1_NQ
    n = tris.shape[0]
    idx = np.arange(n)
    cl = nearfield_pairs(pts, tris, idx, idx, thr)
    rules = {"co": (trr.coincident_quad(nq_co), False, True),
             "ea": (trr.edge_adj_quad(nq_ea), True, True),
             "va": (trr.vertex_adj_quad(nq_va, nq_va, nq_va), True, True),
             "near": (gauss4d_tri(nq_near, nq_near), False, False)}
    far4 = gauss4d_tri(nq_far, nq_far)
    rows, cols, vals = [], [], []
    for c, (rule, adj, check0) in rules.items():
        recs, dofs = cl[c]
        b = orc.pairs(K_NAME, np.float64, rule, pts, tris, recs[:, :5 if adj else 2], PARAMS,
                      adj=adj, check0=check0)
        b = b - orc.pairs(K_NAME, np.float64, far4, pts, tris, recs[:, :2], PARAMS,
                          check0=(c == "co"))
        b = b.reshape(-1, 9, 9)
        r = np.broadcast_to(dofs[:, 0][:, None, None] * 9 + np.arange(9)[None, :, None], b.shape)
        cc = np.broadcast_to(dofs[:, 1][:, None, None] * 9 + np.arange(9)[None, None, :], b.shape)
        rows.append(r.reshape(-1))
        cols.append(cc.reshape(-1))
        vals.append(b.reshape(-1))
    near = scipy.sparse.csr_matrix((np.concatenate(vals), (np.concatenate(rows),
                                    np.concatenate(cols))), shape=(9 * n, 9 * n))
    q = gauss2d_tri(nq_far)
    cmT = cm.T.tocsr()

    def mv(v):
        u = cm @ v
        return cmT @ (orc.farfield_tris(K_NAME, np.float64, q, pts, tris, tris, u, PARAMS) +
                      near @ u)
    m = cm.shape[1]
    A = scipy.sparse.linalg.LinearOperator((m, m), matvec=mv)
    count = [0]

    def cb(_):
        count[0] += 1
    t0 = time.perf_counter()
    scipy.sparse.linalg.gmres(A, cmT @ rhs, rtol=tol, restart=200, callback=cb,
                              callback_type="pr_norm")
    t = time.perf_counter() - t0
    return {"value": 1.0 / t, "unit": "solves/s", "cores": os.cpu_count() or 1, "kind": "port",
            "sample": ("one full solve: scipy GMRES (restart 200, rtol %g, %d iterations) on "
                       "the host with the oracle restatement of the FP64 operator (farfield "
                       "per matvec on %d threads, nearfield blocks assembled beforehand), "
                       "%.2f s" % (tol, count[0], os.cpu_count() or 1, t))}


def run_solve_workload(args, rank, world, torch, dist):
    import tectosaur_b200 as tct
    from tectosaur_b200.ops.sparse_farfield_op import TriToTriDirectFarfieldOp
    from tectosaur_b200.simple_solver import (ConstrainedOperator, free_edge_vertices, gmres,
                                              iterative_solve, shared_vertex_matrix)
    tol = 1e-8
    pts, tris = c1_mesh()
    n = tris.shape[0]
    op = tct.RegularizedSparseIntegralOp(*C1_NQ, K_NAME, K_NAME, PARAMS, pts, tris, np.float64,
                                         TriToTriDirectFarfieldOp)
    cm = shared_vertex_matrix(tris, fixed_vertices=free_edge_vertices(tris))
    rhs = np.random.default_rng(1 + rank).standard_normal(9 * n)
    cop = ConstrainedOperator(op, cm)
    b = torch.empty(cm.shape[1], dtype=torch.float64, device="cuda")
    cop.cmT.dot_device(torch.from_numpy(rhs).cuda(), b)
    # one matvec of the seeded slip vector (seed 0), then the solves
    xs = torch.from_numpy(np.random.default_rng(0).standard_normal(9 * n)).cuda()
    ys = torch.empty_like(xs)
    op.dot_device(xs, ys)
    for _ in range(args.warmup):
        gmres(cop, b, tol=tol, restart=200)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    sampler.start()
    lat, iters = [], []
    cop.n_matvecs = 0
    a = torch.cuda.Event(enable_timing=True)
    e = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    for _ in range(args.steps):
        t0 = time.perf_counter()
        x, info, it, _ = gmres(cop, b, tol=tol, restart=200)
        torch.cuda.synchronize()
        lat.append(time.perf_counter() - t0)
        iters.append(it)
    e.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    total_ms = a.elapsed_time(e)
    if dist is not None:
        tt = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        total_ms = float(tt.item())
    # e2e: the public drop-in with host arrays
    t0 = time.perf_counter()
    for _ in range(args.steps):
        u = iterative_solve(op, cm, rhs, cfg=dict(solver_tol=tol))
    t_e2e = time.perf_counter() - t0
    if rank != 0:
        return
    ms = total_ms / args.steps
    it_mean = float(np.mean(iters))
    nnzb = op.nearfield.bsr.nnzb
    m = cm.shape[1]
    # bytes one GMRES step must move: nearfield blocks + x/y, and the two
    # classical Gram-Schmidt passes over the basis (read twice each)
    avg_basis = min(it_mean, 200) / 2.0 + 1
    bytes_step = nnzb * (81 * 8 + 4) + 2 * 9 * n * 8 + 4 * avg_basis * m * 8
    achieved = bytes_step * it_mean / (ms * 1e-3) / 1e9
    mp = measured_peaks()
    hbm = mp.get("hbm_gbs") if mp else 6650.0
    line = {
        "metric": "BEM solves/s (GMRES to 1e-8)", "value": world * args.steps / (total_ms * 1e-3),
        "unit": "solves/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded mesh and right-hand sides)",
        "config": {"workload": ("plain FP64 solve: make_rect(20, 20) over [-1, 1]^2 (722 "
                                "triangles, 6,498 DOF), RegularizedSparseIntegralOp(6, 6, 6, 2, "
                                "5, 2.5, elasticRH3) with the direct farfield, vertex continuity + "
                                "zero slip on the free edges, GMRES(200) to 1e-8 for a N(0, 1) "
                                "traction"),
                   "n_tris": int(n), "dof": int(9 * n), "free_dof": int(m),
                   "gmres_iterations": it_mean, "latency_ms_p50": 1e3 * float(np.percentile(lat, 50)),
                   "latency_ms_p99": 1e3 * float(np.percentile(lat, 99)),
                   "l2": "small problem: working set fits in L2 (latency-bound solve)",
                   "parallelism": "replicas"},
        "roofline": {"kernel": "whole GMRES step (operator apply + CGS2 orthogonalisation)",
                     "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": None,
                     "peak_source": "MEASURED_PEAKS.json" if mp else "fallback",
                     "algorithmic": "%.3e bytes per GMRES step" % bytes_step},
        "e2e": {"value": args.steps / t_e2e, "unit": "solves/s",
                "h2d_bytes_per_step": int(rhs.nbytes), "d2h_bytes_per_step": int(u.nbytes),
                "api": "simple_solver.iterative_solve(op, cm, numpy rhs) -> numpy"},
        "gpu_launches": int(args.steps * it_mean * 6),
        "clocks": clocks,
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_solve_baseline(pts, tris, cm, rhs, tol)
    print(json.dumps(line), flush=True)


# ---- C3: batched singular / near-singular pair quadrature --------------------
# (singular-class kernel, near-class kernel) per family
C3_FAMILIES = [("elasticU3", "elasticU3"), ("elasticRT3", "elasticT3"),
               ("elasticRA3", "elasticA3"), ("elasticRH3", "elasticH3")]
# FP64 flops per quadrature point of this build's pair integrand
# (csrc/pair_math.cuh, FMA = 2): 42 shared (two barycentric points, D, r^2)
# + the kernel's tensor/separable form + the 81-output accumulation
# (U 241, T/A 283, H 361, RT/RA 971 -- the Levi-Civita surface-curl
# contraction -- and RH 63, whose separable form keeps 7 sums instead of 81).
PAIR_POINT_FLOPS = {"elasticU3": 241, "elasticT3": 283, "elasticA3": 283, "elasticH3": 361,
                    "elasticRT3": 971, "elasticRA3": 971, "elasticRH3": 63}


def _rand_planar_tris(rng, m, max_aspect=5.0):
    """m random triangles in 2-D with v0 at the origin, v1 on +x: edge lengths
    U[0.5, 2], aspect (longest edge / shortest altitude) <= max_aspect."""
    out = np.zeros((m, 3, 2))
    todo = np.arange(m)
    while todo.size:
        k = todo.size
        L1, L2 = rng.uniform(0.5, 2.0, k), rng.uniform(0.5, 2.0, k)
        th = rng.uniform(np.radians(20), np.radians(160), k)
        v2 = np.stack([L2 * np.cos(th), L2 * np.sin(th)], axis=1)
        L3 = np.hypot(v2[:, 0] - L1, v2[:, 1])
        area = 0.5 * L1 * v2[:, 1]
        longest = np.maximum(np.maximum(L1, L2), L3)
        ok = (L3 >= 0.5) & (L3 <= 2.0) & (longest ** 2 / (2 * area) <= max_aspect)
        good = todo[ok]
        out[good, 1, 0] = L1[ok]
        out[good, 2] = v2[ok]
        todo = todo[~ok]
    return out


def c3_pairs(n_pairs=400_000, seed=4):
    """Seeded random triangle pairs: 10 % coincident / 30 % edge-adjacent /
    30 % vertex-adjacent / 30 % separate (parallel, gap U[0.01, 1] x mean edge),
    edge lengths U[0.5, 2], aspect <= 5; per pair a quadrature order U{3..20},
    a kernel family (U / T / A / H, the singular classes taking the
    regularized RT / RA / RH) and nu in {0.25, 0.35}.  Returns the mesh and
    per-class records in the operator's pair-record format."""
    from tectosaur_b200.mesh.find_near_adj import split_adjacent_close
    from tectosaur_b200.nearfield.nearfield_op import resolve_ea_rotation
    rng = np.random.default_rng(seed)
    n = n_pairs
    cls = rng.choice(4, size=n, p=[0.1, 0.3, 0.3, 0.3])  # co, ea, va, near
    fam = rng.integers(0, 4, n)
    nq = rng.integers(3, 21, n)
    nu_id = rng.integers(0, 2, n)
    # a random orthonormal frame per pair
    nrm = rng.standard_normal((n, 3))
    nrm /= np.linalg.norm(nrm, axis=1)[:, None]
    a = rng.standard_normal((n, 3))
    e1 = np.cross(nrm, a)
    e1 /= np.linalg.norm(e1, axis=1)[:, None]
    e2 = np.cross(nrm, e1)
    centre = np.stack([(np.arange(n) % 1000) * 20.0, (np.arange(n) // 1000) * 20.0,
                       np.zeros(n)], axis=1)

    def place(p2, z=0.0):  # (m, 2) in-plane coordinates (+ normal offset) -> 3-D
        return centre + p2[:, :1] * e1 + p2[:, 1:2] * e2 + np.asarray(z).reshape(-1, 1) * nrm

    t1 = _rand_planar_tris(rng, n)
    v = [place(t1[:, k]) for k in range(3)]
    extra = []
    # edge-adjacent: across edge v0 v1, tilted about it by a dihedral angle
    t2 = _rand_planar_tris(rng, n)
    xm = rng.uniform(0.25, 0.75, n) * t1[:, 1, 0]
    h = np.abs(t2[:, 2, 1])
    phi = rng.uniform(-np.radians(80), np.radians(80), n)
    v3 = centre + xm[:, None] * e1 - (h * np.cos(phi))[:, None] * e2 + (h * np.sin(phi))[:, None] * nrm
    # vertex-adjacent: a second triangle at v0 in the other half-plane, tilted
    t3 = _rand_planar_tris(rng, n)
    th3 = np.arctan2(t3[:, 2, 1], t3[:, 2, 0])
    psi = np.pi + 0.2 + rng.uniform(0, 1, n) * (np.pi - 0.4 - th3)
    rot = lambda p, ang: np.stack([p[:, 0] * np.cos(ang) - p[:, 1] * np.sin(ang),
                                   p[:, 0] * np.sin(ang) + p[:, 1] * np.cos(ang)], axis=1)
    tilt = rng.uniform(-np.radians(60), np.radians(60), n)
    def tilted(p):
        q = rot(p, psi)
        return centre + q[:, :1] * e1 + (q[:, 1] * np.cos(tilt))[:, None] * e2 + \
            (q[:, 1] * np.sin(tilt))[:, None] * nrm
    v4, v5 = tilted(t3[:, 1]), tilted(t3[:, 2])
    # separate: a parallel triangle at a small gap
    t4 = _rand_planar_tris(rng, n)
    mean_edge = (t1[:, 1, 0] + np.hypot(*t1[:, 2].T) + np.hypot(t1[:, 2, 0] - t1[:, 1, 0],
                                                               t1[:, 2, 1])) / 3
    gap = rng.uniform(0.01, 1.0, n) * mean_edge
    ang = rng.uniform(0, 2 * np.pi, n)
    shift = rng.uniform(-0.3, 0.3, (n, 2))
    w = [place(rot(t4[:, k], ang) + shift, gap) for k in range(3)]
    pts, tris, t1_idx, t2_idx = [], [], np.zeros(n, np.int64), np.zeros(n, np.int64)
    base = 0
    # vectorised assembly, pair by class
    nv = np.array([3, 4, 5, 6])[cls]
    start = np.concatenate([[0], np.cumsum(nv)])[:-1]
    P = np.zeros((int(nv.sum()), 3))
    for k in range(3):
        P[start + k] = v[k]
    co, ea, va, nr = (cls == 0), (cls == 1), (cls == 2), (cls == 3)
    P[start[ea] + 3] = v3[ea]
    P[start[va] + 3] = v4[va]
    P[start[va] + 4] = v5[va]
    for k in range(3):
        P[start[nr] + 3 + k] = w[k][nr]
    ntri = np.where(co, 1, 2)
    tstart = np.concatenate([[0], np.cumsum(ntri)])[:-1]
    T = np.zeros((int(ntri.sum()), 3), np.int64)
    T[tstart] = start[:, None] + np.arange(3)
    T[tstart[ea] + 1] = np.stack([start[ea] + 1, start[ea], start[ea] + 3], axis=1)
    T[tstart[va] + 1] = np.stack([start[va], start[va] + 3, start[va] + 4], axis=1)
    T[tstart[nr] + 1] = start[nr][:, None] + 3 + np.arange(3)
    t1_idx = tstart
    t2_idx = np.where(co, tstart, tstart + 1)
    close = np.stack([t1_idx[~co], t2_idx[~co]], axis=1)
    near_d, va_d, ea_d = split_adjacent_close(close, T, T)
    ea_rec = resolve_ea_rotation(T, ea_d)
    va_rec = np.hstack([va_d[:, :4], np.zeros((va_d.shape[0], 1), np.int64)])
    near_rec = np.hstack([near_d[:, :2], np.zeros((near_d.shape[0], 3), np.int64)])
    co_rec = np.stack([t1_idx[co], t1_idx[co]] + [np.zeros(int(co.sum()), np.int64)] * 3, axis=1)
    pair_of_tri = np.zeros(T.shape[0], np.int64)
    pair_of_tri[t1_idx] = np.arange(n)
    recs = {"co": co_rec, "ea": ea_rec, "va": va_rec, "near": near_rec}
    owner = {c: pair_of_tri[r[:, 0]] for c, r in recs.items()}
    return P, T, recs, owner, dict(cls=cls, fam=fam, nq=nq, nu_id=nu_id)


def c3_rule(kind, nq):
    from tectosaur_b200.nearfield import triangle_rules as trr
    from tectosaur_b200.util.quadrature import gauss4d_tri
    if kind == "co":
        return (*trr.coincident_quad(nq), False, True)
    if kind == "ea":
        return (*trr.edge_adj_quad(nq), True, True)
    if kind == "va":
        return (*trr.vertex_adj_quad(nq, nq, nq), True, True)
    return (*gauss4d_tri(nq, nq), False, False)


def c3_groups(recs, owner, attr):
    """Per kernel: records, rule ids into a per-kernel rule list, nu ids."""
    groups = {}
    for kind, r in recs.items():
        o = owner[kind]
        for f, (ks, kn) in enumerate(C3_FAMILIES):
            K = kn if kind == "near" else ks
            sel = attr["fam"][o] == f
            if not sel.any():
                continue
            g = groups.setdefault(K, dict(recs=[], keys=[], nu=[]))
            g["recs"].append(r[sel])
            g["keys"].append(np.stack([np.full(int(sel.sum()), ["co", "ea", "va", "near"].index(kind)),
                                       attr["nq"][o[sel]]], axis=1))
            g["nu"].append(attr["nu_id"][o[sel]])
    out = {}
    for K, g in groups.items():
        keys = np.concatenate(g["keys"])
        uk, rid = np.unique(keys, axis=0, return_inverse=True)
        rules = [c3_rule(["co", "ea", "va", "near"][k], int(q)) for k, q in uk]
        out[K] = dict(recs=np.concatenate(g["recs"]), rule_ids=rid.reshape(-1), rules=rules,
                      nu=np.concatenate(g["nu"]))
    return out


def fp64_peak_tflops(torch, lib):
    from tectosaur_b200 import _lib
    out = torch.empty(256, dtype=torch.float64, device="cuda")
    n_blocks, iters = 148 * 16, 2048
    for _ in range(2):
        _lib.check(lib.tct_fp64_fma_probe(_lib.tptr(out), n_blocks, iters, _lib.stream_ptr()),
                   "fp64 probe")
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        _lib.check(lib.tct_fp64_fma_probe(_lib.tptr(out), n_blocks, iters, _lib.stream_ptr()),
                   "fp64 probe")
        b.record()
        b.synchronize()
        best = max(best, n_blocks * 256.0 * iters * 16 / (a.elapsed_time(b) * 1e-3) / 1e12)
    return best


def cpu_pairs_baseline(P, T, groups, flops_total, target_s=12.0):
    """The oracle restatement of the reference's pair kernels (FP64, all host
    threads) on a random sample of each kernel's pairs, extrapolated to the
    whole workload by algorithmic flops."""
    from oracle import oracle as orc
    rng = np.random.default_rng(12)
    psets = np.array([[1.0, 0.25], [1.0, 0.35]])

    def run(frac):
        t_all, fl = 0.0, 0.0
        for K, g in groups.items():
            m = max(1, int(frac * g["recs"].shape[0]))
            pick = rng.choice(g["recs"].shape[0], m, replace=False)
            # one oracle call per (rule, nu) group, so its OpenMP loop has pairs to share
            key = g["rule_ids"][pick] * 2 + g["nu"][pick]
            for k in np.unique(key):
                sel = pick[key == k]
                pts4, wts, adj, c0 = g["rules"][g["rule_ids"][sel[0]]]
                t0 = time.perf_counter()
                orc.pairs(K, np.float64, (pts4, wts), P, T, g["recs"][sel, :5 if adj else 2],
                          psets[g["nu"][sel[0]]], adj=adj, check0=c0)
                t_all += time.perf_counter() - t0
                fl += sel.size * wts.shape[0] * PAIR_POINT_FLOPS[K]
        return t_all, fl
    t, fl = run(2e-5)
    frac = min(2e-5 * target_s / max(t, 1e-3), 1e-2)
    t, fl = run(frac)
    t_full = t * flops_total / fl
    n = sum(g["recs"].shape[0] for g in groups.values())
    return {"value": n / t_full, "unit": "pairs/s", "cores": os.cpu_count() or 1,
            "kind": "port",
            "sample": ("oracle restatement of the reference's pair kernels (FP64, OpenMP all "
                       "threads) on %.2g of each kernel's pairs (%.1f s), extrapolated by "
                       "algorithmic flops to the %d-pair workload (%.0f s)"
                       % (frac, t, n, t_full))}


def run_pairs_workload(args, rank, world, torch, dist):
    from tectosaur_b200 import _lib
    from tectosaur_b200.nearfield.pairs_integrator import PairsIntegrator
    from tectosaur_b200.util.sparse import DeviceBSR9, make_bsr_index
    n_pairs = args.pairs
    t0 = time.perf_counter()
    P, T, recs, owner, attr = c3_pairs(n_pairs, seed=4 + rank)
    groups = c3_groups(recs, owner, attr)
    psets = np.array([[1.0, 0.25], [1.0, 0.35]])
    runs, flops, points = [], 0.0, 0
    for K, g in groups.items():
        pi = PairsIntegrator(K, psets[0], np.float64, 2, 2, P, T)
        plan = pi.batched_plan(g["recs"], g["rule_ids"], g["rules"], g["nu"], psets)
        out = torch.empty(plan["n"] * 81, dtype=torch.float64, device="cuda")
        runs.append((pi, plan, out, K))
        sizes = np.array([r[0].shape[0] for r in g["rules"]])[g["rule_ids"]]
        points += int(sizes.sum())
        flops += float(sizes.sum()) * PAIR_POINT_FLOPS[K]
    t_setup = time.perf_counter() - t0

    def step():
        for pi, plan, out, _ in runs:
            pi.batched_run(plan, out)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    sampler.start()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    for _ in range(args.steps):
        step()
    b.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    total_ms = a.elapsed_time(b)
    if dist is not None:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms = total_ms / args.steps
    # BSR matvec on the assembled blocks (rows = obs triangle, cols = source)
    allrec = np.concatenate([g["recs"] for g in groups.values()])
    blocks = torch.cat([out for _, _, out, _ in runs]).view(-1, 81)
    n_tri = T.shape[0]
    indptr, indices, slot = make_bsr_index(n_tri, allrec[:, 0], allrec[:, 1])
    bsr = DeviceBSR9((9 * n_tri, 9 * n_tri), indptr, indices, np.float64)
    order = torch.from_numpy(np.argsort(slot)).cuda()
    bsr.data.view(81, -1)[:, :blocks.shape[0]] = blocks.index_select(0, order).t()
    xb = torch.from_numpy(np.random.default_rng(5).standard_normal(9 * n_tri)).cuda()
    yb = torch.empty_like(xb)

    def time_bsr():
        for _ in range(3):
            bsr.matvec(xb, yb)
        torch.cuda.synchronize()
        c = torch.cuda.Event(enable_timing=True)
        d = torch.cuda.Event(enable_timing=True)
        c.record()
        for _ in range(20):
            bsr.matvec(xb, yb)
        d.record()
        torch.cuda.synchronize()
        return c.elapsed_time(d) / 20
    # the default shape (a warp per block row), then the autotuned one (rows
    # of one or two blocks: several rows per warp)
    from tectosaur_b200 import autotune
    bsr_ms_default = time_bsr()
    bsr_shape = autotune.tune_bsr(bsr, xb)
    bsr_ms = time_bsr()
    nnzb = bsr.nnzb
    bsr_bytes = nnzb * (81 * 8 + 4) + (n_tri + 1) * 4 + 2 * 9 * n_tri * 8
    # e2e: the public per-call API (plan + upload + launch + copy out)
    t0 = time.perf_counter()
    for _ in range(max(1, min(args.steps, 2))):
        for K, g in groups.items():
            pi = [r[0] for r in runs if r[3] == K][0]
            hb = pi.batched(g["recs"], g["rule_ids"], g["rules"], g["nu"], psets)
    k_e2e = max(1, min(args.steps, 2))
    t_e2e = (time.perf_counter() - t0) / k_e2e
    if rank != 0:
        return
    peak64 = fp64_peak_tflops(torch, _lib.lib)
    achieved = flops / (ms * 1e-3) / 1e12
    mp = measured_peaks()
    hbm = mp.get("hbm_gbs") if mp else 6650.0
    line = {
        "metric": "pair integrals/s (batched singular quadrature)",
        "value": world * n_pairs / (ms * 1e-3), "unit": "pairs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded random triangle pairs)",
        "config": {"workload": ("%d seeded random triangle pairs (10 %% coincident, 30 %% "
                                "edge-adjacent, 30 %% vertex-adjacent, 30 %% separate with gap "
                                "U[0.01, 1] x edge; edges U[0.5, 2], aspect <= 5), order "
                                "U{3..20} per pair, kernels U/T/A/H (RT/RA/RH for the singular "
                                "classes), nu in {0.25, 0.35}, FP64, %d batched launches "
                                "(one per kernel)" % (n_pairs, len(runs))),
                   "quadrature_points": points, "setup_s": t_setup,
                   "bsr": {"blocks": int(nnzb), "ms": bsr_ms, "bytes": int(bsr_bytes),
                           "ms_default_shape": bsr_ms_default,
                           "tuned_shape": {"lanes_per_row": bsr_shape[0],
                                           "ctas_per_sm": bsr_shape[1]},
                           "achieved_gbs": bsr_bytes / (bsr_ms * 1e-3) / 1e9,
                           "blocks_per_s": nnzb / (bsr_ms * 1e-3), "hbm_peak_gbs": hbm},
                   "l2": "inputs larger than L2 (blocks %.0f MB per step)" % (n_pairs * 648 / 1e6),
                   "parallelism": "replicas"},
        "roofline": {"kernel": "pairs_batched<double, K> (all kernels of the step)",
                     "bound": "fp64", "achieved": achieved, "peak": peak64, "unit": "TFLOP/s",
                     "frac": achieved / peak64, "traffic": None,
                     "peak_source": "measured live: FP64 FMA probe (tct_fp64_fma_probe)",
                     "algorithmic": "%.3e flops per step = %.3e quadrature points x per-kernel "
                                    "point flops" % (flops, points)},
        "e2e": {"value": n_pairs / t_e2e, "unit": "pairs/s",
                "h2d_bytes_per_step": int(sum(g["recs"].nbytes for g in groups.values())),
                "d2h_bytes_per_step": int(n_pairs * 81 * 8),
                "api": "PairsIntegrator.batched(records, rule_ids, rules, nu ids, params) -> "
                       "numpy blocks, per kernel"},
        "gpu_launches": args.steps * len(runs),
        "clocks": clocks,
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_pairs_baseline(P, T, groups, flops)
    print(json.dumps(line), flush=True)


def run_panel_workload(args, rank, world, torch, dist):
    """C2 farfield (elasticRH3, or elasticRT3 with --panel-kernel) applied to
    a panel of R right-hand sides on the tensor cores."""
    from tectosaur_b200.ops.sparse_farfield_op import TriToTriDirectFarfieldOp
    R = args.rhs
    K = args.panel_kernel
    pts, tris = c2_mesh(args.grid or 174)
    n = tris.shape[0]
    idx = np.arange(n)
    op = TriToTriDirectFarfieldOp(NQ["nq_far"], K, PARAMS, pts, tris, np.float32, idx, idx)
    X = torch.from_numpy(np.random.default_rng(3 + rank).standard_normal((R, 9 * n))
                         .astype(np.float32)).cuda()
    Y = torch.empty((R, 9 * n), dtype=torch.float32, device="cuda")
    for _ in range(args.warmup):
        op.dot_panel_device(X, Y)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    sampler.start()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    for _ in range(args.steps):
        op.dot_panel_device(X, Y)
    b.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    total_ms = a.elapsed_time(b)
    if dist is not None:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms = total_ms / args.steps
    errs = [int(op.panel_error(16))]
    # the single-vector path on the same mesh, and the panel's error against it
    y1 = torch.empty(9 * n, dtype=torch.float32, device="cuda")
    for _ in range(3):
        op.dot_device(X[0].contiguous(), y1)
    torch.cuda.synchronize()
    c = torch.cuda.Event(enable_timing=True)
    d = torch.cuda.Event(enable_timing=True)
    c.record()
    for _ in range(5):
        op.dot_device(X[0].contiguous(), y1)
    d.record()
    torch.cuda.synchronize()
    single_ms = c.elapsed_time(d) / 5
    rel = []
    for r in sorted({0, R // 2, R - 1}):
        op.dot_device(X[r].contiguous(), y1)
        rel.append(float(torch.linalg.norm(Y[r] - y1) / torch.linalg.norm(y1)))
    # e2e: host panel in, host panel out
    Xh = X.cpu().numpy()
    op.dot_panel(Xh)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(max(1, min(args.steps, 3))):
        Yh = op.dot_panel(Xh)
    t_e2e = (time.perf_counter() - t0) / max(1, min(args.steps, 3))
    if rank != 0:
        return
    # executed tensor work: per panel of width w, 3 split-TF32 products of
    # RH: (n_obs padded to 128) x (7 n_src padded to 56) x 9w;
    # RT: (3 n_obs points padded to 128) x (10 n_src padded to 40) x 3w
    widths, r0 = [], 0
    while r0 < R:
        widths.append(16)
        r0 += 16
    if K == "elasticRT3":
        n_obs_p = (3 * n + 127) // 128 * 128
        n_src_p = (n + 3) // 4 * 4
        mma_flops = sum(3 * 2.0 * n_obs_p * 10 * n_src_p * 3 * w for w in widths)
        kname, b_mb = "rt_main (tcgen05.mma kind::tf32, A in tensor memory, split TF32)", \
            n_src_p * 10 * 3 * 16 * 8 / 1e6
    else:
        n_obs_p = (n + 127) // 128 * 128
        n_src_p = (n + 7) // 8 * 8
        mma_flops = sum(3 * 2.0 * n_obs_p * 7 * n_src_p * 9 * w for w in widths)
        kname, b_mb = "mrhs_main<R> (tcgen05.mma kind::tf32, split TF32)", \
            n_src_p * 7 * 9 * 16 * 8 / 1e6
    mp = measured_peaks()
    bf16 = mp.get("bf16_tflops") if mp else 1590.0
    tf32_peak = bf16 / 2.0
    achieved = mma_flops / (ms * 1e-3) / 1e12
    line = {
        "metric": "farfield vector applies/s (multi-RHS panel, tensor cores)",
        "value": world * R / (ms * 1e-3), "unit": "vector applies/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded mesh and inputs)",
        "config": {"workload": ("direct farfield of the 60k-triangle topographic surface "
                                "(%s, 3-point rule) applied to a panel of %d N(0, 1) "
                                "vectors: kernel scalars on the CUDA cores, contraction with "
                                "the panel by split-TF32 tcgen05.mma (panels of %s)"
                                % (K, R, "+".join(str(w) for w in widths))),
                   "kernel": K,
                   "n_tris": int(n), "rhs": R, "single_vector_ms": single_ms,
                   "speedup_vs_single_vector": single_ms * R / ms,
                   "rel_err_vs_single_vector_fp32": rel, "error_words": errs,
                   "l2": "inputs larger than L2 (panel B operand %.0f MB)" % b_mb,
                   "parallelism": "replicas"},
        "roofline": {"kernel": kname,
                     "bound": "tensor", "achieved": achieved, "peak": tf32_peak,
                     "unit": "TFLOP/s", "frac": achieved / tf32_peak, "traffic": None,
                     "peak_source": "TF32 dense = half of the measured BF16 GEMM rate "
                                    "(MEASURED_PEAKS.json bf16_tflops %.0f)" % bf16,
                     "algorithmic": "%.3e tensor flops per panel apply (3 split products)"
                                    % mma_flops},
        "e2e": {"value": R / t_e2e, "unit": "vector applies/s",
                "h2d_bytes_per_step": int(Xh.nbytes), "d2h_bytes_per_step": int(Yh.nbytes),
                "api": "TriToTriDirectFarfieldOp.dot_panel(numpy (R, 9n)) -> numpy"},
        "gpu_launches": args.steps * len(widths) * 4,
        "clocks": clocks,
    }
    if not args.no_cpu_baseline:
        cb = cpu_direct_far_baseline(pts, tris, K=K)
        cb["unit"] = "vector applies/s"
        line["cpu_baseline"] = cb
    print(json.dumps(line), flush=True)


def c2_point_form(n=174):
    """The 60k-triangle surface's 3-point-rule quadrature points (179,574)
    with their triangle normals: the point form of the C2 configuration."""
    from tectosaur_b200.util.quadrature import gauss2d_tri
    pts, tris = c2_mesh(n)
    q, _ = gauss2d_tri(NQ["nq_far"])
    tp = pts[tris]
    b = np.stack([1 - q[:, 0] - q[:, 1], q[:, 0], q[:, 1]], axis=1)   # (nq, 3)
    P = np.einsum("qb,tbd->tqd", b, tp).reshape(-1, 3)
    nrm = np.cross(tp[:, 2] - tp[:, 0], tp[:, 2] - tp[:, 1])
    nrm /= np.linalg.norm(nrm, axis=1)[:, None]
    Nn = np.repeat(nrm, q.shape[0], axis=0)
    return P, Nn


def run_ptspanel_workload(args, rank, world, torch, dist):
    """The C2 point form (179,574 quadrature points of the 60k-triangle
    surface, elasticT3 and elasticH3) on a panel of R weight vectors on the
    tensor cores, against the single-vector point kernel and the FP64
    oracle on sampled rows."""
    from tectosaur_b200 import _lib
    from tectosaur_b200.farfield import farfield_pts_panel_device
    R = args.rhs
    P, Nn = c2_point_form(args.grid or 174)
    n = P.shape[0]
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    op, on = dev(P), dev(Nn)
    W = dev(np.random.default_rng(3 + rank).standard_normal((R, 3 * n)))
    Y = torch.empty((R, 3 * n), dtype=torch.float32, device="cuda")
    res = {}
    for K in ("elasticH3", "elasticT3"):
        for _ in range(args.warmup):
            farfield_pts_panel_device(K, op, on, op, on, W, PARAMS, out=Y)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.steps):
            farfield_pts_panel_device(K, op, on, op, on, W, PARAMS, out=Y)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / args.steps
        # the single-vector kernel
        y1 = torch.empty(3 * n, dtype=torch.float32, device="cuda")
        params = np.ascontiguousarray(PARAMS, np.float64)
        kid = _lib.kernel_id(K)

        def single(r):
            _lib.check(_lib.lib.tct_farfield_pts(
                kid, _lib.TCT_F32, _lib.tptr(y1), _lib.tptr(op), _lib.tptr(on), n,
                _lib.tptr(op), _lib.tptr(on), n, _lib.tptr(W[r]), _lib.dptr(params),
                _lib.stream_ptr()), "tct_farfield_pts")
        single(0)
        torch.cuda.synchronize()
        c = torch.cuda.Event(enable_timing=True)
        d = torch.cuda.Event(enable_timing=True)
        c.record()
        for _ in range(3):
            single(0)
        d.record()
        torch.cuda.synchronize()
        single_ms = c.elapsed_time(d) / 3
        # FP64 oracle on 256 seeded observation points, columns 0 and R - 1
        from oracle import oracle as orc
        rows = np.sort(np.random.default_rng(19).choice(n, 256, replace=False))
        Wh = W.cpu().numpy().astype(np.float64)
        Yh = Y.cpu().numpy()
        errs = []
        for r in (0, R - 1):
            want = orc.farfield_pts(K, np.float64, P[rows], Nn[rows], P, Nn, Wh[r], PARAMS)
            got = Yh[r].reshape(-1, 3)[rows].reshape(-1)
            errs.append(float(np.linalg.norm(got - want) / np.linalg.norm(want)))
            if r == 0:
                # the single-vector FP32 kernel on the same rows, for scale
                single(0)
                s1 = y1.cpu().numpy().reshape(-1, 3)[rows].reshape(-1)
                err_single = float(np.linalg.norm(s1 - want) / np.linalg.norm(want))
                err_vs_single = float(np.linalg.norm(got - s1) / np.linalg.norm(s1))
        n_pad_o = (n + 127) // 128 * 128
        n_pad_s = (n + 7) // 8 * 8
        panels = (R + 15) // 16
        mma_flops = panels * 3 * 2.0 * n_pad_o * 9 * n_pad_s * 48
        res[K] = {"ms_per_panel_apply": ms, "vector_applies_per_s": R / (ms * 1e-3),
                  "single_vector_ms": single_ms, "speedup_vs_single_vector": single_ms * R / ms,
                  "rel_err_fp64_oracle_256_rows": errs,
                  "single_vector_fp32_rel_err_fp64_oracle": err_single,
                  "rel_diff_vs_single_vector_fp32": err_vs_single,
                  "tensor_tflops_executed": mma_flops / (ms * 1e-3) / 1e12}
    if rank != 0:
        return
    mp = measured_peaks()
    bf16 = mp.get("bf16_tflops") if mp else 1590.0
    tf32_peak = bf16 / 2.0
    hv = res["elasticH3"]
    line = {
        "metric": "point farfield vector applies/s (multi-RHS panel, tensor cores)",
        "value": world * hv["vector_applies_per_s"], "unit": "vector applies/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": hv["ms_per_panel_apply"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded mesh and weights)",
        "config": {"workload": ("point form of the 60k-triangle surface: %d quadrature points "
                                "(3-point rule) with their triangle normals, all-pairs "
                                "elasticH3 / elasticT3 on a panel of %d N(0, 1) weight vectors "
                                "(tct_farfield_pts_panel)" % (n, R)),
                   "n_points": int(n), "rhs": R, "kernels": res, "parallelism": "replicas"},
        "roofline": {"kernel": "pts_panel_main<elasticH3> (tcgen05.mma kind::tf32)",
                     "bound": "tensor", "achieved": hv["tensor_tflops_executed"],
                     "peak": tf32_peak, "unit": "TFLOP/s",
                     "frac": hv["tensor_tflops_executed"] / tf32_peak, "traffic": None,
                     "peak_source": "TF32 dense = half of the measured BF16 GEMM rate"},
        "gpu_launches": args.steps * ((R + 15) // 16) * 4,
    }
    print(json.dumps(line), flush=True)


def run_batch_workload(args, rank, world, torch, dist):
    """Batched mixed-precision solves against the plain FP64 one-at-a-time
    solve on the 722-triangle configuration."""
    import tectosaur_b200 as tct
    from tectosaur_b200.ops.sparse_farfield_op import TriToTriDirectFarfieldOp
    from tectosaur_b200.simple_solver import (free_edge_vertices, iterative_solve,
                                              iterative_solve_batch, shared_vertex_matrix)
    tol = 1e-8
    R = args.rhs if args.rhs != 64 else 16
    if args.grid is None:
        pts, tris = c1_mesh()
    else:
        from tectosaur_b200.mesh.mesh_gen import make_rect
        g = args.grid
        pts, tris = make_rect(g, g, [[-1, -1, 0], [-1, 1, 0], [1, 1, 0], [1, -1, 0]])
    n = tris.shape[0]
    op64 = tct.RegularizedSparseIntegralOp(*C1_NQ, K_NAME, K_NAME, PARAMS, pts, tris,
                                           np.float64, TriToTriDirectFarfieldOp)
    op32 = tct.RegularizedSparseIntegralOp(*C1_NQ, K_NAME, K_NAME, PARAMS, pts, tris,
                                           np.float32, TriToTriDirectFarfieldOp)
    cm = shared_vertex_matrix(tris, fixed_vertices=free_edge_vertices(tris))
    rhs = np.random.default_rng(1 + rank).standard_normal((R, 9 * n))
    rhs_d = torch.from_numpy(rhs).cuda()
    for _ in range(args.warmup):
        iterative_solve_batch(op64, op32, cm, rhs_d, tol=tol)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    sampler.start()
    lat = []
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    for _ in range(args.steps):
        t0 = time.perf_counter()
        U = iterative_solve_batch(op64, op32, cm, rhs_d, tol=tol)
        lat.append(time.perf_counter() - t0)
    b.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    total_ms = a.elapsed_time(b)
    if dist is not None:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    hist = iterative_solve_batch.last
    # the plain path: FP64 operator, one solve at a time, same right-hand sides
    iterative_solve(op64, cm, rhs[0], cfg=dict(solver_tol=tol))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    U64 = [iterative_solve(op64, cm, rhs[r], cfg=dict(solver_tol=tol)) for r in range(R)]
    t_plain = time.perf_counter() - t0
    err = max(float(np.linalg.norm(U[r] - U64[r]) / np.linalg.norm(U64[r])) for r in range(R))
    if rank != 0:
        return
    ms = total_ms / args.steps
    value = world * R * args.steps / (total_ms * 1e-3)
    line = {
        "metric": "BEM solves/s: batched mixed precision (served) vs plain FP64",
        "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 tensor-core farfield panel + f64 refinement",
        "data": "synthetic (seeded mesh and right-hand sides)",
        "config": {"workload": ("%d seeded N(0, 1) tractions on the %d-triangle planar fault "
                                "(make_rect over [-1, 1]^2, elasticRH3, continuity + free "
                                "edges) solved together: batched GMRES on the FP32 operator "
                                "(farfield as one tensor-core panel apply and nearfield as one "
                                "BSR panel launch per step) inside FP64 iterative refinement "
                                "to 1e-8 FP64 residual" % (R, n)),
                   "n_tris": int(n),
                   "rhs_per_batch": R, "plain_fp64_solves_per_s": R / t_plain,
                   "speedup_vs_plain": value / (R / t_plain),
                   "max_rel_diff_vs_plain_fp64": err,
                   "refinement_gmres_steps": hist["gmres_steps"],
                   "refinement_residuals": hist["residuals"],
                   "batch_latency_ms_p50": 1e3 * float(np.percentile(lat, 50)),
                   "batch_latency_ms_p99": 1e3 * float(np.percentile(lat, 99)),
                   "l2": "small problem: working set in L2 (latency-bound solve)",
                   "parallelism": "replicas"},
        "roofline": {"kernel": "whole batched solve (launch- and sync-bound at this size)",
                     "bound": "hbm", "achieved": None, "peak": None, "unit": "GB/s",
                     "frac": None, "traffic": None},
        "e2e": {"value": value, "unit": "solves/s",
                "h2d_bytes_per_step": int(rhs.nbytes), "d2h_bytes_per_step": int(U.nbytes),
                "api": "simple_solver.iterative_solve_batch(op64, op32, cm, rhs panel) -> numpy"},
        "gpu_launches": None,
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def qd_mesh(n=25):
    """The reference's quasidynamic example fault: make_rect(25, 25) over a
    2 x 2 vertical square (1,152 triangles)."""
    from tectosaur_b200.mesh.mesh_gen import make_rect
    return make_rect(n, n, [[-1, 0, 1], [-1, 0, -1], [1, 0, -1], [1, 0, 1]])


def qd_config(n_tris, float_type=np.float32):
    """The configuration of the reference's quasidynamic example run
    (shear modulus 3e10, density 2670, a 0.010, b 0.015, Dc 2e-6, f0 0.6,
    V0 1e-6, plate rate 1e-9, 50 MPa normal stress, time-step tolerance 1e-4,
    the 722-triangle plain method's operator rules, mass rule order 4)."""
    return dict(sm=3e10, pr=0.25, density=2670.0, Dc=2e-6, f0=0.6, V0=1e-6,
                a=np.full(n_tris * 3, 0.010), b=np.full(n_tris * 3, 0.015), plate_rate=1e-9,
                additional_normal_stress=50e6, timestep_tol=1e-4,
                tectosaur_cfg=dict(quad_coincident_order=6, quad_edgeadj_order=6,
                                   quad_vertadj_order=6, quad_near_order=5,
                                   quad_near_threshold=2.5, quad_far_order=2, quad_mass_order=4,
                                   float_type=float_type, use_fmm=False))


def qd_initial(n_tris, seed=9):
    """Zero slip, state 0.7 with a seeded perturbation (which perturbs the
    initial slip rate)."""
    rng = np.random.default_rng(seed)
    return np.concatenate([np.zeros(9 * n_tris), 0.7 + 0.01 * rng.standard_normal(3 * n_tris)])


def cpu_qd_baseline(pts, tris, cfg, y0, n_steps):
    """The oracle (qd_oracle.FullspaceModel: oracle operator composition,
    scipy cg, the rate-state Newton restatement) stepped by scipy's RK23,
    as the reference's Integrator does; nearfield blocks integrated before
    the timing."""
    from scipy.integrate import RK23
    from oracle import qd_oracle
    from tectosaur_b200.ops.mass_op import MassOp, unscaled_normals
    from tectosaur_b200.qd.model import edge_ones_interior
    from tectosaur_b200.simple_solver import free_edge_vertices, shared_vertex_matrix
    import scipy.sparse
    op = cfg["tectosaur_cfg"]
    H = qd_oracle.sparse_op(op["quad_coincident_order"], op["quad_edgeadj_order"],
                            op["quad_vertadj_order"], op["quad_far_order"],
                            op["quad_near_order"], op["quad_near_threshold"], "elasticRH3",
                            [1.0, cfg["pr"]], pts, tris, op["float_type"])
    ones = edge_ones_interior(tris)
    cm_edges = scipy.sparse.diags(ones).tocsc()[:, ones > 0]
    cm = shared_vertex_matrix(tris, fixed_vertices=free_edge_vertices(tris))
    un = unscaled_normals(pts[tris])
    normals = un / np.linalg.norm(un, axis=1)[:, None]
    om = qd_oracle.FullspaceModel(pts, tris, cfg, H, MassOp(4, pts, tris).mat, cm, cm_edges,
                                  normals)
    rk = RK23(om.derivs, 0.0, y0, 1e50, atol=cfg["timestep_tol"], rtol=cfg["timestep_tol"])
    rk.h_abs = 365.25 * 24 * 3600 / 10.0
    t0 = time.perf_counter()
    for _ in range(n_steps):
        rk.step()
    dt = time.perf_counter() - t0
    return {"value": n_steps / dt, "unit": "qd steps/s", "cores": os.cpu_count() or 1,
            "kind": "port",
            "sample": ("%d RK23 steps of the oracle model (oracle operator, scipy cg, Newton "
                       "restatement) from the same initial state, %.1f s" % (n_steps, dt))}


def run_qd_workload(args, rank, world, torch, dist):
    """Quasidynamic rate-and-state time stepping of the reference's example
    fault, the whole state on the device."""
    from tectosaur_b200 import _lib, qd
    pts, tris = qd_mesh()
    n = tris.shape[0]
    cfg = qd_config(n)
    t_build = time.perf_counter()
    model = qd.FullspaceModel((pts, tris), cfg)
    torch.cuda.synchronize()
    t_build = time.perf_counter() - t_build
    y0 = qd_initial(n, seed=9 + rank)
    n_steps = args.qd_steps

    def run():
        integ = qd.Integrator(model, (0.0, y0))
        integ.integrate(n_steps)
        y_end = integ.h_y[-1].cpu().numpy()
        return integ, y_end

    for _ in range(args.warmup):
        run()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    sampler.start()
    l0 = _lib.launch_count() + model.graph_kernel_launches
    e0 = model.n_evals
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    for _ in range(args.steps):
        integ, y_end = run()
    b.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    # the derivative runs as a replayed CUDA graph: its library kernels are
    # counted per replay (FullspaceModel.graph_kernel_launches)
    launches = _lib.launch_count() + model.graph_kernel_launches - l0
    evals = (model.n_evals - e0) / args.steps
    total_ms = a.elapsed_time(b)
    if dist is not None:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * n_steps * args.steps / (total_ms * 1e-3)
    if rank != 0:
        return
    line = {
        "metric": "quasidynamic time steps/s (RK23 with rate-state friction, device-resident)",
        "value": value, "unit": "qd steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 state, f32 elastic operator", "data": "synthetic (seeded initial state)",
        "config": {"workload": ("%d RK23 steps (one bench step = the whole integration from "
                                "the seeded state) of the reference's quasidynamic example: "
                                "make_rect(25, 25) vertical fault, %d triangles, elasticRH3 "
                                "RegularizedSparseIntegralOp(6,6,6,2,5,2.5) FP32, mass order 4, "
                                "a 0.010, b 0.015, Dc 2e-6, V0 1e-6, timestep_tol 1e-4"
                                % (n_steps, n)),
                   "n_tris": n, "qd_steps": n_steps, "rejected_steps": integ.rk23.n_rejected,
                   "derivs_per_run": evals, "t_end_years": integ.h_t[-1] / qd.siay,
                   "last_cg_iterations": model.last_cg_iterations,
                   "newton_failures": model.newton_failures(),
                   "model_build_s": t_build, "l2": "small problem: working set in L2",
                   "parallelism": "replicas"},
        "roofline": {"kernel": "whole stepper (latency-bound at this size)", "bound": "hbm",
                     "achieved": None, "peak": None, "unit": "GB/s", "frac": None,
                     "traffic": None},
        "e2e": {"value": value, "unit": "qd steps/s", "h2d_bytes_per_step": int(y0.nbytes),
                "d2h_bytes_per_step": int(y_end.nbytes),
                "api": "qd.Integrator(model, (0, y0 numpy)).integrate(n); h_y[-1] -> numpy"},
        "gpu_launches": int(launches // args.steps),
        "clocks": clocks,
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_qd_baseline(pts, tris, cfg, y0, 3)
    print(json.dumps(line), flush=True)


def c4_free_surface_problem(pts, tris, n_surf):
    """The C4 free-surface problem: surface displacement unknown (continuity,
    held at zero on the surface's outer edges), fault slip prescribed (unit
    thrust slip up dip: (0, cos 30, -sin 30) in the fault's dip plane).
    Returns (cm, c_rhs) as examples/solve.py:iterative_solve uses them: the
    solution is cm x + c_rhs."""
    from tectosaur_b200.simple_solver import free_edge_vertices, shared_vertex_matrix
    n = tris.shape[0]
    fixed = np.concatenate([free_edge_vertices(tris[:n_surf]), np.unique(tris[n_surf:])])
    cm = shared_vertex_matrix(tris, fixed_vertices=fixed)
    slip = np.zeros((n, 3, 3))
    slip[n_surf:, :, 1] = np.cos(np.radians(30.0))
    slip[n_surf:, :, 2] = -np.sin(np.radians(30.0))
    return cm, slip.reshape(-1)


def run_c4solve_workload(args, rank, world, torch, dist):
    """The FMM-accelerated free-surface solve of the 1M-triangle C4 mesh:
    GMRES on the FP32 operator (FMM farfield, order 8, mac 3, 128 triangles
    per leaf) inside FP64-residual iterative refinement to 1e-6, against the
    plain FP64 GMRES solve."""
    import tectosaur_b200 as tct
    from tectosaur_b200 import _lib
    from tectosaur_b200.fmm.tsfmm import FMMFarfieldOp
    from tectosaur_b200.simple_solver import iterative_solve, iterative_solve_batch
    tol = 1e-6
    grid = args.grid or 707
    pts, tris = c4_mesh(grid)
    n = tris.shape[0]
    n_surf = (grid - 1) ** 2 * 2
    cfg = dict(FMM_CFG)
    if args.fmm_order:
        cfg["order"] = args.fmm_order
    t0 = time.perf_counter()
    op64 = tct.RegularizedSparseIntegralOp(*[NQ[k] for k in ("nq_co", "nq_ea", "nq_va",
                                                               "nq_far", "nq_near", "thr")],
                                           K_NAME, K_NAME, PARAMS, pts, tris, np.float64,
                                           FMMFarfieldOp(cfg["mac"], cfg["pts_per_cell"],
                                                         cfg["order"], mode=cfg["mode"]),
                                           keep_uncorrected=False)
    op32 = op64.astype(np.float32, keep_uncorrected=False)
    torch.cuda.synchronize()
    t_build = time.perf_counter() - t0
    cm, c_rhs = c4_free_surface_problem(pts, tris, n_surf)
    rhs = -op64.dot(c_rhs)
    mem_gb = torch.cuda.memory_allocated() / 1e9

    def solve():
        return iterative_solve_batch(op64, op32, cm, rhs[None, :], tol=tol, restart=200)[0]

    for _ in range(args.warmup):
        solve()
    torch.cuda.synchronize()
    sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    sampler.start()
    l0 = _lib.launch_count()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    for _ in range(args.steps):
        u = solve()
    b.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    hist = iterative_solve_batch.last
    launches = (_lib.launch_count() - l0) // args.steps
    ms = a.elapsed_time(b) / args.steps
    value = world / (ms * 1e-3)
    # the plain path: FP64 GMRES on the FP64 operator, one solve
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    u64 = iterative_solve(op64, cm, rhs, cfg=dict(solver_tol=tol))
    t_plain = time.perf_counter() - t1
    plain_steps = iterative_solve.last["n_iter"]
    diff = float(np.linalg.norm(u - u64) / np.linalg.norm(u64))
    # error of the FMM operator against the direct FP64 farfield (the
    # reference's CPU-runnable algorithm, parity-pinned to the oracle) on
    # 1,024 seeded observation rows: on a random vector, and on the solution
    # itself (the extra residual the solution has under the direct operator)
    from tectosaur_b200.ops.sparse_farfield_op import TriToTriDirectFarfieldOp
    rows = np.sort(np.random.default_rng(41).choice(n, 1024, replace=False))
    direct = TriToTriDirectFarfieldOp(NQ["nq_far"], K_NAME, PARAMS, pts, tris, np.float64, rows,
                                      np.arange(n))
    xr = np.random.default_rng(42).standard_normal(9 * n)

    def rows_of(v):
        return np.asarray(v).reshape(-1, 9)[rows].reshape(-1)
    dref = direct.dot(xr)
    fmm_err = float(np.linalg.norm(rows_of(op64.farfield.dot(xr)) - dref) / np.linalg.norm(dref))
    fmm32_err = float(np.linalg.norm(rows_of(op32.farfield.dot(xr.astype(np.float32))) - dref) /
                      np.linalg.norm(dref))
    du = direct.dot(u)
    sol_err = float(np.linalg.norm(rows_of(op64.farfield.dot(u)) - du) /
                    np.linalg.norm(rows_of(op64.dot(u))))
    # matvec timings (device)
    x32 = torch.randn(9 * n, device="cuda")
    y32 = torch.empty_like(x32)
    op32.dot_device(x32, y32)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    op32.dot_device(x32, y32)
    torch.cuda.synchronize()
    t_mv32 = time.perf_counter() - t2
    if rank != 0:
        return
    line = {
        "metric": "BEM solves/s: FMM solve, FP32 GMRES + FP64 refinement vs plain FP64",
        "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 operator + f64 refinement",
        "data": "synthetic (seeded hills; prescribed uniform fault slip)",
        "config": {"workload": ("free-surface displacement solve of the C4 mesh (%d x %d "
                                "topographic surface over [-50, 50]^2 with three seeded hills "
                                "+ a 30-degree dipping 20 x 10 thrust fault, %d triangles): "
                                "surface DOFs unknown (continuity, zero on the outer edges), "
                                "unit thrust slip prescribed on the fault; elasticRH3 "
                                "RegularizedSparseIntegralOp(6,6,6,1,5,2.5) with the FMM "
                                "farfield (order %d, mac 3, 128 per leaf); FP32 GMRES inside "
                                "FP64-residual refinement to 1e-6" % (grid, grid, n,
                                                                      cfg["order"])),
                   "n_tris": n, "n_free": int(cm.shape[1]),
                   "nearfield_blocks": int(op64.nearfield.bsr.nnzb),
                   "gmres_steps": hist["gmres_steps"], "residuals": hist["residuals"],
                   "plain_fp64_solves_per_s": 1.0 / t_plain,
                   "plain_fp64_gmres_steps": int(plain_steps),
                   "speedup_vs_plain": value / (1.0 / t_plain),
                   "rel_diff_vs_plain_fp64": diff, "fp32_matvec_s": t_mv32,
                   "fmm_order": cfg["order"],
                   "fmm_fp64_rel_err_vs_direct_fp64": fmm_err,
                   "fmm_fp32_rel_err_vs_direct_fp64": fmm32_err,
                   "solution_apply_rel_err_fmm_vs_direct_fp64": sol_err,
                   "error_rows": "1,024 seeded observation rows, direct FP64 farfield",
                   "build_s": t_build, "hbm_gb": mem_gb,
                   "l2": "operator of %.0f GB (FP64 + FP32 nearfield blocks), beyond L2"
                         % mem_gb,
                   "parallelism": "replicas"},
        "roofline": {"kernel": "whole solve (FMM matvecs: see the fmm workload)",
                     "bound": "fp32", "achieved": None, "peak": None, "unit": "TFLOP/s",
                     "frac": None, "traffic": None},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": int(rhs.nbytes),
                "d2h_bytes_per_step": int(u.nbytes),
                "api": "simple_solver.iterative_solve_batch(op64, op32, cm, rhs) -> numpy"},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if not args.no_cpu_baseline:
        cb = cpu_direct_far_baseline(pts, tris, target_s=10.0)
        steps = sum(hist["gmres_steps"])
        cb = dict(cb, value=cb["value"] / max(steps, 1), unit="solves/s",
                  sample=cb["sample"] + "; one solve = %d such applies" % steps)
        line["cpu_baseline"] = cb
    print(json.dumps(line), flush=True)


def run_near_workload(args, rank, world, torch, dist):
    """Near-pair search of the C4 mesh (1,016,894 triangles, threshold 2.5,
    the operator build's first step): get_nearfield_device (octrees, dual
    traversal to leaf pairs, ball tests, row fill and row sort, all on the
    device) against the host search; both give the reference's pair set in
    (obs, src) order.  The host-built plan (host octrees and traversal) is
    timed beside it."""
    from tectosaur_b200 import _lib
    from tectosaur_b200.mesh import find_near_adj as fna
    pts, tris = c4_mesh(args.grid or 707)
    c, r = fna.get_tri_centroids_rs(pts, tris)
    thr = 2.5
    for _ in range(max(1, min(args.warmup, 2))):
        out = fna.get_nearfield_device(c, r, c, r, thr)
    torch.cuda.synchronize()
    sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    sampler.start()
    l0 = _lib.launch_count()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        out = fna.get_nearfield_device(c, r, c, r, thr)
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / args.steps
    clocks = sampler.stop()
    launches = (_lib.launch_count() - l0) // args.steps
    n_pairs = int(out.shape[0])
    t0 = time.perf_counter()
    host_out = out.cpu().numpy()
    d2h = time.perf_counter() - t0
    # the plans alone: octrees + traversal to leaf pairs on the host, and on
    # the device
    t0 = time.perf_counter()
    h = fna.near_plan(c, r, c, r, thr)
    t_plan = time.perf_counter() - t0
    n_leaf_pairs = int(_lib.lib.tct_near_plan_leaf_pairs(h))
    _lib.lib.tct_near_plan_free(h)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    h = fna.near_plan(c, r, c, r, thr, device_tree=True)
    torch.cuda.synchronize()
    t_plan_dev = time.perf_counter() - t0
    _lib.lib.tct_near_plan_free(h)
    # the whole search with the host-built plan
    t0 = time.perf_counter()
    out_h = fna.get_nearfield_device(c, r, c, r, thr, device_tree=False)
    torch.cuda.synchronize()
    t_hostplan = time.perf_counter() - t0
    same_plans = bool(torch.equal(out_h, out))
    del out_h
    if rank != 0:
        return
    line = {
        "metric": "near-pair search pairs/s (get_nearfield, C4 mesh)",
        "value": world * n_pairs / dt, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 tests, int64 pairs",
        "data": "synthetic (seeded hills)",
        "config": {"workload": ("near pairs of the C4 mesh (%d triangles), threshold %.1f: "
                                "octrees, traversal to leaf pairs, tests, fill and per-row "
                                "sort on the device" % (tris.shape[0], thr)),
                   "n_tris": int(tris.shape[0]), "pairs": n_pairs,
                   "leaf_pairs": n_leaf_pairs, "host_plan_s": t_plan,
                   "device_plan_s": t_plan_dev,
                   "search_with_host_plan_s": t_hostplan,
                   "device_plan_equals_host_plan_output": same_plans,
                   "timing": "wall clock (host phases included)", "parallelism": "replicas",
                   "l2": "inputs and pair arrays larger than L2"},
        "roofline": {"kernel": "near_count / near_fill (ball tests)", "bound": "fp64",
                     "achieved": None, "peak": None, "unit": "TFLOP/s", "frac": None,
                     "traffic": None},
        "e2e": {"value": world * n_pairs / (dt + d2h), "unit": "pairs/s",
                "h2d_bytes_per_step": int(c.nbytes + r.nbytes),
                "d2h_bytes_per_step": int(host_out.nbytes),
                "api": "get_nearfield_device(numpy) -> torch, then .cpu()"},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if not args.no_cpu_baseline:
        t0 = time.perf_counter()
        ref = fna.get_nearfield(c, r, c, r, thr)
        th = time.perf_counter() - t0
        line["cpu_baseline"] = {
            "value": ref.shape[0] / th, "unit": "pairs/s", "cores": os.cpu_count() or 1,
            "kind": "port",
            "sample": "the whole search once with the host restatement (tct_find_near_pairs, "
                      "OpenMP on all host threads, bit-exact with the reference's finder): "
                      "%.2f s; identical output: %s" % (th, bool(np.array_equal(ref, host_out)))}
    print(json.dumps(line), flush=True)


def run_interior_workload(args, rank, world, torch, dist):
    """Interior evaluation (InteriorOp.dot) on the reference's interior
    nearfield test configuration, scaled: a make_rect(n, n) fault in the
    z = 0 plane and a 50 x 50 grid of observation points on the y = 0 plane
    through it (tests/test_integral_op.py:219-248 of the reference)."""
    import tectosaur_b200 as tct
    from tectosaur_b200 import _lib
    from tectosaur_b200.util.quadrature import gauss2d_tri
    n = args.grid or 30
    src = tct.make_rect(n, n, [[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]])
    xs = np.linspace(-3, 3, 50)
    X, Z = np.meshgrid(xs, xs)
    obs = np.array([e.flatten() for e in [X, np.zeros_like(X), Z]]).T.copy()
    ns = np.zeros(obs.shape)
    ns[:, 2] = 1.0
    K, nq_vertex, nq_far, nq_near = "elasticT3", 8, 2, 5
    t_build = time.perf_counter()
    op = tct.InteriorOp(obs, ns, src, K, 4, nq_vertex, nq_far, nq_near, PARAMS, np.float32)
    torch.cuda.synchronize()
    t_build = time.perf_counter() - t_build
    v = np.zeros(src[1].shape[0] * 9)
    v.reshape((-1, 3))[:, 0] = 1.0
    vd = torch.from_numpy(v).cuda()
    y = torch.empty(op.shape[0], dtype=torch.float64, device="cuda")
    for _ in range(args.warmup):
        op.dot_device(vd, y)
    torch.cuda.synchronize()
    sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    sampler.start()
    l0 = _lib.launch_count()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    for _ in range(args.steps):
        op.dot_device(vd, y)
    b.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    launches = (_lib.launch_count() - l0) // args.steps
    ms = a.elapsed_time(b) / args.steps
    n_obs = obs.shape[0]
    value = world * n_obs / (ms * 1e-3)
    # e2e: host vector in, host values out
    op.dot(v)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        out = op.dot(v)
    e2e_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    # point-pair work of the farfield kernel (the dominant term)
    nq2 = gauss2d_tri(nq_far)[0].shape[0]
    pairs = n_obs * src[1].shape[0] * nq2
    if rank != 0:
        return
    line = {
        "metric": "interior evaluation points/s (InteriorOp.dot)",
        "value": value, "unit": "points/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 farfield, f64 pair terms", "data": "synthetic",
        "config": {"workload": ("InteriorOp(elasticT3, nq_vertex 8, nq_far 2, nq_near 5) of a "
                                "make_rect(%d, %d) fault (%d triangles) at a 50 x 50 grid of "
                                "points through it, the reference's interior nearfield test "
                                "case" % (n, n, src[1].shape[0])),
                   "n_obs": n_obs, "n_src_tris": int(src[1].shape[0]),
                   "near_pairs": int(op.near_pairs.shape[0]),
                   "vertex_pairs": int(op.vertex_pairs.shape[0]),
                   "point_pairs_per_apply": pairs, "build_s": t_build,
                   "l2": "small problem: working set in L2", "parallelism": "replicas"},
        "roofline": {"kernel": "pts_kernel (triangle-to-point farfield)", "bound": "fp32",
                     "achieved": None, "peak": None, "unit": "TFLOP/s", "frac": None,
                     "traffic": None},
        "e2e": {"value": world * n_obs / (e2e_ms * 1e-3), "unit": "points/s",
                "h2d_bytes_per_step": int(v.nbytes), "d2h_bytes_per_step": int(out.nbytes),
                "api": "InteriorOp.dot(numpy) -> numpy"},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if not args.no_cpu_baseline:
        from oracle import oracle as orc
        M = op.near_mat - op.near_mat_correction + op.vertex_mat
        reps, t0 = 0, time.perf_counter()
        while reps == 0 or time.perf_counter() - t0 < 2.0:
            orc.farfield_tris_to_pts(K, np.float32, gauss2d_tri(nq_far), obs, ns, src[0],
                                     src[1], v, PARAMS)
            M.dot(v)
            reps += 1
        dt = (time.perf_counter() - t0) / reps
        line["cpu_baseline"] = {
            "value": n_obs / dt, "unit": "points/s", "cores": os.cpu_count() or 1,
            "kind": "port",
            "sample": "the whole apply: oracle triangle-to-point farfield of all %d points "
                      "(FP32, all host threads) plus the pair terms' host sparse product, "
                      "%d repetitions, %.3f s each" % (n_obs, reps, dt)}
    print(json.dumps(line), flush=True)


# ---- C5: the served quasidynamic stream ----------------------------------------
C5_LO, C5_HI = 2_000, 200_000
C5_TOL = 1e-8             # FP64 residual of every solve request
C5_FMM_MIN = 60_000       # meshes from this size use the FMM farfield
C5_FMM = dict(mac=3.0, pts_per_cell=128, order=10, mode="fmm")
# the served FP32 correction operator of an FMM mesh: a lower order (its
# FP32 rounding floor, 1e-5 - 3e-5, is above the truncation error of order
# 6 anyway) and a correction tolerance above that floor
C5_INNER_ORDER = 6
C5_INNER_TOL_FMM = 1e-4
C5_SOLVES = (8, 6, 4, 3, 2, 2)   # solve requests per mesh, smallest mesh first
C5_QD_MESHES = 2                  # the smallest meshes (faults) also take qd requests
C5_QD_PER_MESH = 4


def c5_meshes(n_meshes=6, seed=6, lo=C5_LO, hi=C5_HI):
    """The served stream's meshes: one seeded log-uniform triangle count per
    equal log-width stratum of [lo, hi] (so the draw spans the range),
    kinds cycling through a vertical strike-slip fault, a 30-degree dipping
    fault and a topographic surface (Gaussian hill) with a dipping fault
    below it; 2 x 2 (nondimensional) patches."""
    from tectosaur_b200.mesh.mesh_gen import concat_no_dedupe, make_rect
    rng = np.random.default_rng(seed)
    edges = np.exp(np.linspace(np.log(lo), np.log(hi), n_meshes + 1))
    dip = np.radians(30.0)
    out = []
    for i in range(n_meshes):
        n_tris = float(np.exp(rng.uniform(np.log(edges[i]), np.log(edges[i + 1]))))
        kind = ("planar", "dipping", "topo")[i % 3]
        if kind == "planar":
            g = int(round(np.sqrt(n_tris / 2.0))) + 1
            pts, tris = make_rect(g, g, [[-1, 0, -1], [1, 0, -1], [1, 0, 1], [-1, 0, 1]])
        elif kind == "dipping":
            g = int(round(np.sqrt(n_tris / 2.0))) + 1
            pts, tris = make_rect(g, g, [[-1, 0, 0], [1, 0, 0],
                                         [1, 2 * np.cos(dip), -2 * np.sin(dip)],
                                         [-1, 2 * np.cos(dip), -2 * np.sin(dip)]])
        else:
            gs = int(round(np.sqrt(0.75 * n_tris / 2.0))) + 1
            gf = int(round(np.sqrt(0.25 * n_tris / 2.0))) + 1
            sp, st = make_rect(gs, gs, [[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]])
            sp = sp.copy()
            amp, w = rng.uniform(0.1, 0.3), rng.uniform(0.3, 0.6)
            sp[:, 2] = amp * np.exp(-(sp[:, 0] ** 2 + sp[:, 1] ** 2) / (2 * w * w))
            z0, y1 = -0.1, np.cos(dip)
            fp, ft = make_rect(gf, gf, [[-0.5, -0.5, z0], [0.5, -0.5, z0],
                                        [0.5, -0.5 + y1, z0 - np.sin(dip)],
                                        [-0.5, -0.5 + y1, z0 - np.sin(dip)]])
            pts, tris = concat_no_dedupe((sp, st), (fp, ft))
        out.append(("%s-%d" % (kind, tris.shape[0]), np.asarray(pts), np.asarray(tris), kind))
    return out


def c5_stream(torch, quiet=True, seed=7, inner="fmm-low"):
    """Serve the C5 stream (module-level C5_* settings) and time it against
    the plain paths.  Returns a dict of results (no JSON printing).

    Requests: C5_SOLVES[i] traction solves (seeded N(0, 1) right-hand sides,
    FP64 residual C5_TOL, continuity + free-edge constraints) on mesh i, and
    C5_QD_PER_MESH quasidynamic requests (200 RK23 steps of rate-and-state
    friction, a 0.010, b 0.015, Dc 1e-4, V0 1e-6, eta = mu / (2 c_s), seeded
    state perturbation) on each of the C5_QD_MESHES smallest meshes, in a
    seeded order.  Served: serve.SolveServer (continuous batching, 16 slots
    per mesh, FP32 operator in FP64 refinement; FMM farfield from C5_FMM_MIN
    triangles; the FP32 correction operator of an FMM mesh is, with
    inner="fmm-low", the FMM at order C5_INNER_ORDER solved to
    C5_INNER_TOL_FMM, with "fmm" the FMM at the residual's order, with
    "direct" the direct farfield (tensor-core panel) -- the FP64 residual
    always uses the order-C5_FMM FMM, so the converged solution is that
    operator's).  Plain: one
    request at a time in arrival order -- the FP64
    GMRES solve (simple_solver.iterative_solve) and the single-state
    Integrator.  Saturation (all requests at t = 0) gives the throughput;
    Poisson arrivals at 0.7 of the served saturation rate give the served
    latencies, and the plain path's FIFO queue replayed against the same
    arrivals (its measured service times) the plain latencies."""
    import tectosaur_b200 as tct
    from tectosaur_b200 import _lib, qd, serve
    from tectosaur_b200.fmm.tsfmm import FMMFarfieldOp
    from tectosaur_b200.ops.sparse_farfield_op import TriToTriDirectFarfieldOp
    from tectosaur_b200.simple_solver import (free_edge_vertices, iterative_solve,
                                              shared_vertex_matrix)

    def log(*a):
        if not quiet:
            print("[c5]", *a, flush=True)

    meshes = c5_meshes()
    t_build = time.perf_counter()
    srv = serve.SolveServer(slots=16, restart=64)
    specs, fmm_err = {}, {}
    for key, pts, tris, kind in meshes:
        n = tris.shape[0]
        cm = shared_vertex_matrix(tris, fixed_vertices=free_edge_vertices(tris))
        far = (FMMFarfieldOp(C5_FMM["mac"], C5_FMM["pts_per_cell"], C5_FMM["order"],
                             C5_FMM["mode"]) if n >= C5_FMM_MIN else TriToTriDirectFarfieldOp)
        op64 = tct.RegularizedSparseIntegralOp(*C1_NQ, K_NAME, K_NAME, PARAMS, pts, tris,
                                               np.float64, far, keep_uncorrected=False)
        inner_far, inner_tol = None, None
        if n >= C5_FMM_MIN:
            if inner == "direct":
                inner_far = TriToTriDirectFarfieldOp
            elif inner == "fmm-low":
                inner_far = FMMFarfieldOp(C5_FMM["mac"], C5_FMM["pts_per_cell"], C5_INNER_ORDER,
                                          C5_FMM["mode"])
                inner_tol = C5_INNER_TOL_FMM
            else:
                inner_tol = C5_INNER_TOL_FMM
        srv.add_mesh(key, pts, tris, cm, nq=C1_NQ, params=PARAMS, op64=op64,
                     farfield_op_type=far, inner_farfield_op_type=inner_far, inner_tol=inner_tol)
        specs[key] = (op64, cm, n)
        if n >= C5_FMM_MIN:
            # the FMM farfield's error against the direct FP64 farfield on
            # sampled observation rows (the order's truncation error)
            idx = np.arange(n)
            rows = np.sort(np.random.default_rng(31).choice(n, 256, replace=False))
            xr = np.random.default_rng(32).standard_normal(9 * n)
            direct = TriToTriDirectFarfieldOp(C1_NQ[3], K_NAME, PARAMS, pts, tris, np.float64,
                                              rows, idx).dot(xr)
            fm = op64.farfield.dot(xr).reshape(-1, 9)[rows].reshape(-1)
            fmm_err[key] = float(np.linalg.norm(fm - direct) / np.linalg.norm(direct))
        log("built", key, "%.1f s" % (time.perf_counter() - t_build))
    qd_keys = []
    for key, pts, tris, kind in sorted(meshes, key=lambda m: m[2].shape[0])[:C5_QD_MESHES]:
        cfg = c5_qd_config(tris.shape[0])
        model = qd.FullspaceModel((pts, tris), cfg)
        srv.add_qd_mesh(key + "/qd", pts, tris, cfg, model=model)
        specs[key + "/qd"] = (model, None, tris.shape[0])
        qd_keys.append(key + "/qd")
    torch.cuda.synchronize()
    t_build = time.perf_counter() - t_build
    rng = np.random.default_rng(seed)
    stream = []
    for (key, pts, tris, kind), k_req in zip(sorted(meshes, key=lambda m: m[2].shape[0]),
                                              C5_SOLVES):
        for _ in range(k_req):
            stream.append(("solve", key, rng.standard_normal(9 * tris.shape[0])))
    for i, key in enumerate(qd_keys):
        for j in range(C5_QD_PER_MESH):
            stream.append(("qd", key, c5_qd_initial(specs[key][2], seed=100 + 10 * i + j)))
    stream = [stream[i] for i in rng.permutation(len(stream))]
    kinds = [k for k, _, _ in stream]
    n_all = len(stream)

    def arrivals(offsets, qd_steps=C5_QD_STEPS, sub=None):
        arr = []
        for i, (off, (kind, k, payload)) in enumerate(zip(offsets, stream)):
            if sub is not None and i not in sub:
                continue
            arr.append((off, "qd", k, payload, qd_steps) if kind == "qd" else
                       (off, k, payload, C5_TOL))
        return arr

    # warm-up: one request of every mesh (short qd runs) -- builds the
    # resident operators and engines
    first = {}
    for i, (kind, k, _) in enumerate(stream):
        first.setdefault(k, i)
    srv.replay(arrivals([0.0] * n_all, qd_steps=3, sub=set(first.values())))
    torch.cuda.synchronize()
    log("warm-up done")
    l0 = _lib.launch_count()
    t0 = time.perf_counter()
    sat = srv.replay(arrivals([0.0] * n_all))
    torch.cuda.synchronize()
    t_served = time.perf_counter() - t0
    launches = _lib.launch_count() - l0
    assert all(r.error is None for r in sat), [r.error for r in sat if r.error]
    served_rate = n_all / t_served
    log("served saturation %.2f s" % t_served)
    for r, (kind, k, _) in zip(sat, stream):
        log("  %s %s latency %.2f s steps %s refinements %s" % (
            kind, k, r.latency, getattr(r, "gmres_steps", "-"), getattr(r, "refinements", "-")))
    # the plain paths, one request at a time in arrival order
    service, err_solve, err_qd = [], [], []
    for (kind, k, payload), r in zip(stream, sat):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if kind == "solve":
            x = iterative_solve(specs[k][0], specs[k][1], payload, cfg=dict(solver_tol=C5_TOL))
            err_solve.append(float(np.linalg.norm(r.x - x) / np.linalg.norm(x)))
        else:
            integ = qd.Integrator(specs[k][0], (0.0, payload))
            integ.integrate(C5_QD_STEPS)
            y = integ.h_y[-1].cpu().numpy()
            err_qd.append(float(np.linalg.norm(r.y - y) / np.linalg.norm(y)))
        torch.cuda.synchronize()
        service.append(time.perf_counter() - t0)
        log("  plain %s %s %.2f s" % (kind, k, service[-1]))
    plain_rate = n_all / sum(service)
    log("plain %.2f s" % sum(service))
    lam = 0.7 * served_rate
    gaps = np.random.default_rng(11).exponential(1.0 / lam, n_all)
    offs = np.cumsum(gaps) - gaps[0]
    reqs = srv.replay(arrivals(list(offs)))
    fin, plat = 0.0, []
    for off, sv in zip(offs, service):
        fin = max(fin, off) + sv
        plat.append(fin - off)

    def pct(v):
        v = np.asarray(v, dtype=np.float64)
        return {"p50_ms": 1e3 * float(np.percentile(v, 50)),
                "p99_ms": 1e3 * float(np.percentile(v, 99))} if v.size else None
    lat = {}
    for kd in ("solve", "qd"):
        lat[kd] = {"served": pct([r.latency for r, k in zip(reqs, kinds) if k == kd]),
                   "plain": pct([v for v, k in zip(plat, kinds) if k == kd]),
                   "served_saturation": pct([r.latency for r, k in zip(sat, kinds) if k == kd])}
    by_kind = {kd: {"requests": int(sum(1 for k in kinds if k == kd)),
                    "plain_s": float(sum(sv for sv, k in zip(service, kinds) if k == kd))}
               for kd in ("solve", "qd")}
    return {
        "metric": "served vs plain requests/s (solves/s and qd integrations/s)",
        "served_requests_per_s": served_rate, "plain_requests_per_s": plain_rate,
        "speedup_vs_plain": served_rate / plain_rate,
        "served_s": t_served, "plain_s": float(sum(service)),
        "requests": by_kind,
        "meshes": {key: {"n_tris": int(tris.shape[0]), "kind": kind,
                         "farfield": ("fmm p=%d mac %.1f, %d per leaf"
                                      % (C5_FMM["order"], C5_FMM["mac"], C5_FMM["pts_per_cell"])
                                      if tris.shape[0] >= C5_FMM_MIN else "direct"),
                         "served_inner_farfield": (
                             "direct (tensor-core panel)"
                             if tris.shape[0] < C5_FMM_MIN or inner == "direct" else
                             ("fmm p=%d, correction tol %g" % (C5_INNER_ORDER, C5_INNER_TOL_FMM)
                              if inner == "fmm-low" else
                              "fmm p=%d, correction tol %g" % (C5_FMM["order"],
                                                                C5_INNER_TOL_FMM))),
                         "served_gmres_steps_mean": float(np.mean(
                             [r.gmres_steps for r, (k_, m_, _) in zip(sat, stream)
                              if k_ == "solve" and m_ == key] or [0])),
                         "served_refinements_mean": float(np.mean(
                             [r.refinements for r, (k_, m_, _) in zip(sat, stream)
                              if k_ == "solve" and m_ == key] or [0])),
                         "plain_s": float(sum(sv for sv, (k_, m_, _) in zip(service, stream)
                                              if m_ in (key, key + "/qd")))}
                   for key, pts, tris, kind in meshes},
        "qd_meshes": qd_keys, "qd_steps": C5_QD_STEPS, "solve_tol": C5_TOL,
        "max_rel_diff_solve_vs_plain_fp64": max(err_solve) if err_solve else None,
        "max_rel_diff_qd_vs_plain_integrator": max(err_qd) if err_qd else None,
        "fmm_rel_err_vs_direct_fp64": fmm_err,
        "latency_poisson": {"arrival_rate_per_s": lam, "fraction_of_served_saturation": 0.7,
                            **lat},
        "gpu_launches": int(launches),
        "build_s": t_build, "resident_bytes": int(srv.resident_bytes),
        "h2d_bytes": int(sum(p.nbytes for _, _, p in stream)),
        "d2h_bytes": int(sum((r.x if k == "solve" else r.y).nbytes for r, k in zip(sat, kinds))),
    }


C5_QD_STEPS = 200


def c5_qd_config(n_tris, float_type=np.float32):
    """The C5 quasidynamic configuration: the reference example run's
    constants (shear modulus 3e10, density 2670 -> eta = mu / (2 c_s), f0
    0.6, V0 1e-6, plate rate 1e-9, 50 MPa normal stress, step tolerance
    1e-4) with a 0.010, b 0.015, Dc 1e-4 and the plain method's rules."""
    cfg = qd_config(n_tris, float_type)
    cfg["Dc"] = 1e-4
    return cfg


def c5_qd_initial(n_tris, seed):
    """Zero slip and state 0.7 with a seeded perturbation (it perturbs the
    initial slip rate)."""
    return qd_initial(n_tris, seed)


def run_serve_workload(args, rank, world, torch, dist):
    """The C5 served stream as its own line (see c5_stream)."""
    sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    sampler.start()
    res = c5_stream(torch, quiet=(rank != 0), inner=args.c5_inner)
    clocks = sampler.stop()
    if rank != 0:
        return
    line = {
        "metric": "BEM requests/s: served (continuous batching, mixed precision) vs plain",
        "value": res["served_requests_per_s"], "unit": "requests/s", "n_gpus": world,
        "steps": 1, "warmup": 1, "ms_per_step": 1e3 * res["served_s"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 operator (tensor-core farfield panel / FMM) + f64 residual refinement; "
                 "f64 qd state",
        "data": "synthetic (seeded meshes, arrivals, right-hand sides and qd states)",
        "config": {"workload": "C5 served stream (bench.c5_stream)", **{
            k: res[k] for k in ("meshes", "requests", "qd_meshes", "qd_steps", "solve_tol")},
            "parallelism": "replicas"},
        "served": res,
        "e2e": {"value": res["served_requests_per_s"], "unit": "requests/s",
                "h2d_bytes_per_step": res["h2d_bytes"], "d2h_bytes_per_step": res["d2h_bytes"],
                "api": "serve.SolveServer.replay(stream of solve and qd requests) -> numpy"},
        "gpu_launches": res["gpu_launches"], "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def config_block(n_tris, nnzb):
    return {
        "workload": ("direct-farfield 60k-triangle topographic surface (174x174 grid over "
                     "[-10,10]^2, z = 0.5 exp(-(x^2+y^2)/8) + 0.02 N(0,1)), elasticRH3 "
                     "RegularizedSparseIntegralOp(6,6,6,1,5,2.5), 3-point farfield rule on all "
                     "triangle pairs + corrected nearfield"),
        "n_tris": int(n_tris), "dof": int(9 * n_tris), "nearfield_blocks": int(nnzb),
        "kernel": K_NAME, "params": PARAMS, "parallelism": "replicas (independent applies per GPU)",
        "l2": "inputs larger than L2: nearfield blocks %.2f GB per apply" % (nnzb * 324 / 1e9),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="default launch shapes (skip the autotuner in setup)")
    ap.add_argument("--c5-inner", default="fmm-low", choices=["fmm-low", "fmm", "direct"],
                    help="farfield of the served FP32 correction operator on FMM meshes")
    ap.add_argument("--no-served", action="store_true",
                    help="skip the C5 served-vs-plain stream on the default line")
    ap.add_argument("--grid", type=int, default=None,
                    help="vertices per side of the surface grid (174 = the 59,858-triangle "
                         "workload; smaller for profiling; the fmm workload uses 707)")
    ap.add_argument("--workload", default="c2",
                    choices=["c2", "fmm", "solve", "pairs", "panel", "batch", "serve", "qd",
                             "interior", "c4solve", "near", "ptspanel"],
                    help="c2: the operator apply line (default); fmm: the 1M-triangle FMM "
                         "farfield; solve: the 722-triangle FP64 GMRES solve; pairs: the "
                         "400k-pair batched singular quadrature + BSR matvec; panel: the "
                         "C2 farfield on a panel of --rhs vectors (tensor cores); batch: "
                         "batched mixed-precision solves vs the plain FP64 solve")
    ap.add_argument("--rhs", type=int, default=64)
    ap.add_argument("--panel-kernel", default="elasticRH3", choices=["elasticRH3", "elasticRT3"],
                    help="kernel of the panel workload")
    ap.add_argument("--pairs", type=int, default=400_000)
    ap.add_argument("--qd-steps", type=int, default=200,
                    help="RK23 steps per quasidynamic integration (qd workload)")
    ap.add_argument("--fmm-order", type=int, default=None)
    ap.add_argument("--fmm-ppc", type=int, default=None)
    ap.add_argument("--fmm-mode", default=None, choices=["fmm", "treecode"])
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))

    if args.workload in ("fmm", "solve", "pairs", "panel", "batch", "serve", "qd", "interior",
                         "c4solve", "near", "ptspanel"):
        {"fmm": run_fmm_workload, "solve": run_solve_workload, "pairs": run_pairs_workload,
         "panel": run_panel_workload, "batch": run_batch_workload,
         "serve": run_serve_workload, "qd": run_qd_workload,
         "interior": run_interior_workload, "c4solve": run_c4solve_workload,
         "near": run_near_workload, "ptspanel": run_ptspanel_workload}[args.workload](
            args, rank, world, torch, dist)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return

    from tectosaur_b200 import _lib
    pts, tris = c2_mesh(args.grid or 174)
    t_build = time.perf_counter()
    op = build_op(pts, tris)
    torch.cuda.synchronize()
    t_build = time.perf_counter() - t_build
    # launch shapes picked by the autotuner on this operator (setup, untimed)
    t_tune = time.perf_counter()
    shapes = op.autotune() if not args.no_autotune else {}
    t_tune = time.perf_counter() - t_tune
    n = tris.shape[0]
    nnzb = op.nearfield.bsr.nnzb
    x = torch.from_numpy(np.random.default_rng(3 + rank).standard_normal(9 * n)
                         .astype(np.float32)).cuda()
    y = torch.empty_like(x)
    far, near = op.farfield, op.nearfield

    for _ in range(args.warmup):
        op.dot_device(x, y)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    sampler = ClockSampler(local_rank)
    sampler.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    for i in range(args.steps):
        ev[i][0].record()
        far.dot_device(x, y, accumulate=False)
        ev[i][1].record()
        near.dot_device(x, y, accumulate=True)
    end.record()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = sampler.stop()
    total_ms = start.elapsed_time(end)
    far_ms = float(np.mean([a.elapsed_time(b) for a, b in ev]))
    if dist is not None:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = world * args.steps / (total_ms * 1e-3)
    # the nearfield BSR launch alone (the apply's second kernel), CUDA events
    # on the stream it is launched on; its 1.9 GB of blocks are beyond L2
    nev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    torch.cuda.synchronize()
    for i in range(args.steps):
        nev[i][0].record()
        near.dot_device(x, y, accumulate=True)
        nev[i][1].record()
    torch.cuda.synchronize()
    bsr_ms = float(np.mean([a.elapsed_time(b) for a, b in nev]))

    # e2e through the public API with host arrays (copy in, copy out)
    x_host = x.cpu().numpy()
    op.dot(x_host)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        yh = op.dot(x_host)
    t_e2e = time.perf_counter() - t0
    if dist is not None:
        t = torch.tensor([t_e2e], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_e2e = float(t.item())
    e2e = {"value": world * args.steps / t_e2e, "unit": "matvecs/s",
           "h2d_bytes_per_step": int(x_host.nbytes), "d2h_bytes_per_step": int(yh.nbytes),
           "api": "RegularizedSparseIntegralOp.dot(numpy float32) -> numpy"}

    if rank == 0:
        peak_ffma, peak_ffma2 = fp32_peak_tflops(torch, _lib.lib)
        peak = max(peak_ffma, peak_ffma2)
        flops = float(n) * n * 9 * FLOPS_PER_POINT_PAIR_RH
        achieved = flops / (far_ms * 1e-3) / 1e12
        near_ms = ms_per_step - far_ms
        near_bytes = nnzb * (81 * 4 + 4) + (n + 1) * 4 + 2 * 9 * n * 4
        mp = measured_peaks()
        hbm = mp.get("hbm_gbs") if mp else 6650.0
        obs_blocks = (n + 127) // 128
        chunks = max(1, min(-(-1184 // obs_blocks), max(1, n // 128), 32))
        line = {
            "metric": "BEM matvecs/s", "value": value, "unit": "matvecs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded mesh and inputs)",
            "config": config_block(n, nnzb),
            "roofline": {
                "kernel": "far_main_rh2<3, uniform> (packed f32x2 elasticRH3 tri-to-tri "
                          "farfield)",
                "bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": FAR_TRAFFIC_BYTES,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                                  "full-size launch (profiles/far_main_rh2_c2_full.md)",
                "peak_source": "measured live: best of the FP32 FMA probes (scalar FFMA "
                               "%.1f, packed fma.rn.f32x2 %.1f TFLOP/s); MEASURED_PEAKS.json "
                               "has no FP32 figure" % (peak_ffma, peak_ffma2),
                "algorithmic": "%.3e flops per apply = %d^2 tri pairs x 9 point pairs x %g"
                               % (flops, n, FLOPS_PER_POINT_PAIR_RH),
                "far_ms": far_ms,
            },
            "nearfield": {"ms": near_ms, "bytes": near_bytes,
                          "ms_source": "step time minus the farfield launches' event time",
                          "achieved_gbs": near_bytes / (near_ms * 1e-3) / 1e9 if near_ms > 0 else None,
                          "bsr_ms": bsr_ms,
                          "bsr_ms_source": "the bsr9_kernel launch alone, CUDA events, mean "
                                           "of %d launches after the timed steps" % args.steps,
                          "bsr_achieved_gbs": near_bytes / (bsr_ms * 1e-3) / 1e9,
                          "bsr_frac": near_bytes / (bsr_ms * 1e-3) / 1e9 / hbm,
                          "hbm_peak_gbs": hbm, "peak_source": "MEASURED_PEAKS.json" if mp else "fallback",
                          "row_align": int(near.bsr.row_align), "slots": int(near.bsr.stride),
                          "traffic": NEAR_TRAFFIC_BYTES if near.bsr.row_align == 32 else None,
                          "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum "
                                            "of one full-size launch "
                                            "(profiles/bsr9_fp32_c2.md)"},
            "e2e": e2e,
            "gpu_launches": args.steps * (2 + (1 if chunks > 1 else 0) + (1 if nnzb else 0)),
            "clocks": clocks,
            "setup_s": t_build,
            "autotune": dict(shapes, seconds=t_tune),
        }
        classes = c2_classes(pts, tris)
        line["parity"] = c2_parity(pts, tris, y.cpu().numpy(), x.cpu().numpy(), classes)
        if world == 1 and not args.no_served:
            # the north-star comparison: the C5 stream served vs plain
            del op, far, near
            torch.cuda.empty_cache()
            try:
                line["served"] = c5_stream(torch, inner=args.c5_inner)
            except Exception as e:  # keep the matvec line if the stream fails
                line["served"] = {"error": "%s: %s" % (type(e).__name__, e)}
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(pts, tris, classes)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
