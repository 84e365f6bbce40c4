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


def c2_mesh(n=174, seed=2):
    from tectosaur_b200.mesh.mesh_gen import make_rect
    pts, tris = make_rect(n, n, [[-10, -10, 0], [10, -10, 0], [10, 10, 0], [-10, 10, 0]])
    rng = np.random.default_rng(seed)
    pts = pts.copy()
    pts[:, 2] = 0.5 * np.exp(-(pts[:, 0] ** 2 + pts[:, 1] ** 2) / 8.0) + \
        0.02 * rng.standard_normal(pts.shape[0])
    return pts, tris


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
def cpu_apply_sample(pts, tris, n_obs_sample, seed=3, n_threads=None):
    """Time one apply restricted to `n_obs_sample` observation triangles
    (farfield over all sources + their nearfield rows), FP32, with the
    oracle restatement of the reference's kernels on all host threads.
    Returns (seconds_far, seconds_near, n_blocks_sample)."""
    from oracle import oracle as orc
    from tectosaur_b200.nearfield import triangle_rules as trr
    from tectosaur_b200.nearfield.nearfield_op import nearfield_pairs
    from tectosaur_b200.util.quadrature import gauss2d_tri, gauss4d_tri
    n = tris.shape[0]
    rng = np.random.default_rng(seed)
    obs = np.sort(rng.choice(n, size=n_obs_sample, replace=False))
    x = rng.standard_normal(n * 9)
    # nearfield blocks of the sampled rows (assembly: setup, not timed)
    cl = nearfield_pairs(pts, tris, obs, np.arange(n), NQ["thr"])
    rules = {"co": (trr.coincident_quad(NQ["nq_co"]), False, True),
             "ea": (trr.edge_adj_quad(NQ["nq_ea"]), True, True),
             "va": (trr.vertex_adj_quad(NQ["nq_va"], NQ["nq_va"], NQ["nq_va"]), True, True),
             "near": (gauss4d_tri(NQ["nq_near"], NQ["nq_near"]), False, False)}
    far4 = gauss4d_tri(NQ["nq_far"], NQ["nq_far"])
    rows, cols, blocks = [], [], []
    for c, (rule, adj, check0) in rules.items():
        recs, dofs = cl[c]
        if dofs.shape[0] == 0:
            continue
        b = orc.pairs(K_NAME, np.float32, rule, pts, tris, recs[:, :5 if adj else 2], PARAMS,
                      adj=adj, check0=check0, n_threads=n_threads)
        b = b - orc.pairs(K_NAME, np.float32, far4, pts, tris, recs[:, :2], PARAMS,
                          check0=(c == "co"), n_threads=n_threads)
        rows.append(dofs[:, 0])
        cols.append(dofs[:, 1])
        blocks.append(b.reshape(-1, 9, 9))
    rows = np.concatenate(rows)
    cols = np.concatenate(cols)
    blocks = np.concatenate(blocks).astype(np.float32).astype(np.float64)
    t0 = time.perf_counter()
    orc.farfield_tris(K_NAME, np.float32, gauss2d_tri(NQ["nq_far"]), pts, tris[obs], tris, x,
                      PARAMS, n_threads=n_threads)
    t1 = time.perf_counter()
    orc.bcoo_matvec(np.float32, rows, cols, blocks, x, obs.shape[0] * 9, n_threads=n_threads)
    t2 = time.perf_counter()
    return t1 - t0, t2 - t1, rows.shape[0]


def cpu_baseline(pts, tris, nnzb_full, target_s=12.0):
    n = tris.shape[0]
    threads = os.cpu_count() or 1
    probe = 8
    tf, tn, nb = cpu_apply_sample(pts, tris, probe)
    per_obs = max(tf / probe, 1e-6)
    n_s = int(min(max(probe, target_s / per_obs), n // 4))
    tf, tn, nb = cpu_apply_sample(pts, tris, n_s)
    t_full = tf * (n / n_s) + tn * (nnzb_full / max(nb, 1))
    return {
        "value": 1.0 / t_full, "unit": "matvecs/s", "cores": threads, "kind": "port",
        "sample": ("oracle restatement of the reference kernels (FP32, OpenMP %d threads): "
                   "farfield of %d of %d observation triangles against all sources (%.1f s) "
                   "+ BCOO matvec of their %d nearfield blocks (%.3f s), extrapolated by "
                   "triangle count and block count to one full apply (%.1f s)"
                   % (threads, n_s, n, tf, nb, tn, t_full)),
    }


def run_reference(args, rank, world):
    if rank != 0:
        return
    pts, tris = c2_mesh()
    n = tris.shape[0]
    from tectosaur_b200.nearfield.nearfield_op import nearfield_pairs
    cl = nearfield_pairs(pts, tris, np.arange(n), np.arange(n), NQ["thr"])
    nnzb = sum(v[1].shape[0] for v in cl.values())
    threads = os.cpu_count() or 1
    probe = 8
    tf, tn, nb = cpu_apply_sample(pts, tris, probe)
    n_s = int(min(max(probe, 6.0 / max(tf / probe, 1e-6)), n // 4))
    times = []
    for i in range(args.warmup + args.steps):
        tf, tn, nb = cpu_apply_sample(pts, tris, n_s, seed=3 + i)
        if i >= args.warmup:
            times.append(tf * (n / n_s) + tn * (nnzb / max(nb, 1)))
    t = float(np.mean(times))
    value = 1.0 / t
    line = {
        "metric": "BEM matvecs/s", "value": value, "unit": "matvecs/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "impl": "reference",
        "config": config_block(n, nnzb),
        "cpu_baseline": {"value": value, "unit": "matvecs/s", "cores": threads, "kind": "port",
                         "sample": "each step: farfield of %d of %d observation triangles "
                                   "against all sources + their nearfield BCOO rows, "
                                   "extrapolated to one full apply" % (n_s, n)},
        "e2e": {"value": value, "unit": "matvecs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
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
    ap.add_argument("--grid", type=int, default=174,
                    help="vertices per side of the surface grid (174 = the 59,858-triangle "
                         "workload; smaller for profiling)")
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

    from tectosaur_b200 import _lib
    pts, tris = c2_mesh(args.grid)
    t_build = time.perf_counter()
    op = build_op(pts, tris)
    torch.cuda.synchronize()
    t_build = time.perf_counter() - t_build
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
                "kernel": "far_main<float, elasticRH3, 3> (tri-to-tri farfield)",
                "bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": None,
                "peak_source": "measured live: best of the FP32 FMA probes (scalar FFMA "
                               "%.1f, packed fma.rn.f32x2 %.1f TFLOP/s); MEASURED_PEAKS.json "
                               "has no FP32 figure" % (peak_ffma, peak_ffma2),
                "algorithmic": "%.3e flops per apply = %d^2 tri pairs x 9 point pairs x %g"
                               % (flops, n, FLOPS_PER_POINT_PAIR_RH),
                "far_ms": far_ms,
            },
            "nearfield": {"ms": near_ms, "bytes": near_bytes,
                          "achieved_gbs": near_bytes / (near_ms * 1e-3) / 1e9 if near_ms > 0 else None,
                          "hbm_peak_gbs": hbm, "peak_source": "MEASURED_PEAKS.json" if mp else "fallback"},
            "e2e": e2e,
            "gpu_launches": args.steps * (2 + (1 if chunks > 1 else 0) + (1 if nnzb else 0)),
            "clocks": clocks,
            "setup_s": t_build,
        }
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(pts, tris, nnzb)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
