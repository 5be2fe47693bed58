#!/usr/bin/env python3
"""GN iterations/s of HI-SLAM2's 300-keyframe backend bundle adjustment on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one ``droid_backends.ba`` call of the backend workload (300
keyframes, 43x77 grid, 6000 edges, 8 Gauss-Newton iterations, frames 0-9 fixed,
lm=1e-5, ep=1e-2; seeded synthetic inputs, see ``hislam2_b200.synth``), started
from the same initial poses/disparities every step.  ``value`` is the device-
timed throughput with inputs resident in HBM (max over ranks); ``e2e`` repeats
it through the public op with the inputs copied from pinned host memory and
the updated poses/disparities copied back inside the timed region.  The line
also carries the corr-lookup throughput (4-level radius-4 lookup over the
258-edge frontend window), a roofline entry for the dominant kernel timed live
with CUDA events, SM clocks sampled during the timed region and the float64
CPU oracle timed on a bounded sample.

With N > 1 (torchrun) every rank solves its own window: the path has no
exchange step, so ranks are independent replicas ("scaling": "weak").

``--impl reference`` times the reference algorithm's CPU restatement (the
oracle; HI-SLAM2's own ``ba`` needs Eigen, absent here) on the host cores on a
bounded sample of the same workload, and prints the same line with
``"impl": "reference"``.
"""

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "hi-slam2_b200"), ROOT]

import numpy as np  # noqa: E402
import torch  # noqa: E402

METRIC = "GN iters/s (300-kf BA) & corr-lookup GB/s; mixed vs FP32 at ≤1e-5 pose err"
UNIT = "GN iters/s"
WORKLOAD = "backend300"
CONFIG = {"workload": "backend300: 300 keyframes, 43x77 grid, 6000 edges, 8 GN iters, t0=10, lm=1e-5, ep=1e-2",
          "inputs_vs_l2": "targets+weights 318 MB per window > 126 MB L2 (no flush needed)"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the oracle timing leg")
    return ap.parse_args()


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return dict(hbm_gbs=d["hbm_gbs"], bf16_tflops=d["bf16_tflops"],
                    bf16_tflops_sustained=d.get("bf16_tflops_sustained", d["bf16_tflops"]), source="measured")
    return dict(hbm_gbs=6650.0, bf16_tflops=1590.0, bf16_tflops_sustained=1400.0, source="fallback")


# ------------------------------------------------------------------ clocks
class Clocks:
    """Samples nvidia-smi every 50 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits", "-lms", "50",
                 "-i", str(self.gpu)], stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for k, name in enumerate(names):
                    if r[5 + k].strip().lower().startswith("active"):
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------ distributed
def dist_setup(args):
    from hislam2_b200 import replicas
    world, rank, local = replicas.env_ranks()
    if args.impl == "ours":
        replicas.init(world, local, backend="nccl", timeout_s=180)
    return world, rank, local


def max_over_ranks(x, world, dev):
    from hislam2_b200 import replicas
    return replicas.max_over_ranks(x, world, dev)


def barrier(world):
    from hislam2_b200 import replicas
    replicas.barrier(world)


# ----------------------------------------------------------- algorithmic work
def algorithmic_work(p, HW):
    """Per-launch algorithmic bytes / FLOPs of the BA kernels for this problem."""
    ii, jj = p["ii"].cpu().numpy(), p["jj"].cpu().numpy()
    t0, t1 = p["t0"], p["t1"]
    P, E = t1 - t0, len(ii)
    kx = np.unique(np.concatenate([np.arange(t0, t1), ii]))
    M = len(kx)
    inwin = (jj >= t0) & (jj < t1)
    R = np.zeros(M, dtype=np.int64)
    pos = np.searchsorted(kx, ii)
    np.add.at(R, pos[inwin], 1)
    R += ((kx >= t0) & (kx < t1)).astype(np.int64)
    gram_blocks = int(np.sum(R * (R + 1) // 2 + R))
    back_rows = int(np.sum((jj - t0 >= 1) & (jj - t0 < P))) + max(P - 1, 0)
    n = 6 * P
    return {
        "ba_linearize": ("hbm", E * HW * 16 + M * HW * 8 + (P + E) * HW * 24 + M * HW * 8),
        "ba_schur": ("fp32", 2.0 * 36 * HW * gram_blocks),
        "ba_backsub": ("hbm", back_rows * HW * 24 + M * HW * (8 + 4 + 8)),
        "ba_cholesky": ("fp64", n ** 3 / 3.0 + 2.0 * n * n),
    }


def roofline(prof, work, steps, iters, peaks, simt, traffic_table):
    """Roofline entry for the kernel with the largest share of the timed region."""
    name = max((k for k in prof if k in work), key=lambda k: prof[k][1])
    launches, total_ms = prof[name]
    kind, amount = work[name]
    per_launch_s = total_ms / launches / 1e3
    if kind == "hbm":
        achieved, peak, unit = amount / per_launch_s / 1e9, peaks["hbm_gbs"], "GB/s"
        bound = "hbm"
    elif kind == "fp32":
        achieved, peak, unit = amount / per_launch_s / 1e12, simt[0], "TFLOP/s"
        bound = "fp32"
    else:
        achieved, peak, unit = amount / per_launch_s / 1e12, simt[1], "TFLOP/s"
        bound = "fp64"
    share = total_ms / sum(v[1] for v in prof.values())
    tr = traffic_table.get(name)
    return {"kernel": name, "bound": bound, "achieved": round(achieved, 3), "peak": round(peak, 3), "unit": unit,
            "frac": round(achieved / peak, 4), "traffic": tr, "launches": launches,
            "avg_launch_us": round(per_launch_s * 1e6, 2), "share_of_kernel_time": round(share, 3),
            "peak_source": peaks["source"] if bound == "hbm" else "fma probe (hs2_measure_simt_peaks)"}


# ------------------------------------------------------------------- ours
def run_ours(args, world, rank, local):
    import droid_backends
    from hislam2_b200 import _lib, replicas, synth

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    peaks = measured_peaks()
    simt = _lib.measure_simt_peaks()
    p = synth.make_ba_problem(WORKLOAD, seed=replicas.window_seed(rank), device=dev)
    HW = p["disps"].shape[1] * p["disps"].shape[2]
    init_poses, init_disps = p["poses"].clone(), p["disps"].clone()
    poses, disps = init_poses.clone(), init_disps.clone()
    iters = p["iters"]

    def step():
        poses.copy_(init_poses)
        disps.copy_(init_disps)
        droid_backends.ba(poses, disps, p["intrinsics"], p["targets"], p["weights"], p["eta"], p["ii"], p["jj"],
                          p["t0"], p["t1"], iters, p["lm"], p["ep"], False)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    barrier(world)
    clocks = Clocks(local)
    _lib.profile_report(reset=True)
    _lib.profile_enable(True)
    n0 = _lib.launch_count()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = _lib.launch_count() - n0
    _lib.profile_enable(False)
    prof = _lib.profile_report(reset=True)
    barrier(world)
    ms = max_over_ranks(e0.elapsed_time(e1), world, dev)
    value = replicas.throughput(iters * args.steps, ms, world)

    # end to end through the public op: pinned host inputs in, updated state out
    host = {k: p[k].cpu().pin_memory() for k in ("poses", "disps", "intrinsics", "targets", "weights", "eta",
                                                  "ii", "jj")}
    host["poses"].copy_(init_poses.cpu())
    host["disps"].copy_(init_disps.cpu())
    devbuf = {k: torch.empty_like(v, device=dev) for k, v in host.items()}
    out_poses = torch.empty_like(host["poses"]).pin_memory()
    out_disps = torch.empty_like(host["disps"]).pin_memory()
    h2d = sum(v.numel() * v.element_size() for v in host.values())
    d2h = out_poses.numel() * 4 + out_disps.numel() * 4

    def step_e2e():
        for k, v in host.items():
            devbuf[k].copy_(v, non_blocking=True)
        droid_backends.ba(devbuf["poses"], devbuf["disps"], devbuf["intrinsics"], devbuf["targets"],
                          devbuf["weights"], devbuf["eta"], devbuf["ii"], devbuf["jj"], p["t0"], p["t1"], iters,
                          p["lm"], p["ep"], False)
        out_poses.copy_(devbuf["poses"], non_blocking=True)
        out_disps.copy_(devbuf["disps"], non_blocking=True)

    for _ in range(2):
        step_e2e()
    torch.cuda.synchronize()
    barrier(world)
    e0.record()
    for _ in range(args.steps):
        step_e2e()
    e1.record()
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1), world, dev)
    e2e = {"value": round(replicas.throughput(iters * args.steps, ms_e2e, world), 3), "unit": UNIT,
           "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)}

    corr = corr_lookup(args, dev, world, peaks)
    pg = pgba_leg(args, dev, world, rank)

    traffic_path = os.path.join(ROOT, "profiles", "traffic.json")
    traffic = json.load(open(traffic_path)) if os.path.exists(traffic_path) else {}
    roof = roofline(prof, algorithmic_work(p, HW), args.steps, iters, peaks, simt, traffic)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(p, target_seconds=25.0)

    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": max(args.warmup, 3), "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 reduced system)",
                "data": "synthetic (seeded; Replica-shaped 43x77 grid)",
                "config": dict(CONFIG, parallelism="replicas: one independent window per rank" if world > 1 else
                               "single GPU"),
                "e2e": e2e, "gpu_launches": int(launches), "roofline": roof, "cpu_baseline": cpu,
                "corr_lookup": corr, "pgba": pg, "clocks": clk,
                "kernel_ms_per_step": {k: round(v[1] / args.steps, 4) for k, v in sorted(prof.items())},
                "simt_peaks_tflops": {"fp32": round(simt[0], 2), "fp64": round(simt[1], 2)}}
        print(json.dumps(line), flush=True)
    replicas.finalize(world)


def corr_lookup(args, dev, world, peaks):
    """4-level radius-4 lookup of the 258-edge frontend window (fp16 volumes)."""
    import droid_backends
    from hislam2_b200 import synth
    import torch.nn.functional as F

    c = synth.make_corr_problem("frontend", seed=0, device=dev, dtype=torch.float16)
    f, ii, jj = c["fmaps"], c["ii"], c["jj"]
    E, (H, W), r = ii.numel(), f.shape[2:], c["radius"]
    with torch.no_grad():
        vol = torch.matmul((f[ii].flatten(2) / 4.0).transpose(1, 2), f[jj].flatten(2) / 4.0)
        vol = vol.reshape(E * H * W, 1, H, W)
        pyr = []
        for lvl in range(4):
            pyr.append(vol.view(E, H, W, vol.shape[-2], vol.shape[-1]).contiguous())
            if lvl < 3:
                vol = F.avg_pool2d(vol, 2, stride=2)
        del vol
    crd = c["coords"].permute(0, 3, 1, 2).contiguous()
    crds = [(crd / 2 ** i).contiguous() for i in range(4)]
    D, rd = 2 * r + 2, 2 * r + 1
    bytes_per = E * H * W * 4 * (D * D * 2 + rd * rd * 2 + 8)

    def step():
        for lvl in range(4):
            droid_backends.corr_index_forward(pyr[lvl], crds[lvl], r)

    for _ in range(3):
        step()
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), world, dev) / args.steps
    gbs = bytes_per / (ms / 1e3) / 1e9 * world
    del pyr
    torch.cuda.empty_cache()
    return {"value": round(gbs, 2), "unit": "GB/s", "ms_per_lookup": round(ms, 4),
            "config": "258 edges (frontend window), 43x77, 4 levels, radius 4, fp16 volumes",
            "roofline": {"bound": "hbm", "achieved": round(gbs / world, 2), "peak": peaks["hbm_gbs"],
                         "unit": "GB/s", "frac": round(gbs / world / peaks["hbm_gbs"], 4)}}


def pgba_leg(args, dev, world, rank):
    """One Sim3 pose-graph BA step (droid_backends.pgba) on the same 300-keyframe /
    6000-edge window with Sim3 poses and 600 relative-pose factors, device-timed."""
    import droid_backends
    from hislam2_b200 import _lib, replicas, synth

    g = synth.make_pgba_problem(WORKLOAD, seed=replicas.window_seed(rank), device=dev, num_factors=600)
    init = g["disps"].clone()
    disps = init.clone()

    def step():
        disps.copy_(init)
        droid_backends.pgba(g["poses"], disps, g["intrinsics"], g["targets"], g["weights"], g["eta"], g["Hsp"],
                            g["vsp"], g["ii"], g["jj"], g["iip"], g["jjp"], g["t0"], g["t1"], g["lm"], g["ep"])

    for _ in range(3):
        step()
    torch.cuda.synchronize()
    barrier(world)
    _lib.profile_report(reset=True)
    _lib.profile_enable(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    _lib.profile_enable(False)
    prof = _lib.profile_report(reset=True)
    ms = max_over_ranks(e0.elapsed_time(e1), world, dev) / args.steps
    del g, init, disps
    torch.cuda.empty_cache()
    return {"value": round(world * 1e3 / ms, 2), "unit": "pgba steps/s", "ms_per_step": round(ms, 4),
            "config": "backend300 window with Sim3 poses, 600 relative-pose factors, one GN step",
            "kernel_ms_per_step": {k: round(v[1] / args.steps, 4) for k, v in sorted(prof.items())}}


# ------------------------------------------------------------ CPU oracle legs
def oracle_problem_rows(p, rows):
    """The workload restricted to the first `rows` pixel rows (all edges and frames)."""
    f = lambda k: p[k].detach().cpu().numpy()  # noqa: E731
    return dict(poses=f("poses"), disps=f("disps")[:, :rows], intr=f("intrinsics"),
                targets=f("targets")[:, :, :rows], weights=f("weights")[:, :, :rows], eta=f("eta")[:, :rows],
                ii=f("ii"), jj=f("jj"), t0=p["t0"], t1=p["t1"], lm=p["lm"], ep=p["ep"])


def oracle_iteration(q):
    import oracle
    t = time.perf_counter()
    oracle.ba.ba(q["poses"], np.ascontiguousarray(q["disps"]), q["intr"], np.ascontiguousarray(q["targets"]),
                 np.ascontiguousarray(q["weights"]), np.ascontiguousarray(q["eta"]), q["ii"], q["jj"], q["t0"],
                 q["t1"], 1, q["lm"], q["ep"])
    return time.perf_counter() - t


def cpu_baseline(p, target_seconds):
    """One float64 oracle GN iteration on a row band sized for ~target_seconds; GN iters/s of the
    whole 43-row problem extrapolated linearly in pixel rows."""
    H = p["disps"].shape[1]
    t_small = oracle_iteration(oracle_problem_rows(p, 2))
    rows = int(min(H, max(2, round(2 * target_seconds / max(t_small, 1e-3)))))
    dt = oracle_iteration(oracle_problem_rows(p, rows))
    return {"value": round((rows / H) / dt, 6), "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": "1 GN iteration of the 300-kf / 6000-edge problem on %d of %d pixel rows (%.1f s), "
                      "float64 numpy oracle, extrapolated by rows" % (rows, H, dt)}


def run_reference(args, world, rank):
    if rank != 0:
        return
    from hislam2_b200 import synth
    p = synth.make_ba_problem(WORKLOAD, seed=0)
    H = p["disps"].shape[1]
    budget = 150.0 / max(1, args.steps + args.warmup)
    t_small = oracle_iteration(oracle_problem_rows(p, 2))
    rows = int(min(H, max(1, round(2 * budget / max(t_small, 1e-3)))))
    q = oracle_problem_rows(p, rows)
    for _ in range(args.warmup):
        oracle_iteration(q)
    times = [oracle_iteration(q) for _ in range(args.steps)]
    total = float(sum(times))
    value = args.steps * (rows / H) / total
    sample = ("1 GN iteration per step of the 300-kf / 6000-edge problem on %d of %d pixel rows, float64 numpy "
              "oracle (the reference's own ba needs Eigen, absent), extrapolated by rows" % (rows, H))
    line = {"metric": METRIC, "value": round(value, 6), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": dict(CONFIG, parallelism="host cores"), "impl": "reference",
            "cpu_baseline": {"value": round(value, 6), "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(value, 6), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
