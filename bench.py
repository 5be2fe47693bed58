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
258-edge frontend window), the tensor-core all-pairs volume + pyramid of that
window against torch.matmul + avg_pool2d, a Sim3 pgba step, a roofline entry for
the dominant kernel timed live with CUDA events, SM clocks sampled during the
timed region, the pure-PyTorch port of HI-SLAM2's Python BA timed on the host
cores, and the pose / disparity error against the float64 oracle.

With N > 1 (torchrun) every rank solves its own window: the path has no
exchange step, so ranks are independent replicas ("scaling": "weak").

``--impl reference`` times HI-SLAM2's own ``droid_backends.ba`` (compiled
unmodified into oracle/_ref, with a dense stand-in for the Eigen solver it
includes) on the same workload -- its kernels on the GPU, its host loops and
solve on the host -- plus its corr_index_forward on the same lookup, and prints
the same line with ``"impl": "reference"``.
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
    ap.add_argument("--profile-case", default=None,
                    help="run one small pass of a kernel family for a profiler and exit (see PROFILE_CASES)")
    ap.add_argument("--profile-iters", type=int, default=1)
    ap.add_argument("--profile-edges", type=int, default=64)
    return ap.parse_args()


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return dict(hbm_gbs=d["hbm_gbs"], bf16_tflops=d["bf16_tflops"],
                    bf16_tflops_sustained=d.get("bf16_tflops_sustained", d["bf16_tflops"]), source="measured")
    return dict(hbm_gbs=6650.0, bf16_tflops=1590.0, bf16_tflops_sustained=1400.0, source="fallback")


def library_peaks(dev):
    """(fp32, fp64) throughput of cuBLAS SGEMM / DGEMM on this device in TFLOP/s: the
    denominators for kernels bound by the FP32 and FP64 pipes, measured the way the bf16
    GEMM peak is (a library GEMM timed with CUDA events)."""
    out = []
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        for dt, n in ((torch.float32, 8192), (torch.float64, 8192)):
            a = torch.randn(n, n, device=dev, dtype=dt)
            b = torch.randn(n, n, device=dev, dtype=dt)
            c = torch.matmul(a, b)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(3):
                torch.matmul(a, b, out=c)
            e1.record()
            torch.cuda.synchronize()
            out.append(3 * 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
            del a, b, c
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    torch.cuda.empty_cache()
    return tuple(out)


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
            "peak_source": peaks["source"] if bound == "hbm" else "measured cuBLAS %s on this device" %
                           ("SGEMM" if bound == "fp32" else "DGEMM")}


# ------------------------------------------------------------------- ours
def run_ours(args, world, rank, local):
    import droid_backends
    from hislam2_b200 import _lib, replicas, synth

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    peaks = measured_peaks()
    simt = library_peaks(dev)
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
    ms_serial = max_over_ranks(e0.elapsed_time(e1), world, dev)

    # the same steps with the next step's inputs copied on a second stream while the current
    # step computes (two device input sets; each step still copies its own inputs in and
    # its result out inside the timed region)
    cs = torch.cuda.Stream(device=dev)
    main = torch.cuda.current_stream(dev)
    bufs = [devbuf, {k: torch.empty_like(v, device=dev) for k, v in host.items()}]
    outs = [(out_poses, out_disps), (torch.empty_like(out_poses).pin_memory(), torch.empty_like(out_disps).pin_memory())]
    copied = [torch.cuda.Event(), torch.cuda.Event()]
    done = [torch.cuda.Event(), torch.cuda.Event()]

    def issue_copy(k):
        b = k & 1
        with torch.cuda.stream(cs):
            if k >= 2:
                cs.wait_event(done[b])   # step k-2 has finished with this input set
            for name, v in host.items():
                bufs[b][name].copy_(v, non_blocking=True)
            copied[b].record(cs)

    def run_step(k):
        b = k & 1
        main.wait_event(copied[b])
        d = bufs[b]
        droid_backends.ba(d["poses"], d["disps"], d["intrinsics"], d["targets"], d["weights"], d["eta"], d["ii"],
                          d["jj"], p["t0"], p["t1"], iters, p["lm"], p["ep"], False)
        outs[b][0].copy_(d["poses"], non_blocking=True)
        outs[b][1].copy_(d["disps"], non_blocking=True)
        done[b].record(main)

    def pipelined(n):
        cs.wait_stream(main)
        issue_copy(0)
        for k in range(n):
            if k + 1 < n:
                issue_copy(k + 1)
            run_step(k)

    pipelined(3)
    torch.cuda.synchronize()
    barrier(world)
    e0.record()
    pipelined(args.steps)
    e1.record()
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1), world, dev)
    e2e = {"value": round(replicas.throughput(iters * args.steps, ms_e2e, world), 3), "unit": UNIT,
           "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
           "pipelining": "each step's inputs copied from pinned host memory on a second stream while the "
                         "previous step computes (two device input sets), its poses/disparities copied back",
           "serialized": {"value": round(replicas.throughput(iters * args.steps, ms_serial, world), 3),
                          "note": "copy in, compute, copy out on one stream"}}

    corr = corr_lookup(args, dev, world, peaks)
    pg = pgba_leg(args, dev, world, rank)
    alt = altcorr_leg(args, dev, world, peaks)
    step = backend_step_leg(args, dev, world)
    vol = volume_leg(args, dev, world, peaks) if world == 1 else None
    bat = batch_leg(args, dev, world, rank)
    jd = jdsa_leg(args, dev, world, rank)

    traffic_path = os.path.join(ROOT, "profiles", "traffic.json")
    traffic = json.load(open(traffic_path)) if os.path.exists(traffic_path) else {}
    roof = roofline(prof, algorithmic_work(p, HW), args.steps, iters, peaks, simt, traffic)

    cpu, acc = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(p, target_seconds=12.0)
        acc = accuracy_vs_fp64(p, dev, args.steps)

    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": max(args.warmup, 3), "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 reduced system)",
                "data": "synthetic (seeded; Replica-shaped 43x77 grid)",
                "config": dict(CONFIG, parallelism="replicas: one independent window per rank" if world > 1 else
                               "single GPU"),
                "e2e": e2e, "gpu_launches": int(launches), "roofline": roof, "cpu_baseline": cpu,
                "accuracy": acc, "corr_lookup": corr, "altcorr": alt, "backend_step": step, "corr_volume": vol, "batch": bat, "pgba": pg, "jdsa": jd, "clocks": clk,
                "kernel_ms_per_step": {k: round(v[1] / args.steps, 4) for k, v in sorted(prof.items())},
                "library_peaks_tflops": {"sgemm_fp32": round(simt[0], 2), "dgemm_fp64": round(simt[1], 2)}}
        print(json.dumps(line), flush=True)
    replicas.finalize(world)


def device_time(fn, steps, warmup=3):
    """Average device time of fn() in ms (CUDA events on the current stream)."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def torch_pyramid(f, ii, jj, levels=4):
    """CorrBlock's construction in PyTorch (hislam2/modules/corr.py:29-38,63-71)."""
    import torch.nn.functional as F
    E, (H, W) = ii.numel(), f.shape[2:]
    vol = torch.matmul((f[ii].flatten(2) / 4.0).transpose(1, 2), f[jj].flatten(2) / 4.0)
    vol = vol.reshape(E * H * W, 1, H, W)
    pyr = []
    for lvl in range(levels):
        pyr.append(vol.view(E, H, W, vol.shape[-2], vol.shape[-1]))
        if lvl < levels - 1:
            vol = F.avg_pool2d(vol, 2, stride=2)
    return pyr


def frontend_lookup_inputs(dev):
    from hislam2_b200 import synth
    c = synth.make_corr_problem("frontend", seed=0, device=dev, dtype=torch.float16)
    f, ii, jj = c["fmaps"], c["ii"], c["jj"]
    E, (H, W), r = ii.numel(), f.shape[2:], c["radius"]
    with torch.no_grad():
        pyr = [v.contiguous() for v in torch_pyramid(f, ii, jj)]
    crd = c["coords"].permute(0, 3, 1, 2).contiguous()
    crds = [(crd / 2 ** i).contiguous() for i in range(4)]
    D, rd = 2 * r + 2, 2 * r + 1
    bytes_per = E * H * W * 4 * (D * D * 2 + rd * rd * 2 + 8)
    return pyr, crds, r, bytes_per


def corr_lookup(args, dev, world, peaks):
    """4-level radius-4 lookup of the 258-edge frontend window (fp16 volumes)."""
    import droid_backends
    pyr, crds, r, bytes_per = frontend_lookup_inputs(dev)

    def step():
        for lvl in range(4):
            droid_backends.corr_index_forward(pyr[lvl], crds[lvl], r)

    barrier(world)
    ms = max_over_ranks(device_time(step, args.steps), world, dev)
    gbs = bytes_per / (ms / 1e3) / 1e9 * world
    del pyr
    torch.cuda.empty_cache()
    return {"value": round(gbs, 2), "unit": "GB/s", "ms_per_lookup": round(ms, 4),
            "config": "258 edges (frontend window), 43x77, 4 levels, radius 4, fp16 volumes",
            "roofline": {"bound": "hbm", "achieved": round(gbs / world, 2), "peak": peaks["hbm_gbs"],
                         "unit": "GB/s", "frac": round(gbs / world / peaks["hbm_gbs"], 4),
                         "peak_source": peaks["source"]}}


def volume_leg(args, dev, world, peaks):
    """CorrBlock's all-pairs volume + 4-level pyramid of the 258-edge frontend window:
    hislam2_b200's tcgen05 kernel (float16, bfloat16, FP8 e4m3) against torch.matmul +
    F.avg_pool2d on the same inputs, device-timed in the same run."""
    from hislam2_b200 import _lib, backends, synth
    c = synth.make_corr_problem("frontend", seed=0, device=dev, dtype=torch.float16)
    f, ii, jj = c["fmaps"], c["ii"], c["jj"]
    E, (H, W) = ii.numel(), f.shape[2:]
    HW = H * W
    flops = 2.0 * HW * HW * 128 * E
    out_bytes = sum(E * HW * (H >> l) * (W >> l) * 2 for l in range(4))
    in_bytes = 2 * E * HW * 128 * 2
    steps = max(5, min(args.steps, 20))
    res = {"config": "258 edges (frontend window), 43x77, 128 channels, 4 levels",
           "algorithmic": {"gflop": round(flops / 1e9, 2), "write_gb": round(out_bytes / 1e9, 3)}}
    with torch.no_grad():
        for name, dt, prec in (("f16", torch.float16, "native"), ("bf16", torch.bfloat16, "native"),
                               ("e4m3", torch.float16, "e4m3")):
            g = f.to(dt)
            _lib.profile_report(reset=True)
            _lib.profile_enable(True)
            ms = device_time(lambda: backends.corr_volume(g, g, ii, jj, precision=prec), steps)
            _lib.profile_enable(False)
            prof = _lib.profile_report(reset=True)
            kms = prof.get("corr_volume", (1, ms))[1] / prof.get("corr_volume", (1, ms))[0]
            res[name] = {"ms": round(ms, 4), "kernel_ms": round(kms, 4),
                         "tflops": round(flops / (kms / 1e3) / 1e12, 1),
                         "write_gbs": round(out_bytes / (kms / 1e3) / 1e9, 1),
                         "hbm_frac": round((out_bytes + in_bytes) / (kms / 1e3) / 1e9 / peaks["hbm_gbs"], 4)}
            torch.cuda.empty_cache()
        ms_t = device_time(lambda: torch_pyramid(f, ii, jj), steps)
        res["torch_matmul_avgpool_f16"] = {"ms": round(ms_t, 4)}
        res["speedup_vs_torch_f16"] = round(ms_t / res["f16"]["ms"], 2)
        res["roofline"] = {"bound": "hbm", "achieved": round((out_bytes + in_bytes) / (res["f16"]["kernel_ms"] / 1e3)
                                                             / 1e9, 1),
                           "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": res["f16"]["hbm_frac"],
                           "peak_source": peaks["source"]}
    torch.cuda.empty_cache()
    return res


def batch_leg(args, dev, world, rank):
    """The batching workload: 64 independent windows (keyframes 8..40, edges 20..500,
    43x77 or 30x40 grids), 4 LM iterations, each iteration ONE persistent launch over
    all windows, the 4 launches replayed as a CUDA graph; against the same windows
    solved one droid_backends.ba call after another."""
    import droid_backends
    from hislam2_b200 import autotune, backends, replicas, synth
    ws = [{k: (v.to(dev) if torch.is_tensor(v) else v) for k, v in w.items()}
          for w in synth.make_batch_problems(num_windows=64, seed=replicas.window_seed(rank))]
    init = [(w["poses"].clone(), w["disps"].clone()) for w in ws]
    iters, lm, ep = 4, 1e-4, 0.1

    def reset():
        for w, (p0, d0) in zip(ws, init):
            w["poses"].copy_(p0)
            w["disps"].copy_(d0)

    cfg = autotune.best("batch64")
    plan = backends.BABatch(ws, lm, ep, **cfg)
    graph = plan.graph(iters)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = max(3, min(args.steps, 10))
    for _ in range(2):
        reset()
        graph.replay()
    total = 0.0
    for _ in range(reps):
        reset()
        torch.cuda.synchronize()
        e0.record()
        graph.replay()
        e1.record()
        torch.cuda.synchronize()
        total += e0.elapsed_time(e1)
    plan.check()
    ms = max_over_ranks(total / reps, world, dev)

    def sequential():
        for w in ws:
            droid_backends.ba(w["poses"], w["disps"], w["intrinsics"], w["targets"], w["weights"], w["eta"], w["ii"],
                              w["jj"], w["t0"], w["t1"], iters, lm, ep, False)

    reset()
    sequential()
    torch.cuda.synchronize()
    total = 0.0
    for _ in range(3):
        reset()
        torch.cuda.synchronize()
        e0.record()
        sequential()
        e1.record()
        torch.cuda.synchronize()
        total += e0.elapsed_time(e1)
    ms_seq = total / 3
    del graph, plan
    torch.cuda.empty_cache()
    return {"value": round(world * 64 * iters / (ms / 1e3), 1), "unit": "window GN iters/s",
            "ms_per_iteration": round(ms / iters, 4), "iterations": iters, "launch": "cooperative persistent, "
            "one per iteration, CUDA graph", "tuning": cfg,
            "edges_total": int(sum(w["ii"].numel() for w in ws)),
            "sequential_single_window_ms_per_iteration": round(ms_seq / iters, 4),
            "speedup_vs_sequential": round(ms_seq / ms, 2),
            "config": "64 windows, keyframes U{8..40}, edges U{20..500}, 43x77 or 30x40 grids, t0=1, lm=1e-4, ep=0.1"}


def altcorr_leg(args, dev, world, peaks):
    """The backend's memory-light correlation (radius 3, 4 levels, float16 features) over all
    6000 edges of the 300-keyframe window in the global BA loop's chunks of two source
    frames (HI-SLAM2 factor_graph.py:253-260); one step = one pass over every chunk and
    level.  `dropin`: droid_backends.altcorr_forward per chunk and level (it packs the
    call's frames channel-last first); `block`: AltCorrBlock with its pyramid packed once.
    Algorithmic work per edge-pixel-level: D^2 = 64 window dot products of 128 channels."""
    from hislam2_b200 import backends
    from hislam2_b200.corr import AltCorrBlock
    fmaps, pyr, chunks = altcorr_inputs(dev)
    r, L, E, H, W, C = 3, 4, 6000, 43, 77, 128

    def dropin():
        for ci, cj, crd in chunks:
            for lvl in range(L):
                backends.altcorr_forward(pyr[0], pyr[lvl], crd[lvl], ci, cj, r)

    blk = AltCorrBlock(fmaps[None].contiguous(), num_levels=L, radius=r)
    crd5 = [(ci, cj, crd[0].permute(0, 1, 3, 4, 2).contiguous()) for ci, cj, crd in chunks]

    def block():
        with torch.no_grad():
            for ci, cj, crd in crd5:
                blk(crd, ci, cj)

    from hislam2_b200 import synth
    pb = synth.make_ba_problem(WORKLOAD, seed=0, device=dev)
    levels = [lv[0] for lv in pyr]

    def fused():
        for ci, cj, _ in chunks:
            backends.corr_reproject_lookup(levels, pb["poses"], pb["disps"], pb["intrinsics"], ci, cj, r)

    steps = max(3, min(args.steps, 10))
    barrier(world)
    ms_drop = max_over_ranks(device_time(dropin, steps), world, dev)
    ms_blk = max_over_ranks(device_time(block, steps), world, dev)
    ms_fused = max_over_ranks(device_time(fused, steps), world, dev)
    D = 2 * r + 2
    flops = 2.0 * E * H * W * D * D * C * L
    out_bytes = E * H * W * (2 * r + 1) ** 2 * L * 2
    res = {"config": "300 keyframes, 6000 edges, 43x77, 128 channels fp16, radius 3, 4 levels, %d chunks of "
                     "two source frames" % len(chunks),
           "dropin": {"ms_per_pass": round(ms_drop, 3), "edges_per_s": round(E / (ms_drop / 1e3) * world, 1)},
           "block": {"ms_per_pass": round(ms_blk, 3), "edges_per_s": round(E / (ms_blk / 1e3) * world, 1),
                     "tflops": round(flops / (ms_blk / 1e3) / 1e12, 2),
                     "write_gbs": round(out_bytes / (ms_blk / 1e3) / 1e9, 1)},
           "fused_reproject_lookup": {
               "ms_per_pass": round(ms_fused, 3), "edges_per_s": round(E / (ms_fused / 1e3) * world, 1),
               "note": "corr_reproject_lookup per chunk: coordinates reprojected from the current poses and "
                       "disparities inside the kernel (no coordinate or volume tensors), same chunks"},
           "algorithmic": {"gflop": round(flops / 1e9, 1), "write_gb": round(out_bytes / 1e9, 3)}}
    del pyr, chunks, blk, crd5, levels
    torch.cuda.empty_cache()
    return res


def backend_step_leg(args, dev, world):
    """One update step of HI-SLAM2's backend global BA on the 300-keyframe window
    (factor_graph.py:240-277: the radius-3, 4-level correlation of all 6000 edges in
    chunks of two source frames, then cuda_ba with itrs = 2 GN iterations), timed three
    ways on the device (the update network between them is out of scope):
      plain_fp32   float32 features, the direct altcorr kernel (the reference's method:
                   one dot product per window tap), BA in the FP32 form (3xTF32 Gram);
      fp16_packed  float16 features (the reference runtime's dtype) through AltCorrBlock's
                   channel-last path, same BA;
      mixed_tc     bfloat16 features, per chunk the tcgen05 volume pyramid (corr_volume)
                   and the radius-3 lookup (corr_index_forward), BA with the one-product
                   TF32 Gram (its pose error vs FP64 is the `accuracy` entry's mixed form).
    value = GN iterations per second of the whole step (2 / step time)."""
    import droid_backends
    from hislam2_b200 import _lib, backends, synth
    from hislam2_b200.corr import AltCorrBlock, _pool_pyramid
    p = synth.make_ba_problem(WORKLOAD, seed=0, device=dev)
    g = torch.Generator().manual_seed(17)
    K, H, W, C, r, L, itrs = 300, 43, 77, 128, 3, 4, 2
    f32 = (torch.randn(K, C, H, W, generator=g) / np.sqrt(C)).to(dev)
    ii, jj = p["ii"], p["jj"]
    coords = synth.reproject(p["poses_gt"].cpu(), p["disps_gt"].cpu(), p["intrinsics"].cpu(), ii.cpu(), jj.cpu())
    coords = (coords.float() + torch.randn(coords.shape, generator=g)).to(dev)           # [E, H, W, 2]
    chunks = []
    for i in range(0, int(jj.max()) + 1, 2):
        v = ((ii >= i) & (ii < i + 2)).nonzero().flatten()
        if v.numel():
            crd = coords[v][None].contiguous()
            c5 = crd.permute(0, 1, 4, 2, 3).contiguous()
            chunks.append((ii[v].contiguous(), jj[v].contiguous(), crd,
                           [(c5 / 2 ** lvl).contiguous() for lvl in range(L)]))
    init_poses, init_disps = p["poses"].clone(), p["disps"].clone()
    poses, disps = init_poses.clone(), init_disps.clone()

    def ba():
        poses.copy_(init_poses)
        disps.copy_(init_disps)
        droid_backends.ba(poses, disps, p["intrinsics"], p["targets"], p["weights"], p["eta"], p["ii"], p["jj"],
                          p["t0"], p["t1"], itrs, p["lm"], p["ep"], False)

    pyr32 = [lv[None].contiguous() for lv in _pool_pyramid(f32, L)]

    def plain():
        for ci, cj, _, crd in chunks:
            for lvl in range(L):
                backends.altcorr_forward(pyr32[0], pyr32[lvl], crd[lvl], ci, cj, r, path="direct")
        ba()

    blk = AltCorrBlock(f32.half()[None].contiguous(), num_levels=L, radius=r)

    def fp16_packed():
        with torch.no_grad():
            for ci, cj, crd, _ in chunks:
                blk(crd, ci, cj)
        ba()

    fbf = f32.bfloat16().contiguous()

    def mixed_tc():
        for ci, cj, _, crd in chunks:
            levels = backends.corr_volume(fbf, fbf, ci, cj, num_levels=L)
            for lvl in range(L):
                droid_backends.corr_index_forward(levels[lvl], crd[lvl][0], r)
        _lib.set_gram_precision(0)
        try:
            ba()
        finally:
            _lib.set_gram_precision(1)

    res = {"config": "300 keyframes, 6000 edges in %d chunks, 43x77, 128 channels, radius 3, 4 levels, "
                     "itrs = 2 GN iterations per step" % len(chunks), "unit": "GN iters/s"}
    barrier(world)
    for name, fn, n in (("plain_fp32", plain, 1), ("fp16_packed", fp16_packed, 2), ("mixed_tc", mixed_tc, 2)):
        ms = max_over_ranks(device_time(fn, n, warmup=1), world, dev)
        res[name] = {"ms_per_step": round(ms, 2), "gn_iters_per_s": round(itrs * 1e3 / ms * world, 3)}
        torch.cuda.empty_cache()
    for name in ("fp16_packed", "mixed_tc"):
        res[name]["vs_plain"] = round(res[name]["gn_iters_per_s"] / res["plain_fp32"]["gn_iters_per_s"], 2)
    del blk, pyr32, chunks
    torch.cuda.empty_cache()
    return res


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

    # the rest of DepthVideo.cuda_pgba's iteration: the 600 factors' blocks (numeric Sim3
    # Jacobians) before the step and the Sim3 retraction of the window after it
    from hislam2_b200 import pgo
    rel, infos = synth.make_pgo_factors(g["poses"], g["iip"], g["jjp"], seed=replicas.window_seed(rank))
    poses = g["poses"].clone()
    dx = torch.zeros(g["t1"] - g["t0"], 7, device=dev)
    cons = lambda: pgo.global_relative_posesim3_constraints(g["iip"], g["jjp"], poses, rel, infos, pw=1e-3)  # noqa
    retr = lambda: pgo.sim3_retr_(poses, dx, g["t0"], g["t1"])  # noqa: E731
    ms_cons = device_time(cons, args.steps)
    ms_retr = device_time(retr, args.steps)
    del g, init, disps
    torch.cuda.empty_cache()
    return {"value": round(world * 1e3 / ms, 2), "unit": "pgba steps/s", "ms_per_step": round(ms, 4),
            "config": "backend300 window with Sim3 poses, 600 relative-pose factors, one GN step",
            "kernel_ms_per_step": {k: round(v[1] / args.steps, 4) for k, v in sorted(prof.items())},
            "pgo_constraints_ms": round(ms_cons, 4), "sim3_retr_ms": round(ms_retr, 4),
            "loop_note": "one cuda_pgba iteration = pgo_constraints + pgba step + sim3_retr; the "
                         "constraints time includes its info read (one host sync)"}


def jdsa_leg(args, dev, world, rank):
    """The mono-prior alignment step (hislam2_b200.mono.JDSA, one hs2_jdsa call: proj_trans
    plus the per-frame scale solve and depth update) on HI-SLAM2's frontend window, 25
    keyframes at 43x77 with 258 edges and its 2x2 scale grid per frame, device-timed."""
    from hislam2_b200 import _lib, mono, replicas, synth

    g = synth.make_jdsa_problem("frontend", seed=replicas.window_seed(rank), device=dev)
    init = g["dscales"].clone()
    dscales = init.clone()
    disps = g["disps"][None]

    def step():
        dscales.copy_(init)
        mono.JDSA(g["targets"], g["weights"], g["eta"], g["poses"], disps, g["intrinsics"], g["disps_prior"],
                  dscales, g["ii"], g["jj"], g["alpha"])

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
    return {"value": round(world * 1e3 / ms, 2), "unit": "JDSA steps/s", "ms_per_step": round(ms, 4),
            "config": "frontend window: 25 kf, 43x77, 258 edges, 2x2 scale grid, alpha 0.01; the step's "
                      "host sync (torch.unique, info read) included",
            "kernel_ms_per_step": {k: round(v[1] / args.steps, 4) for k, v in sorted(prof.items())}}


# ------------------------------------------------------------ CPU legs
def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def torch_path_iteration(p, rows):
    """One iteration of the pure-PyTorch port of HI-SLAM2's Python BA (geom/ba.py:BA +
    geom/chol.py:schur_solve) on the first `rows` pixel rows of every frame; seconds."""
    from oracle import torch_path
    tg = p["targets"][:, :, :rows].permute(0, 2, 3, 1).contiguous().cpu()
    wt = p["weights"][:, :, :rows].permute(0, 2, 3, 1).contiguous().cpu()
    disps = p["disps"][:, :rows].contiguous().cpu()
    ii, jj = p["ii"].cpu(), p["jj"].cpu()
    M = len(torch.unique(ii))
    eta = p["eta"][:M, :rows].contiguous().cpu()
    t = time.perf_counter()
    torch_path.BA(tg, wt, eta, p["poses"].cpu(), disps, p["intrinsics"].cpu(), ii, jj, p["t0"], ep=p["ep"],
                  lm=p["lm"])
    return time.perf_counter() - t


def cpu_baseline(p, target_seconds):
    """GN iters/s of the pure-PyTorch port on the host cores for the whole 43-row problem,
    from one iteration on each of two pixel-row bands and a linear fit in rows (its work --
    the dense E, E Q E^T and the dzcov term -- grows linearly with the rows; the
    1740x1740 Cholesky is a row-independent constant that the fit's intercept carries)."""
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    H = p["disps"].shape[1]
    r1 = 1
    t1 = torch_path_iteration(p, r1)
    r2 = int(min(H, max(r1 + 1, round(target_seconds / max(t1, 1e-3)))))
    t2 = torch_path_iteration(p, r2)
    slope = max((t2 - t1) / (r2 - r1), 0.0)
    full = t2 + slope * (H - r2)
    return {"value": round(1.0 / full, 6), "unit": UNIT, "cores": threads, "kind": "port",
            "cpu_model": cpu_model(),
            "sample": "one iteration of the pure-PyTorch port of HI-SLAM2's Python BA (geom/ba.py:BA, "
                      "geom/chol.py:schur_solve; float32, dense E, dzcov) on %d and %d of %d pixel rows of the "
                      "300-kf / 6000-edge window (%.2f s, %.2f s), the whole problem's iteration time "
                      "extrapolated linearly in rows (%.1f s)" % (r1, r2, H, t1, t2, full)}


def accuracy_vs_fp64(p, dev, steps, iters=2):
    """Pose / disparity error of ba on the backend300 window after `iters` GN iterations
    against the float64 oracle (the checker), max |x - x_fp64| / max |x_fp64|, for both
    precisions of the tensor-core Schur Gram: 3xTF32 (the FP32 form, the default) and one
    TF32 product (the mixed form), each with its own device-timed GN iterations / s."""
    import droid_backends
    import oracle
    from hislam2_b200 import _lib
    q = {k: (v.to(dev) if torch.is_tensor(v) else v) for k, v in p.items()}
    f = lambda k: p[k].double().cpu().numpy()  # noqa: E731
    t = time.perf_counter()
    r = oracle.ba.ba(f("poses"), f("disps"), f("intrinsics"), f("targets"), f("weights"), f("eta"),
                     p["ii"].cpu().numpy(), p["jj"].cpu().numpy(), p["t0"], p["t1"], iters, p["lm"], p["ep"])
    dt = time.perf_counter() - t
    rel = lambda a, b: float(np.abs(a - b).max() / np.abs(b).max())  # noqa: E731
    poses, disps = q["poses"].clone(), q["disps"].clone()

    def call(n):
        poses.copy_(q["poses"])
        disps.copy_(q["disps"])
        droid_backends.ba(poses, disps, q["intrinsics"], q["targets"], q["weights"], q["eta"], q["ii"], q["jj"],
                          q["t0"], q["t1"], n, q["lm"], q["ep"], False)

    forms = {}
    try:
        for name, prec in (("fp32_3xtf32_gram", 1), ("mixed_1xtf32_gram", 0)):
            _lib.set_gram_precision(prec)
            call(iters)
            torch.cuda.synchronize()
            err = {"pose_err_vs_fp64": rel(poses.double().cpu().numpy(), r.poses),
                   "disp_err_vs_fp64": rel(disps.double().cpu().numpy(), r.disps)}
            ms = device_time(lambda: call(p["iters"]), steps)
            forms[name] = dict(err, gn_iters_per_s=round(p["iters"] * 1e3 / ms, 2))
    finally:
        _lib.set_gram_precision(1)
    return {"iterations": iters, "forms": forms,
            "definition": "max |x - x_fp64| / max |x_fp64| over the [300,7] poses / [300,43,77] disparities "
                          "after %d GN iterations; gn_iters_per_s device-timed at %d iterations per call"
                          % (iters, p["iters"]),
            "oracle_seconds": round(dt, 1)}


def run_reference(args, world, rank):
    """The reference's own ``droid_backends.ba`` (HI-SLAM2 src/droid.cpp + droid_kernels.cu compiled
    unmodified into oracle/_ref, Eigen replaced by the dense stand-in) on the same backend300
    workload: its CUDA kernels on this GPU, its host loops and solve on the host cores.  One step =
    one call of `iters` GN iterations, wall-clocked with a device sync (the op syncs itself)."""
    if rank != 0:
        return
    from hislam2_b200 import synth
    from oracle import build_ref
    ref = build_ref.load() if torch.cuda.is_available() else None
    p = synth.make_ba_problem(WORKLOAD, seed=0)
    common = {"metric": METRIC, "unit": UNIT, "n_gpus": world, "steps": args.steps, "higher_is_better": True,
              "scaling": "weak", "vs_baseline": None, "data": "synthetic (seeded)", "impl": "reference"}
    if ref is None:
        # the reference extension is not built: time the pure-PyTorch port on the host cores instead
        cb = cpu_baseline(p, target_seconds=max(2.0, 120.0 / max(1, args.steps + args.warmup)))
        line = dict(common, value=cb["value"], warmup=args.warmup, ms_per_step=round(1e3 / cb["value"], 3),
                    dtype="f32", config=dict(CONFIG, parallelism="host cores"), cpu_baseline=cb,
                    e2e={"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
        print(json.dumps(line), flush=True)
        return
    dev = torch.device("cuda:0")
    q = {k: (v.to(dev) if torch.is_tensor(v) else v) for k, v in p.items()}
    init_p, init_d = q["poses"].clone(), q["disps"].clone()
    poses, disps = init_p.clone(), init_d.clone()

    def call(iters):
        poses.copy_(init_p)
        disps.copy_(init_d)
        torch.cuda.synchronize()
        t = time.perf_counter()
        ref.ba(poses, disps, q["intrinsics"], q["targets"], q["weights"], q["eta"], q["ii"], q["jj"], q["t0"],
               q["t1"], iters, q["lm"], q["ep"], False)
        torch.cuda.synchronize()
        return time.perf_counter() - t

    t_one = call(1)
    budget = 150.0 / max(1, args.steps + args.warmup)
    iters = int(max(1, min(q["iters"], budget // max(t_one, 1e-3))))
    for _ in range(args.warmup):
        call(iters)
    times = [call(iters) for _ in range(args.steps)]
    total = float(sum(times))
    value = args.steps * iters / total
    corr = reference_corr_lookup(ref, args, dev)
    alt = reference_altcorr(ref, dev)
    line = dict(common, value=round(value, 4), warmup=args.warmup, ms_per_step=round(1e3 * total / args.steps, 3),
                dtype="f32 kernels, f64 host solve",
                config=dict(CONFIG, parallelism="single GPU + host", iterations_per_step=iters),
                cpu_baseline={"value": round(value, 4), "unit": UNIT, "cores": 1, "kind": "reference",
                              "cpu_model": cpu_model(),
                              "sample": "HI-SLAM2's own droid_backends.ba compiled unmodified (Eigen's SimplicialLLT "
                                        "replaced by a dense natural-order LLT stand-in) on the full backend300 "
                                        "window, %d GN iteration(s) per step: CUDA kernels on the GPU, host loops, "
                                        "triplet assembly and the solve on one host core" % iters},
                e2e={"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                corr_lookup=corr, altcorr=alt)
    print(json.dumps(line), flush=True)


def altcorr_inputs(dev, dtype=torch.float16):
    """The backend's correlation workload: 300 keyframes of 128-channel features at 43x77
    (~N(0,1)/sqrt(128)), the 4-level pooled pyramid, and the 6000 edges' reprojected
    coordinates (+ N(0,1) px) in the global BA loop's chunks of two source frames
    (factor_graph.py:253-260), coordinates pre-scaled per level, [1, m, 2, H, W]."""
    from hislam2_b200 import synth
    from hislam2_b200.corr import _pool_pyramid
    p = synth.make_ba_problem(WORKLOAD, seed=0)
    g = torch.Generator().manual_seed(17)
    K, H, W, C, L = 300, 43, 77, 128, 4
    fmaps = (torch.randn(K, C, H, W, generator=g) / np.sqrt(C)).to(dev, dtype)
    pyr = [lv[None].contiguous() for lv in _pool_pyramid(fmaps, L)]
    ii, jj = p["ii"].to(dev), p["jj"].to(dev)
    coords = synth.reproject(p["poses_gt"], p["disps_gt"], p["intrinsics"], p["ii"], p["jj"]).float()
    coords = (coords + torch.randn(coords.shape, generator=g)).permute(0, 3, 1, 2).contiguous().to(dev)
    chunks = []
    for i in range(0, int(p["jj"].max()) + 1, 2):
        v = ((ii >= i) & (ii < i + 2)).nonzero().flatten()
        if v.numel():
            chunks.append((ii[v].contiguous(), jj[v].contiguous(),
                           [(coords[v] / 2 ** lvl)[None].contiguous() for lvl in range(L)]))
    return fmaps, pyr, chunks


def reference_altcorr(ref, dev):
    """The reference's altcorr_forward (src/altcorr_kernel.cu, built in oracle/_ref) over the
    same 6000-edge backend pass as the `altcorr` leg (float16 features, radius 3, 4 levels),
    one pass timed with CUDA events after one warm-up chunk."""
    _, pyr, chunks = altcorr_inputs(dev)

    def run(chs):
        for ci, cj, crd in chs:
            for lvl in range(4):
                ref.altcorr_forward(pyr[0], pyr[lvl], crd[lvl], ci, cj, 3)

    run(chunks[:1])
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    run(chunks)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    del pyr, chunks
    torch.cuda.empty_cache()
    return {"ms_per_pass": round(ms, 2), "edges_per_s": round(6000 / (ms / 1e3), 1),
            "config": "300 keyframes, 6000 edges in chunks of two source frames, 43x77, 128 channels fp16, "
                      "radius 3, 4 levels; one pass"}


def reference_corr_lookup(ref, args, dev):
    """The reference's corr_index_forward on the same 4-level radius-4 frontend lookup as ours."""
    pyr, crds, r, bytes_per = frontend_lookup_inputs(dev)

    E = pyr[0].shape[0]
    halves = [(0, E // 2), (E // 2, E)]   # its 32-bit accessors take < 2^31 elements per volume

    def step():
        for lvl in range(4):
            for a, b in halves:
                ref.corr_index_forward(pyr[lvl][a:b], crds[lvl][a:b], r)

    ms = device_time(step, args.steps)
    del pyr
    torch.cuda.empty_cache()
    return {"value": round(bytes_per / (ms / 1e3) / 1e9, 2), "unit": "GB/s", "ms_per_lookup": round(ms, 4),
            "config": "258 edges (frontend window) in two calls of 129 (the op's 32-bit accessors take < 2^31 "
                      "elements per volume), 43x77, 4 levels, radius 4, fp16 volumes"}


# ------------------------------------------------------------ profiler cases
def profile_ba(args, dev):
    """One backend300 ba call (--profile-iters GN iterations) and one radius-4 fp16
    lookup over the first --profile-edges edges of the frontend window.  About 1 GB
    on the device: small enough for an ncu capture of single kernels."""
    import droid_backends
    from hislam2_b200 import synth
    p = synth.make_ba_problem(WORKLOAD, seed=0, device=dev)
    poses, disps = p["poses"].clone(), p["disps"].clone()
    droid_backends.ba(poses, disps, p["intrinsics"], p["targets"], p["weights"], p["eta"], p["ii"], p["jj"],
                      p["t0"], p["t1"], args.profile_iters, p["lm"], p["ep"], False)
    c = synth.make_corr_problem("frontend", seed=0, device=dev, num_edges=args.profile_edges,
                                dtype=torch.float16)
    f = c["fmaps"]
    H, W = f.shape[2:]
    vol = torch.matmul((f[c["ii"]].flatten(2) / 4).transpose(1, 2), f[c["jj"]].flatten(2) / 4)
    vol = vol.view(-1, H, W, H, W).contiguous()
    droid_backends.corr_index_forward(vol, c["coords"].permute(0, 3, 1, 2).contiguous(), 4)


def profile_volume(args, dev):
    """One corr_volume call (float16, 4 levels) on the first --profile-edges edges of the
    frontend window (about 1.5 GB of pyramid at 64 edges)."""
    from hislam2_b200 import backends, synth
    c = synth.make_corr_problem("frontend", seed=0, device=dev, num_edges=args.profile_edges, dtype=torch.float16)
    for _ in range(args.profile_iters):
        backends.corr_volume(c["fmaps"], c["fmaps"], c["ii"], c["jj"])


def profile_adjoint(args, dev):
    """One ba_adjoint call on the 2 x 7-frame 48x64 clip (the differentiation config)."""
    from hislam2_b200 import backends, synth
    p = synth.make_ba_problem("clips2x7", seed=0, device=dev)
    poses, disps = p["poses"].clone(), p["disps"].clone()
    dx, dz, _ = backends.ba(poses, disps, p["intrinsics"], p["targets"], p["weights"], p["eta"], p["ii"], p["jj"],
                            p["t0"], p["t1"], 1, p["lm"], p["ep"], False)
    backends.ba_adjoint(p["poses"], p["disps"], p["intrinsics"], p["targets"], p["weights"], p["eta"][:dz.shape[0]],
                        p["ii"], p["jj"], p["t0"], p["t1"], p["lm"], p["ep"], dx, torch.ones_like(dx),
                        torch.ones_like(dz))


def profile_batch(args, dev):
    """One batched LM iteration over the first --profile-edges windows of the batching workload."""
    from hislam2_b200 import backends, synth
    ws = [{k: (v.to(dev) if torch.is_tensor(v) else v) for k, v in w.items()}
          for w in synth.make_batch_problems(num_windows=min(64, args.profile_edges), seed=0)]
    plan = backends.BABatch(ws, 1e-4, 0.1)
    plan.run(args.profile_iters)


def profile_altcorr(args, dev):
    """AltCorrBlock (float16, radius 3, 4 levels, pyramid packed channel-last) on the
    first --profile-edges edges of the 300-keyframe window: 4 altcorr_fwd_packed launches."""
    from hislam2_b200 import synth
    from hislam2_b200.corr import AltCorrBlock
    p = synth.make_ba_problem(WORKLOAD, seed=0)
    g = torch.Generator().manual_seed(17)
    f = (torch.randn(1, 300, 128, 43, 77, generator=g) / np.sqrt(128)).half().to(dev)
    E = min(args.profile_edges, p["ii"].numel())
    ii, jj = p["ii"][:E].to(dev), p["jj"][:E].to(dev)
    crd = synth.reproject(p["poses_gt"], p["disps_gt"], p["intrinsics"], p["ii"][:E], p["jj"][:E]).float()
    crd = (crd + torch.randn(crd.shape, generator=g))[None].contiguous().to(dev)
    blk = AltCorrBlock(f, num_levels=4, radius=3)
    with torch.no_grad():
        for _ in range(args.profile_iters):
            blk(crd, ii, jj)


PROFILE_CASES = {"ba": profile_ba, "volume": profile_volume, "adjoint": profile_adjoint, "batch": profile_batch,
                 "altcorr": profile_altcorr}


def main():
    args = parse()
    if args.profile_case is not None:
        dev = torch.device("cuda:0")
        torch.cuda.set_device(dev)
        PROFILE_CASES[args.profile_case](args, dev)
        torch.cuda.synchronize()
        print("profile case %s: done" % args.profile_case)
        return
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
