"""Launch-shape tuner of the batched BA (``backends.BABatch``).

The persistent batched kernel has two shape knobs: the number of pixel splits of each
depth frame's Schur Gram (``gram_split``: more, smaller Gram units balance frames
with many Schur rows across SMs but add atomics into the FP64 system) and the CTAs
per SM of the persistent grid (``ctas_per_sm``: 1 gives each unit a whole SM's
issue slots, 2 overlaps one CTA's waits with another's work).  :func:`tune` times
every candidate on a workload with CUDA events (one LM iteration per launch, after a
warm-up) and returns the table of timings; :func:`save` / :func:`best` keep the
winner per workload name in ``ba_batch_tuning.json`` beside this file, which
``BABatch`` users read through :func:`best`.

    python -m hislam2_b200.autotune        # tunes the 64-window batching workload
"""

import json
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "ba_batch_tuning.json")
CANDIDATES = {"gram_split": [1, 2, 4, 8, 16], "ctas_per_sm": [1, 2]}
DEFAULT = {"gram_split": 4, "ctas_per_sm": 0}


def _time(windows, lm, ep, iters, cfg, reps):
    from . import backends
    init = [(w["poses"].clone(), w["disps"].clone()) for w in windows]

    def reset():
        for w, (p, d) in zip(windows, init):
            w["poses"].copy_(p)
            w["disps"].copy_(d)

    plan = backends.BABatch(windows, lm, ep, gram_split=cfg["gram_split"], ctas_per_sm=cfg["ctas_per_sm"])
    reset()
    plan.run(iters)
    best = None
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(reps):
        reset()
        torch.cuda.synchronize()
        e0.record()
        plan.run(iters)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / iters
        best = ms if best is None else min(best, ms)
    reset()
    plan.check()
    return best


def tune(windows, lm=1e-4, ep=0.1, iters=4, reps=3, candidates=None):
    """[(config, ms per LM iteration)] for every candidate, fastest first."""
    cand = candidates or CANDIDATES
    rows = []
    for gs in cand["gram_split"]:
        for cps in cand["ctas_per_sm"]:
            cfg = {"gram_split": gs, "ctas_per_sm": cps}
            rows.append((cfg, _time(windows, lm, ep, iters, cfg, reps)))
    rows.sort(key=lambda r: r[1])
    return rows


def load():
    if os.path.exists(TABLE):
        with open(TABLE) as f:
            return json.load(f)
    return {}


def best(workload):
    """Tuned knobs for `workload` (a name in the table), else the defaults."""
    entry = load().get(workload)
    return dict(entry["best"]) if entry else dict(DEFAULT)


def save(workload, rows, device_name):
    table = load()
    table[workload] = {"device": device_name, "best": rows[0][0],
                       "timings_ms_per_iteration": [dict(cfg, ms=round(ms, 4)) for cfg, ms in rows]}
    with open(TABLE, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
        f.write("\n")


def main():
    import argparse
    from . import synth
    ap = argparse.ArgumentParser()
    ap.add_argument("--windows", type=int, default=64)
    ap.add_argument("--out", default=None, help="write the table here instead of beside the package")
    a = ap.parse_args()
    global TABLE
    if a.out:
        TABLE = a.out
    dev = torch.device("cuda:0")
    ws = [{k: (v.to(dev) if torch.is_tensor(v) else v) for k, v in w.items()}
          for w in synth.make_batch_problems(num_windows=a.windows, seed=0)]
    rows = tune(ws)
    for cfg, ms in rows:
        print("%-40s %.4f ms / iteration" % (cfg, ms))
    save("batch%d" % a.windows, rows, torch.cuda.get_device_name(dev))
    print("best:", rows[0][0], "->", TABLE)


if __name__ == "__main__":
    main()
