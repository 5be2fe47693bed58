"""Multi-rank plumbing of the BA bench and of multi-window runs, on CPU with the gloo
backend and two ranks: each rank solves its own window with the float64 oracle, the
timing collectives (barrier, MAX reduce) agree on every rank, and windows are spread
over ranks with none lost or solved twice."""

import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from hislam2_b200 import replicas

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "hi-slam2_b200")]
    import oracle
    from hislam2_b200 import replicas as rp, synth

    w, r, _ = rp.env_ranks()
    rp.init(w, r, backend="gloo", timeout_s=60)
    # each rank solves its own window (seeded by rank), one GN iteration of the small frontend
    p = synth.make_ba_problem("frontend_small", seed=rp.window_seed(r))
    f = lambda k: p[k].numpy().astype(np.float64)  # noqa: E731
    poses = oracle.ba.ba(f("poses"), f("disps"), f("intrinsics"), f("targets"), f("weights"), f("eta"),
                         p["ii"].numpy(), p["jj"].numpy(), p["t0"], p["t1"], 1, p["lm"], p["ep"]).poses
    rp.barrier(w)
    fake_ms = 10.0 * (r + 1)                     # stands in for a rank's device-timed duration
    mx = rp.max_over_ranks(fake_ms, w)
    rate = rp.throughput(8, mx, w)
    mine = list(rp.shard(7, w, r))
    np.savez(os.path.join(out_dir, "rank%d.npz" % r), poses=poses, mx=mx, rate=rate, mine=np.array(mine))
    rp.barrier(w)
    rp.finalize(w)


def test_two_gloo_ranks(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [np.load(tmp_path / ("rank%d.npz" % r)) for r in range(world)]
    # the MAX reduce gives the slowest rank's time on every rank, and the rate uses it
    assert all(float(x["mx"]) == 20.0 for x in res)
    assert all(abs(float(x["rate"]) - 8 * world / 0.020) < 1e-9 for x in res)
    # ranks solved different windows
    assert not np.allclose(res[0]["poses"], res[1]["poses"])
    # the windows are covered exactly once
    got = sorted(int(i) for x in res for i in x["mine"])
    assert got == list(range(7))


def test_rank_solves_same_window_as_single_process():
    """A rank's window is the one a single process with that seed would solve."""
    import oracle
    from hislam2_b200 import synth
    p = synth.make_ba_problem("frontend_small", seed=replicas.window_seed(1))
    q = synth.make_ba_problem("frontend_small", seed=1)
    assert torch.equal(p["poses"], q["poses"]) and torch.equal(p["ii"], q["ii"])
    assert oracle is not None


@pytest.mark.parametrize("n,world", [(0, 2), (1, 2), (7, 3), (300, 8), (5, 8)])
def test_shard_covers_once(n, world):
    seen = []
    for r in range(world):
        s = replicas.shard(n, world, r)
        assert len(s) in (n // world, n // world + 1)
        seen.extend(s)
    assert sorted(seen) == list(range(n))


def test_shard_and_throughput_reject_bad_input():
    with pytest.raises(ValueError):
        replicas.shard(4, 2, 2)
    with pytest.raises(ValueError):
        replicas.throughput(8, 0.0, 1)


def test_reference_arm_other_ranks_exit_quietly():
    """Under torchrun only rank 0 of the reference arm runs; the others exit 0 printing nothing."""
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1", MASTER_PORT="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
