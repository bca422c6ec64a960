"""Multi-rank tracer sharding (croma-fp_b200/shard.py) on CPU.

The partition helpers are checked against direct restatements of the
reference's rules, and a world-size-2 gloo run shards one snapshot of
tracers by LPT, advances each shard with the oracle, gathers the rows and
compares them with a single-process run of all tracers: tracers are
independent, so the sharded result must be identical.
"""
import os
import socket
import sys

import numpy as np
import pytest

from conftest import load_package

load_package()
from croma_fp_b200 import config, shard, synth  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def _reference_lpt(weights, nthreads):
    """The assignment loop of src/tracer_fp_batch.c:915-937, transliterated."""
    tasks = sorted(range(len(weights)), key=lambda i: (-int(weights[i]), i))
    loads = [0] * nthreads
    part = [0] * len(weights)
    for i in tasks:
        best = 0
        for t in range(1, nthreads):
            if loads[t] < loads[best]:
                best = t
        part[i] = best
        loads[best] += int(weights[i])
    return np.array(part)


def test_contiguous_covers_every_tracer_once():
    for n, world in ((10, 3), (65536, 8), (5, 8), (1, 1)):
        parts = [shard.contiguous(n, world, r) for r in range(world)]
        allidx = np.concatenate(parts)
        assert np.array_equal(np.sort(allidx), np.arange(n))
        sizes = [p.size for p in parts]
        assert max(sizes) - min(sizes) <= 1


def test_lpt_matches_reference_rule_and_balances():
    rng = np.random.default_rng(3)
    nsub = rng.integers(10, 501, 2000)
    w = shard.task_weights(nsub, shard.coeff_segments(nsub))
    for k in (2, 3, 8):
        part = shard.lpt_assign(w, k)
        assert np.array_equal(part, _reference_lpt(w, k))
        assert shard.imbalance(w, part, k) < 1.01
    idx = [shard.lpt_indices(w, 4, r) for r in range(4)]
    assert np.array_equal(np.sort(np.concatenate(idx)), np.arange(w.size))


def test_coeff_segments_match_oracle():
    import pyoracle
    cfg = config.config1(nb=128)
    o = pyoracle.Oracle(cfg)
    nsub = np.array([1, 2, 3, 4, 7, 8, 15, 16, 31, 63, 64, 65, 100, 500, 1000, 10 ** 6])
    got = shard.coeff_segments(nsub)
    want = np.array([o.coeff_segments(int(n), True) for n in nsub])
    assert np.array_equal(got, want)
    assert np.all(shard.coeff_segments(nsub, allow_interp=False) == 1)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, nt, out_path):
    sys.path.insert(0, HERE)
    sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
    import torch.distributed as dist
    from conftest import load_package as lp
    lp()
    from croma_fp_b200 import config as cf, shard as sd, synth as sy
    import pyoracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        cfg = cf.config0(nsub_max=120)
        w = sy.Workload(cfg, nt, 100, seed=17)
        o = pyoracle.Oracle(cfg)
        isnap = 40
        args = w.snapshot_args(isnap)
        ic = o.ic_row(args[2])
        nsub, _, _, _ = o.nsub(args[5], args[0], np.concatenate([ic[0], [ic[1], ic[2]]]))
        weights = sd.task_weights(nsub, sd.coeff_segments(nsub))
        mine = sd.lpt_indices(weights, world, rank)
        gp, ge = o.grid(0), o.grid(1)
        crp, cre = sy.initial_state((gp[0], gp[1]), (ge[0], ge[1]), nt, cfg.species)
        lc, le = crp[mine].copy(), cre[mine].copy()
        cur, nxt = args[0][:, mine].copy(), args[1][:, mine].copy()
        o.snapshot(cur, nxt, *args[2:], np.zeros_like(lc), np.zeros_like(le), lc, le, mass=w.mass[mine])
        full = sd.gather_rows(le, mine, nt, dist)
        tmax = sd.max_over_ranks(float(rank + 1), dist)
        if rank == 0:
            np.savez(out_path, cre=full, tmax=tmax, sizes=np.array([mine.size]))
    finally:
        dist.destroy_process_group()


def test_sharded_snapshot_equals_single_process(tmp_path):
    import torch.multiprocessing as mp
    import pyoracle
    nt, world = 40, 2
    out = str(tmp_path / "sharded.npz")
    mp.start_processes(_worker, args=(world, _free_port(), nt, out), nprocs=world, join=True,
                       start_method="spawn")
    d = np.load(out)
    assert float(d["tmax"]) == 2.0
    cfg = config.config0(nsub_max=120)
    w = synth.Workload(cfg, nt, 100, seed=17)
    o = pyoracle.Oracle(cfg)
    gp, ge = o.grid(0), o.grid(1)
    crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), nt, cfg.species)
    args = w.snapshot_args(40)
    o.snapshot(*args, np.zeros_like(crp), np.zeros_like(cre), crp, cre, mass=w.mass)
    assert np.array_equal(d["cre"], cre)
