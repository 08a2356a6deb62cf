"""Parameter sweep: instance sharding over ranks and the batched GPU runner.

CPU tests cover the longest-processing-time partition and the N>1 path (two
gloo ranks, each solving its shard with the oracle, results gathered on the
host); the GPU test checks that amcfd_run_batch, with several instances in
flight on one GPU, gives every instance exactly the results of running it alone.
"""
import itertools
import os
import socket

import numpy as np
import pytest

import amcfd
import amcfd_decks as D
import amcfd_sweep as S


def test_shard_covers_every_instance_once_largest_first():
    rng = np.random.default_rng(7)
    costs = [int(c) for c in rng.integers(1, 1000, size=37)]
    for world in (1, 2, 3, 8, 40):
        parts = S.shard(costs, world)
        assert len(parts) == world
        flat = sorted(itertools.chain.from_iterable(parts))
        assert flat == list(range(len(costs)))
        for p in parts:
            assert [costs[q] for q in p] == sorted((costs[q] for q in p), reverse=True)
        assert parts == S.shard(costs, world)  # deterministic


def test_shard_lpt_bound_against_brute_force():
    rng = np.random.default_rng(11)
    for trial in range(20):
        n = int(rng.integers(1, 9))
        costs = [int(c) for c in rng.integers(1, 50, size=n)]
        for world in (2, 3):
            parts = S.shard(costs, world)
            got = max(sum(costs[q] for q in p) for p in parts)
            best = min(max(sum(c for c, a in zip(costs, asg) if a == r) for r in range(world))
                       for asg in itertools.product(range(world), repeat=n))
            assert got * 3 <= best * 4, (costs, world, got, best)


def test_instance_cost_counts_interior_cells_times_steps():
    assert S.instance_cost((12, 8, 6), 3) == 10 * 6 * 4 * 3
    assert S.instance_cost((2, 8, 6), 3) == 0


def test_config2_sweep_decks():
    decks = D.config2(n=64)
    assert len(decks) == 64
    again = D.config2(n=64)
    assert [d.power for d in decks] == [d.power for d in again]  # seeded
    for d in decks:
        nx = d.x_zones[0][1]
        assert 60 <= nx <= 240
        assert 100.0 <= d.power <= 400.0
        assert 40e-6 <= d.radius <= 80e-6
        assert 0.5 <= d.single_track[3] <= 1.5


def _sweep_decks(directory, n=3, steps=2):
    out = []
    for q in range(n):
        d = D.small(f"sw{q}", nx=14 + 2 * q, ny=10, nz=6, steps=steps, power=250.0 + 40 * q)
        out.append(d.write(os.path.join(directory, f"sw{q}")))
    return out


def oracle_runner(paths, steps):
    """Runs a shard on the CPU with the oracle (test infrastructure only)."""
    import oracle_py
    res = []
    for p in paths:
        o = oracle_py.Oracle(amcfd.Deck(p))
        rep = None
        for _ in range(steps):
            rep = o.step()
        res.append({k: rep[k] for k in S.RESULT_KEYS})
    return res


def _gloo_worker(rank, world, port, paths, steps, outdir):
    import datetime
    import json

    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        out = S.run_sweep(paths, steps, runner=oracle_runner)
        with open(os.path.join(outdir, f"rank{rank}.json"), "w") as f:
            json.dump({"results": out["results"], "shards": out["shards"]}, f)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sweep_two_gloo_ranks_match_one_process(tmp_path, oracle_lib):
    import json

    import torch.multiprocessing as mp
    paths = _sweep_decks(str(tmp_path), n=3, steps=2)
    single = S.run_sweep(paths, 2, runner=oracle_runner, rank=0, world=1)
    mp.spawn(_gloo_worker, args=(2, _free_port(), paths, 2, str(tmp_path)), nprocs=2, join=True)
    outs = [json.load(open(os.path.join(tmp_path, f"rank{r}.json"))) for r in range(2)]
    assert outs[0]["results"] == outs[1]["results"]
    assert sorted(len(s) for s in outs[0]["shards"]) == [1, 2]
    for a, b in zip(outs[0]["results"], single["results"]):
        assert a == b


def test_run_batch_rejects_bad_arguments(lib):
    import ctypes as C
    assert lib.amcfd_run_batch(None, 1, 1, 0, None, None) == -1
    arr = (C.c_void_p * 1)(None)
    assert lib.amcfd_run_batch(arr, 1, 1, 0, None, None) == -1
    assert lib.amcfd_run_batch(arr, 0, 1, 0, None, None) == 0
    assert lib.amcfd_run_batch(arr, 1, 1, 65, None, None) == -1


@pytest.mark.gpu
def test_batch_on_one_gpu_equals_instances_alone(tmp_path):
    paths = _sweep_decks(str(tmp_path), n=4, steps=3)
    for prec, order in ((amcfd.PREC_FP64, amcfd.ORDER_EXACT), (amcfd.PREC_FP32, amcfd.ORDER_REDBLACK)):
        out = S.run_sweep(paths, 3, runner=S.gpu_runner(0, prec, order, nthreads=4), rank=0, world=1)
        for q, p in enumerate(paths):
            s = amcfd.Solver(amcfd.Deck(p), order=order, precision=prec)
            for _ in range(3):
                rep = s.step()
            s.close()
            for k in S.RESULT_KEYS:
                assert out["results"][q][k] == rep[k], (q, k, out["results"][q][k], rep[k])


@pytest.mark.gpu
def test_batch_matches_oracle_in_fp64(tmp_path):
    paths = _sweep_decks(str(tmp_path), n=3, steps=2)
    gpu = S.run_sweep(paths, 2, runner=S.gpu_runner(0, amcfd.PREC_FP64, amcfd.ORDER_EXACT), rank=0, world=1)
    ref = S.run_sweep(paths, 2, runner=oracle_runner, rank=0, world=1)
    for a, b in zip(gpu["results"], ref["results"]):
        assert a["niter"] == b["niter"] and a["itertot"] == b["itertot"]
        assert abs(a["tpeak"] - b["tpeak"]) <= 1e-8 * abs(b["tpeak"])
        for k in ("alen", "depth", "width"):
            assert abs(a[k] - b[k]) <= 1e-8 * max(abs(b[k]), 1e-12), (k, a[k], b[k])
