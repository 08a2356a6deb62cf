"""Data-parallel training of the warm-start network.

CPU: two gloo ranks average their gradients with amcfd_warmstart.average_grads
(each rank holds a stand-in network whose gradients are a host array), and
decks are split over ranks so that every rank runs the same number of updates.
GPU: the network's gradient buffer can be replaced exactly (amcfd_net_set_grads),
and training through a one-rank process group gives the same losses and
parameters as training without one.
"""
import os
import socket

import numpy as np
import pytest

import amcfd_warmstart as W


class _HostNet:
    """Stand-in exposing the gradient accessors average_grads uses."""

    def __init__(self, g):
        self.g = np.asarray(g, dtype=np.float32)

    def grads(self):
        return self.g.copy()

    def set_grads(self, g):
        self.g = np.asarray(g, dtype=np.float32).copy()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, outdir):
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(100 + rank)
        net = _HostNet(rng.standard_normal(1000))
        np.save(os.path.join(outdir, f"g{rank}.npy"), net.g)
        W.average_grads(net)
        np.save(os.path.join(outdir, f"avg{rank}.npy"), net.g)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_average_their_gradients(tmp_path):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    g = [np.load(os.path.join(tmp_path, f"g{r}.npy")) for r in range(2)]
    avg = [np.load(os.path.join(tmp_path, f"avg{r}.npy")) for r in range(2)]
    assert np.array_equal(avg[0], avg[1])
    np.testing.assert_allclose(avg[0], (g[0] + g[1]) / 2, rtol=1e-6, atol=1e-7)


def test_decks_split_evenly_over_ranks():
    paths = [f"d{q}" for q in range(6)]
    parts = [W.shard(paths, r, 3) for r in range(3)]
    assert sorted(sum(parts, [])) == sorted(paths)
    assert all(len(p) == 2 for p in parts)
    with pytest.raises(ValueError):
        W.shard(paths, 0, 4)


@pytest.mark.gpu
def test_gradient_buffer_round_trip_and_one_rank_group(tmp_path):
    import datetime

    import torch.distributed as dist

    import amcfd
    import amcfd_decks as D
    net = amcfd.Net(seed=3)
    g = np.linspace(-1.0, 1.0, net.nparams, dtype=np.float32)
    net.set_grads(g)
    assert np.array_equal(net.grads(), g)
    net.close()

    path = D.small("dp", nx=24, ny=14, nz=10, steps=2).write(str(tmp_path))
    a, b = amcfd.Net(seed=5), amcfd.Net(seed=5)
    la = W.train(a, [path], steps=2, updates=2)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        lb = W.train(b, [path], steps=2, updates=2, group=True)
    finally:
        dist.destroy_process_group()
    assert la == lb
    assert np.array_equal(a.params(), b.params())
    a.close()
    b.close()
