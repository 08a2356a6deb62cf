"""Learned warm start: training on fields the solver generates, and evaluation.

Training (``train``): solver instances run in record mode; after every time
step the network takes ``updates`` Adam steps on that step's pair (features
at the start of the step -> realised enthalpy and pressure increments), all on
the GPU with the tensor-core kernels of k_cnn.cu.

Data-parallel training (``train`` with a process group): each rank solves its
own share of the decks and, after every backward pass, the ranks' gradients
are averaged with one all-reduce (NCCL over NVLink for CUDA tensors, or gloo)
before the Adam step, so every rank keeps the same parameters.

Evaluation (``evaluate``): the same deck is solved twice, plainly and with
the network's prediction as the starting guess of every step (rejected when
it raises the step's initial energy residual); the outer-iteration counts,
device times, acceptance counts and the final fields are returned.
"""
from __future__ import annotations

import time
from typing import Dict, List, Sequence

import numpy as np

import amcfd


class DeviceArray:
    """Zero-copy view of a device pointer for torch.as_tensor (FP32)."""

    def __init__(self, ptr: int, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f4",
                                         "data": (int(ptr), False), "version": 3}


def device_view(ptr: int, shape):
    import torch
    return torch.as_tensor(DeviceArray(ptr, shape), device="cuda")


def average_grads(net, group=None) -> None:
    """Replace the network's gradients by their mean over the ranks of `group`
    (torch.distributed; the default group when None).  Every rank must call it
    the same number of times.  The gradients go through a CUDA tensor when the
    group's backend is NCCL, a CPU tensor otherwise."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    if world == 1:
        return
    t = torch.from_numpy(net.grads())
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    net.set_grads((t / world).cpu().numpy())


def shard(deck_paths: Sequence[str], rank: int, world: int) -> List[str]:
    """This rank's decks (every world-th from `rank`); the deck count must divide
    evenly, so that every rank runs the same number of updates (all-reduces)."""
    if len(deck_paths) % world:
        raise ValueError(f"{len(deck_paths)} decks do not split evenly over {world} ranks")
    return list(deck_paths[rank::world])


def train(net: amcfd.Net, deck_paths: Sequence[str], steps: int, lr: float = 1e-3, updates: int = 4,
          precision: int = amcfd.PREC_FP32, order: int = amcfd.ORDER_REDBLACK, device: int = 0,
          group=None) -> List[float]:
    """Online training on every step of every deck; returns the loss history.

    With `group` (a torch.distributed process group, or True for the default
    one) each rank trains on its shard of `deck_paths` and the gradients are
    averaged over the ranks before every Adam step."""
    losses: List[float] = []
    if group is not None:
        import torch.distributed as dist
        grp = None if group is True else group
        deck_paths = shard(deck_paths, dist.get_rank(grp), dist.get_world_size(grp))
    for path in deck_paths:
        s = amcfd.Solver(amcfd.Deck(path), order=order, precision=precision, device=device, use_graphs=1)
        s.ws_attach(net, amcfd.WS_RECORD)
        feat, target = s.ws_buffers()
        nk, nj, ni = s.shape
        for _ in range(steps):
            s.step()
            for _ in range(updates):
                net.forward(feat, (ni, nj, nk))
                losses.append(net.backward(target))
                if group is not None:
                    average_grads(net, None if group is True else group)
                net.adam(lr)
        s.ws_attach(None, amcfd.WS_OFF)
        s.close()
    return losses


def evaluate(net: amcfd.Net, deck_path: str, steps: int, precision: int = amcfd.PREC_FP32,
             order: int = amcfd.ORDER_REDBLACK, device: int = 0, ref_maxit: int = 200,
             mode: int = amcfd.WS_PREDICT) -> Dict:
    """Plain vs warm-started solve of the same deck, both against a reference
    solve that may take up to ``ref_maxit`` outer iterations per step (the
    deck's own limit, 20 in the reference's decks, often stops a step before
    its convergence test passes)."""
    out = {}
    for run in ("plain", "warm", "reference"):
        deck = amcfd.Deck(deck_path)
        if run == "reference":
            deck.params.maxit = ref_maxit
        s = amcfd.Solver(deck, order=order, precision=precision, device=device, use_graphs=1)
        if run == "warm":
            s.ws_attach(net, mode)
        iters, fallback, resorh = [], [], []
        t0 = time.perf_counter()
        for _ in range(steps):
            r = s.step()
            iters.append(r["niter"])
            fallback.append(r["fallback"])
            resorh.append(r["resorh"])
        wall = time.perf_counter() - t0
        acc, rej = s.ws_stats()
        out[run] = {"iters": iters, "fallback": fallback, "resorh": resorh, "wall_s": wall, "accepted": acc,
                     "rejected": rej, "temp": s.get("temp"), "uvel": s.get("uvel"),
                     "dims": (r["alen"], r["depth"], r["width"])}
        s.close()
    p, w, ref = out["plain"], out["warm"], out["reference"]

    def err(a, f):
        return float(np.linalg.norm(a[f] - ref[f]) / max(np.linalg.norm(ref[f]), 1e-300))

    out["summary"] = {
        "steps": steps,
        "iters_plain": float(np.mean(p["iters"])), "iters_warm": float(np.mean(w["iters"])),
        "iters_reference": float(np.mean(ref["iters"])),
        "wall_plain_s": p["wall_s"], "wall_warm_s": w["wall_s"],
        "fallback_rate": w["rejected"] / max(1, w["accepted"] + w["rejected"]),
        "resorh_plain": float(np.mean(p["resorh"])), "resorh_warm": float(np.mean(w["resorh"])),
        "temp_err_plain": err(p, "temp"), "temp_err_warm": err(w, "temp"),
        "uvel_err_plain": err(p, "uvel"), "uvel_err_warm": err(w, "uvel"),
        "dims_plain": p["dims"], "dims_warm": w["dims"], "dims_reference": ref["dims"],
    }
    return out


# Tensor-core FLOPs per cell of one forward pass (padded channels, as executed):
# 2 x 27 taps x sum over layers of cin x cout.
FWD_FLOP_PER_CELL = 2 * 27 * (16 * 32 + 32 * 32 + 32 * 32 + 32 * 16)
# backward on the tensor cores: input-gradient convolutions of layers 3, 2, 1 and
# the weight-gradient contractions of all four layers (as many FLOPs as the forward)
BWD_TC_FLOP_PER_CELL = 2 * 27 * (16 * 32 + 32 * 32 + 32 * 32) + FWD_FLOP_PER_CELL


def bench_network(dims=(202, 102, 62), reps: int = 10, device: int = 0) -> Dict:
    """Forward/backward throughput of the network on a node grid (the config-3
    evaluation grid by default), CUDA-event timed, random features."""
    import torch
    ni, nj, nk = dims
    n = ni * nj * nk
    g = torch.Generator(device="cuda").manual_seed(5)
    feat = torch.randn((n, 11), device="cuda", generator=g)
    target = torch.randn((n, 2), device="cuda", generator=g) * 0.1
    net = amcfd.Net(device=device, seed=5)
    for _ in range(3):
        net.forward(feat.data_ptr(), dims)
        net.backward(target.data_ptr())
    f_ms, b_ms = [], []
    for _ in range(reps):
        net.forward(feat.data_ptr(), dims)
        net.backward(target.data_ptr())
        f, b = net.last_ms()
        f_ms.append(f)
        b_ms.append(b)
    net.close()
    f, b = float(np.median(f_ms)), float(np.median(b_ms))
    return {"cells": n, "fwd_ms": f, "bwd_ms": b,
            "fwd_tflops": FWD_FLOP_PER_CELL * n / (f * 1e-3) / 1e12,
            "bwd_tc_tflops": BWD_TC_FLOP_PER_CELL * n / (b * 1e-3) / 1e12}


if __name__ == "__main__":
    import argparse
    import json
    import os
    import tempfile

    import amcfd_decks as D

    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--bench", action="store_true", help="network throughput on the config-3 grid")
    ap.add_argument("--eval", type=int, default=0, help="train, then evaluate N steps of config 3")
    ap.add_argument("--train-steps", type=int, default=60)
    ap.add_argument("--train-instances", type=int, default=8,
                    help="config-2 instances to train on (of the seeded 64; steps x instances pairs)")
    args = ap.parse_args()
    if args.bench:
        print(json.dumps(bench_network()))
    if args.eval:
        tmp = tempfile.mkdtemp(prefix="amcfd_ws_")
        # training decks: the first config-2 instances of the seeded sweep (draws of
        # grid size, power, speed, radius)
        decks = D.config2(n=64, steps=args.train_steps + 1)[:args.train_instances]
        paths = [d.write(os.path.join(tmp, d.name)) for d in decks]
        net = amcfd.Net(seed=3)
        t0 = time.perf_counter()
        losses = train(net, paths, steps=args.train_steps, lr=1e-3, updates=4)
        train_s = time.perf_counter() - t0
        held = D.config3_eval(steps=args.eval + 1).write(os.path.join(tmp, "config3"))
        ev = evaluate(net, held, args.eval, ref_maxit=60)
        s = ev["summary"]
        s.update({"train_pairs": len(paths) * args.train_steps, "train_s": train_s,
                  "loss_first": losses[0], "loss_last": losses[-1]})
        print(json.dumps(s))
