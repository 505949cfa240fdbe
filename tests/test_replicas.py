"""The multi-rank host logic on CPU with two gloo ranks: the replicas' camera
shares, the max-over-ranks job time, and the view-sharded round's score
exchange and argmax (equal on every rank to the single-process choice)."""
import math
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from splatfield_b200 import replicas


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def scores_for(n_views):
    # Ties on purpose: views 3 and 9 share the maximum; the first must win.
    return [math.sin(1.7 * v) if v not in (3, 9) else 5.0 for v in range(n_views)]


def worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = replicas.max_over_ranks(1.5 + rank, dist)
        n_views = 13
        full = scores_for(n_views)
        local = {v: full[v] for v in replicas.owned_views(n_views, rank, world)}
        merged = replicas.gather_view_scores(local, n_views, dist)
        calls = []
        scores, best = replicas.sharded_round(n_views, lambda views: (calls.append(list(views)),
                                                                      [full[v] for v in views])[1], dist)
        out[rank] = (t, merged, replicas.best_view(merged), scores, best, calls)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_time_and_best_view():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(worker, args=(world, free_port(), out), nprocs=world, join=True, start_method="spawn")
    want_scores = scores_for(13)
    for rank in range(world):
        t, merged, best, scores, best2, calls = out[rank]
        assert t == 2.5
        assert merged == want_scores
        assert best == (3, 5.0)
        # The sharded round: each rank scored only its own views, once.
        assert calls == [replicas.owned_views(13, rank, world)]
        assert scores == want_scores and best2 == (3, 5.0)


def test_replica_share_covers_the_orbit():
    cams = list(range(30))
    shares = [replicas.replica_share(cams, r, 4) for r in range(4)]
    assert all(len(s) == 30 for s in shares)
    # The first 30 / 4 frames of the ranks together visit distinct cameras.
    firsts = [c for s in shares for c in s[:7]]
    assert len(set(firsts)) == len(firsts)
    assert replicas.owned_views(10, 1, 3) == [1, 4, 7]


def test_single_process_fallbacks():
    assert replicas.max_over_ranks(3.0) == 3.0
    assert replicas.gather_view_scores({1: 2.0}, 3) == [-math.inf, 2.0, -math.inf]
    assert replicas.best_view([-math.inf, -math.inf]) == (0, -math.inf)
