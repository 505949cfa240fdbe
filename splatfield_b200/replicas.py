"""Running the render path on several GPUs: one process per GPU.

A frame has no exchange step (every tile needs the whole sorted list of its
splats), so frames run as independent replicas: each rank renders its share
of the cameras and the job time is the slowest rank's. A segmentation round
shards by view: the candidate views are independent given the read-only
splats and posterior, so rank r scores views r, r + world, ... and the one
exchange is an all-gather of the per-view EIG scalars before the argmax
(src/seg/active.rs:113-129 picks the first strictly greatest).

Works with any torch.distributed backend: NCCL with CUDA tensors on GPUs,
gloo with CPU tensors (the tests).
"""
from __future__ import annotations

import math


def replica_share(items, rank: int, world: int):
    """The rank's share of a round-robin list (item i + k * world for rank i),
    cycled to the list's length so every rank does equal work."""
    n = len(items)
    return [items[(rank + world * i) % n] for i in range(n)]


def owned_views(n_views: int, rank: int, world: int) -> list[int]:
    """Views rank ``rank`` scores: v with v % world == rank."""
    return list(range(rank, n_views, world))


def _device(dist):
    import torch

    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")


def max_over_ranks(value: float, dist=None) -> float:
    """The maximum of ``value`` over the ranks (the job time of a step timed
    on every rank); ``value`` itself without a process group."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=_device(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_view_scores(local: dict[int, float], n_views: int, dist=None) -> list[float]:
    """Every view's score on every rank from each rank's owned views (one
    all-reduce of an n_views vector; views a rank does not own hold -inf)."""
    scores = [-math.inf] * n_views
    for v, e in local.items():
        scores[v] = float(e)
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return scores
    import torch

    t = torch.tensor(scores, dtype=torch.float64, device=_device(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def best_view(scores: list[float]):
    """(index, score) of the first strictly greatest score, starting from
    -inf as select_view does; (0, -inf) when no score beats it."""
    best, best_score = 0, -math.inf
    for v, e in enumerate(scores):
        if e > best_score:
            best, best_score = v, e
    return best, best_score


def sharded_round(n_views: int, score_owned, dist=None):
    """One view-sharded round: this rank scores its owned views with
    ``score_owned(views) -> scores`` (a batched round over those views on
    this rank's GPU), then the ranks exchange the scores and pick the best
    view. Returns (all scores, (best view, its score)), equal on every rank.
    Every rank takes the same collective steps: one all-reduce."""
    rank = dist.get_rank() if dist is not None and dist.is_initialized() else 0
    world = dist.get_world_size() if dist is not None and dist.is_initialized() else 1
    views = owned_views(n_views, rank, world)
    local = dict(zip(views, score_owned(views))) if views else {}
    scores = gather_view_scores(local, n_views, dist)
    return scores, best_view(scores)
