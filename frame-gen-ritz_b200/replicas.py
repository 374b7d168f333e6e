"""Multi-GPU plumbing of the V1 path: one process per GPU, frame pairs partitioned across ranks, no collective on the
data path. Frame pairs are independent (a generated frame reads only its own pair), so a job of many pairs shards
across GPUs by pairs; a single frame is never split. The collectives that remain are off the data path:
  - the bench's timing: a barrier around the timed span and the max of the ranks' spans;
  - seed-net training, data-parallel: one all-reduce (sum) of the float32 gradient per step, the 1 / ranks folded
    into the Adam step (fg_seednet_adam_scaled).
Every function works on any torch.distributed backend (NCCL on GPUs; gloo on CPU for the tests) and degrades to the
single-process case when no process group is initialised.
"""
import heapq
import os
import socket
import subprocess
import sys
import time

import torch
import torch.distributed as dist


def world():
    """(rank, world size) of the current process group, (0, 1) without one"""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def pair_cost(width, height, multiplier):
    """the cost of one frame pair for partitioning: the pixels it moves (two frames read, multiplier - 1 generated
    frames written); the estimate and every synthesis are memory-bound passes over the pair's pixels"""
    return width * height * (multiplier + 1)


def shard_by_cost(costs, n_ranks):
    """Partition items of the given costs (bytes a pair moves, or pixels) over n_ranks: longest-processing-time
    greedy, the costliest item first to the least-loaded rank (ties to the lower rank, so every rank computes the same
    partition without communicating). Returns one list of item indices per rank, each in ascending order. The heaviest
    rank carries at most the mean load plus one item's cost."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0, r) for r in range(n_ranks)]
    shards = [[] for _ in range(n_ranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(s) for s in shards]


def round_robin(n_items, n_ranks):
    """item i to rank i mod n_ranks (pairs of equal cost, e.g. one resolution and format)"""
    return [list(range(r, n_items, n_ranks)) for r in range(n_ranks)]


def max_over_ranks(value, device=None):
    """the maximum of a per-rank float (a timed span in ms) over all ranks; every rank gets it"""
    rank, n = world()
    if n == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def timed_span_value(span_ms, items_per_rank, device=None):
    """the whole-job time per item: the slowest rank's span over the items of all ranks (weak scaling: every rank
    processes items_per_rank items in its span)"""
    _, n = world()
    return max_over_ranks(span_ms, device) / (items_per_rank * n)


class GradSync:
    """Data-parallel gradient exchange of the seed net: the flat float32 gradient (SeedNet.grad_buffer(), or any
    flat tensor on the process group's device) is all-reduced in place (sum) once per step; scale() is the factor the
    Adam step applies to it (1 / ranks), so every rank takes the step of the mean gradient over the global batch and
    the ranks' parameters stay identical."""

    def __init__(self):
        self.rank, self.n = world()

    def __call__(self, grad):
        if self.n > 1:
            dist.all_reduce(grad, op=dist.ReduceOp.SUM)
        return grad

    def scale(self):
        return 1.0 / self.n

    def rank_seed(self, seed):
        """the data seed of this rank (distinct crops per rank; the parameter initialisation uses the shared seed)"""
        return seed + 7919 * self.rank


def free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def spawn_ranks(script, argv, n):
    """A script asked for n GPUs without a launcher: run n copies of it, rank r on GPU r, with the variables a launcher
    sets (RANK, LOCAL_RANK, WORLD_SIZE, LOCAL_WORLD_SIZE, MASTER_ADDR = 127.0.0.1, MASTER_PORT). If a rank fails, the
    others are stopped after a grace period (their process group would otherwise end them by its timeout). Returns
    the worst exit code."""
    port = free_port()
    procs = []
    for r in range(n):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(n), LOCAL_WORLD_SIZE=str(n),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, script] + list(argv), env=env))
    failed_at = None
    while any(p.poll() is None for p in procs):
        if failed_at is None and any(p.returncode not in (None, 0) for p in procs):
            failed_at = time.monotonic()
        if failed_at is not None and time.monotonic() - failed_at > 30:
            for p in procs:
                if p.poll() is None:
                    p.kill()
        time.sleep(0.2)
    return max(abs(p.returncode) for p in procs)
