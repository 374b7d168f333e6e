"""The multi-rank path on CPU: two gloo ranks (world size 2) running the host logic that bench.py, batch_bench.py and
seednet_train.py run over NCCL, one process per GPU, on a B200 node.

  - frame pairs are partitioned, not exchanged: every rank computes the same partition alone, every pair lands on
    exactly one rank, and the costliest rank stays within one pair of the mean (the mixed batch's 64 pairs);
  - the timing collective: the max of the ranks' spans over the pairs of all ranks;
  - data-parallel seed-net training: the all-reduced (summed) gradient of the ranks' half-batches, scaled by 1 / ranks,
    is the gradient of the whole batch (the float64 reference net), and one Adam step leaves the ranks' parameters
    identical;
  - the reference arm on a rank other than 0 exits 0 without work or output.
"""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import replicas
import seednet_ref as ref

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WORLD = 2


def c3_costs():
    """the mixed batch's 64 pairs (34 x 720p, 17 x 1080p, 9 x 1440p, 4 x 2160p; multipliers 2 / 3 / 4 cycling): the
    pixels a pair moves, two frames in and m - 1 frames out"""
    sizes = [(1280, 720)] * 34 + [(1920, 1080)] * 17 + [(2560, 1440)] * 9 + [(3840, 2160)] * 4
    return [replicas.pair_cost(w, h, 2 + i % 3) for i, (w, h) in enumerate(sizes)]


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_ranks(fn, *args):
    port = free_port()
    mp.start_processes(fn, args=(WORLD, port) + args, nprocs=WORLD, join=True, start_method="spawn")


def _init(rank, world, port):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)


def _partition_worker(rank, world, port):
    _init(rank, world, port)
    costs = c3_costs()
    mine = replicas.shard_by_cost(costs, world)[rank]
    got = [None] * world
    dist.all_gather_object(got, mine)
    flat = sorted(i for s in got for i in s)
    assert flat == list(range(len(costs))), "every pair on exactly one rank"
    loads = [sum(costs[i] for i in s) for s in got]
    assert max(loads) <= sum(costs) / world + max(costs)
    dist.destroy_process_group()


def _timing_worker(rank, world, port):
    _init(rank, world, port)
    span = 10.0 + 3.0 * rank          # the slower rank sets the job's time
    assert replicas.max_over_ranks(span) == 13.0
    v = replicas.timed_span_value(span, items_per_rank=5)
    assert abs(v - 13.0 / (5 * world)) < 1e-12
    dist.destroy_process_group()


def _dp_worker(rank, world, port, la, lc, tgt, p):
    _init(rank, world, port)
    sync = replicas.GradSync()
    assert (sync.rank, sync.n) == (rank, world)
    seeds = [None] * world
    dist.all_gather_object(seeds, sync.rank_seed(1))
    assert len(set(seeds)) == world, "distinct data per rank"
    B = la.shape[0] // world
    sl = slice(rank * B, (rank + 1) * B)
    g_local, _ = ref.grads(p, ref.pack(la[sl], lc[sl]), tgt[sl])
    g = torch.from_numpy(g_local.copy())
    sync(g)
    g = g.numpy() * sync.scale()
    g_full, _ = ref.grads(p, ref.pack(la, lc), tgt)
    err = np.abs(g - g_full).max() / max(np.abs(g_full).max(), 1e-30)
    assert err < 1e-12, f"data-parallel gradient differs from the whole batch's: {err:.3g}"
    p1, _, _ = ref.adam(p.astype(np.float64), 0.0, 0.0, g, 1, 1e-3)
    got = [None] * world
    dist.all_gather_object(got, p1)
    assert all(np.array_equal(got[0], q) for q in got), "ranks' parameters diverged"
    dist.destroy_process_group()


def test_shard_by_cost_single_process():
    costs = c3_costs()
    for n in range(1, 9):
        shards = replicas.shard_by_cost(costs, n)
        assert sorted(i for s in shards for i in s) == list(range(len(costs)))
        loads = [sum(costs[i] for i in s) for s in shards]
        assert max(loads) <= sum(costs) / n + max(costs)
    assert replicas.shard_by_cost(costs, 1) == [list(range(64))]
    assert replicas.round_robin(5, 2) == [[0, 2, 4], [1, 3]]
    assert replicas.pair_cost(1280, 720, 2) == 1280 * 720 * 3
    with pytest.raises(ValueError):
        replicas.shard_by_cost(costs, 0)
    assert replicas.world() == (0, 1)
    assert replicas.max_over_ranks(2.5) == 2.5


def test_partition_over_gloo_ranks():
    run_ranks(_partition_worker)


def test_timing_max_over_gloo_ranks():
    run_ranks(_timing_worker)


def test_data_parallel_seed_net_step_over_gloo_ranks():
    rng = np.random.default_rng(11)
    B, h, w = 4, 24, 40
    la = (rng.random((B, h, w)) * 255).astype(np.float32)
    lc = np.roll(la, 3, axis=2)
    tgt = np.zeros((B, (h + 7) // 8, (w + 7) // 8, 6), np.float32)
    tgt[..., :4] = rng.uniform(-2, 2, tgt[..., :4].shape)
    tgt[..., 4] = 1.0
    p = ref.init_params(3)
    run_ranks(_dp_worker, la, lc, tgt, p)


def test_reference_arm_on_a_nonzero_rank_exits_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_bench_spawns_its_ranks():
    """`bench.py --gpus 2` without torchrun starts its two ranks itself (the rank plumbing of the timed region: gloo,
    barriers, the max of the spans) and reports n_gpus 2; a launcher with a different rank count is refused."""
    import json
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--gpus", "2", "--dry-run", "--steps", "5",
                        "--warmup", "3"], capture_output=True, text=True, timeout=240)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["n_gpus"] == 2 and line["steps"] == 5 and line["warmup"] == 3
    assert line["value"] * 2 == pytest.approx(line["per_rank_ms_per_pair"], rel=1e-3)
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--gpus", "2", "--dry-run", "--steps", "2"],
                       capture_output=True, text=True, timeout=240, env=env)
    assert r.returncode != 0 and "--gpus 2" in r.stderr
