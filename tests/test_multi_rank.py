"""Multi-rank sharding of the batch, on CPU with the gloo backend (world size 2).

Each rank builds its own share of the lines with the oracle (the GPU ranks run the same shares
through the CUDA path) and the shares, gathered on every rank, must equal the single-rank build of
all lines bit for bit: lines are independent, so sharding needs no collective on the data path.
The uneven-batch partition is checked to cover every problem once and to balance the work.
"""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
dist = pytest.importorskip("torch.distributed")

from ddc_b200.sharding import problem_cost, shard_problems, shard_range  # noqa: E402


def test_shard_range_partitions_lines():
    for n in (0, 1, 7, 1000, 65536):
        for world in (1, 2, 3, 8):
            spans = [shard_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[r][1] == spans[r + 1][0] for r in range(world - 1))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1


def test_shard_problems_balance_uneven_batch():
    from ddc_b200 import workloads as W

    probs = W.config4(count=512)
    costs = [problem_cost(p["ncells"], p["degree"], len(p["coords"])) for p in probs]
    for world in (2, 4, 8):
        parts = shard_problems(costs, world)
        flat = sorted(i for part in parts for i in part)
        assert flat == list(range(len(probs)))
        loads = [sum(costs[i] for i in part) for part in parts]
        assert max(loads) <= sum(costs) / world + max(costs)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        from datetime import timedelta

        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
        from ddc_b200 import workloads as W
        from oracle import oracle as O

        O.lib()
        w = W.config1(B=96, ncells=64, m=16)
        obs = O.BSplines(3, True, rmin=0.0, rmax=1.0, ncells=64)
        ob = O.Builder(obs, obs.greville(O.PERIODIC, O.PERIODIC), O.PERIODIC, O.PERIODIC)
        a, b = shard_range(96, rank, world)
        mine = ob(np.ascontiguousarray(w["vals"][:, a:b]), nthreads=1)
        parts = [None] * world
        dist.all_gather_object(parts, (a, b, mine))
        full = np.concatenate([p[2] for p in sorted(parts, key=lambda p: p[0])], axis=1)
        ref = ob(w["vals"], nthreads=1)
        q.put((rank, bool(np.array_equal(full, ref))))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as exc:  # reported to the parent
        q.put((rank, f"{type(exc).__name__}: {exc}"))


def test_two_rank_sharded_build_equals_single_rank():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert results == {0: True, 1: True}, results


def test_bench_starts_ranks_and_shards_the_batch():
    """`bench.py --gpus 2` starts two ranks itself (torchrun), each rank draws its contiguous shard
    of the global batch, and rank 0 reports n_gpus = 2 with the time as the max over ranks. The CPU
    stub runs the same rank code over gloo with a NumPy step in place of the kernels."""
    import json
    import subprocess
    import sys

    import numpy as np

    from ddc_b200 import workloads as W

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lines = 96
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--gpus", "2", "--cpu-stub", "--steps", "2",
                        "--warmup", "3", "--lines", str(lines)], capture_output=True, text=True, timeout=240)
    assert r.returncode == 0, r.stderr[-2000:]
    out = [json.loads(ln) for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(out) == 1, r.stdout
    line = out[0]
    assert line["n_gpus"] == 2 and line["config"]["global_lines"] == 2 * lines
    assert [s[:2] for s in line["shards"]] == [[0, lines], [lines, 2 * lines]]
    # each rank's inputs are exactly its columns of the global batch
    whole = W.config2(B=2 * lines, m=64, points=np.linspace(0.0, 1.0, 33))
    for (a, b, check) in line["shards"]:
        expect = float(whole["vals"][:, a:b].sum() + whole["coords"][:, a:b].sum())
        assert abs(check - expect) <= 1e-9 * abs(expect)
