"""CPU: the multi-process path (one rank per GPU) with world_size 2 over gloo:
max-over-ranks timing, the barrier, and the instance sharding of the batched
engine (every instance owned by exactly one rank, the same split on every rank,
balanced cost)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from logosq_b200 import replicas, workloads


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port),
                       "WORLD_SIZE": str(world), "RANK": str(rank), "LOCAL_RANK": str(rank)})
    import torch.distributed as dist
    try:
        replicas.init("gloo", timeout_s=60)
        ws, r, _ = replicas.dist_info()
        replicas.barrier()
        step_time = 1.0 + 0.5 * r  # rank 1 is the slow one
        m = replicas.max_over_ranks(step_time)
        recs = workloads.heisenberg_instances(40, seed=4, n_lo=10, n_hi=20)
        costs = [replicas.instance_cost(x["n"], 8 * x["n"]) for x in recs]
        mine = replicas.shard_instances(costs, ws, r)
        q.put((r, ws, m, mine))
    finally:
        if dist.is_initialized():
            dist.destroy_process_group()


def test_world_size_2_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        r, ws, m, mine = q.get(timeout=120)
        out[r] = (ws, m, mine)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(v[0] == 2 for v in out.values())
    assert out[0][1] == out[1][1] == 1.5  # every rank sees the slowest rank's time
    owned = sorted(out[0][2] + out[1][2])
    assert owned == list(range(40)) and not set(out[0][2]) & set(out[1][2])


def test_shard_balance_and_determinism():
    recs = workloads.heisenberg_instances(256, seed=4, n_lo=10, n_hi=20)
    costs = [replicas.instance_cost(x["n"], 8 * x["n"]) for x in recs]
    for world in (1, 2, 4, 8):
        parts = [replicas.shard_instances(costs, world, r) for r in range(world)]
        assert sorted(sum(parts, [])) == list(range(256))
        loads = [sum(costs[i] for i in p) for p in parts]
        # LPT bound: the heaviest rank is within one largest item of the mean
        assert max(loads) <= sum(costs) / world + max(costs)
        assert parts == [replicas.shard_instances(costs, world, r) for r in range(world)]
    with pytest.raises(ValueError):
        replicas.shard_instances(costs, 2, 2)


def test_single_process_fallbacks():
    assert replicas.max_over_ranks(3.25) == 3.25
    assert replicas.job_throughput(10.0, 2.0, 4) == 20.0


from hypothesis import given, settings, strategies as st  # noqa: E402


@settings(max_examples=200, deadline=None)
@given(costs=st.lists(st.floats(0.0, 1e6, allow_nan=False), min_size=0, max_size=60),
       world=st.integers(1, 9))
def test_shard_property(costs, world):
    """Every instance goes to exactly one rank, and the busiest rank's load is
    within the longest-processing-time bound: the average load plus the largest
    single cost."""
    parts = [replicas.shard_instances(costs, world, r) for r in range(world)]
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(costs)))
    if costs:
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) <= sum(costs) / world + max(costs) + 1e-9 * (1 + sum(costs))


def test_instance_cost_counts_gates():
    """Cost = (2P + 1) circuits x (12n - 4) gates x 2^n amplitudes: a 20-qubit
    chain weighs (321 * 236 * 2^20) / (161 * 116 * 2^10) times a 10-qubit one."""
    from logosq_b200 import replicas
    r = replicas.instance_cost(20, 160) / replicas.instance_cost(10, 80)
    assert abs(r - (321 * 236 * 2 ** 20) / (161 * 116 * 2 ** 10)) < 1e-9
    assert replicas.instance_cost(10, 80, ngates=1) == 161 * 2 ** 10
