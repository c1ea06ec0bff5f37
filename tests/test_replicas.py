"""Multi-GPU host logic of the benchmark (replicas only), as two gloo ranks on
CPU: the barrier, the max over ranks of the timed region, and the whole-job
rate = work of all ranks / slowest rank's time."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from tclb_b200.replicas import Replicas

    reps = Replicas("gloo", timeout_s=30)
    reps.barrier()
    # rank r "processed" (r + 1) * 1000 units in (r + 1) * 0.5 s
    rate, t_max = reps.whole_job_rate(units=(rank + 1) * 1000.0, seconds=(rank + 1) * 0.5)
    m = reps.reduce_max(float(rank))
    s = reps.reduce_sum(1.0)
    reps.barrier()
    reps.close()
    out.put((rank, rate, t_max, m, s))


def test_two_gloo_ranks_reduce_and_rate():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=5) for _ in range(world))
    for rank, rate, t_max, m, s in res:
        assert t_max == pytest.approx(1.0)       # slowest rank: 2 * 0.5 s
        assert rate == pytest.approx(3000.0)     # (1000 + 2000) units / 1.0 s
        assert m == 1.0 and s == 2.0


def test_single_process_needs_no_process_group():
    from tclb_b200.replicas import Replicas

    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        os.environ.pop(k, None)
    reps = Replicas("gloo")
    assert reps.world == 1
    assert reps.whole_job_rate(500.0, 2.0) == (250.0, 2.0)
    assert reps.reduce_max(3.5) == 3.5
    reps.barrier()
    reps.close()


def test_partition_cases_balances_work():
    from tclb_b200.replicas import partition_cases

    w = [float(x) for x in [100, 1, 7, 50, 50, 3, 99, 2, 8, 60]]
    parts = partition_cases(w, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(w)))  # every case exactly once
    loads = [sum(w[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(w)
    assert partition_cases(w, 3) == parts  # deterministic: every rank computes the same split
    assert partition_cases(w, 1) == [list(range(len(w)))]


def _agg_main(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from tclb_b200.benchmarks import aggregate_batch, aggregate_serving
    from tclb_b200.replicas import Replicas

    reps = Replicas("gloo", timeout_s=30)
    # rank r: (r+1) * 1e6 updates in (r+1) s, 3 cases, single-case rate 10 + r MLUPS
    b = aggregate_batch(reps, (rank + 1) * 1e6, rank + 1.0, 3, 10.0 + rank)
    rep = {"busy_s": 2.0 + rank, "wall_s": 4.0 + rank, "rounds": 5, "pending": 0}
    tts = [0.1 * (rank + 1), 0.2 * (rank + 1)]
    srv = aggregate_serving(reps, rep, tts, updates=1e6 * (rank + 1), ideal_s=1.0 + rank)
    reps.close()
    out.put((rank, b, srv))


def test_two_gloo_ranks_aggregate_sharded_runs():
    """The whole-job figures of sharded batch and serving runs: work of all
    ranks over the slowest rank, percentiles over every rank's requests."""
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_agg_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=5) for _ in range(world))
    for rank, b, srv in res:
        assert b["time_s"] == pytest.approx(2.0) and b["MLUPS"] == pytest.approx(1.5)  # 3e6 updates / 2 s
        assert b["cases_per_s"] == pytest.approx(3.0)                                   # 6 cases / 2 s
        assert b["fraction_of_single"] == pytest.approx(1.5 / (2 * 10.5))
        assert srv["requests"] == 4 and srv["wall_s"] == pytest.approx(5.0)
        assert srv["busy_s"] == pytest.approx(5.0) and srv["fraction_of_single"] == pytest.approx(3.0 / 5.0)
        assert srv["p50_s"] == pytest.approx(0.2) and srv["rounds"] == 10
