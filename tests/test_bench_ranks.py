"""bench.py's multi-rank plumbing on CPU: two gloo ranks (replicas only, no data-path collective).

Each rank reports its own solve time; the job's time is the slowest rank's, taken with one
all-reduce between barriers. Under torchrun the reference arm runs on rank 0 alone.
"""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, results):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    ranks = bench.Ranks("gloo", "cpu", timeout_s=60)
    assert (ranks.rank, ranks.world) == (rank, world)
    ranks.barrier()
    times = [ranks.max(0.5 + 0.25 * rank), ranks.max(3.0 - rank)]
    ranks.close()
    results[rank] = times


def test_two_gloo_ranks_take_the_slowest_rank():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        results = mgr.dict()
        procs = [ctx.Process(target=_worker, args=(r, world, port, results)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        codes = [p.exitcode for p in procs]
        res = dict(results)
    assert codes == [0] * world, codes
    assert all(res[r] == [0.75, 3.0] for r in range(world)), res


def test_single_process_needs_no_group(monkeypatch):
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    monkeypatch.delenv("RANK", raising=False)
    sys.path.insert(0, ROOT)
    import bench
    ranks = bench.Ranks("gloo", "cpu")
    assert ranks.world == 1 and ranks.dist is None
    assert ranks.max(1.25) == 1.25
    ranks.barrier()
    ranks.close()


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1"])
    sys.path.insert(0, ROOT)
    import bench
    assert bench.main() == 0
    assert capsys.readouterr().out == ""
