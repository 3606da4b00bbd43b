"""The bench's multi-replica host logic on CPU: two gloo ranks (world size 2, 127.0.0.1).

bench.py --gpus N runs N independent replicas, one per GPU, with no data-path collective; the
ranks only meet in barriers and in the two reductions that turn per-rank work and device times
into the whole-job rate (all ranks' units over the slowest rank's time).  The reference arm runs
on rank 0 alone; the other ranks leave without work.
"""
import json
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, port, out_dir):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    D_ = bench.Dist()
    try:
        D_.barrier()
        # rank r processed 3 + r units in 2 + r seconds: whole job 7 units over the slowest 3 s
        rate = bench.job_rate(D_, 3 + rank, 2.0 + rank)
        mx, sm = D_.max(10.0 * (rank + 1)), D_.sum(rank + 1)
        # the reference arm: rank 1 must return at once (it would need a GPU otherwise)
        if rank == 1:
            bench.run_reference(None, D_)
        D_.barrier()
        with open(os.path.join(out_dir, "rank%d.json" % rank), "w") as f:
            json.dump({"rate": rate, "max": mx, "sum": sm, "world": D_.world}, f)
    finally:
        D_.close()


def test_two_gloo_replicas_aggregate_like_the_bench(tmp_path):
    mp = pytest.importorskip("torch.multiprocessing")
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
        assert p.exitcode == 0
    res = [json.load(open(tmp_path / ("rank%d.json" % r))) for r in range(2)]
    for r in res:
        assert r["world"] == 2
        assert r["rate"] == pytest.approx(7.0 / 3.0)
        assert r["max"] == 20.0 and r["sum"] == 3.0
