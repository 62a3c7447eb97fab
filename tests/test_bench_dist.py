"""The multi-process plumbing of bench.py (one process per GPU under torchrun) with the gloo
backend on the host, world size 2: the barrier, the max over ranks every timed number goes
through, and the whole-job rate of the replicas -- all ranks' cell updates over the slowest
rank's time."""
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist(backend="gloo")
    try:
        d.barrier()
        slowest = d.max(1.0 + rank)           # rank r took 1 + r seconds
        rate = bench.whole_job_mlups(d.world, 1000000, 10, slowest)
        d.barrier()
        q.put((rank, d.world, slowest, rate))
    finally:
        d.close()


def test_replicas_take_the_slowest_rank_and_count_every_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, world, slowest, rate in out:
        assert world == 2
        assert slowest == 2.0                  # the max over ranks
        assert abs(rate - 2 * 10.0 / 2.0) < 1e-12  # 2 ranks x 1e6 cells x 10 steps / 2 s = 10 MLUPS
