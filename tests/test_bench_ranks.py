"""The bench's multi-process plumbing (one process per GPU under torchrun)
run as two gloo ranks on the CPU: the process group comes up from the
launcher's environment variables (127.0.0.1), the barrier passes, and the
timing reduction returns the maximum over the ranks on every rank -- the
whole-job figure divides all ranks' cells by that slowest time."""
import argparse
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, port: int, q):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    ws, r, local = bench.dist_init(argparse.Namespace(gpus=2), backend="gloo")
    bench.barrier(ws)
    ms = bench.allmax(ws, 1.5 * (r + 1))       # rank 0 took 1.5 ms, rank 1 3.0 ms
    bench.barrier(ws)
    q.put((r, ws, local, ms))
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out == [(0, 2, 0, 3.0), (1, 2, 1, 3.0)]
