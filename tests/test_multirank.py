"""Multi-rank host logic of bench.py on the CPU: two processes over gloo (127.0.0.1) build their
shards of the serving stream, which must differ (independent systems, no data exchange), and
combine timings and atom counts with the max / sum the benchmark reports (max over ranks for time,
sum for whole-job throughput)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench

    dist = bench.Dist(backend="gloo", timeout_s=60)

    class Args:
        requests = 6
        rate = 50.0
        request_steps = 10

    systems, arrivals = bench.build_stream(Args, dist.rank)
    atoms = sum(sd.n for sd in systems)
    dist.barrier()
    t_max = dist.reduce(1.0 + rank, "max")
    atoms_all = dist.reduce(atoms, "sum")
    out.put((rank, atoms, [sd.n for sd in systems], [int(sd.params.seed) for sd in systems], t_max, atoms_all))
    dist.close()


def test_two_ranks_shard_and_reduce():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, a0, n0, s0, t0, all0), (r1, a1, n1, s1, t1, all1) = res
    assert (r0, r1) == (0, 1)
    assert n0 != n1 and not set(s0) & set(s1)  # distinct shards, distinct random streams
    assert t0 == t1 == 2.0                      # max over ranks
    assert all0 == all1 == a0 + a1              # whole-job atom count


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    d = bench.Dist()
    assert d.world == 1 and d.reduce(3.5, "max") == 3.5
    d.barrier()
    d.close()
