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


def test_gpus_flag_starts_ranks():
    """`bench.py --gpus 2` without a torchrun environment starts two ranks itself (torch's launcher,
    rendezvous on 127.0.0.1); under --impl reference rank 0 alone works and prints the line, the
    other rank exits 0.  gloo stands in for NCCL on the CPU."""
    import json
    import subprocess
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR",
                                                            "MASTER_PORT")}
    env["RBMD_DIST_BACKEND"] = "gloo"
    env["RBMD_ORACLE_THREADS"] = "2"
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0", "--requests", "12"], capture_output=True, text=True,
                       timeout=600, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    lines = [json.loads(ln) for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"


def test_gpus_flag_must_match_world_size():
    import subprocess
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2"], capture_output=True,
                       text=True, timeout=120, env=env, cwd=ROOT)
    assert r.returncode != 0 and "WORLD_SIZE" in r.stderr
