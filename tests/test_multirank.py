"""The N > 1 host logic of bench.py on CPU: two gloo ranks (spawned
processes, 127.0.0.1 rendezvous).  The time step does not shard across GPUs
(one grid per device); bench.py runs one replica per rank and reduces the
device times with max over ranks, which is what is checked here."""
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


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r, w, local = bench.dist_env()
        ms = 10.0 + 5.0 * rank                  # per-rank device time of the timed region
        mx = bench.aggregate(ms, "max")
        sm = bench.aggregate(1.0, "sum")
        bench.barrier()
        # --impl reference: only rank 0 does work
        args = type("A", (), {"steps": 1, "warmup": 0, "n": 8})()
        ref = bench.run_reference(args) if rank != 0 else None
        q.put((r, w, local, mx, sm, ref))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_reduce_max_and_sum():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=100) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert [x[:3] for x in res] == [(0, 2, 0), (1, 2, 1)]
    for _, _, _, mx, sm, ref in res:
        assert mx == 15.0 and sm == 2.0
    assert res[1][5] is None


@pytest.mark.timeout(120)
def test_reference_arm_never_loads_the_cuda_library():
    """bench.py --impl reference times the CPU restatement only: the grid and
    the parameters are made without libntcfd.so, so the process never maps it."""
    import json
    import subprocess
    code = ("import sys, runpy; sys.argv = ['bench.py', '--impl', 'reference', '--n', '12', "
            "'--steps', '2', '--warmup', '1']; sys.path.insert(0, %r); "
            "runpy.run_path(%r, run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); "
            "print('MAPPED', 'libntcfd.so' in maps, 'libntcfd_oracle.so' in maps)"
            % (ROOT, os.path.join(ROOT, "bench.py")))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=110)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["steps"] == 2
    assert line["sweep_rate"]["unit"] == "Mcell-sweeps/s"
    assert lines[-1] == "MAPPED False True"
