"""The N>1 path of bench.py on CPU: world-size-2 gloo ranks.  Every rank
runs its own team on its own data (weak scaling, no data-path collective);
the job's time is the slowest rank's and its throughput counts every rank's
bytes.  The reference arm under torchrun prints one line, from rank 0."""
import json
import os
import socket
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
    first = bench.inputs(seed_base=rank * 100, which=(0,))[0][0, :4].tolist()
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, ms, bench.job_gbs(1e9, 2, world, ms), first))


def test_two_gloo_ranks_time_and_throughput():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, ms0, v0, x0), (r1, ms1, v1, x1) = res
    assert ms0 == ms1 == 15.0          # the slowest rank's time, on every rank
    assert v0 == v1 == 1e9 * 2 * 2 / 0.015 / 1e9
    assert not np.allclose(x0, x1)     # each rank reduces its own data


def test_reference_arm_under_torchrun_prints_one_line():
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "3"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d.get("unavailable") or (d["value"] > 0 and d["cpu_baseline"]["kind"] in ("reference", "port"))
