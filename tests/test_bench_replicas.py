"""The multi-GPU form of bench.py runs independent replicas (the stepper does
not shard): the job time is the slowest rank's, the rate is the sum over
ranks.  Checked here on CPU with two gloo ranks, plus the reference arm's
JSON line (it runs the reference CPU stepper, no GPU)."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = bench.max_over_ranks(1.0 + rank, dist, "cpu")      # rank 1 is the slow one
        out.put((rank, t, bench.replica_throughput(100.0, world, t)))
    finally:
        dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, rate in res:
        assert t == 2.0                     # every rank reports the slowest rank's time
        assert rate == 100.0 * 2 / 2.0      # summed work over the slowest time


def test_reference_arm_json_line():
    import oracle
    if not oracle.reference_available():
        pytest.skip("reference binary not built")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3", "--workload", "c0"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-1500:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == "site-updates/s"
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] == "reference"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
