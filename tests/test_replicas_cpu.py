"""Multi-process host logic of the replica-parallel bench (gloo, 2 ranks, CPU)."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _worker(rank, world, port, q):
    import torch.distributed as dist

    from appearance_b200 import replicas
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r took (1 + r) seconds of device time and (2 + 3 r) end to end
        dev, e2e = replicas.max_over_ranks([1.0 + rank, 2.0 + 3.0 * rank], world)
        value = replicas.job_throughput(100.0, world, dev)
        q.put((rank, dev, e2e, value, replicas.replica_first_frame(rank)))
    finally:
        dist.destroy_process_group()


def _free_port():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_replicas_take_the_slowest_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, dev, e2e, value, first in res:
        assert dev == 2.0 and e2e == 5.0  # max over ranks, on every rank
        assert value == pytest.approx(100.0 * 2 / 2.0)  # all ranks' units over the slowest time
    assert [r[4] for r in res] == [0, 7]  # replicas start at different frames


def test_job_throughput_rejects_zero_time():
    from appearance_b200 import replicas
    with pytest.raises(ValueError):
        replicas.job_throughput(1.0, 1, 0.0)


def test_reference_arm_nonzero_rank_exits_without_output():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "3", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
