"""The replica host logic of multi-GPU runs, as two gloo ranks on CPU."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    from gip_b200.replicas import Replicas
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    R = Replicas(dist)
    R.barrier()
    local = 100.0 + 50.0 * rank          # rank 1 is the slow replica
    q.put((rank, R.max(local), R.sum(1.0), R.job_ms_per_step(local, steps=5)))
    dist.destroy_process_group()


def test_two_rank_replicas_max_and_job_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get() for _ in range(2))
    for rank, mx, sm, job in res:
        assert mx == 150.0 and sm == 2.0
        assert job == 150.0 / (5 * 2)    # 10 replica-steps in the slowest rank's 150 ms


def _failing_worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    from gip_b200.replicas import Replicas
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=5))
    R = Replicas(dist)
    R.barrier()
    if rank == 1:
        os._exit(3)  # a replica dies between steps, with nothing in flight
    try:
        R.max(1.0)
        q.put((rank, "no error"))
    except Exception as e:  # the survivor's next collective ends with an error
        q.put((rank, type(e).__name__))


def test_lost_replica_is_detected_not_waited_for():
    import time
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_failing_worker, args=(r, 2, port, q)) for r in range(2)]
    t0 = time.time()
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
    assert ps[1].exitcode == 3
    rank, what = q.get(timeout=10)
    assert rank == 0 and what != "no error"
    assert time.time() - t0 < 90
