"""world_size-2 gloo test of the multi-rank (replica) path on CPU: every rank takes the same
collective steps; the job time is the max over ranks and the work the sum."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from hpcrack_b200 import replicas
    r, w, _ = replicas.rank_info()
    # rank r took (r + 1) * 100 ms for (r + 1) * 1e6 DoF-iterations
    t, work = replicas.aggregate(100.0 * (r + 1), 1e6 * (r + 1), w)
    thr = replicas.throughput(100.0 * (r + 1), 1e6 * (r + 1), w)
    replicas.barrier(w)
    q.put((r, t, work, thr, replicas.replica_seed(1, r, True), replicas.replica_seed(1, r, False)))
    dist.destroy_process_group()


def test_two_rank_aggregation():
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
    for r, t, work, thr, sd, ss in res:
        assert t == 200.0          # max over ranks
        assert work == 3e6         # sum over ranks
        assert abs(thr - 3e6 / 0.2) < 1e-6
        assert ss == 1 and sd == 1 + 1000 * r
