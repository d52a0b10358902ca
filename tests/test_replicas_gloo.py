"""The N > 1 path of bench.py (replicas, no collective on the data path), on the host:
two gloo ranks on 127.0.0.1 meet at the barrier and reduce their timings to the maximum over
ranks; a rank other than 0 leaves the reference arm without work."""
import os
import socket
import sys

import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime
    sys.path.insert(0, ROOT)
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world))
    torch.distributed.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                                         world_size=world, timeout=datetime.timedelta(seconds=60))
    from slope_stability_octave_b200 import replicas
    r, lr, w = replicas.rank_world()
    replicas.barrier(w)
    out = replicas.max_over_ranks([1.0 + rank, 10.0 - rank], w)
    import bench
    ref = bench.reference_arm(type("A", (), dict(gpus=w, steps=1, warmup=0))(), rank, w) if rank != 0 else None
    torch.distributed.destroy_process_group()
    q.put((rank, r, w, out, ref))


def test_two_gloo_ranks_barrier_and_max_over_ranks():
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
    for rank, r, w, out, ref in res:
        assert r == rank and w == 2
        assert out == [2.0, 10.0]
        assert ref is None


def test_single_process_is_identity():
    sys.path.insert(0, ROOT)
    from slope_stability_octave_b200 import replicas
    assert replicas.max_over_ranks([3.0, 4.0], 1) == [3.0, 4.0]
