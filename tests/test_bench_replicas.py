"""The multi-GPU path of bench.py is N independent replicas: each rank times
its own copy of the workload and rank 0 reports the whole job from the
maximum time over ranks.  These host-side checks run two gloo ranks on the
CPU: process-group set-up from the launcher's environment, the barrier, the
max over ranks, and the reference arm's rule that only rank 0 works."""
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    r, w, local = bench.dist_setup(world)
    bench.barrier(w)
    m = bench.max_over_ranks(1.5 + r, w)
    # the reference arm: ranks other than 0 leave without work
    ref_rc = bench.run_reference(type("A", (), {"steps": 1, "warmup": 3, "gpus": w, "n": 4, "seed": 1})()) \
        if r != 0 else 0
    bench.barrier(w)
    dist.destroy_process_group()
    q.put((r, w, local, m, ref_rc))


def test_two_gloo_replicas():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    out = sorted(q.get(timeout=5) for _ in range(2))
    for p in procs:
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1]
    assert all(o[1] == 2 for o in out)
    assert all(o[3] == 2.5 for o in out)  # max over ranks of 1.5 + rank
    assert all(o[4] == 0 for o in out)
