"""The multi-rank plumbing of bench.py (one process per GPU, replicas of the workload) on CPU: two
gloo ranks rendezvous on 127.0.0.1, meet at the barrier and agree on the max-over-ranks time; the
reference arm's non-zero ranks exit without work."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_init()
    bench.barrier(w)
    m = bench.max_over_ranks(1.5 + r, w)
    out.put((r, w, m, dist.get_backend()))
    dist.destroy_process_group()


def test_two_gloo_ranks_barrier_and_max():
    torch = pytest.importorskip("torch")
    mp = torch.multiprocessing.get_context("spawn")
    q = mp.Queue()
    port = _free_port()
    procs = [mp.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == [(0, 2, 2.5, "gloo"), (1, 2, 2.5, "gloo")]


def test_reference_arm_nonzero_rank_exits_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""


def _sum_rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import datetime
    import numpy as np
    import torch.distributed as dist
    from srsoriginal_b200 import aggregate as A
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    rng = np.random.default_rng(100 + rank)
    mine = rng.lognormal(0.0, 6.0, 50)
    total = A.sum_over_ranks(mine, weight=1.0 / world)
    out.put((rank, mine.tolist(), None if total is None else total.tolist()))
    dist.destroy_process_group()


def test_sum_over_ranks_gloo():
    """The reference's MPI example pattern (workers' spectra summed at rank 0 with add_to_spectrum) on
    two gloo ranks: rank 0 gets the compensated, weighted sum in rank order, rank 1 None."""
    torch = pytest.importorskip("torch")
    import numpy as np
    sys.path.insert(0, ROOT)
    from srsoriginal_b200 import aggregate as A
    mp = torch.multiprocessing.get_context("spawn")
    q = mp.Queue()
    port = _free_port()
    procs = [mp.Process(target=_sum_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, t0), (r1, m1, t1) = got
    assert t1 is None and t0 is not None
    ref = A.SpectrumSum()
    for m in (m0, m1):
        ref.add(np.zeros(len(m)), m, 0.5)
    assert np.array_equal(np.array(t0), ref.flux)
