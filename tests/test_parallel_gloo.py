"""Host logic of the multi-GPU path on CPU: world_size 2 gloo ranks split the
orientations and all-reduce their partial Mueller sums (no GPU)."""
import os

import numpy as np
import pytest


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import sys
        sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                        "bem-cpp_b200"))
        from bem_b200.parallel import allreduce_max, allreduce_sum, orientation_slice
        n_orient, nt = 37, 19
        rng = np.random.default_rng(0)
        terms = rng.standard_normal((n_orient, 16, nt))  # per-orientation w_o M_o terms
        o0, o1 = orientation_slice(n_orient, rank, world)
        part = terms[o0:o1].sum(axis=0)
        total = allreduce_sum(part)
        tmax = allreduce_max(float(rank + 1))
        q.put((rank, o0, o1, total, tmax))
    finally:
        dist.destroy_process_group()


def test_orientation_split_and_mueller_allreduce():
    import torch.multiprocessing as mp
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    (r0, a0, a1, t0, m0), (r1, b0, b1, t1, m1) = res
    assert (a0, a1, b0, b1) == (0, 18, 18, 37)
    rng = np.random.default_rng(0)
    full = rng.standard_normal((37, 16, 19)).sum(axis=0)
    assert np.allclose(t0, full, rtol=1e-13, atol=1e-13) and np.allclose(t1, full, rtol=1e-13, atol=1e-13)
    assert m0 == m1 == 2.0


def test_orientation_slice_covers_all():
    import sys
    from bem_b200.parallel import orientation_slice
    for n in (1, 7, 1395):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                o0, o1 = orientation_slice(n, r, world)
                seen += list(range(o0, o1))
            assert seen == list(range(n))
    with pytest.raises(ValueError):
        orientation_slice(5, 2, 2)


def _worker_particles(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import sys
        sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                        "bem-cpp_b200"))
        from bem_b200.parallel import batch_run_distributed
        particles = [{"id": i} for i in range(11)]
        seen = []

        def run(ps):   # stands in for the device pipeline: one result per particle
            seen.extend(p["id"] for p in ps)
            return [(np.full((4, 4, 3), float(p["id"])), {"status": 0, "rank": rank}) for p in ps]
        out = batch_run_distributed(None, particles, rank, world, run=run)
        q.put((rank, seen, [float(m[0, 0, 0]) for m, _ in out], [i["rank"] for _, i in out]))
    finally:
        dist.destroy_process_group()


def test_particle_split_and_gather():
    import torch.multiprocessing as mp
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker_particles, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, seen0, ids0, who0), (r1, seen1, ids1, who1) = res
    assert seen0 == list(range(0, 5)) and seen1 == list(range(5, 11))    # each particle once
    assert ids0 == ids1 == [float(i) for i in range(11)]                  # gathered in order
    assert who0 == who1 == [0] * 5 + [1] * 6


def _worker_failure(rank, world, port, q):
    # rank 1 fails inside its local work (an exception on the host, before
    # any collective); every rank must still take the same collectives and
    # raise naming rank 1, rather than wait for the process group's timeout
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        import sys
        sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                        "bem-cpp_b200"))
        from bem_b200.parallel import batch_run_distributed, orientation_average_distributed
        msgs = []

        def run(ps):
            if rank == 1:
                raise MemoryError("injected on rank 1")
            return [(np.zeros((4, 4, 3)), {"status": 0}) for _ in ps]
        try:
            batch_run_distributed(None, list(range(6)), rank, world, run=run)
        except RuntimeError as ex:
            msgs.append(str(ex))
        # one orientation: rank 0 has none, rank 1 has it and fails (no device
        # objects here, so its first device call raises)
        try:
            orientation_average_distributed(None, None, None, np.eye(3)[None], np.ones(1), 1.0, 1.0,
                                            ntheta=3, rank=rank, world=world)
        except RuntimeError as ex:
            msgs.append(str(ex))
        # the group is still usable afterwards
        from bem_b200.parallel import allreduce_max
        q.put((rank, msgs, allreduce_max(float(rank))))
    finally:
        dist.destroy_process_group()


def test_a_failing_rank_is_reported_on_every_rank():
    import torch.multiprocessing as mp
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker_failure, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, msgs, mx in res:
        assert len(msgs) == 2, (rank, msgs)
        assert "batch_run_distributed: rank 1 failed: MemoryError: injected on rank 1" in msgs[0]
        assert msgs[1].startswith("orientation_average_distributed: rank 1 failed")
        assert mx == 1.0
