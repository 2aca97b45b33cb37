"""Replica sharding over two ranks (gloo, CPU): the multi-GPU path is
independent instances per rank plus one host gather."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from caustic_b200 import replicas


def test_shard_covers_every_item_once():
    for n in (0, 1, 5, 64):
        for world in (1, 2, 3, 8):
            got = sorted(i for r in range(world) for i in replicas.shard(n, r, world))
            assert got == list(range(n))
    with pytest.raises(ValueError):
        replicas.shard(4, 2, 2)


def _tiny_solve(seed):
    # a CPU oracle solve stands in for the per-GPU solve
    from caustic_b200 import problems
    from oracle import oracle as O

    p = problems.make(3, instance=seed, g=6, res=24)
    prob = O.Problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
    w, st = O.lbfgs_wolfe(prob, np.zeros(p.n), tol=1e-3)
    return w, st.iterations


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        res = replicas.solve_replicas(list(range(5)), _tiny_solve)
        if rank == 0:
            np.save(os.path.join(out_dir, "it.npy"), np.array([r[1] for r in res]))
            np.save(os.path.join(out_dir, "w.npy"), np.concatenate([r[0] for r in res]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_match_one_process(tmp_path):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    local = [_tiny_solve(i) for i in range(5)]
    assert np.array_equal(np.load(tmp_path / "it.npy"), np.array([r[1] for r in local]))
    assert np.array_equal(np.load(tmp_path / "w.npy"), np.concatenate([r[0] for r in local]))


def _gpu_solve(seed):
    # the library's own GPU solve on the rank's device
    from caustic_b200 import capi, problems

    p = problems.make(3, instance=seed, g=12, res=48)
    with capi.Solver(device=0) as s:
        s.set_problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
        w, st = s.solve(np.zeros(p.n), tol=1e-4)
    return w, st.evaluations


def _gpu_worker(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        res = replicas.solve_replicas(list(range(6)), _gpu_solve)
        if rank == 0:
            np.save(os.path.join(out_dir, "ev.npy"), np.array([r[1] for r in res]))
            np.save(os.path.join(out_dir, "w.npy"), np.concatenate([r[0] for r in res]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_two_gpu_ranks_match_one_process(gpu, tmp_path):
    """The replica path with the GPU solve on every rank: two processes
    (gloo for the gather, each solving its share on device 0 -- independent
    solves that never wait on each other) give the single process's weights
    bit for bit."""
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_gpu_worker, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    local = [_gpu_solve(i) for i in range(6)]
    assert np.array_equal(np.load(tmp_path / "ev.npy"), np.array([r[1] for r in local]))
    assert np.array_equal(np.load(tmp_path / "w.npy"), np.concatenate([r[0] for r in local]))
