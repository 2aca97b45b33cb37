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
