"""Host logic of the warm-start pipeline (caustic_b200/warm.py), no GPU:
which levels each start solves."""
import pytest

from caustic_b200 import problems
from caustic_b200.warm import WarmSolver


def test_levels_of_each_start():
    p = problems.make(2, 0, g=128, res=512)          # 16,384 sites
    ml = WarmSolver(start="multilevel")
    assert [q.n for q in ml.chain(p)] == [16384, 4096, 1024]
    z = WarmSolver(start="zero")
    assert [q.n for q in z.chain(p)] == [16384]
    learned = WarmSolver(start="learned", net=object(), net_level_sites=4096, learned_at="level")
    assert [q.n for q in learned.chain(p)] == [16384, 4096]
    # a network for a level finer than the problem starts at the problem itself
    fine = WarmSolver(start="learned", net=object(), net_level_sites=65536, learned_at="level")
    assert [q.n for q in fine.chain(p)] == [16384]
    # averaged down to the coarsest level, the whole chain is solved
    down = WarmSolver(start="learned", net=object(), net_level_sites=4096)
    ch = down.chain(p)
    assert [q.n for q in ch] == [16384, 4096, 1024] and ch[down._net_level(ch)].n == 4096


def test_config2_learned_level_keeps_the_training_resolution():
    """At the benchmark size the 16,384-site level has 4 pixels per site, as
    the network's training problems do (128^2 sites, 512^2 images)."""
    p = problems.make(2)
    ch = WarmSolver(start="learned", net=object(), net_level_sites=16384, learned_at="level").chain(p)
    assert [q.n for q in ch] == [65536, 16384]
    assert tuple(ch[-1].size) == (512, 512)


def test_bad_arguments():
    with pytest.raises(ValueError):
        WarmSolver(start="sideways")
    with pytest.raises(ValueError):
        WarmSolver(start="learned")


def test_restriction_keeps_smooth_fields():
    """Block means of a linear field are the field at the blocks' mean
    positions (what the coarse sites are)."""
    import numpy as np

    from caustic_b200 import multilevel

    p = problems.make(2, 1, g=32, res=128)
    ch = multilevel.chain(p, min_sites=64)
    fine, coarse = ch[0], ch[2]
    w = 0.3 * p.xy[:, 0] - 0.7 * p.xy[:, 1]
    wc = multilevel.restrict(w, fine, coarse)
    ref = 0.3 * coarse.xy[:, 0] - 0.7 * coarse.xy[:, 1]
    assert np.abs(wc - (ref - ref.mean())).max() < 1e-12


class _FakeSolver:
    """Stands in for a pipeline on the host: records which problems it
    solved, in which thread order, and fails on request."""

    def __init__(self, **kw):
        self.device = 0
        self.seen = []
        self.closed = False

    def solve(self, p):
        if p == "boom":
            raise RuntimeError("solve failed")
        self.seen.append(p)
        return (p * 10, p)

    def close(self):
        self.closed = True


def test_pool_round_robin_order_and_errors(monkeypatch):
    """WarmPool hands the problems round robin to its pipelines, returns the
    results in problem order, closes every pipeline, and raises a pipeline's
    error on the calling thread."""
    import torch

    from caustic_b200 import warm

    monkeypatch.setattr(warm, "WarmSolver", _FakeSolver)
    monkeypatch.setattr(torch.cuda, "set_device", lambda d: None)
    with warm.WarmPool(3) as pool:
        out, wall = pool.solve_all(list(range(7)))
        assert [r[1] for r in out] == list(range(7)) and [r[0] for r in out] == [10 * i for i in range(7)]
        assert [s.seen for s in pool.solvers] == [[0, 3, 6], [1, 4], [2, 5]]
        assert wall >= 0.0
        with pytest.raises(RuntimeError, match="solve failed"):
            pool.solve_all([1, "boom", 2])
    assert all(s.closed for s in pool.solvers)
