"""Admission and tick logic of the continuous-batching server, driven by host-only stand-ins
for the device scene and batch (no GPU): budget never exceeded, arrival order kept, every
request stepped exactly K steps, late arrivals joining while others run."""
import time

import numpy as np
import pytest

from diploma_thesis_b200 import scenes, serve


class FakeScene:
    def __init__(self, scene, log):
        self.scene = scene
        self.num_particles = scene.num_particles
        self.steps = 0
        self.budget = None
        self.closed = False
        log.append(self)

    def download_async(self, stream=None):
        return {"steps": np.array(self.steps)}

    def close_async(self, stream=None):
        self.closed = True


class FakeBatch:
    def __init__(self):
        self.members = []
        self.ticks = []
        self.delay = 0.0

    def set_scenes(self, members, steps_left=None):
        assert len({id(m) for m in members}) == len(members)
        for m in members:
            assert not m.closed
        self.members = list(members)
        for i, m in enumerate(self.members):
            m.budget = None if steps_left is None else int(steps_left[i])

    def step(self, k, use_graph=True, stream=None):
        """Scenes with a budget are integrated by at most that many steps, then frozen."""
        assert k >= 1
        for m in self.members:
            assert not m.closed
            n = k if m.budget is None else max(0, min(k, m.budget))
            m.steps += n
            if m.budget is not None:
                m.budget -= n
        self.ticks.append((k, [id(m) for m in self.members]))
        if self.delay:
            time.sleep(self.delay)

    def close(self):
        pass


class FakeEvent:
    def query(self):
        return True

    def synchronize(self):
        pass


class FakeStream:
    def synchronize(self):
        pass

    def record_event(self):
        return FakeEvent()

    def wait_event(self, ev):
        pass


class FakeCtx:
    def check(self, stream=None):
        pass


def _server(budget, **kw):
    log = []
    batch = FakeBatch()
    srv = serve.Server(FakeCtx(), budget, tick_steps=4, keep_results=True,
                       scene_factory=lambda c, sc, st: FakeScene(sc, log), batch=batch,
                       stream=FakeStream(), **kw)
    return srv, batch, log


def _requests(n, ks, spread=0.002):
    pool = [scenes.small_scene(i, nb_side=1 + i % 3) for i in range(3)]
    return [serve.Request(spread * i, i, pool[i % 3], int(ks[i])) for i in range(n)]


def test_every_request_gets_exactly_k_steps():
    rng = np.random.default_rng(0)
    reqs = _requests(12, rng.integers(1, 30, 12))
    srv, batch, log = _server(1e12)
    stats = srv.run(reqs)
    assert stats.completed == 12
    for r in reqs:
        assert int(r.result["steps"]) == r.steps
        assert r.done >= r.admitted >= r.arrival - 1e-9
    assert all(s.closed for s in log)
    assert stats.scene_steps == sum(r.steps for r in reqs)


def test_budget_bounds_residency_and_order_is_fifo():
    reqs = _requests(9, [5] * 9, spread=0.0)
    srv, batch, log = _server(1.0)
    one = srv.cost(reqs[0].scene)[0]
    srv.budget = 2.5 * max(srv.cost(r.scene)[0] for r in reqs)
    stats = srv.run(reqs)
    assert stats.completed == 9
    assert stats.peak_bytes <= srv.budget and one > 0
    for k, ids in batch.ticks:
        members = [s for s in log if id(s) in ids]
        assert sum(srv.cost(s.scene)[0] for s in members) <= srv.budget
    assert max(len(t[1]) for t in batch.ticks) < 9
    admitted = [r.admitted for r in sorted(reqs, key=lambda r: r.rid)]
    assert admitted == sorted(admitted)


def test_late_arrivals_join_running_batch():
    reqs = _requests(2, [400, 10], spread=0.0)
    reqs[1].arrival = 0.02
    srv, batch, log = _server(1e12)
    srv.tick_steps = 1
    batch.delay = 2e-4  # 400 ticks take >= 80 ms, the second request arrives at 20 ms
    stats = srv.run(reqs)
    assert stats.completed == 2
    # the second scene was admitted while the first was still resident, and finished first
    assert reqs[1].admitted < reqs[0].done and reqs[1].done < reqs[0].done
    assert any(len(t[1]) == 2 for t in batch.ticks)


def test_particle_cap_limits_the_batch():
    reqs = _requests(6, [3] * 6, spread=0.0)
    cap = max(r.scene.num_particles for r in reqs)
    srv, batch, log = _server(1e12, max_batch_particles=cap)
    stats = srv.run(reqs)
    assert stats.completed == 6
    for k, ids in batch.ticks:
        members = [s for s in log if id(s) in ids]
        assert sum(s.num_particles for s in members) <= cap


def test_request_that_can_never_fit_is_an_error():
    reqs = _requests(1, [3])
    srv, batch, log = _server(1e12, max_batch_particles=1)
    with pytest.raises(ValueError):
        srv.run(reqs)


def test_frozen_scenes_leave_and_are_freed_after_the_next_member_change():
    rng = np.random.default_rng(3)
    reqs = _requests(8, rng.integers(1, 25, 8), spread=0.0)
    srv, batch, log = _server(1e12)
    srv.tick_steps = 7
    stats = srv.run(reqs)
    assert stats.completed == 8
    for r in reqs:  # budgets freeze every scene after exactly K steps, whatever the tick size
        assert int(r.result["steps"]) == r.steps
    assert all(s.closed for s in log) and batch.members == []
