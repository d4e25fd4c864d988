"""Continuous-batching scheduler logic (SnapshotServer) against a fake batch on the CPU:
FIFO admission against the HBM budget, admission of requests that arrive while others are
resident, every request completed once, latency accounting."""
import itertools

import numpy as np

from philip_b200.serve import SnapshotServer, SolveRequest, poisson_arrivals


class FakeBatch:
    """Budget-accounting stand-in for the device batch: a solve needs `bytes` of the budget,
    advances one step per stepped step, completes when its steps are done."""

    def __init__(self, budget):
        self.budget, self.used = budget, 0
        self.slots, self.ids = {}, itertools.count()
        self.max_used, self.log = 0, []

    def admit(self, mesh, prm, U0, dt, nsteps):
        need = mesh   # the fake request carries its size in place of a mesh
        if self.used + need > self.budget:
            return None
        s = next(self.ids)
        self.slots[s] = [need, 0, nsteps]
        self.used += need
        self.max_used = max(self.max_used, self.used)
        self.log.append(("admit", s, len(self.slots)))
        return s

    @property
    def active(self):
        return sum(1 for v in self.slots.values() if v[1] < v[2])

    def step(self, n):
        for v in self.slots.values():
            v[1] = min(v[2], v[1] + n)

    def fence(self):
        return 0

    def wait(self, t):
        pass

    def poll(self, s):
        v = self.slots[s]
        return v[1] >= v[2]

    def state(self, s, ndofs):
        return np.zeros(1)

    def status(self, s):
        return 0

    def release(self, s):
        self.used -= self.slots.pop(s)[0]


class FakeServer(SnapshotServer):
    def _prepare(self, req):   # the fake request carries (bytes, nsteps)
        return req.tag[0], None, None, 1.0, req.tag[1]    # (bytes, -, -, dt, nsteps)


def _run(budget, reqs, chunk=4):
    clock = itertools.count(0.0, 0.001)
    batch = FakeBatch(budget)
    srv = FakeServer(batch, chunk=chunk, clock=lambda: next(clock))
    return batch, srv.run(reqs)


def test_all_requests_complete_within_budget():
    rng = np.random.default_rng(3)
    t = poisson_arrivals(50.0, 40, rng)
    reqs = [(float(t[i]), SolveRequest(tag=(int(rng.integers(1, 5)), int(rng.integers(5, 60))))) for i in range(40)]
    batch, stats = _run(8, reqs)
    assert len(stats.completed) == 40
    assert batch.max_used <= 8 and batch.used == 0
    for c in stats.completed:
        assert c.admitted >= c.arrival and c.done >= c.admitted and c.latency > 0
    assert stats.percentile(99) >= stats.percentile(50) > 0
    assert stats.solves_per_s > 0


def test_requests_join_while_others_are_resident():
    # a long solve admitted first; a short one arriving later joins before the long one ends
    reqs = [(0.0, SolveRequest(tag=(2, 200))), (0.01, SolveRequest(tag=(2, 10)))]
    batch, stats = _run(8, reqs)
    by_steps = {c.steps: c for c in stats.completed}
    assert by_steps[10].admitted < by_steps[200].done
    assert by_steps[10].done < by_steps[200].done
    assert max(n for (_, _, n) in batch.log) == 2


def test_fifo_admission_waits_for_room():
    # the second request does not fit until the first is released; the third (small) waits behind it
    reqs = [(0.0, SolveRequest(tag=(6, 30))), (0.001, SolveRequest(tag=(6, 5))), (0.002, SolveRequest(tag=(1, 5)))]
    batch, stats = _run(8, reqs)
    done = {c.request.tag: c for c in stats.completed}
    assert done[(6, 5)].admitted >= done[(6, 30)].done
    assert done[(1, 5)].admitted >= done[(6, 5)].admitted
    assert stats.admissions_deferred > 0


class FakeNativeServer:
    """Stand-in for serve.Server (the native loop): every solve is admitted at once and done
    `steps * 1 ms` after its submission; records the order and times of the submissions."""

    def __init__(self):
        import time
        self.t0 = time.perf_counter()
        self.jobs, self.order = {}, []

    def submit_request(self, req):
        import time
        t = len(self.jobs) + 1
        _, _, nsteps = req.prepare()
        self.jobs[t] = (req, time.perf_counter() - self.t0, nsteps)
        self.order.append(t)
        return t

    def wait(self, ticket, timeout=3600.0):
        return 2

    def result(self, ticket, ndofs):
        req, sub, nsteps = self.jobs.pop(ticket)
        return np.zeros(ndofs), 0, (0.0, 1e-3 * nsteps)

    def stats(self):
        return {"queued": 0, "admissions_deferred": 0, "max_resident": 1, "launches": 0}


class _Req:
    def __init__(self, nsteps):
        self.nsteps, self.ndofs = nsteps, 4

    def prepare(self):
        return None, 0.1, self.nsteps


def test_native_serving_loop_accounting():
    from philip_b200.serve import serve_native
    arrivals = [(0.0, _Req(5)), (0.02, _Req(3)), (0.01, _Req(7))]
    srv = FakeNativeServer()
    stats = serve_native(srv, arrivals)
    assert len(stats.completed) == 3 and not srv.jobs           # every ticket collected once
    # submitted in arrival order, each no earlier than its arrival time
    assert [c.request.nsteps for c in sorted(stats.completed, key=lambda c: c.admitted)] == [5, 7, 3]
    for c in stats.completed:
        assert c.admitted >= c.arrival - 1e-9
        assert abs((c.done - c.admitted) - 1e-3 * c.steps) < 1e-12
        assert c.latency >= 1e-3 * c.steps - 1e-9
    assert stats.makespan == max(c.done for c in stats.completed)
