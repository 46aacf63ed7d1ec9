"""The serving loop's host logic (bfvm/serve.py: FIFO admission under a
device-memory budget, one quantum of LOD steps for every resident solve, never
past the end of any of them, retirement and freeing), on the CPU with a fake
batched engine, fake solves and a deterministic clock -- no device involved.
"""
import types

import pytest

from bfvm import serve


class FakeClock:
    """Advances by `dt` seconds per reading."""

    def __init__(self, dt=0.001):
        self.t = 0.0
        self.dt = dt

    def __call__(self):
        self.t += self.dt
        return self.t


class FakeSolve:
    def __init__(self, wl):
        self.wl = wl
        self.steps = 0
        self.closed = False

    def download_field(self):
        return None

    def synchronize(self):
        pass

    def close(self):
        self.closed = True


class FakeBatch:
    """Records members, the quanta stepped and each member's step count."""

    def __init__(self, precision, device):
        self.members = []
        self.quanta = []
        self.max_members = 0

    def set_schedule(self, **kw):
        pass

    def add(self, me):
        assert me not in self.members
        self.members.append(me)
        self.max_members = max(self.max_members, len(self.members))

    def remove(self, me):
        self.members.remove(me)

    def step(self, k, sources=True):
        assert k >= 1 and self.members
        for me in self.members:
            me.steps += k
            assert me.steps <= me.wl.steps, "a solve was stepped past its end"
        self.quanta.append(k)

    def synchronize(self):
        pass

    def close(self):
        pass


def _workload(steps, nbytes, n_values=1000):
    return types.SimpleNamespace(steps=steps, n_values=n_values, nbytes=nbytes)


@pytest.fixture
def fakes(monkeypatch):
    made = []

    def create(wl, precision, device=0):
        me = FakeSolve(wl)
        made.append(me)
        return me

    monkeypatch.setattr(serve, "Batch", FakeBatch)
    monkeypatch.setattr(serve, "create_solve", create)
    monkeypatch.setattr(serve, "estimate_bytes", lambda wl, precision: wl.nbytes)
    return made


def test_budget_fifo_and_exact_step_counts(fakes):
    reqs = [serve.SolveRequest(i, _workload(steps, nbytes), arrival=0.0)
            for i, (steps, nbytes) in enumerate([(100, 40), (30, 40), (250, 40), (7, 30), (64, 10)])]
    srv = serve.Server(budget_bytes=100, quantum=64)
    st = srv.run(reqs, clock=FakeClock())
    assert sorted(r.rid for r in st.results) == [0, 1, 2, 3, 4]
    assert st.rejected == []
    assert st.peak_bytes <= 100
    assert srv.batch.max_members <= 3  # 40 + 40 + 10 fits, a third 40 does not
    # every solve ran exactly its step count and was freed
    for me in fakes:
        assert me.steps == me.wl.steps and me.closed
    # a quantum never exceeds the configured 64 steps
    assert max(srv.batch.quanta) <= 64
    # admission is FIFO: a solve is admitted no earlier than any request ahead of it
    admitted = {r.rid: r.admitted for r in st.results}
    assert admitted[0] <= admitted[1] <= admitted[2] <= admitted[3] <= admitted[4]


def test_requests_larger_than_the_budget_are_rejected(fakes):
    reqs = [serve.SolveRequest(0, _workload(10, 500)), serve.SolveRequest(1, _workload(10, 50)),
            serve.SolveRequest(2, _workload(10, 101))]
    srv = serve.Server(budget_bytes=100, quantum=8)
    st = srv.run(reqs, clock=FakeClock())
    assert sorted(st.rejected) == [0, 2]
    assert [r.rid for r in st.results] == [1]
    assert fakes[0].steps == 10


def test_later_arrivals_wait_for_their_time(fakes):
    clock = FakeClock(dt=0.01)
    reqs = [serve.SolveRequest(0, _workload(5, 10), arrival=0.0), serve.SolveRequest(1, _workload(5, 10), arrival=0.5)]
    st = serve.Server(budget_bytes=100, quantum=4).run(reqs, clock=clock)
    res = {r.rid: r for r in st.results}
    assert res[0].admitted < 0.5 <= res[1].admitted
    assert all(r.latency > 0 for r in st.results)
    s = st.summary()
    assert s["requests"] == 2 and s["updates"] == 2 * 5 * 1000 and s["wall_s"] > 0


def test_cancellation_frees_the_solve_and_leaves_the_others_exact(fakes):
    """Request 1 is cancelled after the second quantum (running) and request
    3 before it is admitted (waiting); both are reported with the steps they
    got, their solves are freed, and every other request runs exactly its
    step count."""
    reqs = [serve.SolveRequest(i, _workload(steps, nbytes), arrival=0.0)
            for i, (steps, nbytes) in enumerate([(300, 30), (500, 30), (90, 30), (200, 60), (40, 10)])]
    srv = serve.Server(budget_bytes=100, quantum=32)

    def on_quantum(server, quanta):
        if quanta == 2:
            server.cancel(1)
            server.cancel(3)

    st = srv.run(reqs, clock=FakeClock(), on_quantum=on_quantum)
    done = dict(st.cancelled)
    assert set(done) == {1, 3}
    assert done[1] == 64 and done[3] == 0  # two quanta of 32, and never admitted
    assert sorted(r.rid for r in st.results) == [0, 2, 4]
    by_steps = {me.wl.steps: me for me in fakes}
    assert 200 not in by_steps  # request 3 was never created
    assert by_steps[500].closed and by_steps[500].steps == 64
    for steps in (300, 90, 40):
        assert by_steps[steps].steps == steps and by_steps[steps].closed
    assert st.summary()["cancelled"] == 2


def test_cancelling_an_unknown_or_finished_request_changes_nothing(fakes):
    reqs = [serve.SolveRequest(0, _workload(10, 10)), serve.SolveRequest(1, _workload(20, 10))]
    srv = serve.Server(budget_bytes=100, quantum=8)
    srv.cancel(99)
    st = srv.run(reqs, clock=FakeClock())
    assert sorted(r.rid for r in st.results) == [0, 1] and st.cancelled == []
