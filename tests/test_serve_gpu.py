"""Serving loop: continuous batching, memory-budget admission, and results that
do not depend on what else is being served."""
import numpy as np
import pytest

from bfvm import workloads as W
from bfvm.serve import (Server, SolveRequest, create_solve, estimate_bytes, poisson_arrivals,
                        run_one_at_a_time)


def _requests(n, seed=11, keep=True, **kw):
    arr = poisson_arrivals(n, rate=2000.0, seed=seed)
    args = dict(edge_lo=16, edge_hi=40, steps_lo=20, steps_hi=70, agents_hi=2000)
    args.update(kw)
    return [SolveRequest(i, W.serve_request(i, seed=seed, **args), float(arr[i]), keep) for i in range(n)]


def _alone(req, precision):
    me = create_solve(req.workload, precision)
    me.simulate_diffusion_decay(int(req.workload.steps), sources=True)
    out = me.download_field()
    me.close()
    return out


def test_poisson_arrivals_are_seeded_and_increasing():
    a = poisson_arrivals(50, rate=10.0, seed=3)
    assert np.all(np.diff(a) > 0)
    assert np.array_equal(a, poisson_arrivals(50, rate=10.0, seed=3))
    assert 2.0 < a[-1] < 10.0


def test_estimate_grows_with_size_and_agents():
    small = W.serve_request(0, edge_lo=16, edge_hi=16, agents_hi=0, steps_lo=1, steps_hi=1)
    big = W.serve_request(0, edge_lo=64, edge_hi=64, agents_hi=0, steps_lo=1, steps_hi=1)
    assert 0 < estimate_bytes(small, "fp32") < estimate_bytes(big, "fp32")
    assert estimate_bytes(big, "fp32") < estimate_bytes(big, "fp64")
    field_fp64 = big.n_values * 8
    assert estimate_bytes(big, "fp64") >= 2 * field_fp64   # field + transfer buffer


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_results_same_alone_and_in_mix(precision):
    reqs = _requests(7, seed=21)
    srv = Server(precision, quantum=8)
    st = srv.run(reqs)
    srv.close()
    assert sorted(r.rid for r in st.results) == list(range(7))
    assert st.quanta > len(reqs)  # members joined and left at different steps
    for res in st.results:
        req = reqs[res.rid]
        alone = _alone(req, precision)
        assert np.array_equal(res.field, alone), f"request {res.rid} differs in the mix"
        assert res.finished >= res.admitted >= res.arrival - 1e-9


@pytest.mark.gpu
def test_budget_limits_residency_and_rejects_oversized():
    reqs = _requests(6, seed=31, keep=False)
    sizes = [estimate_bytes(r.workload, "fp32") for r in reqs]
    budget = max(sizes) + min(sizes)  # never more than about two at a time
    huge = SolveRequest(99, W.serve_request(99, seed=31, edge_lo=120, edge_hi=120, steps_lo=2, steps_hi=2,
                                            agents_hi=0), 0.0, False)
    assert estimate_bytes(huge.workload, "fp32") > budget
    srv = Server("fp32", budget_bytes=budget, quantum=16)
    st = srv.run(reqs + [huge])
    srv.close()
    assert st.rejected == [99]
    assert sorted(r.rid for r in st.results) == list(range(6))
    assert st.peak_bytes <= budget


@pytest.mark.gpu
def test_one_at_a_time_path_gives_the_same_fp64_results():
    reqs = _requests(4, seed=41)
    srv = Server("fp64", quantum=16)
    st = srv.run(reqs)
    srv.close()
    base = run_one_at_a_time(reqs, "fp64")
    got = {r.rid: r.field for r in st.results}
    for r in base.results:
        assert np.array_equal(r.field, got[r.rid])
    summ = st.summary()
    assert summ["requests"] == 4 and summ["p99_s"] >= summ["p50_s"] > 0


@pytest.mark.gpu
def test_cancelled_request_leaves_the_others_unchanged():
    """One request is cancelled while it runs in the batch; every other
    result is bit-identical to the same request served alone."""
    reqs = _requests(5, seed=51, steps_lo=60, steps_hi=90)
    srv = Server("fp64", quantum=8)

    def on_quantum(server, quanta):
        if quanta == 3:
            server.cancel(2)

    st = srv.run(reqs, on_quantum=on_quantum)
    srv.close()
    assert [rid for rid, _ in st.cancelled] == [2]
    assert 0 < st.cancelled[0][1] < reqs[2].workload.steps
    assert sorted(r.rid for r in st.results) == [0, 1, 3, 4]
    for res in st.results:
        assert np.array_equal(res.field, _alone(reqs[res.rid], "fp64")), res.rid
