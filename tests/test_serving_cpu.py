"""Serving layer logic (idx2_b200.serving) on the CPU: schedule, admission under the memory
budget, batching of queued requests, latency accounting, with a simulated clock and a fake
decoder (no GPU)."""
import numpy as np

from idx2_b200.serving import Request, Server, output_dims, poisson_schedule, request_cost


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += max(dt, 1e-9)


def test_output_dims_rounding():
    # first rounded down, last rounded up to the stride (GetGrid)
    assert output_dims((5, 0, 0), (13, 7, 0), (2, 0, 0)) == (4, 8, 1)
    assert output_dims((0, 0, 0), (31, 31, 31), (0, 0, 0)) == (32, 32, 32)


def test_schedule_is_seeded_and_in_range():
    a = poisson_schedule(200, 2000.0, (2048, 2048, 1024), seed=3)
    b = poisson_schedule(200, 2000.0, (2048, 2048, 1024), seed=3)
    assert [r.first for r in a] == [r.first for r in b]
    arr = np.array([r.arrival for r in a])
    assert np.all(np.diff(arr) > 0)
    assert 0.05 < arr[-1] < 0.2  # about 200 / 2000 s
    for r in a:
        for f, l, d in zip(r.first, r.last, (2048, 2048, 1024)):
            assert 0 <= f <= l < d and 32 <= l - f + 1 <= 512
        assert all(0 <= x <= 3 for x in r.downsampling)
        assert 1e-6 <= r.tolerance <= 1e-1
        assert r.cost >= r.out_bytes > 0


def _reqs(costs, gap=0.0):
    return [Request(i * gap, (0, 0, 0), (31, 31, 31), (0, 0, 0), 1e-3, c, c) for i, c in enumerate(costs)]


def test_admission_respects_budget_and_order():
    s = Server(lambda b: 0.0, budget=100)
    q = _reqs([40, 40, 30, 10])
    assert [r.cost for r in s.admit(q)] == [40, 40]  # the third would exceed 100
    s2 = Server(lambda b: 0.0, budget=100, max_batch=1)
    assert len(s2.admit(q)) == 1


def test_batched_beats_one_at_a_time_when_decode_has_fixed_cost():
    clk = FakeClock()
    calls = []

    def decode(batch):
        calls.append(len(batch))
        clk.t += 0.002 + 0.0001 * len(batch)  # fixed launch cost + per-request cost
        return 0.0

    sched = _reqs([1] * 200, gap=0.0005)  # 2000 req/s
    one = Server(decode, budget=10**9, clock=clk, sleep=clk.sleep).run([Request(**r.__dict__) for r in sched],
                                                                      batched=False)
    clk.t = 0.0
    calls.clear()
    bat = Server(decode, budget=10**9, clock=clk, sleep=clk.sleep).run([Request(**r.__dict__) for r in sched],
                                                                      batched=True)
    assert one.requests == bat.requests == 200
    assert bat.batches < one.batches == 200
    assert bat.p99_ms < one.p99_ms


def test_oversized_requests_are_rejected():
    clk = FakeClock()
    srv = Server(lambda b: 0.0, budget=50, clock=clk, sleep=clk.sleep)
    st = srv.run(_reqs([10, 60, 10], gap=0.001))
    assert st.rejected == 1 and st.requests == 2


def test_request_cost_counts_bricks():
    ob, cost = request_cost((0, 0, 0), (63, 63, 63), (0, 0, 0), 4)
    assert ob == 64 ** 3 * 4 and cost > ob
