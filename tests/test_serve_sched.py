"""The serving scheduler (exmarg_b200.serve.Scheduler): admission by workspace budget, on the CPU."""

from exmarg_b200.serve import Scheduler, workspace_bytes


def test_admission_respects_budget_and_worker_limit():
    cost = {"a": 40, "b": 70}
    s = Scheduler(budget=100, cost=lambda k: cost[k], max_workers=3)
    for i in range(4):
        s.push(("a", i), "a")
    s.push(("b", 0), "b")
    got = []
    while True:
        g = s.admit()
        if g[0] is None:
            break
        got.append(g)
    # two 'a' workers fit (80 of 100); a third 'a' or a 'b' worker would exceed the budget
    assert [g[0] for g in got] == [("a", 0), ("a", 1)]
    assert s.used == 80 and s.n_workers() == 2
    assert all(g[3] for g in got)                       # both were new workers
    s.release(got[0][2])
    g = s.admit()                                       # the freed 'a' worker takes the next 'a' request
    assert g[0] == ("a", 2) and g[2] == got[0][2] and not g[3]
    assert s.used == 80


def test_out_of_order_admission_when_the_head_is_blocked():
    cost = {"big": 90, "small": 10}
    s = Scheduler(budget=100, cost=lambda k: cost[k], max_workers=4)
    s.push("big0", "big")
    s.push("big1", "big")
    s.push("small0", "small")
    a = s.admit()
    assert a[0] == "big0"
    b = s.admit()                                       # big1 cannot start, small0 can
    assert b[0] == "small0"
    assert s.admit()[0] is None
    s.release(a[2])
    c = s.admit()
    assert c[0] == "big1" and c[2] == a[2]


def test_workspace_estimate_grows_with_the_bank():
    small = workspace_bytes(256, 16384, 53, 87, 1969, 2048)
    big = workspace_bytes(2048, 32768, 53, 87, 3937, 2048)
    assert 0 < small < big
    assert 8e9 < big < 20e9


def test_idle_workers_of_another_bank_are_evicted():
    cost = {"a": 60, "b": 60}
    s = Scheduler(budget=100, cost=lambda k: cost[k], max_workers=4)
    s.push("a0", "a")
    a = s.admit()
    s.release(a[2])                                     # an idle 'a' worker holds 60 of 100
    s.push("b0", "b")
    b = s.admit()
    assert b[0] == "b0" and b[3] and b[4] == [a[2]]     # the idle 'a' worker was evicted for it
    assert s.used == 60
    s.push("a1", "a")
    assert s.admit()[0] is None                         # 'b' is busy: nothing to evict


def test_recost_follows_live_workers():
    cost = {"a": 50}
    s = Scheduler(budget=100, cost=lambda k: cost[k], max_workers=4)
    for i in range(2):
        s.push(i, "a")
    assert s.admit()[0] == 0 and s.admit()[0] == 1
    assert s.used == 100
    s.recost("a", 30, cost.__setitem__)                  # measured smaller than estimated
    assert cost["a"] == 30 and s.used == 60
    s.push(2, "a")
    assert s.admit()[0] == 2 and s.used == 90


def test_idle_worker_with_queued_work_is_kept():
    cost = {"a": 60, "b": 60}
    s = Scheduler(budget=100, cost=lambda k: cost[k], max_workers=4)
    s.push("a0", "a")
    a = s.admit()
    s.release(a[2])
    s.push("b0", "b")
    s.push("a1", "a")                                   # 'a' has queued work: its idle worker stays
    g = s.admit()
    assert g[0] == "a1" and g[2] == a[2] and g[4] == []
    assert s.admit()[0] is None                         # b0 waits for the budget


def test_busy_bank_waits_instead_of_evicting():
    cost = {"a": 40, "b": 40}
    s = Scheduler(budget=100, cost=lambda k: cost[k], max_workers=2)
    s.push("a0", "a")
    s.push("b0", "b")
    a = s.admit()
    b = s.admit()
    s.release(b[2])                                     # 'b' idle, 'a' busy
    s.push("a1", "a")
    g = s.admit()
    assert g[0] is None and g[4] == []                  # no second 'a' worker at the price of 'b''s
    s.release(a[2])
    assert s.admit()[0] == "a1"


def test_a_worker_that_cannot_open_fails_its_request_and_frees_its_budget(monkeypatch):
    # the server's host logic with fakes for the device: bank 'bad' cannot get a worker (its context runs
    # out of memory); its request must fail with that error instead of waiting forever, the slot and budget
    # must come back, and the other bank's requests are served
    from types import SimpleNamespace

    import numpy as np
    import pytest

    from exmarg_b200 import serve

    class FakeWorker:
        def __init__(self, parent, bank, store, prior, ymin, graph=False):
            if bank.name == "bad":
                raise MemoryError("no room for the workspace")
            self.ctx = SimpleNamespace(bytes=10)

        def prioritise(self, rank):
            pass

        def run(self, segments, row, seed, n_loud, n_random):
            return np.array([[float(seed)]]), np.array([1.5])

        def close(self):
            pass

    monkeypatch.setattr(serve._lib, "context", lambda device: object())
    monkeypatch.setattr(serve, "upload_store", lambda store, ctx: None)
    monkeypatch.setattr(serve, "_Worker", FakeWorker)
    store = SimpleNamespace(tables=[SimpleNamespace(shape=(87, 49, 200, 219))] * 3)
    bank = lambda name: SimpleNamespace(name=name, u=np.zeros(16), n_time=16384, W=np.zeros((16, 100)))
    srv = serve.Server(store, {"good": bank("good"), "bad": bank("bad")}, hbm_budget=1 << 40, max_workers=2)
    reqs = [serve.Request(0, "bad", None, seed=3), serve.Request(1, "good", None, seed=4),
            serve.Request(2, "good", None, seed=5)]
    srv.serve(reqs)
    with pytest.raises(MemoryError, match="no room"):
        reqs[0].future.result(timeout=0)
    assert [r.future.result(timeout=0)[1] for r in reqs[1:]] == [1.5, 1.5]
    assert srv.n_created == 1 and srv.sched.n_workers() == 1
    assert srv.sched.used == 10                           # the good worker's measured size only
    assert not srv.sched.busy
