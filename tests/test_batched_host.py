"""Host scheduling of BatchedFloorPolicy.run_many, without a GPU: with stand-in
workers and a stand-in for the CUDA stream calls, state k goes to worker
k mod width, each worker takes its states in order on its own thread and
stream, rows come back in input order, on_result sees every state on its
worker, and a worker's exception is raised on the calling thread."""

import contextlib
import threading
import types

import pytest

from gpu_fem import policy as pol


class _Stream:
    def __init__(self, name):
        self.name = name
        self.waited = []

    def wait_stream(self, other):
        self.waited.append(other.name)


def _fake_torch(current):
    cuda = types.SimpleNamespace()
    local = threading.local()
    cuda.current_stream = lambda: getattr(local, "s", current)

    @contextlib.contextmanager
    def stream(s):
        old = getattr(local, "s", current)
        local.s = s
        try:
            yield
        finally:
            local.s = old

    cuda.stream = stream
    return types.SimpleNamespace(cuda=cuda), local


class _Worker:
    def __init__(self, i, fail_on=None, local=None):
        self.i, self.seen, self.fail_on, self.local = i, [], fail_on, local

    def run(self, density, binary=False):
        if density == self.fail_on:
            raise RuntimeError(f"state {density} failed")
        self.seen.append((density, self.local.s.name, threading.get_ident()))
        return {"state": density, "worker": self.i, "binary": binary}


def _batched(width, monkeypatch, fail_on=None):
    caller = _Stream("caller")
    torch, local = _fake_torch(caller)
    monkeypatch.setattr(pol._lib, "require_cuda", lambda: torch)
    b = object.__new__(pol.BatchedFloorPolicy)
    b.width = width
    b.workers = [_Worker(i, fail_on, local) for i in range(width)]
    b.streams = [_Stream(f"s{i}") for i in range(width)]
    return b, caller


def test_round_robin_in_order_on_own_streams(monkeypatch):
    b, caller = _batched(3, monkeypatch)
    got = []
    rows = b.run_many(list(range(10)), binary=True, on_result=lambda k, w, r: got.append((k, w.i)))
    assert [r["state"] for r in rows] == list(range(10))
    assert all(r["worker"] == k % 3 and r["binary"] for k, r in enumerate(rows))
    for i, w in enumerate(b.workers):
        assert [s for s, _, _ in w.seen] == list(range(i, 10, 3))
        assert {name for _, name, _ in w.seen} == {f"s{i}"}
        assert len({t for _, _, t in w.seen}) == 1
    assert sorted(got) == [(k, k % 3) for k in range(10)]
    # every worker stream waits for the caller's inputs, the caller for every worker
    assert all(s.waited == ["caller"] for s in b.streams)
    assert caller.waited == ["s0", "s1", "s2"]


def test_fewer_states_than_workers(monkeypatch):
    b, _ = _batched(4, monkeypatch)
    rows = b.run_many([7, 8])
    assert [r["state"] for r in rows] == [7, 8] and [r["worker"] for r in rows] == [0, 1]
    assert b.workers[2].seen == [] and b.workers[3].seen == []


def test_worker_error_reaches_the_caller(monkeypatch):
    b, _ = _batched(2, monkeypatch, fail_on=5)
    with pytest.raises(RuntimeError, match="state 5 failed"):
        b.run_many(list(range(8)))
