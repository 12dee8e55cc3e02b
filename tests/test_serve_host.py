"""Host logic of the served loop on the CPU: admission against the budget, eviction, continuous
batching and per-client order.

The device side is replaced by fakes (handles, batches, CUDA events and streams) that record
what the loop asks of them; a fake batch finishes after it has been polled twice, so requests
that arrive meanwhile have to wait for the next batch slot.
"""
import collections

import pytest
import torch

from reproducibility_icpp23_scalable_gpu_deduplication_b200 import serve

LOG = collections.defaultdict(list)


class FakeEvent:
    def record(self, stream=None):
        pass

    def query(self):
        return True

    def synchronize(self):
        pass


class FakeStream:
    def wait_event(self, ev):
        pass

    def synchronize(self):
        LOG["stream_syncs"].append(self)


class FakeHandle:
    grow = 0              # bytes a handle's memory grows by per checkpoint

    def __init__(self, chunk_size, hash_kind):
        self.client = None
        self.closed = False
        self.count = 0
        self.mem = 100
        LOG["created"].append(self)

    def checkpoint_device(self, buf, make_baseline=False):
        assert not self.closed
        self.count += 1
        self.mem += self.grow
        LOG["checkpoints"].append((self, self.count, int(buf[0])))

    def memory(self):
        return self.mem

    @property
    def current_id(self):       # ids count this handle's checkpoints, from 0
        return self.count

    def diff_device(self):
        return 0, 32

    def diff_checksum(self):
        return self.count

    def close(self):
        assert not self.closed
        self.closed = True


class FakeListHandle(FakeHandle):
    pass


class FakeBatch:
    def __init__(self, **params):
        self.inflight = 0
        self.polls = 0

    def launch(self, handles, buffers, make_baseline=None, stream=None):
        assert self.inflight == 0 and len(handles) == len(buffers)
        assert len(set(map(id, handles))) == len(handles), "a client twice in one batch"
        LOG["batches"].append(len(handles))
        for h, b, mb in zip(handles, buffers, make_baseline):
            h.checkpoint_device(b, mb)
        self.inflight = len(handles)
        self.polls = 0

    def done(self):
        self.polls += 1
        return self.polls >= 2

    def wait(self, check_status=True):
        n, self.inflight = self.inflight, 0
        return [0] * n

    def close(self):
        pass


@pytest.fixture
def fakes(monkeypatch):
    LOG.clear()
    FakeHandle.grow = 0
    monkeypatch.setattr(torch.cuda, "Event", FakeEvent)
    monkeypatch.setattr(torch.cuda, "Stream", FakeStream)
    monkeypatch.setattr(torch.cuda, "current_stream", lambda *a: FakeStream())
    monkeypatch.setattr(serve, "CheckpointBatch", FakeBatch)
    monkeypatch.setattr(serve, "TreeDeduplicator", FakeHandle)
    monkeypatch.setattr(serve, "ListDeduplicator", FakeListHandle)
    monkeypatch.setattr(serve, "estimate_memory", lambda nbytes, cs: 100)
    monkeypatch.setattr(serve, "reserve_map_memory", lambda nbytes: None)
    return LOG


def drive(srv, clients, rounds, burst=3):
    """every client submits `rounds` requests, interleaved; buffer k of client c holds c*100+k"""
    order = [c for k in range(rounds) for c in range(clients)]
    count = [0] * clients
    reqs = []
    for i, c in enumerate(order):
        while srv.busy(c):
            srv.step()
        reqs.append(srv.submit(c, torch.full((64,), c * 100 + count[c], dtype=torch.int32)))
        count[c] += 1
        if i % burst == burst - 1:
            srv.step()
    srv.drain()
    return reqs


def per_client_in_order(log):
    seen = collections.defaultdict(list)
    for h, n, v in log["checkpoints"]:
        seen[v // 100].append(v % 100)
    return all(vs == sorted(vs) and vs == list(range(len(vs))) for vs in seen.values())


def test_continuous_batching(fakes):
    srv = serve.CheckpointServer(hbm_budget=10_000, max_batch=3, max_inflight=2)
    reqs = drive(srv, clients=5, rounds=4)
    assert all(r.rc == 0 and r.done is not None for r in reqs)
    assert per_client_in_order(fakes)
    assert srv.batches == len(fakes["batches"]) < len(reqs)        # requests shared batches
    assert max(fakes["batches"]) <= 3 and max(fakes["batches"]) > 1
    assert len(fakes["created"]) == 5                              # one resident handle per client
    assert all(r.admitted <= r.launched <= r.done for r in reqs)
    assert srv.idle() and len(srv.completed) == len(reqs)
    srv.close()
    assert all(h.closed for h in fakes["created"])


def test_one_request_per_client_in_flight(fakes):
    """a client's later requests wait behind its launched one, in arrival order"""
    srv = serve.CheckpointServer(hbm_budget=10_000, max_batch=8, max_inflight=2)
    r = [srv.submit(0, torch.full((8,), k, dtype=torch.int32)) for k in range(3)]
    srv.step()
    assert r[0].launched is not None and r[1].launched is None
    srv.drain()
    assert r[0].done <= r[1].launched and r[1].done <= r[2].launched
    assert [v for _, _, v in fakes["checkpoints"]] == [0, 1, 2]
    srv.close()


def test_admission_evicts_least_recently_used(fakes):
    """a budget of two clients' state: never exceeded, idle clients evicted, an evicted client
    comes back on a fresh handle (its next request is a baseline)"""
    srv = serve.CheckpointServer(hbm_budget=250, max_batch=4, max_inflight=2)
    reqs = drive(srv, clients=4, rounds=3, burst=1)
    assert all(r.rc == 0 for r in reqs)
    assert srv.peak_resident <= 250
    assert sum(1 for c in srv.clients.values() if c.handle is not None) <= 2
    assert len(fakes["created"]) > 4
    assert sum(h.closed for h in fakes["created"]) == len(fakes["created"]) - 2
    assert per_client_in_order(fakes)
    srv.close()


def test_waits_without_eviction(fakes):
    srv = serve.CheckpointServer(hbm_budget=150, evict=False)
    r0 = srv.submit(0, torch.zeros(8, dtype=torch.int32))
    r1 = srv.submit(1, torch.ones(8, dtype=torch.int32))
    for _ in range(10):
        srv.step()
    assert r0.done is not None and r0.rc == 0
    assert r1.admitted is None and not srv.idle()
    srv.close()


def test_map_growth_keeps_reservation_honest(fakes):
    """a handle whose memory grows past its estimate raises the resident total by the growth"""
    FakeHandle.grow = 40
    srv = serve.CheckpointServer(hbm_budget=10_000)
    drive(srv, clients=2, rounds=3)
    assert srv.resident == sum(c.handle.memory() for c in srv.clients.values())
    assert srv.resident == 2 * (100 + 3 * 40)
    srv.close()


def test_plain_loop_serves_in_arrival_order(fakes):
    srv = serve.CheckpointServer(hbm_budget=10_000, plain=True)
    reqs = drive(srv, clients=3, rounds=3)
    assert not fakes["batches"] and srv.batches == len(reqs)
    done = sorted(reqs, key=lambda r: r.done)
    assert [r.seq for r in done] == sorted(r.seq for r in reqs)
    srv.close()


@pytest.mark.parametrize("plain", [False, True])
def test_list_approach_builds_list_handles(fakes, plain):
    srv = serve.CheckpointServer(hbm_budget=10_000, approach="list", plain=plain)
    drive(srv, clients=3, rounds=2)
    assert fakes["created"] and all(type(h) is FakeListHandle for h in fakes["created"])
    srv.close()


def test_percentile():
    assert serve.percentile([3, 1, 2], 50) == 2
    assert serve.percentile([1, 2, 3, 4], 100) == 4
    assert serve.percentile([1, 2, 3, 4], 0) == 1
    assert serve.percentile([0, 10], 25) == 2.5
    assert serve.percentile([], 50) is None


class FailingBatch(FakeBatch):
    """reports a device failure for the handles in `fail` (once each)"""
    fail = set()

    def launch(self, handles, buffers, make_baseline=None, stream=None):
        LOG["launch_flags"].append([(h, bool(mb)) for h, mb in zip(handles, make_baseline)])
        self.handles = list(handles)
        super().launch(handles, buffers, make_baseline, stream)

    def wait(self, check_status=True):
        rcs = super().wait(check_status)
        for i, h in enumerate(self.handles):
            if h in self.fail:
                self.fail.discard(h)
                rcs[i] = -7
        return rcs


def flags_of(log, handle):
    return [mb for batch in log["launch_flags"] for h, mb in batch if h is handle]


def test_baselines_chosen_by_the_loop(fakes, monkeypatch):
    """first request on a handle, a length change, a client's request and a failed request each
    make the client's next (or own) checkpoint a baseline; everything else is incremental"""
    monkeypatch.setattr(serve, "CheckpointBatch", FailingBatch)
    srv = serve.CheckpointServer(hbm_budget=10_000, max_batch=4)
    buf = lambda n, v=0: torch.full((n,), v, dtype=torch.uint8)
    srv.submit(0, buf(64))
    srv.submit(1, buf(64))
    srv.drain()
    h0, h1 = srv.clients[0].handle, srv.clients[1].handle
    FailingBatch.fail = {h1}
    srv.submit(0, buf(64, 1))                   # incremental
    srv.submit(1, buf(64, 1))                   # fails on the device
    srv.drain()
    srv.submit(0, buf(128))                     # length change
    srv.submit(1, buf(64, 2))                   # after a failure
    srv.drain()
    srv.submit(0, buf(128, 3), make_baseline=True)
    srv.submit(1, buf(64, 3))
    srv.drain()
    assert flags_of(fakes, h0) == [True, False, True, True]
    assert flags_of(fakes, h1) == [True, False, True, False]
    rcs = [r.rc for r in srv.completed]
    assert rcs.count(-7) == 1 and rcs.count(0) == len(rcs) - 1
    assert [r.baseline for r in srv.completed if r.client == 1] == [True, False, True, False]
    srv.close()


def test_empty_buffer_rejected_at_submit(fakes):
    srv = serve.CheckpointServer(hbm_budget=10_000)
    with pytest.raises(ValueError):
        srv.submit(0, torch.empty(0, dtype=torch.uint8))
    assert srv.idle() and not srv.busy(0)
    srv.close()


def test_client_moves_to_a_new_handle_at_the_id_limit(fakes, monkeypatch):
    """a client that has used up a handle's checkpoint ids continues on a new handle, starting
    with a baseline; the old handle is closed"""
    monkeypatch.setattr(serve, "MAX_CHECKPOINTS_PER_HANDLE", 3)
    monkeypatch.setattr(serve, "CheckpointBatch", FailingBatch)
    FailingBatch.fail = set()
    srv = serve.CheckpointServer(hbm_budget=10_000)
    for k in range(7):
        srv.submit(0, torch.full((64,), k, dtype=torch.uint8))
        srv.drain()
    hs = fakes["created"]
    assert len(hs) == 3 and hs[0].closed and hs[1].closed and not hs[2].closed
    assert [h.count for h in hs] == [3, 3, 1]
    assert [r.baseline for r in srv.completed] == [True, False, False, True, False, False, True]
    # each request carries the id its diff has on its handle (the index to restart it by)
    assert [r.chkpt_id for r in srv.completed] == [0, 1, 2, 0, 1, 2, 0]
    assert all(r.rc == 0 for r in srv.completed)
    srv.close()


class RaisingBatch(FakeBatch):
    """a launch that fails as a whole (as a CUDA error at launch would)"""
    raise_for = set()

    def launch(self, handles, buffers, make_baseline=None, stream=None):
        LOG["launch_flags"].append([(h, bool(mb)) for h, mb in zip(handles, make_baseline)])
        if any(h in self.raise_for for h in handles):
            self.raise_for.clear()
            err = RuntimeError("launch failed")
            err.code = -2
            raise err
        super().launch(handles, buffers, make_baseline, stream)


def test_failed_launch_completes_its_requests(fakes, monkeypatch):
    """a batch whose launch raises completes its requests with the error code; the loop keeps
    serving, and those clients' next requests are baselines"""
    monkeypatch.setattr(serve, "CheckpointBatch", RaisingBatch)
    srv = serve.CheckpointServer(hbm_budget=10_000, max_batch=4)
    buf = lambda v: torch.full((64,), v, dtype=torch.uint8)
    for c in range(2):
        srv.submit(c, buf(0))
    srv.drain()
    h0, h1 = srv.clients[0].handle, srv.clients[1].handle
    RaisingBatch.raise_for = {h0}
    r = [srv.submit(c, buf(1)) for c in range(2)]
    srv.drain()
    assert [x.rc for x in r] == [-2, -2] and all(x.done is not None for x in r)
    # the slot's stream was synchronised before those clients became idle again
    assert len(fakes["stream_syncs"]) == 1
    assert not srv.busy(0) and not srv.busy(1)
    r2 = [srv.submit(c, buf(2)) for c in range(2)]
    srv.drain()
    assert [x.rc for x in r2] == [0, 0] and [x.baseline for x in r2] == [True, True]
    assert flags_of(fakes, h0) == [True, False, True] and flags_of(fakes, h1) == [True, False, True]
    srv.close()
