"""Served form: a request loop over many clients' checkpoint requests, with continuous batching.

The reference has no server; its driver checkpoints one buffer per call
(src/dedup_files.cpp:98-102 -> TreeDeduplicator::checkpoint, src/tree_approach.cpp:1705).  Here
clients submit "checkpoint my device buffer now" requests as they arrive.  The loop

* keeps each client's Merkle tree and digest map resident on the device between its requests
  (one ``TreeDeduplicator`` handle per client, or ``ListDeduplicator`` with
  ``approach="list"``), so every request after the first is an incremental checkpoint against
  that client's own previous one;
* admits a request when its client's state fits in the HBM budget (the handle's device bytes:
  ``estimate_memory`` before its first checkpoint, ``memory()`` after), evicting the least
  recently used idle clients when allowed (an evicted client's next request is a baseline);
* launches every admitted request whose client is idle as one batch (``CheckpointBatch``) as
  soon as a batch slot is free, while the batches already launched keep running on their own
  streams: requests that arrive during a batch join the next one (continuous batching), and up
  to ``max_inflight`` batches overlap on the device;
* completes a batch when its device work is done and stamps each request's completion time; with
  ``enable_host_copy`` a request completes once its diff has been copied back to pinned host
  memory (the copies of a batch run on its slot's stream while later batches compute).

A client has at most one request in flight; its later requests wait in arrival order.  Each
request's diff is exactly what its client's handle gives when it checkpoints the same buffers
alone, one request at a time.  A request is taken as a baseline (``Request.baseline``) when
its client asks for one, when it is the client's first on its handle, when its buffer length
differs from the client's previous request (the handle takes a new length only as a baseline)
and after a failed request of the client (its tree and map may be part-way updated); so one
client's bad request never fails a batch that other clients' requests share.

``plain=True`` serves the same requests the drop-in way instead: one request at a time, in
arrival order, each through its client's handle (``checkpoint_device``).
"""
import collections
import time

from ._lib import HASH_MURMUR3
from .batch import CheckpointBatch
from .tree import ListDeduplicator, TreeDeduplicator, estimate_memory, reserve_map_memory

__all__ = ["CheckpointServer", "Request"]

# a handle's checkpoint ids run 0..8190 (they keep counting across baselines; the digest map
# stores them in 13 bits): a client that reaches the end continues on a new handle
MAX_CHECKPOINTS_PER_HANDLE = 8191


class Request:
    __slots__ = ("client", "buffer", "nbytes", "make_baseline", "arrival", "admitted", "launched", "done", "rc",
                 "diff_len", "checksum", "ready", "seq", "host", "launch_s", "batch_size", "baseline", "chkpt_id")

    def __init__(self, client, buffer, make_baseline, arrival, seq):
        self.client, self.buffer, self.make_baseline, self.arrival, self.seq = client, buffer, make_baseline, arrival, seq
        self.nbytes = buffer.numel() * buffer.element_size()
        self.admitted = self.launched = self.done = None
        self.rc = None
        self.diff_len = None
        self.checksum = None
        self.ready = None
        self.host = None          # the diff in pinned host memory (with enable_host_copy)
        self.launch_s = None      # host seconds its batch's launch call took
        self.batch_size = 1
        self.baseline = None      # whether it ran as a baseline (set at launch)
        self.chkpt_id = None      # the checkpoint id its diff carries on its client's handle (the
                                  # index to restart it by among that handle's diffs)

    @property
    def latency(self):
        return None if self.done is None else self.done - self.arrival


class _Client:
    __slots__ = ("handle", "reserved", "last_use", "busy", "pending", "outstanding", "host", "nbytes", "rebase",
                 "taken")

    def __init__(self):
        self.handle = None
        self.reserved = 0
        self.last_use = 0.0
        self.busy = False                     # a request of this client is in a launched batch
        self.pending = collections.deque()   # admitted, not launched
        self.outstanding = 0                 # submitted, not completed
        self.host = None                     # pinned buffer for diff copy-back
        self.nbytes = None                   # buffer length of the last launched request
        self.rebase = False                  # the next request runs as a baseline
        self.taken = 0                       # checkpoints launched on the current handle


class CheckpointServer:
    def __init__(self, hbm_budget=150e9, chunk_size=128, hash_kind=HASH_MURMUR3, max_batch=64, max_inflight=2,
                 evict=True, plain=False, checksum=False, clock=time.perf_counter, map_reserve=0, approach="tree",
                 **batch_params):
        """`map_reserve`: bytes of device memory kept mapped for digest maps
        (``reserve_growth``), so a client whose map grows does not pay for fresh driver
        allocations (tens of ms per GB) inside its request; released by ``close``.
        `approach`: "tree" (``TreeDeduplicator`` per client) or "list" (``ListDeduplicator``)."""
        import torch

        self.budget = int(hbm_budget)
        self.cs, self.kind = int(chunk_size), int(hash_kind)
        self.max_batch, self.plain, self.evict, self.checksum = int(max_batch), plain, evict, checksum
        self.clock = clock
        if approach not in ("tree", "list"):
            raise ValueError(f"approach must be 'tree' or 'list', not {approach!r}")
        self.Dedup = ListDeduplicator if approach == "list" else TreeDeduplicator
        self.clients = collections.defaultdict(_Client)
        self.waiting = collections.deque()       # arrived, not admitted (arrival order)
        self.resident = 0                        # bytes reserved by resident clients
        self.peak_resident = 0
        self.completed = []
        self.copying = []                        # (event, requests) whose diffs are being copied back
        self.to_host = False
        self.batches = 0
        self.seq = 0
        params = {"graph_cache": 256}
        params.update(batch_params)
        self.map_reserve = 0
        if map_reserve:
            self.reserve_growth(map_reserve)
        self.slots = [] if plain else [
            (CheckpointBatch(**params), torch.cuda.Stream(), []) for _ in range(max(1, int(max_inflight)))]

    # -- client side
    def submit(self, client, buffer, make_baseline=False, arrival=None):
        """Queue one checkpoint of `buffer` (a CUDA tensor the client will not touch until the
        request completes) for `client`.  Work queued on the current stream before this call is
        ordered before the checkpoint."""
        import torch

        r = Request(client, buffer, bool(make_baseline), self.clock() if arrival is None else arrival, self.seq)
        if r.nbytes == 0:
            raise ValueError("an empty buffer cannot be checkpointed")
        self.seq += 1
        r.ready = torch.cuda.Event()
        r.ready.record(torch.cuda.current_stream())
        self.waiting.append(r)
        self.clients[client].outstanding += 1
        return r

    def reserve_growth(self, nbytes):
        """Map `nbytes` of unused device memory for digest maps now.  New clients' baseline maps
        are carved from it too, so a server calls this once its clients are resident (after their
        first requests) to keep the memory for later map growth."""
        reserve_map_memory(int(nbytes))
        self.map_reserve = int(nbytes)

    def busy(self, client):
        """True while a request of `client` is not completed (its buffer must stay unchanged)."""
        c = self.clients.get(client)
        return bool(c and c.outstanding)

    def idle(self):
        return (not self.waiting and not any(c.pending for c in self.clients.values())
                and not any(reqs for _, _, reqs in self.slots) and not self.copying)

    def close(self):
        for b, _, reqs in self.slots:
            if reqs:
                b.wait(check_status=False)
            b.close()
        for c in self.clients.values():
            if c.handle is not None:
                c.handle.close()
                c.handle = None
        self.clients.clear()
        if self.map_reserve:
            reserve_map_memory(0)
            self.map_reserve = 0

    # -- loop
    def step(self):
        """One pass of the loop: complete finished batches, admit, launch.  Returns requests completed."""
        if self.plain:
            return self._step_plain()
        done = self._complete()
        self._admit()
        self._launch()
        return done

    def drain(self, poll=0.0):
        while not self.idle():
            self.step()
            if poll:
                time.sleep(poll)

    # -- internals
    def _need(self, c, r):
        if c.handle is not None:
            return 0
        return estimate_memory(r.nbytes, self.cs)

    def _evict_for(self, need):
        idle = [(c.last_use, cid) for cid, c in self.clients.items()
                if c.handle is not None and not c.busy and not c.pending]
        idle.sort()
        for _, cid in idle:
            if self.resident + need <= self.budget:
                break
            c = self.clients[cid]
            c.handle.close()
            c.handle = None
            c.nbytes = None
            self.resident -= c.reserved
            c.reserved = 0

    def _admit(self):
        keep = collections.deque()
        blocked = set()
        while self.waiting:
            r = self.waiting.popleft()
            c = self.clients[r.client]
            if r.client in blocked:
                keep.append(r)
                continue
            need = self._need(c, r)
            if need and self.resident + need > self.budget and self.evict:
                self._evict_for(need)
            if need and self.resident + need > self.budget:
                keep.append(r)          # waits for memory; later requests of this client wait behind it
                blocked.add(r.client)
                continue
            if c.handle is None:
                c.handle = self.Dedup(self.cs, self.kind)
                c.rebase = True         # a handle's first checkpoint is its baseline
                c.taken = 0
                c.reserved = need
                self.resident += need
                self.peak_resident = max(self.peak_resident, self.resident)
            r.admitted = self.clock()
            c.pending.append(r)
        self.waiting = keep

    def _launch(self):
        for slot in self.slots:
            b, stream, reqs = slot
            if reqs:
                continue
            heads = sorted((c.pending[0].seq, cid) for cid, c in self.clients.items() if c.pending and not c.busy)
            if not heads:
                return
            batch = [self.clients[cid].pending.popleft() for _, cid in heads[:self.max_batch]]
            for r in batch:
                stream.wait_event(r.ready)
                self._take(self.clients[r.client], r)
            now = self.clock()
            for r in batch:
                r.launched = now
            try:
                b.launch([self.clients[r.client].handle for r in batch], [r.buffer for r in batch],
                         [r.baseline for r in batch], stream=stream)
            except Exception as e:   # noqa: BLE001 - the status travels with the requests
                # nothing of the batch runs: its requests complete now with the error, and
                # their clients' next requests are baselines.  Handles prepared before the
                # failure may have queued work on this slot's stream; it completes before their
                # clients become idle (their next batch may run on another slot's stream).
                stream.synchronize()
                done = self.clock()
                for r in batch:
                    r.done = done
                    self._finish(r, getattr(e, "code", -8))
                self.batches += 1
                continue
            host = self.clock() - now
            for r in batch:
                r.launch_s = host
                r.batch_size = len(batch)
            reqs.extend(batch)
            self.batches += 1

    def _take(self, c, r):
        """`r` is about to run on its client's handle: decide whether it runs as a baseline"""
        if c.taken >= MAX_CHECKPOINTS_PER_HANDLE:
            c.handle.close()
            c.handle = self.Dedup(self.cs, self.kind)
            c.taken, c.rebase = 0, True
        r.baseline = r.make_baseline or c.rebase or (c.nbytes is not None and c.nbytes != r.nbytes)
        c.nbytes, c.rebase, c.busy = r.nbytes, False, True
        c.taken += 1

    def _finish(self, r, rc):
        c = self.clients[r.client]
        r.rc = rc
        if rc != 0:
            c.rebase = True
        if rc == 0:
            r.diff_len = c.handle.diff_device()[1]
            r.chkpt_id = c.handle.current_id - 1
            if self.checksum:
                r.checksum = c.handle.diff_checksum()
            used = c.handle.memory()
            if used > c.reserved:              # maps grow: keep the reservation honest
                self.resident += used - c.reserved
                c.reserved = used
                self.peak_resident = max(self.peak_resident, self.resident)
        c.busy = False
        c.outstanding -= 1
        c.last_use = r.done
        r.buffer = None
        self.completed.append(r)

    def _host_buffer(self, c, n):
        import torch

        if c.host is None or c.host.numel() < n:
            c.host = torch.empty(int(n * 1.25) + 4096, dtype=torch.uint8, pin_memory=True)
        return c.host

    def enable_host_copy(self, sizes=None, fraction=0.25):
        """From now on a request completes when its diff is in pinned host memory (``Request.host``,
        a view of the client's buffer, valid until its next request completes).  `sizes`
        (client -> buffer bytes) pre-allocates each client's pinned buffer at `fraction` of it."""
        self.to_host = True
        for cid, nbytes in (sizes or {}).items():
            self._host_buffer(self.clients[cid], int(nbytes * fraction))

    def _complete(self):
        import torch

        out = []
        for b, stream, reqs in self.slots:
            if not reqs or not b.done():
                continue
            rcs = b.wait(check_status=False)
            now = self.clock()
            if self.to_host:
                # copy the diffs back on the slot's stream; the requests complete when that lands
                for r, rc in zip(reqs, rcs):
                    r.rc = rc
                    if rc == 0:
                        h = self.clients[r.client].handle
                        buf = self._host_buffer(self.clients[r.client], h.diff_device()[1])
                        r.host = buf[:h.copy_diff_async(buf, stream)]
                ev = torch.cuda.Event()
                ev.record(stream)
                self.copying.append((ev, list(reqs)))
            else:
                for r, rc in zip(reqs, rcs):
                    r.done = now
                    self._finish(r, rc)
                    out.append(r)
            reqs.clear()
        keep = []
        for ev, reqs in self.copying:
            if ev.query():
                now = self.clock()
                for r in reqs:
                    r.done = now
                    self._finish(r, r.rc)
                    out.append(r)
            else:
                keep.append((ev, reqs))
        self.copying = keep
        return out

    def _step_plain(self):
        self._admit()
        nxt = None
        for c in self.clients.values():
            if c.pending and (nxt is None or c.pending[0].seq < nxt.seq):
                nxt = c.pending[0]
        if nxt is None:
            return []
        c = self.clients[nxt.client]
        c.pending.popleft()
        nxt.launched = self.clock()
        nxt.ready.synchronize()
        self._take(c, nxt)
        rc = 0
        try:
            c.handle.checkpoint_device(nxt.buffer, nxt.baseline)
        except Exception as e:   # noqa: BLE001 - the status travels with the request
            rc = getattr(e, "code", -8)
        if rc == 0 and self.to_host:
            buf = self._host_buffer(c, c.handle.diff_device()[1])
            nxt.host = buf[:len(c.handle.copy_diff(buf.numpy()))]
        nxt.done = self.clock()
        self._finish(nxt, rc)
        self.batches += 1
        return [nxt]


def percentile(values, q):
    """q-th percentile (0..100) by linear interpolation between order statistics."""
    v = sorted(values)
    if not v:
        return None
    k = (len(v) - 1) * q / 100.0
    lo = int(k)
    hi = min(lo + 1, len(v) - 1)
    return v[lo] + (v[hi] - v[lo]) * (k - lo)
