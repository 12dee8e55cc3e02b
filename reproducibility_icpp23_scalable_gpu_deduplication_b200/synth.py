"""Seeded synthetic checkpoint series with the shapes of the reference's workloads.

The reference measures on HiPC graph-application checkpoints that are not available here;
these generators stand in for them with the buffer sizes, chunk sizes and change patterns of
the five benchmark configurations:

  plain_64m   : 64 MiB uint8, chunk 128 B, 5 checkpoints; rewrite 5% of chunks in runs of
                1-64 (uniform starts), copy 2% single chunks from other offsets, zero 1%
  plain_4g    : 4 GiB uint8, chunk {64..4096} B, 20 checkpoints; change 1% of chunks in runs
                Geometric(1/32) capped at 1024, plus 0.5% shifted single-chunk copies
  md5_f32_8g  : 8 GiB float32 N(0, 0.02), chunk 256 B, MD5, 10 checkpoints; N(0, 1e-4) noise on
                30% of the 64 KiB blocks, a fixed 10% of 4 KiB pages zero, 5% of the buffer
                copies of one 1 MiB block at 256 B-aligned offsets
  batched     : 256 buffers log-uniform in [1 MiB, 512 MiB] (multiple of 128 B), chunk 128 B,
                10 checkpoints; change U[0.5%, 20%] in runs U[1,256] + 1% shifted copies
  served      : 64 clients log-uniform in [4 MiB, 2 GiB], chunk 128 B, Poisson arrivals at
                200 req/s; change U[0.5%, 20%] in runs U[1,512] + 1% shifted copies

Random bytes are counter-based (splitmix64 finaliser over (seed, stream, word index)), so the
numpy (host) and torch (device) generators produce identical bytes; edit plans come from
numpy's PCG64 seeded by (seed, config, buffer, checkpoint).  Copy sources are read before the
checkpoint's own edits are applied.  Float data (md5_f32_8g) uses numpy's normal generator on
the host and torch.randn on the device: same distribution, not the same bytes.
"""
import math

import numpy as np

SEED = 1931   # src/data_generation.cpp:142-143 of the reference

GOLDEN = 0x9E3779B97F4A7C15
M1 = 0xBF58476D1CE4E5B9
M2 = 0x94D049BB133111EB
C_STREAM = 0x632BE59BD9B4E019
MASK64 = (1 << 64) - 1


# ----------------------------------------------------------------------------- counter PRNG
def _mix64_np(z):
    z = (z ^ (z >> np.uint64(30))) * np.uint64(M1)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(M2)
    return z ^ (z >> np.uint64(31))


def stream_keys_np(seed, streams):
    s = np.asarray(streams, dtype=np.uint64)
    with np.errstate(over="ignore"):
        return _mix64_np(np.uint64(seed) ^ _mix64_np(s + np.uint64(C_STREAM)))


def words_np(seed, streams, nwords):
    """uint64 [len(streams), nwords]: word j of stream i."""
    keys = stream_keys_np(seed, streams)
    j = np.arange(1, nwords + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        return _mix64_np(keys[:, None] + j[None, :] * np.uint64(GOLDEN))


def _s64(c):
    return c - (1 << 64) if c >= (1 << 63) else c


def _lsr(z, k):
    return (z >> k) & ((1 << (64 - k)) - 1)


def _mix64_t(z):
    z = (z ^ _lsr(z, 30)) * _s64(M1)
    z = (z ^ _lsr(z, 27)) * _s64(M2)
    return z ^ _lsr(z, 31)


def words_torch(seed, streams, nwords, device):
    """Same words as words_np, computed on the device with int64 wrap-around arithmetic."""
    import torch

    s = torch.as_tensor(np.asarray(streams, dtype=np.uint64).view(np.int64), device=device)
    keys = _mix64_t(_s64(seed) ^ _mix64_t(s + _s64(C_STREAM)))
    j = torch.arange(1, nwords + 1, dtype=torch.int64, device=device)
    return _mix64_t(keys[:, None] + j[None, :] * _s64(GOLDEN))


def words_torch_t(seed, streams, nwords):
    """words_torch for streams already in a device int64 tensor (bit patterns of the uint64 ids)."""
    import torch

    keys = _mix64_t(_s64(seed) ^ _mix64_t(streams + _s64(C_STREAM)))
    j = torch.arange(1, nwords + 1, dtype=torch.int64, device=streams.device)
    return _mix64_t(keys[:, None] + j[None, :] * _s64(GOLDEN))


def chunk_bytes_np(seed, streams, cs):
    w = words_np(seed, streams, (cs + 7) // 8)
    return w.view(np.uint8).reshape(len(streams), -1)[:, :cs]


def chunk_bytes_torch(seed, streams, cs, device):
    import torch

    w = words_torch(seed, streams, (cs + 7) // 8, device)
    return w.view(torch.uint8).reshape(len(streams), -1)[:, :cs]


def _stream_id(tag, ckpt, index):
    return (np.uint64(tag) << np.uint64(56)) | (np.uint64(ckpt) << np.uint64(40)) | np.asarray(index, np.uint64)


# ----------------------------------------------------------------------------- edit plans
def plan_rng(seed, config, buf, ckpt):
    return np.random.Generator(np.random.PCG64(np.random.SeedSequence([seed, config, buf, ckpt])))


def _unique_last(dst, src):
    """keep the last write to each destination (sequential-assignment semantics)"""
    if dst.size == 0:
        return dst, src
    rev_d = dst[::-1]
    u, first_in_rev = np.unique(rev_d, return_index=True)
    return u, src[::-1][first_in_rev]


def runs_to_chunks(starts, lens):
    if len(starts) == 0:
        return np.zeros(0, np.int64)
    idx = np.repeat(np.asarray(starts, np.int64), lens) + (np.arange(int(np.sum(lens))) -
                                                           np.repeat(np.cumsum(lens) - lens, lens))
    return np.unique(idx)


def sample_runs(rng, n, quota, draw_len):
    starts, lens, total = [], [], 0
    while total < quota:
        L = int(min(draw_len(), quota - total, n))
        s = int(rng.integers(0, n - L + 1))
        starts.append(s)
        lens.append(L)
        total += L
    return np.asarray(starts, np.int64), np.asarray(lens, np.int64)


def shifted_copies(rng, n, count):
    if count <= 0 or n < 2:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    dst = rng.integers(0, n, count, dtype=np.int64)
    src = rng.integers(0, n - 1, count, dtype=np.int64)
    src = src + (src >= dst)
    return _unique_last(dst, src)


def plan_plain_64m(rng, n):
    rew_s, rew_l = sample_runs(rng, n, round(0.05 * n), lambda: rng.integers(1, 65))
    cdst, csrc = shifted_copies(rng, n, round(0.02 * n))
    zero = np.unique(rng.integers(0, n, round(0.01 * n), dtype=np.int64))
    return {"rewrite": runs_to_chunks(rew_s, rew_l), "copy_dst": cdst, "copy_src": csrc, "zero": zero}


def plan_plain_4g(rng, n):
    rew_s, rew_l = sample_runs(rng, n, round(0.01 * n), lambda: min(int(rng.geometric(1.0 / 32)), 1024))
    cdst, csrc = shifted_copies(rng, n, round(0.005 * n))
    return {"rewrite": runs_to_chunks(rew_s, rew_l), "copy_dst": cdst, "copy_src": csrc,
            "zero": np.zeros(0, np.int64)}


def plan_varied(rng, n, max_run):
    rate = rng.uniform(0.005, 0.20)
    rew_s, rew_l = sample_runs(rng, n, max(1, round(rate * n)), lambda: rng.integers(1, max_run + 1))
    cdst, csrc = shifted_copies(rng, n, round(0.01 * n))
    return {"rewrite": runs_to_chunks(rew_s, rew_l), "copy_dst": cdst, "copy_src": csrc,
            "zero": np.zeros(0, np.int64)}


# ----------------------------------------------------------------------------- byte series
class ByteSeries:
    """A uint8 buffer evolving through seeded checkpoints, on the host (numpy) or device (torch).

    ckpt 0 is uniform random bytes; each later checkpoint applies `plan(rng, n)`:
    shifted copies (sources read before the edits), fresh random runs, zero chunks.
    """

    def __init__(self, nbytes, chunk_size, plan, config_id, buf_id=0, seed=SEED, device=None):
        self.nbytes = int(nbytes)
        self.cs = int(chunk_size)
        self.n = (self.nbytes + self.cs - 1) // self.cs
        self.plan = plan
        self.config_id = config_id
        self.buf_id = buf_id
        self.seed = seed
        self.device = device
        self.ckpt = -1
        self.data = None
        self.last_plan = None

    def _fill_random(self):
        total_words = (self.nbytes + 7) // 8
        step = 1 << 24   # words per generation block
        nblk = (total_words + step - 1) // step
        if self.device is None:
            out = np.empty(nblk * step * 8, np.uint8)
            for b in range(nblk):
                w = words_np(self.seed, [int(_stream_id(1, 0, self.buf_id * 4096 + b))], step)[0]
                out[b * step * 8:(b + 1) * step * 8] = w.view(np.uint8)
            self.data = out[:self.nbytes].copy()
        else:
            import torch

            self.data = torch.empty(self.nbytes, dtype=torch.uint8, device=self.device)
            for b in range(nblk):
                w = words_torch(self.seed, [int(_stream_id(1, 0, self.buf_id * 4096 + b))], step, self.device)[0]
                lo = b * step * 8
                hi = min(self.nbytes, lo + step * 8)
                self.data[lo:hi] = w.view(torch.uint8)[:hi - lo]

    def _full_chunk_view(self):
        nfull = self.nbytes // self.cs
        return self.data[:nfull * self.cs].reshape(nfull, self.cs), nfull

    def next(self):
        """Advance to the next checkpoint; returns the buffer (numpy array or CUDA tensor)."""
        self.ckpt += 1
        if self.ckpt == 0:
            self._fill_random()
            return self.data
        rng = plan_rng(self.seed, self.config_id, self.buf_id, self.ckpt)
        p = self.plan(rng, self.n)
        nfull = self.nbytes // self.cs
        # only whole chunks are edited; the short tail chunk (if any) never changes
        keep = lambda a: a[a < nfull] if a.size else a  # noqa: E731
        cm = (p["copy_dst"] < nfull) & (p["copy_src"] < nfull)
        p = {"rewrite": keep(p["rewrite"]), "copy_dst": p["copy_dst"][cm], "copy_src": p["copy_src"][cm],
             "zero": keep(p["zero"])}
        self.last_plan = p
        view, _ = self._full_chunk_view()
        # fresh content of a rewritten chunk depends on (seed, buffer, checkpoint, chunk index)
        streams = _stream_id(2, self.ckpt, p["rewrite"]) if p["rewrite"].size else None
        if self.device is None:
            src_rows = view[p["copy_src"]].copy()
            if streams is not None:
                view[p["rewrite"]] = chunk_bytes_np(self.seed + self.buf_id, streams, self.cs)
            view[p["copy_dst"]] = src_rows
            view[p["zero"]] = 0
        else:
            import torch

            dev = self.device
            src_rows = view[torch.as_tensor(p["copy_src"], device=dev)].clone()
            if streams is not None:
                view[torch.as_tensor(p["rewrite"], device=dev)] = chunk_bytes_torch(self.seed + self.buf_id, streams,
                                                                                     self.cs, dev)
            view[torch.as_tensor(p["copy_dst"], device=dev)] = src_rows
            if p["zero"].size:
                view[torch.as_tensor(p["zero"], device=dev)] = 0
        return self.data


def plain_64m(nbytes=64 << 20, chunk_size=128, device=None, seed=SEED):
    return ByteSeries(nbytes, chunk_size, plan_plain_64m, 1, 0, seed, device)


def plain_4g(nbytes=4 << 30, chunk_size=128, device=None, seed=SEED):
    return ByteSeries(nbytes, chunk_size, plan_plain_4g, 2, 0, seed, device)


def varied(nbytes, chunk_size=128, max_run=256, config_id=4, buf_id=0, device=None, seed=SEED):
    return ByteSeries(nbytes, chunk_size, lambda r, n: plan_varied(r, n, max_run), config_id, buf_id, seed, device)


def batched_sizes(count=256, lo=1 << 20, hi=512 << 20, align=128, seed=SEED, config_id=4):
    rng = plan_rng(seed, config_id, 999999, 0)
    s = np.exp(rng.uniform(math.log(lo), math.log(hi), count))
    return [max(align, int(x) // align * align) for x in s]


def served_sizes(count=64, lo=4 << 20, hi=2 << 30, align=128, seed=SEED):
    return batched_sizes(count, lo, hi, align, seed, config_id=5)


def poisson_arrivals(rate_hz, count, seed=SEED):
    rng = plan_rng(seed, 5, 888888, 0)
    return np.cumsum(rng.exponential(1.0 / rate_hz, count))


class DeviceSeries:
    """A device buffer whose checkpoints are edited on the device: only a handful of scalars and run
    bounds are drawn on the host, so a request loop can advance many clients in real time.

    ckpt 0 is uniform random bytes; each later checkpoint rewrites a fraction of the whole chunks,
    drawn uniform in `rate`, as runs of 1..`max_run` chunks with fresh bytes, and copies `shift`
    of the chunks verbatim from other offsets (sources read before the edits).  Deterministic in
    (seed, client, checkpoint).
    """

    def __init__(self, nbytes, chunk_size, client, seed=SEED, device="cuda", max_run=512, rate=(0.005, 0.20),
                 shift=0.01):
        self.nbytes, self.cs, self.client, self.seed = int(nbytes), int(chunk_size), int(client), seed
        self.device, self.max_run, self.rate, self.shift = device, int(max_run), rate, shift
        self.nfull = self.nbytes // self.cs
        self.ckpt = -1
        self.data = None

    def next(self):
        import torch

        self.ckpt += 1
        dev = self.device
        if self.ckpt == 0:
            self.data = torch.empty(self.nbytes, dtype=torch.uint8, device=dev)
            step = 1 << 24
            total_words = (self.nbytes + 7) // 8
            for b in range((total_words + step - 1) // step):
                w = words_torch(self.seed, [int(_stream_id(3, 0, self.client * 4096 + b))], step, dev)[0]
                lo = b * step * 8
                hi = min(self.nbytes, lo + step * 8)
                self.data[lo:hi] = w.view(torch.uint8)[:hi - lo]
            return self.data
        n = self.nfull
        if n == 0:
            return self.data
        view = self.data[:n * self.cs].view(n, self.cs)
        rng = plan_rng(self.seed, 6, self.client, self.ckpt)
        rate = rng.uniform(*self.rate)
        nruns = max(1, round(rate * n / ((1 + self.max_run) / 2)))
        lens = rng.integers(1, self.max_run + 1, nruns)
        starts = rng.integers(0, n, nruns)
        total = int(lens.sum())
        L = torch.as_tensor(lens, device=dev)
        S = torch.as_tensor(starts, device=dev)
        idx = torch.repeat_interleave(S, L, output_size=total)
        idx += torch.arange(total, device=dev) - torch.repeat_interleave(torch.cumsum(L, 0) - L, L, output_size=total)
        idx.clamp_(max=n - 1)   # a run past the end rewrites the last chunk (same bytes every time)
        m = round(self.shift * n) if n > 1 else 0
        if m:
            g = torch.Generator(device=dev)
            g.manual_seed(int(rng.integers(1 << 62)))
            dst = torch.randperm(n, generator=g, device=dev)[:m]
            src = torch.randint(0, n - 1, (m,), generator=g, device=dev)
            src += (src >= dst).to(src.dtype)
            rows = view[src].clone()
        # fresh bytes in slices, so the temporaries stay small and are reused from the allocator
        tag = (2 << 56) | (self.ckpt << 40)
        step = 1 << 16
        for lo in range(0, total, step):
            part = idx[lo:lo + step]
            w = words_torch_t(self.seed + self.client, part | tag, (self.cs + 7) // 8)
            view[part] = w.view(torch.uint8).reshape(part.numel(), -1)[:, :self.cs]
        if m:
            view[dst] = rows
        return self.data


def duplicate_heavy(n_chunks, chunk_size, checkpoints, seed=SEED):
    """Buffers with few distinct chunk values (equal chunks and equal subtrees at many depths,
    all-zero pages): every chunk of checkpoint k holds one of four byte patterns, drawn per
    chunk from numpy's PCG64 seeded by (seed, checkpoint)."""
    bufs = []
    for k in range(checkpoints):
        rng = plan_rng(seed, 7, n_chunks, k)
        pat = rng.integers(0, 4, n_chunks)
        b = np.zeros((n_chunks, chunk_size), np.uint8)
        for v in range(1, 4):
            b[pat == v] = v + (k % 3)
        bufs.append(b.reshape(-1))
    return bufs


# ----------------------------------------------------------------------------- float32 / MD5
class FloatSeries:
    """Training-state-like float32 buffer (md5_f32_8g)."""

    BLOCK = 64 << 10
    PAGE = 4 << 10
    REPEAT = 1 << 20

    def __init__(self, nbytes=8 << 30, device=None, seed=SEED):
        assert nbytes % self.BLOCK == 0
        self.nbytes = int(nbytes)
        self.device = device
        self.seed = seed
        self.ckpt = -1
        self.data = None
        rng = plan_rng(seed, 3, 0, 0)
        npages = self.nbytes // self.PAGE
        self.zero_pages = np.sort(rng.choice(npages, size=npages // 10, replace=False))

    def next(self):
        self.ckpt += 1
        rng = plan_rng(self.seed, 3, 1, self.ckpt)
        nvals = self.nbytes // 4
        nblocks = self.nbytes // self.BLOCK
        vals_per_block = self.BLOCK // 4
        if self.device is None:
            if self.ckpt == 0:
                self.data = rng.normal(0.0, 0.02, nvals).astype(np.float32)
            else:
                blocks = rng.choice(nblocks, size=int(0.3 * nblocks), replace=False)
                v = self.data.reshape(nblocks, vals_per_block)
                v[blocks] += rng.normal(0.0, 1e-4, (blocks.size, vals_per_block)).astype(np.float32)
            b = self.data.view(np.uint8)
        else:
            import torch

            g = torch.Generator(device=self.device)
            g.manual_seed(int(rng.integers(0, 2**62)))
            if self.ckpt == 0:
                self.data = torch.empty(nvals, dtype=torch.float32, device=self.device)
                step = 1 << 28
                for lo in range(0, nvals, step):
                    hi = min(nvals, lo + step)
                    self.data[lo:hi] = torch.randn(hi - lo, generator=g, device=self.device) * 0.02
            else:
                blocks = rng.choice(nblocks, size=int(0.3 * nblocks), replace=False)
                v = self.data.view(nblocks, vals_per_block)
                bt = torch.as_tensor(blocks, device=self.device)
                for lo in range(0, bt.numel(), 16384):
                    sel = bt[lo:lo + 16384]
                    v[sel] += torch.randn((sel.numel(), vals_per_block), generator=g, device=self.device) * 1e-4
            b = self.data.view(torch.uint8)
        # 5% of the buffer: copies of one 1 MiB block at 256 B-aligned offsets
        ncopies = int(0.05 * self.nbytes) // self.REPEAT
        src = int(rng.integers(0, (self.nbytes - self.REPEAT) // 256)) * 256
        dsts = rng.integers(0, (self.nbytes - self.REPEAT) // 256, ncopies) * 256
        block = b[src:src + self.REPEAT].clone() if self.device is not None else b[src:src + self.REPEAT].copy()
        for d in dsts:
            b[int(d):int(d) + self.REPEAT] = block
        # fixed 10% of 4 KiB pages are zero at every checkpoint
        pv = b.reshape(-1, self.PAGE)
        if self.device is None:
            pv[self.zero_pages] = 0
        else:
            import torch

            pv[torch.as_tensor(self.zero_pages, device=self.device)] = 0
        return b
