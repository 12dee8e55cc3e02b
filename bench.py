#!/usr/bin/env python
"""Tree-dedup ingest throughput: one incremental checkpoint of the 4 GiB plain workload per step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--chunk-size CS] [--impl reference]

Workload (the GPU configuration the metric is quoted on): a 4 GiB uint8 buffer, chunk 128 B,
a 20-checkpoint series: checkpoint 0 uniform random (the baseline), each later checkpoint
changes 1% of the chunks in Geometric(1/32) runs capped at 1024 plus 0.5% shifted single-chunk
copies (seeded synthetic data; the reference's HiPC datasets are not available).  A step is
one incremental checkpoint: hash + label + Merkle forest + map + diff assembly, inputs resident
in HBM (each step's buffer is materialised before the timed region; 4 GiB > L2, so no flush).

`value`    : ingested GB/s (all ranks' bytes / max over ranks of the device time of K steps)
`e2e`      : the same metric through the public API with host buffers: pinned host -> device
             copy of the step's buffer, checkpoint, diff copied back to pinned host memory
`roofline` : the dominant kernel (chunk hashing + labelling) against measured HBM bandwidth
`cpu_baseline` / --impl reference: the CPU restatement of the reference algorithm (oracle/),
             OpenMP-parallel hashing with all host threads, on the workload's full buffer: an
             untimed baseline and warm-up checkpoints, then timed incremental checkpoints

Multi-GPU (torchrun): every rank deduplicates its own buffer (independent replicas, like the
reference's MPI driver); nothing crosses ranks but the barrier and the max-time reduction.
"""
import argparse
import collections
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

GB = 1e9


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=16)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--workload", default="plain_4g", choices=["plain_4g", "md5_f32_8g", "plain_64m"],
                   help="plain form: the 4 GiB Murmur3 series (default), the 8 GiB float32 MD5 series, or "
                        "the 64 MiB CPU-runnable series (5%% rewritten, 2%% shifted, 1%% zeroed per checkpoint)")
    p.add_argument("--chunk-size", type=int, default=None, help="default 128 (plain_4g) / 256 (md5_f32_8g)")
    p.add_argument("--approach", default="tree", choices=["tree", "list"],
                   help="the tree approach (default) or the list approach (ListDeduplicator), in every "
                        "form and in the reference arm")
    p.add_argument("--nbytes", type=int, default=None, help="default 4 GiB (plain_4g) / 8 GiB (md5_f32_8g)")
    p.add_argument("--e2e-steps", type=int, default=2)
    p.add_argument("--cpu-sample-bytes", type=int, default=0,
                   help="CPU baseline buffer size (0 = the workload's full size)")
    p.add_argument("--cpu-steps", type=int, default=3,
                   help="timed incremental checkpoints of the cpu_baseline leg (after a baseline and one warm-up)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--leaf-stages", type=int, default=0, help="TMA ring depth (0 = library default)")
    p.add_argument("--leaf-ctas", type=int, default=0, help="hashing CTAs per SM (0 = library default)")
    p.add_argument("--leaf-unit", type=int, default=0, help="staged segment width (0 = library default)")
    p.add_argument("--form", default="plain", choices=["plain", "batched", "served"],
                   help="plain: one 4 GiB buffer (default); batched: 256 uneven buffers per step through "
                        "b2d_batch_checkpoint vs one at a time; served: Poisson request loop")
    p.add_argument("--buffers", type=int, default=256, help="batched form: number of buffers")
    p.add_argument("--max-buffer", type=int, default=512 << 20, help="batched form: largest buffer size")
    p.add_argument("--no-autotune", action="store_true")
    p.add_argument("--tune-batches", type=int, default=12, help="batched form: most autotuning batches")
    p.add_argument("--capacity-waves", type=int, default=4, help="served form: waves of the capacity run")
    p.add_argument("--no-forms", action="store_true",
                   help="plain form: skip the bounded batched and served legs the default line carries")
    p.add_argument("--forms-steps", type=int, default=4,
                   help="plain form: timed batches of the bounded batched leg (after 2 warm-up batches)")
    p.add_argument("--forms-requests", type=int, default=400,
                   help="plain form: requests of the bounded served leg (Poisson, --rate per second)")
    p.add_argument("--no-restart", action="store_true", help="plain form: skip the restart measurement")
    p.add_argument("--no-plain", action="store_true", help="batched form: skip the one-at-a-time pass")
    p.add_argument("--graph", type=int, default=None, choices=[0, 1, 2],
                   help="plain form: 0 launch kernels one by one, 1 replay a CUDA graph, 2 graph without "
                        "phase-timing events (default: the library's)")
    p.add_argument("--clients", type=int, default=64, help="served form: clients")
    p.add_argument("--requests", type=int, default=1000, help="served form: requests in the stream")
    p.add_argument("--rate", type=float, default=200.0, help="served form: aggregate arrivals per second")
    p.add_argument("--client-max-buffer", type=int, default=2 << 30, help="served form: largest client buffer")
    p.add_argument("--map-reserve", type=float, default=20e9,
                   help="device bytes kept mapped for digest-map growth after the warm-up (all forms)")
    p.add_argument("--hbm-budget", type=float, default=150e9, help="served form: device bytes for client state")
    p.add_argument("--map-headroom", type=int, default=None,
                   help="plain form: digest-map size at the baseline over its minimum, percent (default: 400 for "
                        "md5_f32_8g, whose series adds about 0.3 N entries per checkpoint, so the baseline's table "
                        "holds all 20 checkpoints; the library default 150 otherwise)")
    a = p.parse_args()
    md5 = a.workload == "md5_f32_8g"
    if a.map_headroom is None:
        a.map_headroom = 400 if md5 else 0
    if a.chunk_size is None:
        a.chunk_size = 256 if md5 else 128
    if a.nbytes is None:
        a.nbytes = (8 << 30) if md5 else ((64 << 20) if a.workload == "plain_64m" else (4 << 30))
    return a


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """Polls SM clock and clock-event reasons through NVML while the timed region runs."""

    REASONS = {
        0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
        0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown",
        0x100: "display_clock_setting",
    }

    def __init__(self, index):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        try:
            import pynvml

            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                r = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for bit, name in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.0005)

    def __enter__(self):
        if self.nv:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        if self.nv:
            self._stop.set()
            self.t.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons - {"gpu_idle"}), "samples": len(self.samples)}


def workload_series(workload, nbytes, cs, device, seed):
    from reproducibility_icpp23_scalable_gpu_deduplication_b200 import synth

    if workload == "md5_f32_8g":
        return synth.FloatSeries(nbytes=nbytes, device=device, seed=seed)
    if workload == "plain_64m":
        return synth.plain_64m(nbytes=nbytes, chunk_size=cs, device=device, seed=seed)
    return synth.plain_4g(nbytes=nbytes, chunk_size=cs, device=device, seed=seed)


def cpu_baseline_run(nbytes, cs, steps, threads, workload="plain_4g", approach="tree", warmup=1, device=None):
    """The oracle (sequential restatement of the reference) on the host, all threads hashing.

    One definition for every CPU figure: an untimed baseline, `warmup` untimed incremental
    checkpoints, then `steps` timed incremental checkpoints of the same series; returns (ingest
    GB/s over the timed checkpoints, their seconds).  With `device` the series' bytes are generated
    there and copied to host memory before each checkpoint (same bytes for the byte workloads,
    faster than generating 4 GiB with numpy); only the oracle's checkpoint calls are timed."""
    from oracle import oracle as O
    from reproducibility_icpp23_scalable_gpu_deduplication_b200 import synth

    s = workload_series(workload, nbytes, cs, device, synth.SEED)

    def host_next():
        b = s.next()
        return b if device is None else b.view(-1).cpu().numpy()

    cls = O.OracleListDeduplicator if approach == "list" else O.OracleTreeDeduplicator
    o = cls(cs, O.HASH_MD5 if workload == "md5_f32_8g" else O.HASH_MURMUR3, threads=threads)
    o.checkpoint(host_next(), True)
    for _ in range(max(0, warmup)):
        o.checkpoint(host_next(), False)
    t = 0.0
    for _ in range(steps):
        b = host_next()
        t0 = time.perf_counter()
        o.checkpoint(b, False)
        t += time.perf_counter() - t0
    o.close()
    return steps * nbytes / t / GB, t


def cpu_sample_text(nbytes, workload, cs, warmup, steps):
    return (f"{nbytes / 2**30:g} GiB buffer of the {workload} series, chunk {cs} B: an untimed baseline and "
            f"{warmup} untimed incremental checkpoint(s), then the mean of {steps} timed incremental checkpoints")


def leaf_traffic(cs):
    """DRAM bytes per leaf launch from the committed ncu summary, scaled to this workload."""
    path = os.path.join(ROOT, "profiles", "leaf_traffic.json")
    try:
        with open(path) as f:
            t = json.load(f)
        e = t.get(str(cs))
        return e["bytes_per_input_byte"] if e else None
    except Exception:
        return None


def run_reference(args, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    steps = max(1, args.steps)
    warm = max(1, args.warmup)
    nbytes = args.cpu_sample_bytes or args.nbytes
    gbps, t = cpu_baseline_run(nbytes, args.chunk_size, steps, threads, args.workload, args.approach, warmup=warm)
    line = {
        "impl": "reference", "metric": f"{args.approach}-dedup ingest GB/s", "value": round(gbps, 4), "unit": "GB/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": warm, "ms_per_step": round(1e3 * t / steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": args.workload, "nbytes": nbytes, "chunk_size": args.chunk_size,
                   "hash": "md5" if args.workload == "md5_f32_8g" else "murmur3", "approach": args.approach},
        "cpu_baseline": {"value": round(gbps, 4), "unit": "GB/s", "cores": threads, "kind": "port",
                         "sample": cpu_sample_text(nbytes, args.workload, args.chunk_size, warm, steps)},
        "e2e": {"value": round(gbps, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def batched_series(sizes, dev, seed):
    from reproducibility_icpp23_scalable_gpu_deduplication_b200 import synth

    return [synth.varied(n, 128, max_run=256, config_id=4, buf_id=i, device=dev, seed=seed)
            for i, n in enumerate(sizes)]


def run_batched(args, rank, world, dev, emit=True):
    """256 buffers of log-uniform sizes: the batch API against the same buffers one at a time.
    Prints the line (emit) and returns it."""
    import torch

    from reproducibility_icpp23_scalable_gpu_deduplication_b200 import (CheckpointBatch, ListDeduplicator,
                                                                        TreeDeduplicator, replicas, synth)
    from reproducibility_icpp23_scalable_gpu_deduplication_b200.tree import reserve_map_memory

    Dedup = ListDeduplicator if args.approach == "list" else TreeDeduplicator

    sizes = synth.batched_sizes(count=args.buffers, hi=args.max_buffer)
    total = sum(sizes)
    chunks = sum((n + 127) // 128 for n in sizes)
    stream = torch.cuda.current_stream()
    seed = synth.SEED + rank
    ckpts = 1 + args.warmup + args.steps

    def series_pass(step_fn, tune_fn=None):
        ss = batched_series(sizes, dev, seed)
        hs = [Dedup(128) for _ in sizes]
        times, sums, launches, dbytes = [], [], 0, []
        grows0 = 0
        for c in range(ckpts):
            bufs = [s.next() for s in ss]
            torch.cuda.synchronize()
            if world > 1:
                import torch.distributed as dist

                dist.barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            nl = step_fn(hs, bufs, c == 0)
            e1.record(stream)
            torch.cuda.synchronize()
            if c > args.warmup:
                times.append(e0.elapsed_time(e1))
                launches += nl
                dbytes.append(sum(h.diff_device()[1] for h in hs))
            sums.append([h.diff_checksum() for h in hs])
            if c == args.warmup:
                # the maps' baselines are in place: keep device memory mapped for their growth
                # (as a long-running service does), and count the growths of the timed steps
                if args.map_reserve > 0:
                    reserve_map_memory(int(args.map_reserve))
                grows0 = sum(h.map_stats()[2] for h in hs)
        grows = sum(h.map_stats()[2] for h in hs) - grows0
        for h in hs:
            h.close()
        del ss, bufs
        torch.cuda.empty_cache()
        series_pass.diff_bytes = statistics.mean(dbytes) if dbytes else 0
        return times, sums, launches, grows

    def plain_step(hs, bufs, base):
        n = 0
        for h, b in zip(hs, bufs):
            h.checkpoint_device(b, base)
            n += h.last_launch_count()
        return n

    batch = CheckpointBatch()
    if not args.no_autotune:
        # tuning series: a baseline, then incremental batches until the tuner settles
        batch.set_param("autotune", 1)
        ss = batched_series(sizes, dev, seed + 1000)
        hs = [Dedup(128) for _ in sizes]
        for c in range(args.tune_batches):
            batch.checkpoint(hs, [s.next() for s in ss])
            if batch.get_param("tuned"):
                break
        for h in hs:
            h.close()
        del ss
        torch.cuda.empty_cache()
    tuned = {k: batch.get_param(k) for k in ("shared", "leaf_stages", "leaf_ctas_per_sm", "tiles_per_pop",
                                              "warp_bands", "map_headroom_pct")}

    def batch_step(hs, bufs, base):
        batch.checkpoint(hs, bufs)
        return batch.launch_count()

    with ClockSampler(int(dev.index or 0)) as clk:
        t_plain, s_plain, l_plain, g_plain = (series_pass(plain_step) if not args.no_plain
                                              else ([float("nan")], None, 0, 0))
        t_batch, s_batch, l_batch, g_batch = series_pass(batch_step)
    same = s_plain == s_batch or args.no_plain
    ms_b, ms_p = statistics.mean(t_batch), statistics.mean(t_plain)
    rate_b, ms_b = replicas.throughput(ms_b, total, dev)
    rate_p, ms_p = replicas.throughput(ms_p, total, dev) if not args.no_plain else (float("nan"), ms_p)
    value = rate_b / GB
    plain = rate_p / GB
    peak, peak_kind = measured_peak()
    # algorithmic bytes of a step, as the plain form's step fraction counts them: every buffer
    # read, a prior digest read and a digest written per chunk, and the diffs written
    diff_b = int(series_pass.diff_bytes)
    alg = total + 32 * chunks + diff_b
    line = {
        "metric": f"{args.approach}-dedup batched ingest GB/s", "value": round(value, 2), "unit": "GB/s", "n_gpus": world,
        "steps": len(t_batch), "warmup": args.warmup, "ms_per_step": round(ms_b, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded; reference datasets unavailable)",
        "config": {"workload": f"batched_{len(sizes)}", "buffers": len(sizes), "total_bytes": total,
                   "min_buffer": min(sizes), "max_buffer": max(sizes), "chunk_size": 128, "hash": "murmur3",
                   "approach": args.approach, "checkpoints": ckpts, "change": "uniform [0.5%, 20%] in runs of 1-256 chunks + 1% shifted",
                   "l2": f"inputs {total / 2**30:.1f} GiB > L2, no flush", "tuned": tuned},
        "plain_same_workload": None if args.no_plain else {
            "value": round(plain, 2), "unit": "GB/s", "ms_per_step": round(ms_p, 4), "gpu_launches": l_plain},
        "speedup_vs_plain": None if args.no_plain else round(value / plain, 3),
        "map_growth": {"reserved_bytes": int(args.map_reserve), "grows_in_timed_steps": {"batched": g_batch,
                                                                                        "one_at_a_time": g_plain}},
        "parity": ("not compared (--no-plain)" if args.no_plain else ("identical" if same else "MISMATCH") +
                   f": diff checksums of {len(sizes)} buffers x {ckpts} checkpoints, batched vs one at a time"),
        "e2e": None,
        "gpu_launches": l_batch,
        "roofline": {"bound": "hbm", "kernel": "whole batch (graph)", "achieved": round(alg / (ms_b * 1e-3) / GB, 1),
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": round(alg / (ms_b * 1e-3) / GB / peak, 4), "traffic": None,
                     "algorithmic_bytes": alg, "diff_bytes_per_step": diff_b},
        "clocks": clk.summary(),
    }
    if rank == 0 and emit:
        print(json.dumps(line), flush=True)
    batch.close()
    if not same and emit:
        sys.exit(3)
    return line


def serve_stream(server_kw, sizes, clients, arrivals, dev, warm_rounds=2, reserve=0):
    """Drive one CheckpointServer through a request stream; returns (requests, wall seconds)."""
    import torch

    from reproducibility_icpp23_scalable_gpu_deduplication_b200 import synth
    from reproducibility_icpp23_scalable_gpu_deduplication_b200.serve import CheckpointServer

    series = [synth.DeviceSeries(n, 128, c, device=dev) for c, n in enumerate(sizes)]
    srv = CheckpointServer(**server_kw)
    # every client's baseline and first incremental checkpoints before the stream (resident state)
    for _ in range(warm_rounds):
        for c in range(len(sizes)):
            srv.submit(c, series[c].next())
        srv.drain()
    if reserve:
        srv.reserve_growth(reserve)     # clients resident: keep memory mapped for map growth
    srv.enable_host_copy({c: n for c, n in enumerate(sizes)})   # a request ends with its diff on the host
    torch.cuda.synchronize()
    srv.completed.clear()
    clock = srv.clock
    # clients act independently: a client submits its next request once it is due and its
    # previous one has completed (its buffer is free to edit); nobody waits for another client
    due = [collections.deque() for _ in sizes]
    for c, a in zip(clients, arrivals):
        due[int(c)].append(float(a))
    active = {c for c in range(len(sizes)) if due[c]}
    reqs, submitted = [], []
    t0 = clock()
    while active:
        now = clock() - t0
        for c in sorted(active, key=lambda c: due[c][0]):
            if due[c][0] <= now and not srv.busy(c):
                a = due[c].popleft()
                buf = series[c].next()
                submitted.append(clock())
                reqs.append(srv.submit(c, buf, arrival=t0 + a))
                if not due[c]:
                    active.discard(c)
        srv.step()
    srv.drain()
    wall = max(r.done for r in reqs) - t0
    batches = srv.batches
    service = [r.done - t for r, t in zip(reqs, submitted)]
    grows = sum(c.handle.map_stats()[2] for c in srv.clients.values() if c.handle is not None)
    queue = sorted(1e3 * (r.launched - t) for r, t in zip(reqs, submitted))
    execu = sorted(1e3 * (r.done - r.launched) for r in reqs)
    print(json.dumps({"diag": "served_stream", "plain": bool(server_kw.get("plain")), "map_grows_total": grows,
                      "queue_ms_p50_p99_max": [queue[len(queue) // 2], queue[int(0.99 * len(queue))], queue[-1]],
                      "exec_ms_p50_p99_max": [execu[len(execu) // 2], execu[int(0.99 * len(execu))], execu[-1]],
                      "slowest": sorted(((round(1e3 * (r.done - t), 1), r.client, r.nbytes >> 20,
                                          round(1e3 * (r.launch_s or 0), 2), r.batch_size,
                                          round(1e3 * (r.done - r.launched), 1))
                                         for r, t in zip(reqs, submitted)), reverse=True)[:8]}),
          file=sys.stderr, flush=True)
    srv.close()
    del series
    torch.cuda.empty_cache()
    return reqs, wall, batches, service


def serve_capacity(server_kw, sizes, waves, dev, warm_rounds=2):
    """Saturation: every client's next buffer is edited and resident, then all clients submit at
    once and the loop drains them; repeated `waves` times.  Returns (requests, busy seconds,
    batches, service times)."""
    import torch

    from reproducibility_icpp23_scalable_gpu_deduplication_b200 import synth
    from reproducibility_icpp23_scalable_gpu_deduplication_b200.serve import CheckpointServer

    series = [synth.DeviceSeries(n, 128, c, device=dev) for c, n in enumerate(sizes)]
    srv = CheckpointServer(**server_kw)
    for _ in range(warm_rounds):
        for c in range(len(sizes)):
            srv.submit(c, series[c].next())
        srv.drain()
    reqs, service, busy = [], [], 0.0
    b0 = srv.batches
    for _ in range(waves):
        bufs = [s.next() for s in series]
        torch.cuda.synchronize()
        t = srv.clock()
        wave = [srv.submit(c, bufs[c], arrival=t) for c in range(len(sizes))]
        srv.drain()
        busy += max(r.done for r in wave) - t
        reqs += wave
        service += [r.done - t for r in wave]
    batches = srv.batches - b0
    srv.close()
    del series, bufs
    torch.cuda.empty_cache()
    return reqs, busy, batches, service


def run_served(args, rank, world, dev, emit=True):
    """64 clients, Poisson arrivals: the continuous-batching loop against the one-at-a-time loop.
    Prints the line (emit) and returns it."""
    from reproducibility_icpp23_scalable_gpu_deduplication_b200 import synth
    from reproducibility_icpp23_scalable_gpu_deduplication_b200.serve import percentile

    sizes = synth.served_sizes(count=args.clients, hi=args.client_max_buffer)
    rng = np.random.default_rng(synth.SEED + rank)
    n = args.requests
    clients = rng.integers(0, len(sizes), n)
    arrivals = synth.poisson_arrivals(args.rate, n, seed=synth.SEED + rank)
    budget = args.hbm_budget
    kw = {"hbm_budget": budget, "max_batch": 64, "max_inflight": 2, "approach": args.approach}

    def summarize(reqs, wall, batches, service):
        lat = [1e3 * r.latency for r in reqs]
        svc = [1e3 * v for v in service]
        byt = sum(r.nbytes for r in reqs)
        return {"value": round(byt / wall / GB, 2), "unit": "GB/s", "p50_ms": round(percentile(lat, 50), 3),
                "p99_ms": round(percentile(lat, 99), 3), "max_ms": round(max(lat), 3),
                "service_p50_ms": round(percentile(svc, 50), 3), "service_p99_ms": round(percentile(svc, 99), 3),
                "requests": len(reqs), "batches": batches, "failed": sum(1 for r in reqs if r.rc != 0),
                "wall_s": round(wall, 3)}

    with ClockSampler(int(dev.index or 0)) as clk:
        served = summarize(*serve_stream(kw, sizes, clients, arrivals, dev, reserve=args.map_reserve))
        plain = summarize(*serve_stream(dict(kw, plain=True), sizes, clients, arrivals, dev,
                                        reserve=args.map_reserve))
        # capacity: all clients' requests waiting at once (unbounded arrival rate), 4 waves
        cap_served = summarize(*serve_capacity(kw, sizes, args.capacity_waves, dev))
        cap_plain = summarize(*serve_capacity(dict(kw, plain=True), sizes, args.capacity_waves, dev))
    line = {
        "metric": f"{args.approach}-dedup served GB/s", "value": served["value"], "unit": "GB/s", "n_gpus": world,
        "steps": n, "warmup": 2, "ms_per_step": served["p50_ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded; reference datasets unavailable)",
        "config": {"workload": f"served_{len(sizes)}_clients", "clients": len(sizes), "rate_hz": args.rate,
                   "requests": n, "client_bytes_total": sum(sizes), "min_buffer": min(sizes),
                   "max_buffer": max(sizes), "chunk_size": 128, "hash": "murmur3", "approach": args.approach,
                   "hbm_budget": budget, "map_growth_reserve": args.map_reserve,
                   "change": "uniform [0.5%, 20%] in runs of 1-512 chunks + 1% shifted, edited on the device",
                   "latency": "scheduled arrival -> diff in pinned host memory (includes the client's wait "
                              "for its own previous request and its device-side edit of its buffer); "
                              "service_*: submission -> diff on the host; capacity: diffs stay on the device"},
        "latency_ms": {"p50": served["p50_ms"], "p99": served["p99_ms"], "max": served["max_ms"]},
        "served": served, "plain_same_stream": plain,
        "capacity": {"mode": f"all {len(sizes)} clients submit at once, buffers edited and resident; "
                             f"{args.capacity_waves} waves",
                     "served": cap_served, "plain": cap_plain,
                     "speedup_vs_plain": round(cap_served["value"] / cap_plain["value"], 3)},
        "e2e": None, "clocks": clk.summary(),
    }
    if rank == 0 and emit:
        print(json.dumps(line), flush=True)
    return line


def bounded_forms(args, rank, world, dev):
    """The batched form (all 256 buffers, 2 warm-up and --forms-steps timed batches after at most
    8 autotuning batches: a baseline and the tuner's 7) and the served form (64 clients, --forms-requests Poisson requests, 2
    capacity waves), summarised as two keys of the plain line."""
    import copy

    import torch

    b_args = copy.copy(args)
    b_args.warmup, b_args.steps, b_args.tune_batches = 2, max(1, args.forms_steps), 8
    b = run_batched(b_args, rank, world, dev, emit=False)
    torch.cuda.empty_cache()
    s_args = copy.copy(args)
    s_args.requests, s_args.capacity_waves = max(1, args.forms_requests), 2
    sv = run_served(s_args, rank, world, dev, emit=False)
    torch.cuda.empty_cache()
    batched = {k: b[k] for k in ("value", "unit", "ms_per_step", "steps", "speedup_vs_plain", "parity",
                                 "gpu_launches", "map_growth")}
    batched["one_at_a_time"] = b["plain_same_workload"]
    batched["roofline_frac"] = b["roofline"]["frac"]
    batched["config"] = {k: b["config"][k] for k in ("workload", "buffers", "total_bytes", "checkpoints", "change",
                                                      "tuned")}
    served = {"value": sv["value"], "unit": sv["unit"], "latency_ms": sv["latency_ms"],
              "one_at_a_time": {k: sv["plain_same_stream"][k] for k in ("value", "p50_ms", "p99_ms", "max_ms")},
              "capacity": {"value": sv["capacity"]["served"]["value"],
                           "one_at_a_time": sv["capacity"]["plain"]["value"],
                           "speedup_vs_plain": sv["capacity"]["speedup_vs_plain"]},
              "config": {k: sv["config"][k] for k in ("workload", "clients", "rate_hz", "requests", "hbm_budget",
                                                       "latency")}}
    return {"batched": batched, "served": served}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.form != "plain":
        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dev = torch.device("cuda", local)
        if world > 1:
            import datetime

            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
        if args.form == "batched":
            run_batched(args, rank, world, dev)
        else:
            run_served(args, rank, world, dev)
        if world > 1:
            dist.destroy_process_group()
        return

    import torch
    import torch.distributed as dist

    from reproducibility_icpp23_scalable_gpu_deduplication_b200 import (HASH_MD5, HASH_MURMUR3, ListDeduplicator,
                                                                        TreeDeduplicator, replicas, synth)
    from reproducibility_icpp23_scalable_gpu_deduplication_b200.tree import parse_header, reserve_map_memory

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    cs = args.chunk_size
    nbytes = args.nbytes
    n_chunks = (nbytes + cs - 1) // cs

    md5 = args.workload == "md5_f32_8g"
    series = workload_series(args.workload, nbytes, cs, dev, synth.SEED + rank)
    Dedup = ListDeduplicator if args.approach == "list" else TreeDeduplicator
    dd = Dedup(cs, HASH_MD5 if md5 else HASH_MURMUR3)
    if args.leaf_stages:
        dd.set_param("leaf_stages", args.leaf_stages)
    if args.leaf_ctas:
        dd.set_param("leaf_ctas_per_sm", args.leaf_ctas)
    if args.leaf_unit:
        dd.set_param("leaf_unit", args.leaf_unit)
    if args.graph is not None:
        dd.set_param("graph", args.graph)
    if args.map_headroom:
        dd.set_param("map_headroom_pct", args.map_headroom)
    dd.checkpoint_device(series.next(), make_baseline=True)          # checkpoint 0: baseline
    for _ in range(args.warmup):
        dd.checkpoint_device(series.next())
    # the map's baseline is in place: keep device memory mapped for its growth (a long-running
    # user's steady state; an unreserved growth is dominated by its allocation)
    if args.map_reserve > 0:
        reserve_map_memory(int(args.map_reserve))
    grows0 = dd.map_stats()[2]
    # the steps' inputs are materialised in HBM before they are timed, in groups that fit half of
    # the free device memory (one group for the 4 GiB workload, two for the 8 GiB MD5 one); each
    # group is timed on the device and the group times add up
    free_b, _ = torch.cuda.mem_get_info(dev)
    group = replicas.agree_min(max(1, min(args.steps, int(0.5 * free_b) // nbytes)), dev)

    stream = torch.cuda.current_stream()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    leaf_s, forest_s, gather_s, diff_bytes, launches = [], [], [], [], 0
    # inputs smaller than 2x the 126 MB L2: flush L2 before each step (outside the timed spans)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev) if nbytes < (256 << 20) else None
    step_ms, group_ms = [], []
    with ClockSampler(local) as clk:
        done = 0
        while done < args.steps:
            bufs = [series.next().clone() for _ in range(min(group, args.steps - done))]
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize()
            start.record(stream)
            for b in bufs:
                if flush is not None:
                    flush.fill_(1)
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                diff_bytes.append(dd.checkpoint_device(b))
                if flush is not None:
                    e1.record(stream)
                    e1.synchronize()
                    step_ms.append(e0.elapsed_time(e1))
                ph, path = dd.phase_times()
                leaf_s.append(ph[0])
                forest_s.append(ph[1])
                gather_s.append(ph[2])
                launches += dd.last_launch_count()
            stop.record(stream)
            torch.cuda.synchronize()
            group_ms.append(start.elapsed_time(stop))
            done += len(bufs)
            del bufs
    if world > 1:
        dist.barrier()
    ms = sum(group_ms) if flush is None else sum(step_ms)
    grows_timed = dd.map_stats()[2] - grows0
    del flush
    # replicas: the slowest rank's time, every rank's bytes
    rate, ms_max = replicas.throughput(ms, args.steps * nbytes, dev)
    value = rate / GB
    leaf_ms = 1e3 * statistics.mean(leaf_s)   # 0 when the graph runs without timing events

    # end to end through the public API: each step copies its input from pinned host memory to
    # the device and checkpoints it with the host-diff call, which brings the diff back into the
    # library's pinned host buffer (read through a view, no further host copy).  One untimed step
    # first sizes the host-side staging.
    e2e_bufs = [torch.empty(nbytes, dtype=torch.uint8, pin_memory=True) for _ in range(args.e2e_steps)]
    dbuf = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    if e2e_bufs:
        e2e_bufs[-1].copy_(series.next().view(torch.uint8).reshape(-1))
        dbuf.copy_(e2e_bufs[-1], non_blocking=True)
        dd.checkpoint(dbuf, copy=False)
        torch.cuda.synchronize()
    for hb in e2e_bufs:
        hb.copy_(series.next().view(torch.uint8).reshape(-1))
    d2h = []
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for hb in e2e_bufs:
        dbuf.copy_(hb, non_blocking=True)
        d2h.append(len(dd.checkpoint(dbuf, copy=False)))
    e1.record(stream)
    torch.cuda.synchronize()
    e_ms = e0.elapsed_time(e1)
    e2e_value = replicas.throughput(e_ms, len(e2e_bufs) * nbytes, dev)[0] / GB if e2e_bufs else None
    del e2e_bufs

    # restart: rebuild the last checkpoint of a fresh 4-checkpoint series from its diffs held in
    # pinned host memory (host -> device copies and scatter inside the timed span)
    restart = None
    if not args.no_restart:
        rs = workload_series(args.workload, nbytes, cs, dev, synth.SEED + rank + 17)
        rd = Dedup(cs, HASH_MD5 if md5 else HASH_MURMUR3)
        diffs = []
        for k in range(4):
            x = rs.next()
            rd.checkpoint_device(x, k == 0)
            pin = torch.empty(rd.diff_device()[1], dtype=torch.uint8).pin_memory()
            diffs.append(rd.copy_diff(pin.numpy()))
        out = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        rd.restart(out, diffs, 3)
        torch.cuda.synchronize()
        r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        r0.record(stream)
        rd.restart(out, diffs, 3)
        r1.record(stream)
        torch.cuda.synchronize()
        r_ms = r0.elapsed_time(r1)
        ok = bool(torch.equal(out, x.view(torch.uint8).reshape(-1)[:nbytes]))
        # the same chain with the diffs resident in device memory
        ddiffs = [torch.from_numpy(dh).to(dev) for dh in diffs]
        out.zero_()
        rd.restart_device(out, ddiffs, 3)
        torch.cuda.synchronize()
        r0.record(stream)
        rd.restart_device(out, ddiffs, 3)
        r1.record(stream)
        torch.cuda.synchronize()
        rd_ms = r0.elapsed_time(r1)
        ok_d = bool(torch.equal(out, x.view(torch.uint8).reshape(-1)[:nbytes]))
        # restart roofline: the output written once, every output chunk read once from some
        # diff's data section, and every diff's header and region lists read
        hdrs = [parse_header(dh) for dh in diffs]
        meta = sum(32 + 4 * h["num_first_ocur"] + 8 * (h["num_prior_chkpts"] + h["num_shift_dupl"]) for h in hdrs)
        alg = 2 * nbytes + meta
        peak_r, peak_kind_r = measured_peak()
        restart = {"value": round(nbytes / (r_ms * 1e-3) / GB, 2), "unit": "GB/s", "ms": round(r_ms, 3),
                   "diffs": 4, "h2d_bytes": int(sum(d.nbytes for d in diffs)), "identical": ok,
                   "device_diffs": {"value": round(nbytes / (rd_ms * 1e-3) / GB, 2), "unit": "GB/s",
                                    "ms": round(rd_ms, 3), "identical": ok_d,
                                    "roofline": {"bound": "hbm", "algorithmic_bytes": alg,
                                                 "achieved": round(alg / (rd_ms * 1e-3) / GB, 1), "peak": peak_r,
                                                 "peak_kind": peak_kind_r, "unit": "GB/s",
                                                 "frac": round(alg / (rd_ms * 1e-3) / GB / peak_r, 4)}}}
        del ddiffs
        rd.close()
        del rs, diffs, out, x
        torch.cuda.empty_cache()

    peak, peak_kind = measured_peak()
    alg_leaf = nbytes + 32 * n_chunks              # read the buffer, read + write a digest per chunk
    achieved = alg_leaf / (leaf_ms * 1e-3) / GB if leaf_ms > 0 else 0.0
    tb = leaf_traffic(cs)
    roofline = {"bound": "hbm", "kernel": f"leaf_tma_kernel (chunk {cs} B)" if path else "leaf_generic_kernel",
                "achieved": round(achieved, 1), "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": round(tb * nbytes) if tb else None,
                "algorithmic_bytes": alg_leaf, "launch_ms": round(leaf_ms, 4),
                "step_frac": round(((nbytes + 32 * n_chunks + statistics.mean(diff_bytes)) /
                                    (ms_max * 1e-3 / args.steps) / GB) / peak, 4)}
    line = {
        "metric": f"{args.approach}-dedup ingest GB/s", "value": round(value, 2), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded; reference datasets unavailable)",
        "config": {"workload": args.workload, "nbytes": nbytes, "chunk_size": cs, "hash": "md5" if md5 else "murmur3",
                   "approach": args.approach, "checkpoints": 1 + args.warmup + args.steps,
                   "timed_groups": f"{len(group_ms)} (inputs of a group resident in HBM before it is timed)",
                   "map_growth": {"reserved_bytes": int(args.map_reserve), "grows_in_timed_steps": grows_timed,
                                  "baseline_headroom_pct": args.map_headroom or 150},
                   "l2": (f"inputs {nbytes / 2**30:.2f} GiB > L2, no flush" if nbytes >= (256 << 20) else
                          "L2 flushed (512 MiB write) before each step, outside the timed spans"),
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": round(e2e_value, 2) if e2e_value else None, "unit": "GB/s", "h2d_bytes_per_step": nbytes,
                "d2h_bytes_per_step": int(statistics.mean(d2h)) if d2h else 0},
        "gpu_launches": launches,
        "restart": restart,
        "roofline": roofline,
        "clocks": clk.summary(),
        "diff_bytes_per_step": int(statistics.mean(diff_bytes)),
        "phases_ms": {"leaf": round(leaf_ms, 4), "forest": round(1e3 * statistics.mean(forest_s), 4),
                      "gather": round(1e3 * statistics.mean(gather_s), 4)},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        cpu_bytes = args.cpu_sample_bytes or nbytes
        torch.cuda.empty_cache()
        gbps, _ = cpu_baseline_run(cpu_bytes, cs, args.cpu_steps, threads, args.workload, args.approach,
                                   warmup=1, device=dev)
        line["cpu_baseline"] = {"value": round(gbps, 4), "unit": "GB/s", "cores": threads, "kind": "port",
                                "sample": cpu_sample_text(cpu_bytes, args.workload, cs, 1, args.cpu_steps)}
    if world == 1 and args.workload == "plain_4g" and not args.no_forms:
        # the batched and served forms, bounded to a few batches and a few hundred requests, so
        # the default line carries them next to the plain form
        dd.close()
        del series
        torch.cuda.empty_cache()
        line.update(bounded_forms(args, rank, world, dev))
    if rank == 0:
        print(json.dumps(line), flush=True)
    dd.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
