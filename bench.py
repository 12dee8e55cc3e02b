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
             OpenMP-parallel hashing with all host threads, on a bounded sample of the workload

Multi-GPU (torchrun): every rank deduplicates its own buffer (independent replicas, like the
reference's MPI driver); nothing crosses ranks but the barrier and the max-time reduction.
"""
import argparse
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
    p.add_argument("--chunk-size", type=int, default=128)
    p.add_argument("--nbytes", type=int, default=4 << 30)
    p.add_argument("--e2e-steps", type=int, default=2)
    p.add_argument("--cpu-sample-bytes", type=int, default=512 << 20)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--leaf-stages", type=int, default=0, help="TMA ring depth (0 = library default)")
    p.add_argument("--leaf-ctas", type=int, default=0, help="hashing CTAs per SM (0 = library default)")
    return p.parse_args()


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


def cpu_baseline_run(nbytes, cs, steps, threads):
    """The oracle (sequential restatement of the reference) on the host, all threads hashing."""
    from oracle import oracle as O
    from reproducibility_icpp23_scalable_gpu_deduplication_b200 import synth

    s = synth.plain_4g(nbytes=nbytes, chunk_size=cs)
    o = O.OracleTreeDeduplicator(cs, O.HASH_MURMUR3, threads=threads)
    o.checkpoint(s.next(), True)
    t = 0.0
    for _ in range(steps):
        b = s.next()
        t0 = time.perf_counter()
        o.checkpoint(b, False)
        t += time.perf_counter() - t0
    return steps * nbytes / t / GB, t


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
    gbps, t = cpu_baseline_run(args.cpu_sample_bytes, args.chunk_size, steps, threads)
    sample = (f"{args.cpu_sample_bytes >> 20} MiB buffer with the 4 GiB workload's change pattern, chunk "
              f"{args.chunk_size} B, {steps} incremental checkpoints after an untimed baseline")
    line = {
        "impl": "reference", "metric": "tree-dedup ingest GB/s", "value": round(gbps, 4), "unit": "GB/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup, "ms_per_step": round(1e3 * t / steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": "plain_4g", "nbytes": args.nbytes, "chunk_size": args.chunk_size,
                   "hash": "murmur3"},
        "cpu_baseline": {"value": round(gbps, 4), "unit": "GB/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": round(gbps, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    import torch.distributed as dist

    from reproducibility_icpp23_scalable_gpu_deduplication_b200 import TreeDeduplicator, synth

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    cs = args.chunk_size
    nbytes = args.nbytes
    n_chunks = (nbytes + cs - 1) // cs

    series = synth.plain_4g(nbytes=nbytes, chunk_size=cs, device=dev, seed=synth.SEED + rank)
    dd = TreeDeduplicator(cs)
    if args.leaf_stages:
        dd.set_param("leaf_stages", args.leaf_stages)
    if args.leaf_ctas:
        dd.set_param("leaf_ctas_per_sm", args.leaf_ctas)
    dd.checkpoint_device(series.next(), make_baseline=True)          # checkpoint 0: baseline
    for _ in range(args.warmup):
        dd.checkpoint_device(series.next())
    bufs = [series.next().clone() for _ in range(args.steps)]
    torch.cuda.synchronize()

    stream = torch.cuda.current_stream()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    leaf_s, diff_bytes, launches = [], [], 0
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        start.record(stream)
        for b in bufs:
            diff_bytes.append(dd.checkpoint_device(b))
            ph, path = dd.phase_times()
            leaf_s.append(ph[0])
            launches += dd.last_launch_count()
        stop.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = start.elapsed_time(stop)
    t = torch.tensor([ms], device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * args.steps * nbytes / (ms_max * 1e-3) / GB
    leaf_ms = 1e3 * statistics.mean(leaf_s)
    del bufs

    # end to end through the public API: host buffers in pinned memory, diff back to the host
    e2e_bufs = []
    for _ in range(args.e2e_steps):
        e2e_bufs.append(series.next().cpu().pin_memory())
    dbuf = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    d2h = []
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for hb in e2e_bufs:
        dbuf.copy_(hb, non_blocking=True)
        d2h.append(len(dd.checkpoint(dbuf)))
    e1.record(stream)
    torch.cuda.synchronize()
    e_ms = e0.elapsed_time(e1)
    te = torch.tensor([e_ms], device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * len(e2e_bufs) * nbytes / (float(te.item()) * 1e-3) / GB if e2e_bufs else None

    peak, peak_kind = measured_peak()
    alg_leaf = nbytes + 32 * n_chunks              # read the buffer, read + write a digest per chunk
    achieved = alg_leaf / (leaf_ms * 1e-3) / GB
    tb = leaf_traffic(cs)
    roofline = {"bound": "hbm", "kernel": f"leaf_tma_kernel (chunk {cs} B)" if path else "leaf_generic_kernel",
                "achieved": round(achieved, 1), "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": round(tb * nbytes) if tb else None,
                "algorithmic_bytes": alg_leaf, "launch_ms": round(leaf_ms, 4),
                "step_frac": round(((nbytes + 32 * n_chunks + statistics.mean(diff_bytes)) /
                                    (ms_max * 1e-3 / args.steps) / GB) / peak, 4)}
    line = {
        "metric": "tree-dedup ingest GB/s", "value": round(value, 2), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded; reference datasets unavailable)",
        "config": {"workload": "plain_4g", "nbytes": nbytes, "chunk_size": cs, "hash": "murmur3",
                   "checkpoints": 1 + args.warmup + args.steps, "l2": "inputs 4 GiB > L2, no flush",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": round(e2e_value, 2) if e2e_value else None, "unit": "GB/s", "h2d_bytes_per_step": nbytes,
                "d2h_bytes_per_step": int(statistics.mean(d2h)) if d2h else 0},
        "gpu_launches": launches,
        "roofline": roofline,
        "clocks": clk.summary(),
        "diff_bytes_per_step": int(statistics.mean(diff_bytes)),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        gbps, _ = cpu_baseline_run(args.cpu_sample_bytes, cs, 2, threads)
        line["cpu_baseline"] = {"value": round(gbps, 4), "unit": "GB/s", "cores": threads, "kind": "port",
                                "sample": f"{args.cpu_sample_bytes >> 20} MiB buffer with this workload's change "
                                          f"pattern, 2 incremental checkpoints after a baseline"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    dd.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
