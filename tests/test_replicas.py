"""The replica path of bench.py on CPU: two gloo ranks, each with its own measurement; the job
reports the slowest rank's time and everyone's work (no data crosses ranks)."""
import os

import pytest
import torch.multiprocessing as mp


def _rank(rank, world, port, q):
    import torch.distributed as dist

    from reproducibility_icpp23_scalable_gpu_deduplication_b200 import replicas, synth

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # each rank's buffer comes from its own seed (independent replicas)
        s = synth.plain_64m(nbytes=1 << 16, seed=synth.SEED + rank)
        first = bytes(s.next()[:64])
        ms = 10.0 * (rank + 1)
        rate, ms_max = replicas.throughput(ms, 1000 * (rank + 1))
        group = replicas.agree_min(5 + 3 * rank)   # e.g. inputs per timed group, from free memory
        q.put((rank, rate, ms_max, first, replicas.world(), group))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, rate0, ms0, b0, w0, g0), (r1, rate1, ms1, b1, w1, g1) = out
    assert w0 == w1 == 2
    assert g0 == g1 == 5                            # every rank groups its timed steps alike
    assert ms0 == ms1 == 20.0                       # the slowest rank's time
    assert rate0 == rate1 == pytest.approx(3000 / 0.020)   # everyone's units
    assert b0 != b1                                 # replicas checkpoint different data
