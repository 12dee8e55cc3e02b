"""The staged hashing kernel's bounded barrier waits, made to give up.

Every wait of the TMA hashing kernel on its shared-memory ring is bounded: when it runs out the
kernel records B2D_ERR_TIMEOUT, the producer waits for the copies it still has in flight (they
write into the CTA's shared memory) and the CTA exits; nothing traps or hangs.  The parameter
``leaf_wait_polls`` replaces the bound by that many non-blocking polls, so a wait runs out at
the first stage (a bulk copy from HBM takes far longer than one poll).  After the timeout the
handle accepts only a baseline, and that baseline and the checkpoints after it are bit-exact
with the oracle: the context stays usable.
"""
import numpy as np
import pytest

from oracle import oracle as O
from reproducibility_icpp23_scalable_gpu_deduplication_b200 import B2DError, TreeDeduplicator, synth

pytestmark = pytest.mark.gpu

B2D_ERR_LEN_CHANGED = -10
B2D_ERR_TIMEOUT = -7


def to_dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("where", ["baseline", "incremental"])
def test_wait_gives_up_and_handle_recovers(cuda, where):
    s = synth.plain_64m(nbytes=16 << 20)
    bufs = [s.next().copy() for _ in range(4)]
    g = TreeDeduplicator(128)
    if where == "incremental":
        assert g.checkpoint(to_dev(bufs[0]), True) == O.OracleTreeDeduplicator(128).checkpoint(bufs[0], True)
    g.set_param("leaf_wait_polls", 1)
    with pytest.raises(B2DError) as e:
        g.checkpoint(to_dev(bufs[1]), where == "baseline")
    assert e.value.code == B2D_ERR_TIMEOUT
    _, path = g.phase_times()
    assert path == 1, "the staged (TMA) hashing kernel ran"
    g.set_param("leaf_wait_polls", 0)
    if where == "incremental":
        # the tree and map may be part-way updated: only a baseline is accepted next (a handle
        # whose first checkpoint failed takes any checkpoint as its baseline anyway)
        with pytest.raises(B2DError) as e:
            g.checkpoint(to_dev(bufs[1]), False)
        assert e.value.code == B2D_ERR_LEN_CHANGED
    # the oracle takes the same sequence: bufs[1] as a baseline, then bufs[2], bufs[3] (the failed
    # call did not advance the handle's checkpoint id)
    o = O.OracleTreeDeduplicator(128)
    if where == "incremental":
        o.checkpoint(bufs[0], True)
    for i, b in enumerate(bufs[1:]):
        assert g.checkpoint(to_dev(b), i == 0) == o.checkpoint(b, i == 0), i
    g.close()
