"""Failure detection without a GPU fault: the dependency-level pass bounds
every wait on a neighbour's level.  A host-side injection holds one path
node's level back (it is never published); its dependants' waits run out
after a few hundred polls, the run returns an error naming the wait, and the
same simulation object runs normally afterwards (the context stays usable)."""
import numpy as np
import pytest

from g2s_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def test_level_wait_runs_out_and_is_reported(g2s, gpu):
    ti = syn.grf((40, 40), (6, 6), seed=3)
    di = np.full((24, 24), np.nan, np.float32)
    ref = g2s.Simulation(ti, di, [0], n=12, k=1.2, seed=5)
    ref.run()
    want, want_idx, _ = ref.read()
    ref.close()

    sim = g2s.Simulation(ti, di, [0], n=12, k=1.2, seed=5)
    # path node 0 is an informed neighbour of the nodes simulated next to it
    sim.set_level_wait(spin_limit=256, hold_node=0)
    with pytest.raises(RuntimeError, match="wait limit"):
        sim.run()
    sim.set_level_wait(0, -1)
    sim.run()
    out, idx, _ = sim.read()
    sim.close()
    assert np.array_equal(out, want) and np.array_equal(idx, want_idx)


def test_level_wait_arguments_checked(g2s):
    ti = syn.grf((20, 20), (4, 4), seed=3)
    di = np.full((8, 8), np.nan, np.float32)
    try:
        sim = g2s.Simulation(ti, di, [0], n=6, k=1.2, seed=5)
    except RuntimeError:
        pytest.skip("no CUDA device")
    with pytest.raises(RuntimeError):
        sim.set_level_wait(100, 64)   # 64 path nodes: indices 0..63
    sim.close()
