"""Device blocks kept from ended simulations (qsk_sim_destroy hands the
buffers over after a device synchronisation; DBuf::alloc takes them): a
simulation built on blocks another job left behind (other grid, other TI,
other path) gives the same output as the oracle, and the blocks are
reused."""
import numpy as np
import pytest

from g2s_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def run(g2s, ti, di, types, n, seed, tensor=None):
    sim = g2s.Simulation(ti, di, types, n=n, k=1.2, seed=seed)
    if tensor:
        sim.set_tensor(tensor, audit=0.0)
    sim.run()
    out = sim.read()
    sim.close()
    return out


def test_simulation_on_kept_blocks_equals_oracle(g2s, gpu, oracle):
    g2s.blocks_release()
    ti = syn.grf((64, 64), (6, 6), seed=3)
    di = np.full((48, 48), np.nan, np.float32)
    other = syn.channels2d((80, 80), n_channels=6, seed=4)
    run(g2s, other, np.full((60, 60), np.nan, np.float32), [1], 24, 9)   # leaves its blocks behind
    kept = g2s.blocks_info(0)
    assert kept["bytes"] > 0 and kept["blocks"] > 0
    v, i, _ = run(g2s, ti, di, [0], 16, 100)
    after = g2s.blocks_info(0)
    assert after["hits"] > kept["hits"]
    o = oracle.simulate(ti, di, [0], 16, 1.2, 100, mode=0)
    assert np.array_equal(v, o["sim"], equal_nan=True)
    assert np.array_equal(i.ravel(), o["id"])


def test_tensor_form_on_kept_blocks_is_unchanged(g2s, gpu):
    ti = syn.channels2d((96, 96), n_channels=8, seed=5)
    di = np.full((64, 64), np.nan, np.float32)
    g2s.blocks_release()
    first = run(g2s, ti, di, [1], 32, 7, tensor="bf16")
    run(g2s, syn.grf((70, 70), (5, 5), seed=6), np.full((50, 50), np.nan, np.float32), [0], 20, 3, tensor="bf16")
    again = run(g2s, ti, di, [1], 32, 7, tensor="bf16")
    for a, b in zip(first, again):
        assert np.array_equal(a, b, equal_nan=True)


def test_limit_zero_keeps_nothing(g2s, gpu):
    g2s.blocks_release()
    g2s.blocks_set_limit(0)
    try:
        run(g2s, syn.grf((40, 40), (5, 5), seed=1), np.full((32, 32), np.nan, np.float32), [0], 12, 2)
        assert g2s.blocks_info(0)["bytes"] == 0
    finally:
        g2s.blocks_set_limit(8 << 30)
    run(g2s, syn.grf((40, 40), (5, 5), seed=1), np.full((32, 32), np.nan, np.float32), [0], 12, 2)
    assert g2s.blocks_info(0)["bytes"] > 0
    g2s.blocks_release()
    assert g2s.blocks_info(0)["bytes"] == 0
