"""Autotuner on the GPU: tuning a small job shape chooses settings whose
audit passes, persists them, answers the second call from the cache, and a
simulation run with them stays within the regret bound."""
import numpy as np
import pytest

from g2s_b200 import autotune as at
from g2s_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def test_tune_persist_and_apply(g2s, gpu, tmp_path):
    ti = syn.grf((128, 128), (10, 10), seed=3)
    path = str(tmp_path / "tune.json")
    res = at.tune(ti, [0], n=30, k=1.2, grid=(96, 96), cache=path)
    print(res)
    assert not res["cached"] and res["ok"] and res["regret"] <= 0.001 * res["audited"]
    assert res["width"] in (0, 8, 16, 32) and res["batch"] in (2048, 4096, 8192) and res["prefix"] >= 64
    assert res["runs"] >= 7
    again = at.tune(ti, [0], n=30, k=1.2, grid=(96, 96), cache=path)
    assert again["cached"] and again["width"] == res["width"] and again["prefix"] == res["prefix"]
    di = np.full((96, 96), np.nan, np.float32)
    sim = g2s.Simulation(ti, di, [0], n=30, k=1.2, seed=77)
    at.apply(sim, res, audit=1.0)
    sim.run()
    info = sim.info()
    assert info["tensor_prefix"] == res["prefix"] and info["audited"] > 0
    assert info["regret"] <= 0.01 * info["audited"]
    sim.close()
