"""Several training images in the batched engine (-ti a b [c], -ii): every
level's nodes mapped against each TI, each TI's k best with the same seed,
merged and drawn on the GPU as G2S does with one CUDA device per TI
(quantileSamplingModule.hpp:90-126).  The simulation and the index image
(TI cell * nTI + TI) equal the oracle's several-TI simulation bit for bit
(the oracle is pinned to the reference in test_oracle_multi_ti.py)."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["multi_ti", "multi_ti_ii", "multi_ti3", "multi_ti_eq"])
def test_batched_several_tis_equal_oracle(g2s, gpu, oracle, name):
    g = golden(name)
    nti = int(g["nti"])
    tis = [g[f"ti{i}"] for i in range(nti)]
    types = [int(t) for t in g["types"]]
    sim = g2s.Simulation(tis[0], g["di"], types, n=int(g["n"]), k=float(g["k"]), seed=int(g["seed"]),
                         extra_tis=tis[1:], ii=g.get("ii"))
    sim.run()
    out, idx, _ = sim.read()
    sim.close()
    o = oracle.simulate_multi(tis, g["di"], types, int(g["n"]), float(g["k"]), int(g["seed"]), ii=g.get("ii"))
    assert np.array_equal(out, o["sim"])
    assert np.array_equal(idx.ravel(), o["id"])
    assert len(np.unique(idx.ravel() % nti)) > 1


def test_batched_several_tis_rejections(g2s, gpu):
    g = golden("multi_ti")
    tis = [g["ti0"], g["ti1"]]
    sim = g2s.Simulation(tis[0], g["di"], [0], n=12, k=1.2, seed=7, extra_tis=tis[1:])
    with pytest.raises(RuntimeError):
        sim.set_tensor("bf16")
    sim.close()
    with pytest.raises(RuntimeError):   # 2 TIs x ceil(9) candidates > 16
        g2s.Simulation(tis[0], g["di"], [0], n=12, k=9.0, seed=7, extra_tis=tis[1:])
    with pytest.raises(RuntimeError):   # -ii naming a third TI
        g2s.Simulation(tis[0], g["di"], [0], n=12, k=1.2, seed=7, extra_tis=tis[1:],
                       ii=np.full(g["di"].shape, 2.0, np.float32))


def test_one_call_qs_with_several_tis_equals_oracle(g2s, gpu, oracle):
    """The one-call API with a list of training images and -ii."""
    g = golden("multi_ti_ii")
    tis = [g["ti0"], g["ti1"]]
    out, idx = g2s.qs(tis, g["di"], [0], k=float(g["k"]), n=int(g["n"]), s=int(g["seed"]), ii=g["ii"])
    o = oracle.simulate_multi(tis, g["di"], [0], int(g["n"]), float(g["k"]), int(g["seed"]), ii=g["ii"])
    assert np.array_equal(out, o["sim"])
    assert np.array_equal(idx.ravel(), o["id"])
