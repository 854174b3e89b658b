"""Several simulations in one call (qsk_jobs_run): jobs over different TIs,
uneven grids and neighbour counts run on their own streams from a pool of
host threads; each job's output must be bit-identical to the same job run
alone, with direct launches and with the batch chain captured in a CUDA
graph (qsk_sim_set_graph)."""
import numpy as np
import pytest

from g2s_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def job_specs():
    grf = syn.grf((96, 96), (8, 8), seed=11)
    chan = syn.channels2d((100, 100), n_channels=8, seed=12)
    biv = syn.bivariate(syn.grf((96, 96), (8, 8), seed=13))
    tis = [(grf, [0]), (chan, [1]), (biv, [0, 1])]
    sides = [40, 64, 80, 50, 72, 90]
    ns = [20, 40, 12, 30]
    specs = []
    for j in range(6):
        ti, types = tis[j % 3]
        shape = (sides[j], sides[j]) + ((2,) if len(types) > 1 else ())
        specs.append(dict(ti=ti, types=types, di=np.full(shape, np.nan, np.float32), n=ns[j % 4], k=1.2,
                          seed=100 + j, tensor="bf16" if j == 4 else None))
    return specs


def make(g2s, sp, graph=False):
    sim = g2s.Simulation(sp["ti"], sp["di"], sp["types"], n=sp["n"], k=sp["k"], seed=sp["seed"])
    if sp["tensor"]:
        sim.set_tensor(sp["tensor"], audit=0.0)
    if graph:
        sim.set_graph(True)
    return sim


def single_runs(g2s, specs):
    out = []
    for sp in specs:
        sim = make(g2s, sp)
        sim.run()
        out.append(sim.read())
        sim.close()
    return out


@pytest.mark.parametrize("graph", [False, True])
def test_jobs_equal_single_runs(g2s, gpu, graph):
    specs = job_specs()
    ref = single_runs(g2s, specs)
    sims = [make(g2s, sp, graph) for sp in specs]
    status = g2s.run_jobs(sims, threads=4)
    assert list(status) == [0] * len(specs)
    for j, (sim, (v0, i0, c0)) in enumerate(zip(sims, ref)):
        v, i, c = sim.read()
        assert np.array_equal(v, v0, equal_nan=True), j
        assert np.array_equal(i, i0), j
        assert np.array_equal(c, c0), j
        info = sim.info()
        if graph and not specs[j]["tensor"]:
            assert info["graph_nodes"] > 0
        else:
            assert info["graph_nodes"] == 0
        sim.close()


def test_jobs_plain_equal_oracle(g2s, gpu, oracle):
    """The plain jobs of the batch against the CPU oracle as well."""
    specs = [sp for sp in job_specs() if not sp["tensor"]][:3]
    sims = [make(g2s, sp) for sp in specs]
    g2s.run_jobs(sims, threads=3)
    for sp, sim in zip(specs, sims):
        v, i, _ = sim.read()
        o = oracle.simulate(sp["ti"], sp["di"], sp["types"], sp["n"], sp["k"], sp["seed"], mode=0)
        assert np.array_equal(v, o["sim"], equal_nan=True)
        assert np.array_equal(i.ravel(), o["id"])
        sim.close()


def test_jobs_error_names_the_job(g2s, gpu):
    sp = job_specs()[0]
    a = make(g2s, sp)
    with pytest.raises(ValueError):
        g2s.run_jobs([a, a])
    a.close()
