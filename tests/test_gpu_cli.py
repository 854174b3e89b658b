"""qs_b200, the G2S `qs` command line on the GPU engine, end to end: grids
written as .bgrid into a data directory, the command run as a process, its
<id>.bgrid / id_<id>.bgrid outputs compared with the reference's results."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden

pytestmark = pytest.mark.gpu

EXE = os.path.join(ROOT, "g2s_b200", "qs_b200")


def run_cli(g2s, tmp_path, g, args, grids):
    env = dict(os.environ, G2S_DATA_DIR=str(tmp_path))
    types = [int(t) for t in g["types"]]
    g2s.write_bgrid(str(tmp_path / "ti.bgrid"), g["ti"], types)
    g2s.write_bgrid(str(tmp_path / "di.bgrid"), g["di"], types)
    for name, (arr, ty) in grids.items():
        g2s.write_bgrid(str(tmp_path / (name + ".bgrid")), arr, ty)
    r = subprocess.run([EXE, "-ti", "ti", "-di", "di", "-id", "job", "-W_CUDA", "0"] + args, capture_output=True,
                       text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "compuattion time" in r.stderr
    sim, _ = g2s.read_bgrid(str(tmp_path / "job.bgrid"))
    idx, _ = g2s.read_bgrid(str(tmp_path / "id_job.bgrid"))
    return sim, idx


def test_cli_equals_reference(g2s, gpu, tmp_path):
    g = golden("grf2d_small")
    sim, idx = run_cli(g2s, tmp_path, g, ["-k", "1.2", "-n", "20", "-s", "100"], {})
    assert np.array_equal(idx.ravel(), g["idx"].ravel())
    assert np.array_equal(sim, g["sim"])


def test_cli_local_controls_equal_reference(g2s, gpu, tmp_path):
    g = golden("grf2d_ni")
    sim, idx = run_cli(g2s, tmp_path, g, ["-k", "1.2", "-s", "100", "-ni", "ni"], {"ni": (g["ni"], [0])})
    assert np.array_equal(idx.ravel(), g["idx"].ravel())


def test_cli_kernels_equal_oracle(g2s, gpu, oracle, tmp_path):
    g = golden("grf2d_kii")
    sim, idx = run_cli(g2s, tmp_path, g, ["-k", "1.2", "-n", "20", "-s", "100", "-ki", "k0", "k1", "-kii", "kii"],
                       {"k0": (g["k0"], [0]), "k1": (g["k1"], [0]), "kii": (g["kii"], [0])})
    o = oracle.simulate(g["ti"], g["di"], [0], 20, 1.2, 100, kii=g["kii"],
                        kernels=[(g["k0"], g["k0"].shape[::-1]), (g["k1"], g["k1"].shape[::-1])])
    assert np.array_equal(idx.ravel(), o["id"])


def test_cli_full_simulation_equals_reference(g2s, gpu, tmp_path):
    g = golden("grf2d_fs")
    sim, idx = run_cli(g2s, tmp_path, g, ["-k", "1.2", "-n", "20", "-s", "100", "-fs"], {})
    assert np.array_equal(idx.ravel(), g["idx"].ravel())
    assert np.array_equal(sim, g["sim"])


def test_auto_qs_cli_equals_calibrate(g2s, gpu, oracle, tmp_path):
    """auto_qs_b200 (the G2S auto_qs command line): im_1/2/3 images equal to the
    oracle's calibration for the same setups, seed and iteration counts."""
    from g2s_b200 import synthetic as syn
    exe = os.path.join(ROOT, "g2s_b200", "auto_qs_b200")
    ti = syn.grf((48, 48), (5, 5), seed=4)
    r = np.arange(9) - 4
    k = np.exp(-(r[:, None] ** 2 + r[None, :] ** 2) / 10.0).astype(np.float32)
    g2s.write_bgrid(str(tmp_path / "ti.bgrid"), ti, [0])
    g2s.write_bgrid(str(tmp_path / "k.bgrid"), k, [0])
    env = dict(os.environ, G2S_DATA_DIR=str(tmp_path))
    res = subprocess.run([exe, "-ti", "ti", "-ki", "k", "-maxk", "2", "-maxn", "8", "-densities", "0.1", "0.5",
                          "-maxIter", "20", "-minIter", "6", "-s", "9", "-id", "cal", "-W_CUDA", "0"],
                         capture_output=True, text=True, env=env, timeout=300)
    assert res.returncode == 0, res.stderr
    assert "compuattion time" in res.stderr
    m, _ = g2s.read_bgrid(str(tmp_path / "im_1_cal.bgrid"))
    d, _ = g2s.read_bgrid(str(tmp_path / "im_2_cal.bgrid"))
    n, _ = g2s.read_bgrid(str(tmp_path / "im_3_cal.bgrid"))
    om, od, on, _ = oracle.calibrate(ti, [0], [k], g2s.default_neighbour_counts(8), [0.1, 0.5], max_k=2, power=2.0,
                                     max_iter=20, min_iter=6, seed=9)
    assert np.array_equal(np.asarray(n).view(np.uint32).reshape(on.shape) if np.asarray(n).dtype == np.float32
                          else np.asarray(n).reshape(on.shape), on)
    assert np.array_equal(np.asarray(m).reshape(om.shape), om, equal_nan=True)
    assert np.array_equal(np.asarray(d).reshape(od.shape), od, equal_nan=True)


@pytest.mark.parametrize("name", ["multi_ti_ii", "multi_ti3"])
def test_cli_several_tis_equal_oracle(g2s, gpu, oracle, tmp_path, name):
    """-ti a b [c] (and -ii) on the batched engine: the simulation and the
    index image (TI cell * nTI + TI) equal the oracle's several-TI run."""
    g = golden(name)
    nti = int(g["nti"])
    types = [int(t) for t in g["types"]]
    tis = [g[f"ti{i}"] for i in range(nti)]
    for i, t in enumerate(tis):
        g2s.write_bgrid(str(tmp_path / f"ti{i}.bgrid"), t, types)
    g2s.write_bgrid(str(tmp_path / "di.bgrid"), g["di"], types)
    args = [EXE, "-ti"] + [f"ti{i}" for i in range(nti)] + ["-di", "di", "-k", str(float(g["k"])), "-n",
                                                              str(int(g["n"])), "-s", str(int(g["seed"])),
                                                              "-id", "job", "-W_CUDA", "0"]
    ii = g["ii"] if "ii" in g else None
    if ii is not None:
        g2s.write_bgrid(str(tmp_path / "ii.bgrid"), ii, [0])
        args += ["-ii", "ii"]
    r = subprocess.run(args, capture_output=True, text=True, env=dict(os.environ, G2S_DATA_DIR=str(tmp_path)),
                       timeout=300)
    assert r.returncode == 0, r.stderr
    sim, _ = g2s.read_bgrid(str(tmp_path / "job.bgrid"))
    idx, _ = g2s.read_bgrid(str(tmp_path / "id_job.bgrid"))
    o = oracle.simulate_multi(tis, g["di"], types, int(g["n"]), float(g["k"]), int(g["seed"]), ii=ii)
    assert np.array_equal(sim, o["sim"])
    assert np.array_equal(idx.ravel(), o["id"])
