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
