"""G2S .bgrid grids: the library's reader and writer against grids written by
the reference's own DataImage::write (tests/golden/ref_written*, made by
tests/golden/make_golden.py bgrid), round trips, and the command line's
argument checks (no GPU needed: it stops before any device work)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT


@pytest.mark.parametrize("ext", [".bgrid", ".bgrid.gz"])
def test_reads_reference_written_grids(g2s, ext):
    arr, types = g2s.read_bgrid(os.path.join(GOLDEN, "ref_written" + ext))
    want = np.load(os.path.join(GOLDEN, "ref_written_values.npy"))
    assert types == [0, 1]
    assert arr.shape == want.shape
    assert np.array_equal(arr, want, equal_nan=True)


@pytest.mark.parametrize("compress", [False, True])
def test_write_then_read(g2s, tmp_path, compress):
    rng = np.random.default_rng(5)
    a = rng.standard_normal((3, 4, 6)).astype(np.float32)
    p = str(tmp_path / ("g.bgrid.gz" if compress else "g.bgrid"))
    g2s.write_bgrid(p, a, [0], compress=compress)
    b, t = g2s.read_bgrid(p)
    assert t == [0] and np.array_equal(a, b)
    ix = rng.integers(0, 2 ** 32 - 1, (4, 5), dtype=np.uint32)
    q = str(tmp_path / "ix.bgrid")
    g2s.write_bgrid(q, ix, [0])
    c, _ = g2s.read_bgrid(q)
    assert c.dtype == np.uint32 and np.array_equal(c, ix)


def test_written_file_matches_reference_bytes(g2s, tmp_path):
    """Same serialised bytes as the reference for the same grid."""
    want = np.load(os.path.join(GOLDEN, "ref_written_values.npy"))
    p = str(tmp_path / "w.bgrid")
    g2s.write_bgrid(p, want, [0, 1])
    with open(p, "rb") as f, open(os.path.join(GOLDEN, "ref_written.bgrid"), "rb") as g:
        assert f.read() == g.read()


def test_rejects_truncated_grid(g2s, tmp_path):
    with open(os.path.join(GOLDEN, "ref_written.bgrid"), "rb") as f:
        raw = f.read()
    p = tmp_path / "bad.bgrid"
    p.write_bytes(raw[:-4])
    with pytest.raises(RuntimeError, match="not a valid"):
        g2s.read_bgrid(str(p))


def _cli():
    exe = os.path.join(ROOT, "g2s_b200", "qs_b200")
    if not os.path.exists(exe):
        pytest.fail("g2s_b200/qs_b200 is missing: python -m g2s_b200.build cli")
    return exe


def test_cli_rejects_unimplemented_flags(tmp_path):
    r = subprocess.run([_cli(), "-ti", "a", "-di", "c", "-n", "5", "-k", "1.2", "-csim"], capture_output=True, text=True)
    assert r.returncode == 1 and "-csim" in r.stderr


def test_cli_checks_several_training_images(g2s, tmp_path):
    """-ti a b: every training image must match the grid in dimensions and
    variables, and an -ii grid must have the simulation grid's cells."""
    env = dict(os.environ, G2S_DATA_DIR=str(tmp_path))
    g2s.write_bgrid(str(tmp_path / "a.bgrid"), np.zeros((8, 8), np.float32), [0])
    g2s.write_bgrid(str(tmp_path / "b.bgrid"), np.zeros((8, 8, 2), np.float32), [0, 0])
    g2s.write_bgrid(str(tmp_path / "c.bgrid"), np.full((6, 6), np.nan, np.float32), [0])
    g2s.write_bgrid(str(tmp_path / "ii.bgrid"), np.zeros((5, 5), np.float32), [0])
    r = subprocess.run([_cli(), "-ti", "a", "b", "-di", "c", "-n", "5", "-k", "1.2"], capture_output=True, text=True,
                       env=env)
    assert r.returncode == 1 and "differ in dimensions or variables" in r.stderr
    r = subprocess.run([_cli(), "-ti", "a", "a", "-di", "c", "-n", "5", "-k", "1.2", "-ii", "ii"], capture_output=True,
                       text=True, env=env)
    assert r.returncode == 1 and "-ii grid size" in r.stderr


def test_cli_reports_missing_grid(tmp_path):
    env = dict(os.environ, G2S_DATA_DIR=str(tmp_path))
    r = subprocess.run([_cli(), "-ti", "nothere", "-di", "c", "-n", "5", "-k", "1.2"], capture_output=True, text=True,
                       env=env)
    assert r.returncode == 1 and "not found" in r.stderr
