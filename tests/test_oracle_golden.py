"""The CPU oracle against the G2S reference's own outputs (tests/golden,
generated by tests/golden/make_golden.py from the reference build)."""
import numpy as np
import pytest

from conftest import golden


@pytest.mark.parametrize("name", ["grf2d_small", "grf3d_small", "grf1d_small"])
def test_oracle_sequential_equals_reference(oracle, name):
    g = golden(name)
    types = [int(t) for t in g["types"]]
    out = oracle.simulate(g["ti"], g["di"], types, int(g["n"]), float(g["k"]), int(g["seed"]), mode=0)
    # continuous and mixed small cases: the reference's FFT rounding never
    # decides a draw here, so the whole simulation is identical
    assert np.array_equal(out["sim"], g["sim"])
    assert np.array_equal(out["id"], g["idx"].ravel())


@pytest.mark.parametrize("name", ["grf2d_small", "cat2d_small", "bivar2d_small", "grf3d_small", "grf2d_k3",
                                  "cat3_small", "grf1d_small", "bivar3d_small"])
def test_oracle_teacher_forced_outside_near_ties(oracle, name):
    g = golden(name)
    types = [int(t) for t in g["types"]]
    tf = oracle.simulate(g["ti"], g["sim"], types, int(g["n"]), float(g["k"]), int(g["seed"]), mode=1,
                         want_fp64=True, di_init=g["di"])
    order, seeds, post, begin = oracle.path(g["di"], len(types), int(g["seed"]))
    ref_cells = g["idx"].ravel()[order[begin:]]
    mismatch = tf["cell"] != ref_cells
    assert not np.any(mismatch & ~tf["near_tie"]), "draw differs from the reference outside near-ties"


def test_oracle_three_facies_weighted_kernel_outside_near_ties(oracle):
    """Three categories (codes 0, 1, 2) with a Gaussian -ki weight kernel:
    real-valued weights leave fewer match-score ties than unit weights, so
    a large share of the nodes is decided, and every decided node draws the
    reference's TI cell."""
    g = golden("cat3_ki")
    kern = g["kernel"]
    tf = oracle.simulate(g["ti"], g["sim"], [1], int(g["n"]), float(g["k"]), int(g["seed"]), mode=1,
                         want_fp64=True, di_init=g["di"], kernel=kern, kdims=kern.shape[::-1])
    order, seeds, post, begin = oracle.path(g["di"], 1, int(g["seed"]))
    ref_cells = g["idx"].ravel()[order[begin:]]
    decided = ~tf["near_tie"]
    assert decided.sum() > 0.3 * len(ref_cells)
    assert np.array_equal(tf["cell"][decided], ref_cells[decided])
    assert set(np.unique(g["sim"])) == {0.0, 1.0, 2.0}


def test_oracle_config0_prefix_teacher_forced(oracle):
    """Config 0 (200x200, n=50, k=1.2): first 1500 path nodes teacher-forced."""
    g = golden("config0")
    tf = oracle.simulate(g["ti"], g["sim"], [0], 50, 1.2, 100, mode=1, want_fp64=True, di_init=g["di"],
                         node_begin=0, node_end=1500)
    order, seeds, post, begin = oracle.path(g["di"], 1, 100)
    ref_cells = g["idx"].ravel()[order[begin:begin + 1500]]
    mismatch = tf["cell"] != ref_cells
    assert not np.any(mismatch & ~tf["near_tie"])
    fx = golden("config0_oracle_tf")
    assert np.array_equal(tf["cell"], fx["cell"][:1500])


def test_config0_fixture_near_ties_cover_all_mismatches():
    g = golden("config0")
    fx = golden("config0_oracle_tf")
    from oracle import qs_oracle as qo
    order, seeds, post, begin = qo.path(g["di"], 1, 100)
    ref_cells = g["idx"].ravel()[order[begin:]]
    mismatch = fx["cell"] != ref_cells
    assert mismatch.sum() <= fx["near_tie"].sum()
    assert not np.any(mismatch & ~fx["near_tie"])
    assert fx["near_tie"].mean() < 0.01


def test_reference_output_is_ti_values():
    for name in ["grf2d_small", "cat2d_small", "config0"]:
        g = golden(name)
        ti = g["ti"].reshape(-1)
        assert np.array_equal(ti[g["idx"].ravel()], g["sim"].ravel())


def local_kwargs(g):
    """Local controls stored in a fixture -> oracle / simulation keyword arguments."""
    kw = {}
    n = np.asarray(g["n"])
    if n.ndim > 0:
        kw["n_per_var"] = [int(x) for x in n]
    if "ni" in g:
        kw["ni"] = g["ni"]
    if "kvi" in g:
        kw["kvi"] = g["kvi"]
    if "kii" in g:
        kw["kii"] = g["kii"]
    return kw


def local_n(g):
    n = np.asarray(g["n"])
    return int(n.max()) if n.ndim > 0 else max(int(n), 0)


def local_kernels(g):
    if "kii" not in g:
        return {}
    return {"kernels": [(g["k0"], g["k0"].shape[::-1]), (g["k1"], g["k1"].shape[::-1])]}


@pytest.mark.parametrize("name", ["grf2d_ni", "grf2d_kvi"])
def test_oracle_local_controls_equal_reference(oracle, name):
    """-ni / -kvi / -kii with two -ki kernels: the whole simulation equals the
    reference's (these continuous cases have no near-tie on the path; the -kii
    cases have early near-ties and are checked teacher-forced below)."""
    g = golden(name)
    kw = local_kwargs(g)
    kw.update(local_kernels(g))
    out = oracle.simulate(g["ti"], g["di"], [0], local_n(g), float(g["k"]), int(g["seed"]), mode=0, **kw)
    assert np.array_equal(out["id"], g["idx"].ravel())
    assert np.array_equal(out["sim"], g["sim"])


@pytest.mark.parametrize("name", ["grf2d_ni", "grf2d_kvi", "grf2d_kii", "grf2d_local", "bivar2d_n2", "bivar2d_ni2"])
def test_oracle_local_controls_teacher_forced(oracle, name):
    """Every local-control case (-n n1 n2, -ni with one or two counts, -kvi,
    -kii): teacher-forced against the reference, identical outside FP64
    near-ties."""
    g = golden(name)
    types = [int(t) for t in g["types"]]
    tf = oracle.simulate(g["ti"], g["sim"], types, local_n(g), float(g["k"]), int(g["seed"]), mode=1,
                         want_fp64=True, di_init=g["di"], **local_kwargs(g), **local_kernels(g))
    order, seeds, post, begin = oracle.path(g["di"], len(types), int(g["seed"]))
    ref_cells = g["idx"].ravel()[order[begin:]]
    mismatch = tf["cell"] != ref_cells
    assert not np.any(mismatch & ~tf["near_tie"])
    assert mismatch.sum() <= 0.05 * mismatch.size


def full_kwargs(g):
    n = np.asarray(g["n"])
    return (int(n.max()), {"n_per_var": [int(x) for x in n]}) if n.ndim > 0 else (int(n), {})


def test_oracle_full_simulation_equals_reference(oracle):
    """-fs, one variable: the whole simulation equals the reference's."""
    g = golden("grf2d_fs")
    out = oracle.simulate(g["ti"], g["di"], [0], int(g["n"]), float(g["k"]), int(g["seed"]), full=True)
    assert np.array_equal(out["id"], g["idx"].ravel())
    assert np.array_equal(out["sim"], g["sim"])


@pytest.mark.parametrize("name", ["grf2d_fs", "bivar2d_fs", "bivar2d_fs_n2"])
def test_oracle_full_simulation_teacher_forced(oracle, name):
    """-fs teacher-forced on the reference's output: identical outside FP64
    near-ties (the bivariate cases have a categorical variable)."""
    g = golden(name)
    types = [int(t) for t in g["types"]]
    n, kw = full_kwargs(g)
    tf = oracle.simulate(g["ti"], g["sim"], types, n, float(g["k"]), int(g["seed"]), mode=1, want_fp64=True,
                         di_init=g["di"], full=True, **kw)
    order, seeds, post, begin = oracle.path(g["di"], len(types), int(g["seed"]), full=True)
    ref_cells = g["idx"].ravel()[order[begin:]]
    mismatch = tf["cell"] != ref_cells
    assert not np.any(mismatch & ~tf["near_tie"])
    assert mismatch.sum() <= 0.05 * mismatch.size
