"""Generate the golden fixtures of tests/golden/ from the G2S reference.

Runs the reference CPU QuickSampling (compiled from the G2S sources by
oracle/Makefile, FFTW replaced by the project FFT shim) on seeded synthetic
inputs and stores inputs + outputs (simulation grid, index image and the
reference's own reported compute time).  Needs oracle/_ref/libg2sref.so,
which is built only where the G2S sources are present:

    make -C oracle && python tests/golden/make_golden.py
    python tests/golden/make_golden.py multi     # several training images
    python tests/golden/make_golden.py kernel    # one -ki weight kernel
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402
from g2s_b200 import synthetic as syn  # noqa: E402

CASES = {
    # name: (ti builder, di shape, types, k, n, seed)
    "grf2d_small": (lambda: syn.grf((64, 64), (8, 8), seed=1), (40, 40), [0], 1.2, 20, 100),
    "cat2d_small": (lambda: syn.channels2d((80, 80), n_channels=6, seed=3), (40, 40), [1], 1.5, 20, 100),
    "bivar2d_small": (lambda: syn.bivariate(syn.grf((64, 64), (8, 8), seed=2), 0.7), (32, 32, 2), [0, 1], 1.2, 16, 7),
    "grf3d_small": (lambda: syn.grf((16, 20, 24), (5, 6, 6), seed=4), (8, 12, 12), [0], 1.2, 12, 11),
    "grf1d_small": (lambda: syn.grf((400,), (8,), seed=17), (150,), [0], 1.2, 10, 33),
    # 3-D bivariate (continuous + indicator), the kind of data of configuration 4
    "bivar3d_small": (lambda: syn.bivariate(syn.grf((16, 20, 24), (4, 6, 6), seed=23)), (8, 10, 12, 2), [0, 1],
                      1.5, 14, 41),
    "grf2d_k3": (lambda: syn.grf((48, 48), (6, 6), seed=5), (30, 30), [0], 3.0, 12, 3),
    # three facies (codes 0, 1, 2: a GRF cut at its terciles), categorical
    "cat3_small": (lambda: facies3(syn.grf((64, 64), (7, 7), seed=9)), (36, 36), [1], 1.5, 16, 21),
    # configuration 0: 200x200 GRF (range 12), unconditional 200x200, n=50, k=1.2, seed 100
    "config0": (lambda: syn.grf((200, 200), (12, 12), seed=1), (200, 200), [0], 1.2, 50, 100),
}

# cases with extra qs flags: name -> (ti builder, di shape, types, k, n, seed, extra flags)
EXTRA = {
    "grf2d_nv": (lambda: syn.grf((64, 64), (8, 8), seed=1), (40, 40), [0], 1.2, 20, 100, ["-nV"]),
    "grf2d_holes": (lambda: holes(syn.grf((64, 64), (8, 8), seed=6), seed=6), (40, 40), [0], 1.2, 20, 100, []),
    "grf2d_holes_nv": (lambda: holes(syn.grf((60, 70), (7, 7), seed=8), seed=8), (36, 44), [0], 1.5, 16, 5, ["-nV"]),
}


def _local_arrays(dshape, seed, what):
    """Seeded local-control images for a grid of numpy shape dshape."""
    rng = np.random.default_rng(seed)
    sp = dshape[:2]
    out = {}
    if "ni" in what:
        out["ni"] = rng.integers(3, 30, sp).astype(np.float32)
    if "ni2" in what:
        out["ni"] = np.stack([rng.integers(2, 20, sp), rng.integers(2, 20, sp)], -1).astype(np.float32)
    if "kvi" in what:
        out["kvi"] = rng.choice(np.array([1.0, 1.5, 2.0, 3.0, 0.0], np.float32), sp)
    if "kii" in what:
        out["k0"] = np.ones((15, 15), np.float32)
        yy, xx = np.meshgrid(np.arange(21) - 10, np.arange(21) - 10, indexing="ij")
        out["k1"] = np.exp(-np.hypot(yy, xx) / 4).astype(np.float32)
        out["kii"] = rng.integers(0, 2, sp).astype(np.float32)
    return out


# local controls (-n per variable, -ni, -kvi, -kii with a -ki list):
# name -> (ti builder, di shape, types, k, n (int or list), seed, images wanted)
LOCAL = {
    "grf2d_ni": (lambda: syn.grf((60, 70), (6, 6), seed=3), (24, 28), [0], 1.2, None, 100, ["ni"]),
    "grf2d_kvi": (lambda: syn.grf((60, 70), (6, 6), seed=3), (24, 28), [0], 1.2, 20, 100, ["kvi"]),
    "grf2d_kii": (lambda: syn.grf((60, 70), (6, 6), seed=3), (24, 28), [0], 1.2, 20, 100, ["kii"]),
    "grf2d_local": (lambda: syn.grf((60, 70), (6, 6), seed=3), (24, 28), [0], 1.2, None, 100, ["ni", "kvi", "kii"]),
    "bivar2d_n2": (lambda: syn.bivariate(syn.grf((60, 70), (6, 6), seed=5)), (20, 22, 2), [0, 1], 1.2, [12, 25], 100, []),
    "bivar2d_ni2": (lambda: syn.bivariate(syn.grf((60, 70), (6, 6), seed=5)), (20, 22, 2), [0, 1], 1.2, None, 100,
                    ["ni2"]),
}


# -fs (one path node per cell value): name -> (ti builder, di shape, types, k, n (int or list), seed)
FULL = {
    "grf2d_fs": (lambda: syn.grf((60, 70), (6, 6), seed=3), (24, 28), [0], 1.2, 20, 100),
    "bivar2d_fs": (lambda: syn.bivariate(syn.grf((60, 70), (6, 6), seed=5)), (16, 18, 2), [0, 1], 1.2, 15, 100),
    "bivar2d_fs_n2": (lambda: syn.bivariate(syn.grf((60, 70), (6, 6), seed=5)), (16, 18, 2), [0, 1], 1.2, [10, 20],
                      100),
}


def make_full(names=None):
    for name, (mk, dshape, types, k, n, seed) in FULL.items():
        if names and name not in names:
            continue
        ti = mk()
        di = np.full(dshape, np.nan, np.float32)
        args = ["-k", str(k), "-s", str(seed), "-j", "1", "-fs", "-n"] + [str(x) for x in np.ravel(n)]
        sim, idx, ms, _ = ref.run_qs(ti, di, types, args, job_id=3300 + len(name))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), ti=ti, di=di, types=np.array(types), k=k,
                            n=np.array(n), seed=seed, sim=sim, idx=idx, ref_ms=ms)
        print(name, ti.shape, dshape, idx.shape)


def make_bgrid():
    """Grids written by the reference's own DataImage::write (gzip and plain),
    copied out of its data directory, for the .bgrid reader tests."""
    import shutil
    rng = np.random.default_rng(12)
    a = rng.standard_normal((5, 7, 2)).astype(np.float32)
    a[1, 2, 0] = np.nan
    for compressed, ext in ((True, ".bgrid.gz"), (False, ".bgrid")):
        name = f"g2sb200_bgrid_{int(compressed)}"
        ref.write_image(name, a, [0, 1], compressed=compressed)
        src = os.path.realpath(f"/tmp/G2S/data/{name}{ext}")
        shutil.copyfile(src, os.path.join(HERE, f"ref_written{ext}"))
    np.save(os.path.join(HERE, "ref_written_values.npy"), a)
    print("bgrid fixtures", a.shape)


# one weight kernel (-ki): name -> (ti builder, di shape, types, k, n, seed, kernel builder).  Real-valued
# weights make categorical match scores rarely tie, so most nodes are decided
KERNEL = {
    "cat3_ki": (lambda: facies3(syn.grf((64, 64), (7, 7), seed=9)), (36, 36), [1], 1.5, 16, 21,
                lambda: gauss_kernel(15, 3.0)),
}


def gauss_kernel(size, sigma):
    r = np.arange(size) - size // 2
    yy, xx = np.meshgrid(r, r, indexing="ij")
    return np.exp(-(yy * yy + xx * xx) / (2.0 * sigma * sigma)).astype(np.float32)


def make_kernel(names=None):
    for name, (mk, dshape, types, k, n, seed, kmk) in KERNEL.items():
        if names and name not in names:
            continue
        ti = mk()
        di = np.full(dshape, np.nan, np.float32)
        kern = kmk()
        args = ["-k", str(k), "-n", str(n), "-s", str(seed), "-j", "1"]
        sim, idx, ms, _ = ref.run_qs(ti, di, types, args, images={"-ki": [(kern, [0])]}, job_id=3300 + len(name))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), ti=ti, di=di, types=np.array(types), k=k, n=n,
                            seed=seed, sim=sim, idx=idx, ref_ms=ms, kernel=kern)
        print(name, ti.shape, dshape, "kernel", kern.shape)


def make_local(names=None):
    for name, (mk, dshape, types, k, n, seed, what) in LOCAL.items():
        if names and name not in names:
            continue
        ti = mk()
        di = np.full(dshape, np.nan, np.float32)
        arrs = _local_arrays(dshape, seed + len(name), what)
        args = ["-k", str(k), "-s", str(seed), "-j", "1"]
        if n is not None:
            args += ["-n"] + [str(x) for x in np.ravel(n)]
        images = {}
        if "ni" in arrs:
            images["-ni"] = [(arrs["ni"], [0] * (1 if arrs["ni"].ndim == 2 else arrs["ni"].shape[-1]))]
        if "kvi" in arrs:
            images["-kvi"] = [(arrs["kvi"], [0])]
        if "kii" in arrs:
            images["-ki"] = [(arrs["k0"], [0]), (arrs["k1"], [0])]
            images["-kii"] = [(arrs["kii"], [0])]
        sim, idx, ms, _ = ref.run_qs(ti, di, types, args, images=images, job_id=3100 + len(name))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), ti=ti, di=di, types=np.array(types), k=k,
                            n=np.array(-1 if n is None else n), seed=seed, sim=sim, idx=idx, ref_ms=ms, **arrs)
        print(name, ti.shape, dshape, sorted(arrs))


def facies3(field):
    """Three categories: a continuous field cut at its terciles (codes 0, 1, 2)."""
    lo, hi = np.quantile(field, [1.0 / 3.0, 2.0 / 3.0])
    return np.where(field < lo, 0.0, np.where(field < hi, 1.0, 2.0)).astype(np.float32)


def holes(field, seed):
    """Missing training-image values: a few NaN rectangles."""
    rng = np.random.default_rng(seed)
    f = field.copy()
    ny, nx = f.shape
    for _ in range(6):
        y, x = rng.integers(0, ny - 8), rng.integers(0, nx - 8)
        f[y:y + int(rng.integers(2, 8)), x:x + int(rng.integers(2, 8))] = np.nan
    return f


def main(names=None):
    cases = {k: v + ([],) for k, v in CASES.items()}
    cases.update(EXTRA)
    for name, (mk, dshape, types, k, n, seed, extra) in cases.items():
        if names and name not in names:
            continue
        ti = mk()
        di = np.full(dshape, np.nan, np.float32)
        sim, idx, ms, _ = ref.run_qs(ti, di, types, ["-k", str(k), "-n", str(n), "-s", str(seed), "-j", "1"] + extra)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), ti=ti, di=di, types=np.array(types), k=k, n=n,
                            seed=seed, sim=sim, idx=idx, ref_ms=ms, nv=("-nV" in extra))
        print(name, ti.shape, dshape, "ref ms", ms)




# several training images in one run (-ti with more than one grid; -ii the TI
# index image): name -> (TI builders, di shape, types, k, n, seed, ii builder)
# TI shapes whose spectrum length ny*(nx/2+1) is a multiple of 8 (exact in the
# reference build)
MULTI = {
    "multi_ti": ([lambda: syn.grf((48, 48), (6, 6), seed=11), lambda: syn.grf((40, 40), (6, 6), seed=12)],
                 (32, 32), [0], 1.2, 12, 7, None),
    "multi_ti_ii": ([lambda: syn.grf((48, 48), (6, 6), seed=11), lambda: syn.grf((40, 40), (6, 6), seed=12)],
                    (32, 32), [0], 1.2, 12, 7, lambda: np.repeat((np.arange(32) >= 16)[None, :], 32, 0)),
    # equal sizes: the reference CPU device's unnormalised scores (N x S)
    # share one N, so its merge orders candidates as the true scores do
    "multi_ti_eq": ([lambda: syn.grf((48, 48), (6, 6), seed=11), lambda: syn.grf((48, 48), (6, 6), seed=13)],
                    (32, 32), [0], 1.5, 12, 8, None),
    "multi_ti3": ([lambda: syn.grf((40, 40), (5, 5), seed=13), lambda: syn.grf((48, 48), (5, 5), seed=14),
                   lambda: syn.grf((32, 32), (5, 5), seed=15)], (30, 30), [0], 2.5, 10, 9, None),
}


def make_multi(names=None):
    """The reference `qs` with several `-ti` grids (and `-ii`): its cross-TI
    merge of the per-TI k best (quantileSamplingModule.hpp:90-126) and
    index image `index * nTI + TI` (simulation.hpp:658)."""
    for name, (mks, dshape, types, k, n, seed, mkii) in MULTI.items():
        if names and name not in names:
            continue
        tis = [mk() for mk in mks]
        di = np.full(dshape, np.nan, np.float32)
        images = {"-ti": [(t, types) for t in tis[1:]]}
        ii = None
        if mkii is not None:
            ii = mkii().astype(np.float32)
            images["-ii"] = [(ii, [0])]
        sim, idx, ms, _ = ref.run_qs(tis[0], di, types, ["-k", str(k), "-n", str(n), "-s", str(seed), "-j", "1"],
                                     images=images)
        extra = {f"ti{i}": t for i, t in enumerate(tis)}
        if ii is not None:
            extra["ii"] = ii
        np.savez_compressed(os.path.join(HERE, name + ".npz"), di=di, types=np.array(types), k=k, n=n, seed=seed,
                            nti=len(tis), sim=sim, idx=idx, ref_ms=ms, **extra)
        print(name, [t.shape for t in tis], dshape, "from TI", np.bincount((idx.ravel() % len(tis)).astype(int)))


def oracle_teacher_config0():
    """Teacher-forced oracle evaluation of every config-0 path node against the
    reference's completed grid: chosen TI cell and FP64 near-tie flag."""
    from oracle import qs_oracle as qo
    g = np.load(os.path.join(HERE, "config0.npz"))
    di = g["di"]
    tf = qo.simulate(g["ti"], g["sim"], [0], int(g["n"]), float(g["k"]), int(g["seed"]), mode=1, want_fp64=True,
                     di_init=di)
    np.savez_compressed(os.path.join(HERE, "config0_oracle_tf.npz"), cell=tf["cell"], near_tie=tf["near_tie"],
                        gap=tf["gap"].astype(np.float32))
    print("config0 oracle teacher-forced: near-ties", int(tf["near_tie"].sum()))


if __name__ == "__main__":
    args = sys.argv[1:]
    if args == ["teacher"]:
        oracle_teacher_config0()
    elif args[:1] == ["local"]:
        make_local(args[1:])
    elif args[:1] == ["full"]:
        make_full(args[1:])
    elif args == ["bgrid"]:
        make_bgrid()
    elif args[:1] == ["multi"]:
        make_multi(args[1:])
    elif args[:1] == ["kernel"]:
        make_kernel(args[1:])
    else:
        main(args)
