"""The encoder oracle (oracle/encoder_oracle.py) against central finite
differences: the hand-written float64 gradient of the symmetric InfoNCE loss
is the reference the GPU's backward kernels are checked against, so it is
checked first, on random weights and inputs (CPU only)."""
import numpy as np

from oracle import encoder_oracle as eo


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    D0 = 64 * 5
    w = eo.init_weights(D0, seed=1)
    B = 6
    xq = rng.standard_normal((B, D0))
    xp = xq + 0.3 * rng.standard_normal((B, D0))
    loss, g = eo.loss_grad(w, xq, xp, tau=0.1)
    assert np.isfinite(loss) and loss > 0
    off, n = eo.layout(D0)
    # a few coordinates of every parameter block
    picks = np.concatenate([rng.integers(off[b], off[b + 1], 4) for b in range(eo.NBLOCKS)])
    h = 1e-6
    for i in picks:
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (eo.loss_grad(wp, xq, xp, tau=0.1)[0] - eo.loss_grad(wm, xq, xp, tau=0.1)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_oracle_positive_pairs_lower_the_loss():
    rng = np.random.default_rng(2)
    D0 = 64 * 6
    w = eo.init_weights(D0, seed=3)
    x = rng.standard_normal((16, D0))
    same, _ = eo.loss_grad(w, x, x, tau=0.05)
    other, _ = eo.loss_grad(w, x, rng.standard_normal((16, D0)), tau=0.05)
    assert same < other
