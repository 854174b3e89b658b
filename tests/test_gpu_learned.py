"""Learned proposal: the encoder's FP32 forward and backward kernels against
the float64 CPU oracle (oracle/encoder_oracle.py), training on pairs the
exact path draws, and the learned map inside the simulation audited on the
plain path (regret), with and without training."""
import numpy as np
import pytest

from g2s_b200 import synthetic as syn
from oracle import encoder_oracle as eo

pytestmark = pytest.mark.gpu


def test_encoder_gradient_matches_oracle(g2s, gpu):
    """FP32 products on the CUDA cores: the gradient of every parameter
    block within 1e-3 (relative norm) of the float64 oracle."""
    enc = g2s.Encoder(nvar=2, seed=7).set_tensor_cores(False)
    assert enc.input_dim == 64 * 6
    w = enc.weights()
    rng = np.random.default_rng(1)
    B = 16
    xq = rng.standard_normal((B, enc.input_dim)).astype(np.float32)
    xp = (xq + 0.5 * rng.standard_normal(xq.shape)).astype(np.float32)
    loss, g = enc.loss_grad(xq, xp, tau=0.1)
    loss_ref, g_ref = eo.loss_grad(w.astype(np.float64), xq, xp, tau=0.1)
    assert abs(loss - loss_ref) <= 1e-4 * abs(loss_ref) + 1e-5
    off, n = eo.layout(enc.input_dim)
    assert g.size == n
    for b in range(eo.NBLOCKS):
        a, r = g[off[b]:off[b + 1]].astype(np.float64), g_ref[off[b]:off[b + 1]]
        rel = np.linalg.norm(a - r) / max(np.linalg.norm(r), 1e-12)
        assert rel < 1e-3, (b, rel)
    enc.close()


def test_encoder_embedding_matches_oracle_forward(g2s, gpu):
    enc = g2s.Encoder(nvar=1, seed=3).set_tensor_cores(False)
    x = np.random.default_rng(4).standard_normal((300, enc.input_dim)).astype(np.float32)
    for head in ("query", "pattern"):
        y = enc.embed(x, head)
        ref, _ = eo.forward(enc.weights().astype(np.float64), x, enc.input_dim, head)
        assert np.abs(y - ref).max() < 1e-4 * max(1.0, np.abs(ref).max())
    enc.close()


def test_encoder_tensor_cores_match_oracle_at_bf16_precision(g2s, gpu):
    """The default mode: every product on the tensor cores (operands rounded
    to BF16, FP32 accumulation).  Embeddings within 2 % of the largest
    float64 oracle value, the loss within 1 % and every parameter block's
    gradient within 5 % (relative norm): the rounding of BF16 operands,
    not a layout error (which is O(1))."""
    enc = g2s.Encoder(nvar=2, seed=7)
    w = enc.weights().astype(np.float64)
    rng = np.random.default_rng(1)
    x = rng.standard_normal((300, enc.input_dim)).astype(np.float32)
    for head in ("query", "pattern"):
        ref, _ = eo.forward(w, x, enc.input_dim, head)
        assert np.abs(enc.embed(x, head) - ref).max() < 2e-2 * np.abs(ref).max()
    B = 64
    xq = rng.standard_normal((B, enc.input_dim)).astype(np.float32)
    xp = (xq + 0.5 * rng.standard_normal(xq.shape)).astype(np.float32)
    loss, g = enc.loss_grad(xq, xp, tau=0.5)
    loss_ref, g_ref = eo.loss_grad(w, xq, xp, tau=0.5)
    assert abs(loss - loss_ref) <= 1e-2 * abs(loss_ref)
    off, n = eo.layout(enc.input_dim)
    for b in range(eo.NBLOCKS):
        a, r = g[off[b]:off[b + 1]].astype(np.float64), g_ref[off[b]:off[b + 1]]
        rel = np.linalg.norm(a - r) / max(np.linalg.norm(r), 1e-12)
        assert rel < 5e-2, (b, rel)
    enc.close()


def bivariate_ti(shape, seed):
    return syn.bivariate(syn.grf(shape, (6, 6), seed=seed))


def trained_encoder(g2s, epochs=30, tis=20):
    """An encoder trained on pairs drawn by the exact path on other TIs
    (seeds 1000+i), teacher-forced on completed grids of other seeds."""
    enc = g2s.Encoder(nvar=2, seed=11)
    for i in range(tis):
        ti = bivariate_ti((128, 128), 1000 + i)
        done = bivariate_ti((96, 96), 2000 + i)
        di = np.full(done.shape, np.nan, np.float32)
        sim = g2s.Simulation(ti, di, [0, 1], n=24, k=1.5, seed=5 + i)
        enc.add_pairs(sim, done, np.arange(96 * 96, dtype=np.int32))
        sim.close()
    assert enc.pairs() > 0.9 * tis * 96 * 96
    first = enc.train(epochs=1, batch=1024, lr=1e-3, tau=1.0, seed=1)
    last = enc.train(epochs=epochs - 1, batch=1024, lr=1e-3, tau=1.0, seed=2)
    return enc, first, last


def test_training_lowers_the_loss(g2s, gpu):
    enc, first, last = trained_encoder(g2s, epochs=12, tis=2)
    print(f"InfoNCE loss: first epoch {first:.3f}, after training {last:.3f}")
    assert last < 0.9 * first
    enc.close()


def run_learned(g2s, enc, ti, done, di):
    sim = g2s.Simulation(ti, di, [0, 1], n=24, k=1.5, seed=100)
    sim.set_learned(enc, shortlist=256, audit=1.0)
    sim.run_teacher(done)
    out = sim.read()
    info = sim.info()
    sim.close()
    return out, info


def test_learned_simulation_regret_and_what_training_gains(g2s, gpu):
    """On a TI it was not trained on: every node with neighbours is drawn by
    the proposal or, failing its confidence check, by the exact map; the
    plain path audits all of them (regret within 1 %).  The trained network
    passes the check for a large share of the nodes; the same network
    untrained (its proposal scores do not predict the exact scores) for
    almost none: what training gains is the share of nodes spared the full
    scan."""
    ti = bivariate_ti((128, 128), 1)
    done = bivariate_ti((64, 64), 2)
    di = np.full(done.shape, np.nan, np.float32)
    enc, _, _ = trained_encoder(g2s)
    raw = g2s.Encoder(nvar=2, seed=11)
    (_, _, cells), info = run_learned(g2s, enc, ti, done, di)
    (_, _, cells0), info0 = run_learned(g2s, raw, ti, done, di)
    conf = info["tensor_nodes"] - info["learned_fallback"]
    conf0 = info0["tensor_nodes"] - info0["learned_fallback"]
    for name, i in (("trained", info), ("untrained", info0)):
        print(f"{name}: {i['tensor_nodes'] - i['learned_fallback']} of {i['tensor_nodes']} proposal nodes confident, "
              f"regret {i['regret']} / {i['audited']} (+{i['regret_near']} near)")
    assert info["tensor_nodes"] > 0.9 * info["nodes"]
    assert info["regret"] <= 0.01 * info["audited"]
    assert info0["regret"] <= 0.01 * info0["audited"]
    assert conf > 0.2 * info["tensor_nodes"] and conf > 10 * max(conf0, 1)
    enc.close()
    raw.close()


def test_query_and_pattern_features_align(g2s, gpu):
    """The TI is the completed grid itself, so every node has a TI cell of
    mismatch 0 (its own) and the exact path (k = 1) draws a cell of mismatch
    0.  At stencil scale 1 the node's entries must then equal that cell's
    entries wherever the node has a neighbour: the node and TI-cell feature
    kernels read the same offsets, values and layout."""
    done = bivariate_ti((48, 48), 3)
    di = np.full(done.shape, np.nan, np.float32)
    enc = g2s.Encoder(nvar=2, seed=1).set_scales(1)
    sim = g2s.Simulation(done.copy(), di, [0, 1], n=16, k=1.0, seed=4)
    added = enc.add_pairs(sim, done, np.arange(48 * 48, dtype=np.int32))
    sim.close()
    q, p = enc.get_pairs()
    assert len(q) == added > 0.99 * 48 * 48
    q = q.reshape(len(q), 64, 6)
    p = p.reshape(len(p), 64, 6)
    mask = q[:, :, 2] > 0
    assert mask.sum() > 10 * len(q)
    assert np.all(p[:, :, 2][mask] == 1.0)
    assert np.array_equal(q[:, :, :2][mask], p[:, :, :2][mask])
    assert np.array_equal(q[:, :, 3:], p[:, :, 3:])   # entry offsets
    enc.close()
