"""Autotuner host logic on the CPU: the coordinate search picks the fastest
candidate whose regret audit passes, audits only candidates that would
replace the best, and the JSON cache answers a tuned shape without a GPU."""
import numpy as np

from g2s_b200 import autotune as at


def fake_run(times, regret_of=lambda p: 0, auto_prefix=512):
    calls = []

    def run(p, audit):
        calls.append((dict(p), audit))
        prefix = p["prefix"] or auto_prefix
        width = p["width"] or 8
        r = {"ms": times(width, prefix, p["batch"]), "prefix": prefix}
        if audit:
            r.update(regret=regret_of(dict(p, width=width, prefix=prefix)), audited=1000)
        return r
    return run, calls


def test_search_finds_the_fastest_passing_candidate():
    # fastest overall: width 32, prefix 256, batch 8192; width 32 fails the audit
    def times(w, t, b):
        return 100.0 - {8: 0, 16: 10, 32: 20}[w] - {64: 1, 128: 2, 256: 5, 512: 0, 1024: -5}[t] - {2048: -3, 4096: 0, 8192: 4}[b]
    run, calls = fake_run(times, regret_of=lambda p: 5 if p["width"] == 32 else 0)
    res = at.search(run, max_regret=0.0)
    assert (res["width"], res["prefix"], res["batch"]) == (16, 256, 8192)
    assert res["ok"] and res["regret"] == 0
    assert res["ms"] == times(16, 256, 8192)
    # audits only for the automatic choice and the candidates that became the best
    assert len([p for p, a in calls if a]) <= 7


def test_search_keeps_the_automatic_choice_when_nothing_is_faster():
    run, _ = fake_run(lambda w, t, b: 1.0 + 0.01 * (w != 8) + 0.01 * (t != 512) + 0.01 * (b != 4096))
    res = at.search(run)
    assert (res["width"], res["prefix"], res["batch"]) == (0, 512, 4096)
    assert res["ok"]


def test_regret_budget_is_a_fraction_of_the_audited_nodes():
    run, _ = fake_run(lambda w, t, b: 10.0 - w, regret_of=lambda p: 3 if p["width"] == 32 else 0)
    assert at.search(run, max_regret=0.0)["width"] == 16
    run, _ = fake_run(lambda w, t, b: 10.0 - w, regret_of=lambda p: 3 if p["width"] == 32 else 0)
    assert at.search(run, max_regret=0.005)["width"] == 32


def test_cache_roundtrip_answers_without_a_gpu(tmp_path):
    path = str(tmp_path / "t" / "tune.json")
    ti = np.zeros((64, 64), np.float32)
    key = at.shape_key(ti.shape, [0], 40, 1.2, "bf16", "TestGPU")
    at.save(path, {key: {"width": 16, "prefix": 256, "batch": 2048, "ms": 1.5}})
    res = at.tune(ti, [0], 40, 1.2, cache=path, device_name="TestGPU")
    assert res["cached"] and (res["width"], res["prefix"], res["batch"]) == (16, 256, 2048)
    assert at.load(str(tmp_path / "missing.json")) == {}
    other = at.shape_key(ti.shape, [0], 60, 1.2, "bf16", "TestGPU")
    assert other != key


def test_a_failing_automatic_choice_is_replaced_by_a_passing_candidate():
    # the automatic choice (width 8) is fastest but fails; width 16 passes
    run, _ = fake_run(lambda w, t, b: float(w), regret_of=lambda p: 9 if p["width"] == 8 else 0)
    res = at.search(run, max_regret=0.0)
    assert res["width"] == 16 and res["ok"]
