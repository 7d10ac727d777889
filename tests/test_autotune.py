"""The serving autotuner's choice, budget and cache logic (CPU; a fake timing function stands in
for the device), and its key on a real map."""

import json

import numpy as np
import pytest

import h2factory_b200 as h2
from h2factory_b200 import autotune, methods
from h2factory_b200.trees import build_tree


def _core(p=3, maxvalues=24, precision="fp32"):
    rng = np.random.default_rng(0)
    tree = build_tree(rng.random((600, 3)), maxvalues=maxvalues, root_center=[0.5] * 3, root_halfsize=0.5)
    return methods.interpolation_core(tree, methods.laplace, p, precision=precision)


class FakeDevice:
    """Throughput grows with the block and saturates; latency grows with block x in-flight."""

    def __init__(self):
        self.calls = 0

    def __call__(self, core, block, inflight):
        self.calls += 1
        rate = 1000.0 * block / (1.0 + 0.05 * block) * (1.0 + 0.1 * (inflight - 1))
        p99 = 0.5 * block * inflight
        return rate, p99


def test_key_of_real_map():
    core = _core(p=3, maxvalues=24, precision="fp32")
    k = autotune.key_of(core, 16)
    assert k.order == 3 and k.nrhs == 16 and k.dtype == "fp32/real"
    counts = np.diff(core.test.value_ptr)
    assert k.leaf_size == counts.max() <= 24


def test_choice_budget_and_ties():
    core = _core()
    dev = FakeDevice()
    t = autotune.Autotuner(measure=dev)
    best = t.choose(core, 16, blocks=(1, 2, 4, 8, 16, 32), inflight=(1, 2))
    assert (best["block"], best["inflight"]) == (16, 2)  # 32 exceeds the clients' 16
    assert len(best["trials"]) == 5 * 2 and best["budget_met"]
    capped = t.choose(core, 16, blocks=(1, 2, 4, 8, 16), inflight=(1, 2), p99_budget_ms=4.0)
    assert capped["p99_ms"] <= 4.0 and (capped["block"], capped["inflight"]) == (8, 1)
    none = t.choose(core, 16, blocks=(4, 8), inflight=(1,), p99_budget_ms=0.1)
    assert not none["budget_met"] and none["block"] == 4  # lowest latency when nothing fits
    with pytest.raises(ValueError):
        t.choose(core, 1, blocks=(2, 4))


def test_cache_is_reused_across_tuners(tmp_path):
    core = _core()
    path = str(tmp_path / "tune.json")
    dev = FakeDevice()
    a = autotune.Autotuner(cache_path=path, measure=dev).choose(core, 8, blocks=(2, 4, 8), inflight=(1, 2))
    n = dev.calls
    saved = json.load(open(path))
    assert len(saved) == 1 and list(saved.values())[0]["block"] == a["block"]
    b = autotune.Autotuner(cache_path=path, measure=dev).choose(core, 8, blocks=(2, 4, 8), inflight=(1, 2))
    assert dev.calls == n and b["block"] == a["block"] and b["inflight"] == a["inflight"]
    # another shape (order) is another key: measured again
    autotune.Autotuner(cache_path=path, measure=dev).choose(_core(p=4), 8, blocks=(2, 4, 8), inflight=(1, 2))
    assert dev.calls > n and len(json.load(open(path))) == 2


def test_server_params():
    core = _core()
    p = autotune.Autotuner(measure=FakeDevice()).server_params(core, 8, blocks=(1, 8), inflight=(1, 3))
    assert p == {"max_block": 8, "slots": 3}
