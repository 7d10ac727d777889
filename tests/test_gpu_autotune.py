"""The serving autotuner timing candidates on the device (GPU): a choice among the candidates,
recorded in the cache file, with blocks of several right-hand sides faster per right-hand side
than single ones on a launch-bound small map."""

import json

import pytest

from h2factory_b200 import autotune
from test_gpu_parity import CASES

pytestmark = pytest.mark.gpu


def test_autotune_on_device(tmp_path):
    core = CASES["toeplitz-laplace"]()
    path = str(tmp_path / "tune.json")
    t = autotune.Autotuner(cache_path=path,
                           measure=lambda c, b, f: autotune.measure_on_device(c, b, f, steps=6, warmup=2))
    c = t.choose(core, 8, blocks=(1, 4, 8), inflight=(1, 2))
    assert (c["block"], c["inflight"]) in {(b, f) for b in (1, 4, 8) for f in (1, 2)}
    rates = {(tr["block"], tr["inflight"]): tr["rhs_per_s"] for tr in c["trials"]}
    assert all(r > 0 for r in rates.values())
    assert rates[(8, 1)] > rates[(1, 1)]
    assert json.load(open(path))[autotune.key_of(core, 8).text()]["block"] == c["block"]
