"""The launch autotuner (sfb200.autotune) against a simulated plan on the CPU: it applies and caches
the fastest candidate, skips candidates the library refuses, and its cache round-trips a file."""
import numpy as np
import pytest

from sfb200 import _abi, autotune
from sfb200.api import plan_description
from sfb200 import synthetic


class FakePlan:
    """set_launch / set_option / stats like _lib.Plan; the 'kernel time' depends on the launch."""

    def __init__(self, refuse=()):
        self.launch = (0, -1, 0)
        self.order = -1
        self.refuse = set(refuse)
        self.runs = 0

    def set_launch(self, tile, priv, bps):
        if (tile, priv) in self.refuse:
            raise ValueError("refused")
        self.launch = (tile, priv, bps)

    def set_option(self, opt, value):
        assert opt == _abi.OPT_POINT_ORDER
        self.order = value

    def ms(self):
        tile, priv, _ = self.launch
        return 10.0 - (tile == 256) * 2.0 - (priv == 3) * 3.0 - (self.order == -1) * 1.0

    def stats(self):
        return {"kernel_ms": self.ms()}

    def run(self):
        self.runs += 1


def desc_of(name="c1", n=4000):
    w = synthetic.config(name, n=n)
    d, keep = plan_description(w.ops, w.u.shape[0], w.distance_bins, w.value_bins, w.metric, "mixed", w.x.dtype,
                               w.u.dtype)
    return d, keep


def test_picks_and_caches_the_fastest_candidate():
    autotune.clear()
    d, keep = desc_of()
    p = FakePlan()
    r = autotune.tune(p, d, p.run, 4000)
    assert r["choice"] == (256, 3, -1)
    assert (p.launch[:2], p.order) == ((256, 3), -1)
    assert autotune.lookup(autotune.shape_key(d, 4000)) == (256, 3, -1)
    assert len(r["timings"]) == len(autotune.CANDIDATES_1D)
    assert p.runs == len(autotune.CANDIDATES_1D) * 3  # one warm-up and two timed runs each


def test_refused_candidates_are_skipped():
    autotune.clear()
    d, keep = desc_of()
    p = FakePlan(refuse={(256, 3)})
    r = autotune.tune(p, d, p.run, 4000)
    assert r["choice"] == (128, 3, -1)


def test_shape_key_separates_size_classes_and_joint():
    d, _ = desc_of("c1", 4000)
    dj, _ = desc_of("c3", 3000)
    assert autotune.shape_key(d, 4000) == autotune.shape_key(d, 4090)   # same log2 class
    assert autotune.shape_key(d, 4000) != autotune.shape_key(d, 40000)
    assert autotune.shape_key(d, 4000) != autotune.shape_key(dj, 4000)


def test_cache_file_round_trip(tmp_path):
    autotune.clear()
    d, _ = desc_of()
    p = FakePlan()
    autotune.tune(p, d, p.run, 4000)
    f = tmp_path / "tune.json"
    autotune.save(str(f))
    autotune.clear()
    assert autotune.lookup(autotune.shape_key(d, 4000)) is None
    autotune.load(str(f))
    assert autotune.lookup(autotune.shape_key(d, 4000)) == (256, 3, -1)
