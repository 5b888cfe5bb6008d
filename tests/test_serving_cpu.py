"""Host logic of the serving loop that needs no GPU: the Poisson trace, the
warm-up trace, the latency summary and the OR-join argument check."""
import types

import numpy as np
import pytest

from yallasql_b200 import serving


def fake_catalog(ntables=8):
    return types.SimpleNamespace(ntables=ntables)


def test_trace_is_seeded_and_follows_the_mix():
    cat = fake_catalog()
    a = serving.make_trace(4000, 500.0, cat, seed=4)
    b = serving.make_trace(4000, 500.0, cat, seed=4)
    assert [(r.klass, r.table, r.param, r.arrival) for r in a] == [(r.klass, r.table, r.param, r.arrival) for r in b]
    counts = {k: sum(r.klass == k for r in a) / len(a) for k in serving.CLASSES}
    for k, p in zip(serving.CLASSES, serving.MIX):
        assert abs(counts[k] - p) < 0.03
    gaps = np.diff([r.arrival for r in a])
    assert (gaps >= 0).all() and abs(gaps.mean() - 1 / 500.0) < 0.2 / 500.0
    burst = serving.make_trace(50, 0.0, cat, seed=4)
    assert all(r.arrival == 0.0 for r in burst)


def test_warm_trace_covers_every_class_and_table():
    cat = fake_catalog(5)
    w = serving.warm_trace(cat)
    assert {(r.klass, r.table) for r in w} == {(k, t) for k in serving.CLASSES for t in range(5)}
    assert len({r.rid for r in w}) == len(w)
    assert all(r.arrival == 0.0 for r in w)


def test_summary_latencies():
    reqs = [serving.Request(i, "filter", 0, arrival=0.01 * i) for i in range(100)]
    for i, r in enumerate(reqs):
        r.done = r.arrival + (0.002 if i < 99 else 0.5)
    s = serving.summary(reqs)
    assert s["queries"] == 100
    assert s["p50_ms"] == pytest.approx(2.0)
    assert s["p99_ms"] > 2.0 and s["mean_ms"] == pytest.approx((99 * 2.0 + 500.0) / 100)
    assert s["span_s"] == pytest.approx(0.99 + 0.5)


def test_or_join_groups_must_match_conditions():
    from yallasql_b200 import ops
    with pytest.raises(ValueError):
        ops._disjunct([0, 1, 1], [(0, 0, 0), (1, 1, 0)])
    arr = ops._disjunct([0, 1], [(0, 0, 0), (1, 1, 0)])
    assert list(arr) == [0, 1]
