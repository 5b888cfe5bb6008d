"""Serving form: every request's result is the same when it runs alone (plain
form, one request at a time) and when it runs in the mix (continuous
batching: overlapping streams, co-launched filter requests, staged
subqueries). Float SUM/AVG are compared at 1e-6 relative; everything else
exactly."""
import copy

import pytest
import torch

from yallasql_b200 import serving

pytestmark = pytest.mark.gpu

REL = 1e-6


def close(a, b):
    if a is None or b is None:
        return a is None and b is None
    if isinstance(a, float) or isinstance(b, float):
        return abs(a - b) <= REL * max(1.0, abs(a))
    return a == b


@pytest.mark.parametrize("share", [True, False])
@pytest.mark.parametrize("rate", [0.0, 2000.0])
def test_results_same_alone_and_in_mix(cuda, rate, share):
    """With `share`, identical pending requests ride on one dispatch, filter
    requests on one table share a scan and ORDER BY reuses a table's resident
    permutation: every request's result is still the one it gets alone."""
    cat = serving.Catalog(ntables=4, lo=1_000, hi=200_000, seed=4)
    plans = serving.Plans()
    trace = serving.make_trace(80, rate, cat, seed=4)
    alone = copy.deepcopy(trace)
    serving.serve_plain(alone, cat, plans, keep=True)
    mixed = copy.deepcopy(trace)
    stats = serving.serve_continuous(mixed, cat, plans, slots=4, keep=True, share=share)
    assert stats["queries"] == len(trace)
    seen = set()
    for a, m in zip(alone, mixed):
        assert a.rid == m.rid and a.klass == m.klass
        seen.add(a.klass)
        if a.klass in ("filter", "join"):
            assert len(a.result) == len(m.result)
            assert all(close(x, y) for x, y in zip(a.result, m.result)), (a.rid, a.result, m.result)
        elif a.klass == "order":
            for ca, cm in zip(a.result.columns, m.result.columns):
                assert torch.equal(ca.data, cm.data)
        else:
            assert a.result[0] == m.result[0]
            assert torch.equal(a.result[1], m.result[1]) and torch.equal(a.result[2], m.result[2])
        assert m.done >= m.arrival
    assert seen == set(serving.CLASSES)


def test_slot_buffers_reused_across_requests(cuda):
    """Without keep, ORDER BY and subquery requests write into their slot's
    reused buffers; the counts and aggregates still match the plain form."""
    cat = serving.Catalog(ntables=4, lo=1_000, hi=200_000, seed=6)
    plans = serving.Plans()
    trace = serving.make_trace(80, 0.0, cat, seed=6)
    alone = copy.deepcopy(trace)
    serving.serve_plain(alone, cat, plans)
    mixed = copy.deepcopy(trace)
    serving.serve_continuous(mixed, cat, plans, slots=4)
    for a, m in zip(alone, mixed):
        if a.klass in ("filter", "join"):
            assert all(close(x, y) for x, y in zip(a.result, m.result)), (a.rid, a.result, m.result)
        else:
            assert a.result == m.result, (a.rid, a.result, m.result)
    assert len(cat._slots) == 4 and any(b._order is not None for b in cat._slots.values())
