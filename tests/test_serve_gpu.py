"""GPU: the continuous-batching server. Every request's result -- in a mix of
k=10 and k=100 requests, 30% of them filtered, batched as they arrive onto
several streams -- must equal a search of that query alone, bit for bit."""

import numpy as np
import pytest

import nsparse
import oracle as O
from helpers import sq_spec
from nsparse_b200 import synth

pytestmark = pytest.mark.gpu

SPEC = "seismic,lambda=2000|beta=200|alpha=0.4|seed=7"


def corpus():
    docs = synth.docs_config0(20000, seed=21)
    qs = synth.queries_config2(400, seed=22)
    return docs, qs


def alone(idx, qs, i, k, cut, hf, bits=None, n_docs=0):
    p = nsparse.SeismicSearchParameters(cut, hf)
    if bits is not None:
        p.set_id_selector(nsparse.BitmapIDSelector(n_docs, bits))
    r = qs.rows(i, i + 1)
    return idx.search(1, r.indptr, r.indices, r.values, k, p)


def mixed_trace(qs, rng, rate_qps):
    k_per = np.where(rng.random(qs.n) < 0.5, 10, 100).astype(np.int32)
    filtered = rng.random(qs.n) < 0.3
    arrivals = np.cumsum(rng.exponential(1e6 / rate_qps, qs.n))
    return k_per, filtered, arrivals


@pytest.mark.parametrize("kind", ["fp32", "sq8"])
def test_mixed_requests_equal_searches_alone(kind):
    docs, qs = corpus()
    vmin, vmax = float(docs.values.min()), float(docs.values.max())
    spec = SPEC if kind == "fp32" else sq_spec(vmin, vmax, lam=2000, beta=200)
    idx = nsparse.index_factory(docs.dim, spec)
    idx.add(docs.n, docs.indptr, docs.indices, docs.values)
    idx.build()
    rng = np.random.default_rng(5)
    bits = O.bitmap_from_ids(docs.n, rng.choice(docs.n, docs.n // 10, replace=False))
    srv = nsparse.Server(idx, max_batch=48, slots=3)
    fid = srv.add_filter(bits)
    k_per, filtered, arrivals = mixed_trace(qs, rng, rate_qps=20000)
    fper = np.where(filtered, fid, -1).astype(np.int32)
    D, L, lat = srv.replay(qs.indptr, qs.indices, qs.values, k_per, arrivals, cut=12,
                           heap_factor=0.9, filter_per=fper)
    st = srv.stats()
    srv.close()
    assert st["requests"] == qs.n and st["batches"] > 1 and st["max_batch"] > 1
    assert (lat > 0).all()
    for i in range(qs.n):
        k = int(k_per[i])
        Da, La = alone(idx, qs, i, k, 12, 0.9, bits if filtered[i] else None, docs.n)
        np.testing.assert_array_equal(L[i, :k], La[0].astype(np.int64))
        np.testing.assert_array_equal(D[i, :k], Da[0])
        assert (L[i, k:] == -1).all()


def test_submit_wait_external_ids_and_tiny_budget():
    docs, qs = corpus()
    idx = nsparse.index_factory(docs.dim, SPEC)
    idx.add(docs.n, docs.indptr, docs.indices, docs.values)
    idx.build()
    rng = np.random.default_rng(9)
    ext = rng.integers(1 << 40, 1 << 62, docs.n, dtype=np.int64)
    # a budget below one request's bytes still admits one request per launch
    srv = nsparse.Server(idx, max_batch=8, slots=2, scratch_budget_bytes=64)
    srv.set_external_ids(ext)
    tickets = []
    for i in range(40):
        r = qs.rows(i, i + 1)
        tickets.append(srv.submit(r.indices, r.values, k=10, cut=10, heap_factor=0.8))
    for i, t in enumerate(tickets):
        d, l, lat = srv.wait(t)
        Da, La = alone(idx, qs, i, 10, 10, 0.8)
        np.testing.assert_array_equal(d, Da[0])
        want = np.where(La[0] >= 0, ext[np.maximum(La[0], 0)], -1)
        np.testing.assert_array_equal(l, want)
        assert lat > 0
    assert srv.stats()["max_batch"] == 1
    srv.close()
    with pytest.raises(ValueError):
        nsparse.Server(idx, max_batch=-1)
