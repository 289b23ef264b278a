"""GPU: the batched SEISMIC search step captured as a CUDA graph
(nsp_search_graph_*). Every replay must return what the ordinary search
returns, bit for bit (for fp32 the reference's own golden results) -- through
host buffers and through device buffers the caller binds -- and the graph must
refuse to run on an index changed since its capture."""

import numpy as np
import pytest
import torch

import nsparse
from helpers import CUT, HF, K, SEISMIC, golden, golden_corpus, sq_spec

pytestmark = pytest.mark.gpu


def built(spec):
    docs, qs = golden_corpus()
    idx = nsparse.index_factory(docs.dim, spec)
    idx.add(docs.n, docs.indptr, docs.indices, docs.values)
    idx.build()
    return idx, docs, qs


def max_row(qs):
    return int(np.diff(qs.indptr).max())


def expected(kind):
    """The index and the results the graph must reproduce: for fp32 the
    reference's golden results; for SQ the ordinary search's (uint8 scores
    tie often and the reference orders ties by unspecified library
    internals, so its golden rows pin SQ only through the oracle, ties by
    lower id, which the ordinary search matches in the search tests)."""
    g = golden()
    params = nsparse.SeismicSearchParameters(CUT, HF)
    if kind == "fp32":
        idx, docs, qs = built(SEISMIC)
        D0, L0 = idx.search(qs.n, qs.indptr, qs.indices, qs.values, K, params)
        np.testing.assert_array_equal(L0, g["seismic_L"])
        np.testing.assert_array_equal(D0, g["seismic_D"])
    else:
        idx, docs, qs = built(sq_spec(g["sq_vmin"], g["sq_vmax"]))
        D0, L0 = idx.search(qs.n, qs.indptr, qs.indices, qs.values, K, params)
    return idx, docs, qs, params, D0, L0


@pytest.mark.parametrize("kind", ["fp32", "sq8"])
def test_graph_replays_match_reference_golden(kind):
    idx, docs, qs, params, want_D, want_L = expected(kind)
    docs_scored = nsparse.last_search_stats().docs_scored

    graph = nsparse.SearchGraph(idx, qs.n, qs.nnz, max_row(qs), K, params)
    for _ in range(3):  # replays of the same step
        D, L = graph.search(qs.n, qs.indptr, qs.indices, qs.values)
        np.testing.assert_array_equal(L, want_L)
        np.testing.assert_array_equal(D, want_D)
        st = nsparse.last_search_stats()
        assert st.docs_scored == docs_scored and st.launches == 1
    # a smaller batch: the graph's other rows are empty and unread
    part = qs.rows(10, 47)
    D, L = graph.search(part.n, part.indptr, part.indices, part.values)
    np.testing.assert_array_equal(L, want_L[10:47])
    np.testing.assert_array_equal(D, want_D[10:47])
    # rows arrive in any term order, as the ordinary search takes them
    r = qs.rows(3, 4)
    perm = np.arange(r.nnz)[::-1]
    D, L = graph.search(1, r.indptr, r.indices[perm], r.values[perm])
    np.testing.assert_array_equal(L[0], want_L[3])
    np.testing.assert_array_equal(D[0], want_D[3])
    graph.close()


def test_graph_with_selector_matches_reference_golden():
    g = golden()
    idx, docs, qs = built(SEISMIC)
    p = nsparse.SeismicSearchParameters(CUT, HF)
    p.set_id_selector(nsparse.SetIDSelector(g["filter_ids"]))
    graph = nsparse.SearchGraph(idx, qs.n, qs.nnz, max_row(qs), K, p)
    D, L = graph.search(qs.n, qs.indptr, qs.indices, qs.values)
    np.testing.assert_array_equal(L, g["filter_L"])
    np.testing.assert_array_equal(D, g["filter_D"])
    # the exact-match path (a selector of at most k ids) is not a graph step
    p2 = nsparse.SeismicSearchParameters(CUT, HF)
    p2.set_id_selector(nsparse.SetIDSelector(g["exact_ids"]))
    with pytest.raises(ValueError):
        nsparse.SearchGraph(idx, 4, qs.nnz, max_row(qs), K, p2)


@pytest.mark.parametrize("kind", ["fp32", "sq8"])
def test_graph_on_caller_device_buffers(kind):
    idx, docs, qs, params, want_D, want_L = expected(kind)
    dev = torch.device("cuda", 0)
    n, cap = qs.n, qs.nnz + 64
    ip = torch.zeros(n + 1, dtype=torch.int32, device=dev)
    ix = torch.zeros(cap, dtype=torch.int16, device=dev)
    vv = torch.zeros(cap, dtype=torch.float32, device=dev)
    d = torch.full((n, K), 7.0, dtype=torch.float32, device=dev)
    lab = torch.full((n, K), 7, dtype=torch.int32, device=dev)
    bufs = {"indptr": ip.data_ptr(), "indices": ix.data_ptr(), "values": vv.data_ptr(),
            "distances": d.data_ptr(), "labels": lab.data_ptr()}
    graph = nsparse.SearchGraph(idx, n, cap, max_row(qs), K, params, device_buffers=bufs)
    assert graph.buffers() == bufs
    stream = torch.cuda.Stream(device=dev)
    with torch.cuda.stream(stream):
        # two different batches through the same buffers: the second half of
        # the queries first, then all of them
        for lo in (n // 2, 0):
            sub = qs.rows(lo, n)
            rows = np.concatenate([sub.indptr, np.full(n - sub.n, sub.indptr[-1])])
            ip.copy_(torch.from_numpy(rows.astype(np.int32)))
            ix[:sub.nnz].copy_(torch.from_numpy(sub.indices.view(np.int16)))
            vv[:sub.nnz].copy_(torch.from_numpy(sub.values))
            graph.launch(stream.cuda_stream)
            graph.sync(stream.cuda_stream)
            np.testing.assert_array_equal(lab.cpu().numpy()[:sub.n], want_L[lo:])
            np.testing.assert_array_equal(d.cpu().numpy()[:sub.n], want_D[lo:])
            # rows past the batch are empty queries: padding
            assert (lab.cpu().numpy()[sub.n:] == -1).all()
    graph.close()


def test_graph_refuses_changed_index_and_bad_arguments():
    idx, docs, qs = built(SEISMIC)
    params = nsparse.SeismicSearchParameters(CUT, HF)
    graph = nsparse.SearchGraph(idx, 8, qs.nnz, max_row(qs), K, params)
    part = qs.rows(0, 8)
    graph.search(part.n, part.indptr, part.indices, part.values)
    with pytest.raises(ValueError):  # more rows than the graph holds
        graph.search(qs.n, qs.indptr, qs.indices, qs.values)
    short = nsparse.SearchGraph(idx, 8, qs.nnz, 2, K, params)
    with pytest.raises(ValueError):  # a row longer than max_row_nnz
        short.search(part.n, part.indptr, part.indices, part.values)
    short.close()
    plain = nsparse.SeismicSearchParameters(CUT, HF)
    plain.set_engine(plain=True)
    with pytest.raises(ValueError):
        nsparse.SearchGraph(idx, 8, qs.nnz, max_row(qs), K, plain)
    idmap = nsparse.index_factory(docs.dim, "idmap," + SEISMIC)
    idmap.add_with_ids(docs.n, docs.indptr, docs.indices, docs.values,
                       np.arange(docs.n, dtype=np.int32))
    idmap.build()
    with pytest.raises(ValueError):
        nsparse.SearchGraph(idmap, 8, qs.nnz, max_row(qs), K, params)
    # added docs make the device copy stale, and the next search replaces it:
    # the graph must be recaptured
    more = docs.rows(0, 5)
    idx.add(more.n, more.indptr, more.indices, more.values)
    with pytest.raises(RuntimeError):
        graph.search(part.n, part.indptr, part.indices, part.values)
    idx.search(part.n, part.indptr, part.indices, part.values, K, params)
    with pytest.raises(RuntimeError):
        graph.launch()
    graph.close()
    fresh = nsparse.SearchGraph(idx, 8, qs.nnz, max_row(qs), K, params)
    D, L = fresh.search(part.n, part.indptr, part.indices, part.values)
    D2, L2 = idx.search(part.n, part.indptr, part.indices, part.values, K, params)
    np.testing.assert_array_equal(L, L2)
    np.testing.assert_array_equal(D, D2)
    fresh.close()
