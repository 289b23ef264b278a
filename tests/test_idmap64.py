"""IDMapIndex with 64-bit external ids (an engine extension: the reference's
idx_t is 32 bits, nsparse/id_map_index.h:98-108). Host-side behaviour on CPU:
ids that fit 32 bits keep the reference's IDMP file byte for byte; wider ids
are written under the IDM8 tag with 64-bit ids and read back; the 32-bit
search refuses an index whose ids it cannot return. Search through the map on
the GPU: labels are the external ids of the delegate's results, and 64-bit
selectors filter by external id."""

import struct

import numpy as np
import pytest

import nsparse
import oracle as O
from helpers import CUT, HF, K, SEISMIC, golden_corpus, ref_index

need_ref = pytest.mark.skipif(not O.ref_available(), reason="reference library not built")


def _wide_ids(n, seed=5):
    rng = np.random.default_rng(seed)
    return rng.choice(np.int64(1) << 62, n, replace=False).astype(np.int64) + (1 << 40)


@need_ref
def test_narrow_64bit_ids_write_the_reference_file(tmp_path):
    docs, _ = golden_corpus()
    ids = np.arange(docs.n, dtype=np.int32) * 13 + 5
    spec = "idmap," + SEISMIC
    ours = nsparse.index_factory(docs.dim, spec)
    ours.add_with_ids64(docs.n, docs.indptr, docs.indices, docs.values, ids.astype(np.int64))
    nsparse.write_index(ours, str(tmp_path / "o.idx"))
    ref_index(docs, spec, build=False, ids=ids).write(str(tmp_path / "r.idx"))
    assert open(tmp_path / "o.idx", "rb").read() == open(tmp_path / "r.idx", "rb").read()


def test_wide_ids_round_trip_under_their_own_tag(tmp_path):
    docs, _ = golden_corpus()
    ids = _wide_ids(docs.n)
    idx = nsparse.index_factory(docs.dim, "idmap," + SEISMIC)
    half = docs.n // 2
    a, b = docs.rows(0, half), docs.rows(half, docs.n)
    idx.add_with_ids64(a.n, a.indptr, a.indices, a.values, ids[:half])
    idx.add_with_ids64(b.n, b.indptr, b.indices, b.values, ids[half:])
    assert idx.num_vectors() == docs.n
    p = tmp_path / "w.idx"
    nsparse.write_index(idx, str(p))
    raw = open(p, "rb").read()
    assert raw[:4] == b"IDM8"
    (m,) = struct.unpack_from("<Q", raw, 8)
    assert m == docs.n
    np.testing.assert_array_equal(np.frombuffer(raw, np.int64, m, 16), ids)
    back = nsparse.read_index(str(p))
    assert back.id() == "IDMP" and back.num_vectors() == docs.n
    p2 = tmp_path / "w2.idx"
    nsparse.write_index(back, str(p2))
    assert open(p2, "rb").read() == raw


def test_32bit_search_refuses_wide_ids_before_any_device_work():
    docs, qs = golden_corpus()
    idx = nsparse.index_factory(docs.dim, "idmap," + SEISMIC)
    idx.add_with_ids64(docs.n, docs.indptr, docs.indices, docs.values, _wide_ids(docs.n))
    with pytest.raises(ValueError, match="64 bits"):
        idx.search(qs.n, qs.indptr, qs.indices, qs.values, K)
    with pytest.raises(TypeError):
        idx.add_with_ids64(1, docs.indptr[:2], docs.indices, docs.values,
                           np.zeros(1, np.int32))


def test_set_selector64_membership():
    ids = np.array([3, -7, (1 << 40) + 1, 2**31 - 1], np.int64)
    sel = nsparse.SetIDSelector64(ids)
    assert sel.is_member(3) and sel.is_member(-7) and sel.is_member(2**31 - 1)
    assert not sel.is_member(4)


@pytest.mark.gpu
def test_search64_returns_external_ids_and_filters_by_them(tmp_path):
    docs, qs = golden_corpus()
    ids = _wide_ids(docs.n)
    params = nsparse.SeismicSearchParameters(CUT, HF)
    plain = nsparse.index_factory(docs.dim, SEISMIC)
    plain.add(docs.n, docs.indptr, docs.indices, docs.values)
    plain.build()
    D0, L0 = plain.search(qs.n, qs.indptr, qs.indices, qs.values, K, params)
    idx = nsparse.index_factory(docs.dim, "idmap," + SEISMIC)
    idx.add_with_ids64(docs.n, docs.indptr, docs.indices, docs.values, ids)
    idx.build()
    D, L = idx.search64(qs.n, qs.indptr, qs.indices, qs.values, K, params)
    np.testing.assert_array_equal(D, D0)
    np.testing.assert_array_equal(L, np.where(L0 >= 0, ids[np.maximum(L0, 0)], -1))
    # a 64-bit selector over external ids = the internal selector of the same docs
    keep = np.arange(0, docs.n, 4)
    p = nsparse.SeismicSearchParameters(CUT, HF)
    p.set_id_selector(nsparse.SetIDSelector64(ids[keep]))
    D, L = idx.search64(qs.n, qs.indptr, qs.indices, qs.values, K, p)
    p0 = nsparse.SeismicSearchParameters(CUT, HF)
    p0.set_id_selector(nsparse.SetIDSelector(keep.astype(np.int32)))
    D0, L0 = plain.search(qs.n, qs.indptr, qs.indices, qs.values, K, p0)
    np.testing.assert_array_equal(D, D0)
    np.testing.assert_array_equal(L, np.where(L0 >= 0, ids[np.maximum(L0, 0)], -1))
    # and its complement
    n = nsparse.SeismicSearchParameters(CUT, HF)
    inner = nsparse.SetIDSelector64(ids[keep])
    n.set_id_selector(nsparse.NotIDSelector(inner))
    D, L = idx.search64(qs.n, qs.indptr, qs.indices, qs.values, K, n)
    n0 = nsparse.SeismicSearchParameters(CUT, HF)
    inner0 = nsparse.SetIDSelector(keep.astype(np.int32))
    n0.set_id_selector(nsparse.NotIDSelector(inner0))
    D0, L0 = plain.search(qs.n, qs.indptr, qs.indices, qs.values, K, n0)
    np.testing.assert_array_equal(L, np.where(L0 >= 0, ids[np.maximum(L0, 0)], -1))
    # a few selected ids: the exact-match path (selector size <= k)
    few = nsparse.SeismicSearchParameters(CUT, HF)
    few.set_id_selector(nsparse.SetIDSelector64(ids[[5, 17, 900]]))
    D, L = idx.search64(qs.n, qs.indptr, qs.indices, qs.values, K, few)
    few0 = nsparse.SeismicSearchParameters(CUT, HF)
    few0.set_id_selector(nsparse.SetIDSelector(np.array([5, 17, 900], np.int32)))
    D0, L0 = plain.search(qs.n, qs.indptr, qs.indices, qs.values, K, few0)
    np.testing.assert_array_equal(D, D0)
    np.testing.assert_array_equal(L, np.where(L0 >= 0, ids[np.maximum(L0, 0)], -1))
    # written and read back: the same results
    path = tmp_path / "w.idx"
    nsparse.write_index(idx, str(path))
    back = nsparse.read_index(str(path))
    D2, L2 = back.search64(qs.n, qs.indptr, qs.indices, qs.values, K, params)
    D1, L1 = idx.search64(qs.n, qs.indptr, qs.indices, qs.values, K, params)
    np.testing.assert_array_equal(L2, L1)
    np.testing.assert_array_equal(D2, D1)


@pytest.mark.gpu
def test_server_over_a_wide_idmap_returns_64bit_labels():
    docs, qs = golden_corpus()
    ids = _wide_ids(docs.n)
    idx = nsparse.index_factory(docs.dim, "idmap," + SEISMIC)
    idx.add_with_ids64(docs.n, docs.indptr, docs.indices, docs.values, ids)
    idx.build()
    params = nsparse.SeismicSearchParameters(CUT, HF)
    D0, L0 = idx.search64(qs.n, qs.indptr, qs.indices, qs.values, K, params)
    srv = nsparse.Server(idx, max_batch=64, slots=2)
    try:
        for q in range(8):
            s, e = int(qs.indptr[q]), int(qs.indptr[q + 1])
            t = srv.submit(qs.indices[s:e], qs.values[s:e], k=K, cut=CUT, heap_factor=HF)
            D, L, _ = srv.wait(t)
            np.testing.assert_array_equal(np.asarray(L, np.int64), L0[q])
            np.testing.assert_array_equal(D, D0[q])
    finally:
        srv.close()
