"""GPU parity: every search path through the C ABI against the oracle and the
reference's golden results.

Tolerances: BrutalIndex / InvertedIndex / SEISMIC fp32 scores are bit-identical
to the oracle (the kernels sum in the reference's order); InvertedIndex scores
are within 1e-5 relative of the reference's own MaxScore sums; SEISMIC ids and
scores equal the oracle's bit for bit; SEISMIC-SQ integer code sums are exact.
"""

import numpy as np
import pytest

import nsparse
import oracle as O
from helpers import CUT, HF, K, SEISMIC, golden, golden_corpus, oracle_seismic_from_file, recall, \
    ref_file, sq_codes, sq_exact_scores, sq_spec, unsorted_rows
from nsparse_b200 import synth

pytestmark = pytest.mark.gpu


def make(spec, docs, build=True, ids=None):
    idx = nsparse.index_factory(docs.dim, spec)
    if ids is None:
        idx.add(docs.n, docs.indptr, docs.indices, docs.values)
    else:
        idx.add_with_ids(docs.n, docs.indptr, docs.indices, docs.values, ids)
    if build:
        idx.build()
    return idx


def search(idx, qs, k=K, params=None):
    return idx.search(qs.n, qs.indptr, qs.indices, qs.values, k, params)


def search_each(idx, qs, k=K, params=None):
    D = np.empty((qs.n, k), np.float32)
    L = np.empty((qs.n, k), np.int32)
    for q in range(qs.n):
        r = qs.rows(q, q + 1)
        D[q], L[q] = search(idx, r, k, params)
    return D, L


# ------------------------------------------------------------- exact -------

def test_brutal_matches_reference_golden():
    g = golden()
    docs, qs = golden_corpus()
    idx = make("brutal", docs, build=False)
    D, L = search(idx, qs)
    np.testing.assert_array_equal(L, g["brutal_L"])
    np.testing.assert_array_equal(D, g["brutal_D"])
    assert nsparse.last_search_stats().launches >= 1


def test_inverted_matches_reference_golden():
    g = golden()
    docs, qs = golden_corpus()
    idx = make("inverted", docs)
    D, L = search(idx, qs)
    np.testing.assert_array_equal(L, g["inverted_L"])
    np.testing.assert_allclose(D, g["inverted_D"], rtol=1e-5, atol=1e-6)
    Do, Lo = O.exact_search(docs, qs, K, 1)
    np.testing.assert_array_equal(D, Do)


def test_inverted_filter_matches_reference_golden():
    g = golden()
    docs, qs = golden_corpus()
    idx = make("inverted", docs)
    p = nsparse.SearchParameters()
    p.set_id_selector(nsparse.SetIDSelector(g["filter_ids"]))
    D, L = search(idx, qs, params=p)
    np.testing.assert_array_equal(L, g["inv_filter_L"])
    np.testing.assert_allclose(D, g["inv_filter_D"], rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("k", [1, 10, 37, 100])
def test_exact_paths_match_oracle_medium(k):
    docs = synth.docs_config0(30000, seed=5)
    qs = synth.queries_config0(150, seed=5)
    b = make("brutal", docs, build=False)
    D, L = search(b, qs, k)
    Do, Lo = O.exact_search(docs, qs, k, 0)
    np.testing.assert_array_equal(L, Lo)
    np.testing.assert_array_equal(D, Do)
    v = make("inverted", docs)
    D, L = search(v, qs, k)
    Do, Lo = O.exact_search(docs, qs, k, 1)
    np.testing.assert_array_equal(L, Lo)
    np.testing.assert_array_equal(D, Do)


@pytest.mark.parametrize("k", [10, 200])
def test_exact_paths_unsorted_rows_and_large_k(k):
    """Term-at-a-time scoring needs strictly ascending rows and k <= 128; an
    index with unsorted or repeated terms, or a larger k, takes the tile kernel.
    Every combination equals the oracle bit for bit."""
    base = synth.docs_config0(20000, seed=8)
    qs = synth.queries_config0(100, seed=8)
    for docs in (base, unsorted_rows(base, 9)):
        b = make("brutal", docs, build=False)
        D, L = search(b, qs, k)
        Do, Lo = O.exact_search(docs, qs, k, 0)
        np.testing.assert_array_equal(L, Lo)
        np.testing.assert_array_equal(D, Do)
        v = make("inverted", docs)
        D, L = search(v, qs, k)
        Do, Lo = O.exact_search(docs, qs, k, 1)
        np.testing.assert_array_equal(L, Lo)
        np.testing.assert_array_equal(D, Do)


def test_exact_paths_selector_empty_queries_and_readd():
    """Across several doc chunks: a 10% selector on the inverted index, empty
    query rows (brutal: the first k docs at score 0; inverted: padding), and a
    second add(), after which the postings follow the grown index."""
    docs = synth.docs_config0(40000, seed=11)
    qs = synth.queries_config0(80, seed=11)
    ip = qs.indptr.copy()
    keep = np.ones(qs.nnz, bool)
    for q in (3, 40):  # empty rows 3 and 40
        keep[ip[q]:ip[q + 1]] = False
    lens = np.diff(ip)
    lens[[3, 40]] = 0
    qe = synth.Csr(qs.dim, np.concatenate([[0], np.cumsum(lens)]).astype(np.int32),
                   qs.indices[keep], qs.values[keep])
    rng = np.random.default_rng(12)
    ids = np.sort(rng.choice(docs.n, docs.n // 10, replace=False)).astype(np.int32)
    v = make("inverted", docs)
    p = nsparse.SearchParameters()
    p.set_id_selector(nsparse.SetIDSelector(ids))
    D, L = search(v, qe, 10, p)
    Do, Lo = O.exact_search(docs, qe, 10, 1, sel_bits=O.bitmap_from_ids(docs.n, ids))
    np.testing.assert_array_equal(L, Lo)
    np.testing.assert_array_equal(D, Do)
    assert (L[[3, 40]] == -1).all()
    b = make("brutal", docs, build=False)
    D, L = search(b, qe, 10)
    Do, Lo = O.exact_search(docs, qe, 10, 0)
    np.testing.assert_array_equal(L, Lo)
    np.testing.assert_array_equal(D, Do)
    np.testing.assert_array_equal(L[3], np.arange(10))
    more = synth.docs_config0(15000, seed=13)
    b.add(more.n, more.indptr, more.indices, more.values)
    grown = synth.Csr(docs.dim, np.concatenate([docs.indptr, more.indptr[1:] + docs.nnz]).astype(np.int32),
                      np.concatenate([docs.indices, more.indices]),
                      np.concatenate([docs.values, more.values]))
    D, L = search(b, qs, 10)
    Do, Lo = O.exact_search(grown, qs, 10, 0)
    np.testing.assert_array_equal(L, Lo)
    np.testing.assert_array_equal(D, Do)


def test_brutal_ignores_selector_and_pads():
    docs, qs = golden_corpus()
    idx = make("brutal", docs, build=False)
    p = nsparse.SearchParameters()
    p.set_id_selector(nsparse.SetIDSelector(np.arange(50, dtype=np.int32)))
    _, L1 = search(idx, qs, params=p)
    _, L0 = search(idx, qs)
    np.testing.assert_array_equal(L1, L0)
    small = make("brutal", docs.rows(0, 3), build=False)
    D, L = search(small, qs, 10)
    assert (L[:, 3:] == -1).all() and (D[:, 3:] == -1.0).all()


def test_inverted_not_selector_and_short_rows():
    docs, qs = golden_corpus()
    idx = make("inverted", docs)
    _, L0 = search(idx, qs)
    banned = L0[:, :3].ravel()
    p = nsparse.SearchParameters()
    inner = nsparse.SetIDSelector(banned.astype(np.int32))
    p.set_id_selector(nsparse.NotIDSelector(inner))
    _, L = search(idx, qs, params=p)
    assert not np.isin(L[L >= 0], banned).any()
    Do, Lo = O.exact_search(docs, qs, K, 1, sel_bits=~O.bitmap_from_ids(docs.n, banned))
    np.testing.assert_array_equal(L, Lo)


# ----------------------------------------------------------- SEISMIC ------

@pytest.fixture(scope="module")
def seismic_file(tmp_path_factory):
    docs, _ = golden_corpus()
    p = tmp_path_factory.mktemp("idx") / "s.idx"
    ref_file(docs, SEISMIC, p)
    return p


def test_seismic_matches_reference_golden(seismic_file):
    g = golden()
    _, qs = golden_corpus()
    idx = nsparse.read_index(str(seismic_file))
    D, L = search(idx, qs, params=nsparse.SeismicSearchParameters(CUT, HF))
    np.testing.assert_array_equal(L, g["seismic_L"])
    np.testing.assert_array_equal(D, g["seismic_D"])
    st = nsparse.last_search_stats()
    assert st.docs_scored > 0 and st.bytes > 0 and st.launches == 1


def test_seismic_plain_equals_batched(seismic_file):
    _, qs = golden_corpus()
    idx = nsparse.read_index(str(seismic_file))
    p = nsparse.SeismicSearchParameters(CUT, HF)
    Db, Lb = search(idx, qs, params=p)
    p.set_engine(plain=True)
    Dp, Lp = search(idx, qs, params=p)
    assert nsparse.last_search_stats().launches == qs.n
    np.testing.assert_array_equal(Lp, Lb)
    np.testing.assert_array_equal(Dp, Db)
    p2 = nsparse.SeismicSearchParameters(CUT, HF)
    De, Le = search_each(idx, qs, params=p2)
    np.testing.assert_array_equal(Le, Lb)
    np.testing.assert_array_equal(De, Db)
    for wpb in (1, 2, 8, 16, 32):
        p3 = nsparse.SeismicSearchParameters(CUT, HF)
        p3.set_engine(False, wpb)
        Dw, Lw = search(idx, qs, params=p3)
        np.testing.assert_array_equal(Lw, Lb)
        np.testing.assert_array_equal(Dw, Db)


@pytest.mark.parametrize("variant,stage", [(0, 0), (1, 0), (1, 2048), (1, 128), (2, 0), (2, 32),
                                           (3, 0), (4, 64), (5, 0)])
@pytest.mark.parametrize("kind", ["fp32", "sq8"])
def test_seismic_kernel_variants_agree(tmp_path, variant, stage, kind):
    """Direct row loads, bulk-copy staging, and staging buffers so small that
    most rows are scored from HBM in their place: identical results."""
    docs, qs = golden_corpus()
    spec = SEISMIC if kind == "fp32" else sq_spec(float(docs.values.min()),
                                                  float(docs.values.max()))
    ref_file(docs, spec, tmp_path / "v.idx")
    idx = nsparse.read_index(str(tmp_path / "v.idx"))
    base = nsparse.SeismicSearchParameters(CUT, HF)
    base.set_kernel(0, 0)
    D0, L0 = search(idx, qs, params=base)
    p = nsparse.SeismicSearchParameters(CUT, HF)
    p.set_kernel(variant, stage)
    D, L = search(idx, qs, params=p)
    np.testing.assert_array_equal(L, L0)
    np.testing.assert_array_equal(D, D0)
    p.set_engine(plain=True)
    Dp, Lp = search(idx, qs.rows(0, 8), params=p)
    np.testing.assert_array_equal(Lp, L0[:8])
    sel = nsparse.SetIDSelector(np.arange(0, docs.n, 3, dtype=np.int32))
    p2 = nsparse.SeismicSearchParameters(CUT, HF)
    p2.set_kernel(variant, stage)
    p2.set_id_selector(sel)
    b2 = nsparse.SeismicSearchParameters(CUT, HF)
    b2.set_kernel(0, 0)
    b2.set_id_selector(sel)
    np.testing.assert_array_equal(search(idx, qs, params=p2)[1], search(idx, qs, params=b2)[1])


@pytest.mark.parametrize("kind", ["fp32", "sq8"])
def test_cta_kernel_batches_split_blocks_and_sorts_in_hbm(tmp_path, kind):
    """One CTA per query: blocks of hundreds of docs split across batches of
    32, the first list (up to 200 blocks) sorted in global scratch, selector
    filtering, 1, 2, 4 and 8 lanes per doc -- results equal the oracle's bit for
    bit at every batch size."""
    docs = synth.docs_config0(20000, seed=5)
    qs = synth.queries_config0(200, seed=6)
    vmin, vmax = float(docs.values.min()), float(docs.values.max())
    spec = ("seismic,lambda=2000|beta=200|alpha=0.4|seed=7" if kind == "fp32"
            else sq_spec(vmin, vmax, lam=2000, beta=200))
    idx = make(spec, docs)
    nsparse.write_index(idx, str(tmp_path / "c.idx"))
    codes = None if kind == "fp32" else O.sq_encode_u8(vmin, vmax, qs.values)
    ids = np.arange(0, docs.n, 2, dtype=np.int32)
    Do, Lo = oracle_seismic_from_file(tmp_path / "c.idx", qs, K, CUT, HF, codes=codes)
    Dos, Los = oracle_seismic_from_file(tmp_path / "c.idx", qs, K, CUT, HF, codes=codes,
                                        sel_bits=O.bitmap_from_ids(docs.n, ids))
    if kind != "fp32":
        scale = np.float32(O.sq_scale(vmin, vmax, vmin, vmax))
        Do = np.where(Lo >= 0, (Do * scale).astype(np.float32), Do)
        Dos = np.where(Los >= 0, (Dos * scale).astype(np.float32), Dos)
    for variant, batch in ((2, 0), (2, 32), (2, 96), (2, 4096), (3, 64), (4, 0), (4, 32), (5, 0),
                           (5, 64)):
        p = nsparse.SeismicSearchParameters(CUT, HF)
        p.set_kernel(variant, batch)
        D, L = search(idx, qs, params=p)
        np.testing.assert_array_equal(L, Lo)
        np.testing.assert_array_equal(D, Do)
        p.set_id_selector(nsparse.SetIDSelector(ids))
        Ds, Ls = search(idx, qs, params=p)
        np.testing.assert_array_equal(Ls, Los)
        np.testing.assert_array_equal(Ds, Dos)


def test_cta_kernel_non_finite_query_value(seismic_file):
    """A query value of +inf: row padding must not turn sums into NaN."""
    _, qs = golden_corpus()
    vals = qs.values.copy()
    vals[qs.indptr[3]] = np.inf
    qi = synth.Csr(qs.dim, qs.indptr, qs.indices, vals)
    Do, Lo = oracle_seismic_from_file(seismic_file, qi, K, CUT, HF)
    idx = nsparse.read_index(str(seismic_file))
    for variant in (2, 3, 4, 5):
        p = nsparse.SeismicSearchParameters(CUT, HF)
        p.set_kernel(variant, 0)
        D, L = search(idx, qi, params=p)
        np.testing.assert_array_equal(L, Lo)
        np.testing.assert_array_equal(D, Do)


def test_autotune_picks_a_shape_and_keeps_results(seismic_file):
    """The autotuner's choice is one of the CTA-per-query shapes and the
    searches that follow it return the same ids and scores."""
    _, qs = golden_corpus()
    idx = nsparse.read_index(str(seismic_file))
    p = nsparse.SeismicSearchParameters(CUT, HF)
    D0, L0 = search(idx, qs, params=p)
    c = idx.autotune(qs.n, qs.indptr, qs.indices, qs.values, K, p)
    assert 2 <= c["variant"] <= 5 and c["batch_docs"] in (256, 512, 640, 1024)
    assert c["warps_per_block"] in (4, 8) and c["kernel_ms"] > 0
    assert c["ctas_per_query"] in (1, 2, 4, 8)
    D1, L1 = search(idx, qs, params=p)
    np.testing.assert_array_equal(L1, L0)
    np.testing.assert_array_equal(D1, D0)
    # one-query launches take the tuned split
    p1 = nsparse.SeismicSearchParameters(CUT, HF)
    p1.set_engine(plain=True)
    D2, L2 = search(idx, qs.rows(0, 8), params=p1)
    np.testing.assert_array_equal(L2, L0[:8])
    np.testing.assert_array_equal(D2, D0[:8])


def test_seismic_filter_and_exact_path_match_golden(seismic_file):
    g = golden()
    _, qs = golden_corpus()
    idx = nsparse.read_index(str(seismic_file))
    p = nsparse.SeismicSearchParameters(CUT, HF)
    p.set_id_selector(nsparse.SetIDSelector(g["filter_ids"]))
    D, L = search(idx, qs, params=p)
    np.testing.assert_array_equal(L, g["filter_L"])
    np.testing.assert_array_equal(D, g["filter_D"])
    p = nsparse.SeismicSearchParameters(CUT, HF)
    p.set_id_selector(nsparse.SetIDSelector(g["exact_ids"]))
    D, L = search(idx, qs.rows(0, 4), params=p)
    np.testing.assert_array_equal(L, g["exact_L"])
    np.testing.assert_array_equal(D, g["exact_D"])


@pytest.mark.parametrize("cut,hf,k", [(1, 1.0, 10), (3, 0.7, 5), (12, 0.95, 100), (200, 2.0, 10)])
def test_seismic_matches_oracle_params(seismic_file, cut, hf, k):
    _, qs = golden_corpus()
    idx = nsparse.read_index(str(seismic_file))
    D, L = search(idx, qs, k, nsparse.SeismicSearchParameters(cut, hf))
    Do, Lo = oracle_seismic_from_file(seismic_file, qs, k, cut, hf)
    np.testing.assert_array_equal(L, Lo)
    np.testing.assert_array_equal(D, Do)


def test_seismic_medium_corpus_matches_oracle_and_reference(tmp_path):
    docs = synth.docs_config0(20000, seed=3)
    qs = synth.queries_config0(300, seed=3)
    spec = "seismic,lambda=400|beta=40|alpha=0.4|seed=7"
    r = ref_file(docs, spec, tmp_path / "m.idx")
    idx = nsparse.read_index(str(tmp_path / "m.idx"))
    D, L = search(idx, qs, params=nsparse.SeismicSearchParameters(10, 0.8))
    Do, Lo = oracle_seismic_from_file(tmp_path / "m.idx", qs, K, 10, 0.8)
    np.testing.assert_array_equal(L, Lo)
    np.testing.assert_array_equal(D, Do)
    Dr, Lr = r.search(qs, K, param_kind=2, cut=10, heap_factor=0.8)
    same = (Lr == L).all(axis=1)
    assert same.mean() >= 0.99
    np.testing.assert_array_equal(Dr[same], D[same])
    _, Lt = O.exact_search(docs, qs, K, 1)
    assert recall(L, Lt) >= recall(Lr, Lt) - 0.005


def test_seismic_sq_matches_oracle_and_scores_exact(tmp_path):
    g = golden()
    docs, qs = golden_corpus()
    vmin, vmax = float(g["sq_vmin"]), float(g["sq_vmax"])
    ref_file(docs, sq_spec(vmin, vmax), tmp_path / "q.idx")
    idx = nsparse.read_index(str(tmp_path / "q.idx"))
    D, L = search(idx, qs, params=nsparse.SeismicSearchParameters(CUT, HF))
    codes = O.sq_encode_u8(vmin, vmax, qs.values)
    Do, Lo = oracle_seismic_from_file(tmp_path / "q.idx", qs, K, CUT, HF, codes=codes)
    scale = np.float32(O.sq_scale(vmin, vmax, vmin, vmax))
    np.testing.assert_array_equal(L, Lo)
    np.testing.assert_array_equal(D, np.where(Lo >= 0, (Do * scale).astype(np.float32), Do))
    exact = sq_exact_scores(docs, codes, qs, L, vmin, vmax) * scale
    np.testing.assert_array_equal(D[L >= 0], exact[L >= 0])
    _, Lt = O.exact_search(docs, qs, K, 1)
    assert recall(L, Lt) >= recall(g["sq_L"], Lt) - 0.02


def test_seismic_sq_query_range_override(tmp_path):
    g = golden()
    docs, qs = golden_corpus()
    vmin, vmax = float(g["sq_vmin"]), float(g["sq_vmax"])
    ref_file(docs, sq_spec(vmin, vmax), tmp_path / "q.idx")
    idx = nsparse.read_index(str(tmp_path / "q.idx"))
    qmin, qmax = 0.0, float(qs.values.max())
    D, L = search(idx, qs, params=nsparse.SeismicSQSearchParameters(qmin, qmax, CUT, HF))
    codes = O.sq_encode_u8(qmin, qmax, qs.values)
    Do, Lo = oracle_seismic_from_file(tmp_path / "q.idx", qs, K, CUT, HF, codes=codes)
    scale = np.float32(O.sq_scale(vmin, vmax, qmin, qmax))
    np.testing.assert_array_equal(L, Lo)
    np.testing.assert_array_equal(D, np.where(Lo >= 0, (Do * scale).astype(np.float32), Do))


def _sq16_expect(path, docs, qs, vmin, vmax, qmin, qmax, cut=CUT, hf=HF, k=K):
    codes = sq_codes(qmin, qmax, qs.values, 16)
    Do, Lo = oracle_seismic_from_file(path, qs, k, cut, hf, codes=codes)
    scale = np.float32(O.sq_scale(vmin, vmax, qmin, qmax, 16))
    return codes, scale, Lo, np.where(Lo >= 0, (Do * scale).astype(np.float32), Do)


def test_seismic_sq16_matches_oracle_and_scores_exact(tmp_path):
    """16-bit codes on the device (uint16 code table, int64 doc sums,
    scalar_quantizer.h:108-118, distance.h:49-57): ids and scores equal the
    oracle's, every score is the exact int64 code sum decoded, batched and one
    query per launch, every kernel variant."""
    docs, qs = golden_corpus()
    vmin, vmax = float(docs.values.min()), float(docs.values.max())
    path = tmp_path / "q16.idx"
    r = ref_file(docs, sq_spec(vmin, vmax, bits=16), path)
    idx = nsparse.read_index(str(path))
    codes, scale, Lo, Do = _sq16_expect(path, docs, qs, vmin, vmax, vmin, vmax)
    for variant in (-1, 0, 1, 2, 3, 5):
        p = nsparse.SeismicSearchParameters(CUT, HF)
        p.set_kernel(variant, 0)
        D, L = search(idx, qs, params=p)
        np.testing.assert_array_equal(L, Lo)
        np.testing.assert_array_equal(D, Do)
    plain = nsparse.SeismicSearchParameters(CUT, HF)
    plain.set_engine(plain=True)
    D, L = search(idx, qs, params=plain)
    np.testing.assert_array_equal(L, Lo)
    np.testing.assert_array_equal(D, Do)
    exact = sq_exact_scores(docs, codes, qs, L, vmin, vmax, 16) * scale
    np.testing.assert_array_equal(D[L >= 0], exact[L >= 0])
    # the reference's own search of the same file: the same rows
    Dr, Lr = r.search(qs, K, param_kind=2, cut=CUT, heap_factor=HF)
    same = (Lr == L).all(axis=1)
    assert same.mean() >= 0.95
    np.testing.assert_array_equal(Dr[same], D[same])


def test_seismic_sq16_query_range_and_k100(tmp_path):
    docs, qs = golden_corpus()
    vmin, vmax = float(docs.values.min()), float(docs.values.max())
    path = tmp_path / "q16.idx"
    ref_file(docs, sq_spec(vmin, vmax, bits=16), path)
    idx = nsparse.read_index(str(path))
    qmin, qmax = 0.0, float(qs.values.max())
    _, _, Lo, Do = _sq16_expect(path, docs, qs, vmin, vmax, qmin, qmax)
    D, L = search(idx, qs, params=nsparse.SeismicSQSearchParameters(qmin, qmax, CUT, HF))
    np.testing.assert_array_equal(L, Lo)
    np.testing.assert_array_equal(D, Do)
    _, _, Lo, Do = _sq16_expect(path, docs, qs, vmin, vmax, vmin, vmax, k=100)
    D, L = search(idx, qs, k=100, params=nsparse.SeismicSearchParameters(CUT, HF))
    np.testing.assert_array_equal(L, Lo)
    np.testing.assert_array_equal(D, Do)


def test_seismic_sq16_device_build(tmp_path):
    """A 16-bit index built on the device: the file it writes reads back in
    the reference, and the engine's search of it equals the oracle's."""
    docs, qs = golden_corpus()
    vmin, vmax = float(docs.values.min()), float(docs.values.max())
    idx = make(sq_spec(vmin, vmax, bits=16), docs)
    path = tmp_path / "dev16.idx"
    nsparse.write_index(idx, str(path))
    _, _, Lo, Do = _sq16_expect(path, docs, qs, vmin, vmax, vmin, vmax)
    D, L = search(idx, qs, params=nsparse.SeismicSearchParameters(CUT, HF))
    np.testing.assert_array_equal(L, Lo)
    np.testing.assert_array_equal(D, Do)
    r = O.RefIndex.read(str(path))
    Dr, Lr = r.search(qs, K, param_kind=2, cut=CUT, heap_factor=HF)
    r.close()
    same = (Lr == L).all(axis=1)
    assert same.mean() >= 0.95
    np.testing.assert_array_equal(Dr[same], D[same])


@pytest.mark.parametrize("kind", ["fp32", "sq8", "fp32-selector"])
def test_counting_pass_counts_each_scored_row_once_per_query(tmp_path, kind):
    """The kernel scores a doc met again in a later cut list again (the
    reference skips it with its visited set, seismic_index.cpp:104-107). Its
    counting pass stamps visited docs: the docs it counts once per query are
    exactly the oracle's scored docs, the rest of its scored docs are exactly
    the oracle's revisits, and results do not change."""
    docs, qs = golden_corpus()
    path = tmp_path / "c.idx"
    codes = None
    if kind == "sq8":
        vmin, vmax = float(docs.values.min()), float(docs.values.max())
        ref_file(docs, sq_spec(vmin, vmax), path)
        codes = O.sq_encode_u8(vmin, vmax, qs.values)
    else:
        ref_file(docs, SEISMIC, path)
    idx = nsparse.read_index(str(path))
    sel = bits = None
    if kind == "fp32-selector":
        keep = np.arange(0, docs.n, 2, dtype=np.int32)
        sel = nsparse.SetIDSelector(keep)
        bits = O.bitmap_from_ids(docs.n, keep)

    def params(count):
        p = nsparse.SeismicSearchParameters(CUT, HF)
        p.set_kernel(4, 0)
        if sel is not None:
            p.set_id_selector(sel)
        p.set_count_unique(count)
        return p

    D, L = search(idx, qs, params=params(False))
    st = nsparse.last_search_stats()
    D2, L2 = search(idx, qs, params=params(True))
    st2 = nsparse.last_search_stats()
    np.testing.assert_array_equal(L2, L)
    np.testing.assert_array_equal(D2, D)
    _, Lo, ost = oracle_seismic_from_file(path, qs, K, CUT, HF, codes=codes, sel_bits=bits,
                                          want_stats=True)
    np.testing.assert_array_equal(L, Lo)
    assert st2.unique_docs == int(ost[:, 0].sum())
    assert st2.docs_scored == st.docs_scored and st2.row_bytes == st.row_bytes
    if sel is None:
        assert st2.docs_scored - st2.unique_docs == int(ost[:, 3].sum())
    assert 0 < st2.unique_row_bytes <= st2.row_bytes < st2.bytes
    assert st2.reference_bytes == st2.bytes - st2.row_bytes + st2.unique_row_bytes


def test_idmap_seismic_returns_external_ids(tmp_path):
    g = golden()
    docs, qs = golden_corpus()
    ext = (np.arange(docs.n, dtype=np.int32) * 7 + 1000)
    ref_file(docs, "idmap," + SEISMIC, tmp_path / "i.idx", ids=ext)
    idx = nsparse.read_index(str(tmp_path / "i.idx"))
    D, L = search(idx, qs, params=nsparse.SeismicSearchParameters(CUT, HF))
    want = np.where(g["seismic_L"] >= 0, ext[np.maximum(g["seismic_L"], 0)], -1)
    np.testing.assert_array_equal(L, want)
    np.testing.assert_array_equal(D, g["seismic_D"])
    # selector in external ids, translated for the delegate
    p = nsparse.SeismicSearchParameters(CUT, HF)
    allowed = ext[g["filter_ids"]]
    sel = nsparse.SetIDSelector(allowed)
    p.set_id_selector(sel)
    D, L = search(idx, qs, params=p)
    want = np.where(g["filter_L"] >= 0, ext[np.maximum(g["filter_L"], 0)], -1)
    np.testing.assert_array_equal(L, want)
    assert p.get_id_selector() is sel


def test_search_before_build_is_padding():
    docs, qs = golden_corpus()
    idx = nsparse.index_factory(docs.dim, SEISMIC)
    idx.add(docs.n, docs.indptr, docs.indices, docs.values)
    D, L = search(idx, qs)
    assert (L == -1).all() and (D == -1.0).all()


def test_unsorted_and_empty_query_rows(seismic_file):
    docs, qs = golden_corpus()
    idx = nsparse.read_index(str(seismic_file))
    p = nsparse.SeismicSearchParameters(CUT, HF)
    D0, L0 = search(idx, qs, params=p)
    # reverse each row's term order: canonicalisation restores the same result
    ip, ix, v = qs.indptr, qs.indices.copy(), qs.values.copy()
    for q in range(qs.n):
        s, e = ip[q], ip[q + 1]
        ix[s:e] = ix[s:e][::-1].copy()
        v[s:e] = v[s:e][::-1].copy()
    D1, L1 = idx.search(qs.n, ip, ix, v, K, p)
    np.testing.assert_array_equal(L1, L0)
    # an empty row returns padding, its neighbours are unaffected
    ip2 = np.concatenate([[0], [0], ip[1:3]]).astype(np.int32)
    D2, L2 = idx.search(3, ip2, qs.indices, qs.values, K, p)
    assert (L2[0] == -1).all()
    np.testing.assert_array_equal(L2[1:], L0[:2])
