"""GPU: a query split over a thread-block cluster (2, 4 or 8 CTAs per query:
the leader walks the query, every CTA scores each batch of its candidates).
Results must equal the oracle's bit for bit, batched and one query per
launch, with selectors, small and large batches, k = 10 and 100."""

import numpy as np
import pytest

import nsparse
import oracle as O
from helpers import CUT, HF, K, golden_corpus, oracle_seismic_from_file, ref_file, sq_spec
from nsparse_b200 import synth

pytestmark = pytest.mark.gpu


def make(spec, docs):
    idx = nsparse.index_factory(docs.dim, spec)
    idx.add(docs.n, docs.indptr, docs.indices, docs.values)
    idx.build()
    return idx


def search(idx, qs, k, params):
    return idx.search(qs.n, qs.indptr, qs.indices, qs.values, k, params)


def params(split, variant=-1, batch=0, plain=False, sel=None, cut=CUT, hf=HF):
    p = nsparse.SeismicSearchParameters(cut, hf)
    p.set_kernel(variant, batch)
    p.set_split(split)
    if plain:
        p.set_engine(plain=True)
    if sel is not None:
        p.set_id_selector(sel)
    return p


@pytest.mark.parametrize("kind", ["fp32", "sq8"])
def test_split_query_matches_oracle(tmp_path, kind):
    docs = synth.docs_config0(20000, seed=5)
    qs = synth.queries_config0(200, seed=6)
    vmin, vmax = float(docs.values.min()), float(docs.values.max())
    spec = ("seismic,lambda=2000|beta=200|alpha=0.4|seed=7" if kind == "fp32"
            else sq_spec(vmin, vmax, lam=2000, beta=200))
    idx = make(spec, docs)
    nsparse.write_index(idx, str(tmp_path / "c.idx"))
    codes = None if kind == "fp32" else O.sq_encode_u8(vmin, vmax, qs.values)
    ids = np.arange(0, docs.n, 2, dtype=np.int32)
    scale = None if kind == "fp32" else np.float32(O.sq_scale(vmin, vmax, vmin, vmax))

    def oracle(k, sel_bits=None, cut=CUT, hf=HF):
        D, L = oracle_seismic_from_file(tmp_path / "c.idx", qs, k, cut, hf, codes=codes,
                                        sel_bits=sel_bits)
        if scale is not None:
            D = np.where(L >= 0, (D * scale).astype(np.float32), D)
        return D, L

    Do, Lo = oracle(K)
    Dos, Los = oracle(K, O.bitmap_from_ids(docs.n, ids))
    for split in (2, 4, 8):
        for variant, batch in ((-1, 0), (2, 32), (4, 0), (4, 96), (5, 4096)):
            D, L = search(idx, qs, K, params(split, variant, batch))
            np.testing.assert_array_equal(L, Lo)
            np.testing.assert_array_equal(D, Do)
        D, L = search(idx, qs, K, params(split, sel=nsparse.SetIDSelector(ids)))
        np.testing.assert_array_equal(L, Los)
        np.testing.assert_array_equal(D, Dos)
        sub = qs.rows(0, 12)
        D, L = search(idx, sub, K, params(split, plain=True))
        assert nsparse.last_search_stats().launches == sub.n
        np.testing.assert_array_equal(L, Lo[:12])
        np.testing.assert_array_equal(D, Do[:12])
    Dk, Lk = oracle(100, cut=12, hf=0.95)
    for split in (1, 4):
        D, L = search(idx, qs, 100, params(split, cut=12, hf=0.95))
        np.testing.assert_array_equal(L, Lk)
        np.testing.assert_array_equal(D, Dk)


def test_split_query_golden_and_non_finite(tmp_path):
    """The golden corpus through a reference-built index file, and a query
    value of +inf (row padding masked out) on a split query."""
    docs, qs = golden_corpus()
    ref_file(docs, "seismic,lambda=200|beta=20|alpha=0.4|seed=7", tmp_path / "g.idx")
    idx = nsparse.read_index(str(tmp_path / "g.idx"))
    D0, L0 = search(idx, qs, K, params(1))
    vals = qs.values.copy()
    vals[qs.indptr[3]] = np.inf
    qi = synth.Csr(qs.dim, qs.indptr, qs.indices, vals)
    Do, Lo = oracle_seismic_from_file(tmp_path / "g.idx", qi, K, CUT, HF)
    for split in (2, 8):
        D, L = search(idx, qs, K, params(split))
        np.testing.assert_array_equal(L, L0)
        np.testing.assert_array_equal(D, D0)
        D, L = search(idx, qi, K, params(split, variant=4))
        np.testing.assert_array_equal(L, Lo)
        np.testing.assert_array_equal(D, Do)
