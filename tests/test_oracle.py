"""Pins the C oracle (oracle/nsp_oracle.c) before any GPU result is compared
with it: against known answers from the reference's own unit tests, against
the golden results the reference produced (tests/golden/small.npz), and, where
the compiled reference is present, against the reference directly."""

import numpy as np
import pytest

import oracle as O
from helpers import CUT, HF, K, SEISMIC, golden, golden_corpus, oracle_seismic_from_file, \
    sq_codes, sq_exact_scores, \
    recall, ref_file, ref_index, sq_spec, unsorted_rows
from nsparse_b200 import synth

need_ref = pytest.mark.skipif(not O.ref_available(), reason="reference library not built")


# --- known answers restated from the reference's tests ---------------------

def test_quantizer_known_answers():
    # tests/scalar_quantizer_test.cpp:82-135 (range [0, 1], 8 bit)
    codes = O.sq_encode_u8(0.0, 1.0, np.array([0.0, 1.0, 0.5, -0.5, 1.5], np.float32))
    assert codes.tolist() == [0, 255, 128, 0, 255]
    # tests/scalar_quantizer_test.cpp:286-307 (decode_dot_product scale)
    assert abs(65025.0 * O.sq_scale(0.0, 1.0, 0.0, 1.0) - 1.0) < 1e-3
    assert abs(65025.0 * O.sq_scale(0.0, 2.0, 0.0, 4.0) - 8.0) < 1e-3
    assert O.sq_scale(0.0, 1.0, 0.0, 1.0) * 0.0 == 0.0


def test_query_cut_known_answers():
    # tests/vector_process_test.cpp:16-75
    assert O.cut([0, 1, 2, 3, 4], np.array([1, 5, 3, 2, 4], np.float32), 3).tolist() == [1, 4, 2]
    assert O.cut([10, 20, 30], np.array([3, 1, 2], np.float32), 3).tolist() == [10, 20, 30]
    assert O.cut([5, 6], np.array([2, 1], np.float32), 5).tolist() == [5, 6]
    assert O.cut([42], np.array([7], np.float32), 1).tolist() == [42]
    assert len(O.cut([1, 2, 3, 4], np.array([5, 5, 5, 5], np.float32), 2)) == 2


def _csr(dim, rows):
    from nsparse_b200.synth import Csr
    indptr = np.cumsum([0] + [len(r) for r in rows]).astype(np.int32)
    idx = np.array([t for r in rows for t, _ in r], np.uint16)
    val = np.array([v for r in rows for _, v in r], np.float32)
    return Csr(dim, indptr, idx, val)


def test_dot_product_known_answers():
    # tests/distance_test.cpp:40-73: 2*5 = 10; 1+4+9 = 14; 1+0+6 = 7
    docs = _csr(5, [[(3, 2.0)], [(0, 1.0), (2, 2.0), (4, 3.0)]])
    q = _csr(5, [[(3, 5.0)], [(0, 1.0), (2, 2.0), (4, 3.0)]])
    D, L = O.exact_search(docs, q, 2, 0)
    assert D[0, 0] == 10.0 and L[0, 0] == 0
    assert D[1, 0] == 14.0 and L[1, 0] == 1
    q2 = _csr(3, [[(0, 1.0), (2, 2.0)]])
    d2 = _csr(3, [[(0, 1.0), (1, 2.0), (2, 3.0)]])
    D, _ = O.exact_search(d2, q2, 1, 0)
    assert D[0, 0] == 7.0


# --- golden results of the reference ---------------------------------------

@need_ref
def test_exact_oracle_matches_reference_on_unsorted_rows():
    """Rows stored out of term order, some repeating a term: the reference's
    BrutalIndex sums each row in stored order (utils/distance.h:29-37), and so
    does the oracle, bit for bit. The GPU tests compare both exact kernels
    with the oracle on these rows."""
    docs = unsorted_rows(synth.docs_config0(3000, seed=8), 9)
    qs = synth.queries_config0(60, seed=8)
    r = O.RefIndex(docs.dim, "brutal", variant="generic")
    r.add(docs)
    Dr, Lr = r.search(qs, 37)
    r.close()
    D, L = O.exact_search(docs, qs, 37, 0)
    np.testing.assert_array_equal(L, Lr)
    np.testing.assert_array_equal(D, Dr)


def test_exact_oracle_matches_reference_golden():
    g = golden()
    docs, qs = golden_corpus()
    D, L = O.exact_search(docs, qs, K, 0)
    np.testing.assert_array_equal(L, g["brutal_L"])
    np.testing.assert_array_equal(D, g["brutal_D"])  # bit-identical fp32
    D, L = O.exact_search(docs, qs, K, 1)
    np.testing.assert_array_equal(L, g["inverted_L"])
    np.testing.assert_allclose(D, g["inverted_D"], rtol=1e-5, atol=1e-5)
    bits = O.bitmap_from_ids(docs.n, g["filter_ids"])
    D, L = O.exact_search(docs, qs, K, 1, sel_bits=bits)
    np.testing.assert_array_equal(L, g["inv_filter_L"])
    np.testing.assert_allclose(D, g["inv_filter_D"], rtol=1e-5, atol=1e-5)


@need_ref
def test_seismic_oracle_matches_reference_golden(tmp_path):
    g = golden()
    docs, qs = golden_corpus()
    ref_file(docs, SEISMIC, tmp_path / "s.idx")
    import hashlib
    assert hashlib.sha256(open(tmp_path / "s.idx", "rb").read()).hexdigest() == \
        str(g["seismic_file_sha"]), "seeded reference build is not reproducible"
    D, L = oracle_seismic_from_file(tmp_path / "s.idx", qs, K, CUT, HF)
    np.testing.assert_array_equal(L, g["seismic_L"])
    np.testing.assert_array_equal(D, g["seismic_D"])
    bits = O.bitmap_from_ids(docs.n, g["filter_ids"])
    D, L = oracle_seismic_from_file(tmp_path / "s.idx", qs, K, CUT, HF, sel_bits=bits)
    np.testing.assert_array_equal(L, g["filter_L"])
    np.testing.assert_array_equal(D, g["filter_D"])


@need_ref
def test_seismic_sq_oracle_matches_reference_golden(tmp_path):
    g = golden()
    docs, qs = golden_corpus()
    vmin, vmax = float(g["sq_vmin"]), float(g["sq_vmax"])
    ref_file(docs, sq_spec(vmin, vmax), tmp_path / "q.idx")
    codes = O.sq_encode_u8(vmin, vmax, qs.values)
    D, L = oracle_seismic_from_file(tmp_path / "q.idx", qs, K, CUT, HF, codes=codes)
    scale = np.float32(O.sq_scale(vmin, vmax, vmin, vmax))
    Dd = np.where(L >= 0, (D * scale).astype(np.float32), D)
    # uint8 codes tie constantly; the oracle orders them by the reference's own
    # TopKHolder and std::ranges::sort steps, so rows match position by position
    np.testing.assert_array_equal(L, g["sq_L"])
    np.testing.assert_array_equal(Dd, g["sq_D"])
    exact = sq_exact_scores(docs, codes, qs, L, vmin, vmax) * scale
    np.testing.assert_array_equal(Dd[L >= 0], exact[L >= 0])
    _, Lt = O.exact_search(docs, qs, K, 1)
    assert recall(L, Lt) >= recall(g["sq_L"], Lt) - 0.02


@need_ref
def test_quantizer_matches_reference_encoder():
    L = O.ref_lib("generic")
    rng = np.random.default_rng(3)
    vals = np.concatenate([rng.lognormal(0, 0.8, 5000), [-1, 0, 1e9, 0.5]]).astype(np.float32)
    want = np.empty(len(vals), np.uint8)
    assert L.ref_sq_encode(8, 0.0158, 84.475, vals.ctypes.data, want.ctypes.data, len(vals)) == 0
    np.testing.assert_array_equal(O.sq_encode_u8(0.0158, 84.475, vals), want)


@need_ref
def test_quantizer_16bit_matches_reference_encoder():
    L = O.ref_lib("generic")
    rng = np.random.default_rng(4)
    vals = np.concatenate([rng.lognormal(0, 0.8, 5000), [-1, 0, 1e9, 0.5]]).astype(np.float32)
    want = np.empty(len(vals), np.uint16)
    assert L.ref_sq_encode(16, 0.0158, 84.475, vals.ctypes.data, want.ctypes.data,
                           len(vals)) == 0
    np.testing.assert_array_equal(O.sq_encode_u16(0.0158, 84.475, vals), want)
    # tests/scalar_quantizer_test.cpp (range [0, 1]): ends and midpoint
    got = O.sq_encode_u16(0.0, 1.0, np.array([0.0, 1.0, 0.5, -0.5, 1.5], np.float32))
    assert got.tolist() == [0, 65535, 32768, 0, 65535]
    assert abs(65535.0 * 65535.0 * O.sq_scale(0.0, 1.0, 0.0, 1.0, 16) - 1.0) < 1e-3


@need_ref
def test_seismic_sq16_oracle_matches_reference(tmp_path):
    """16-bit codes (SeismicScalarQuantizedIndex with quantizer=16bit): the
    oracle over the reference's own file returns the reference's rows, and
    every returned score is the exact int64 code sum, decoded."""
    docs, qs = golden_corpus()
    vmin, vmax = float(docs.values.min()), float(docs.values.max())
    r = ref_file(docs, sq_spec(vmin, vmax, bits=16), tmp_path / "q16.idx")
    assert O.read_index_file(str(tmp_path / "q16.idx"))["vectors"]["esz"] == 2
    codes = sq_codes(vmin, vmax, qs.values, 16)
    D, L = oracle_seismic_from_file(tmp_path / "q16.idx", qs, K, CUT, HF, codes=codes)
    scale = np.float32(O.sq_scale(vmin, vmax, vmin, vmax, 16))
    Dd = np.where(L >= 0, (D * scale).astype(np.float32), D)
    Dr, Lr = r.search(qs, K, param_kind=2, cut=CUT, heap_factor=HF)
    np.testing.assert_array_equal(L, Lr)
    np.testing.assert_array_equal(Dd, Dr)
    exact = sq_exact_scores(docs, codes, qs, L, vmin, vmax, 16) * scale
    np.testing.assert_array_equal(Dd[L >= 0], exact[L >= 0])


@need_ref
def test_cut_matches_reference_with_tied_values():
    """Tied weights (uint8 codes tie constantly): which terms the cut keeps and
    their order are the reference's TopKHolder's."""
    L = O.ref_lib("generic")
    rng = np.random.default_rng(11)
    for n in (3, 10, 25, 120, 200):
        idx = np.sort(rng.choice(30522, n, replace=False)).astype(np.uint16)
        for levels in (1, 2, 4, 16):
            w8 = rng.integers(0, levels, n).astype(np.uint8)
            w32 = w8.astype(np.float32) * 0.5
            for cut in (1, 3, 5, 10, 12, 200):
                for w, fn in ((w8, L.ref_top_k_tokens_u8), (w32, L.ref_top_k_tokens_f32)):
                    out = np.empty(max(n, cut), np.uint16)
                    cnt = np.zeros(1, np.int32)
                    assert fn(idx.ctypes.data, w.ctypes.data, n, cut, out.ctypes.data,
                              cnt.ctypes.data) == 0
                    np.testing.assert_array_equal(O.cut(idx, w, cut), out[:cnt[0]])


@need_ref
def test_seismic_sq8_oracle_rows_equal_reference_under_ties(tmp_path):
    """A 20k-doc SEISMIC-SQ index: uint8 block scores, doc scores and query
    codes tie constantly, and the oracle's rows equal the reference's row for
    row (ids, order and scores)."""
    from nsparse_b200 import synth
    docs = synth.docs_config2(20000, seed=5)
    qs = synth.queries_config2(300, seed=6)
    vmin, vmax = float(docs.values.min()), float(docs.values.max())
    spec = sq_spec(vmin, vmax, lam=600, beta=60)
    r = ref_file(docs, spec, tmp_path / "t.idx")
    codes = O.sq_encode_u8(vmin, vmax, qs.values)
    for cut, hf in ((12, 0.9), (5, 0.7), (30, 1.0)):
        D, Lo = oracle_seismic_from_file(tmp_path / "t.idx", qs, K, cut, hf, codes=codes)
        scale = np.float32(O.sq_scale(vmin, vmax, vmin, vmax))
        Dd = np.where(Lo >= 0, (D * scale).astype(np.float32), D)
        Dr, Lr = r.search(qs, K, param_kind=2, cut=cut, heap_factor=hf)
        np.testing.assert_array_equal(Lo, Lr)
        np.testing.assert_array_equal(Dd, Dr)


@need_ref
def test_cut_matches_reference_on_distinct_values():
    L = O.ref_lib("generic")
    rng = np.random.default_rng(5)
    for n in (3, 10, 25, 120):
        idx = np.sort(rng.choice(30522, n, replace=False)).astype(np.uint16)
        w = rng.permutation(n).astype(np.float32) + 1.0  # distinct: order is defined
        for cut in (1, 5, 10, 12, 200):
            out = np.empty(max(n, cut), np.uint16)
            cnt = np.zeros(1, np.int32)
            assert L.ref_top_k_tokens_f32(idx.ctypes.data, w.ctypes.data, n, cut,
                                          out.ctypes.data, cnt.ctypes.data) == 0
            np.testing.assert_array_equal(O.cut(idx, w, cut), out[:cnt[0]])


@need_ref
def test_seismic_oracle_recall_equals_reference_medium(tmp_path):
    """A 20k-doc corpus: oracle and reference return the same rows."""
    from nsparse_b200 import synth
    docs = synth.docs_config0(20000, seed=3)
    qs = synth.queries_config0(100, seed=3)
    spec = "seismic,lambda=400|beta=40|alpha=0.4|seed=7"
    r = ref_file(docs, spec, tmp_path / "m.idx")
    Dr, Lr = r.search(qs, K, param_kind=2, cut=10, heap_factor=0.8)
    Do, Lo = oracle_seismic_from_file(tmp_path / "m.idx", qs, K, 10, 0.8)
    np.testing.assert_array_equal(Lr, Lo)
    np.testing.assert_array_equal(Dr, Do)
    _, Lt = O.exact_search(docs, qs, K, 1)
    assert recall(Lo, Lt) == pytest.approx(recall(Lr, Lt), abs=0.01)
