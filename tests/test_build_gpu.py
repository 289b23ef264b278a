"""The SEISMIC build on the device against the reference's build.

fp32: with a fixed seed the device-built index file is byte-identical to the
one the reference writes (posting truncation, centroid draw, assignment,
summaries and transposes all agree). Where values tie, posting truncation
still agrees (the host repeats the reference's unstable sort for those
lists); only a summary's alpha cut may keep another of several equal maxima.

uint8 (SEISMIC-SQ): codes tie constantly, and the reference breaks ties in its
posting truncation and summary cut with an unstable sort, so whole files are
not comparable. Instead each list is checked through the reference's own
functions: given the engine's kept list and centroids, the reference's
assigner (cluster/kmeans_utils.cpp) produces the engine's blocks exactly, and
its summarizer (cluster/inverted_list_clusters.cpp) produces summaries with
the engine's entry counts and values.
"""

import hashlib

import numpy as np
import pytest

import nsparse
import oracle as O
from helpers import CUT, HF, K, SEISMIC, golden, golden_corpus, recall, ref_file, sq_spec
from nsparse_b200 import synth

pytestmark = pytest.mark.gpu


def device_build(docs, spec, path=None):
    idx = nsparse.index_factory(docs.dim, spec)
    idx.add(docs.n, docs.indptr, docs.indices, docs.values)
    idx.build()
    if path is not None:
        nsparse.write_index(idx, str(path))
    return idx


def sha(path):
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def test_fp32_build_is_byte_identical_to_reference_golden(tmp_path):
    g = golden()
    docs, qs = golden_corpus()
    idx = device_build(docs, SEISMIC, tmp_path / "d.idx")
    assert sha(tmp_path / "d.idx") == str(g["seismic_file_sha"])
    D, L = idx.search(qs.n, qs.indptr, qs.indices, qs.values, K,
                      nsparse.SeismicSearchParameters(CUT, HF))
    np.testing.assert_array_equal(L, g["seismic_L"])
    np.testing.assert_array_equal(D, g["seismic_D"])


@pytest.mark.parametrize("spec", [
    "seismic,lambda=400|beta=40|alpha=0.4|seed=7",
    "seismic,lambda=-1|beta=-1|alpha=0.5|seed=3",
    "seismic,lambda=50|beta=0|alpha=0.2|seed=11",
    "seismic,lambda=0|beta=8|alpha=0.9|seed=5",
])
def test_fp32_build_matches_reference_file(tmp_path, spec):
    docs = synth.docs_config0(20000, seed=3)
    ref_file(docs, spec, tmp_path / "r.idx")
    device_build(docs, spec, tmp_path / "d.idx")
    a = open(tmp_path / "r.idx", "rb").read()
    b = open(tmp_path / "d.idx", "rb").read()
    if a != b:
        n_blocks, n_diff = _lists_match_up_to_cut_ties(tmp_path / "r.idx", tmp_path / "d.idx")
        pytest.fail(f"{n_diff} of {n_blocks} block summaries differ from the reference's")


def test_fp32_build_with_tied_values_matches_reference_lists(tmp_path):
    """Values on a coarse grid tie constantly. A posting list longer than
    lambda keeps its top lambda in the order the reference's unstable sort
    leaves them (the host repeats that sort for lists whose kept values tie),
    so every list's docs and block offsets equal the reference's -- ties
    across the cut included. Where equal maxima straddle a block summary's
    alpha cut, the host repeats the reference's sort of that block's pairs,
    so the summaries -- and the whole file -- are the reference's too."""
    base = synth.docs_config0(20000, seed=3)
    docs = synth.Csr(base.dim, base.indptr, base.indices,
                     (np.round(base.values * 4) / 4 + 0.25).astype(np.float32))
    spec = "seismic,lambda=100|beta=10|alpha=0.4|seed=7"
    ref_file(docs, spec, tmp_path / "r.idx")
    device_build(docs, spec, tmp_path / "d.idx")
    f = O.read_index_file(str(tmp_path / "r.idx"))
    assert sum(len(c["docs"]) == 100 for c in f["lists"]) > 500  # many truncated lists
    n_blocks, n_diff = _lists_match_up_to_cut_ties(tmp_path / "r.idx", tmp_path / "d.idx")
    assert n_diff == 0, f"{n_diff} of {n_blocks} block summaries differ from the reference's"
    assert sha(tmp_path / "r.idx") == sha(tmp_path / "d.idx")


def _lists_match_up_to_cut_ties(ref_path, dev_path):
    """Every list's docs and offsets equal; a block summary that differs
    keeps the same values and differs only in terms whose value is the
    block's smallest kept one (equal maxima straddling the alpha cut, which
    the reference leaves to its unstable sort). Returns (blocks, differing)."""
    ra, rb = O.read_index_file(str(ref_path)), O.read_index_file(str(dev_path))
    np.testing.assert_array_equal(ra["vectors"]["values"], rb["vectors"]["values"])
    n_blocks = n_diff = 0
    for la, lb in zip(ra["lists"], rb["lists"]):
        np.testing.assert_array_equal(la["docs"], lb["docs"])        # truncation + assignment
        np.testing.assert_array_equal(la["offsets"], lb["offsets"])
        for blk in range(len(la["offsets"]) - 1 if len(la["offsets"]) else 0):
            n_blocks += 1
            ta, va = _block_summary(la, blk)
            tb, vb = _block_summary(lb, blk)
            if np.array_equal(ta, tb) and np.array_equal(va, vb):
                continue
            n_diff += 1
            np.testing.assert_array_equal(np.sort(va), np.sort(vb))  # same kept values
            boundary = va.min()
            only = set(ta.tolist()) ^ set(tb.tolist())
            vals = dict(zip(ta.tolist(), va.tolist()))
            vals.update(zip(tb.tolist(), vb.tolist()))
            assert all(vals[t] == boundary for t in only), "summary differs beyond a tie"
    return n_blocks, n_diff


def _block_summary(lst, blk):
    """(terms, values) of one block's summary from a list's CSC arrays."""
    m = lst["csc_cluster"] == blk
    col = np.searchsorted(lst["term_ptr"], np.nonzero(m)[0], side="right") - 1
    return lst["term_ids"][col], lst["csc_value"][m]


def test_seeded_build_is_reproducible_and_seed_matters(tmp_path):
    docs, qs = golden_corpus()
    device_build(docs, SEISMIC, tmp_path / "a.idx")
    device_build(docs, SEISMIC, tmp_path / "b.idx")
    assert sha(tmp_path / "a.idx") == sha(tmp_path / "b.idx")
    device_build(docs, SEISMIC.replace("seed=7", "seed=8"), tmp_path / "c.idx")
    assert sha(tmp_path / "a.idx") != sha(tmp_path / "c.idx")


def _posting_codes(docs, codes, t):
    rows = np.repeat(np.arange(docs.n), np.diff(docs.indptr))
    m = docs.indices == t
    return rows[m].astype(np.int32), codes[m]


def test_sq_build_assignment_and_summaries_match_reference(tmp_path):
    docs, _ = golden_corpus()
    vmin, vmax = float(docs.values.min()), float(docs.values.max())
    lam, beta, alpha = 200, 20, 0.4
    device_build(docs, sq_spec(vmin, vmax, lam, beta), tmp_path / "q.idx")
    f = O.read_index_file(str(tmp_path / "q.idx"))
    codes = O.sq_encode_u8(vmin, vmax, docs.values)
    L = O.ref_lib("generic")
    P = lambda a: a.ctypes.data  # noqa: E731
    lists = f["lists"]
    checked = 0
    rng = np.random.default_rng(0)
    cand = [t for t, c in enumerate(lists) if c["n_clusters"] >= 2]
    for t in rng.choice(cand, size=min(120, len(cand)), replace=False):
        c = lists[t]
        ids, vals = _posting_codes(docs, codes, t)
        if len(ids) > lam:
            order = np.lexsort((ids, -vals.astype(np.int64)))[:lam]
            kept = ids[order]
        else:
            kept = ids
        off = c["offsets"]
        blocks = [c["docs"][off[b]:off[b + 1]] for b in range(len(off) - 1)]
        assert sorted(np.concatenate(blocks).tolist()) == sorted(kept.tolist())
        cents = np.array([b[0] for b in blocks], np.int32)
        out_docs = np.empty(len(kept), np.int32)
        out_off = np.empty(len(cents) + 1, np.int32)
        kept = np.ascontiguousarray(kept, np.int32)
        assert L.ref_map_docs_to_clusters(docs.dim, 1, docs.n, P(docs.indptr), P(docs.indices),
                                          P(codes), P(kept), len(kept), P(cents), len(cents),
                                          P(out_docs), P(out_off)) == 0
        ref_blocks = [out_docs[out_off[b]:out_off[b + 1]] for b in range(len(cents))]
        for mine, theirs in zip(blocks, ref_blocks):
            np.testing.assert_array_equal(mine, theirs)
        # summaries of these clusters
        cap = 1 << 22
        buf = np.empty(cap, np.uint8)
        n = L.ref_summarize(docs.dim, 1, docs.n, P(docs.indptr), P(docs.indices), P(codes),
                            P(c["docs"]), P(off), len(off) - 1, alpha, P(buf), cap)
        assert n > 0
        r = O._read_clusters(O._Rd(bytes(buf[:n])))
        mine_cnt = np.bincount(c["csc_cluster"], minlength=len(off) - 1)
        ref_cnt = np.bincount(r["csc_cluster"], minlength=len(off) - 1)
        np.testing.assert_array_equal(mine_cnt, ref_cnt)
        for b in range(len(off) - 1):
            mv = np.sort(c["csc_value"][c["csc_cluster"] == b])
            rv = np.sort(r["csc_value"][r["csc_cluster"] == b])
            np.testing.assert_array_equal(mv, rv)
        checked += 1
    assert checked > 50


@pytest.mark.parametrize("lam,beta,alpha", [(400, 2, 0.4), (400, 40, 0.1), (400, 40, 1.0),
                                             (400, 2, 1.5), (60, 1, 0.7)])
def test_sq_summaries_match_reference_on_large_blocks_and_edge_alphas(tmp_path, lam, beta,
                                                                        alpha):
    """uint8 summaries are made per block in shared memory, by a hash-table
    kernel (blocks of up to 3,072 entries) or a per-term-table kernel (larger
    blocks: beta 1-2 puts 60-200 docs in a block). For every list, the
    reference's summarizer over the engine's blocks gives each block the
    engine's entry count and values, at an alpha that keeps little (0.1),
    one that ends at the last nonzero maximum (1.0) and one no running sum
    reaches (1.5: every pair kept)."""
    docs = synth.docs_config0(6000, seed=9)
    vmin, vmax = float(docs.values.min()), float(docs.values.max())
    spec = (f"seismic_sq,quantizer=8bit|vmin={vmin!r}|vmax={vmax!r}|lambda={lam}|beta={beta}|"
            f"alpha={alpha}|seed=7")
    device_build(docs, spec, tmp_path / "q.idx")
    f = O.read_index_file(str(tmp_path / "q.idx"))
    codes = O.sq_encode_u8(vmin, vmax, docs.values)
    L = O.ref_lib("generic")
    P = lambda a: a.ctypes.data  # noqa: E731
    lens = np.diff(docs.indptr)
    lists = [c for c in f["lists"] if len(c["offsets"]) >= 2]
    largest = [c for c in lists if lens[c["docs"]].sum() > 3072]  # lists with a large block
    rng = np.random.default_rng(2)
    sample = [lists[i] for i in rng.choice(len(lists), min(150, len(lists)), replace=False)]
    big = 0
    checked = 0
    cap = 1 << 24
    buf = np.empty(cap, np.uint8)
    for c in largest[:150] + sample:
        off = c["offsets"]
        n = L.ref_summarize(docs.dim, 1, docs.n, P(docs.indptr), P(docs.indices), P(codes),
                            P(c["docs"]), P(off), len(off) - 1, alpha, P(buf), cap)
        assert n > 0
        r = O._read_clusters(O._Rd(bytes(buf[:n])))
        nb = len(off) - 1
        np.testing.assert_array_equal(np.bincount(c["csc_cluster"], minlength=nb),
                                      np.bincount(r["csc_cluster"], minlength=nb))
        for b in range(nb):
            np.testing.assert_array_equal(np.sort(c["csc_value"][c["csc_cluster"] == b]),
                                          np.sort(r["csc_value"][r["csc_cluster"] == b]))
            big += int(lens[c["docs"][off[b]:off[b + 1]]].sum() > 3072)
        checked += 1
    assert checked > 100
    if beta <= 2:
        assert big > 0  # the per-term-table kernel ran


def test_sq_build_full_size_lists_match_reference_assigner(tmp_path):
    """The 8.8M-doc build's list shape at 1M docs: postings capped at 6,000 and
    600 blocks per full list (uint8 codes, config-2 generator). For the 12
    longest lists and 12 other full ones, the reference's assigner, given the engine's kept list and
    centroids, produces the engine's blocks exactly."""
    docs = synth.docs_config2(1_000_000, seed=3)
    vmin, vmax = float(docs.values.min()), float(docs.values.max())
    lam, beta = 6000, 600
    device_build(docs, sq_spec(vmin, vmax, lam, beta), tmp_path / "big.idx")
    f = O.read_index_file(str(tmp_path / "big.idx"))
    lists = f["lists"]
    codes = O.sq_encode_u8(vmin, vmax, docs.values)
    full = [t for t, c in enumerate(lists) if c["n_clusters"] == beta]
    assert len(full) >= 24
    n_trunc = 0
    by_len = sorted(full, key=lambda t: -len(lists[t]["docs"]))
    rest = np.random.default_rng(1).choice(by_len[12:], 12, replace=False)
    chosen = np.array(sorted(list(by_len[:12]) + list(rest)))
    pos = np.flatnonzero(np.isin(docs.indices, chosen))
    rows = (np.searchsorted(docs.indptr, pos, side="right") - 1).astype(np.int32)
    terms = docs.indices[pos]
    L = O.ref_lib("generic")
    P = lambda a: a.ctypes.data  # noqa: E731
    for t in chosen:
        m = terms == t
        ids, vals = rows[m], codes[pos[m]]
        # a list longer than the cap keeps its top codes in value order
        # (inverted_lists.cpp:110-132); a shorter one keeps doc order
        kept = ids[np.lexsort((ids, -vals.astype(np.int64)))[:lam]] if len(ids) > lam else ids
        c = lists[t]
        off = c["offsets"]
        blocks = [c["docs"][off[b]:off[b + 1]] for b in range(len(off) - 1)]
        assert sorted(np.concatenate(blocks).tolist()) == sorted(kept.tolist())
        cents = np.array([b[0] for b in blocks], np.int32)
        out_docs = np.empty(len(kept), np.int32)
        out_off = np.empty(len(cents) + 1, np.int32)
        kept = np.ascontiguousarray(kept, np.int32)
        assert L.ref_map_docs_to_clusters(docs.dim, 1, docs.n, P(docs.indptr), P(docs.indices),
                                          P(codes), P(kept), len(kept), P(cents), len(cents),
                                          P(out_docs), P(out_off)) == 0
        for b in range(len(cents)):
            np.testing.assert_array_equal(blocks[b], out_docs[out_off[b]:out_off[b + 1]])
        n_trunc += len(ids) > lam
    assert n_trunc >= 4  # capped lists among those checked


def test_sq_build_search_recall_matches_reference(tmp_path):
    docs = synth.docs_config0(20000, seed=4)
    qs = synth.queries_config0(200, seed=4)
    vmin, vmax = float(docs.values.min()), float(docs.values.max())
    spec = sq_spec(vmin, vmax, 400, 40)
    idx = device_build(docs, spec)
    r = ref_file(docs, spec, tmp_path / "r.idx")
    D, L = idx.search(qs.n, qs.indptr, qs.indices, qs.values, K,
                      nsparse.SeismicSearchParameters(10, 0.8))
    _, Lr = r.search(qs, K, param_kind=2, cut=10, heap_factor=0.8)
    _, Lt = O.exact_search(docs, qs, K, 1)
    assert recall(L, Lt) >= recall(Lr, Lt) - 0.01


def test_build_rejects_out_of_range_terms():
    docs, _ = golden_corpus()
    idx = nsparse.index_factory(1000, SEISMIC)
    idx.add(docs.n, docs.indptr, docs.indices, docs.values)
    with pytest.raises(ValueError, match="term_id out of range"):
        idx.build()


def test_build_of_tiny_and_empty_inputs(tmp_path):
    docs, qs = golden_corpus()
    small = docs.rows(0, 3)
    idx = device_build(small, SEISMIC, tmp_path / "s.idx")
    ref_file(small, SEISMIC, tmp_path / "r.idx")
    assert sha(tmp_path / "s.idx") == sha(tmp_path / "r.idx")
    D, L = idx.search(qs.n, qs.indptr, qs.indices, qs.values, 10)
    assert (L[:, 3:] == -1).all()
