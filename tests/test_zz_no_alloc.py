"""The SEISMIC search entry point that allocates nothing
(nsp_index_search_device_noalloc), for callers that cannot allocate device
memory per call -- an engine inside a host that accounts for every device byte
against a fixed budget, or a loop that cannot absorb cudaMalloc/cudaFree
stalls. It must return exactly what nsp_index_search_device returns, call
after call, while its scratch lives in the library's fixed device array; and a
caller's wrong row bound must cost padding and a status code, never memory
outside the kernel's buffers.

Collected last (file name), so a run that stops at the first failure has
already run every other test; it builds its own indexes, so it also passes
alone in a fresh process.
"""

import ctypes

import numpy as np
import pytest
import torch

import nsparse
from helpers import CUT, HF, K, SEISMIC, golden_corpus, sq_spec
from nsparse_b200 import synth

pytestmark = pytest.mark.gpu

_P = ctypes.c_void_p
_fn = nsparse._L.nsp_index_search_device_noalloc
_fn.restype = ctypes.c_int
_fn.argtypes = [_P, ctypes.c_int32, _P, _P, _P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int,
                _P, _P, _P, _P, _P]


def _resident_index(spec, docs, qs, params):
    idx = nsparse.index_factory(docs.dim, spec)
    idx.add(docs.n, docs.indptr, docs.indices, docs.values)
    idx.build()
    idx.search(qs.n, qs.indptr, qs.indices, qs.values, K, params)  # uploads the index
    return idx


def _device_inputs(qs):
    dev = torch.device("cuda", 0)
    return (torch.from_numpy(qs.indptr).to(dev),
            torch.from_numpy(qs.indices.view(np.int16)).to(dev),
            torch.from_numpy(qs.values).to(dev))


def _outputs(n):
    dev = torch.device("cuda", 0)
    return (torch.full((n, K), 7.0, dtype=torch.float32, device=dev),
            torch.full((n, K), 7, dtype=torch.int32, device=dev))


def _status():
    return torch.full((1,), -5, dtype=torch.int32, device=torch.device("cuda", 0))


def _noalloc(idx, qs, inputs, nnz, max_nnz, params, stream, status):
    ip, ix, v = inputs
    d, l = _outputs(qs.n)
    rc = _fn(idx._h, qs.n, ip.data_ptr(), ix.data_ptr(), v.data_ptr(), nnz, max_nnz, K,
             d.data_ptr(), l.data_ptr(), params._h, stream.cuda_stream,
             None if status is None else status.data_ptr())
    assert rc == 0, nsparse._L.nsp_last_error().decode()
    return d, l


def _device_search(idx, qs, inputs, max_nnz, params, stream):
    ip, ix, v = inputs
    d, l = _outputs(qs.n)
    idx.search_device(qs.n, ip.data_ptr(), ix.data_ptr(), v.data_ptr(), max_nnz, K,
                      d.data_ptr(), l.data_ptr(), params, stream.cuda_stream)
    return d, l


@pytest.mark.parametrize("kind", ["fp32", "sq8", "sq8-query-range"])
def test_noalloc_search_matches_device_search_on_consecutive_calls(kind):
    docs, qs = golden_corpus()
    params = nsparse.SeismicSearchParameters(CUT, HF)
    if kind == "fp32":
        spec = SEISMIC
    else:
        vmin, vmax = float(docs.values.min()), float(docs.values.max())
        spec = sq_spec(vmin, vmax)
        if kind == "sq8-query-range":
            # the query quantizer's own range (SeismicSQSearchParameters)
            params = nsparse.SeismicSQSearchParameters(0.5 * vmin, 0.8 * vmax, CUT, HF)
    idx = _resident_index(spec, docs, qs, params)
    inputs = _device_inputs(qs)
    max_nnz = int(np.diff(qs.indptr).max())
    stream = torch.cuda.Stream()
    ref_d, ref_l = _device_search(idx, qs, inputs, max_nnz, params, stream)
    results = []
    for _ in range(2):
        st = _status()
        results.append((_noalloc(idx, qs, inputs, qs.nnz, max_nnz, params, stream, st), st))
    stream.synchronize()
    want_d, want_l = ref_d.cpu().numpy(), ref_l.cpu().numpy()
    for (d, l), st in results:
        # SEISMIC results are bit-identical between launches of the same kernel
        np.testing.assert_array_equal(l.cpu().numpy(), want_l)
        np.testing.assert_array_equal(d.cpu().numpy(), want_d)
        assert int(st.item()) == 0


def test_noalloc_caps_its_grid_to_the_fixed_array():
    # One list of ~14,000 single-doc blocks: a CTA's block-score rows, visiting
    # order and sort keys take ~0.6 MB, so only a few dozen CTAs fit the 32 MiB
    # array and the persistent grid is capped well below a full wave; queries
    # are still shared out by work stealing.
    docs = synth.docs_config0(20000, seed=3)
    qs = synth.queries_config0(600, seed=4)
    spec = "seismic,lambda=20000|beta=20000|alpha=0.4|seed=7"
    params = nsparse.SeismicSearchParameters(CUT, HF)
    idx = _resident_index(spec, docs, qs.rows(0, 8), params)
    counts = np.bincount(docs.indices.astype(np.int64), minlength=docs.dim)
    assert counts.max() >= 10000, "the corpus no longer has one very long list"
    inputs = _device_inputs(qs)
    max_nnz = int(np.diff(qs.indptr).max())
    stream = torch.cuda.Stream()
    ref_d, ref_l = _device_search(idx, qs, inputs, max_nnz, params, stream)
    st = _status()
    d, l = _noalloc(idx, qs, inputs, qs.nnz, max_nnz, params, stream, st)
    stream.synchronize()
    np.testing.assert_array_equal(l.cpu().numpy(), ref_l.cpu().numpy())
    np.testing.assert_array_equal(d.cpu().numpy(), ref_d.cpu().numpy())
    assert int(st.item()) == 0


@pytest.mark.parametrize("kind", ["fp32", "sq8"])
def test_noalloc_wrong_row_bounds_give_padding_and_a_status(kind):
    docs, qs = golden_corpus()
    params = nsparse.SeismicSearchParameters(CUT, HF)
    spec = SEISMIC if kind == "fp32" else sq_spec(float(docs.values.min()),
                                                  float(docs.values.max()))
    idx = _resident_index(spec, docs, qs, params)
    inputs = _device_inputs(qs)
    lens = np.diff(qs.indptr)
    max_nnz = int(lens.max())
    stream = torch.cuda.Stream()
    ref_d, ref_l = _device_search(idx, qs, inputs, max_nnz, params, stream)
    stream.synchronize()
    want_d, want_l = ref_d.cpu().numpy(), ref_l.cpu().numpy()
    # an understated row bound (and none at all): rows longer than it come
    # back as padding, every other row as before, and the status says so
    for bound in (int(np.median(lens)), 0):
        st = _status()
        d, l = _noalloc(idx, qs, inputs, qs.nnz, bound, params, stream, st)
        stream.synchronize()
        d, l = d.cpu().numpy(), l.cpu().numpy()
        long_rows = lens > max(bound, 1)
        assert long_rows.any() and int(st.item()) == 3
        assert (l[long_rows] == -1).all() and (d[long_rows] == -1.0).all()
        np.testing.assert_array_equal(l[~long_rows], want_l[~long_rows])
        np.testing.assert_array_equal(d[~long_rows], want_d[~long_rows])
    # a declared nnz short of d_indptr[n]: rows that end past it are padding
    cut_at = int(qs.indptr[qs.n // 2])
    st = _status()
    d, l = _noalloc(idx, qs, inputs, cut_at, max_nnz, params, stream, st)
    stream.synchronize()
    d, l = d.cpu().numpy(), l.cpu().numpy()
    past = qs.indptr[1:] > cut_at
    assert past.any() and int(st.item()) == 3
    assert (l[past] == -1).all() and (d[past] == -1.0).all()
    np.testing.assert_array_equal(l[~past], want_l[~past])
    # the status word is optional: the same call without it still pads
    d2, l2 = _noalloc(idx, qs, inputs, cut_at, max_nnz, params, stream, None)
    stream.synchronize()
    np.testing.assert_array_equal(l2.cpu().numpy(), l)


def test_noalloc_rejects_what_it_cannot_hold():
    docs, qs = golden_corpus()
    params = nsparse.SeismicSearchParameters(CUT, HF)
    spec = sq_spec(float(docs.values.min()), float(docs.values.max()))
    idx = _resident_index(spec, docs, qs, params)
    ip, ix, v = _device_inputs(qs)
    d, l = _outputs(qs.n)
    max_nnz = int(np.diff(qs.indptr).max())
    # codes of 2 * nnz bytes beyond the fixed array: refused before any launch
    rc = _fn(idx._h, qs.n, ip.data_ptr(), ix.data_ptr(), v.data_ptr(), 1 << 25, max_nnz, K,
             d.data_ptr(), l.data_ptr(), params._h, None, None)
    assert rc == 1 and "too large" in nsparse._L.nsp_last_error().decode()
    sel = nsparse.SetIDSelector(np.arange(50, dtype=np.int32))
    p2 = nsparse.SeismicSearchParameters(CUT, HF)
    p2.set_id_selector(sel)
    rc = _fn(idx._h, qs.n, ip.data_ptr(), ix.data_ptr(), v.data_ptr(), qs.nnz, max_nnz, K,
             d.data_ptr(), l.data_ptr(), p2._h, None, None)
    assert rc == 1 and "selector" in nsparse._L.nsp_last_error().decode()
    fresh = nsparse.index_factory(docs.dim, SEISMIC)
    fresh.add(docs.n, docs.indptr, docs.indices, docs.values)
    rc = _fn(fresh._h, qs.n, ip.data_ptr(), ix.data_ptr(), v.data_ptr(), qs.nnz, max_nnz, K,
             d.data_ptr(), l.data_ptr(), params._h, None, None)
    assert rc == 1 and "resident" in nsparse._L.nsp_last_error().decode()
    torch.cuda.synchronize()
    assert (l.cpu().numpy() == 7).all(), "a refused call wrote results"
