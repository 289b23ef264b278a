"""The SEISMIC search entry point that allocates nothing
(nsp_index_search_device_noalloc), for callers that cannot allocate device
memory per call -- an engine inside a host that accounts for every device byte
against a fixed budget, or a loop that cannot absorb cudaMalloc/cudaFree
stalls. It must return exactly what nsp_index_search_device returns, call
after call, while its scratch lives in the library's fixed device array.

Collected last (file name), so a run that stops at the first failure has
already run every other test; it builds its own index, so it also passes alone
in a fresh process.
"""

import ctypes

import numpy as np
import pytest
import torch

import nsparse
from helpers import CUT, HF, K, SEISMIC, golden_corpus, sq_spec

pytestmark = pytest.mark.gpu

_P = ctypes.c_void_p
_fn = nsparse._L.nsp_index_search_device_noalloc
_fn.restype = ctypes.c_int
_fn.argtypes = [_P, ctypes.c_int32, _P, _P, _P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int,
                _P, _P, _P, _P]


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


@pytest.mark.parametrize("kind", ["fp32", "sq8"])
def test_noalloc_search_matches_device_search_on_consecutive_calls(kind):
    docs, qs = golden_corpus()
    params = nsparse.SeismicSearchParameters(CUT, HF)
    if kind == "fp32":
        spec = SEISMIC
    else:
        spec = sq_spec(float(docs.values.min()), float(docs.values.max()))
    idx = _resident_index(spec, docs, qs, params)
    ip, ix, v = _device_inputs(qs)
    max_nnz = int(np.diff(qs.indptr).max())
    stream = torch.cuda.Stream()
    ref_d, ref_l = _outputs(qs.n)
    idx.search_device(qs.n, ip.data_ptr(), ix.data_ptr(), v.data_ptr(), max_nnz, K,
                      ref_d.data_ptr(), ref_l.data_ptr(), params, stream.cuda_stream)
    results = []
    for _ in range(2):
        d, l = _outputs(qs.n)
        rc = _fn(idx._h, qs.n, ip.data_ptr(), ix.data_ptr(), v.data_ptr(), qs.nnz, max_nnz, K,
                 d.data_ptr(), l.data_ptr(), params._h, stream.cuda_stream)
        assert rc == 0, nsparse._L.nsp_last_error().decode()
        results.append((d, l))
    stream.synchronize()
    want_d, want_l = ref_d.cpu().numpy(), ref_l.cpu().numpy()
    for d, l in results:
        # SEISMIC results are bit-identical between launches of the same kernel
        np.testing.assert_array_equal(l.cpu().numpy(), want_l)
        np.testing.assert_array_equal(d.cpu().numpy(), want_d)


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
             d.data_ptr(), l.data_ptr(), params._h, None)
    assert rc == 1 and "too large" in nsparse._L.nsp_last_error().decode()
    sel = nsparse.SetIDSelector(np.arange(50, dtype=np.int32))
    p2 = nsparse.SeismicSearchParameters(CUT, HF)
    p2.set_id_selector(sel)
    rc = _fn(idx._h, qs.n, ip.data_ptr(), ix.data_ptr(), v.data_ptr(), qs.nnz, max_nnz, K,
             d.data_ptr(), l.data_ptr(), p2._h, None)
    assert rc == 1 and "selector" in nsparse._L.nsp_last_error().decode()
    fresh = nsparse.index_factory(docs.dim, SEISMIC)
    fresh.add(docs.n, docs.indptr, docs.indices, docs.values)
    rc = _fn(fresh._h, qs.n, ip.data_ptr(), ix.data_ptr(), v.data_ptr(), qs.nnz, max_nnz, K,
             d.data_ptr(), l.data_ptr(), params._h, None)
    assert rc == 1 and "resident" in nsparse._L.nsp_last_error().decode()
    torch.cuda.synchronize()
    assert (l.cpu().numpy() == 7).all(), "a refused call wrote results"
