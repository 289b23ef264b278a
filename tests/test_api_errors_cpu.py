"""Argument and state errors of the index API against the reference compiled
from its sources: for every index type, the same calls succeed or raise the
same exception class (ValueError for std::invalid_argument, RuntimeError for
std::runtime_error, as swignsparse.swig:47-59 maps them). All of these fail
or finish before any device work.

Building an empty InvertedIndex, SeismicIndex or SeismicScalarQuantizedIndex
crashes the reference (a segmentation fault in its build), so that call is
not made on the reference side."""

import ctypes

import numpy as np
import pytest

import nsparse
import oracle as O

ERRORS = {0: None, 1: "ValueError", 2: "RuntimeError", 3: "IndexError", 4: "MemoryError"}
SPECS = ["brutal", "inverted", "seismic,lambda=4|beta=2|alpha=0.4|seed=1",
         "seismic_sq,quantizer=8bit|vmin=0|vmax=4|lambda=4|beta=2|alpha=0.4|seed=1",
         "idmap,brutal", "idmap,inverted"]
CRASHES_WHEN_EMPTY = ("inverted", "idmap,inverted", "seismic")

IP = np.array([0, 2, 3], np.int32)
IX = np.array([0, 5, 20], np.uint16)
IX_OUT = np.array([0, 5, 16], np.uint16)  # 16 = the dimension: accepted by add, rejected at build
VV = np.array([1, 2, 3], np.float32)
IDS = np.array([7, 9], np.int32)
QIP = np.array([0, 1], np.int32)
QIX = np.array([0], np.uint16)
QV = np.array([1], np.float32)


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def _ours(call):
    try:
        call()
        return None
    except Exception as e:  # noqa: BLE001 -- the class is the result
        return type(e).__name__


def _cases(spec, tmp_path):
    mk = lambda: nsparse.index_factory(16, spec)  # noqa: E731
    path = str(tmp_path / "e.idx")
    return {
        "add_zero": (lambda: mk().add(0, IP, IX, VV), lambda L, h: L.ref_add(h, 0, _p(IP), _p(IX), _p(VV))),
        "add_negative": (lambda: mk().add(-1, IP, IX, VV),
                         lambda L, h: L.ref_add(h, -1, _p(IP), _p(IX), _p(VV))),
        "add": (lambda: mk().add(2, IP, IX, VV), lambda L, h: L.ref_add(h, 2, _p(IP), _p(IX), _p(VV))),
        "add_term_at_dim": (lambda: mk().add(2, IP, IX_OUT, VV),
                            lambda L, h: L.ref_add(h, 2, _p(IP), _p(IX_OUT), _p(VV))),
        "add_with_ids": (lambda: mk().add_with_ids(2, IP, IX, VV, IDS),
                         lambda L, h: L.ref_add_with_ids(h, 2, _p(IP), _p(IX), _p(VV), _p(IDS))),
        "build_empty": (lambda: mk().build(), lambda L, h: L.ref_build(h)),
        "write_empty": (lambda: nsparse.write_index(mk(), path),
                        lambda L, h: L.ref_write_index(h, path.encode())),
        "search_k0": (lambda: mk().search(1, QIP, QIX, QV, 0),
                      lambda L, h: L.ref_search(h, 1, _p(QIP), _p(QIX), _p(QV), 0, None, None, 0, 10,
                                                1.0, 0.0, 1.0, 0, 0, None)),
        "search_k_negative": (lambda: mk().search(1, QIP, QIX, QV, -2),
                              lambda L, h: L.ref_search(h, 1, _p(QIP), _p(QIX), _p(QV), -2, None, None,
                                                        0, 10, 1.0, 0.0, 1.0, 0, 0, None)),
    }


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("spec", SPECS)
def test_api_errors_match_reference(spec, tmp_path):
    L = O.ref_lib("generic")
    for name, (ours_call, ref_call) in _cases(spec, tmp_path).items():
        if name == "build_empty" and spec.startswith(CRASHES_WHEN_EMPTY):
            continue
        ours = _ours(ours_call)
        h = L.ref_index_factory(16, spec.encode())
        try:
            ref = ERRORS[ref_call(L, h)]
        finally:
            L.ref_index_free(h)
        assert ours == ref, name


@pytest.mark.parametrize("spec", ["seismic,lambda=10|beta=2|alpha=0.4|seed=1",
                                  "seismic_sq,quantizer=8bit|vmin=0.0|vmax=2.0|lambda=10|beta=2|"
                                  "alpha=0.4|seed=1"])
def test_seismic_build_rejects_out_of_range_terms_before_the_device(spec):
    """build() checks every stored term against the dimension first (one scan,
    kept for later calls), so a bad corpus fails with the reference's
    exception and no device is needed to find out."""
    idx = nsparse.index_factory(10, spec)
    idx.add(2, np.array([0, 2, 3], np.int32), np.array([1, 20, 3], np.uint16),
            np.ones(3, np.float32))
    with pytest.raises(ValueError, match="term_id out of range"):
        idx.build()
    with pytest.raises(ValueError, match="term_id out of range"):
        idx.build()
