"""CSR files in the reference's two layouts (nsparse/utils/csr_layout.h), host
side only, checked against the reference compiled from its sources:

* csr_layout::convert writes the same native file, byte for byte, and
  rejects the same malformed inputs with the same exception type
  (tests/csr_layout_test.cpp in the reference lists the cases);
* SeismicIndex::read_csr(path, Residency::kMmap) reads the native layout
  with the mapped reader's checks (tests/mmap_index_test.cpp), and the
  vectors it holds afterwards are written out exactly as the reference
  writes its own, while a quantized index refuses the mapped residency.
"""

import os

import numpy as np
import pytest

import nsparse
import oracle as O
from nsparse_b200 import synth

need_ref = pytest.mark.skipif(not O.ref_available(), reason="reference library not built")
SEISMIC = "seismic,lambda=200|beta=20|alpha=0.4|seed=7"
ERRORS = {1: ValueError, 2: RuntimeError, 3: IndexError, 4: MemoryError}


def write_interchange(path, rows, cols, nnz, indptr, indices, values, extra=b""):
    with open(path, "wb") as f:
        f.write(np.array([rows, cols, nnz], np.int64).tobytes())
        f.write(np.asarray(indptr, np.int64).tobytes())
        f.write(np.asarray(indices, np.int32).tobytes())
        f.write(np.asarray(values, np.float32).tobytes())
        f.write(extra)


def write_native(path, rows, cols, nnz, indptr, indices, values):
    """The native layout written directly (as the reference's tests do),
    including files whose header disagrees with their arrays."""
    with open(path, "wb") as f:
        f.write(np.array([rows, cols, nnz], np.int64).tobytes())
        f.write(np.asarray(indptr, np.int32).tobytes())
        f.write(np.asarray(indices, np.uint16).tobytes())
        f.write(b"\0" * nsparse.padding(f.tell()))
        f.write(np.asarray(values, np.float32).tobytes())


def corpus_file(path, docs):
    write_interchange(path, docs.n, docs.dim, docs.nnz, docs.indptr, docs.indices, docs.values)


def ours_convert(src, dst):
    try:
        nsparse.convert(src, dst)
        return None
    except Exception as e:  # noqa: BLE001 -- the class is the result
        return type(e)


def ref_convert(src, dst):
    rc, _ = O.ref_csr_convert(src, dst)
    return None if rc == 0 else ERRORS[rc]


def test_layout_sizes():
    assert nsparse.padding(24) == 0 and nsparse.padding(26) == 2 and nsparse.padding(27) == 1
    assert nsparse.native_path("x.csr") == "x.csr.mcsr"
    assert nsparse.interchange_file_size(2, 4) == 72  # 24 + 16 + 16 + 16
    assert nsparse.native_file_size(2, 4) == 56       # 24 + 8 + 8, no padding, 16
    assert nsparse.native_file_size(4, 3) == 60  # 24 + 16 + 6, 2 bytes of padding, 12


@need_ref
@pytest.mark.parametrize("case", ["corpus", "odd", "even", "empty", "chunks"])
def test_convert_writes_the_reference_file(tmp_path, case):
    if case == "corpus":
        corpus_file(tmp_path / "a.csr", synth.docs_config0(500, seed=3))
    elif case == "odd":
        write_interchange(tmp_path / "a.csr", 3, 4, 3, [0, 2, 2, 3], [0, 2, 1], [1.5, 2.5, 3.5])
    elif case == "even":
        write_interchange(tmp_path / "a.csr", 2, 4, 2, [0, 1, 2], [0, 3], [1.0, 2.0])
    elif case == "empty":
        write_interchange(tmp_path / "a.csr", 2, 4, 0, [0, 0, 0], [], [])
    else:  # more nonzeros than one streamed chunk
        n = 70001
        rng = np.random.default_rng(1)
        write_interchange(tmp_path / "a.csr", 1, 30522, n, [0, n], rng.integers(0, 30522, n),
                          rng.random(n))
    assert ours_convert(tmp_path / "a.csr", tmp_path / "ours.mcsr") is None
    assert ref_convert(tmp_path / "a.csr", tmp_path / "ref.mcsr") is None
    assert open(tmp_path / "ours.mcsr", "rb").read() == open(tmp_path / "ref.mcsr", "rb").read()


@need_ref
@pytest.mark.parametrize("case", [
    "missing", "short_header", "zero_rows", "zero_cols", "negative_nnz", "short_file",
    "trailing_bytes", "native_input", "indptr_start", "indptr_end", "negative_indptr",
    "negative_term", "term_beyond_cols", "term_wider_than_u16", "unwritable_destination"])
def test_convert_rejects_what_the_reference_rejects(tmp_path, case):
    src, dst = tmp_path / "a.csr", tmp_path / "out.mcsr"
    if case == "short_header":
        open(src, "wb").write(b"\0" * 10)
    elif case == "zero_rows":
        write_interchange(src, 0, 4, 0, [0], [], [])
    elif case == "zero_cols":
        write_interchange(src, 1, 0, 0, [0, 0], [], [])
    elif case == "negative_nnz":
        write_interchange(src, 1, 4, -1, [0, 0], [], [])
    elif case == "short_file":
        write_interchange(src, 2, 4, 3, [0, 1, 3], [0, 1], [1.0, 2.0])
    elif case == "trailing_bytes":
        write_interchange(src, 1, 4, 1, [0, 1], [0], [1.0], extra=b"\0" * 4)
    elif case == "native_input":
        write_native(src, 1, 4, 4, [0, 4], [0, 1, 2, 3], [1, 2, 3, 4])
        os.truncate(src, os.path.getsize(src) - 4)  # 60 bytes: neither layout's size
    elif case == "indptr_start":
        write_interchange(src, 1, 4, 1, [1, 1], [0], [1.0])
    elif case == "indptr_end":
        write_interchange(src, 2, 4, 2, [0, 1, 1], [0, 1], [1.0, 2.0])
    elif case == "negative_indptr":
        write_interchange(src, 2, 4, 1, [0, -1, 1], [0], [1.0])
    elif case == "negative_term":
        write_interchange(src, 1, 4, 1, [0, 1], [-1], [1.0])
    elif case == "term_beyond_cols":
        write_interchange(src, 1, 4, 1, [0, 1], [4], [1.0])
    elif case == "term_wider_than_u16":
        write_interchange(src, 1, 70000, 1, [0, 1], [65536], [1.0])
    elif case == "unwritable_destination":
        write_interchange(src, 1, 4, 1, [0, 1], [0], [1.0])
        dst = tmp_path / "no_such_dir" / "out.mcsr"
    ours, ref = ours_convert(src, dst), ref_convert(src, dst)
    assert ref is not None
    assert ours is ref


@need_ref
def test_mapped_read_holds_the_reference_vectors(tmp_path):
    docs = synth.docs_config0(800, seed=4)
    corpus_file(tmp_path / "a.csr", docs)
    nsparse.convert(tmp_path / "a.csr", tmp_path / "a.mcsr")
    ours = nsparse.index_factory(docs.dim, SEISMIC)
    ours.read_csr(tmp_path / "a.mcsr", nsparse.Residency_kMmap)
    assert ours.num_vectors() == docs.n
    ref = O.RefIndex(docs.dim, SEISMIC)
    ref.read_csr(tmp_path / "a.mcsr", 1)
    nsparse.write_index(ours, tmp_path / "ours.idx")
    ref.write(tmp_path / "ref.idx")
    assert open(tmp_path / "ours.idx", "rb").read() == open(tmp_path / "ref.idx", "rb").read()
    # in-memory residency on the same index type takes the interchange file
    again = nsparse.index_factory(docs.dim, SEISMIC)
    again.read_csr(tmp_path / "a.csr", nsparse.Residency_kInMemory)
    assert again.num_vectors() == docs.n


def _ours_read(dim, path, residency, spec=SEISMIC, twice=False):
    idx = nsparse.index_factory(dim, spec)
    try:
        idx.read_csr(path, residency)
        if twice:
            idx.read_csr(path, residency)
        return None
    except Exception as e:  # noqa: BLE001
        return type(e)


def _ref_read(dim, path, residency, spec=SEISMIC, twice=False):
    r = O.RefIndex(dim, spec)
    try:
        for _ in range(2 if twice else 1):
            rc = r.L.ref_read_csr(r.h, str(path).encode(), int(residency))
            if rc != 0:
                return ERRORS[rc]
        return None
    finally:
        r.close()


@need_ref
@pytest.mark.parametrize("case", [
    "ok", "missing", "widened", "truncated", "zero_rows", "cols_beyond_dim", "indptr_end",
    "decreasing_indptr", "unchecked_term", "second_load"])
def test_mapped_read_checks_as_the_reference(tmp_path, case):
    p = tmp_path / "m.mcsr"
    dim = 4
    twice = False
    if case in ("ok", "second_load"):
        write_native(p, 3, 4, 3, [0, 2, 2, 3], [0, 2, 1], [1.5, 2.5, 3.5])
        twice = case == "second_load"
    elif case == "widened":
        write_interchange(p, 2, 4, 2, [0, 1, 2], [0, 1], [1.0, 2.0])
    elif case == "truncated":
        write_native(p, 2, 4, 3, [0, 1, 3], [0, 1], [1.0, 2.0])
    elif case == "zero_rows":
        write_native(p, 0, 4, 0, [0], [], [])
    elif case == "cols_beyond_dim":
        write_native(p, 1, 8, 1, [0, 1], [0], [1.0])
    elif case == "indptr_end":
        write_native(p, 2, 4, 3, [0, 1, 2], [0, 1, 2], [1.0, 2.0, 3.0])
    elif case == "decreasing_indptr":
        write_native(p, 3, 4, 2, [0, 2, 1, 2], [0, 1], [1.0, 2.0])
    elif case == "unchecked_term":  # the mapped reader trusts convert() to have checked terms
        write_native(p, 1, 4, 1, [0, 1], [4], [1.0])
    ours = _ours_read(dim, p, 1, twice=twice)
    ref = _ref_read(dim, p, 1, twice=twice)
    assert ours is ref
    if case == "second_load":
        assert ours is RuntimeError
    if case in ("ok", "unchecked_term"):
        assert ours is None


@need_ref
def test_quantized_index_refuses_the_mapped_residency(tmp_path):
    write_native(tmp_path / "m.mcsr", 1, 4, 1, [0, 1], [0], [1.0])
    spec = "seismic_sq,quantizer=8bit|vmin=0.0|vmax=2.0|lambda=10|beta=2|alpha=0.4|seed=1"
    assert _ours_read(4, tmp_path / "m.mcsr", 1, spec) is ValueError
    assert _ref_read(4, tmp_path / "m.mcsr", 1, spec) is ValueError


@need_ref
@pytest.mark.parametrize("spec", [
    "brutal", "inverted", "idmap,seismic,lambda=10|beta=2|alpha=0.4|seed=1",
    "seismic_sq,quantizer=8bit|vmin=0.0|vmax=2.0|lambda=10|beta=2|alpha=0.4|seed=1",
    "seismic,lambda=10|beta=2|alpha=0.4|seed=1"])
def test_read_csr_layout_and_residency_matrix(tmp_path, spec):
    """Every index type, either layout, either residency: loads the same
    vectors or raises the same exception class as the reference (only a
    seismic index reads the native layout, and only under kMmap)."""
    write_interchange(tmp_path / "i.csr", 2, 4, 2, [0, 1, 2], [0, 3], [1.0, 2.0])
    write_native(tmp_path / "n.mcsr", 2, 4, 2, [0, 1, 2], [0, 3], [1.0, 2.0])
    for path in (tmp_path / "i.csr", tmp_path / "n.mcsr"):
        for res in (0, 1):
            idx = nsparse.index_factory(4, spec)
            try:
                idx.read_csr(path, res)
                ours = idx.num_vectors()
            except Exception as e:  # noqa: BLE001
                ours = type(e)
            r = O.RefIndex(4, spec)
            rc = r.L.ref_read_csr(r.h, str(path).encode(), res)
            ref = r.num_vectors() if rc == 0 else ERRORS[rc]
            r.close()
            assert ours == ref, (path.name, res)
