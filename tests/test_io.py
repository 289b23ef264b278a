"""Index files move both ways between the reference and this engine: a file the
reference wrote loads here and is written back byte for byte (no GPU needed:
loading and writing are host-side). Corrupt files are rejected on the host."""

import os

import numpy as np
import pytest

import nsparse
from nsparse_b200 import synth
import oracle as O
from helpers import SEISMIC, golden_corpus, ref_file, ref_index, sq_spec

need_ref = pytest.mark.skipif(not O.ref_available(), reason="reference library not built")


def _roundtrip_bytes(src, dst):
    idx = nsparse.read_index(str(src))
    nsparse.write_index(idx, str(dst))
    return open(src, "rb").read(), open(dst, "rb").read(), idx


@need_ref
@pytest.mark.parametrize("kind", ["seismic", "seismic_sq", "idmap", "inverted"])
def test_reference_file_roundtrip_is_byte_identical(kind, tmp_path):
    docs, _ = golden_corpus()
    if kind == "seismic":
        spec, ids = SEISMIC, None
    elif kind == "seismic_sq":
        spec, ids = sq_spec(float(docs.values.min()), float(docs.values.max())), None
    elif kind == "idmap":
        spec, ids = "idmap," + SEISMIC, (np.arange(docs.n, dtype=np.int32) * 7 + 1000)
    else:
        spec, ids = "inverted", None
    ref_file(docs, spec, tmp_path / "ref.idx", ids=ids)
    a, b, idx = _roundtrip_bytes(tmp_path / "ref.idx", tmp_path / "ours.idx")
    assert idx.num_vectors() == docs.n
    assert len(a) == len(b)
    assert a == b
    # and the reference reads ours back
    back = O.RefIndex.read(str(tmp_path / "ours.idx"))
    assert back.num_vectors() == docs.n


@need_ref
def test_mmap_flag_is_accepted(tmp_path):
    docs, _ = golden_corpus()
    ref_file(docs, SEISMIC, tmp_path / "s.idx")
    idx = nsparse.read_index(str(tmp_path / "s.idx"), nsparse.kUseMmap)
    assert idx.num_vectors() == docs.n and idx.id() == "SEIS"


@need_ref
def test_unbuilt_index_roundtrip(tmp_path):
    docs, _ = golden_corpus()
    r = ref_index(docs, SEISMIC, build=False)
    r.write(str(tmp_path / "u.idx"))
    a, b, _ = _roundtrip_bytes(tmp_path / "u.idx", tmp_path / "v.idx")
    assert a == b


@need_ref
# 4, 8, -16 and -1 are cuts the reference's own reader accepts without error
# (it returns an index built from what it read); the engine rejects every cut.
@pytest.mark.parametrize("cut_at", [3, 4, 8, 10, 100, 5000, -16, -1])
def test_truncated_file_is_rejected(tmp_path, cut_at):
    docs, _ = golden_corpus()
    ref_file(docs, SEISMIC, tmp_path / "s.idx")
    data = open(tmp_path / "s.idx", "rb").read()
    (tmp_path / "t.idx").write_bytes(data[:cut_at] if cut_at > 0 else data[:len(data) + cut_at])
    with pytest.raises(RuntimeError):
        nsparse.read_index(str(tmp_path / "t.idx"))


@need_ref
def test_corrupt_doc_id_is_rejected(tmp_path):
    docs, _ = golden_corpus()
    ref_file(docs, SEISMIC, tmp_path / "s.idx")
    f = O.read_index_file(str(tmp_path / "s.idx"))
    data = bytearray(open(tmp_path / "s.idx", "rb").read())
    # locate the first non-empty list's docs array and poison one id
    first = next(i for i, c in enumerate(f["lists"]) if len(c["docs"]) > 0)
    needle = f["lists"][first]["docs"].tobytes()
    pos = bytes(data).find(needle)
    assert pos > 0
    data[pos:pos + 4] = np.int32(docs.n + 5).tobytes()
    (tmp_path / "c.idx").write_bytes(bytes(data))
    with pytest.raises(RuntimeError, match="corrupt index file"):
        nsparse.read_index(str(tmp_path / "c.idx"))


def test_unknown_fourcc_is_rejected(tmp_path):
    p = tmp_path / "x.idx"
    p.write_bytes(b"ABCD" + np.int32(64).tobytes() + b"\0" * 64)
    with pytest.raises(RuntimeError, match="Unknown index type"):
        nsparse.read_index(str(p))


def test_missing_file(tmp_path):
    with pytest.raises(RuntimeError, match="Failed to open"):
        nsparse.read_index(str(tmp_path / "nope.idx"))


@need_ref
@pytest.mark.parametrize("bits", [8, 16])
def test_quantized_add_writes_the_reference_codes(tmp_path, bits):
    """A quantized index encodes on add, on the host: with either code width
    the unbuilt index this engine writes is the reference's byte for byte
    (header with quantizer type and range, codes, CSR layout), including
    values outside the range (clamped) and at its ends."""
    docs, _ = golden_corpus()
    vals = docs.values.copy()
    vals[:4] = [-1.0, 0.0, 1e9, float(docs.values.max())]
    docs = type(docs)(docs.dim, docs.indptr, docs.indices, vals)
    vmin, vmax = 0.05, 9.5
    spec = (f"seismic_sq,quantizer={bits}bit|vmin={vmin!r}|vmax={vmax!r}|"
            "lambda=200|beta=20|alpha=0.4|seed=7")
    ref_index(docs, spec, build=False).write(str(tmp_path / "r.idx"))
    ours = nsparse.index_factory(docs.dim, spec)
    ours.add(docs.n, docs.indptr, docs.indices, docs.values)
    nsparse.write_index(ours, str(tmp_path / "o.idx"))
    assert open(tmp_path / "o.idx", "rb").read() == open(tmp_path / "r.idx", "rb").read()


@need_ref
@pytest.mark.parametrize("bits", [8, 16])
def test_quantized_add_of_a_large_batch_writes_the_reference_codes(tmp_path, bits):
    """A batch of more than 4M values is encoded by several host threads (each
    value on its own): the written index still equals the reference's byte
    for byte."""
    docs = synth.docs_config0(100_000, seed=5)  # ~13M values
    assert docs.nnz > 3 * (1 << 22)
    vmin, vmax = float(docs.values.min()), float(np.quantile(docs.values, 0.99))
    spec = (f"seismic_sq,quantizer={bits}bit|vmin={vmin!r}|vmax={vmax!r}|"
            "lambda=200|beta=20|alpha=0.4|seed=7")
    ref_index(docs, spec, build=False).write(str(tmp_path / "r.idx"))
    ours = nsparse.index_factory(docs.dim, spec)
    ours.add(docs.n, docs.indptr, docs.indices, docs.values)
    nsparse.write_index(ours, str(tmp_path / "o.idx"))
    assert open(tmp_path / "o.idx", "rb").read() == open(tmp_path / "r.idx", "rb").read()


@need_ref
@pytest.mark.parametrize("delegate", [
    "seismic,lambda=200|beta=20|alpha=0.4|seed=7", "inverted",
    "seismic_sq,quantizer=16bit|vmin=0.1|vmax=8|lambda=200|beta=20|alpha=0.4|seed=7"])
def test_idmap_add_with_ids_writes_the_reference_file(tmp_path, delegate):
    """add_with_ids on an IDMapIndex, written before any build: the external
    id table and the delegate's vectors equal the reference's byte for byte."""
    docs, _ = golden_corpus()
    ids = np.arange(docs.n, dtype=np.int32) * 13 + 5
    spec = "idmap," + delegate
    ours = nsparse.index_factory(docs.dim, spec)
    ours.add_with_ids(docs.n, docs.indptr, docs.indices, docs.values, ids)
    nsparse.write_index(ours, str(tmp_path / "o.idx"))
    ref_index(docs, spec, build=False, ids=ids).write(str(tmp_path / "r.idx"))
    assert open(tmp_path / "o.idx", "rb").read() == open(tmp_path / "r.idx", "rb").read()
