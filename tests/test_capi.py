"""The C ABI without a GPU: the library loads, exports what include/nsparse_c.h
declares, and its host-side behaviour (factory, argument checks, selectors,
parameters, error mapping) matches the reference's API
(python_tests/test_error_paths.py)."""

import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import nsparse
from helpers import ROOT

HEADER = os.path.join(ROOT, "include", "nsparse_c.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(nsp_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(nsparse.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", nsparse.LIB_PATH], capture_output=True,
                         text=True).stdout
    exported = set(re.findall(r" T (nsp_[a-z_]+)", out))
    assert set(declared_symbols()) <= exported


def small_csr(n=5, dim=64, nnz=4, seed=0):
    rng = np.random.default_rng(seed)
    indptr = np.arange(0, (n + 1) * nnz, nnz, dtype=np.int32)
    idx = np.concatenate([np.sort(rng.choice(dim, nnz, replace=False)) for _ in range(n)])
    vals = rng.uniform(0.1, 1.0, n * nnz).astype(np.float32)
    return indptr, idx.astype(np.uint16), vals


@pytest.mark.parametrize("desc,msg", [("nonsense", "Unknown index type"),
                                      ("", "Description cannot be null or empty"),
                                      ("idmap", "idmap requires a delegate index type")])
def test_bad_index_spec_raises(desc, msg):
    with pytest.raises(ValueError, match=msg):
        nsparse.index_factory(64, desc)


@pytest.mark.parametrize("desc,cls,fourcc", [
    ("brutal", nsparse.BrutalIndex, "BRUT"),
    ("inverted", nsparse.InvertedIndex, "INVT"),
    ("seismic,lambda=10|beta=2|alpha=0.4", nsparse.SeismicIndex, "SEIS"),
    ("seismic_sq,quantizer=8bit|vmin=0|vmax=1", nsparse.SeismicScalarQuantizedIndex, "SESQ"),
    ("idmap,seismic", nsparse.IDMapIndex, "IDMP"),
])
def test_factory_types(desc, cls, fourcc):
    idx = nsparse.index_factory(64, desc)
    assert isinstance(idx, cls)
    assert idx.id() == fourcc
    # IDMapIndex keeps dimension 0, as the reference's constructor leaves it
    assert idx.get_dimension() == (0 if fourcc == "IDMP" else 64)
    assert idx.num_vectors() == 0


def test_add_counts_vectors_without_gpu():
    idx = nsparse.index_factory(64, "brutal")
    ip, ix, v = small_csr()
    idx.add(5, ip, ix, v)
    idx.add(5, ip, ix, v)
    assert idx.num_vectors() == 10


def test_add_rejects_bad_arguments():
    idx = nsparse.index_factory(64, "inverted")
    ip, ix, v = small_csr()
    with pytest.raises(ValueError, match="must be positive"):
        idx.add(0, ip, ix, v)
    with pytest.raises(TypeError, match="float32"):
        idx.add(5, ip, ix, v.astype(np.float64))
    with pytest.raises(TypeError, match="int32"):
        idx.add(5, ip.astype(np.int64), ix, v)


def test_non_positive_k_raises():
    idx = nsparse.index_factory(64, "inverted")
    ip, ix, v = small_csr()
    with pytest.raises(ValueError, match="must be positive"):
        idx.search(5, ip, ix, v, 0)


def test_build_on_brutal_raises():
    idx = nsparse.index_factory(64, "brutal")
    with pytest.raises(RuntimeError, match="not implemented"):
        idx.build()


def test_term_id_out_of_range_raises_at_build():
    idx = nsparse.index_factory(64, "inverted")
    ip, ix, v = small_csr()
    ix = ix.copy()
    ix[0] = 64
    idx.add(5, ip, ix, v)  # accepted at add, as in the reference
    with pytest.raises(ValueError, match="term_id out of range"):
        idx.build()


def test_write_index_on_brutal_raises(tmp_path):
    idx = nsparse.index_factory(64, "brutal")
    ip, ix, v = small_csr()
    idx.add(5, ip, ix, v)
    with pytest.raises(RuntimeError, match="does not support"):
        nsparse.write_index(idx, str(tmp_path / "b.idx"))
    assert not (tmp_path / "b.idx").exists()


def test_add_with_ids_needs_idmap():
    idx = nsparse.index_factory(64, "brutal")
    ip, ix, v = small_csr()
    with pytest.raises(RuntimeError, match="add_with_ids not implemented"):
        idx.add_with_ids(5, ip, ix, v, np.arange(5, dtype=np.int32))
    m = nsparse.index_factory(64, "idmap,brutal")
    m.add_with_ids(5, ip, ix, v, np.arange(100, 105, dtype=np.int32))
    assert m.num_vectors() == 5


def test_selectors_membership():
    s = nsparse.SetIDSelector(np.array([1, 5, 9], np.int32))
    assert s.is_member(5) and not s.is_member(4)
    a = nsparse.ArrayIDSelector(np.array([2, 3], np.int32))
    assert a(3) and not a(1)
    n = nsparse.NotIDSelector(s)
    assert n.is_member(4) and not n.is_member(9)
    bits = np.zeros(2, np.uint64)
    bits[0] = np.uint64(0b1010)
    b = nsparse.BitmapIDSelector(70, bits)
    assert b.is_member(1) and b.is_member(3) and not b.is_member(2) and not b.is_member(100)


def test_search_params():
    p = nsparse.SeismicSearchParameters(12, 0.9)
    assert (p.cut, p.heap_factor) == (12, pytest.approx(0.9))
    s = nsparse.SetIDSelector(np.array([1], np.int32))
    p.set_id_selector(s)
    assert p.get_id_selector() is s
    p.set_engine(plain=True, warps_per_block=2)
    with pytest.raises(ValueError):
        p.set_engine(False, 99)
    q = nsparse.SeismicSQSearchParameters(0.0, 2.0, 10, 1.0)
    assert q.vmax == 2.0


def test_kernel_and_engine_knobs_are_validated():
    p = nsparse.SeismicSearchParameters(10, 1.0)
    for variant, tuning in ((-1, 0), (0, 0), (1, 4096), (2, 256), (5, 8192)):
        p.set_kernel(variant, tuning)
    for variant, tuning in ((-2, 0), (6, 0), (2, 8193), (1, 1 << 20), (3, -1)):
        with pytest.raises(ValueError):
            p.set_kernel(variant, tuning)
    p.set_engine(False, 32)
    with pytest.raises(ValueError):
        p.set_engine(False, 33)
    for split in (0, 1, 2, 4, 8):
        p.set_split(split)
    for split in (-1, 3, 16):
        with pytest.raises(ValueError):
            p.set_split(split)


def test_autotune_and_server_need_a_seismic_index():
    idx = nsparse.index_factory(64, "brutal")
    ip, ix, v = small_csr()
    idx.add(5, ip, ix, v)
    with pytest.raises(ValueError, match="seismic"):
        idx.autotune(5, ip, ix, v, 3)
    with pytest.raises(ValueError, match="seismic"):
        nsparse.Server(idx)
    with pytest.raises(ValueError, match="must not be negative"):
        nsparse.Server(nsparse.index_factory(64, "seismic"), max_batch=-1)


def test_quantizer_range_is_validated():
    with pytest.raises(ValueError, match="vmax must be greater than vmin"):
        nsparse.index_factory(64, "seismic_sq,quantizer=8bit|vmin=1|vmax=1")
    with pytest.raises(ValueError, match="finite"):
        nsparse.index_factory(64, "seismic_sq,quantizer=8bit|vmin=0|vmax=inf")


def test_read_csr_errors(tmp_path):
    idx = nsparse.index_factory(64, "brutal")
    with pytest.raises(ValueError, match="does not exist"):
        idx.read_csr(str(tmp_path / "missing.csr"))
    # interchange layout: int64 header, int64 indptr, int32 indices, f32 values
    p = tmp_path / "ok.csr"
    with open(p, "wb") as f:
        np.array([2, 64, 3], np.int64).tofile(f)
        np.array([0, 2, 3], np.int64).tofile(f)
        np.array([1, 5, 7], np.int32).tofile(f)
        np.array([0.5, 0.25, 1.0], np.float32).tofile(f)
    idx.read_csr(str(p))
    assert idx.num_vectors() == 2
    bad = tmp_path / "bad.csr"
    with open(bad, "wb") as f:
        np.array([2, 64, 3], np.int64).tofile(f)
        np.array([0, 2, 3], np.int64).tofile(f)
        np.array([1, 5, 70], np.int32).tofile(f)
        np.array([0.5, 0.25, 1.0], np.float32).tofile(f)
    with pytest.raises(ValueError, match="out of range"):
        nsparse.index_factory(64, "brutal").read_csr(str(bad))


def test_import_fails_loudly_without_the_engine_library(tmp_path):
    """No fallback: a copy of the Python package with no built library beside
    it refuses to import."""
    import shutil
    import subprocess
    import sys
    src = os.path.join(ROOT, "neural-sparse-cpp_b200", "python", "nsparse")
    dst = tmp_path / "pkg" / "python" / "nsparse"
    shutil.copytree(src, dst, ignore=shutil.ignore_patterns("__pycache__"))
    r = subprocess.run([sys.executable, "-c", "import nsparse"], cwd=str(dst.parent),
                       capture_output=True, text=True)
    assert r.returncode != 0
    assert "ImportError" in r.stderr and "engine library not found" in r.stderr
