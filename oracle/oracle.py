"""TEST INFRASTRUCTURE -- the checker, never the product.

ctypes access to
  * ``_bin/libnsp_oracle.so``: the plain-C restatement (nsp_oracle.c), and
  * ``_ref/libnsparse_ref_<variant>.so``: the reference library compiled from
    its own sources (Makefile target ``ref``), wrapped by ref_harness.cpp,
plus a reader for the reference's index file layout (io/index_io.cpp:88-163,
sparse_vectors.cpp:206-231, cluster/inverted_list_clusters.cpp:333-363,
io/align.h:43-104) that flattens a SEISMIC index into the arrays
``nspo_seismic_search`` takes.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.
"""

from __future__ import annotations

import ctypes
import os
import struct
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
P = ctypes.c_void_p
I32 = ctypes.c_int32
I64 = ctypes.c_int64


def _ptr(a):
    return None if a is None else a.ctypes.data


# ---------------------------------------------------------------- C oracle --

_OR = None


def lib():
    global _OR
    if _OR is None:
        L = ctypes.CDLL(os.path.join(HERE, "_bin", "libnsp_oracle.so"))
        L.nspo_exact_search.restype = ctypes.c_int
        L.nspo_exact_search.argtypes = [ctypes.c_int, I32, P, P, P, I32, P, P, P,
                                        ctypes.c_int, ctypes.c_int, P, P, P]
        L.nspo_seismic_search.restype = ctypes.c_int
        L.nspo_seismic_search.argtypes = [
            ctypes.c_int, ctypes.c_int, I32, P, P, P, I32, P, P, P, P, P, P, P, P,
            I32, P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_float, P, P, P, P]
        L.nspo_sq_encode_u8.restype = None
        L.nspo_sq_encode_u8.argtypes = [ctypes.c_float, ctypes.c_float, P, P, I64]
        L.nspo_sq_encode_u16.restype = None
        L.nspo_sq_encode_u16.argtypes = [ctypes.c_float, ctypes.c_float, P, P, I64]
        L.nspo_sq_scale.restype = ctypes.c_float
        L.nspo_sq_scale.argtypes = [ctypes.c_int] + [ctypes.c_float] * 4
        L.nspo_cut.restype = ctypes.c_int
        L.nspo_cut.argtypes = [P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P]
        _OR = L
    return _OR


def bitmap_from_ids(n_docs: int, ids) -> np.ndarray:
    bits = np.zeros((n_docs + 64) // 64, dtype=np.uint64)
    ids = np.asarray(ids, dtype=np.int64)
    ids = ids[(ids >= 0) & (ids < n_docs)]
    np.bitwise_or.at(bits, ids >> 6, np.left_shift(np.uint64(1), (ids & 63).astype(np.uint64)))
    return bits


def exact_search(docs, queries, k, mode, sel_bits=None):
    """mode 0 = brutal semantics, 1 = inverted semantics (positive only)."""
    n_q = queries.n
    D = np.empty((n_q, k), dtype=np.float32)
    L = np.empty((n_q, k), dtype=np.int32)
    rc = lib().nspo_exact_search(docs.dim, docs.n, _ptr(docs.indptr), _ptr(docs.indices),
                                 _ptr(docs.values), n_q, _ptr(queries.indptr),
                                 _ptr(queries.indices), _ptr(queries.values), k, mode,
                                 _ptr(sel_bits), _ptr(D), _ptr(L))
    assert rc == 0
    return D, L


@dataclass
class SeismicArrays:
    """A SEISMIC index flattened over its posting lists (one list per term)."""

    esz: int
    list_block_ptr: np.ndarray  # int64 [n_lists+1]
    block_doc_ptr: np.ndarray   # int64 [n_blocks+1]
    docs: np.ndarray            # int32
    list_term_ptr: np.ndarray   # int64 [n_lists+1]
    sum_terms: np.ndarray       # uint16
    sum_run_ptr: np.ndarray     # int64 [n_terms_total+1]
    sum_block: np.ndarray       # uint16 (block id local to its list)
    sum_val: np.ndarray         # float32 or uint8

    @property
    def n_lists(self):
        return len(self.list_block_ptr) - 1


def seismic_search(fwd, fwd_values, arrays: SeismicArrays, queries_indptr,
                   queries_indices, queries_values, k, cut, heap_factor,
                   sel_bits=None, want_stats=False):
    """fwd: Csr-like (dim, n, indptr, indices); fwd_values float32, uint16 or
    uint8 codes; queries_values float32 (esz 4), uint16 codes (esz 2) or uint8
    codes (esz 1)."""
    n_q = len(queries_indptr) - 1
    D = np.empty((n_q, k), dtype=np.float32)
    L = np.empty((n_q, k), dtype=np.int32)
    stats = np.zeros((n_q, 4), dtype=np.int64) if want_stats else None
    a = arrays
    rc = lib().nspo_seismic_search(
        fwd.dim, a.esz, fwd.n, _ptr(fwd.indptr), _ptr(fwd.indices), _ptr(fwd_values),
        a.n_lists, _ptr(a.list_block_ptr), _ptr(a.block_doc_ptr), _ptr(a.docs),
        _ptr(a.list_term_ptr), _ptr(a.sum_terms), _ptr(a.sum_run_ptr),
        _ptr(a.sum_block), _ptr(a.sum_val), n_q, _ptr(queries_indptr),
        _ptr(queries_indices), _ptr(queries_values), k, cut, heap_factor,
        _ptr(sel_bits), _ptr(D), _ptr(L), _ptr(stats))
    assert rc == 0
    return (D, L, stats) if want_stats else (D, L)


def sq_encode_u8(vmin, vmax, vals):
    vals = np.ascontiguousarray(vals, dtype=np.float32)
    out = np.empty(len(vals), dtype=np.uint8)
    lib().nspo_sq_encode_u8(vmin, vmax, _ptr(vals), _ptr(out), len(vals))
    return out


def sq_encode_u16(vmin, vmax, vals):
    vals = np.ascontiguousarray(vals, dtype=np.float32)
    out = np.empty(len(vals), dtype=np.uint16)
    lib().nspo_sq_encode_u16(vmin, vmax, _ptr(vals), _ptr(out), len(vals))
    return out


def sq_scale(vmin, vmax, qvmin, qvmax, qbits=8):
    return lib().nspo_sq_scale(qbits, vmin, vmax, qvmin, qvmax)


def cut(idx, vals, n_cut):
    idx = np.ascontiguousarray(idx, dtype=np.uint16)
    esz = {np.dtype(np.float32): 4, np.dtype(np.uint16): 2}.get(np.dtype(vals.dtype), 1)
    out = np.empty(max(len(idx), n_cut), dtype=np.uint16)
    n = lib().nspo_cut(_ptr(idx), _ptr(vals), esz, len(idx), n_cut, _ptr(out))
    return out[:n]


# ------------------------------------------------------ compiled reference --

_REF = {}


def ref_available(variant: str = "generic") -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", f"libnsparse_ref_{variant}.so"))


def ref_lib(variant: str = "generic"):
    if variant not in _REF:
        L = ctypes.CDLL(os.path.join(HERE, "_ref", f"libnsparse_ref_{variant}.so"))
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_index_factory.restype = P
        L.ref_index_factory.argtypes = [ctypes.c_int, ctypes.c_char_p]
        L.ref_index_free.argtypes = [P]
        L.ref_add.argtypes = [P, I32, P, P, P]
        L.ref_add_with_ids.argtypes = [P, I32, P, P, P, P]
        L.ref_build.argtypes = [P]
        L.ref_num_vectors.restype = I64
        L.ref_num_vectors.argtypes = [P]
        L.ref_search.argtypes = [P, I32, P, P, P, ctypes.c_int, P, P, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                 ctypes.c_float, ctypes.c_int, I64, P]
        L.ref_write_index.argtypes = [P, ctypes.c_char_p]
        L.ref_read_csr.argtypes = [P, ctypes.c_char_p, ctypes.c_int]
        L.ref_csr_convert.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
        L.ref_factory_status.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_char_p]
        L.ref_read_index.restype = P
        L.ref_read_index.argtypes = [ctypes.c_char_p, ctypes.c_int]
        L.ref_set_threads.argtypes = [ctypes.c_int]
        L.ref_max_threads.restype = ctypes.c_int
        L.ref_kmeans_train.argtypes = [ctypes.c_int, ctypes.c_int, I32, P, P, P, P, I32,
                                       ctypes.c_int, ctypes.c_uint32, P, P, P]
        L.ref_map_docs_to_clusters.argtypes = [ctypes.c_int, ctypes.c_int, I32, P, P, P,
                                               P, I32, P, ctypes.c_int, P, P]
        L.ref_summarize.restype = I64
        L.ref_summarize.argtypes = [ctypes.c_int, ctypes.c_int, I32, P, P, P, P, P,
                                    ctypes.c_int, ctypes.c_float, P, I64]
        L.ref_prune_and_keep.argtypes = [ctypes.c_int, I32, P, P, I32, P, P]
        L.ref_top_k_tokens_f32.argtypes = [P, P, ctypes.c_int, ctypes.c_int, P, P]
        L.ref_top_k_tokens_u8.argtypes = [P, P, ctypes.c_int, ctypes.c_int, P, P]
        L.ref_sq_encode.argtypes = [ctypes.c_int, ctypes.c_float, ctypes.c_float, P, P, I64]
        L.ref_sq_decode_dot.restype = ctypes.c_float
        L.ref_sq_decode_dot.argtypes = [ctypes.c_int] + [ctypes.c_float] * 5
        _REF[variant] = L
    return _REF[variant]


class RefError(Exception):
    pass


def ref_csr_convert(interchange_path, native_path, variant="generic"):
    """The reference's csr_layout::convert; returns (status, message)."""
    L = ref_lib(variant)
    rc = L.ref_csr_convert(str(interchange_path).encode(), str(native_path).encode())
    return rc, (L.ref_last_error().decode() if rc else "")


class RefIndex:
    """The reference's own Index, driven through its public C++ API."""

    def __init__(self, dim, spec, variant="generic", handle=None):
        self.L = ref_lib(variant)
        self.h = handle if handle is not None else self.L.ref_index_factory(dim, spec.encode())
        if not self.h:
            raise RefError(self.L.ref_last_error().decode())

    def _check(self, rc):
        if rc != 0:
            raise RefError(self.L.ref_last_error().decode())

    def add(self, csr):
        self._check(self.L.ref_add(self.h, csr.n, _ptr(csr.indptr), _ptr(csr.indices),
                                   _ptr(csr.values)))

    def add_with_ids(self, csr, ids):
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        self._check(self.L.ref_add_with_ids(self.h, csr.n, _ptr(csr.indptr),
                                            _ptr(csr.indices), _ptr(csr.values), _ptr(ids)))

    def build(self):
        self._check(self.L.ref_build(self.h))

    def num_vectors(self):
        return self.L.ref_num_vectors(self.h)

    def search(self, q, k, param_kind=0, cut=10, heap_factor=1.0, vmin=0.0, vmax=1.0,
               sel_kind=0, sel_ids=None):
        D = np.empty((q.n, k), dtype=np.float32)
        L = np.empty((q.n, k), dtype=np.int32)
        sel = None if sel_ids is None else np.ascontiguousarray(sel_ids, dtype=np.int32)
        self._check(self.L.ref_search(self.h, q.n, _ptr(q.indptr), _ptr(q.indices),
                                      _ptr(q.values), k, _ptr(D), _ptr(L), param_kind, cut,
                                      heap_factor, vmin, vmax, sel_kind,
                                      0 if sel is None else len(sel), _ptr(sel)))
        return D, L

    def write(self, path):
        self._check(self.L.ref_write_index(self.h, str(path).encode()))

    def read_csr(self, path, residency=0):
        """Index::read_csr; residency 1 = Residency::kMmap."""
        self._check(self.L.ref_read_csr(self.h, str(path).encode(), int(residency)))

    @classmethod
    def read(cls, path, flags=0, variant="generic"):
        L = ref_lib(variant)
        h = L.ref_read_index(str(path).encode(), flags)
        if not h:
            raise RefError(L.ref_last_error().decode())
        return cls(0, "", variant=variant, handle=h)

    def close(self):
        if self.h:
            self.L.ref_index_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------- reference file reader --

class _Rd:
    def __init__(self, buf: bytes, pos: int = 0):
        self.b = buf
        self.p = pos

    def u(self, fmt):
        v = struct.unpack_from("<" + fmt, self.b, self.p)
        self.p += struct.calcsize("<" + fmt)
        return v[0]

    def pad(self, a):
        self.p += (a - self.p % a) % a

    def arr(self, dtype, count, align=None):
        dt = np.dtype(dtype)
        self.pad(align or dt.itemsize)
        nbytes = dt.itemsize * count
        out = np.frombuffer(self.b, dtype=dt, count=count, offset=self.p).copy()
        self.p += nbytes
        return out


def _read_sparse_vectors(r: _Rd):
    n = r.u("Q")
    if n == 0:
        return None
    dim = r.u("Q")
    esz = r.u("Q")
    indptr = r.arr(np.int32, n + 1)
    nnz = int(indptr[-1])
    indices = r.arr(np.uint16, nnz)
    vbytes = r.arr(np.uint8, nnz * esz, align=esz)
    vdt = {4: np.float32, 2: np.uint16, 1: np.uint8}[esz]
    return dict(n=n, dim=dim, esz=esz, indptr=indptr, indices=indices,
                values=vbytes.view(vdt))


def _read_clusters(r: _Rd):
    n_docs = r.u("Q")
    docs = r.arr(np.int32, n_docs)
    n_off = r.u("Q")
    offsets = r.arr(np.int32, n_off)
    n_clusters = r.u("Q")
    esz = r.u("Q")
    n_terms = r.u("Q")
    if n_terms > 0:
        term_ids = r.arr(np.uint16, n_terms)
        term_ptr = r.arr(np.int32, n_terms + 1)
    else:
        term_ids = np.zeros(0, np.uint16)
        term_ptr = np.zeros(1, np.int32)
    nnz = r.u("Q")
    csc_cluster = r.arr(np.uint16, nnz)
    vbytes = r.arr(np.uint8, nnz * esz, align=esz)
    vdt = {4: np.float32, 2: np.uint16, 1: np.uint8}[esz]
    return dict(docs=docs, offsets=offsets, n_clusters=n_clusters, esz=esz,
                term_ids=term_ids, term_ptr=term_ptr, csc_cluster=csc_cluster,
                csc_value=vbytes.view(vdt))


def read_index_file(path):
    """Parses a SEIS / SESQ / IDMP file written by the reference's write_index."""
    buf = open(path, "rb").read()
    return _read_index(_Rd(buf))


def _read_index(r: _Rd):
    fourcc = r.b[r.p:r.p + 4].decode()
    r.p += 4
    dim = r.u("i")
    out = dict(kind=fourcc, dim=dim)
    if fourcc == "IDMP":
        m = r.u("Q")
        out["ids"] = np.frombuffer(r.b, np.int32, m, r.p).copy()
        r.p += 4 * m
        out["delegate"] = _read_index(r)
        return out
    if fourcc == "SESQ":
        out["qtype"] = r.u("B")
        out["vmin"] = r.u("f")
        out["vmax"] = r.u("f")
    if fourcc in ("SEIS", "SESQ"):
        out["vectors"] = _read_sparse_vectors(r)
        n_lists = r.u("Q")
        out["lists"] = [_read_clusters(r) for _ in range(n_lists)]
        return out
    raise ValueError(f"unsupported index kind {fourcc}")


def flatten_lists(lists, esz) -> SeismicArrays:
    lbp, bdp, docs, ltp, terms, rp, blk, val = [0], [0], [], [0], [], [0], [], []
    for c in lists:
        nb = int(c["n_clusters"]) if len(c["offsets"]) else 0
        off = c["offsets"]
        if nb > 0:
            docs.append(c["docs"])
            bdp.extend((off[1:nb + 1] + bdp[-1]).tolist())
        lbp.append(lbp[-1] + nb)
        nt = len(c["term_ids"])
        terms.append(c["term_ids"])
        rp.extend((c["term_ptr"][1:nt + 1] + rp[-1]).tolist())
        ltp.append(ltp[-1] + nt)
        blk.append(c["csc_cluster"])
        val.append(c["csc_value"])
    vdt = {4: np.float32, 2: np.uint16, 1: np.uint8}[esz]
    cat = lambda xs, dt: np.ascontiguousarray(np.concatenate(xs) if xs else np.zeros(0, dt), dtype=dt)
    return SeismicArrays(
        esz=esz,
        list_block_ptr=np.asarray(lbp, np.int64),
        block_doc_ptr=np.asarray(bdp, np.int64),
        docs=cat(docs, np.int32),
        list_term_ptr=np.asarray(ltp, np.int64),
        sum_terms=cat(terms, np.uint16),
        sum_run_ptr=np.asarray(rp, np.int64),
        sum_block=cat(blk, np.uint16),
        sum_val=cat(val, vdt),
    )
