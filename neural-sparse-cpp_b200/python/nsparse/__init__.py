"""nsparse: the reference library's Python API over the B200 engine.

Mirrors the SWIG module of opensearch-project/neural-sparse-cpp
(nsparse/python/swignsparse.swig, class_wrappers.py): ``index_factory``,
``Index.add / add_with_ids / build / search / num_vectors / get_dimension``,
``SearchParameters`` and its SEISMIC subclasses, the id selectors,
``write_index / read_index`` and ``kUseMmap``. Search returns
``(distances, labels)`` as ``(n, k)`` float32 / int32 arrays.

Everything goes through the C ABI of ``lib/libnsparse_b200.so``
(include/nsparse_c.h); the library must be built first
(``python neural-sparse-cpp_b200/build.py``). C++ exceptions arrive as the
Python exceptions the reference's SWIG layer raises: ValueError, RuntimeError,
IndexError, MemoryError.
"""

from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

__version__ = "0.1.0"

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.abspath(os.path.join(_HERE, "..", "..", "lib", "libnsparse_b200.so"))

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"nsparse engine library not found at {LIB_PATH}; build it with "
        "`python neural-sparse-cpp_b200/build.py`")

_L = ctypes.CDLL(LIB_PATH)
_P = ctypes.c_void_p
_I32 = ctypes.c_int32


def _sig(name, *argtypes):
    f = getattr(_L, name)
    f.restype = ctypes.c_int
    f.argtypes = list(argtypes)
    return f


_L.nsp_last_error.restype = ctypes.c_char_p
_L.nsp_last_error.argtypes = []
_sig("nsp_index_factory", ctypes.c_int, ctypes.c_char_p, ctypes.POINTER(_P))
_sig("nsp_index_free", _P)
_sig("nsp_index_add", _P, _I32, _P, _P, _P)
_sig("nsp_index_add_with_ids", _P, _I32, _P, _P, _P, _P)
_sig("nsp_index_add_with_ids64", _P, _I32, _P, _P, _P, _P)
_sig("nsp_index_search64", _P, _I32, _P, _P, _P, ctypes.c_int, _P, _P, _P)
_sig("nsp_id_selector_set64_new", ctypes.c_size_t, _P, ctypes.POINTER(_P))
_sig("nsp_index_build", _P)
_sig("nsp_index_search", _P, _I32, _P, _P, _P, ctypes.c_int, _P, _P, _P)
_sig("nsp_index_num_vectors", _P, ctypes.POINTER(ctypes.c_int64))
_sig("nsp_index_dimension", _P, ctypes.POINTER(_I32))
_sig("nsp_index_fourcc", _P, ctypes.c_char_p)
_sig("nsp_index_read_csr", _P, ctypes.c_char_p, ctypes.c_int)
_sig("nsp_csr_convert", ctypes.c_char_p, ctypes.c_char_p)
_sig("nsp_write_index", _P, ctypes.c_char_p)
_sig("nsp_read_index", ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(_P))
_sig("nsp_id_selector_set_new", ctypes.c_size_t, _P, ctypes.POINTER(_P))
_sig("nsp_id_selector_array_new", ctypes.c_size_t, _P, ctypes.POINTER(_P))
_sig("nsp_id_selector_not_new", _P, ctypes.POINTER(_P))
_sig("nsp_id_selector_bitmap_new", ctypes.c_int64, _P, ctypes.POINTER(_P))
_sig("nsp_id_selector_is_member", _P, _I32, ctypes.POINTER(ctypes.c_int))
_sig("nsp_id_selector_free", _P)
_sig("nsp_search_params_new", ctypes.POINTER(_P))
_sig("nsp_seismic_search_params_new", ctypes.c_int, ctypes.c_float, ctypes.POINTER(_P))
_sig("nsp_seismic_sq_search_params_new", ctypes.c_float, ctypes.c_float, ctypes.c_int,
     ctypes.c_float, ctypes.POINTER(_P))
_sig("nsp_search_params_set_id_selector", _P, _P)
_sig("nsp_search_params_set_engine", _P, ctypes.c_int, ctypes.c_int)
_sig("nsp_search_params_set_kernel", _P, ctypes.c_int, ctypes.c_int)
_sig("nsp_search_params_set_split", _P, ctypes.c_int)
_sig("nsp_search_params_set_count_unique", _P, ctypes.c_int)
_sig("nsp_search_params_free", _P)
_sig("nsp_index_search_device", _P, _I32, _P, _P, _P, _I32, ctypes.c_int, _P, _P, _P, _P)
_sig("nsp_device_info", ctypes.POINTER(_I32), ctypes.c_char_p, ctypes.c_size_t)
_sig("nsp_index_autotune", _P, _I32, _P, _P, _P, ctypes.c_int, _P, ctypes.POINTER(ctypes.c_int),
     ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float),
     ctypes.POINTER(ctypes.c_int))


class _Stats(ctypes.Structure):
    _fields_ = [("docs_scored", ctypes.c_uint64), ("blocks_visited", ctypes.c_uint64),
                ("bytes", ctypes.c_uint64), ("lists_probed", ctypes.c_uint64),
                ("kernel_ms", ctypes.c_float), ("launches", ctypes.c_int32),
                ("row_bytes", ctypes.c_uint64), ("unique_docs", ctypes.c_uint64),
                ("unique_row_bytes", ctypes.c_uint64)]


_sig("nsp_last_search_stats", ctypes.POINTER(_Stats))

_ERRORS = {1: ValueError, 2: RuntimeError, 3: IndexError, 4: MemoryError}

kUseMmap = 1

# Residency of Index.read_csr (nsparse/types.h), under the names the
# reference's SWIG module gives the scoped enum.
Residency_kInMemory = 0
Residency_kMmap = 1

# CSR file layouts (nsparse/utils/csr_layout.h), flattened into the module
# as the reference's SWIG interface flattens them.
kHeaderBytes = 24
kNativeSuffix = ".mcsr"


def padding(pos):
    """Zero bytes that bring file position `pos` to a 4-byte boundary."""
    return (4 - pos % 4) % 4


def interchange_file_size(indptr_size, nnz):
    return kHeaderBytes + 8 * indptr_size + 8 * nnz


def native_values_offset(indptr_size, nnz):
    head = kHeaderBytes + 4 * indptr_size + 2 * nnz
    return head + padding(head)


def native_file_size(indptr_size, nnz):
    return native_values_offset(indptr_size, nnz) + 4 * nnz


def native_path(path):
    return str(path) + kNativeSuffix


def convert(interchange_path, native_path):
    """Rewrites an interchange CSR file (scipy's int64 indptr / int32 indices
    / float values) in the native layout that read_csr(path,
    Residency_kMmap) takes."""
    _check(_L.nsp_csr_convert(str(interchange_path).encode(), str(native_path).encode()))


def _check(rc):
    if rc != 0:
        msg = _L.nsp_last_error().decode(errors="replace")
        raise _ERRORS.get(rc, RuntimeError)(msg)


def _ptr(a):
    return a.ctypes.data if a is not None else None


def _typed(a, dtype, name):
    """Buffer check of the reference's typemaps: a wrong dtype is an error."""
    a = np.asarray(a)
    if a.dtype != np.dtype(dtype):
        raise TypeError(f"Expected {np.dtype(dtype).name} array for {name}")
    return np.ascontiguousarray(a)


# ------------------------------------------------------------ selectors --

class IDSelector:
    """Base of the id selectors (reference: nsparse/id_selector.h:22-86)."""

    _h = None

    def is_member(self, id_):
        out = ctypes.c_int()
        _check(_L.nsp_id_selector_is_member(self._h, int(id_), ctypes.byref(out)))
        return bool(out.value)

    def __call__(self, id_):
        return self.is_member(id_)

    def __del__(self):
        h, self._h = self._h, None
        if h and _L is not None:  # at interpreter exit the module may be gone
            _L.nsp_id_selector_free(h)


class SetIDSelector(IDSelector):
    def __init__(self, ids):
        ids = _typed(ids, np.int32, "indices")
        h = _P()
        _check(_L.nsp_id_selector_set_new(len(ids), _ptr(ids), ctypes.byref(h)))
        self._h = h.value


class SetIDSelector64(IDSelector):
    """Extension: a set of 64-bit ids, for an IDMapIndex whose external ids
    need them."""

    def __init__(self, ids):
        ids = _typed(ids, np.int64, "indices")
        h = _P()
        _check(_L.nsp_id_selector_set64_new(len(ids), _ptr(ids), ctypes.byref(h)))
        self._h = h.value


class ArrayIDSelector(IDSelector):
    def __init__(self, ids):
        ids = _typed(ids, np.int32, "indices")
        h = _P()
        _check(_L.nsp_id_selector_array_new(len(ids), _ptr(ids), ctypes.byref(h)))
        self._h = h.value


class NotIDSelector(IDSelector):
    def __init__(self, selector):
        h = _P()
        _check(_L.nsp_id_selector_not_new(selector._h, ctypes.byref(h)))
        self._h = h.value
        self._inner = selector  # the C++ object borrows it


class BitmapIDSelector(IDSelector):
    """Extension: membership bitmap over ids [0, n_bits), bit d of word d // 64."""

    def __init__(self, n_bits, bits):
        bits = _typed(bits, np.uint64, "bits")
        if len(bits) * 64 < n_bits:
            raise ValueError("bitmap shorter than n_bits")
        h = _P()
        _check(_L.nsp_id_selector_bitmap_new(int(n_bits), _ptr(bits), ctypes.byref(h)))
        self._h = h.value


# ----------------------------------------------------------- parameters --

class SearchParameters:
    """Reference: nsparse/index.h:21-28."""

    def __init__(self):
        h = _P()
        _check(_L.nsp_search_params_new(ctypes.byref(h)))
        self._h = h.value
        self._sel = None

    def set_id_selector(self, selector):
        _check(_L.nsp_search_params_set_id_selector(self._h, None if selector is None else selector._h))
        self._sel = selector

    def get_id_selector(self):
        return self._sel

    def set_engine(self, plain=False, warps_per_block=0):
        """Extension: plain=True runs one kernel launch per query."""
        _check(_L.nsp_search_params_set_engine(self._h, int(bool(plain)), int(warps_per_block)))

    def set_kernel(self, variant=-1, tuning=0):
        """Extension: SEISMIC kernel variant (-1 auto, 0 warp per query with
        direct loads, 1 warp per query with bulk-copy staging, 2-5 CTA per
        query with 1, 2, 4 or 8 lanes per doc) and its tuning value (variant 1:
        staging buffer bytes; variants 2-5: candidate docs per batch; 0 =
        default). Results do not depend on either."""
        _check(_L.nsp_search_params_set_kernel(self._h, int(variant), int(tuning)))

    def set_split(self, ctas_per_query=0):
        """Extension: CTAs per query of SEISMIC variants 2-5 (0 auto, 1, or a
        cluster of 2, 4 or 8 CTAs scoring each query together)."""
        _check(_L.nsp_search_params_set_split(self._h, int(ctas_per_query)))

    def set_count_unique(self, on=True):
        """Extension: a batched SEISMIC search becomes a counting pass (slower,
        same results) whose stats also count each scored doc's row once per
        query, as the reference's visited set does."""
        _check(_L.nsp_search_params_set_count_unique(self._h, int(bool(on))))

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h and _L is not None:  # at interpreter exit the module may be gone
            _L.nsp_search_params_free(h)


class SeismicSearchParameters(SearchParameters):
    """Reference: nsparse/seismic_index.h:26-32 (cut=10, heap_factor=1.0)."""

    def __init__(self, cut=10, heap_factor=1.0):
        h = _P()
        _check(_L.nsp_seismic_search_params_new(int(cut), float(heap_factor), ctypes.byref(h)))
        self._h = h.value
        self._sel = None
        self.cut = int(cut)
        self.heap_factor = float(heap_factor)


class SeismicSQSearchParameters(SeismicSearchParameters):
    """Reference: nsparse/seismic_scalar_quantized_index.h:27-33."""

    def __init__(self, vmin, vmax, cut=10, heap_factor=1.0):
        h = _P()
        _check(_L.nsp_seismic_sq_search_params_new(float(vmin), float(vmax), int(cut),
                                                   float(heap_factor), ctypes.byref(h)))
        self._h = h.value
        self._sel = None
        self.vmin = float(vmin)
        self.vmax = float(vmax)
        self.cut = int(cut)
        self.heap_factor = float(heap_factor)


# ---------------------------------------------------------------- index --

class Index:
    """Reference: nsparse/index.h:30-68 with the SWIG search wrapper
    (class_wrappers.py:22-58)."""

    def __init__(self, handle):
        self._h = handle

    def add(self, n, indptr, indices, values):
        indptr = _typed(indptr, np.int32, "indptr")
        indices = _typed(indices, np.uint16, "indices")
        values = _typed(values, np.float32, "values")
        _check(_L.nsp_index_add(self._h, int(n), _ptr(indptr), _ptr(indices), _ptr(values)))

    def add_with_ids(self, n, indptr, indices, values, ids):
        indptr = np.ascontiguousarray(indptr, dtype=np.int32)
        indices = np.ascontiguousarray(indices, dtype=np.uint16)
        values = np.ascontiguousarray(values, dtype=np.float32)
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        _check(_L.nsp_index_add_with_ids(self._h, int(n), _ptr(indptr), _ptr(indices),
                                         _ptr(values), _ptr(ids)))

    def add_with_ids64(self, n, indptr, indices, values, ids):
        """Extension: add_with_ids with 64-bit external ids (IDMapIndex)."""
        indptr = _typed(indptr, np.int32, "indptr")
        indices = _typed(indices, np.uint16, "indices")
        values = _typed(values, np.float32, "values")
        ids = _typed(ids, np.int64, "ids")
        _check(_L.nsp_index_add_with_ids64(self._h, int(n), _ptr(indptr), _ptr(indices),
                                           _ptr(values), _ptr(ids)))

    def search64(self, n, indptr, indices, values, k, params=None):
        """Extension: search with int64 labels (an IDMapIndex's 64-bit ids)."""
        indptr = np.ascontiguousarray(indptr, dtype=np.int32)
        indices = np.ascontiguousarray(indices, dtype=np.uint16)
        values = np.ascontiguousarray(values, dtype=np.float32)
        n, k = int(n), int(k)
        if n <= 0 or k <= 0:
            raise ValueError("value must be positive")
        distances = np.empty((n, k), dtype=np.float32)
        labels = np.empty((n, k), dtype=np.int64)
        _check(_L.nsp_index_search64(self._h, n, _ptr(indptr), _ptr(indices), _ptr(values), k,
                                     _ptr(distances), _ptr(labels),
                                     None if params is None else params._h))
        return distances, labels

    def build(self):
        _check(_L.nsp_index_build(self._h))

    def search(self, n, indptr, indices, values, k, params=None):
        indptr = np.ascontiguousarray(indptr, dtype=np.int32)
        indices = np.ascontiguousarray(indices, dtype=np.uint16)
        values = np.ascontiguousarray(values, dtype=np.float32)
        n, k = int(n), int(k)
        if n <= 0 or k <= 0:
            # same message the C++ layer gives; allocation below needs n, k > 0
            raise ValueError("value must be positive")
        distances = np.empty((n, k), dtype=np.float32)
        labels = np.empty((n, k), dtype=np.int32)
        _check(_L.nsp_index_search(self._h, n, _ptr(indptr), _ptr(indices), _ptr(values), k,
                                   _ptr(distances), _ptr(labels),
                                   None if params is None else params._h))
        return distances, labels

    def search_device(self, n, d_indptr, d_indices, d_values, max_row_nnz, k, d_distances,
                      d_labels, params=None, stream=None):
        """Extension: device pointers in and out (ints), enqueued on `stream`."""
        _check(_L.nsp_index_search_device(self._h, int(n), d_indptr, d_indices, d_values,
                                          int(max_row_nnz), int(k), d_distances, d_labels,
                                          None if params is None else params._h, stream))

    def autotune(self, n, indptr, indices, values, k, params=None):
        """Extension: times the SEISMIC kernel's launch shapes on these sample
        queries and keeps the fastest for later searches that leave the kernel
        to the engine. Returns the choice as a dict."""
        indptr = np.ascontiguousarray(indptr, dtype=np.int32)
        indices = np.ascontiguousarray(indices, dtype=np.uint16)
        values = np.ascontiguousarray(values, dtype=np.float32)
        v, b, w, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        ms = ctypes.c_float()
        _check(_L.nsp_index_autotune(self._h, int(n), _ptr(indptr), _ptr(indices), _ptr(values),
                                     int(k), None if params is None else params._h,
                                     ctypes.byref(v), ctypes.byref(b), ctypes.byref(w),
                                     ctypes.byref(ms), ctypes.byref(c)))
        return {"variant": v.value, "batch_docs": b.value, "warps_per_block": w.value,
                "kernel_ms": ms.value, "ctas_per_query": c.value}

    def num_vectors(self):
        out = ctypes.c_int64()
        _check(_L.nsp_index_num_vectors(self._h, ctypes.byref(out)))
        return out.value

    def get_dimension(self):
        out = _I32()
        _check(_L.nsp_index_dimension(self._h, ctypes.byref(out)))
        return out.value

    def id(self):
        buf = ctypes.create_string_buffer(4)
        _check(_L.nsp_index_fourcc(self._h, buf))
        return buf.raw.decode()

    def read_csr(self, file_path, residency=0):
        _check(_L.nsp_index_read_csr(self._h, str(file_path).encode(), int(residency)))

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h and _L is not None:  # at interpreter exit the module may be gone
            _L.nsp_index_free(h)


class BrutalIndex(Index):
    pass


class InvertedIndex(Index):
    pass


class SeismicIndex(Index):
    pass


class SeismicScalarQuantizedIndex(Index):
    pass


class IDMapIndex(Index):
    pass


_BY_FOURCC = {"BRUT": BrutalIndex, "INVT": InvertedIndex, "SEIS": SeismicIndex,
              "SESQ": SeismicScalarQuantizedIndex, "IDMP": IDMapIndex}


def _wrap(handle):
    idx = Index(handle)
    cls = _BY_FOURCC.get(idx.id(), Index)
    idx.__class__ = cls
    return idx


def index_factory(dim, description):
    """Reference: nsparse/index_factory.cpp:63-153."""
    h = _P()
    desc = description.encode() if description is not None else None
    _check(_L.nsp_index_factory(int(dim), desc, ctypes.byref(h)))
    return _wrap(h.value)


def write_index(index, file_name):
    _check(_L.nsp_write_index(index._h, str(file_name).encode()))


def read_index(file_name, io_flags=0):
    h = _P()
    _check(_L.nsp_read_index(str(file_name).encode(), int(io_flags), ctypes.byref(h)))
    return _wrap(h.value)


@dataclass
class SearchStats:
    docs_scored: int
    blocks_visited: int
    bytes: int             # every byte read, rows as often as scored
    lists_probed: int
    kernel_ms: float
    launches: int
    row_bytes: int = 0     # the rows' share of `bytes`
    unique_docs: int = 0   # counting pass only: docs counted once per query
    unique_row_bytes: int = 0

    @property
    def reference_bytes(self) -> int:
        """The reference's algorithmic bytes (each scored row once per query:
        its visited set); meaningful after a counting pass."""
        return self.bytes - self.row_bytes + self.unique_row_bytes


def last_search_stats() -> SearchStats:
    """Extension: work counters and device time of this thread's last search."""
    s = _Stats()
    _check(_L.nsp_last_search_stats(ctypes.byref(s)))
    return SearchStats(s.docs_scored, s.blocks_visited, s.bytes, s.lists_probed, s.kernel_ms,
                       s.launches, s.row_bytes, s.unique_docs, s.unique_row_bytes)


def device_info():
    n = _I32()
    buf = ctypes.create_string_buffer(256)
    _check(_L.nsp_device_info(ctypes.byref(n), buf, 256))
    return n.value, buf.value.decode()


# ------------------------------------------------------------ serving ----

class _ServerConfig(ctypes.Structure):
    _fields_ = [("max_batch", ctypes.c_int32), ("slots", ctypes.c_int32),
                ("scratch_budget_bytes", ctypes.c_int64)]


_sig("nsp_server_new", _P, ctypes.POINTER(_ServerConfig), ctypes.POINTER(_P))
_sig("nsp_server_free", _P)
_sig("nsp_server_add_filter", _P, _P, ctypes.c_int64, ctypes.POINTER(_I32))
_sig("nsp_server_set_external_ids", _P, _P, ctypes.c_int64)
_sig("nsp_server_submit", _P, _I32, _P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_float, _I32,
     ctypes.POINTER(ctypes.c_int64))
_sig("nsp_server_wait", _P, ctypes.c_int64, _P, _P, ctypes.POINTER(ctypes.c_double))
_sig("nsp_server_replay", _P, _I32, _P, _P, _P, _P, _P, _P, ctypes.c_int, ctypes.c_float,
     ctypes.c_int, _P, _P, _P)
_sig("nsp_server_stats", _P, ctypes.POINTER(ctypes.c_int64))


class Server:
    """Extension: continuous-batching serving loop over a seismic index (or an
    IDMapIndex over one). Single-query requests with their own k and optional
    doc filter are batched by the engine as they arrive; each result equals a
    search of that query alone. Keep the index alive and unchanged while the
    server runs."""

    def __init__(self, index, max_batch=0, slots=0, scratch_budget_bytes=0):
        self._index = index
        cfg = _ServerConfig(int(max_batch), int(slots), int(scratch_budget_bytes))
        h = _P()
        _check(_L.nsp_server_new(index._h, ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h.value

    def add_filter(self, bits):
        """A doc filter: uint64 bitmap over internal doc ids. Returns its id."""
        bits = np.ascontiguousarray(bits, dtype=np.uint64)
        out = _I32()
        _check(_L.nsp_server_add_filter(self._h, _ptr(bits), bits.size, ctypes.byref(out)))
        return out.value

    def set_external_ids(self, ids):
        ids = np.ascontiguousarray(ids, dtype=np.int64)
        _check(_L.nsp_server_set_external_ids(self._h, _ptr(ids), ids.size))

    def submit(self, terms, values, k=10, cut=10, heap_factor=1.0, filter_id=-1):
        terms = np.ascontiguousarray(terms, dtype=np.uint16)
        values = np.ascontiguousarray(values, dtype=np.float32)
        t = ctypes.c_int64()
        _check(_L.nsp_server_submit(self._h, terms.size, _ptr(terms), _ptr(values), int(k),
                                    int(cut), float(heap_factor), int(filter_id), ctypes.byref(t)))
        return t.value, int(k)

    def wait(self, ticket):
        """ticket: what submit() returned. Returns (distances, labels, latency_us)."""
        t, k = ticket
        d = np.empty(k, dtype=np.float32)
        l = np.empty(k, dtype=np.int64)
        lat = ctypes.c_double()
        _check(_L.nsp_server_wait(self._h, t, _ptr(d), _ptr(l), ctypes.byref(lat)))
        return d, l, lat.value

    def replay(self, indptr, indices, values, k_per, arrival_us, cut=10, heap_factor=1.0,
               filter_per=None):
        """Submits row i at arrival_us[i] (microseconds from the call) and waits
        for all. Returns (distances, labels, latency_us), max(k_per) per row."""
        indptr = np.ascontiguousarray(indptr, dtype=np.int32)
        indices = np.ascontiguousarray(indices, dtype=np.uint16)
        values = np.ascontiguousarray(values, dtype=np.float32)
        k_per = np.ascontiguousarray(k_per, dtype=np.int32)
        arrival_us = np.ascontiguousarray(arrival_us, dtype=np.float64)
        n = len(indptr) - 1
        ks = int(k_per.max())
        fp = None if filter_per is None else np.ascontiguousarray(filter_per, dtype=np.int32)
        d = np.empty((n, ks), dtype=np.float32)
        l = np.empty((n, ks), dtype=np.int64)
        lat = np.empty(n, dtype=np.float64)
        _check(_L.nsp_server_replay(self._h, n, _ptr(indptr), _ptr(indices), _ptr(values),
                                    _ptr(k_per), _ptr(fp), _ptr(arrival_us), int(cut),
                                    float(heap_factor), ks, _ptr(d), _ptr(l), _ptr(lat)))
        return d, l, lat

    def stats(self):
        out = (ctypes.c_int64 * 4)()
        _check(_L.nsp_server_stats(self._h, out))
        return {"batches": out[0], "requests": out[1], "max_batch": out[2],
                "max_in_flight_bytes": out[3]}

    def close(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            _L.nsp_server_free(h)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _GraphBuffers(ctypes.Structure):
    _fields_ = [("indptr", _P), ("indices", _P), ("values", _P), ("distances", _P),
                ("labels", _P)]


_sig("nsp_search_graph_new", _P, _I32, _I32, _I32, ctypes.c_int, _P,
     ctypes.POINTER(_GraphBuffers), ctypes.POINTER(_P))
_sig("nsp_search_graph_free", _P)
_sig("nsp_search_graph_buffers", _P, ctypes.POINTER(_GraphBuffers))
_sig("nsp_search_graph_launch", _P, _P)
_sig("nsp_search_graph_sync", _P, _P)
_sig("nsp_search_graph_search", _P, _I32, _P, _P, _P, _P, _P)


class SearchGraph:
    """Extension: one batched SEISMIC search step of `n` query rows captured
    as a CUDA graph and replayed per batch (k, parameters and selector fixed
    at capture). `device_buffers`: a dict of device pointers (ints) "indptr",
    "indices", "values", "distances", "labels" the caller keeps alive, or None
    for buffers the graph owns. Keep the index alive and unchanged while the
    graph is used."""

    def __init__(self, index, n, nnz_cap, max_row_nnz, k, params=None, device_buffers=None):
        self._index, self._params = index, params
        self.n, self.k = int(n), int(k)
        b = None
        if device_buffers is not None:
            b = _GraphBuffers(*(device_buffers[f] for f in
                                ("indptr", "indices", "values", "distances", "labels")))
        h = _P()
        _check(_L.nsp_search_graph_new(index._h, self.n, int(nnz_cap), int(max_row_nnz), self.k,
                                       None if params is None else params._h,
                                       None if b is None else ctypes.byref(b), ctypes.byref(h)))
        self._h = h.value

    def buffers(self):
        b = _GraphBuffers()
        _check(_L.nsp_search_graph_buffers(self._h, ctypes.byref(b)))
        return {f: getattr(b, f) for f, _ in _GraphBuffers._fields_}

    def launch(self, stream=None):
        """Replays the step on `stream` (a cudaStream_t as int; None: the
        graph's own stream) and returns."""
        _check(_L.nsp_search_graph_launch(self._h, stream))

    def sync(self, stream=None):
        _check(_L.nsp_search_graph_sync(self._h, stream))

    def search(self, n, indptr, indices, values):
        """Host rows in (at most the graph's n), (distances, labels) out."""
        indptr = np.ascontiguousarray(indptr, dtype=np.int32)
        indices = np.ascontiguousarray(indices, dtype=np.uint16)
        values = np.ascontiguousarray(values, dtype=np.float32)
        n = int(n)
        if n <= 0:
            raise ValueError("value must be positive")
        distances = np.empty((n, self.k), dtype=np.float32)
        labels = np.empty((n, self.k), dtype=np.int32)
        _check(_L.nsp_search_graph_search(self._h, n, _ptr(indptr), _ptr(indices), _ptr(values),
                                          _ptr(distances), _ptr(labels)))
        return distances, labels

    def close(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            _L.nsp_search_graph_free(h)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
