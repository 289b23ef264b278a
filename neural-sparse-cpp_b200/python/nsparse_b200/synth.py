"""Seeded synthetic sparse corpora standing in for MS MARCO SPLADE vectors.

The generator itself is C (``synth/nsp_synth.c``, built into
``synth/libnsp_synth.so``, apart from the engine library); this module sizes
the buffers and names the workload shapes used by the benchmarks and tests:

* ``docs_config0`` -- doc nnz lognormal(median 110, sigma 0.6) clipped to
  [10, 400]; Zipf(1.1) terms over the 30,522-term vocabulary without
  replacement, sorted; values lognormal(0, 0.8) float32.
* ``queries_config0`` -- same terms/values, nnz lognormal(median 25, sigma 0.6)
  clipped to [3, 120].
* ``docs_config2`` / ``queries_config2`` -- median 120 doc nnz; query nnz
  uniform on [5, 200].
"""

from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

VOCAB = 30522

_LIB = None
_PATH = os.path.abspath(os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "..",
                                     "synth", "libnsp_synth.so"))


def use_library(path: str) -> None:
    """Loads the generator from `path` (the same C source built elsewhere)
    instead of the package's own build; call before the first corpus."""
    global _PATH
    if _LIB is not None:
        raise RuntimeError("the generator library is already loaded")
    _PATH = os.path.abspath(path)


def _lib():
    global _LIB
    if _LIB is None:
        lib = ctypes.CDLL(_PATH)
        lib.nsp_synth_indptr.restype = ctypes.c_int64
        lib.nsp_synth_indptr.argtypes = [
            ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int64, ctypes.c_int,
            ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
            ctypes.c_int, ctypes.c_void_p,
        ]
        lib.nsp_synth_fill.restype = ctypes.c_int
        lib.nsp_synth_fill.argtypes = [
            ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int64, ctypes.c_int,
            ctypes.c_double, ctypes.c_double, ctypes.c_double,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
        ]
        _LIB = lib
    return _LIB


@dataclass
class Csr:
    """A CSR batch in the reference's dtypes: int32 indptr, uint16 indices,
    float32 values."""

    dim: int
    indptr: np.ndarray
    indices: np.ndarray
    values: np.ndarray

    @property
    def n(self) -> int:
        return len(self.indptr) - 1

    @property
    def nnz(self) -> int:
        return int(self.indptr[-1])

    def rows(self, lo: int, hi: int) -> "Csr":
        s, e = int(self.indptr[lo]), int(self.indptr[hi])
        return Csr(
            self.dim,
            np.ascontiguousarray(self.indptr[lo:hi + 1] - s, dtype=np.int32),
            np.ascontiguousarray(self.indices[s:e]),
            np.ascontiguousarray(self.values[s:e]),
        )


def generate(n: int, *, seed: int, stream: int, dim: int = VOCAB,
             nnz_kind: str = "lognormal", median: float = 110.0,
             sigma: float = 0.6, lo: int = 10, hi: int = 400,
             zipf_s: float = 1.1, val_mu: float = 0.0,
             val_sigma: float = 0.8) -> Csr:
    lib = _lib()
    indptr = np.empty(n + 1, dtype=np.int32)
    kind = 0 if nnz_kind == "lognormal" else 1
    p0, p1 = (median, sigma) if kind == 0 else (0.0, 0.0)
    nnz = lib.nsp_synth_indptr(seed, stream, n, kind, p0, p1, lo, hi, dim,
                               indptr.ctypes.data)
    if nnz < 0:
        raise ValueError("synthetic corpus does not fit int32 offsets")
    indices = np.empty(max(nnz, 1), dtype=np.uint16)
    values = np.empty(max(nnz, 1), dtype=np.float32)
    rc = lib.nsp_synth_fill(seed, stream, n, dim, zipf_s, val_mu, val_sigma,
                            indptr.ctypes.data, indices.ctypes.data,
                            values.ctypes.data)
    if rc != 0:
        raise RuntimeError("synthetic corpus generation failed")
    return Csr(dim, indptr, indices[:nnz], values[:nnz])


def docs_config0(n: int, seed: int = 0, dim: int = VOCAB) -> Csr:
    return generate(n, seed=seed, stream=0, dim=dim, median=110.0, sigma=0.6,
                    lo=10, hi=400)


def queries_config0(n: int, seed: int = 0, dim: int = VOCAB) -> Csr:
    return generate(n, seed=seed, stream=1, dim=dim, median=25.0, sigma=0.6,
                    lo=3, hi=120)


def docs_config2(n: int, seed: int = 0, dim: int = VOCAB) -> Csr:
    return generate(n, seed=seed, stream=0, dim=dim, median=120.0, sigma=0.6,
                    lo=10, hi=400)


def queries_config2(n: int, seed: int = 0, dim: int = VOCAB) -> Csr:
    return generate(n, seed=seed, stream=1, dim=dim, nnz_kind="uniform",
                    lo=5, hi=200)
