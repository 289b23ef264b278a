"""Generates tests/golden/small.npz from the reference library itself.

Run in a container where the reference compiled from its sources exists
(``make -f oracle/Makefile ref``): python tests/golden/make_golden.py

The corpus is not stored: it is regenerated from (seed, n) by the seeded
generator and pinned by a checksum. Stored are the reference's own results on
it for every index type, computed by the generic (scalar) build of the
reference, whose float sums are sequential and whose uint8 sums are exact.
"""

from __future__ import annotations

import hashlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "neural-sparse-cpp_b200", "python"))

import oracle as O  # noqa: E402
from nsparse_b200 import synth  # noqa: E402

N_DOCS = 2000
N_QUERIES = 64
SEED = 11
K = 10
SEISMIC = "seismic,lambda=200|beta=20|alpha=0.4|seed=7"
CUT, HF = 10, 0.8


def corpus():
    return synth.docs_config0(N_DOCS, seed=SEED), synth.queries_config0(N_QUERIES, seed=SEED)


def checksum(csr):
    h = hashlib.sha256()
    for a in (csr.indptr, csr.indices, csr.values):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def sq_spec(docs):
    vmin, vmax = float(docs.values.min()), float(docs.values.max())
    return (f"seismic_sq,quantizer=8bit|vmin={vmin!r}|vmax={vmax!r}|lambda=200|beta=20|"
            f"alpha=0.4|seed=7"), vmin, vmax


def main():
    docs, qs = corpus()
    out = {"docs_sha": np.array(checksum(docs)), "queries_sha": np.array(checksum(qs))}
    r = O.RefIndex(docs.dim, "brutal")
    r.add(docs)
    out["brutal_D"], out["brutal_L"] = r.search(qs, K)
    r = O.RefIndex(docs.dim, "inverted")
    r.add(docs)
    r.build()
    out["inverted_D"], out["inverted_L"] = r.search(qs, K)
    r = O.RefIndex(docs.dim, SEISMIC)
    r.add(docs)
    r.build()
    out["seismic_D"], out["seismic_L"] = r.search(qs, K, param_kind=2, cut=CUT, heap_factor=HF)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "s.idx")
        r.write(p)
        out["seismic_file_sha"] = np.array(hashlib.sha256(open(p, "rb").read()).hexdigest())
    spec, vmin, vmax = sq_spec(docs)
    r = O.RefIndex(docs.dim, spec)
    r.add(docs)
    r.build()
    out["sq_D"], out["sq_L"] = r.search(qs, K, param_kind=2, cut=CUT, heap_factor=HF)
    out["sq_vmin"], out["sq_vmax"] = np.float32(vmin), np.float32(vmax)
    # exact-match path: query 0's reference top-k as an enumerable selector
    seis = O.RefIndex(docs.dim, SEISMIC)
    seis.add(docs)
    seis.build()
    ids = out["seismic_L"][0][out["seismic_L"][0] >= 0].astype(np.int32)
    out["exact_ids"] = ids
    out["exact_D"], out["exact_L"] = seis.search(qs.rows(0, 4), K, param_kind=2, cut=CUT,
                                                 heap_factor=HF, sel_kind=1, sel_ids=ids)
    # filtered search (selector larger than k): every 3rd doc
    allowed = np.arange(0, N_DOCS, 3, dtype=np.int32)
    out["filter_ids"] = allowed
    out["filter_D"], out["filter_L"] = seis.search(qs, K, param_kind=2, cut=CUT, heap_factor=HF,
                                                   sel_kind=1, sel_ids=allowed)
    inv = O.RefIndex(docs.dim, "inverted")
    inv.add(docs)
    inv.build()
    out["inv_filter_D"], out["inv_filter_L"] = inv.search(qs, K, param_kind=1, sel_kind=1,
                                                          sel_ids=allowed)
    np.savez_compressed(os.path.join(HERE, "small.npz"), **out)
    print("wrote", os.path.join(HERE, "small.npz"))


if __name__ == "__main__":
    main()
