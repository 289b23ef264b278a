"""Shared fixtures-by-function for the tests: the golden corpus, reference-
built indexes (through the compiled reference in oracle/_ref) and result
comparisons."""

from __future__ import annotations

import hashlib
import os

import numpy as np

import oracle as O
from nsparse_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "small.npz")

# Parameters the golden file was made with (tests/golden/make_golden.py).
N_DOCS, N_QUERIES, SEED, K = 2000, 64, 11, 10
SEISMIC = "seismic,lambda=200|beta=20|alpha=0.4|seed=7"
CUT, HF = 10, 0.8


def checksum(csr):
    h = hashlib.sha256()
    for a in (csr.indptr, csr.indices, csr.values):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def golden():
    return np.load(GOLDEN)


def golden_corpus():
    g = golden()
    docs = synth.docs_config0(N_DOCS, seed=SEED)
    qs = synth.queries_config0(N_QUERIES, seed=SEED)
    assert checksum(docs) == str(g["docs_sha"]), "generator output drifted from the golden corpus"
    assert checksum(qs) == str(g["queries_sha"])
    return docs, qs


def sq_spec(vmin, vmax, lam=200, beta=20, bits=8):
    return (f"seismic_sq,quantizer={bits}bit|vmin={float(vmin)!r}|vmax={float(vmax)!r}|"
            f"lambda={lam}|beta={beta}|alpha=0.4|seed=7")


def sq_codes(vmin, vmax, vals, bits=8):
    """The reference's ScalarQuantizer::encode (8- or 16-bit), via the oracle."""
    return (O.sq_encode_u16 if bits == 16 else O.sq_encode_u8)(vmin, vmax, vals)


def ref_index(docs, spec, build=True, ids=None):
    r = O.RefIndex(docs.dim, spec)
    if ids is None:
        r.add(docs)
    else:
        r.add_with_ids(docs, ids)
    if build:
        r.build()
    return r


def ref_file(docs, spec, path, ids=None):
    r = ref_index(docs, spec, ids=ids)
    r.write(str(path))
    return r


class Fwd:
    """Forward-index view the C oracle takes."""

    def __init__(self, dim, n, indptr, indices):
        self.dim, self.n, self.indptr, self.indices = dim, n, indptr, indices


def oracle_seismic_from_file(path, qs, k, cut, hf, codes=None, sel_bits=None, want_stats=False):
    f = O.read_index_file(str(path))
    if f["kind"] == "IDMP":
        f = f["delegate"]
    v = f["vectors"]
    esz = v["esz"]
    A = O.flatten_lists(f["lists"], esz)
    fw = Fwd(f["dim"], v["n"], v["indptr"], v["indices"])
    qv = qs.values if codes is None else codes
    return O.seismic_search(fw, v["values"], A, qs.indptr, qs.indices, qv, k, cut, hf,
                            sel_bits=sel_bits, want_stats=want_stats)


def recall(L, T):
    vals = []
    for a, b in zip(L, T):
        want = {int(x) for x in b if x >= 0}
        if not want:
            continue
        vals.append(len({int(x) for x in a if x >= 0} & want) / len(want))
    return float(np.mean(vals)) if vals else 1.0


def sq_exact_scores(docs, q_codes, qs, labels, vmin, vmax, bits=8):
    """Exact integer code dot products (as float32) of each (query, label);
    int64 sums, as the reference sums 16-bit codes (utils/distance.h:49-57)."""
    d_codes = sq_codes(vmin, vmax, docs.values, bits)
    out = np.zeros(labels.shape, np.float32)
    for q in range(labels.shape[0]):
        qd = np.zeros(docs.dim, np.int64)
        s, e = qs.indptr[q], qs.indptr[q + 1]
        qd[qs.indices[s:e]] = q_codes[s:e]
        for j, d in enumerate(labels[q]):
            if d < 0:
                continue
            a, b = docs.indptr[d], docs.indptr[d + 1]
            out[q, j] = np.float32(int(np.dot(d_codes[a:b].astype(np.int64), qd[docs.indices[a:b]])))
    return out


def unsorted_rows(docs, seed):
    """The same docs with every row's elements in a random order, and a
    repeated term (at a new value) appended to every tenth row: rows that
    are not strictly ascending, summed by the reference in stored order."""
    rng = np.random.default_rng(seed)
    ip, ix, vv = [0], [], []
    for d in range(docs.n):
        s, e = int(docs.indptr[d]), int(docs.indptr[d + 1])
        perm = rng.permutation(e - s)
        t, v = docs.indices[s:e][perm], docs.values[s:e][perm]
        if d % 10 == 0 and e > s:
            t = np.append(t, t[0])
            v = np.append(v, np.float32(rng.lognormal(0.0, 0.8)))
        ix.append(t)
        vv.append(v)
        ip.append(ip[-1] + len(t))
    return synth.Csr(docs.dim, np.array(ip, np.int32), np.concatenate(ix).astype(np.uint16),
                     np.concatenate(vv).astype(np.float32))
