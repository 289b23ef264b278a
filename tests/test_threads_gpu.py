"""Concurrent searches of one index from several host threads (the reference's
threading contract: `search` may be called concurrently, each call with its
own scratch, seismic_index.cpp:192-217; results must not depend on the number
of threads, python_tests/test_threading.py:110-150).

Each host thread gets its own engine workspace (CUDA stream, device and pinned
scratch); the index's device images are shared read-only. Every search a
thread runs must equal, bit for bit, the same search run alone on one thread
-- including the first searches of a freshly built index, which race to upload
its device images under the index's lock.
"""

import threading

import numpy as np
import pytest

import nsparse
from helpers import CUT, HF, K, SEISMIC, golden_corpus, sq_spec

pytestmark = pytest.mark.gpu

N_THREADS = 8
ROUNDS = 6


def _tasks(qs, n_docs):
    """(name, query rows, k, params factory): mixed batch sizes, k, cuts,
    heap factors, a selector, and the one-query-per-launch path."""
    sel_ids = np.arange(0, n_docs, 3, dtype=np.int32)

    def p(cut, hf, plain=False, select=False):
        def make():
            prm = nsparse.SeismicSearchParameters(cut, hf)
            if plain:
                prm.set_engine(plain=True)
            if select:
                prm.set_id_selector(nsparse.SetIDSelector(sel_ids))
            return prm
        return make

    return [
        ("all-k10", qs, 10, p(CUT, HF)),
        ("all-k100", qs, 100, p(CUT, 0.9)),
        ("half-cut5", qs.rows(0, qs.n // 2), K, p(5, 1.0)),
        ("tail-sel", qs.rows(qs.n // 4, qs.n), K, p(CUT, HF, select=True)),
        ("few-plain", qs.rows(0, 6), K, p(CUT, HF, plain=True)),
        ("one", qs.rows(3, 4), K, p(12, 0.7)),
    ]


def _run(idx, task):
    _, q, k, make = task
    return idx.search(q.n, q.indptr, q.indices, q.values, k, make())


@pytest.mark.parametrize("kind", ["fp32", "sq8", "brutal"])
def test_concurrent_searches_equal_single_threaded(kind):
    docs, qs = golden_corpus()
    if kind == "fp32":
        spec = SEISMIC
    elif kind == "sq8":
        spec = sq_spec(float(docs.values.min()), float(docs.values.max()))
    else:
        spec = "brutal"

    def build():
        idx = nsparse.index_factory(docs.dim, spec)
        idx.add(docs.n, docs.indptr, docs.indices, docs.values)
        if kind != "brutal":  # BrutalIndex has no build step (Index::build throws, index.cpp:30)
            idx.build()
        return idx

    tasks = _tasks(qs, docs.n)
    if kind == "brutal":
        # exact search takes k and a selector, not SEISMIC parameters
        sel = np.arange(0, docs.n, 3, dtype=np.int32)

        def bp(select):
            def make():
                prm = nsparse.SearchParameters()
                if select:
                    prm.set_id_selector(nsparse.SetIDSelector(sel))
                return prm
            return make
        tasks = [(n, q, k, bp(n == "tail-sel")) for n, q, k, _ in tasks]

    alone = build()
    want = [_run(alone, t) for t in tasks]

    # a fresh index: the threads' first searches race to upload it
    shared = build()
    errors, got = [], {}

    def worker(tid):
        try:
            rng = np.random.default_rng(tid)
            for r in range(ROUNDS):
                for j in rng.permutation(len(tasks)):
                    got[(tid, r, int(j))] = _run(shared, tasks[j])
        except Exception as e:  # surfaced below, with the thread's id
            errors.append((tid, repr(e)))

    threads = [threading.Thread(target=worker, args=(t,)) for t in range(N_THREADS)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    assert len(got) == N_THREADS * ROUNDS * len(tasks)
    for (tid, r, j), (D, L) in got.items():
        np.testing.assert_array_equal(L, want[j][1], err_msg=f"thread {tid} task {tasks[j][0]}")
        np.testing.assert_array_equal(D, want[j][0], err_msg=f"thread {tid} task {tasks[j][0]}")
