"""bench.py's reference arm (--impl reference: the reference's own CPU search,
compiled from its sources) runs here on a small corpus and prints one JSON
line carrying the keys the benchmark contract names."""

import json
import os
import subprocess
import sys

import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not O.ref_available("generic"), reason="reference library not built")
@pytest.mark.parametrize("workload", ["sq8-8.8m", "fp32-1m"])
def test_reference_arm_prints_one_contract_line(workload):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--workload", workload, "--docs", "20000", "--queries", "300",
                        "--steps", "2", "--warmup", "1"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT, check=True)
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config", "impl",
                "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["steps"] == 2 and d["value"] > 0
    assert d["config"]["docs"] == 20000
    assert d["dtype"] == ("u8" if workload == "sq8-8.8m" else "f32")
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"]
    lat = cb["per_query_1_thread"]
    assert lat["queries"] > 0 and 0 < lat["p50_ms"] <= lat["p99_ms"]


def test_row_parity_separates_tied_rows():
    sys.path.insert(0, ROOT)
    import numpy as np

    import bench
    D = np.array([[3.0, 2.0, 1.0], [5.0, 5.0, 4.0], [2.0, 1.0, -1.0]], np.float32)
    L = np.array([[7, 8, 9], [1, 2, 3], [4, 5, -1]], np.int32)
    # row 1 is tied (two scores of 5.0): its ids may come in either order
    Lr = np.array([[7, 8, 9], [2, 1, 3], [4, 5, -1]], np.int32)
    p = bench.row_parity(D, L, D.copy(), Lr)
    assert p["rows_identical_frac"] == 2 / 3 and p["rows_same_scores_frac"] == 1.0
    assert p["untied_rows"] == 2 and p["score_mismatches_untied_rows"] == 0
    Dr = D.copy()
    Dr[0, 1] = 2.5
    p = bench.row_parity(D, L, Dr, Lr)
    assert p["score_mismatches_untied_rows"] == 1 and p["untied_rows_identical_frac"] == 0.5


def test_exact_score_check_flags_a_wrong_score():
    sys.path.insert(0, ROOT)
    import numpy as np

    import bench
    from nsparse_b200 import synth
    docs = synth.docs_config2(1500, seed=0)
    qs = synth.queries_config2(12, seed=1)
    vmin, vmax = float(docs.values.min()), float(docs.values.max())
    dc = O.sq_encode_u8(vmin, vmax, docs.values).astype(np.int64)
    qc = O.sq_encode_u8(vmin, vmax, qs.values).astype(np.int64)
    rng = np.float32(vmax) - np.float32(vmin)
    dec = np.float32(rng * rng) / np.float32(255.0 * 255.0)
    D = np.zeros((qs.n, 10), np.float32)
    L = np.zeros((qs.n, 10), np.int32)
    for q in range(qs.n):
        dense = np.zeros(docs.dim, np.int64)
        s, e = qs.indptr[q], qs.indptr[q + 1]
        dense[qs.indices[s:e]] = qc[s:e]
        sc = np.array([int(np.dot(dc[docs.indptr[d]:docs.indptr[d + 1]],
                                  dense[docs.indices[docs.indptr[d]:docs.indptr[d + 1]]]))
                       for d in range(docs.n)])
        o = np.lexsort((np.arange(docs.n), -sc))[:10]
        L[q], D[q] = o, (sc[o].astype(np.float32) * dec).astype(np.float32)
    assert bench.sq_exact_check(docs, qs, D, L, vmin, vmax, qs.n) == \
        {"scores_checked": 10 * qs.n, "scores_not_exact": 0}
    D[3, 2] = np.nextafter(D[3, 2], np.float32(np.inf))
    assert bench.sq_exact_check(docs, qs, D, L, vmin, vmax, qs.n)["scores_not_exact"] == 1
