"""The build's host tie order against the reference's posting truncation.

For fp32 posting lists whose kept values tie, the SEISMIC build takes the
kept order from nsp::reference_kept_order (csrc/ref_order.cpp): the
reference's own std::ranges::sort over (value, doc) pairs in doc order. Here
that function is compiled into a small driver, and on a corpus whose values
sit on a coarse grid (ties everywhere) every truncated list must equal the
reference's InvertedList::prune_and_keep_doc_ids
(invlists/inverted_lists.cpp:110-132), called through the reference library
compiled from its sources (oracle/_ref).
"""

import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle as O
from nsparse_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "neural-sparse-cpp_b200", "csrc")

DRIVER = r"""
#include <cstdio>
#include <fstream>
#include <vector>
#include "ref_order.h"
extern "C" int ref_prune_and_keep(int esz, int32_t n, const int32_t* doc_ids,
                                  const uint8_t* value_bytes, int32_t lambda,
                                  int32_t* out_ids, int32_t* out_n);
template <class T> std::vector<T> rd(const std::string& p) {
    std::ifstream f(p, std::ios::binary | std::ios::ate);
    const size_t n = f.tellg();
    f.seekg(0);
    std::vector<T> v(n / sizeof(T));
    f.read(reinterpret_cast<char*>(v.data()), n);
    return v;
}
int main(int argc, char** argv) {
    const std::string d = argv[1];
    const int cap = std::atoi(argv[2]);
    nsp::HostCsr h;
    h.dim = std::atoi(argv[3]);
    h.esz = 4;
    h.indptr = rd<int32_t>(d + "/indptr.bin");
    h.indices = rd<uint16_t>(d + "/indices.bin");
    h.values = rd<uint8_t>(d + "/values.bin");
    const auto post = rd<int64_t>(d + "/post.bin");
    const auto lists = rd<int32_t>(d + "/lists.bin");
    std::vector<int32_t> out;
    nsp::reference_kept_order(h, post, lists, cap, out);
    std::vector<std::vector<int32_t>> ids(h.dim);
    std::vector<std::vector<float>> vals(h.dim);
    const float* v = reinterpret_cast<const float*>(h.values.data());
    for (size_t doc = 0; doc + 1 < h.indptr.size(); ++doc)
        for (int32_t e = h.indptr[doc]; e < h.indptr[doc + 1]; ++e) {
            ids[h.indices[e]].push_back(static_cast<int32_t>(doc));
            vals[h.indices[e]].push_back(v[e]);
        }
    std::vector<int32_t> ref(cap);
    int bad = 0;
    for (size_t j = 0; j < lists.size(); ++j) {
        const int t = lists[j];
        int32_t n = 0;
        if (ref_prune_and_keep(4, static_cast<int32_t>(ids[t].size()), ids[t].data(),
                               reinterpret_cast<const uint8_t*>(vals[t].data()), cap, ref.data(),
                               &n) != 0 || n != cap)
            return 2;
        for (int i = 0; i < cap; ++i)
            if (ref[i] != out[j * cap + i]) { ++bad; break; }
    }
    std::printf("%zu %d\n", lists.size(), bad);
    return 0;
}
"""


@pytest.mark.skipif(not O.ref_available("generic") or shutil.which("g++") is None,
                    reason="needs the reference library (oracle/_ref) and g++")
def test_host_tie_order_equals_reference_truncation(tmp_path):
    base = synth.docs_config0(30000, seed=21)
    values = (np.round(base.values * 4) / 4 + 0.25).astype(np.float32)
    cap = 200
    df = np.bincount(base.indices, minlength=base.dim)
    post = np.concatenate([[0], np.cumsum(df)]).astype(np.int64)
    lists = np.flatnonzero(df > cap).astype(np.int32)
    assert len(lists) > 100
    base.indptr.astype(np.int32).tofile(tmp_path / "indptr.bin")
    base.indices.astype(np.uint16).tofile(tmp_path / "indices.bin")
    values.tofile(tmp_path / "values.bin")
    post.tofile(tmp_path / "post.bin")
    lists.tofile(tmp_path / "lists.bin")
    src = tmp_path / "driver.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "driver"
    ref_dir = os.path.join(ROOT, "oracle", "_ref")
    subprocess.run(["g++", "-O2", "-std=c++20", f"-I{CSRC}", f"-I{os.path.join(ROOT, 'include')}",
                    "-I/usr/local/cuda/include", str(src), os.path.join(CSRC, "ref_order.cpp"),
                    os.path.join(ref_dir, "libnsparse_ref_generic.so"), f"-Wl,-rpath,{ref_dir}",
                    "-lpthread", "-o", str(exe)], check=True)
    r = subprocess.run([str(exe), str(tmp_path), str(cap), str(base.dim)], capture_output=True,
                       text=True, check=True)
    n, bad = map(int, r.stdout.split())
    assert n == len(lists) and bad == 0


SUMMARY_DRIVER = r"""
#include <algorithm>
#include <cstdio>
#include <fstream>
#include <vector>
#include "ref_order.h"
template <class T> std::vector<T> rd(const std::string& p) {
    std::ifstream f(p, std::ios::binary | std::ios::ate);
    const size_t n = f.tellg();
    f.seekg(0);
    std::vector<T> v(n / sizeof(T));
    f.read(reinterpret_cast<char*>(v.data()), n);
    return v;
}
int main(int argc, char** argv) {
    const std::string d = argv[1];
    nsp::HostCsr h;
    h.dim = std::atoi(argv[2]);
    const float alpha = std::atof(argv[3]);
    h.esz = 4;
    h.indptr = rd<int32_t>(d + "/indptr.bin");
    h.indices = rd<uint16_t>(d + "/indices.bin");
    h.values = rd<uint8_t>(d + "/values.bin");
    const auto cdocs = rd<int32_t>(d + "/cdocs.bin");
    const auto coff = rd<int32_t>(d + "/coff.bin");
    for (size_t c = 0; c + 1 < coff.size(); ++c) {
        auto kept = nsp::reference_summary_kept(h, cdocs.data() + coff[c],
                                                static_cast<size_t>(coff[c + 1] - coff[c]), alpha);
        std::sort(kept.begin(), kept.end());
        for (auto t : kept) std::printf("%u ", t);
        std::printf("\n");
    }
    return 0;
}
"""


def _first_k_by_term(docs, values, cdocs, alpha):
    """The kept terms if ties at the cut went by ascending term (the device
    order before the host settles ties), float32 arithmetic in the
    reference's order."""
    acc, order = {}, []
    total = np.float32(0)
    for d in cdocs:
        for e in range(docs.indptr[d], docs.indptr[d + 1]):
            t, v = int(docs.indices[e]), np.float32(values[e])
            if t not in acc:
                acc[t] = max(np.float32(0), v)
                order.append(t)
                total = np.float32(total + acc[t])
            elif v > acc[t]:
                total = np.float32(total + np.float32(v - acc[t]))
                acc[t] = v
    pairs = sorted(order, key=lambda t: (-acc[t], t))
    addup = np.float32(0)
    for j, t in enumerate(pairs):
        addup = np.float32(addup + acc[t])
        if np.float32(addup / total) >= np.float32(alpha):
            return sorted(pairs[:j + 1])
    return sorted(pairs)


@pytest.mark.skipif(not O.ref_available("generic") or shutil.which("g++") is None,
                    reason="needs the reference library (oracle/_ref) and g++")
def test_host_summary_cut_equals_reference_summarize_under_ties(tmp_path):
    """nsp::reference_summary_kept (the build's host step for fp32 blocks whose
    alpha cut falls between equal maxima) keeps the terms the reference's
    InvertedListClusters::summarize keeps, block by block, on values that tie
    constantly -- including blocks where taking the tied terms by ascending
    term would keep others."""
    base = synth.docs_config0(4000, seed=5)
    values = (np.round(base.values * 4) / 4 + 0.25).astype(np.float32)
    alpha = 0.4
    rng = np.random.default_rng(9)
    sizes = rng.integers(3, 30, 300)
    cdocs = rng.integers(0, base.n, int(sizes.sum())).astype(np.int32)
    coff = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    L = O.ref_lib("generic")
    cap = 1 << 26
    buf = np.empty(cap, np.uint8)
    n = L.ref_summarize(base.dim, 4, base.n, base.indptr.ctypes.data, base.indices.ctypes.data,
                        values.ctypes.data, cdocs.ctypes.data, coff.ctypes.data, len(sizes),
                        alpha, buf.ctypes.data, cap)
    assert n > 0
    ref = O._read_clusters(O._Rd(buf[:n].tobytes()))
    col_of = np.repeat(np.arange(len(ref["term_ids"])), np.diff(ref["term_ptr"]))
    want = [sorted(ref["term_ids"][col_of[ref["csc_cluster"] == c]].tolist())
            for c in range(len(sizes))]
    for name, a in (("indptr", base.indptr.astype(np.int32)),
                    ("indices", base.indices.astype(np.uint16)), ("values", values),
                    ("cdocs", cdocs), ("coff", coff)):
        a.tofile(tmp_path / f"{name}.bin")
    src = tmp_path / "sdriver.cpp"
    src.write_text(SUMMARY_DRIVER)
    exe = tmp_path / "sdriver"
    subprocess.run(["g++", "-O2", "-std=c++20", f"-I{CSRC}", f"-I{os.path.join(ROOT, 'include')}",
                    "-I/usr/local/cuda/include", str(src), os.path.join(CSRC, "ref_order.cpp"),
                    "-lpthread", "-o", str(exe)], check=True)
    r = subprocess.run([str(exe), str(tmp_path), str(base.dim), str(alpha)], capture_output=True,
                       text=True, check=True)
    got = [[int(x) for x in line.split()] for line in r.stdout.splitlines()]
    assert got == want
    by_term = [_first_k_by_term(base, values, cdocs[coff[c]:coff[c + 1]], alpha)
               for c in range(len(sizes))]
    assert sum(a != b for a, b in zip(by_term, want)) > 0, "no block exercised a tie at the cut"
