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
