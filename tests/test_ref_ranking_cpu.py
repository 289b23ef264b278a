"""The restated ranking order (csrc/ref_ranking.cuh) against the reference's.

The first list's visiting order is the reference's std::ranges::sort of block
indices by summary score (seismic_common.h:105-115), an unstable sort: with
uint8 codes block scores tie constantly, and the visiting order of tied blocks
decides which docs the pruned walk reaches. The top-k holder is the
reference's TopKHolder (utils/ranker.h), a std::priority_queue whose sift
steps decide which of several equal scores is dropped and in which order
equal scores come out. Here the header is compiled for the host and checked,
on tie-heavy inputs, against:

* std::ranges::sort with the reference's comparator (the same call the
  reference makes), for the one-thread sort and for the split a warp runs
  (its lanes' ranges emulated on the host);
* std::make_heap + std::sort_heap (the depth-budget fallback);
* the reference's own TopKHolder, included from the reference's sources.
"""

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "neural-sparse-cpp_b200", "csrc")
REFERENCE = os.environ.get("NSP_REFERENCE_DIR", "/root/reference")
SHIM = os.path.join(ROOT, "oracle", "absl_shim")

DRIVER = r"""
#include <algorithm>
#include <cstdio>
#include <numeric>
#include <queue>
#include <random>
#include <vector>
#include "ref_ranking.cuh"
#ifdef WITH_REFERENCE
#include "nsparse/utils/ranker.h"
#endif
using namespace nsp::ranking;

static std::vector<int> ref_order(const std::vector<float>& s) {
    std::vector<int> o(s.size());
    std::iota(o.begin(), o.end(), 0);
    std::ranges::sort(o, [&](int a, int b) { return s[a] > s[b]; });
    return o;
}

static std::vector<Blk> blks(const std::vector<float>& s) {
    std::vector<Blk> a(s.size());
    for (size_t i = 0; i < s.size(); ++i) a[i] = Blk{s[i], static_cast<int32_t>(i)};
    return a;
}

// the warp split: 32 lanes' ranges after kSortSplitRounds rounds, each lane
// then finishing its range
static void split_sort(std::vector<Blk>& a) {
    const int n = static_cast<int>(a.size());
    SortRange r[32];
    for (int j = 0; j < 32; ++j) r[j] = SortRange{0, j == 0 ? n : 0, n > 0 ? 2 * floor_log2(n) : 0};
    for (int round = 0; round < kSortSplitRounds; ++round) {
        const int active = 1 << round;
        int cut[32];
        for (int j = 0; j < 32; ++j) cut[j] = j < active ? split_cut(a.data(), r[j]) : -1;
        SortRange p[32];
        int pc[32];
        for (int j = 0; j < 32; ++j) {
            p[j] = r[j >> 1];
            pc[j] = cut[j >> 1];
        }
        for (int j = 0; j < 2 * active && j < 32; ++j) r[j] = split_child(p[j], pc[j], (j & 1) != 0);
    }
    for (int j = 0; j < 32; ++j)
        if (r[j].l > r[j].f) sort_range(a.data(), r[j].f, r[j].l, r[j].d);
}

int main() {
    std::mt19937 rng(12345);
    int bad = 0, cases = 0;
    std::vector<int> sizes;
    for (int n = 0; n <= 70; ++n) sizes.push_back(n);
    for (int n : {100, 127, 128, 129, 255, 256, 400, 511, 600, 1000, 2047, 4000, 6000})
        sizes.push_back(n);
    for (int n : sizes) {
        for (int rep = 0; rep < 12; ++rep) {
            std::vector<float> s(n);
            const int kind = rep % 6;
            const int levels = 1 + static_cast<int>(rng() % (kind == 0 ? 3 : 40));
            for (int i = 0; i < n; ++i) {
                switch (kind) {
                    case 0: case 1: case 2: s[i] = static_cast<float>(rng() % levels); break;
                    case 3: s[i] = static_cast<float>(i % levels); break;             // saw
                    case 4: s[i] = static_cast<float>(std::min(i, n - 1 - i) % levels); break;  // organ pipe
                    default: s[i] = (rng() % 4 == 0) ? -0.0f : static_cast<float>(rng() % 5) * 0.5f;
                }
            }
            const std::vector<int> want = ref_order(s);
            std::vector<Blk> a = blks(s), b = blks(s);
            sort_blocks_like_reference(a.data(), n);
            split_sort(b);
            ++cases;
            for (int i = 0; i < n; ++i)
                if (a[i].b != want[i] || b[i].b != want[i]) { ++bad; break; }
        }
    }
    // depth-budget fallback: make_heap + sort_heap with the same comparator
    for (int n : {2, 3, 17, 33, 100, 257}) {
        for (int rep = 0; rep < 20; ++rep) {
            std::vector<float> s(n);
            for (int i = 0; i < n; ++i) s[i] = static_cast<float>(rng() % 7);
            std::vector<Blk> a = blks(s), w = blks(s);
            heap_sort_range(a.data(), 0, n);
            auto cmp = [](const Blk& x, const Blk& y) { return x.s > y.s; };
            std::make_heap(w.begin(), w.end(), cmp);
            std::sort_heap(w.begin(), w.end(), cmp);
            ++cases;
            for (int i = 0; i < n; ++i)
                if (a[i].b != w[i].b) { ++bad; break; }
        }
    }
#ifdef WITH_REFERENCE
    // the top-k holder: offers with many equal scores
    for (int k : {1, 2, 3, 7, 10, 16, 33, 100}) {
        for (int rep = 0; rep < 40; ++rep) {
            const int offers = 1 + static_cast<int>(rng() % 600);
            const int levels = 1 + static_cast<int>(rng() % 12);
            nsparse::detail::TopKHolder<int> ref(k);
            std::vector<float> hs(k);
            std::vector<int32_t> hid(k);
            TopK h{hs.data(), hid.data()};
            int n = 0;
            for (int i = 0; i < offers; ++i) {
                const float sc = static_cast<float>(rng() % levels);
                ref.add(sc, i);
                topk_add(h, n, k, sc, i);
                if (static_cast<int>(ref.size()) != n || (n > 0 && ref.peek_score() != hs[0])) {
                    ++bad;
                    break;
                }
            }
            auto [rs, ri] = ref.top_k_items_descending();
            std::vector<float> os(n);
            std::vector<int32_t> oi(n);
            topk_drain_descending(h, n, os.data(), oi.data());
            ++cases;
            if (static_cast<int>(ri.size()) != n) { ++bad; continue; }
            for (int i = 0; i < n; ++i)
                if (ri[i] != oi[i] || rs[i] != os[i]) { ++bad; break; }
        }
    }
#endif
    std::printf("%d %d\n", cases, bad);
    return 0;
}
"""


def _build(tmp_path, with_reference):
    src = tmp_path / "ranking.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "ranking"
    cmd = ["g++", "-O2", "-std=c++20", f"-I{CSRC}", str(src), "-o", str(exe)]
    if with_reference:
        cmd[4:4] = ["-DWITH_REFERENCE", f"-I{REFERENCE}", f"-I{SHIM}"]
    subprocess.run(cmd, check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, check=True)
    return tuple(map(int, r.stdout.split()))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_block_order_equals_std_ranges_sort(tmp_path):
    cases, bad = _build(tmp_path, with_reference=False)
    assert cases > 1000 and bad == 0


@pytest.mark.skipif(shutil.which("g++") is None
                    or not os.path.exists(os.path.join(REFERENCE, "nsparse", "utils", "ranker.h")),
                    reason="needs g++ and the reference's sources")
def test_topk_holder_equals_reference_ranker(tmp_path):
    cases, bad = _build(tmp_path, with_reference=True)
    assert cases > 1000 and bad == 0
