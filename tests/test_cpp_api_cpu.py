"""Source compatibility of the C++ API (include/nsparse/*.h): one client
program written against the reference's API (index_factory, add, num_vectors,
id, write_index / read_index, selectors, search parameters, the CSR layouts
and read_csr under the mapped residency, exception types) is compiled
unchanged twice -- against this engine's headers and libnsparse_b200.so, and
against the reference's headers and the reference library compiled from its
sources (oracle/_ref) -- and both builds must print the same lines and write
the same index file. Nothing here needs a GPU: the calls are host-side."""

import os
import shutil
import subprocess

import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFERENCE = os.environ.get("NSP_REFERENCE_DIR", "/root/reference")

CLIENT = r"""
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "nsparse/id_selector.h"
#include "nsparse/index.h"
#include "nsparse/index_factory.h"
#include "nsparse/io/index_io.h"
#include "nsparse/seismic_index.h"
#include "nsparse/seismic_scalar_quantized_index.h"
#include "nsparse/utils/csr_layout.h"

int main(int argc, char** argv) {
    const std::string dir = argv[1];
    const char* spec = "seismic,lambda=10|beta=2|alpha=0.4|seed=3";
    // 3 docs over 8 terms
    std::vector<nsparse::idx_t> indptr = {0, 2, 3, 5};
    std::vector<nsparse::term_t> indices = {0, 5, 2, 1, 7};
    std::vector<float> values = {1.5f, 0.5f, 2.0f, 0.25f, 3.0f};

    std::unique_ptr<nsparse::Index> idx(nsparse::index_factory(8, spec));
    idx->add(3, indptr.data(), indices.data(), values.data());
    const auto id = idx->id();
    std::printf("vectors %zu dim %d id %c%c%c%c\n", idx->num_vectors(), idx->get_dimension(),
                id[0], id[1], id[2], id[3]);
    std::string path = dir + "/c.idx";
    nsparse::write_index(idx.get(), path.data());
    std::unique_ptr<nsparse::Index> back(nsparse::read_index(path.data(), 0));
    std::printf("read back %zu\n", back->num_vectors());

    std::vector<nsparse::idx_t> ids = {1, 4};
    nsparse::SetIDSelector set(ids.size(), ids.data());
    nsparse::NotIDSelector not_set(&set);
    std::printf("selectors %d %d %d %d\n", set.is_member(1), set.is_member(2),
                not_set.is_member(1), not_set.is_member(2));

    nsparse::SeismicSearchParameters sp(10, 0.8f);
    nsparse::SeismicSQSearchParameters sqp(0.0f, 4.0f, 12, 0.9f);
    std::printf("params %d %.2f %d %.2f %.1f %.1f\n", sp.cut, sp.heap_factor, sqp.cut,
                sqp.heap_factor, sqp.vmin, sqp.vmax);

    try {
        std::unique_ptr<nsparse::Index> bad(nsparse::index_factory(8, "nonsense"));
        std::printf("no exception\n");
    } catch (const std::invalid_argument&) {
        std::printf("invalid_argument\n");
    }

    namespace cl = nsparse::csr_layout;
    std::printf("layout %zu %zu %zu %s\n", cl::kHeaderBytes, cl::interchange_file_size(4, 5),
                cl::native_file_size(4, 5), cl::native_path("x").c_str());
    {
        std::ofstream f(dir + "/m.csr", std::ios::binary);
        const int64_t header[3] = {3, 8, 5};
        f.write(reinterpret_cast<const char*>(header), sizeof(header));
        for (auto v : indptr) {
            const int64_t w = v;
            f.write(reinterpret_cast<const char*>(&w), sizeof(w));
        }
        for (auto t : indices) {
            const int32_t w = t;
            f.write(reinterpret_cast<const char*>(&w), sizeof(w));
        }
        f.write(reinterpret_cast<const char*>(values.data()), values.size() * sizeof(float));
    }
    cl::convert(dir + "/m.csr", cl::native_path(dir + "/m.csr"));
    std::unique_ptr<nsparse::Index> mapped(nsparse::index_factory(8, spec));
    mapped->read_csr(cl::native_path(dir + "/m.csr").c_str(), nsparse::Residency::kMmap);
    std::printf("mapped %zu\n", mapped->num_vectors());
    try {
        mapped->read_csr(cl::native_path(dir + "/m.csr").c_str(), nsparse::Residency::kMmap);
        std::printf("no exception\n");
    } catch (const std::runtime_error&) {
        std::printf("runtime_error on a second mapped load\n");
    }
    return 0;
}
"""


def _build_and_run(tmp_path, name, includes, lib):
    src = tmp_path / "client.cpp"
    src.write_text(CLIENT)
    exe = tmp_path / f"client_{name}"
    subprocess.run(["g++", "-std=c++20", "-O1", *[f"-I{i}" for i in includes], str(src), lib,
                    f"-Wl,-rpath,{os.path.dirname(lib)}", "-o", str(exe)], check=True)
    out = tmp_path / name
    out.mkdir()
    r = subprocess.run([str(exe), str(out)], capture_output=True, text=True, check=True)
    return r.stdout, open(out / "c.idx", "rb").read()


@pytest.mark.skipif(shutil.which("g++") is None or not O.ref_available("generic")
                    or not os.path.isdir(os.path.join(REFERENCE, "nsparse")),
                    reason="needs g++, the reference sources and the reference library")
def test_reference_api_client_builds_and_agrees_against_both_libraries(tmp_path):
    ours = _build_and_run(tmp_path, "ours", [os.path.join(ROOT, "include"), "/usr/local/cuda/include"],
                          os.path.join(ROOT, "neural-sparse-cpp_b200", "lib", "libnsparse_b200.so"))
    ref = _build_and_run(tmp_path, "ref", [REFERENCE, os.path.join(ROOT, "oracle", "absl_shim")],
                         os.path.join(ROOT, "oracle", "_ref", "libnsparse_ref_generic.so"))
    assert "vectors 3 dim 8 id SEIS" in ours[0] and "mapped 3" in ours[0]
    assert ours[0] == ref[0]
    assert ours[1] == ref[1]
