"""include/nsparse_c.h is plain C: a C11 program (gcc, -Wall -Werror) includes
it, links libnsparse_b200.so and drives the host-side entry points an FFI
binding calls first -- factory, add, counts, the fourcc, selectors, search
parameters, write/read of an index file, CSR conversion and the mapped read,
and an error status with its message. No GPU is needed for these calls."""

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "neural-sparse-cpp_b200", "lib", "libnsparse_b200.so")

PROGRAM = r"""
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "nsparse_c.h"

#define CHECK(x) do { if ((x) != NSP_OK) { printf("fail %s: %s\n", #x, nsp_last_error()); return 1; } } while (0)

int main(int argc, char** argv) {
    (void)argc;
    char path[4096], csr[4096], mcsr[4096];
    snprintf(path, sizeof path, "%s/c.idx", argv[1]);
    snprintf(csr, sizeof csr, "%s/m.csr", argv[1]);
    snprintf(mcsr, sizeof mcsr, "%s/m.csr.mcsr", argv[1]);
    const int32_t indptr[] = {0, 2, 3, 5};
    const uint16_t indices[] = {0, 5, 2, 1, 7};
    const float values[] = {1.5f, 0.5f, 2.0f, 0.25f, 3.0f};

    nsp_index_t* idx = NULL;
    CHECK(nsp_index_factory(8, "seismic,lambda=10|beta=2|alpha=0.4|seed=3", &idx));
    CHECK(nsp_index_add(idx, 3, indptr, indices, values));
    int64_t n = 0;
    int32_t dim = 0;
    char cc[4];
    CHECK(nsp_index_num_vectors(idx, &n));
    CHECK(nsp_index_dimension(idx, &dim));
    CHECK(nsp_index_fourcc(idx, cc));
    printf("vectors %lld dim %d id %.4s\n", (long long)n, dim, cc);
    CHECK(nsp_write_index(idx, path));
    nsp_index_t* back = NULL;
    CHECK(nsp_read_index(path, 0, &back));
    CHECK(nsp_index_num_vectors(back, &n));
    printf("read back %lld\n", (long long)n);

    const int32_t ids[] = {1, 4};
    nsp_id_selector_t* set = NULL;
    nsp_id_selector_t* not_set = NULL;
    CHECK(nsp_id_selector_set_new(2, ids, &set));
    CHECK(nsp_id_selector_not_new(set, &not_set));
    int a = 0, b = 0;
    CHECK(nsp_id_selector_is_member(set, 4, &a));
    CHECK(nsp_id_selector_is_member(not_set, 4, &b));
    printf("selectors %d %d\n", a, b);
    nsp_search_params_t* params = NULL;
    CHECK(nsp_seismic_search_params_new(10, 0.8f, &params));
    CHECK(nsp_search_params_set_id_selector(params, set));

    FILE* f = fopen(csr, "wb");
    const int64_t header[3] = {3, 8, 5};
    fwrite(header, sizeof header, 1, f);
    for (int i = 0; i < 4; ++i) { int64_t w = indptr[i]; fwrite(&w, sizeof w, 1, f); }
    for (int i = 0; i < 5; ++i) { int32_t w = indices[i]; fwrite(&w, sizeof w, 1, f); }
    fwrite(values, sizeof values, 1, f);
    fclose(f);
    CHECK(nsp_csr_convert(csr, mcsr));
    nsp_index_t* mapped = NULL;
    CHECK(nsp_index_factory(8, "seismic,lambda=10|beta=2|alpha=0.4|seed=3", &mapped));
    CHECK(nsp_index_read_csr(mapped, mcsr, 1));
    CHECK(nsp_index_num_vectors(mapped, &n));
    printf("mapped %lld\n", (long long)n);

    nsp_index_t* bad = NULL;
    const nsp_status_t st = nsp_index_factory(8, "nonsense", &bad);
    printf("status %d message %s\n", (int)st, nsp_last_error());

    CHECK(nsp_search_params_free(params));
    CHECK(nsp_id_selector_free(not_set));
    CHECK(nsp_id_selector_free(set));
    CHECK(nsp_index_free(mapped));
    CHECK(nsp_index_free(back));
    CHECK(nsp_index_free(idx));
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None or not os.path.exists(LIB),
                    reason="needs gcc and the built library")
def test_header_is_plain_c_and_host_calls_work(tmp_path):
    src = tmp_path / "client.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "client"
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", "-pedantic",
                    f"-I{os.path.join(ROOT, 'include')}", str(src), LIB,
                    f"-Wl,-rpath,{os.path.dirname(LIB)}", "-o", str(exe)], check=True)
    r = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, check=True)
    assert r.stdout.splitlines() == [
        "vectors 3 dim 8 id SEIS",
        "read back 3",
        "selectors 1 0",
        "mapped 3",
        "status 1 message Unknown index type: nonsense",
    ]
