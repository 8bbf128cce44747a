"""The C++ examples in INTEGRATION.md compile against include/rtscan_b200.h:
each block is wrapped in a function whose parameters declare the names the
block uses, and the whole file is syntax-checked with g++ (no GPU needed),
so the documented calls cannot drift from the ABI."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# parameters each block (in document order) expects from its surroundings
PARAMS = [
    "const char *text, uint64_t len",
    "rts_ctx *ctx, const rts_term *terms, const int32_t *offsets, int32_t nq, uint32_t *dev_bitmaps, "
    "uint64_t stride_words, uint64_t *dev_counts, void *stream, const uint32_t *const *host_cols, int32_t ncols, "
    "uint64_t nrows, uint32_t *host_bitmaps, uint64_t *host_counts, const rts_term *t, int32_t nt, "
    "uint32_t *host_bitmap",
    "rts_ctx *ctx, const uint32_t *dev_bitmap, uint64_t nrows, uint32_t *dev_rows, uint64_t capacity, "
    "uint64_t *dev_count, void *stream, int32_t col_price, int32_t col_discount, uint64_t *dev_sum128, "
    "const rts_term *terms, int32_t nterms, int32_t c, rts_term *coded_terms",
]


def test_cpp_examples_compile(tmp_path):
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("no g++")
    with open(os.path.join(ROOT, "INTEGRATION.md")) as f:
        blocks = re.findall(r"```c\+\+\n(.*?)```", f.read(), re.S)
    assert len(blocks) == len(PARAMS), "a C++ block was added or removed: list its parameters here"
    src = ["#include <cstdint>", "#include <vector>", '#include "rtscan_b200.h"']
    for i, (block, params) in enumerate(zip(blocks, PARAMS)):
        body = "\n".join(l for l in block.splitlines() if not l.startswith("#include"))
        src.append(f"void example_{i}({params}) {{\n{body}\n}}")
    path = tmp_path / "examples.cpp"
    path.write_text("\n".join(src) + "\n")
    r = subprocess.run([gxx, "-std=c++17", "-fsyntax-only", "-Wall", "-I", os.path.join(ROOT, "include"), str(path)],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-3000:]
