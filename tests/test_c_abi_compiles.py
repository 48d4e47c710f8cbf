"""The C-ABI as a C or C++ includer sees it, without a GPU: include/mpf.h compiles
as strict C99 in the plain-C smoke caller (tests/native/c_abi_smoke.c), and the C++
shim that INTEGRATION.md gives for the reference's hybrid_init / hybrid_runpf /
hybrid_free (runpf.h:795, 606, 984) compiles against mpf.h and stand-ins for the
reference's host types (tests/native/ref_types_stub.h)."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NATIVE = os.path.join(ROOT, "tests", "native")
CUDA_INC = "/usr/local/cuda/include"


def _need(tool):
    if not shutil.which(tool):
        pytest.skip(f"{tool} not available")


def test_c_smoke_caller_compiles_as_c99(tmp_path):
    _need("gcc")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", os.path.join(ROOT, "include"),
                    "-c", os.path.join(NATIVE, "c_abi_smoke.c"), "-o", str(tmp_path / "smoke.o")], check=True)


def test_header_compiles_as_cxx(tmp_path):
    _need("g++")
    src = tmp_path / "inc.cpp"
    src.write_text('#include "mpf.h"\nint main() { mpf_options o; mpf_default_options(&o); return o.max_it_nr; }\n')
    subprocess.run(["g++", "-std=c++11", "-Wall", "-Werror", "-pedantic", "-I", os.path.join(ROOT, "include"),
                    "-fsyntax-only", str(src)], check=True)


def test_integration_shim_compiles(tmp_path):
    _need("g++")
    if not os.path.exists(os.path.join(CUDA_INC, "cuda_runtime_api.h")):
        pytest.skip("CUDA headers not available")
    with open(os.path.join(ROOT, "INTEGRATION.md")) as f:
        doc = f.read()
    blocks = [b for b in re.findall(r"```cpp\n(.*?)```", doc, re.S) if "mpf_create(" in b]
    assert len(blocks) == 1, "INTEGRATION.md should hold exactly one C++ shim block"
    src = tmp_path / "shim.cpp"
    src.write_text('#include "ref_types_stub.h"\n' + blocks[0])
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), "-I", NATIVE,
                    "-I", CUDA_INC, "-c", str(src), "-o", str(tmp_path / "shim.o")], check=True)
