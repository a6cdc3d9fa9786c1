"""Builds handler modules on the CPU (nvcc cross-compiles for sm_100a): the
CMake function RTSPATIAL_COMPILE_SHADERS called exactly as the reference's own
projects call theirs (test/CMakeLists.txt:8-9: include dir, header name,
output dir, result variable; the result added to a target's sources), and the
Python compiler on a user header that includes <optix.h> as handler headers
written for the reference do.  Loading and running the modules is covered by
tests/test_gpu_handler_modules.py."""
import os
import shutil
import subprocess

import pytest

from rtspatial_b200 import handlers

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("cmake") is None, reason="cmake not installed")
def test_cmake_function_compiles_the_counting_module(tmp_path):
    src = tmp_path / "proj"
    src.mkdir()
    (src / "CMakeLists.txt").write_text(f"""
cmake_minimum_required(VERSION 3.18)
project(handler_module_user LANGUAGES NONE)
include("{ROOT}/cmake/rtspatial_shaders.cmake")
RTSPATIAL_COMPILE_SHADERS("{ROOT}/include/rtspatial/default_handlers" "counting_handlers.h"
        "${{CMAKE_BINARY_DIR}}/tests_ptx" PROGRAM_MODULES)
add_custom_target(shaders ALL DEPENDS ${{PROGRAM_MODULES}})
""")
    build = tmp_path / "build"
    subprocess.check_call(["cmake", "-S", str(src), "-B", str(build)], stdout=subprocess.DEVNULL)
    subprocess.check_call(["cmake", "--build", str(build)], stdout=subprocess.DEVNULL)
    cubin = build / "tests_ptx" / handlers.MODULE_FILE
    assert cubin.exists() and cubin.stat().st_size > 10_000
    # an ELF image with the module's entry points and version marker
    data = cubin.read_bytes()
    assert data[:4] == b"\x7fELF"
    for name in (b"rts_handler_query_v1_w16", b"rts_module_abi_version",
                 b"rts_module_builtin_handler"):
        assert name in data


def test_python_compiler_takes_a_reference_style_header(tmp_path):
    out = handlers.compile_module(os.path.join(ROOT, "tests", "cpp", "handlers",
                                               "pair_append_handlers.h"), str(tmp_path), force=True)
    data = open(out, "rb").read()
    assert data[:4] == b"\x7fELF" and b"rts_handler_query_v1_w4" in data
