"""Multi-cell kernels of the particle-cell and sampling pyramids, the pulling
scheme, the equivalence step and the sampling gather, checked on the CPU
against the library's own per-cell forms.

The helpers and kernels are taken verbatim from libapr_b200/csrc/structure.cu
(and the status codes and idx3 from kernels.cuh / common.cuh), compiled with
g++ behind the host stand-ins of tests/cpp/bytewise_prelude.hpp, and run
thread by thread by tests/cpp/bytewise_main.cpp: the word-wide status tests
against the per-byte rules for every byte value in every position, and whole
launches of set_filler8, eqopt8 (both min types), fill_parent4,
pyramid_fill4, pyr_mean_u16x2 and gather4 against set_filler, eqopt,
fill_parent, pyramid_fill, pyr_mean_u16 and gather on random levels.  The GPU
parity tests compare the same kernels with the oracle on real volumes; this
test also covers status bytes and row shapes those volumes never produce.
"""
import os
import re
import shutil
import subprocess

import pytest

from tests.conftest import ROOT

CSRC = os.path.join(ROOT, "libapr_b200", "csrc")
CPP = os.path.join(ROOT, "tests", "cpp")


def _read(name):
    with open(os.path.join(CSRC, name)) as f:
        return f.read()


def _block(src, start):
    """The definition that opens with `start`, through its closing brace at column 0."""
    a = src.index(start)
    return src[a:src.index("\n}\n", a) + 3]


def _line(src, start):
    a = src.index(start)
    return src[a:src.index("\n", a) + 1]


def _translation_unit():
    st, kc, cc = _read("structure.cu"), _read("kernels.cuh"), _read("common.cuh")
    assert re.search(r"struct LevelDims \{\s*int yn, xn, zn;\s*\};", st), "LevelDims changed: update the prelude"
    a = kc.index("constexpr uint8_t kEmpty")
    status = kc[a:kc.index(";", a) + 1] + "\n"
    parts = [status, _block(cc, "__host__ __device__ __forceinline__ size_t idx3(")]
    parts += [_block(st, s) for s in (
        "__device__ __forceinline__ void cell_of(",
        "template <int MODE>\n__device__ __forceinline__ bool dil_source(",
        "__device__ __forceinline__ uint32_t bytes_eq(",
    )]
    parts += [_line(st, "__device__ __forceinline__ unsigned high_bits4("),
              _line(st, "__device__ __forceinline__ uint32_t nibble_high_bytes(")]
    parts += [_block(st, s) for s in (
        "__device__ __forceinline__ uint32_t bytes_in_1_to(",
        "template <int MODE>\n__device__ __forceinline__ uint32_t dil_source4(",
        "template <int MODE>\n__device__ __forceinline__ unsigned dil_bits16(",
        "template <int MODE>\n__device__ __forceinline__ uint32_t dil_target4(",
        "__device__ __forceinline__ bool row_group(",
        "__global__ void set_filler_kernel(",
        "__global__ void set_filler8_kernel(",
        "__global__ void eqopt_kernel(",
        "__global__ void eqopt8_kernel(",
        "__global__ void fill_parent_kernel(",
        "__global__ void fill_parent4_kernel(",
        "__global__ void pyramid_fill_kernel(",
        "__global__ void pyramid_fill4_kernel(",
        "__global__ void pyr_mean_u16_kernel(",
        "__global__ void pyr_mean_u16x2_kernel(",
        "__global__ void gather_kernel(",
        "__global__ void gather4_kernel(",
    )]
    with open(os.path.join(CPP, "bytewise_prelude.hpp")) as f:
        prelude = f.read()
    with open(os.path.join(CPP, "bytewise_main.cpp")) as f:
        main = f.read()
    return prelude + "\n".join(parts) + main


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_byte_parallel_kernels_match_per_cell_kernels(tmp_path):
    src = tmp_path / "bytewise_check.cpp"
    src.write_text(_translation_unit())
    exe = str(tmp_path / "bytewise_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-o", exe, str(src)], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "helpers 0, launches 0 + pyramids 0 of" in r.stdout and "gathers 0 mismatched" in r.stdout, r.stdout
