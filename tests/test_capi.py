"""CPU tests of the C ABI: the library loads, exports every symbol include/*.h declares,
and its host-only entry points behave (no GPU is touched here)."""
from __future__ import annotations

import ctypes as C
import glob
import os
import re
import subprocess

import pytest

from conftest import ROOT

from btc_b200 import _lib


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        names |= set(re.findall(r"^BTC_API\s+[\w\s\*]+?\b(btc_\w+)\s*\(", text, flags=re.M))
    return names


def test_library_is_built():
    assert os.path.exists(_lib.LIB_PATH), "run __graft_entry__.build() first"


def test_every_declared_symbol_is_exported():
    decl = declared_symbols()
    assert len(decl) >= 19
    L = _lib.lib()
    for name in sorted(decl):
        assert hasattr(L, name), name
    assert decl == set(_lib.EXPORTS) | (decl - set(_lib.EXPORTS)), "EXPORTS list out of date"
    assert set(_lib.EXPORTS) <= decl


def test_dynamic_symbol_table_has_only_the_abi():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    btc = {s for s in exported if s.startswith("btc_")}
    assert btc == declared_symbols()


def test_library_is_sm100a_only():
    """The shared library carries sm_100a code only (cuobjdump is not used: the list of
    architectures comes from the build flags recorded in the Makefile)."""
    mk = open(os.path.join(ROOT, "btc-tc-artifact_b200", "Makefile")).read()
    assert "arch=compute_100a,code=sm_100a" in mk
    assert "sm_90" not in mk and "sm_80" not in mk


def test_host_only_calls():
    L = _lib.lib()
    assert L.btc_abi_version() >> 16 == 1
    assert L.btc_strerror(0) == b"ok"
    assert L.btc_strerror(_lib.BTC_E_RANGE) == b"vertex id out of range"
    assert L.btc_default_tau(128) == 1024 and L.btc_default_tau(32) == 64


@pytest.mark.parametrize("nnz,rows,mode,want", [
    (131_000, 16_384, 0, 32),        # avg 8 < 15
    (3_298_428, 262_144, 0, 32),     # avg 12.6 < 15 (the reference's choice for the stencil)
    (64_153_542, 2_395_930, 0, 128), # avg 26.8, rows >= 50k
    (2_000_000, 40_000, 0, 32),      # rows < 50k
    (10, 10, 1, 32),
    (10, 10, 2, 128),
])
def test_btc_lite_policy(nnz, rows, mode, want):
    """apps/btc_tc_lite.cu:45-65."""
    assert _lib.lib().btc_lite_select_tile_cols(nnz, rows, mode) == want


def test_bad_arguments_rejected_without_gpu():
    L = _lib.lib()
    out = C.c_void_p(None)
    # null output handle and bad tile width are rejected before any CUDA call
    assert L.btc_build_bitbsr(None, None, 0, 0, 128, 0, None, None) == _lib.BTC_E_INVAL
    assert L.btc_count(None, -1, None, None, None) == _lib.BTC_E_INVAL
    assert L.btc_bitbsr_info(None, None) == _lib.BTC_E_INVAL
    L.btc_free(None)
    s = _lib.BtcBcsrDevice()
    L.btc_bcsr_free(C.byref(s))  # zeroed struct: no-op
    assert L.btc_bcsr_get_result(C.byref(s), None) == _lib.BTC_E_INVAL
    del out


def test_header_compiles_as_c_and_cpp(tmp_path):
    src = tmp_path / "t.c"
    src.write_text('#include "btc_c.h"\nint main(void){btc_bcsr_device d; (void)d; return 0;}\n')
    inc = os.path.join(ROOT, "include")
    subprocess.run(["g++", "-x", "c", "-std=c99", "-Wall", "-Werror", "-I", inc, "-c", str(src),
                    "-o", str(tmp_path / "t.o")], check=True)
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I", inc, "-c", str(src),
                    "-o", str(tmp_path / "t2.o")], check=True)


def test_compat_app_is_built_and_prints_usage():
    """apps/btc_tc_lite.cu (the reference's BTC-Lite CLI over include/btc_compat.hpp)."""
    app = os.path.join(os.path.dirname(_lib.LIB_PATH), "btc_tc_lite")
    assert os.path.exists(app)
    out = subprocess.run([app], capture_output=True, text=True)
    assert out.returncode == 1 and "Usage" in out.stdout


def test_compat_header_compiles_with_nvcc(tmp_path):
    """include/btc_compat.hpp gives the reference's namespace-btc names and signatures."""
    src = tmp_path / "c.cu"
    src.write_text(
        '#include "btc_compat.hpp"\n'
        "struct Coo { int num_rows; size_t num_entries;\n"
        "  thrust::device_vector<int> row_indices, column_indices; };\n"
        "unsigned long long f(Coo& coo) {\n"
        "  btc::BCSR_16x128_Device a; btc::convert_coo_to_bcsr_16x128_gpu(a, coo);\n"
        "  float ms; unsigned long long c = btc::count_triangles_16x128_adaptive(a, 2048, &ms);\n"
        "  btc::BCSR_16x32_Device b; btc::convert_coo_to_bcsr_16x32_gpu(b, coo);\n"
        "  c += btc::count_triangles_16x32_adaptive(b); c += a.get_result(); a.reset_result();\n"
        "  a.free(); b.free(); return c; }\n")
    subprocess.run(["nvcc", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-I",
                    os.path.join(ROOT, "include"), "-c", str(src), "-o", str(tmp_path / "c.o")],
                   check=True)
