"""The reference's own application sources (apps/btc_tc_lite.cu, apps/btc_tc_adaptive_16x128.cu),
unchanged, built against the engine through the include/btc_overlay headers by
oracle/ref/Makefile: the reference's I/O, formats and CPU count come from its tree, the
preprocess, Bit-BSR build and count from libbtc_b200.so.

CPU side: the binaries exist, link libbtc_b200.so and answer like the reference's
(usage text).  GPU side (-m gpu): each binary, fed a graph in the reference's binary CSR
format (graphs.write_bin_csr, btc/utils/io/read.h:255-299), prints the golden count on its
"Triangles (GPU)" line (and btc_tc_adaptive_16x128 with -v 1 the reference's own CPU count
on "Triangles (CPU)"), for every reorder mode the reference reads from BTC_REORDER.
"""
from __future__ import annotations

import os
import re
import subprocess

import pytest

from conftest import ROOT, golden_graph, load_golden

REF_OUT = os.path.join(ROOT, "oracle", "_ref")
APPS = ["btc_tc_lite", "btc_tc_adaptive_16x128"]


def _app(name):
    p = os.path.join(REF_OUT, f"ref_app_{name}")
    if not os.path.exists(p):
        pytest.skip(f"{p} not built (oracle/ref/Makefile needs a reference checkout)")
    return p


@pytest.mark.parametrize("name", APPS)
def test_app_links_the_engine(name):
    app = _app(name)
    ldd = subprocess.run(["ldd", app], capture_output=True, text=True).stdout
    lib = [l for l in ldd.splitlines() if "libbtc_b200.so" in l]
    assert lib and "not found" not in lib[0], ldd
    assert os.path.realpath(lib[0].split("=>")[1].split("(")[0].strip()) == os.path.realpath(
        os.path.join(ROOT, "btc-tc-artifact_b200", "btc_b200", "lib", "libbtc_b200.so"))
    out = subprocess.run([app], capture_output=True, text=True, timeout=60)
    assert "Usage" in out.stdout + out.stderr


def test_recipe_compiles_the_reference_sources_in_place():
    """The recipe names the reference's own app sources and the overlay ahead of its root
    (no copy of a reference source lives in this repository)."""
    mk = open(os.path.join(ROOT, "oracle", "ref", "Makefile")).read()
    assert "$(REF)/apps/%.cu" in mk
    assert mk.index("include/btc_overlay") < mk.index("-I$(REF) $<")


CASES = ["K33", "stencil27_10", "er_1000_8_s3", "rmat_12_16_s7", "sbm_2000_8_s2"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", APPS)
@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("reorder", ["0", "8", "9"])
def test_app_prints_the_golden_count(tmp_path, name, case, reorder):
    from btc_b200 import graphs as G
    from oracle import oracle as O
    app = _app(name)
    src, dst, n = golden_graph(case)
    rp, col, _ = O.lower_csr(src, dst, n)
    path = tmp_path / f"{case}.bin"
    G.write_bin_csr(str(path), rp, col, n)
    env = dict(os.environ, BTC_REORDER=reorder)
    out = subprocess.run([app, "-i", str(path), "-w", "1", "-r", "3", "-v", "1"], capture_output=True,
                         text=True, timeout=300, env=env)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    want = load_golden()[case]["count"]
    gpu = [int(x) for x in re.findall(r"Triangles \(GPU\): (\d+)", out.stdout)]
    cpu = [int(x) for x in re.findall(r"Triangles \(CPU\): (\d+)", out.stdout)]
    assert gpu and all(c == want for c in gpu), out.stdout[-2000:]
    if name == "btc_tc_adaptive_16x128":  # the app with the reference's -v CPU check
        assert cpu and all(c == want for c in cpu), out.stdout[-2000:]
