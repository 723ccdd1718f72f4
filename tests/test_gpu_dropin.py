"""The drop-in surface, run end to end: the MBE_GPU command line and a caller
written against include/mbe_finder.h the way the reference's own main is
written (src/main.cu:126-148: CSRBiGraph::Read, new IterFinderGpu6(graph,
bound_height, bound_size), Execute, PrintResult).

Both read an .adj file of the small configuration (2k x 3k Chung-Lu, seed 1)
and must report the oracle's count (pinned against the reference's own CPU
enumerators in tests/golden/golden.json) in the reference's output line
"maximal nodes:<n>", with the set hash beside it.  The caller is compiled by
g++ in the CPU suite too, so a header that no longer compiles fails without
a GPU.
"""
import json
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "gmbe_b200", "MBE_GPU")
LIBDIR = os.path.join(ROOT, "gmbe_b200")

# A caller shaped like the reference's src/main.cu:18-23 (FinderTest) and
# 126-148 (read the graph, construct the finder with its bounds, run it).
CALLER = r"""
#include <cstdio>
#include <cstdlib>
#include "mbe_finder.h"

static void FinderTest(BicliqueFinder* finder) {
  finder->Execute();
  finder->PrintResult();
}

int main(int argc, char** argv) {
  Option opt;
  opt.uvtrans = atoi(argv[2]);
  opt.order = atoi(argv[3]);
  opt.fast_mode = 1;
  CSRBiGraph* graph = new CSRBiGraph();
  if (graph->Read(argv[1], opt) != MBE_OK) return 1;
  IterFinderGpu6* finder = new IterFinderGpu6(graph, atoi(argv[4]), atoi(argv[5]));
  FinderTest(finder);
  if (finder->status() != MBE_OK) {
    fprintf(stderr, "%s\n", finder->last_error().c_str());
    return 1;
  }
  printf("caller count %llu hash 0x%016llx\n", finder->maximal_nodes(),
         (unsigned long long)finder->result().set_hash);
  delete finder;
  graph->Reset();
  delete graph;
  return 0;
}
"""


def _golden(name):
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        for c in json.load(f)["cases"]:
            if c["name"] == name:
                return c["oracle_count"], int(c["oracle_set_hash"], 16)
    raise KeyError(name)


@pytest.fixture(scope="module")
def gm():
    import gmbe_b200
    return gmbe_b200


@pytest.fixture(scope="module")
def small_adj(tmp_path_factory, gm):
    path = tmp_path_factory.mktemp("dropin") / "small.adj"
    gm.write_adj(str(path), gm.config_graph("small"))
    return str(path)


@pytest.fixture(scope="module")
def caller(tmp_path_factory):
    d = tmp_path_factory.mktemp("caller")
    src, exe = d / "caller.cpp", d / "caller"
    src.write_text(CALLER)
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-o",
                    str(exe), str(src), "-L", LIBDIR, "-lgmbe", f"-Wl,-rpath,{LIBDIR}"],
                   check=True)
    return str(exe)


def _maximal_nodes(out):
    m = re.search(r"^maximal nodes:(\d+)$", out, re.M)
    assert m, out
    return int(m.group(1))


def test_caller_compiles_against_the_finder_header(caller):
    assert os.access(caller, os.X_OK)


@pytest.mark.gpu
@pytest.mark.last
@pytest.mark.parametrize("args", [["-s", "2"], ["-s", "2", "-m", "5", "-n", "100"],
                                  ["-s", "0"], ["-s", "2", "-p"]])
def test_cli_reports_the_oracle_count(small_adj, args):
    count, h = _golden("config_small")
    p = subprocess.run([CLI, "-i", small_adj, "-t", "1", "-o", "1", "-f"] + args,
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    assert _maximal_nodes(p.stdout) == count
    assert re.search(r"^set hash: 0x([0-9a-f]{16})$", p.stdout, re.M).group(1) == f"{h:016x}"
    assert re.search(r"^Total processing time: [0-9.]+ seconds$", p.stdout, re.M)
    if "-p" in args:
        assert len(re.findall(r"^SM exit: [0-9.]+$", p.stdout, re.M)) == 2


def test_cli_reports_a_missing_file(tmp_path):
    # The file is read before any device call: no GPU needed.
    p = subprocess.run([CLI, "-i", str(tmp_path / "none.adj"), "-s", "2"], capture_output=True,
                       text=True, timeout=120)
    assert p.returncode != 0


@pytest.mark.gpu
@pytest.mark.last
@pytest.mark.parametrize("flags", [("1", "1", "20", "1500"), ("0", "1", "20", "1500"),
                                   ("1", "2", "8", "64")])
def test_reference_style_caller(caller, small_adj, flags):
    count, h = _golden("config_small")
    p = subprocess.run([caller, small_adj, *flags], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    assert _maximal_nodes(p.stdout) == count
    m = re.search(r"^caller count (\d+) hash 0x([0-9a-f]{16})$", p.stdout, re.M)
    assert (int(m.group(1)), int(m.group(2), 16)) == (count, h)
