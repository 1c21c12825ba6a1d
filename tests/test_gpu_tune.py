"""The autotuner's decision cache: one entry per matrix signature including
the longest row, so the FSAI factor G and its transpose (same rows, entries
and columns) are timed and stored apart; lines of another format in the
cache file are ignored.  The cache is read once per process, so each case
runs in a child process with its own cache file."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build_in_child(cache, precision):
    code = (
        "import sys\n"
        f"sys.path.insert(0, {ROOT!r})\n"
        "import chronoslab_b200 as cb\n"
        "from chronoslab_b200 import problems as PB\n"
        "A, X = PB.elasticity_q1(16, return_coords=True)\n"
        f"with cb.Hierarchy(A, PB.rbm_test_space(X), cb.params(precision={precision})) as h:\n"
        "    print(h.level_info(0)['nnz_G'], h.level_info(0)['n'])\n")
    env = dict(os.environ, CHRONOS_TUNE_CACHE=str(cache))
    out = subprocess.run([sys.executable, "-c", code], env=env, check=True, timeout=900,
                         capture_output=True, text=True)
    nnz_g, n = map(int, out.stdout.split()[-2:])
    return nnz_g, n


def _entries(cache):
    rows = []
    for line in cache.read_text().splitlines():
        f = line.split()
        if f and f[0] == "v2" and len(f) == 8:
            rows.append((f[1], int(f[2]), int(f[3]), int(f[4]), int(f[5]), int(f[6]), int(f[7])))
    return rows


def test_g_and_its_transpose_are_tuned_apart(lib, tmp_path):
    cache = tmp_path / "tune.txt"
    cache.write_text("h 1000 5000 1000 1 8\nnot a cache line\n")    # another format: ignored
    nnz_g, n = _build_in_child(cache, 1)
    ent = _entries(cache)
    g_like = [e for e in ent if e[1] == n and e[2] == nnz_g and e[3] == n and e[4] == 1]
    assert len(g_like) == 2                           # G and G' of level 1
    assert g_like[0][5] != g_like[1][5]               # different longest rows
    # a second process finds both decisions and adds none
    before = len(ent)
    _build_in_child(cache, 1)
    assert len(_entries(cache)) == before
