"""The C ABI library loads without a GPU and exports every declared symbol."""
import ctypes
import os
import re

import numpy as np
import pytest

import chronoslab_b200 as cb
from chronoslab_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:int|void|const char \*)\s*(chronos_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 30
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(_lib.SIGNATURES), "ctypes table out of sync with the header"


def test_params_struct_layout_matches(lib):
    p = cb.params()
    assert p.nLevMax == 10 and p.maxCoarseSZ == 1000 and p.nstep == 15 and p.step_size == 1
    assert p.epsilon == 1e-3 and p.SoC_type == b"DOM" and p.soc_tau == 0.01
    assert p.proltype == b"BAMG" and p.maxrownrm == 5.0 and p.eps_prol == 1e-10
    assert p.precision == cb.CHRONOS_FP32 and p.seed == 5489 and p.fsai_fabs == 0
    assert p.tol == 1e-8 and p.itmax == 15000


def test_last_error_and_status(lib):
    with pytest.raises(cb.ChronosError) as e:
        cb.readDefaultParams("/nonexistent/aspAMG.fnames")
    assert e.value.code == -6 and "cannot open" in str(e.value)


def test_bad_csr_rejected(lib):
    import scipy.sparse as sp
    A = sp.csr_matrix(np.eye(3))
    # columns out of order are rejected by the host validation, before any GPU use
    bad = sp.csr_matrix((np.ones(2), np.array([1, 0]), np.array([0, 2, 2, 2])), shape=(3, 3))
    bad.has_sorted_indices = True          # lie to skip scipy's sort
    ip = bad.indptr.astype(np.int32)
    ix = bad.indices.astype(np.int32)
    dv = bad.data.astype(np.float64)
    h = ctypes.c_void_p()
    ok = ctypes.c_int()
    code = lib.chronos_fsai_pattern(3, ip.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                    ix.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                    dv.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                    15, 1, 1e-3, 1, 0, ctypes.byref(ok), ctypes.byref(h))
    assert code == -1 and "increasing" in _lib.last_error()
    assert cb.version().startswith("chronos_b200")


def test_hierarchy_file_rejected_before_any_gpu_work(lib, tmp_path):
    """chronos_hier_load checks the file's header before touching the GPU: a
    file of another kind, a truncated one and a missing one are CHRONOS_EIO."""
    import chronoslab_b200 as cb
    bad = tmp_path / "not_a_hierarchy.bin"
    bad.write_bytes(b"0123456789abcdef" * 4)
    short = tmp_path / "truncated.bin"
    short.write_bytes(b"CHRNHIER\x01\x00")
    for p in (bad, short, tmp_path / "missing.bin"):
        with pytest.raises(cb.ChronosError) as e:
            cb.Hierarchy.load(str(p))
        assert e.value.code == -6


C_CALLER = r"""
#include "chronos_b200.h"
#include <stdio.h>
#include <string.h>

int main(int argc, char **argv) {
  chronos_params p;
  chronos_params_default(&p);
  if (p.nLevMax <= 0 || strcmp(p.smoother_method, "AFSAI_SYM") != 0) return 2;
  /* a status, not an exception, for a bad argument; the message is kept */
  if (chronos_amg_setup(&p, 0, 0, 0, 0, 0, 0, 0) != CHRONOS_EINVAL) return 3;
  char msg[256];
  chronos_last_error(msg, (int)sizeof msg);
  if (strlen(msg) == 0) return 4;
  chronos_hier *h = 0;
  if (chronos_hier_load(argv[argc - 1], &h) != CHRONOS_EIO || h) return 5;
  printf("ok %d %s\n", p.nLevMax, p.smoother_method);
  return 0;
}
"""


def test_header_is_c_and_library_links_from_c(lib, tmp_path):
    """include/chronos_b200.h compiles as C99 (-pedantic, warnings as
    errors) and a C caller links against the library and gets statuses and
    messages back without a GPU."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if not gcc:
        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "caller.c"
    src.write_text(C_CALLER)
    exe = tmp_path / "caller"
    libdir = os.path.join(root, "chronoslab_b200")
    subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror",
                    "-I", os.path.join(root, "include"), str(src), "-L", libdir,
                    "-lchronos_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    r = subprocess.run([str(exe), str(tmp_path / "missing.chh")], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert r.stdout.startswith("ok ")
