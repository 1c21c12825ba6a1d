"""Failures injected from the host (no GPU fault, trap or hang): a right-hand
side holding a NaN, and device allocations that fail mid-setup under a cap.
Each call returns its status and the library stays usable."""
import os
import subprocess
import sys

import numpy as np
import pytest

import chronoslab_b200 as cb
from chronoslab_b200 import problems as PB

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("prec", [cb.CHRONOS_FP32, cb.CHRONOS_FP64])
def test_nan_rhs_stops_with_flag_and_next_solve_is_clean(lib, prec):
    """PCG_CJ on a right-hand side with a NaN stops after its first step (the
    device-side loop ends on a non-finite p'r) and the call returns
    CHRONOS_EBREAKDOWN; the same handle then solves a clean right-hand side
    exactly as before."""
    A = PB.poisson7(14)
    n = A.shape[0]
    b = PB.uniform_rhs(n, seed=3)
    bad = b.copy()
    bad[n // 2] = np.nan
    with cb.Hierarchy(A, np.ones((n, 1)), cb.params(precision=prec)) as h:
        x0, it0, _, f0, _ = h.pcg(b, itmax=200, tol=1e-8)
        with pytest.raises(cb.ChronosError) as e:
            h.pcg(bad, itmax=200, tol=1e-8)
        assert e.value.code == -5                    # CHRONOS_EBREAKDOWN
        assert "iteration 1" in str(e.value) or "iteration 0" in str(e.value)
        x1, it1, _, f1, _ = h.pcg(b, itmax=200, tol=1e-8)
    assert f0 == f1 == 0 and it1 == it0
    assert np.array_equal(x1, x0)


def test_allocation_cap_reports_enomem_and_frees(lib, tmp_path):
    """Under CHRONOS_DEVICE_ALLOC_CAP (read once per process, so in a child
    process) a setup that needs more than the cap fails with CHRONOS_ENOMEM,
    leaves no device memory held, and a setup that fits then works."""
    out = tmp_path / "result.txt"
    code = (
        "import sys\n"
        f"sys.path.insert(0, {ROOT!r})\n"
        "import numpy as np\n"
        "import chronoslab_b200 as cb\n"
        "from chronoslab_b200 import problems as PB\n"
        "A, X = PB.elasticity_q1(36, return_coords=True)\n"
        "res = []\n"
        "try:\n"
        "    cb.Hierarchy(A, PB.rbm_test_space(X), cb.params(precision=cb.CHRONOS_FP32))\n"
        "    res.append('built')\n"
        "except cb.ChronosError as e:\n"
        "    res.append(str(e.code))\n"
        "res.append(str(cb.device_bytes()))\n"
        "A, X = PB.elasticity_q1(8, return_coords=True)\n"
        "b = PB.elasticity_rhs(A, X, seed=0)\n"
        "with cb.Hierarchy(A, PB.rbm_test_space(X), cb.params(precision=cb.CHRONOS_FP32)) as h:\n"
        "    x, it, _, flag, _ = h.pcg(b, itmax=300, tol=1e-8)\n"
        "    res.append(str(flag))\n"
        "    res.append(str(np.linalg.norm(b - A @ x) / np.linalg.norm(b) <= 1e-8))\n"
        "res.append(str(cb.device_bytes()))\n"
        f"open({str(out)!r}, 'w').write(' '.join(res))\n")
    env = dict(os.environ, CHRONOS_DEVICE_ALLOC_CAP=str(512 << 20),
               CHRONOS_TUNE_CACHE=str(tmp_path / "tune.txt"))
    subprocess.run([sys.executable, "-c", code], env=env, check=True, timeout=900)
    failed, held, flag, ok, held_after = out.read_text().split()
    assert failed == "-3"             # CHRONOS_ENOMEM
    assert held == "0" and held_after == "0"
    assert flag == "0" and ok == "True"
