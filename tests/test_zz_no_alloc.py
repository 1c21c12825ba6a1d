"""chronos_fsai_numeric_noalloc: the FSAI numeric phase for callers that cannot
let the library allocate device memory (their own memory pool owns the GPU, or
a cudaFree's device-wide synchronisation would stall their other streams).

The caller owns every buffer (here torch allocates them, outside the call);
the entry point keeps its scratch in a static device array.  Its values must
match the allocating entry point chronos_fsai_numeric, on two calls in a row
(the second call reuses the scratch the first one left behind).

Malformed patterns (an empty G row, a G row without its diagonal last) are
rejected on the device before any value is written: sentinels placed on both
sides of the output stay as they were.

This file is collected last so that a failure here leaves every other test run.
"""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import rowwise_close
import chronoslab_b200 as cb

pytestmark = pytest.mark.gpu


def _device_csr(torch, M, dev):
    return (torch.from_numpy(M.indptr.astype(np.int32)).to(dev),
            torch.from_numpy(M.indices.astype(np.int32)).to(dev),
            torch.from_numpy(np.ascontiguousarray(M.data, dtype=np.float64)).to(dev))


def test_fsai_numeric_noalloc_matches_allocating_entry(lib, cubo, cubo_ref):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    A = cubo["Af"]
    G = cubo_ref["G"]                    # reference pattern: strictly-lower ascending, diagonal last
    ref_vals, ref_ok = cb.fsai_numeric(A, G)
    assert ref_ok

    ap, ai, av = _device_csr(torch, A, dev)
    gp = torch.from_numpy(G.indptr.astype(np.int32)).to(dev)
    gi = torch.from_numpy(G.indices.astype(np.int32)).to(dev)
    stream = torch.cuda.Stream(device=dev)
    held = cb.device_bytes()
    for call in range(2):
        out = torch.full((G.nnz,), float("nan"), dtype=torch.float64, device=dev)
        ok = ctypes.c_int(-1)
        torch.cuda.synchronize()
        code = lib.chronos_fsai_numeric_noalloc(
            A.shape[0], ctypes.c_void_p(ap.data_ptr()), ctypes.c_void_p(ai.data_ptr()),
            ctypes.c_void_p(av.data_ptr()), ctypes.c_void_p(gp.data_ptr()),
            ctypes.c_void_p(gi.data_ptr()), ctypes.c_void_p(out.data_ptr()), ctypes.byref(ok),
            ctypes.c_void_p(stream.cuda_stream))
        assert code == 0, cb.last_error() if hasattr(cb, "last_error") else code
        assert ok.value == 1, f"call {call}"
        vals = out.cpu().numpy()
        got = sp.csr_matrix((vals, G.indices, G.indptr), shape=G.shape)
        want = sp.csr_matrix((ref_vals, G.indices, G.indptr), shape=G.shape)
        assert rowwise_close(got, want, 1e-10), f"call {call}"
    # the library's own device memory is what it was before the two calls
    assert cb.device_bytes() == held


def _call_noalloc(lib, torch, dev, n, ap, ai, av, gp_np, gi_np, out, pad):
    gp = torch.from_numpy(np.ascontiguousarray(gp_np, dtype=np.int32)).to(dev)
    gi = torch.from_numpy(np.ascontiguousarray(gi_np, dtype=np.int32)).to(dev)
    ok = ctypes.c_int(-1)
    torch.cuda.synchronize()
    code = lib.chronos_fsai_numeric_noalloc(
        n, ctypes.c_void_p(ap.data_ptr()), ctypes.c_void_p(ai.data_ptr()),
        ctypes.c_void_p(av.data_ptr()), ctypes.c_void_p(gp.data_ptr()),
        ctypes.c_void_p(gi.data_ptr()), ctypes.c_void_p(out.data_ptr() + pad * 8),
        ctypes.byref(ok), None)
    torch.cuda.synchronize()
    return code


def _drop_entries(G, drop):
    """G's pattern without the entries whose positions are in `drop`."""
    keep = np.ones(G.nnz, dtype=bool)
    keep[list(drop)] = False
    rows = np.repeat(np.arange(G.shape[0]), np.diff(G.indptr))[keep]
    indptr = np.zeros(G.shape[0] + 1, dtype=np.int64)
    np.add.at(indptr, rows + 1, 1)
    return np.cumsum(indptr), G.indices[keep]


@pytest.mark.parametrize("case", ["empty_row0", "empty_row", "no_diagonal"])
def test_fsai_numeric_noalloc_rejects_malformed_pattern(lib, cubo, cubo_ref, case):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    A = cubo["Af"]
    G = cubo_ref["G"]
    n = A.shape[0]
    r = 0 if case == "empty_row0" else n // 2
    lo, hi = int(G.indptr[r]), int(G.indptr[r + 1])
    drop = range(lo, hi) if case.startswith("empty") else [hi - 1]
    gp, gi = _drop_entries(G, drop)
    assert gp[-1] == gi.size
    ap, ai, av = _device_csr(torch, A, dev)
    pad = 64
    out = torch.full((gi.size + 2 * pad,), 7.25, dtype=torch.float64, device=dev)
    code = _call_noalloc(lib, torch, dev, n, ap, ai, av, gp, gi, out, pad)
    assert code == -1, (case, code)
    assert bool(torch.all(out == 7.25)), "a value was written for a rejected pattern"
    # the same buffers with the intact pattern still work afterwards
    out = torch.full((G.nnz + 2 * pad,), 7.25, dtype=torch.float64, device=dev)
    code = _call_noalloc(lib, torch, dev, n, ap, ai, av, G.indptr, G.indices, out, pad)
    assert code == 0
    o = out.cpu().numpy()
    assert np.all(o[:pad] == 7.25) and np.all(o[pad + G.nnz:] == 7.25)
    assert np.all(np.isfinite(o[pad:pad + G.nnz]))


def test_fsai_numeric_noalloc_rejects_oversize(lib):
    ok = ctypes.c_int(-1)
    code = lib.chronos_fsai_numeric_noalloc((1 << 20) + 1, ctypes.c_void_p(8), ctypes.c_void_p(8),
                                            ctypes.c_void_p(8), ctypes.c_void_p(8),
                                            ctypes.c_void_p(8), ctypes.c_void_p(8),
                                            ctypes.byref(ok), None)
    assert code == -1
