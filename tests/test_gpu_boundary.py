"""The C ABI's stream, operator and layout arguments (include/chronos_b200.h).

* Solve calls order their device work on the caller's stream: two handles
  solved from two host threads on two torch streams at once give the same
  bits as one after the other, and work the caller queues on its stream
  before and after a call is ordered with the call's work with no host
  synchronisation in between.
* chronos_pcg takes PCG_CJ's operator prodA (PCG_CJ.m:1) as a CSR, as the
  reference passes @(x)A*x separately from the preconditioner
  (aspAMG_main.m:199-202).
* chronos_fsai_numeric takes 0- or 1-based CSR and returns FP64 or FP32 values.
* chronos_amg_setup takes A in host or device memory.
"""
import threading

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import rowwise_close
import chronoslab_b200 as cb
from chronoslab_b200 import problems as PB
from oracle import amg_oracle as O

pytestmark = pytest.mark.gpu


def _problems():
    A1 = PB.poisson7(24)
    A2, X = PB.elasticity_q1(12, return_coords=True)
    return [(A1, np.ones((A1.shape[0], 1)), PB.uniform_rhs(A1.shape[0], seed=3), 1),
            (A2, PB.rbm_test_space(X), PB.elasticity_rhs(A2, X, seed=4), 6)]


def test_two_handles_on_two_streams_concurrently(lib):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    probs = _problems()
    hs = [cb.Hierarchy(A, TV, cb.params(precision=cb.CHRONOS_FP32, ntv=ntv))
          for A, TV, _, ntv in probs]
    try:
        bs = [torch.from_numpy(b).to(dev) for _, _, b, _ in probs]
        # sequential reference results (this also builds each handle's graph)
        seq = []
        for h, b in zip(hs, bs):
            x = torch.zeros_like(b)
            it, flag, _ = h.pcg_dev(b.data_ptr(), x.data_ptr())
            torch.cuda.synchronize()
            seq.append((x.cpu().numpy(), it, flag))
        streams = [torch.cuda.Stream(device=dev) for _ in hs]
        for rep in range(3):
            xs = [torch.zeros_like(b) for b in bs]
            torch.cuda.synchronize()
            out = [None] * len(hs)

            def run(k):
                out[k] = hs[k].pcg_dev(bs[k].data_ptr(), xs[k].data_ptr(), stream=streams[k])

            ths = [threading.Thread(target=run, args=(k,)) for k in range(len(hs))]
            for t in ths:
                t.start()
            for t in ths:
                t.join()
            for k, s in enumerate(streams):
                with torch.cuda.stream(s):
                    got = xs[k].cpu().numpy()          # queued after the solve on s
                assert out[k][0] == seq[k][1] and out[k][1] == seq[k][2] == 0
                assert np.array_equal(got, seq[k][0]), (rep, k)
    finally:
        for h in hs:
            h.close()


def test_work_is_ordered_on_the_callers_stream(lib):
    """b is produced and x consumed by kernels queued on the caller's stream
    around the call, with no host synchronisation in between; a long kernel
    queued first makes a missing wait show as a wrong solution."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    A, TV, b_np, ntv = _problems()[1]
    with cb.Hierarchy(A, TV, cb.params(precision=cb.CHRONOS_FP64, ntv=ntv)) as h:
        x_ref, it_ref, _, _, _ = h.pcg(b_np)
        s = torch.cuda.Stream(device=dev)
        b_host = torch.from_numpy(b_np).pin_memory()
        big = torch.empty(64 << 20, dtype=torch.float32, device=dev)
        torch.cuda.synchronize()
        with torch.cuda.stream(s):
            for _ in range(20):                  # a few ms of work queued ahead of b
                big.mul_(1.0000001)
            b = torch.empty(b_np.size, dtype=torch.float64, device=dev)
            b.copy_(b_host, non_blocking=True)
            x = torch.zeros_like(b)
        it, flag, _ = h.pcg_dev(b.data_ptr(), x.data_ptr(), stream=s)
        with torch.cuda.stream(s):
            y = x * 2.0                          # consumer queued on the same stream
        torch.cuda.synchronize()
        assert it == it_ref and flag == 0
        assert np.array_equal(y.cpu().numpy(), 2.0 * x_ref)
        # the host-buffer entry points take the stream too
        xv = h.vcycle(b_np, stream=s)
        assert np.array_equal(xv, h.vcycle(b_np))
        xp, itp, _, flp, _ = h.pcg(b_np, stream=s)
        assert itp == it_ref and np.array_equal(xp, x_ref)
        X, its, fls, _ = h.pcg_block(np.stack([b_np, -b_np], axis=1), stream=s)
        assert list(fls) == [0, 0]


def test_pcg_operator_argument(lib, cubo):
    """PCG_CJ with prodA given: the operator itself gives the same solve as
    the hierarchy's own; the unmodified Cubo operator with the preconditioner
    of the Dirichlet-fixed one (as the reference's tests pair them) matches
    the oracle's PCG_CJ on the GPU's levels within one iteration; a scaled
    operator 2A leaves the iterates' count unchanged and halves x."""
    A0, Af = cubo["A"], cubo["Af"]
    n = Af.shape[0]
    b = PB.uniform_rhs(n, seed=7)
    with cb.Hierarchy(Af, cubo["TV0"], cb.params(precision=cb.CHRONOS_FP64)) as h:
        x1, it1, rv1, f1, _ = h.pcg(b, tol=1e-8)
        x2, it2, rv2, f2, _ = h.pcg(b, tol=1e-8, A=Af)
        assert (it1, f1) == (it2, f2) and np.allclose(x1, x2, rtol=0, atol=1e-12 * abs(x1).max())
        x3, it3, _, f3, _ = h.pcg(b, tol=1e-8, A=2.0 * Af)
        assert f3 == 0 and abs(it3 - it1) <= 1
        assert np.linalg.norm(2.0 * x3 - x1) <= 1e-7 * np.linalg.norm(x1)
        x4, it4, _, f4, _ = h.pcg(b, tol=1e-8, A=A0)
        parts = []
        for l in range(h.nlevels):
            p = {"A": h.export(l, "A")}
            if l < h.nlevels - 1:
                p.update(G=h.export(l, "G"), P=h.export(l, "P"), omega=h.level_info(l)["omega"])
            parts.append(p)
        Ho = O.hierarchy_from_parts(parts)
        xo, ito, _, flo = O.pcg_cj(lambda r: O.amg_vcycle(Ho, r), lambda v: A0 @ v, b,
                                   np.zeros(n), 1000, 1e-8)
        assert f4 == flo and abs(it4 - ito) <= 1
        assert np.linalg.norm(b - A0 @ x4) <= 1e-8 * np.linalg.norm(b) * 1.01
        # after a call with an operator the hierarchy's own operator is back
        x5, it5, _, _, _ = h.pcg(b, tol=1e-8)
        assert it5 == it1 and np.array_equal(x5, x1)
        with pytest.raises(cb.ChronosError):
            h.pcg(b, A=sp.identity(n - 1, format="csr"))


@pytest.mark.parametrize("base", [0, 1])
def test_fsai_numeric_base_and_fp32_output(lib, cubo, cubo_ref, base):
    A, G = cubo["Af"], cubo_ref["G"]
    v64, ok = cb.fsai_numeric(A, G, base=base)
    assert ok
    ref = sp.csr_matrix((cubo_ref["G"].data, G.indices, G.indptr), shape=G.shape)
    assert rowwise_close(sp.csr_matrix((v64, G.indices, G.indptr), shape=G.shape), ref, 1e-10)
    v32, ok32 = cb.fsai_numeric(A, G, base=base, precision=cb.CHRONOS_FP32)
    assert ok32 and v32.dtype == np.float32
    assert np.array_equal(v32, v64.astype(np.float32))


def test_setup_from_device_memory(lib):
    """The same hierarchy from A and TV0 in device memory as from host memory:
    level sizes, operators and the solve bit for bit."""
    torch = pytest.importorskip("torch")
    import ctypes as C
    from chronoslab_b200._lib import check
    dev = torch.device("cuda", 0)
    A, X = PB.elasticity_q1(10, return_coords=True)
    TV = PB.rbm_test_space(X)
    b = PB.elasticity_rhs(A, X, seed=0)
    prm = cb.params(precision=cb.CHRONOS_FP32)
    A = sp.csr_matrix(A)
    A.sort_indices()
    ip = torch.from_numpy(A.indptr.astype(np.int32)).to(dev)
    ix = torch.from_numpy(A.indices.astype(np.int32)).to(dev)
    dv = torch.from_numpy(np.ascontiguousarray(A.data, dtype=np.float64)).to(dev)
    tv = torch.from_numpy(np.ascontiguousarray(TV.T).ravel()).to(dev)
    torch.cuda.synchronize()
    lib_ = cb._lib.load()
    hd = C.c_void_p()
    check(lib_.chronos_amg_setup(C.byref(prm), A.shape[0], C.cast(ip.data_ptr(), C.POINTER(C.c_int)),
                                 C.cast(ix.data_ptr(), C.POINTER(C.c_int)),
                                 C.cast(dv.data_ptr(), C.POINTER(C.c_double)), TV.shape[1],
                                 C.cast(tv.data_ptr(), C.POINTER(C.c_double)), C.byref(hd)))
    dev_h = cb.Hierarchy.__new__(cb.Hierarchy)
    dev_h._lib, dev_h._h, dev_h.n, dev_h.prm = lib_, hd, A.shape[0], prm
    with dev_h, cb.Hierarchy(A, TV, prm) as host_h:
        assert dev_h.nlevels == host_h.nlevels
        for l in range(host_h.nlevels):
            Ad, Ah = dev_h.export(l, "A"), host_h.export(l, "A")
            assert (Ad != Ah).nnz == 0
        xd, itd, _, _, _ = dev_h.pcg(b)
        xh, ith, _, _, _ = host_h.pcg(b)
        assert itd == ith and np.array_equal(xd, xh)


def test_vcycle_on_device_vectors_fp64_and_fp32(lib):
    """chronos_vcycle_dev: FP64 device vectors give chronos_vcycle's result
    bit for bit; FP32 vectors on an FP32 hierarchy (read and written
    directly) agree with the FP64-vector V-cycle to 2e-5; on an FP64
    hierarchy FP32 vectors give the FP64 cycle of the same input rounded once
    to FP32.  Two columns at once."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    A, TV, b_np, ntv = _problems()[1]
    B = np.stack([b_np, np.roll(b_np, 7)], axis=1)
    for prec in (cb.CHRONOS_FP32, cb.CHRONOS_FP64):
        with cb.Hierarchy(A, TV, cb.params(precision=prec, ntv=ntv)) as h:
            ref = h.vcycle(B)
            bd = torch.from_numpy(np.ascontiguousarray(B.T)).to(dev)
            xd = torch.zeros_like(bd)
            h.vcycle_dev(bd.data_ptr(), xd.data_ptr(), cb.CHRONOS_FP64, nrhs=2)
            torch.cuda.synchronize()
            assert np.array_equal(xd.cpu().numpy().T, ref)
            b32 = bd.to(torch.float32)
            x32 = torch.zeros_like(b32)
            h.vcycle_dev(b32.data_ptr(), x32.data_ptr(), cb.CHRONOS_FP32, nrhs=2)
            torch.cuda.synchronize()
            got = x32.cpu().numpy().T.astype(np.float64)
            if prec == cb.CHRONOS_FP32:
                for j in range(2):
                    assert np.linalg.norm(got[:, j] - ref[:, j]) <= 2e-5 * np.linalg.norm(ref[:, j])
            else:
                want = h.vcycle(b32.cpu().numpy().T.astype(np.float64)).astype(np.float32)
                assert np.array_equal(x32.cpu().numpy().T, want)
            with pytest.raises(cb.ChronosError):
                h.vcycle_dev(bd.data_ptr(), xd.data_ptr(), 7)

