"""On-disk formats of the reference through the C ABI (host code, no GPU):
example_cpp binary CSR (Cpp_EMIN/readMat.cpp) and Chronos .Ext_bin
(DumpChronos.cpp), against independent Python writers/parsers of the same
layouts and the reference's own example file when it is present."""
import os
import struct

import numpy as np
import pytest
import scipy.sparse as sp

import chronoslab_b200 as cb
from chronoslab_b200._lib import ChronosError
from oracle import amg_oracle as O

from oracle.refdir import reference_file

REF_BIN = reference_file("sources", "Preconditioner", "AMG", "prolong", "EMIN", "example_cpp",
                         "matrix.bin")


def random_matrix(n, seed, density=0.05):
    A = sp.random(n, n, density=density, random_state=seed, format="csr")
    A = (A + sp.eye(n)).tocsr()
    A.sort_indices()
    return A


def write_matrix_bin_py(path, A):
    """Header {int32 rows, int32 entries}, records {int32 i, int32 j, f64 a}, 1-based."""
    C = A.tocoo()
    order = np.lexsort((C.col, C.row))
    with open(path, "wb") as f:
        f.write(struct.pack("<ii", A.shape[0], C.nnz))
        for k in order:
            f.write(struct.pack("<iid", int(C.row[k]) + 1, int(C.col[k]) + 1, float(C.data[k])))


def parse_ext_bin_py(path):
    with open(path, "rb") as f:
        nr, nt = struct.unpack("<qq", f.read(16))
        rec = np.frombuffer(f.read(24 * nt),
                            dtype=np.dtype([("i", "<i8"), ("j", "<i8"), ("a", "<f8")]))
    return sp.csr_matrix((rec["a"], (rec["i"] - 1, rec["j"] - 1)), shape=(nr, nr))


def test_matrix_bin_roundtrip(lib, tmp_path):
    A = random_matrix(300, 1)
    p = tmp_path / "m.bin"
    write_matrix_bin_py(p, A)
    B = cb.read_matrix_bin(str(p))
    assert B.shape == A.shape
    assert np.array_equal(B.indptr, A.indptr) and np.array_equal(B.indices, A.indices)
    assert np.array_equal(B.data, A.data)


def test_ext_bin_roundtrip(lib, tmp_path):
    A = random_matrix(257, 2)
    p = tmp_path / "ChronosMatrix.Ext_bin"
    cb.write_ext_bin(str(p), A)
    assert os.path.getsize(p) == 16 + 24 * A.nnz
    assert (parse_ext_bin_py(p) != A).nnz == 0
    B = cb.read_ext_bin(str(p))
    assert np.array_equal(B.indptr, A.indptr) and np.array_equal(B.indices, A.indices)
    assert np.array_equal(B.data, A.data)


def test_tv_ext_bin(lib, tmp_path):
    TV = np.random.default_rng(3).standard_normal((123, 6))
    p = tmp_path / "ChronosTV0.Ext_bin"
    cb.write_tv_ext_bin(str(p), TV)
    with open(p, "rb") as f:
        nr, nc = struct.unpack("<qq", f.read(16))
        vals = np.frombuffer(f.read(), dtype="<f8")
    assert (nr, nc) == TV.shape and np.array_equal(vals, TV.ravel())   # row by row
    assert np.array_equal(cb.read_tv_ext_bin(str(p)), TV)
    # the reference dumper's test-space files end after the header
    q = tmp_path / "header_only.Ext_bin"
    q.write_bytes(struct.pack("<qq", 123, 6))
    assert cb.read_tv_ext_bin(str(q)).shape == (123, 0)


def test_format_errors(lib, tmp_path):
    A = random_matrix(50, 4)
    p = tmp_path / "m.bin"
    write_matrix_bin_py(p, A)
    data = p.read_bytes()
    (tmp_path / "short.bin").write_bytes(data[:-10])
    with pytest.raises(ChronosError) as e:
        cb.read_matrix_bin(str(tmp_path / "short.bin"))
    assert e.value.code == -6
    with pytest.raises(ChronosError):
        cb.read_ext_bin(str(tmp_path / "missing.Ext_bin"))
    bad = tmp_path / "bad.Ext_bin"
    bad.write_bytes(struct.pack("<qq", 10, 1) + struct.pack("<qqd", 11, 1, 1.0))
    with pytest.raises(ChronosError):
        cb.read_ext_bin(str(bad))


@pytest.mark.skipif(REF_BIN is None, reason="reference example file not present")
def test_reads_reference_example_matrix(lib):
    """The reference's own example_cpp/matrix.bin (Cubo level 1) read through
    the C ABI equals the oracle's restatement of readBinaryMatrix."""
    B = cb.read_matrix_bin(REF_BIN)
    R = O.read_bin_matrix(REF_BIN).tocsr()
    R.sum_duplicates()
    R.sort_indices()
    assert B.shape == R.shape and B.nnz == R.nnz
    assert np.array_equal(B.indptr, R.indptr) and np.array_equal(B.indices, R.indices)
    assert np.array_equal(B.data, R.data)
