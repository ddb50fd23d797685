"""BSR files read straight into device memory (jxcpr_bsr_read_device): the arrays equal the host
readers' (jxf_BSRMatrixRead / _Binary) bit for bit for 1- and 0-based files, row- and column-major
blocks, 2x2 and 3x3, the writer's own %.17e text format included; malformed files return an error
status; a solver set up from the device arrays solves exactly as from host arrays."""
import ctypes

import numpy as np
import pytest

from jxpamg_all_b200 import lib
from jxpamg_all_b200.solver import CprGmres
from tests.dropin_util import BSRMatrix, write_bsr_binary, write_bsr_text

pytestmark = pytest.mark.gpu
P = ctypes.c_void_p


def so():
    s = lib.load()
    s.jxcpr_bsr_read_device.argtypes = [ctypes.c_char_p, ctypes.c_int, P, P, P, P, P, P, P, P]
    s.jxcpr_bsr_free_device.argtypes = [P, P, P]
    s.jxf_BSRMatrixRead.restype = ctypes.POINTER(BSRMatrix)
    s.jxf_BSRMatrixRead.argtypes = [ctypes.c_char_p]
    s.jxf_BSRMatrixRead_Binary.restype = ctypes.POINTER(BSRMatrix)
    s.jxf_BSRMatrixRead_Binary.argtypes = [ctypes.c_char_p]
    s.jxf_BSRMatrixPrint.argtypes = [ctypes.POINTER(BSRMatrix), ctypes.c_char_p]
    s.jxf_BSRMatrixDestroy.argtypes = [ctypes.POINTER(BSRMatrix)]
    return s


def cudart():
    lib.load()  # the library brings the CUDA runtime into the process
    rt = ctypes.CDLL("libcudart.so.12")
    rt.cudaMemcpy.argtypes = [P, P, ctypes.c_size_t, ctypes.c_int]
    return rt


def to_host(ptr, n, dtype):
    out = np.zeros(n, dtype)
    if n:
        assert cudart().cudaMemcpy(out.ctypes.data, ptr, out.nbytes, 2) == 0  # device to host
    return out


def read_device(path, binary):
    s = so()
    rows, cols, bs = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    nnzb = ctypes.c_longlong()
    ia, ja, a = P(), P(), P()
    st = s.jxcpr_bsr_read_device(str(path).encode(), binary, ctypes.byref(rows), ctypes.byref(cols),
                                 ctypes.byref(bs), ctypes.byref(nnzb), ctypes.byref(ia), ctypes.byref(ja),
                                 ctypes.byref(a), None)
    return st, dict(rows=rows.value, cols=cols.value, bs=bs.value, nnzb=nnzb.value, ia=ia, ja=ja, a=a)


def host_arrays(d):
    bn = d["bs"] * d["bs"]
    return (to_host(d["ia"], d["rows"] + 1, np.int32), to_host(d["ja"], d["nnzb"], np.int32),
            to_host(d["a"], d["nnzb"] * bn, np.float64))


def free(d):
    so().jxcpr_bsr_free_device(d["ia"], d["ja"], d["a"])


def host_reader(path, binary):
    s = so()
    M = (s.jxf_BSRMatrixRead_Binary if binary else s.jxf_BSRMatrixRead)(str(path).encode())
    A = M.contents
    bn = A.block_size * A.block_size
    out = (np.ctypeslib.as_array(A.i, (A.num_rows + 1,)).copy(), np.ctypeslib.as_array(A.j, (A.num_nonzeros,)).copy(),
           np.ctypeslib.as_array(A.data, (A.num_nonzeros * bn,)).copy())
    s.jxf_BSRMatrixDestroy(M)
    return out


@pytest.mark.parametrize("name", ["tiny", "small", "tiny3", "c0"])
@pytest.mark.parametrize("one_based", [True, False])
@pytest.mark.parametrize("column_major", [False, True])
@pytest.mark.parametrize("binary", [0, 1])
def test_device_reader_equals_host_reader(tmp_path, systems, name, one_based, column_major, binary):
    s = systems(name)
    p = tmp_path / ("A.bin" if binary else "A.txt")
    (write_bsr_binary if binary else write_bsr_text)(str(p), s, one_based=one_based, column_major=column_major)
    st, d = read_device(p, binary)
    assert st == 0, lib.load().jxcpr_last_error()
    assert (d["rows"], d["cols"], d["bs"], d["nnzb"]) == (s.num_block_rows, s.num_block_rows, s.block_size, s.nnzb)
    ia, ja, a = host_arrays(d)
    free(d)
    hia, hja, ha = host_reader(p, binary)
    assert np.array_equal(ia, hia) and np.array_equal(ja, hja)
    assert np.array_equal(a.view(np.int64), ha.view(np.int64))  # bit for bit
    assert np.array_equal(ia, s.ia) and np.array_equal(ja, s.ja) and np.array_equal(a, s.a)


def test_writer_format_and_wide_value_range(tmp_path, systems):
    """The library's own writer prints %.17e (18 significant digits); values spread over the whole
    FP64 range, subnormals and signed zeros included, come back bit for bit."""
    s = systems("small")
    rng = np.random.default_rng(5)
    vals = s.a.copy()
    vals[: len(vals) // 2] = rng.standard_normal(len(vals) // 2) * 10.0 ** rng.integers(-307, 307, len(vals) // 2)
    vals[:40] = rng.integers(1, 2 ** 52, 40, dtype=np.int64).view(np.float64)  # subnormal
    vals[40:44] = [0.0, -0.0, np.finfo(np.float64).max, -np.finfo(np.float64).tiny]
    p0 = tmp_path / "in.txt"
    from types import SimpleNamespace

    t = SimpleNamespace(block_size=s.block_size, num_block_rows=s.num_block_rows, nnzb=s.nnzb, ia=s.ia, ja=s.ja,
                        a=vals)
    write_bsr_text(str(p0), t)
    s_ = so()
    M = s_.jxf_BSRMatrixRead(str(p0).encode())
    p = tmp_path / "out.txt"
    assert s_.jxf_BSRMatrixPrint(M, str(p).encode()) == 0  # %.17e
    s_.jxf_BSRMatrixDestroy(M)
    st, d = read_device(p, 0)
    assert st == 0, lib.load().jxcpr_last_error()
    _, _, a = host_arrays(d)
    free(d)
    assert np.array_equal(a.view(np.int64), vals.view(np.int64))


def test_tokens_left_to_strtod(tmp_path):
    """Values the device does not convert (more than 19 significant digits, inf) are converted on the
    host with strtod."""
    p = tmp_path / "wide.txt"
    p.write_text("1 1 1\n1\n0\n2\n1\n2\n1\n1\n1\n0.123456789012345678901234567890e2\n")
    st, d = read_device(p, 0)
    assert st == 0, lib.load().jxcpr_last_error()
    _, _, a = host_arrays(d)
    free(d)
    assert a[0] == float("0.123456789012345678901234567890e2")


@pytest.mark.parametrize("text", [
    "3 3 2\n2\n0\n4\n1 2 3\n",                              # too few numbers
    "1 3 1\n1\n0\n2\n1 2\n1\n1\n1\n5.0\n",                  # largest column 0, 3 columns declared
    "1 1 1\n1\n0\n2\n1 2\n1\n1\n1\n5.0x\n",                 # malformed value
    "1 1 1\n1\n0\n3\n1 2\n1\n1\n1\n5.0\n",                  # row-pointer length disagrees
    "x 1 1\n",                                              # malformed header
])
def test_malformed_files_report_errors(tmp_path, text):
    p = tmp_path / "bad.txt"
    p.write_text(text)
    st, _ = read_device(p, 0)
    assert st == 4
    assert b"bsr read" in lib.load().jxcpr_last_error()
    st, _ = read_device(tmp_path / "missing.txt", 0)
    assert st == 4


def test_solver_from_device_arrays(tmp_path, systems):
    s = systems("c0")
    p = tmp_path / "c0.bin"
    write_bsr_binary(str(p), s)
    st, d = read_device(p, 1)
    assert st == 0
    G = CprGmres(decouple=1)
    G.setup(d["ia"].value, d["ja"].value, d["a"].value, d["bs"], nb=d["rows"], nnzb=d["nnzb"], device=True)
    x, it, rel, conv = G.solve(s.b)
    G.close()
    free(d)
    H = CprGmres(decouple=1).setup(s.ia, s.ja, s.a, s.block_size)
    xh, ith, relh, convh = H.solve(s.b)
    H.close()
    assert conv and it == ith and np.array_equal(x, xh)
