"""The reference-named C interface on the CPU: the header compiles and links a
caller written against it, and the BSR readers / writers (host code) parse the
reference's text and binary formats."""
import ctypes
import os

import numpy as np

from jxpamg_all_b200 import lib
from tests.dropin_util import BSRMatrix, build_driver, write_bsr_binary, write_bsr_text


def _so():
    so = lib.load()
    so.jxf_BSRMatrixRead.restype = ctypes.POINTER(BSRMatrix)
    so.jxf_BSRMatrixRead.argtypes = [ctypes.c_char_p]
    so.jxf_BSRMatrixRead_Binary.restype = ctypes.POINTER(BSRMatrix)
    so.jxf_BSRMatrixRead_Binary.argtypes = [ctypes.c_char_p]
    so.jxf_BSRMatrixPrint.argtypes = [ctypes.POINTER(BSRMatrix), ctypes.c_char_p]
    so.jxf_BSRMatrixPrint_Binary.argtypes = [ctypes.POINTER(BSRMatrix), ctypes.c_char_p]
    so.jxf_BSRMatrixDestroy.argtypes = [ctypes.POINTER(BSRMatrix)]
    return so


def _arrays(p):
    A = p.contents
    bn = A.block_size * A.block_size
    ia = np.ctypeslib.as_array(A.i, (A.num_rows + 1,)).copy()
    ja = np.ctypeslib.as_array(A.j, (A.num_nonzeros,)).copy()
    a = np.ctypeslib.as_array(A.data, (A.num_nonzeros * bn,)).copy()
    return ia, ja, a, A.block_size


def test_driver_compiles_against_dropin_header(tmp_path):
    assert os.path.exists(build_driver(tmp_path))


def test_text_reader_formats(tmp_path, systems):
    so = _so()
    s = systems("tiny3")
    for one_based in (True, False):
        for cm in (False, True):
            p = tmp_path / f"A_{one_based}_{cm}.txt"
            write_bsr_text(str(p), s, one_based=one_based, column_major=cm)
            M = so.jxf_BSRMatrixRead(str(p).encode())
            ia, ja, a, bs = _arrays(M)
            assert bs == 3 and np.array_equal(ia, s.ia) and np.array_equal(ja, s.ja) and np.array_equal(a, s.a)
            so.jxf_BSRMatrixDestroy(M)


def test_binary_reader_and_writers_roundtrip(tmp_path, systems):
    so = _so()
    s = systems("small")
    for cm in (False, True):
        p = tmp_path / f"A_{cm}.bin"
        write_bsr_binary(str(p), s, column_major=cm)
        M = so.jxf_BSRMatrixRead_Binary(str(p).encode())
        ia, ja, a, _ = _arrays(M)
        assert np.array_equal(ia, s.ia) and np.array_equal(ja, s.ja) and np.array_equal(a, s.a)
        for writer, reader, ext in ((so.jxf_BSRMatrixPrint, so.jxf_BSRMatrixRead, "txt"),
                                    (so.jxf_BSRMatrixPrint_Binary, so.jxf_BSRMatrixRead_Binary, "bin")):
            q = tmp_path / f"round.{ext}"
            assert writer(M, str(q).encode()) == 0
            M2 = reader(str(q).encode())
            i2, j2, a2, _ = _arrays(M2)
            assert np.array_equal(i2, s.ia) and np.array_equal(j2, s.ja) and np.array_equal(a2, s.a)
            so.jxf_BSRMatrixDestroy(M2)
        so.jxf_BSRMatrixDestroy(M)


def test_malformed_files_return_null(tmp_path):
    so = _so()
    p = tmp_path / "bad.txt"
    p.write_text("3 3 2\n2\n0\n4\n1 2 3\n")  # truncated
    assert not so.jxf_BSRMatrixRead(str(p).encode())
    assert b"malformed" in so.jxcpr_last_error()
    assert not so.jxf_BSRMatrixRead(str(tmp_path / "missing.txt").encode())
    q = tmp_path / "badcols.txt"
    q.write_text("1 3 1\n1\n0\n2\n1 2\n1\n1\n1\n5.0\n")  # max column 0 but 3 columns declared
    assert not so.jxf_BSRMatrixRead(str(q).encode())
