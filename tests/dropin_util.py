"""Helpers for the drop-in (reference-named C interface) tests."""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "jxpamg_all_b200")


class BSRMatrix(ctypes.Structure):
    """jxf_BSRMatrix as laid out in include/jxcpr_dropin.h."""
    _fields_ = [("data", ctypes.POINTER(ctypes.c_double)), ("i", ctypes.POINTER(ctypes.c_int)),
                ("j", ctypes.POINTER(ctypes.c_int)), ("big_j", ctypes.POINTER(ctypes.c_int)),
                ("block_size", ctypes.c_int), ("num_rows", ctypes.c_int), ("num_cols", ctypes.c_int),
                ("num_nonzeros", ctypes.c_int), ("owns_data", ctypes.c_int)]


def build_driver(tmpdir):
    exe = os.path.join(str(tmpdir), "dropin_driver")
    cmd = ["gcc", "-O1", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "dropin", "driver.c"), "-L", LIBDIR, "-ljxcpr_b200",
           f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


def write_bsr_text(path, s, one_based=True, column_major=False):
    bs, nb, nnz = s.block_size, s.num_block_rows, s.nnzb
    base = 1 if one_based else 0
    vals = s.a.reshape(nnz, bs, bs)
    if column_major:
        vals = vals.transpose(0, 2, 1)
    with open(path, "w") as f:
        f.write(f"{nb} {nb} {nnz}\n{bs}\n{1 if column_major else 0}\n{nb + 1}\n")
        f.write("\n".join(str(int(v) + base) for v in s.ia) + "\n")
        f.write(f"{nnz}\n" + "\n".join(str(int(v) + base) for v in s.ja) + "\n")
        f.write(f"{nnz * bs * bs}\n" + "\n".join(repr(float(v)) for v in vals.reshape(-1)) + "\n")


def write_bsr_binary(path, s, one_based=True, column_major=False):
    bs, nb, nnz = s.block_size, s.num_block_rows, s.nnzb
    base = 1 if one_based else 0
    vals = s.a.reshape(nnz, bs, bs)
    if column_major:
        vals = vals.transpose(0, 2, 1)
    with open(path, "wb") as f:
        np.array([nb, nb, nnz, bs, 1 if column_major else 0, nb + 1], np.int32).tofile(f)
        (s.ia.astype(np.int32) + base).tofile(f)
        np.array([nnz], np.int32).tofile(f)
        (s.ja.astype(np.int32) + base).tofile(f)
        np.array([nnz * bs * bs], np.int32).tofile(f)
        np.ascontiguousarray(vals, np.float64).reshape(-1).tofile(f)


def bsr_to_scalar_csr(s, one_based=True, diag_last=True):
    """Scalar CSR of the BSR system (unknowns interleaved per cell, every block entry stored);
    each row's diagonal is put LAST so the interface has to move it to the front."""
    bs = s.block_size
    rows_ia, ja, a = [0], [], []
    for I in range(s.num_block_rows):
        for q in range(bs):
            entries = []
            for k in range(s.ia[I], s.ia[I + 1]):
                J = s.ja[k]
                for m in range(bs):
                    entries.append((J * bs + m, s.a[k * bs * bs + q * bs + m]))
            r = I * bs + q
            entries.sort(key=lambda e: (e[0] == r) if diag_last else 0)
            ja += [c for c, _ in entries]
            a += [v for _, v in entries]
            rows_ia.append(len(ja))
    base = 1 if one_based else 0
    return (np.array(rows_ia, np.int32) + base, np.array(ja, np.int32) + base, np.array(a, np.float64))
