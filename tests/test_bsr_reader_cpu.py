"""The number conversion of the device BSR text reader, run on the host (jxcpr_parse_double_host):
every decimal token it converts must give the nearest FP64 bit for bit, as a correctly rounding
strtod does (Python's float() is one); tokens it cannot convert exactly are handed to strtod."""
import ctypes
import struct

import numpy as np
import pytest

from jxpamg_all_b200 import lib


def conv(tok):
    so = lib.load()
    so.jxcpr_parse_double_host.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    out = ctypes.c_double()
    b = tok.encode()
    st = so.jxcpr_parse_double_host(b, len(b), ctypes.byref(out))
    return st, out.value


def bits(x):
    return struct.unpack("<Q", struct.pack("<d", x))[0]


@pytest.mark.parametrize("fmt", ["%.17e", "%.16e", "%.15e", "%.17g", "%g", "%.3e", "repr"])
def test_formatted_doubles_round_trip(fmt):
    rng = np.random.default_rng(7)
    raw = rng.integers(0, 2 ** 63, 4000, dtype=np.int64).view(np.float64)
    scaled = rng.standard_normal(4000) * 10.0 ** rng.integers(-300, 300, 4000)
    subn = rng.integers(1, 2 ** 52, 500, dtype=np.int64).view(np.float64)
    for x in np.concatenate([raw, scaled, subn, -raw[:500]]):
        if not np.isfinite(x):
            continue
        tok = repr(float(x)) if fmt == "repr" else fmt % x
        st, v = conv(tok)
        assert st == 0, tok
        assert bits(v) == bits(float(tok)), tok


def test_random_decimal_strings():
    rng = np.random.default_rng(11)
    for _ in range(20000):
        nd = int(rng.integers(1, 20))
        digits = "".join(str(d) for d in rng.integers(0, 10, nd))
        cut = int(rng.integers(0, nd + 1))
        tok = ("-" if rng.random() < 0.5 else "") + digits[:cut] + "." + digits[cut:] + f"e{int(rng.integers(-360, 330))}"
        if tok.lstrip("-").startswith(".e") or tok.lstrip("-") == ".":
            continue
        st, v = conv(tok)
        assert st == 0, tok
        assert bits(v) == bits(float(tok)), tok


@pytest.mark.parametrize("tok", ["9007199254740993", "9007199254740992.5", "1.7976931348623157e308",
                                 "1.7976931348623159e308", "2.2250738585072011e-308", "4.9406564584124654e-324",
                                 "2.4703282292062327e-324", "2.4703282292062328e-324", "1e23", "0.1", "-0.0",
                                 "0e0", "1e-400", "1e400", "+5", "123456789012345678", "7.0E+2"])
def test_edge_cases(tok):
    st, v = conv(tok)
    assert st == 0
    assert bits(v) == bits(float(tok))


def test_forms_left_to_strtod_and_malformed_tokens():
    assert conv("1.23456789012345678901e5")[0] == 1  # more than 19 significant digits
    assert conv("inf")[0] == 1 and conv("nan")[0] == 1
    for bad in ("", "-", ".", "e5", "1e", "1.2.3", "0x10", "1e+", "abc", "1,5"):
        assert conv(bad)[0] in (1, 2), bad
        assert conv(bad)[0] == 2 or bad == "0x10", bad
