"""Writes pow5_table.inc: 128-bit normalised approximations of 5^q, q = -342..308, for the decimal
to binary64 conversion of the device BSR reader (the Eisel-Lemire method, D. Lemire, "Number parsing
at a gigabyte per second", Software: Practice and Experience 51(8), 2021).  Entry q is a 128-bit
integer with its top bit set: 5^q truncated to its leading 128 bits for q >= 0; for q < 0, 2^b / 5^-q
rounded up and truncated to 128 bits.  Exact integer arithmetic; run it to regenerate the table.

    python jxpamg_all_b200/csrc/make_pow5_table.py > jxpamg_all_b200/csrc/pow5_table.inc
"""

Q_MIN, Q_MAX = -342, 308


def entry(q):
    if q >= 0:
        v = 5 ** q
        while v < (1 << 127):
            v <<= 1
        while v >= (1 << 128):
            v >>= 1
        return v
    p5 = 5 ** (-q)
    z = p5.bit_length()  # smallest z with 2^z > p5 (p5 is never a power of two)
    b = z + 127 if q >= -27 else 2 * z + 2 * 64
    c = (1 << b) // p5 + 1
    while c >= (1 << 128):
        c >>= 1
    return c


def main():
    print("// Generated by make_pow5_table.py: 128-bit normalised 5^q, q = %d..%d (high, low)." % (Q_MIN, Q_MAX))
    print("static const unsigned long long kPow5Table[%d] = {" % (2 * (Q_MAX - Q_MIN + 1)))
    for q in range(Q_MIN, Q_MAX + 1):
        v = entry(q)
        assert (1 << 127) <= v < (1 << 128)
        print("    0x%016xULL, 0x%016xULL,  // q = %d" % (v >> 64, v & ((1 << 64) - 1), q))
    print("};")


if __name__ == "__main__":
    main()
