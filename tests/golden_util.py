"""Loading of the golden fixtures produced by tests/golden/make_golden.py."""
import hashlib
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = [("small", 1), ("c0", 1), ("c0", 5), ("tiny3", 1)]


def load(name, decouple):
    return dict(np.load(os.path.join(GOLDEN, f"{name}_dec{decouple}.npz")))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
