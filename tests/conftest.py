import os
import sys

# The reference library's results depend on its OpenMP thread count; pin it to 1
# before any library is loaded.
os.environ.setdefault("OMP_NUM_THREADS", "1")

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the product library's kernels")
    config.addinivalue_line("markers", "ref: needs the reference library compiled into oracle/_ref")


def pytest_collection_modifyitems(config, items):
    import oracle

    if not oracle.ref_available():
        skip = pytest.mark.skip(reason="reference library not built in oracle/_ref")
        for it in items:
            if "ref" in it.keywords:
                it.add_marker(skip)


@pytest.fixture(scope="session")
def systems():
    """Seeded synthetic systems shared by the tests (built once per session)."""
    from jxpamg_all_b200 import synth

    cache = {}

    def get(name):
        if name not in cache:
            cache[name] = synth.config_system(name)
        return cache[name]

    return get
