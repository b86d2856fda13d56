"""Shared fixtures.

CPU tests (default) check the seeded model generator, pin the oracle
restatement against the reference's own C code (oracle/_ref, when it was
built) and against committed golden vectors, and check that the C-ABI
library loads and exports every declared symbol.  Tests marked `gpu` run the
CUDA library through its C ABI and compare it with the oracle.
"""
import os
import subprocess
import sys

# The reference's OpenMP Gauss-Seidel and marker reduction depend on the
# thread count; parity is defined for one thread.  Must be set before the
# reference library is loaded.
os.environ.setdefault("OMP_NUM_THREADS", "1")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import pytest  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libp2cuda.so")


def _ensure_oracle():
    from oracle import oracle as O
    if not O.available():
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "all"], check=True,
                       stdout=subprocess.DEVNULL)
    return O


@pytest.fixture(scope="session")
def oracle_mod():
    return _ensure_oracle()


@pytest.fixture(scope="session")
def gpu_available():
    try:
        import torch  # noqa: F401
        return torch.cuda.is_available()
    except Exception:
        return False
