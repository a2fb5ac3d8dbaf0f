import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_golden(name):
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test collected on a machine without CUDA")
    return torch


# Achieved parity figures (differences against the oracle) recorded by the
# tests and printed in the terminal summary, so that a run's output states
# what was measured, not only that the bounds held.
_PARITY = []


def record_parity(test: str, quantity: str, value, bound=None):
    _PARITY.append((test, quantity, value, bound))


def pytest_terminal_summary(terminalreporter, exitstatus, config):
    if not _PARITY:
        return
    tr = terminalreporter
    tr.write_sep("-", "parity figures (achieved vs bound)")
    for test, q, v, b in _PARITY:
        vs = f"{v:.3e}" if isinstance(v, float) else str(v)
        bs = "" if b is None else (f" (bound {b:.1e})" if isinstance(b, float) else f" ({b})")
        tr.write_line(f"{test}: {q} = {vs}{bs}")
