import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
ORACLE_DIR = os.path.join(ROOT, "oracle")
if ORACLE_DIR not in sys.path:
    sys.path.insert(0, ORACLE_DIR)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def wct():
    return importlib.import_module("wire-cell-toolkit_b200")


@pytest.fixture(scope="session")
def synth():
    return importlib.import_module("wire-cell-toolkit_b200.synth")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.lib()
    return O


def rel_l2(a, b):
    import numpy as np
    dt = np.complex128 if np.iscomplexobj(a) or np.iscomplexobj(b) else np.float64
    a = np.asarray(a, dtype=dt)
    b = np.asarray(b, dtype=dt)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def parity_log(entry):
    """Append one measured parity figure (a dict) as a JSON line to the file
    named by WCT_PARITY_LOG, when that variable is set."""
    import json
    path = os.environ.get("WCT_PARITY_LOG")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(entry) + "\n")
