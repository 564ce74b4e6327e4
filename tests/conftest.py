import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a); calls the C ABI")
    config.addinivalue_line("markers", "slow: full-size parity case (minutes of CPU oracle time)")


def rel_l2(a, b):
    """Relative L2 error |a - b| / |b| in float64 (elsa's isApprox criterion,
    test_routines/testHelpers.h:190-206)."""
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def cuda():
    """torch with a CUDA device; GPU tests fail loudly when there is none."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    from elsa_b200 import build
    build.build()
    return torch


def record_parity(case, **fields):
    """Append one parity result (relative L2 distances, bounds) as a JSON line to the file named
    by ELSA_PARITY_RECORD; a no-op when it is unset. The committed parity record is made from
    these lines."""
    import json
    path = os.environ.get("ELSA_PARITY_RECORD")
    if not path:
        return
    entry = {"case": case}
    for k, v in fields.items():
        entry[k] = float(v) if isinstance(v, (np.floating, np.integer)) else v
    with open(path, "a") as f:
        f.write(json.dumps(entry, sort_keys=True) + "\n")
