import glob
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_golden(path):
    z = np.load(path)
    meta = json.loads(bytes(z["meta"]).decode())
    return meta, z["points"], z["offsets"], z["ids"]


def golden_cases():
    """Fixtures with float32 points (the reference-run fixtures ref_*.npz hold
    no points: their streams are regenerated, see test_reference_pin.py)."""
    return sorted(p for p in glob.glob(os.path.join(GOLDEN_DIR, "*.npz"))
                  if not os.path.basename(p).startswith(("dbl_", "ref_")))


def golden_cases_f64():
    """Fixtures with double points (double storage, RTOD's double predicate)."""
    return sorted(glob.glob(os.path.join(GOLDEN_DIR, "dbl_*.npz")))


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.build()
    return oracle
